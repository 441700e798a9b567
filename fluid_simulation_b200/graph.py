"""Whole-frame CUDA graphs of the drop-in solvers.

A PBF or DFSPH substep launches only kernels and device-side memsets/copies
(DFSPH takes its iteration decisions on the device), and a WCSPH substep at a
given dt does too, so a display frame of substeps can be recorded once and
replayed as a single graph launch.  States ping-pong as in the reference
harness (simulation.py:192-196); with an even number of substeps the frame's
result is back in ``state_a``.  The reference archive captures PBF the same
way with two graphs for the two ping-pong orders
(backup/examples/newton_pbf_test.py:224-250).
"""

from __future__ import annotations

import ctypes as C
import math

import torch

from . import _lib


class FrameGraph:
    def __init__(self, solver, state_a, state_b, dt: float, substeps: int = 4, warmup: bool = True):
        if substeps < 1:
            raise ValueError("substeps must be >= 1")
        self.solver = solver
        self.state_a, self.state_b = state_a, state_b
        self.dt = float(dt)
        self.substeps = int(substeps)
        dev = solver.model.device
        self.stream = torch.cuda.Stream(device=dev)
        if warmup:
            # one eager frame on the capture stream: compiles nothing, but runs every
            # first-call path (context sizing) outside the capture
            self.stream.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(self.stream):
                self._frame()
            torch.cuda.current_stream(dev).wait_stream(self.stream)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._frame()

    def _frame(self):
        a, b = self.state_a, self.state_b
        for _ in range(self.substeps):
            self.solver.step(a, b, None, None, self.dt)
            a, b = b, a
        self.result = a

    def replay(self):
        """One frame (``substeps`` substeps) as one graph launch on the current stream."""
        self.graph.replay()
        return self.result


class DeviceFrameLoop:
    """The WCSPH / DFSPH dam-break frame loop with its substep rule on the device.

    The reference harness (simulation.py:155-196) reads max |v| (and for
    WCSPH max |a|) back to the host before every substep to choose its dt.
    Here a frame clock in device memory carries the time left in the frame;
    one CUDA graph records ``graph_substeps`` pairs of [evaluate the rule on
    the device (fs_frame_clock_advance), clocked substep
    (fs_wcsph_substep_clocked / fs_dfsph_substep_clocked)],
    and a frame replays that graph until the clock reports the frame done:
    one read of the clock per replay instead of one per substep.  Substeps
    after the end of the frame copy their input through, so the result is
    always back in ``sim.state_0`` (``graph_substeps`` is even).  The dt
    sequence, and hence every state, is the one of ``sim.step()``.
    """

    MAX_SUBSTEPS = 4096  # the harness's own limit per frame

    def __init__(self, sim, graph_substeps: int = 64):
        if sim.method not in ("wcsph", "dfsph"):
            raise NotImplementedError("the device-side substep rule drives the CFL solvers (WCSPH, DFSPH)")
        if graph_substeps < 2 or graph_substeps % 2:
            raise ValueError("graph_substeps must be even and >= 2")
        from .solver import _common as cm

        self.sim = sim
        self.m = int(graph_substeps)
        model, solver = sim.model, sim.solver
        dev = model.device
        n = model.particle_count
        self.clock = torch.zeros(C.sizeof(_lib.FrameClock), dtype=torch.uint8, device=dev)
        start = _lib.FrameClock()
        start.run_substeps = 1 if sim.total_substeps else 0
        self.clock.copy_(torch.frombuffer(bytearray(bytes(start)), dtype=torch.uint8))
        mat = sim.material
        wcsph = sim.method == "wcsph"
        sound = math.sqrt(mat["stiffness"] * mat["exponent"] / sim.scene.spec.density) if wcsph else 0.0
        self.rule = _lib.CflRule(sim.frame_dt, sim.frame_dt / sim.substeps, 0 if wcsph else 1, 1 if wcsph else 0,
                                 float(solver.smoothing_length), sound, float(mat["viscosity"]),
                                 float(sim.scene.spacing))
        self._ms = cm.model_struct(model, wcsph=wcsph)
        a, b = sim.state_0, sim.state_1
        need = ("rho", "pressure") if wcsph else tuple(vars(a.sph))
        self._si = [cm.state_struct(s, n, dev, need=need) for s in (a, b)]
        lib_fn = "fs_wcsph_substep_clocked" if wcsph else "fs_dfsph_substep_clocked"
        self._v = [s.particle_qd for s in (a, b)]
        self._params = solver.params(0.0)
        self._acc = solver._particle_accel
        self._ctx = cm.grid_ctx(model, "DeviceFrameLoop")
        self.stream = torch.cuda.Stream(device=dev)
        self.graph = torch.cuda.CUDAGraph()
        lib = _lib.load()
        self.stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.graph(self.graph, stream=self.stream):
            st = self.stream.cuda_stream
            ck = self.clock.data_ptr()
            for k in range(self.m):
                i, o = k % 2, 1 - k % 2
                _lib.check(lib.fs_frame_clock_advance(ck, C.byref(self.rule), self._v[i].data_ptr(), n,
                                                      self._acc.data_ptr(), n, st), "clock advance")
                _lib.check(getattr(lib, lib_fn)(self._ctx, C.byref(self._ms), C.byref(self._si[i]),
                                                C.byref(self._si[o]), C.byref(self._params), self._acc.data_ptr(),
                                                ck, st), "clocked substep")
        torch.cuda.current_stream(dev).wait_stream(self.stream)
        self.replays = 0

    def read_clock(self) -> _lib.FrameClock:
        return _lib.FrameClock.from_buffer_copy(self.clock.cpu().numpy().tobytes())

    def step(self):
        """One display frame."""
        sim = self.sim
        lib = _lib.load()
        st = torch.cuda.current_stream(sim.model.device).cuda_stream
        _lib.check(lib.fs_frame_clock_start(self.clock.data_ptr(), sim.frame_dt, st), "clock start")
        while True:
            self.graph.replay()
            self.replays += 1
            c = self.read_clock()
            if c.fault & 1:
                raise RuntimeError(f"Non-finite velocity or WCSPH acceleration at frame {sim.frame}")
            if c.fault:
                raise RuntimeError("CFL step cannot safely complete this frame")
            if not c.remaining > 1.0e-12:
                break
            if c.substeps >= self.MAX_SUBSTEPS:
                raise RuntimeError("CFL step cannot safely complete this frame")
        sim.frame += 1
        sim.sim_time = sim.frame * sim.frame_dt
        sim.last_substeps = int(c.substeps)
        sim.total_substeps += int(c.substeps)
