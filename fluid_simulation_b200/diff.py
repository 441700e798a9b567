"""Differentiable WCSPH rollouts: hand-written adjoint of the WCSPH substep
behind ``torch.autograd.Function``.

``DiffWCSPH(model, config, dt).rollout(x0, v0, stiffness, viscosity,
rest_density, steps)`` advances ``steps`` substeps of the drop-in WCSPH step
(fs_wcsph_substep, the reference's SolverWCSPH.step) and returns the final
positions and velocities as tensors that autograd can differentiate with
respect to the initial positions and velocities and the per-particle (or
scalar) stiffness, viscosity and rest density.

Memory: the rollout is cut into segments of ``checkpoint_every`` substeps.
The forward keeps a checkpoint (positions, velocities) at the start of every
segment, and the full record (inputs, rho, pressure, acceleration of each
substep: 44 bytes per particle and substep) of as many trailing segments as
fit in ``record_bytes`` (default: a quarter of the free device memory when
the simulator is made; 0 keeps only the last segment's record).  The backward
walks the segments from last to first; a segment without a record is first
replayed from its checkpoint (the grid is rebuilt by every replayed
substep), then its substeps are differentiated in reverse with
fs_wcsph_substep_adjoint, which holds each substep's neighbour set fixed.
Replays are bit-identical to the forward (deterministic grid build and
reductions), so the gradient depends neither on ``checkpoint_every`` nor on
``record_bytes``.

Every full segment (k substeps forward, or k adjoint substeps) is recorded
once as a CUDA graph over the segment's fixed buffers and replayed after its
first eager run, so a rollout costs one graph launch per segment and pass.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .solver import _common as cm
from .solver.sph.solver_wcsph import SolverWCSPH


class _Segment:
    """Device record of up to k substeps: states 0..k, and rho, pressure,
    accel of substeps 0..k-1, with their C-ABI structs prebuilt."""

    def __init__(self, n, k, device):
        f = dict(dtype=torch.float32, device=device)
        self.x = [torch.empty(n, 3, **f) for _ in range(k + 1)]
        self.v = [torch.empty(n, 3, **f) for _ in range(k + 1)]
        self.rho = [torch.empty(n, **f) for _ in range(k)]
        self.p = [torch.empty(n, **f) for _ in range(k)]
        self.a = [torch.empty(n, 3, **f) for _ in range(k)]
        self.si, self.so = [], []
        for t in range(k):
            si = _lib.State()
            si.particle_q, si.particle_qd = self.x[t].data_ptr(), self.v[t].data_ptr()
            so = _lib.State()
            so.particle_q, so.particle_qd = self.x[t + 1].data_ptr(), self.v[t + 1].data_ptr()
            so.rho, so.pressure = self.rho[t].data_ptr(), self.p[t].data_ptr()
            self.si.append(si)
            self.so.append(so)


class DiffWCSPH:
    """Differentiable rollouts of the WCSPH substep on ``model`` (its
    ``particle_grid``: a HashGrid, or a WorldGrid for batched scenes)."""

    def __init__(self, model, config: SolverWCSPH.SphConfig, dt: float, checkpoint_every: int = 10,
                 use_graphs: bool = True, record_bytes: int | None = None):
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        cm.require_cuda(model, "DiffWCSPH")
        cm.attach_grid(model, "DiffWCSPH")
        self.model = model
        self.config = config
        self.dt = float(dt)
        self.k = int(checkpoint_every)
        self.use_graphs = bool(use_graphs)
        self._solver = SolverWCSPH(model, config)  # parameters only
        self.params = self._solver.params(self.dt)
        n = model.particle_count
        self.n = n
        self.seg_bytes = 44 * n * self.k + 24 * n
        if record_bytes is None:
            record_bytes = torch.cuda.mem_get_info(model.device)[0] // 4
        self.max_records = max(1, int(record_bytes) // max(1, self.seg_bytes))
        self._segs = [_Segment(n, self.k, model.device)]  # [0]: replay buffer; [1:]: kept records
        f = dict(dtype=torch.float32, device=model.device)
        self._xb = [torch.zeros(n, 3, **f), torch.zeros(n, 3, **f)]
        self._vb = [torch.zeros(n, 3, **f), torch.zeros(n, 3, **f)]
        # parameter fields and their gradient accumulators at fixed addresses
        # (recorded graphs hold the pointers)
        sph = model.sph
        for name in ("stiffness", "viscosity", "rest_density"):
            setattr(sph, name, getattr(sph, name).detach().clone().contiguous())
        self.grad = {name: torch.zeros(n, **f) for name in ("stiffness", "viscosity", "rest_density")}
        self._graphs = {}
        self._seen = set()

    # ------------------------------------------------------------- pieces --
    def _model_struct(self):
        return cm.model_struct(self.model, wcsph=True)

    def _run(self, key, fn):
        """fn() eagerly the first time, then recorded as a CUDA graph and
        replayed (all buffers fn touches are fixed)."""
        if not self.use_graphs:
            fn()
            return
        g = self._graphs.get(key)
        if g is not None:
            g.replay()
            return
        fn()
        if key in self._seen:
            return
        self._seen.add(key)
        dev = self.model.device
        stream = torch.cuda.Stream(device=dev)
        stream.wait_stream(torch.cuda.current_stream(dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            fn()
        torch.cuda.current_stream(dev).wait_stream(stream)
        self._graphs[key] = g

    def _buffer(self, b):
        while len(self._segs) <= b:
            self._segs.append(_Segment(self.n, self.k, self.model.device))
        return self._segs[b]

    def _forward_segment(self, ms, steps, b):
        """buffer b: x[0], v[0] -> x[steps], recording every substep."""
        lib = _lib.load()
        ctx = cm.grid_ctx(self.model, "DiffWCSPH")
        s = self._buffer(b)

        def fn():
            st = cm.stream_of(self.model.device)
            for t in range(steps):
                _lib.check(lib.fs_wcsph_substep(ctx, C.byref(ms), C.byref(s.si[t]), C.byref(s.so[t]),
                                                C.byref(self.params), s.a[t].data_ptr(), st), "DiffWCSPH forward")
        self._run(("f", b, steps), fn)

    def _backward_segment(self, ms, steps, b, xb, vb):
        """Adjoint of buffer b's substeps steps-1..0; xb/vb hold dL/d(state
        after the segment) on entry and dL/d(state before it) on exit;
        parameter gradients accumulate into self.grad."""
        lib = _lib.load()
        ctx = cm.grid_ctx(self.model, "DiffWCSPH")
        s = self._buffer(b)
        gB, gnu, grho0 = (self.grad[k].data_ptr() for k in ("stiffness", "viscosity", "rest_density"))
        cur_final = steps % 2

        def fn():
            st = cm.stream_of(self.model.device)
            cur = 0
            for t in reversed(range(steps)):
                nxt = 1 - cur
                _lib.check(lib.fs_wcsph_substep_adjoint(
                    ctx, C.byref(ms), C.byref(s.si[t]), s.rho[t].data_ptr(), s.p[t].data_ptr(), s.a[t].data_ptr(),
                    self._xb[cur].data_ptr(), self._vb[cur].data_ptr(), self._xb[nxt].data_ptr(),
                    self._vb[nxt].data_ptr(), gB, gnu, grho0, C.byref(self.params), st), "DiffWCSPH backward")
                cur = nxt
        self._xb[0].copy_(xb)
        self._vb[0].copy_(vb)
        self._run(("b", b, steps), fn)
        xb.copy_(self._xb[cur_final])
        vb.copy_(self._vb[cur_final])

    # ------------------------------------------------------------ rollout --
    def rollout(self, x0, v0, stiffness, viscosity, rest_density, steps: int):
        """(x_T, v_T) after ``steps`` substeps; differentiable in every input.
        stiffness / viscosity / rest_density: scalars or per-particle [n]."""
        return _Rollout.apply(x0, v0, stiffness, viscosity, rest_density, self, int(steps))


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, stiffness, viscosity, rest_density, sim: DiffWCSPH, steps: int):
        sph = sim.model.sph
        for name, val in (("stiffness", stiffness), ("viscosity", viscosity), ("rest_density", rest_density)):
            getattr(sph, name).copy_(torch.as_tensor(val, dtype=torch.float32).detach())  # scalars broadcast
        ms = sim._model_struct()
        k = sim.k
        nseg = (steps + k - 1) // k
        first_kept = nseg - min(nseg, sim.max_records)  # segments >= first_kept keep their record
        checkpoints, lengths, buffers = [], [], []
        x = x0.detach().to(torch.float32).contiguous()
        v = v0.detach().to(torch.float32).contiguous()
        for si in range(nseg):
            m = min(k, steps - si * k)
            b = si - first_kept + 1 if si >= first_kept else 0
            s = sim._buffer(b)
            s.x[0].copy_(x)
            s.v[0].copy_(v)
            checkpoints.append(None if b else (x.clone(), v.clone()))
            sim._forward_segment(ms, m, b)
            x, v = s.x[m], s.v[m]
            lengths.append(m)
            buffers.append(b)
        ctx.sim, ctx.checkpoints, ctx.lengths, ctx.buffers = sim, checkpoints, lengths, buffers
        ctx.shapes = tuple(torch.as_tensor(t).dim() for t in (stiffness, viscosity, rest_density))
        return x.clone(), v.clone()

    @staticmethod
    def backward(ctx, gx, gv):
        sim = ctx.sim
        n, dev = sim.n, sim.model.device
        f = dict(dtype=torch.float32, device=dev)
        xb = (gx if gx is not None else torch.zeros(n, 3, **f)).to(torch.float32).contiguous().clone()
        vb = (gv if gv is not None else torch.zeros(n, 3, **f)).to(torch.float32).contiguous().clone()
        for g in sim.grad.values():
            g.zero_()
        ms = sim._model_struct()
        for si in reversed(range(len(ctx.lengths))):
            m, b = ctx.lengths[si], ctx.buffers[si]
            if b == 0:  # no record kept: replay the segment from its checkpoint
                s = sim._buffer(0)
                cx, cv = ctx.checkpoints[si]
                s.x[0].copy_(cx)
                s.v[0].copy_(cv)
                sim._forward_segment(ms, m, 0)
            sim._backward_segment(ms, m, b, xb, vb)
        grads = [sim.grad[k].clone() for k in ("stiffness", "viscosity", "rest_density")]
        red = [g.sum() if d == 0 else g for g, d in zip(grads, ctx.shapes)]
        return xb, vb, red[0], red[1], red[2], None, None
