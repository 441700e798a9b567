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

import torch


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
