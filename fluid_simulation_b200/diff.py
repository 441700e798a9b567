"""Differentiable WCSPH rollouts: hand-written adjoint of the WCSPH substep
behind ``torch.autograd.Function``.

``DiffWCSPH(model, config, dt).rollout(x0, v0, stiffness, viscosity,
rest_density, steps)`` advances ``steps`` substeps of the drop-in WCSPH step
(fs_wcsph_substep, the reference's SolverWCSPH.step) and returns the final
positions and velocities as tensors that autograd can differentiate with
respect to the initial positions and velocities and the per-particle (or
scalar) stiffness, viscosity and rest density.

Memory: the forward keeps a checkpoint (positions, velocities) every
``checkpoint_every`` substeps and the full record of the last segment
(inputs, rho, pressure, acceleration of each substep).  The backward walks
the segments from last to first; each earlier segment is first replayed from
its checkpoint (the grid is rebuilt by every replayed substep), then its
substeps are differentiated in reverse with fs_wcsph_substep_adjoint, which
holds each substep's neighbour set fixed.  Replays are bit-identical to the
forward (deterministic grid build and reductions), so the gradient does not
depend on ``checkpoint_every``.
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

    def __init__(self, model, config: SolverWCSPH.SphConfig, dt: float, checkpoint_every: int = 10):
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        cm.require_cuda(model, "DiffWCSPH")
        cm.attach_grid(model, "DiffWCSPH")
        self.model = model
        self.config = config
        self.dt = float(dt)
        self.k = int(checkpoint_every)
        self._solver = SolverWCSPH(model, config)  # parameters only
        self.params = self._solver.params(self.dt)
        n = model.particle_count
        self.n = n
        self.seg = _Segment(n, self.k, model.device)
        f = dict(dtype=torch.float32, device=model.device)
        self._xb = [torch.zeros(n, 3, **f), torch.zeros(n, 3, **f)]
        self._vb = [torch.zeros(n, 3, **f), torch.zeros(n, 3, **f)]
        self.launches = 0

    # ------------------------------------------------------------- pieces --
    def _model_struct(self):
        return cm.model_struct(self.model, wcsph=True)

    def _forward_segment(self, ms, steps):
        """seg.x[0], seg.v[0] -> seg.x[steps], recording every substep."""
        lib = _lib.load()
        ctx = cm.grid_ctx(self.model, "DiffWCSPH")
        st = cm.stream_of(self.model.device)
        s = self.seg
        for t in range(steps):
            _lib.check(lib.fs_wcsph_substep(ctx, C.byref(ms), C.byref(s.si[t]), C.byref(s.so[t]), C.byref(self.params),
                                            s.a[t].data_ptr(), st), "DiffWCSPH forward")

    def _backward_segment(self, ms, steps, xb, vb, gB, gnu, grho0):
        """Adjoint of seg substeps steps-1..0; xb/vb hold dL/d(state after
        the segment) on entry and dL/d(state before it) on exit."""
        lib = _lib.load()
        ctx = cm.grid_ctx(self.model, "DiffWCSPH")
        st = cm.stream_of(self.model.device)
        s = self.seg
        cur = 0
        self._xb[0].copy_(xb)
        self._vb[0].copy_(vb)
        for t in reversed(range(steps)):
            nxt = 1 - cur
            _lib.check(lib.fs_wcsph_substep_adjoint(
                ctx, C.byref(ms), C.byref(s.si[t]), s.rho[t].data_ptr(), s.p[t].data_ptr(), s.a[t].data_ptr(),
                self._xb[cur].data_ptr(), self._vb[cur].data_ptr(), self._xb[nxt].data_ptr(),
                self._vb[nxt].data_ptr(), gB.data_ptr(), gnu.data_ptr(), grho0.data_ptr(), C.byref(self.params), st),
                "DiffWCSPH backward")
            cur = nxt
        xb.copy_(self._xb[cur])
        vb.copy_(self._vb[cur])

    # ------------------------------------------------------------ rollout --
    def rollout(self, x0, v0, stiffness, viscosity, rest_density, steps: int):
        """(x_T, v_T) after ``steps`` substeps; differentiable in every input.
        stiffness / viscosity / rest_density: scalars or per-particle [n]."""
        return _Rollout.apply(x0, v0, stiffness, viscosity, rest_density, self, int(steps))


def _per_particle(t, n, device):
    t = torch.as_tensor(t, dtype=torch.float32, device=device)
    return t.detach().expand(n).contiguous() if t.dim() == 0 else t.detach().contiguous()


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, stiffness, viscosity, rest_density, sim: DiffWCSPH, steps: int):
        n, dev = sim.n, sim.model.device
        sph = sim.model.sph
        sph.stiffness = _per_particle(stiffness, n, dev)
        sph.viscosity = _per_particle(viscosity, n, dev)
        sph.rest_density = _per_particle(rest_density, n, dev)
        ms = sim._model_struct()
        k = sim.k
        s = sim.seg
        checkpoints = []
        x = x0.detach().to(torch.float32).contiguous()
        v = v0.detach().to(torch.float32).contiguous()
        done = 0
        while done < steps:
            m = min(k, steps - done)
            s.x[0].copy_(x)
            s.v[0].copy_(v)
            checkpoints.append((s.x[0].clone(), s.v[0].clone()) if done + m < steps else None)
            sim._forward_segment(ms, m)
            x, v = s.x[m], s.v[m]
            done += m
        ctx.sim, ctx.steps, ctx.checkpoints = sim, steps, checkpoints
        ctx.shapes = tuple(torch.as_tensor(t).dim() for t in (stiffness, viscosity, rest_density))
        ctx.last = steps - (len(checkpoints) - 1) * k if steps else 0
        return x.clone(), v.clone()

    @staticmethod
    def backward(ctx, gx, gv):
        sim, steps, k = ctx.sim, ctx.steps, ctx.sim.k
        n, dev = sim.n, sim.model.device
        f = dict(dtype=torch.float32, device=dev)
        xb = (gx if gx is not None else torch.zeros(n, 3, **f)).to(torch.float32).contiguous().clone()
        vb = (gv if gv is not None else torch.zeros(n, 3, **f)).to(torch.float32).contiguous().clone()
        gB, gnu, grho0 = (torch.zeros(n, **f) for _ in range(3))
        ms = sim._model_struct()
        s = sim.seg
        nseg = len(ctx.checkpoints)
        for si in reversed(range(nseg)):
            m = ctx.last if si == nseg - 1 else k
            if si != nseg - 1:  # replay this segment from its checkpoint
                cx, cv = ctx.checkpoints[si]
                s.x[0].copy_(cx)
                s.v[0].copy_(cv)
                sim._forward_segment(ms, m)
            sim._backward_segment(ms, m, xb, vb, gB, gnu, grho0)
        red = [g.sum() if d == 0 else g for g, d in zip((gB, gnu, grho0), ctx.shapes)]
        return xb, vb, red[0], red[1], red[2], None, None
