"""Shared host plumbing of the drop-in solvers: argument checks and the
conversion of Model/State tensors to the C-ABI structs."""

from __future__ import annotations

import ctypes as C

import torch

from .. import _lib
from ..newton_shim import HashGrid, ModelBuilder, Model, vec3


def ptr(t, name, dtype=torch.float32, cols=None, n=None, device=None, optional=False):
    """Device pointer of a contiguous tensor after checking dtype/shape/device."""
    if t is None:
        if optional:
            return None
        raise ValueError(f"{name} is required")
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch tensor (got {type(t).__name__})")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype} (got {t.dtype})")
    if device is not None and t.device != device:
        raise ValueError(f"{name} is on {t.device}, the model is on {device}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if n is not None:
        want = (n, cols) if cols else (n,)
        if tuple(t.shape) != want:
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {want}")
    return t.data_ptr()


def require_cuda(model: Model, solver: str):
    if model.device.type != "cuda":
        raise RuntimeError(f"{solver} runs on CUDA devices only (B200 kernels; there is no CPU path): "
                           f"model.device = {model.device}")


def attach_grid(model: Model, solver: str):
    """Reference behaviour (solver_wcsph.py:398-402): a model with more than one
    particle gets HashGrid(128,128,128) unless it has a grid, then reserve(N)."""
    if model.particle_count > 1:
        if model.particle_grid is None:
            model.particle_grid = HashGrid(128, 128, 128, device=model.device)
        model.particle_grid.reserve(model.particle_count)


def copy_passthrough_state(state_in, state_out):
    """_copy_passthrough_state, solver_wcsph.py:412-420."""
    if getattr(state_in, "body_count", 0):
        state_out.body_q.copy_(state_in.body_q)
        state_out.body_qd.copy_(state_in.body_qd)
        state_out.body_f.copy_(state_in.body_f)
    if getattr(state_in, "joint_q", None) is not None and getattr(state_out, "joint_q", None) is not None:
        state_out.joint_q.copy_(state_in.joint_q)
    if getattr(state_in, "joint_qd", None) is not None and getattr(state_out, "joint_qd", None) is not None:
        state_out.joint_qd.copy_(state_in.joint_qd)


def model_struct(model: Model, wcsph: bool = False) -> _lib.Model:
    n = model.particle_count
    d = model.device
    sph = model.sph
    g = model.gravity
    return _lib.Model(
        n, int(g.shape[0]),
        ptr(model.particle_flags, "model.particle_flags", torch.int32, n=n, device=d),
        ptr(sph.particle_mask, "model.sph.particle_mask", torch.int32, n=n, device=d),
        ptr(model.particle_world, "model.particle_world", torch.int32, n=n, device=d, optional=True),
        ptr(model.particle_mass, "model.particle_mass", n=n, device=d),
        ptr(g, "model.gravity", cols=3, n=int(g.shape[0]), device=d),
        ptr(sph.rest_density, "model.sph.rest_density", n=n, device=d),
        ptr(sph.surface_tension, "model.sph.surface_tension", n=n, device=d),
        ptr(sph.viscosity, "model.sph.viscosity", n=n, device=d),
        ptr(getattr(sph, "stiffness", None), "model.sph.stiffness", n=n, device=d, optional=not wcsph),
        ptr(getattr(sph, "exponent", None), "model.sph.exponent", n=n, device=d, optional=not wcsph),
    )


_VEC = {"v_star", "delta_p"}


def state_struct(state, n: int, device, need=(), optional=()) -> _lib.State:
    s = _lib.State()
    s.particle_q = ptr(state.particle_q, "state.particle_q", cols=3, n=n, device=device)
    s.particle_qd = ptr(state.particle_qd, "state.particle_qd", cols=3, n=n, device=device)
    for name in tuple(need) + tuple(optional):
        t = getattr(state.sph, name, None)
        dt = torch.int32 if name == "neighbor_count" else torch.float32
        setattr(s, name, ptr(t, f"state.sph.{name}", dt, cols=3 if name in _VEC else None, n=n, device=device,
                             optional=name in optional))
    return s


def stream_of(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def register(builder: ModelBuilder, model_attrs, state_attrs):
    """Add (name, dtype, default) custom attributes in the `sph` namespace."""
    for assignment, attrs in ((Model.AttributeAssignment.MODEL, model_attrs),
                              (Model.AttributeAssignment.STATE, state_attrs)):
        for name, dtype, default in attrs:
            builder.add_custom_attribute(ModelBuilder.CustomAttribute(
                name=name, frequency=Model.AttributeFrequency.PARTICLE, assignment=assignment, dtype=dtype,
                default=default, namespace="sph"))


def particle_radius(config, model) -> float:
    return float(config.particle_radius if config.particle_radius > 0.0 else model.particle_max_radius)


def grid_ctx(model: Model, solver: str):
    grid = model.particle_grid
    if grid is None:
        raise RuntimeError(f"{solver} requires model.particle_grid to be available for particle neighborhoods.")
    if not isinstance(grid, HashGrid):
        raise TypeError(f"{solver}: model.particle_grid must be a fluid_simulation_b200 HashGrid")
    if grid.capacity < model.particle_count:
        grid.reserve(model.particle_count)
    return grid._ctx


__all__ = ["ptr", "require_cuda", "attach_grid", "copy_passthrough_state", "model_struct", "state_struct",
           "stream_of", "register", "particle_radius", "grid_ctx", "vec3", "C"]
