"""Minimal stand-in for the parts of newton 1.6.0 the reference solvers use.

newton (and warp) are not available, so the drop-in solvers work on these
objects, whose attribute names match the Newton ones the reference reads:

* ``Model``: ``particle_count``, ``particle_q``, ``particle_qd``,
  ``particle_mass``, ``particle_radius``, ``particle_flags``,
  ``particle_world``, ``particle_max_radius``, ``gravity`` ([W,3]),
  ``particle_grid``, ``device``, ``sph`` (MODEL custom attributes),
  ``state()``, ``set_gravity()``.
* ``State``: ``particle_q``, ``particle_qd``, ``body_count``, ``joint_q``,
  ``joint_qd``, ``sph`` (STATE custom attributes).
* ``ModelBuilder``: ``add_custom_attribute(ModelBuilder.CustomAttribute(...))``,
  ``add_particles(pos, vel, mass, radius, flags, custom_attributes)``,
  ``add_ground_plane`` (no-op for the particle path), ``finalize(device)``.
* ``HashGrid(dim_x, dim_y, dim_z)``: the ``wp.HashGrid`` object the solvers
  keep in ``model.particle_grid``; ``reserve(n)`` / ``build(points, radius)``
  run on the GPU through ``libfluid_b200.so``.

Arrays are torch tensors in original particle order: vec3 -> float32 [N,3],
float -> float32 [N], int -> int32 [N].  A Newton/Warp user hands the same
memory over with ``wp.to_torch`` (zero copy).
"""

from __future__ import annotations

import ctypes as C
import enum
import types
from dataclasses import dataclass
from typing import Any

import torch

from . import _lib


class vec3:  # noqa: N801 - Newton/Warp type name
    """dtype marker for [N,3] float32 attributes (warp ``wp.vec3``)."""


float32 = torch.float32
int32 = torch.int32


class ParticleFlags(enum.IntFlag):
    ACTIVE = 1


class Axis(enum.IntEnum):
    X = 0
    Y = 1
    Z = 2


def torch_dtype(dtype):
    if dtype is vec3:
        return torch.float32
    if dtype in (float, torch.float32):
        return torch.float32
    if dtype in (int, torch.int32):
        return torch.int32
    raise TypeError(f"unsupported attribute dtype {dtype!r}")


class Control:
    pass


class Contacts:
    pass


class State:
    def __init__(self):
        self.particle_q: torch.Tensor | None = None
        self.particle_qd: torch.Tensor | None = None
        self.body_count = 0
        self.body_q = self.body_qd = self.body_f = None
        self.joint_q = None
        self.joint_qd = None
        self.sph = types.SimpleNamespace()

    @property
    def particle_count(self) -> int:
        return 0 if self.particle_q is None else int(self.particle_q.shape[0])


class Model:
    class AttributeFrequency(enum.Enum):
        PARTICLE = "particle"

    class AttributeAssignment(enum.Enum):
        MODEL = "model"
        STATE = "state"

    def __init__(self, device="cuda:0"):
        self.device = torch.device(device)
        self.particle_count = 0
        self.particle_q = self.particle_qd = None
        self.particle_mass = self.particle_radius = None
        self.particle_flags = self.particle_world = None
        self.particle_max_radius = 0.0
        self.gravity = torch.zeros(1, 3, dtype=torch.float32, device=self.device)
        self.particle_grid = None
        self.sph = types.SimpleNamespace()
        self._state_attrs: list[ModelBuilder.CustomAttribute] = []
        self._state_values: dict[str, Any] = {}

    def set_gravity(self, g, world: int | None = None):
        g = torch.as_tensor(g, dtype=torch.float32, device=self.device).reshape(-1, 3)
        if world is None:
            self.gravity[:] = g[0] if g.shape[0] == 1 else g
        else:
            self.gravity[world] = g[0]

    def state(self) -> State:
        s = State()
        if self.particle_q is not None:
            s.particle_q = self.particle_q.clone()
            s.particle_qd = self.particle_qd.clone()
        for a in self._state_attrs:
            val = self._state_values.get(a.key)
            if val is None:
                val = _filled(a, self.particle_count, self.device)
            else:
                val = val.clone()
            setattr(s.sph, a.name, val)
        return s


def _filled(attr, n, device):
    dt = torch_dtype(attr.dtype)
    shape = (n, 3) if attr.dtype is vec3 else (n,)
    t = torch.empty(shape, dtype=dt, device=device)
    d = attr.default
    if attr.dtype is vec3:
        t[:] = torch.as_tensor(d if d is not None else (0.0, 0.0, 0.0), dtype=dt)
    else:
        t.fill_(0 if d is None else d)
    return t


class ModelBuilder:
    @dataclass
    class CustomAttribute:
        name: str
        frequency: Any = None
        assignment: Any = None
        dtype: Any = float
        default: Any = None
        namespace: str | None = None

        @property
        def key(self) -> str:
            return f"{self.namespace}:{self.name}" if self.namespace else self.name

    @dataclass
    class ShapeConfig:
        density: float = 0.0
        mu: float = 0.0

    def __init__(self, up_axis=Axis.Z, gravity: float = -9.81):
        self.up_axis = up_axis
        self.default_particle_radius = 0.1
        self.custom_attributes: dict[str, ModelBuilder.CustomAttribute] = {}
        self._pos, self._vel, self._mass, self._radius, self._flags, self._world = [], [], [], [], [], []
        self._attr_values: dict[str, list] = {}
        self.gravity = gravity

    def add_custom_attribute(self, attr: "ModelBuilder.CustomAttribute") -> None:
        if attr.namespace not in (None, "sph"):
            raise ValueError(f"namespace {attr.namespace!r} is not supported by the particle shim")
        self.custom_attributes[attr.key] = attr

    def add_particles(self, pos, vel, mass, radius=None, flags=None, custom_attributes=None, world=0):
        n = len(pos)
        self._pos.extend([tuple(map(float, p)) for p in pos])
        self._vel.extend([tuple(map(float, v)) for v in vel])
        self._mass.extend([float(m) for m in mass])
        r = radius if radius is not None else [self.default_particle_radius] * n
        self._radius.extend([float(x) for x in r])
        self._flags.extend([int(f) for f in (flags if flags is not None else [int(ParticleFlags.ACTIVE)] * n)])
        self._world.extend([int(world)] * n)
        start = len(self._pos) - n
        for key, values in (custom_attributes or {}).items():
            if key not in self.custom_attributes:
                raise KeyError(f"custom attribute {key!r} was not registered")
            col = self._attr_values.setdefault(key, [None] * start)
            col.extend(values)
        for col in self._attr_values.values():
            col.extend([None] * (len(self._pos) - len(col)))

    def add_ground_plane(self, cfg=None):
        return -1  # shapes are not part of the particle path

    def finalize(self, device="cuda:0") -> Model:
        m = Model(device)
        dev = m.device
        n = len(self._pos)
        m.particle_count = n
        m.particle_q = torch.tensor(self._pos, dtype=torch.float32, device=dev).reshape(n, 3)
        m.particle_qd = torch.tensor(self._vel, dtype=torch.float32, device=dev).reshape(n, 3)
        m.particle_mass = torch.tensor(self._mass, dtype=torch.float32, device=dev)
        m.particle_radius = torch.tensor(self._radius, dtype=torch.float32, device=dev)
        m.particle_flags = torch.tensor(self._flags, dtype=torch.int32, device=dev)
        m.particle_world = torch.tensor(self._world, dtype=torch.int32, device=dev)
        m.particle_max_radius = max(self._radius) if self._radius else 0.0
        m.gravity = torch.tensor([[0.0, 0.0, self.gravity]], dtype=torch.float32, device=dev)
        for key, a in self.custom_attributes.items():
            vals = self._attr_values.get(key)
            t = _filled(a, n, dev)
            if vals is not None:
                idx = [k for k, v in enumerate(vals) if v is not None]
                if idx:
                    src = torch.tensor([vals[k] for k in idx], dtype=t.dtype, device=dev)
                    t[torch.tensor(idx, device=dev)] = src.reshape(t[idx].shape)
            if a.assignment == Model.AttributeAssignment.STATE:
                m._state_attrs.append(a)
                m._state_values[a.key] = t
            else:
                setattr(m.sph, a.name, t)
        return m


def model_from_arrays(x, v, mass, *, device="cuda:0", flags=None, world=None, gravity=((0.0, 0.0, -10.0),),
                      radius=None, attributes: dict | None = None, state_attributes=(), solver_cls=None) -> Model:
    """Build a Model directly from arrays (no per-particle Python lists).

    With ``solver_cls`` the solver's custom attributes are registered: MODEL
    attributes take the value in ``attributes`` or their default, STATE
    attributes are created by ``model.state()``."""
    if solver_cls is not None:
        b = ModelBuilder()
        solver_cls.register_custom_attributes(b)
        attributes = dict(attributes or {})
        extra = []
        for a in b.custom_attributes.values():
            if a.assignment == Model.AttributeAssignment.STATE:
                extra.append(a)
            elif a.name not in attributes:
                attributes[a.name] = a.default
        state_attributes = tuple(state_attributes) + tuple(extra)
    dev = torch.device(device)
    x = torch.as_tensor(x, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
    n = x.shape[0]
    m = Model(dev)
    m.particle_count = n
    m.particle_q = x
    m.particle_qd = torch.as_tensor(v, dtype=torch.float32, device=dev).reshape(n, 3).contiguous()
    m.particle_mass = torch.as_tensor(mass, dtype=torch.float32, device=dev).expand(n).contiguous()
    rad = torch.as_tensor(0.0 if radius is None else radius, dtype=torch.float32, device=dev).expand(n).contiguous()
    m.particle_radius = rad
    m.particle_max_radius = float(rad.max()) if n else 0.0
    m.particle_flags = (torch.ones(n, dtype=torch.int32, device=dev) if flags is None
                        else torch.as_tensor(flags, dtype=torch.int32, device=dev).contiguous())
    m.particle_world = (torch.zeros(n, dtype=torch.int32, device=dev) if world is None
                        else torch.as_tensor(world, dtype=torch.int32, device=dev).contiguous())
    m.gravity = torch.as_tensor(gravity, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
    for name, val in (attributes or {}).items():
        dt = torch.int32 if name == "particle_mask" else torch.float32
        setattr(m.sph, name, torch.as_tensor(val, dtype=dt, device=dev).expand(n).contiguous())
    for a in state_attributes:
        m._state_attrs.append(a)
    return m


class HashGrid:
    """``wp.HashGrid`` replacement backed by an ``fs_context`` (grid tables and
    the solvers' cell-sorted scratch live in it)."""

    def __init__(self, dim_x=128, dim_y=128, dim_z=128, device="cuda:0", rounding: int = 0):
        self.dims = (int(dim_x), int(dim_y), int(dim_z))
        self.rounding = int(rounding)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("HashGrid needs a CUDA device: the B200 grid has no CPU implementation")
        self._ctx = C.c_void_p()
        self.capacity = 0
        self.num_points = -1

    @property
    def id(self) -> int:
        return int(self._ctx.value or 0)

    def reserve(self, num_points: int) -> None:
        num_points = int(num_points)
        if self._ctx.value and num_points <= self.capacity:
            return
        lib = _lib.load()
        self._destroy()
        cfg = _lib.GridConfig(*self.dims, self.rounding)
        dev = self.device.index if self.device.index is not None else torch.cuda.current_device()
        _lib.check(lib.fs_context_create(C.byref(self._ctx), num_points, C.byref(cfg), dev), "HashGrid.reserve")
        self.capacity = num_points

    def build(self, points: torch.Tensor, radius: float) -> None:
        n = int(points.shape[0])
        if n > self.capacity:
            self.reserve(n)
        pts = points.contiguous()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(_lib.load().fs_grid_build(self._ctx, pts.data_ptr(), n, float(radius), stream), "HashGrid.build")
        self.num_points = n

    def tables(self):
        """(point_ids, point_cells, cell_starts, cell_ends) of the last build."""
        n = self.num_points
        nc = self.dims[0] * self.dims[1] * self.dims[2]
        t = [torch.empty(k, dtype=torch.int32, device=self.device) for k in (n, n, nc, nc)]
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(_lib.load().fs_grid_tables(self._ctx, *[x.data_ptr() for x in t], stream), "HashGrid.tables")
        return tuple(t)

    def candidates(self, queries: torch.Tensor, radius: float):
        """CSR (offsets, candidates) of ``hash_grid_query`` for each query point."""
        q = queries.contiguous()
        nq = q.shape[0]
        lib = _lib.load()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        counts = torch.empty(nq, dtype=torch.int64, device=self.device)
        _lib.check(lib.fs_grid_candidates(self._ctx, q.data_ptr(), nq, float(radius), counts.data_ptr(), None, None,
                                          stream), "HashGrid.candidates")
        offsets = torch.zeros(nq + 1, dtype=torch.int64, device=self.device)
        offsets[1:] = torch.cumsum(counts, 0)
        total = int(offsets[-1])
        cand = torch.empty(max(total, 1), dtype=torch.int32, device=self.device)
        _lib.check(lib.fs_grid_candidates(self._ctx, q.data_ptr(), nq, float(radius), counts.data_ptr(),
                                          offsets.data_ptr(), cand.data_ptr(), stream), "HashGrid.candidates")
        return offsets, cand[:total]

    def status(self) -> int:
        word = C.c_uint32(0)
        _lib.check(_lib.load().fs_status_read(self._ctx, C.byref(word)), "HashGrid.status")
        return int(word.value)

    def clear_status(self) -> None:
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(_lib.load().fs_status_clear(self._ctx, stream), "HashGrid.clear_status")

    def _destroy(self):
        if self._ctx.value:
            _lib.load().fs_context_destroy(self._ctx)
            self._ctx = C.c_void_p()
            self.capacity = 0

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass


class WorldGrid(HashGrid):
    """Segmented grid of a batched model: one box of cells per world
    (``Model.particle_world``), keyed (world, cell), and one tank of walls
    per world.  Drop it in as ``model.particle_grid`` and the WCSPH, DFSPH
    and PBF solvers advance every world in one launch per pass; the walls of
    each world replace the solver config's ``bound_*``, and DFSPH takes its
    iteration decisions per world.

    ``boxes``: one ``(cell_lo[3], dims[3], (bound_width, bound_height,
    bound_length))`` per world: the box covers the cells whose coordinate
    ``int(x / h)`` (truncating, as the reference's hash grid) lies in
    ``[cell_lo, cell_lo + dims)``, h = the solver's smoothing length.  A
    particle outside its box is binned into the nearest edge cell: clamping
    keeps adjacent cells adjacent, so every neighbour within h is still
    found, but that cell's contents and order (and DFSPH's candidate counts)
    differ from the scene's own hash grid (``Batch.boxes`` adds a margin
    for that)."""

    def __init__(self, boxes, device="cuda:0"):
        super().__init__(1, 1, 1, device=device, rounding=1)
        self.boxes = [(tuple(map(int, lo)), tuple(map(int, dims)), tuple(map(float, walls)))
                      for lo, dims, walls in boxes]
        if not self.boxes:
            raise ValueError("WorldGrid needs at least one world")
        self.num_cells = sum(d[0] * d[1] * d[2] for _, d, _ in self.boxes)

    @property
    def num_worlds(self) -> int:
        return len(self.boxes)

    def _world_boxes(self):
        arr = (_lib.WorldBox * len(self.boxes))()
        for k, (lo, dims, walls) in enumerate(self.boxes):
            arr[k].cell_lo[:] = lo
            arr[k].dims[:] = dims
            arr[k].bound_width, arr[k].bound_height, arr[k].bound_length = walls
        return arr

    def reserve(self, num_points: int) -> None:
        num_points = int(num_points)
        if self._ctx.value and num_points <= self.capacity:
            return
        lib = _lib.load()
        self._destroy()
        dev = self.device.index if self.device.index is not None else torch.cuda.current_device()
        boxes = self._world_boxes()
        _lib.check(lib.fs_context_create_worlds(C.byref(self._ctx), num_points, boxes, len(self.boxes), dev),
                   "WorldGrid.reserve")
        self.capacity = num_points

    def build(self, points: torch.Tensor, radius: float, world: torch.Tensor = None) -> None:
        if world is None:
            raise ValueError("WorldGrid.build needs the particle_world array")
        n = int(points.shape[0])
        if n > self.capacity:
            self.reserve(n)
        pts = points.contiguous()
        w = world.to(torch.int32).contiguous()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(_lib.load().fs_grid_build_worlds(self._ctx, pts.data_ptr(), w.data_ptr(), n, float(radius), stream),
                   "WorldGrid.build")
        self.num_points = n

    def tables(self):
        n = self.num_points
        nc = self.num_cells
        t = [torch.empty(k, dtype=torch.int32, device=self.device) for k in (n, n, nc, nc)]
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(_lib.load().fs_grid_tables(self._ctx, *[x.data_ptr() for x in t], stream), "WorldGrid.tables")
        return tuple(t)

    def candidates(self, queries: torch.Tensor, radius: float, qworld: torch.Tensor = None):
        if qworld is None:
            raise ValueError("WorldGrid.candidates needs the world of each query")
        q = queries.contiguous()
        qw = qworld.to(torch.int32).contiguous()
        nq = q.shape[0]
        lib = _lib.load()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        counts = torch.empty(nq, dtype=torch.int64, device=self.device)
        _lib.check(lib.fs_grid_candidates_worlds(self._ctx, q.data_ptr(), qw.data_ptr(), nq, float(radius),
                                                 counts.data_ptr(), None, None, stream), "WorldGrid.candidates")
        offsets = torch.zeros(nq + 1, dtype=torch.int64, device=self.device)
        offsets[1:] = torch.cumsum(counts, 0)
        total = int(offsets[-1])
        cand = torch.empty(max(total, 1), dtype=torch.int32, device=self.device)
        _lib.check(lib.fs_grid_candidates_worlds(self._ctx, q.data_ptr(), qw.data_ptr(), nq, float(radius),
                                                 counts.data_ptr(), offsets.data_ptr(), cand.data_ptr(), stream),
                   "WorldGrid.candidates")
        return offsets, cand[:total]


class SolverBase:
    def __init__(self, model: Model):
        self.model = model

    def update_contacts(self, contacts) -> None:
        del contacts
