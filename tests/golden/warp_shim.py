"""Substitute ``warp`` / ``newton`` runtime for executing the reference solver
source on the CPU, one Python call per thread, in FP32.

Used only by ``make_golden.py`` (fixture generation in a container that has
the reference sources); nothing at test time imports it.  warp-lang 1.17.0 and
newton 1.6.0 are not installable here, so this module provides the subset of
their API that ``solver/sph/solver_wcsph.py``, ``solver/sph/solver_dfsph.py``,
``solver/pbf/solver_pbf.py`` and the particle-separation kernels of
``solver/apic/solver_apic.py`` use:

* ``@wp.kernel`` / ``@wp.func`` keep the Python function; ``wp.launch`` runs
  the kernel body for tid = 0..dim-1, converting scalar arguments to the
  annotated Warp type (``float`` -> float32).
* arrays hold numpy float32 / int32 data; ``vec3`` values are float32 triples
  with warp's component-wise arithmetic (``vec / s`` divides each component).
* ``wp.HashGrid`` restates warp's published hash-grid algorithm (truncating
  float-to-int conversion of ``p * (1/radius)``, 2^20 origin shift, modulo the
  grid dims, x-fastest linearisation, stable sort by cell, 27-cell query
  visited z/y/x without distance filtering).
* ``newton`` provides ``ParticleFlags.ACTIVE`` (bit 0), ``SolverBase``,
  ``ModelBuilder.CustomAttribute`` and the attribute enums.

numpy >= 2 keeps float32 scalar arithmetic in float32 when mixed with Python
floats (NEP 50), which gives per-operation float32 rounding.
"""

from __future__ import annotations

import contextlib
import enum
import inspect
import math
import sys
import types

import numpy as np

f32 = np.float32


# ------------------------------------------------------------------ vec3 ----
class vec3:
    __slots__ = ("c",)

    def __init__(self, *args):
        if len(args) == 1:
            v = f32(args[0])
            self.c = [v, v, v]
        elif len(args) == 3:
            self.c = [f32(a) for a in args]
        elif len(args) == 0:
            self.c = [f32(0.0)] * 3
        else:
            raise TypeError("vec3 takes 0, 1 or 3 arguments")

    @staticmethod
    def _of(a, b, c):
        v = vec3.__new__(vec3)
        v.c = [a, b, c]
        return v

    def __getitem__(self, k):
        return self.c[k]

    def __setitem__(self, k, val):
        self.c = list(self.c)
        self.c[k] = f32(val)

    def __add__(self, o):
        return vec3._of(self.c[0] + o.c[0], self.c[1] + o.c[1], self.c[2] + o.c[2])

    def __sub__(self, o):
        return vec3._of(self.c[0] - o.c[0], self.c[1] - o.c[1], self.c[2] - o.c[2])

    def __neg__(self):
        return vec3._of(-self.c[0], -self.c[1], -self.c[2])

    def __mul__(self, s):
        s = f32(s)
        return vec3._of(self.c[0] * s, self.c[1] * s, self.c[2] * s)

    def __rmul__(self, s):
        s = f32(s)
        return vec3._of(s * self.c[0], s * self.c[1], s * self.c[2])

    def __truediv__(self, s):
        s = f32(s)
        return vec3._of(self.c[0] / s, self.c[1] / s, self.c[2] / s)

    def __repr__(self):
        return f"vec3({self.c[0]}, {self.c[1]}, {self.c[2]})"


def dot(a, b):
    return a.c[0] * b.c[0] + a.c[1] * b.c[1] + a.c[2] * b.c[2]


def length(a):
    return f32(np.sqrt(dot(a, a)))


def _num(x):
    return isinstance(x, (float, np.floating))


def clamp(x, a, b):
    """warp's clamp: x limited to [a, b] (min(max(x, a), b); the ranges used
    here all have a <= b)."""
    return min(max(x, a), b)


def max(a, b):  # noqa: A001 - warp name
    r = a if a > b else b
    return f32(r) if (_num(a) or _num(b)) else r


def min(a, b):  # noqa: A001 - warp name
    r = a if a < b else b
    return f32(r) if (_num(a) or _num(b)) else r


def pow(a, b):  # noqa: A001 - warp name
    with np.errstate(all="ignore"):
        return np.power(f32(a), f32(b))


def isfinite(x):
    return bool(np.isfinite(x))


# A Python float: kernels mix it with float32 operands, which rounds it to
# float32 there (NEP 50), while host-side calls of a wp.func (SolverPBF._w_delta_q)
# evaluate in double, as warp does for functions called from Python scope.
pi = math.pi
inf = float("inf")
int32 = np.int32
uint64 = np.uint64
float32 = np.float32


# ----------------------------------------------------------------- arrays ----
class array:
    """Annotation form ``wp.array(dtype=...)`` and runtime container."""

    def __init__(self, data=None, dtype=float, device=None):
        self.dtype = dtype
        if data is None:
            self.data = None
            return
        self.data = np.array(data, dtype=_np_dtype(dtype), copy=True)
        if dtype is vec3:
            self.data = self.data.reshape(-1, 3)

    @property
    def shape(self):
        return (self.data.shape[0],)

    def __len__(self):
        return self.data.shape[0]

    def __getitem__(self, i):
        if self.dtype is vec3:
            r = self.data[i]
            return vec3._of(r[0], r[1], r[2])
        return self.data[i]

    def __setitem__(self, i, val):
        if self.dtype is vec3:
            self.data[i, 0], self.data[i, 1], self.data[i, 2] = val.c
        else:
            self.data[i] = val

    def numpy(self):
        return self.data.copy()

    def assign(self, values):
        self.data[...] = np.asarray(values, dtype=self.data.dtype).reshape(self.data.shape)

    def zero_(self):
        self.data[...] = 0


def _np_dtype(dtype):
    if dtype is vec3 or dtype in (float, np.float32):
        return np.float32
    if dtype in (int, np.int32):
        return np.int32
    return dtype


def empty(n, dtype=float, device=None):
    shape = (n, 3) if dtype is vec3 else (n,)
    return array(np.zeros(shape, _np_dtype(dtype)), dtype=dtype)


def zeros(n, dtype=float, device=None):
    return empty(n, dtype, device)


def from_numpy(a, dtype=float, device=None):
    return array(a, dtype=dtype)


def copy(dst, src):
    dst.data[...] = src.data


@contextlib.contextmanager
def ScopedDevice(device):  # noqa: N802 - warp name
    yield


# ------------------------------------------------------------ kernels ----
def func(f):
    return f


def kernel(f):
    f.__warp_kernel__ = True
    return f


_tid = 0


def tid():
    return _tid


def _convert(value, annotation):
    if annotation is float or annotation is np.float32:
        return f32(value)
    if annotation is int or annotation is np.int32:
        return int(value)
    if annotation is bool:
        return bool(value)
    if annotation is vec3:
        return value if isinstance(value, vec3) else vec3(*value)
    if annotation is np.uint64:
        return int(value)
    return value


def launch(kernel, dim, inputs=(), outputs=(), device=None):
    global _tid
    params = list(inspect.signature(kernel).parameters.values())
    args = list(inputs) + list(outputs)
    if len(args) != len(params):
        raise TypeError(f"{kernel.__name__}: expected {len(params)} args, got {len(args)}")
    conv = [_convert(a, p.annotation) for a, p in zip(args, params)]
    for t in range(int(dim)):
        _tid = t
        kernel(*conv)


# ------------------------------------------------------------ hash grid ----
_grids: dict[int, "HashGrid"] = {}


def _to_cell(v):
    v = f32(v)
    if v != v:
        return 0
    if v > f32(536870912.0):
        return 536870912
    if v < f32(-536870912.0):
        return -536870912
    return int(v)  # truncation toward zero, as warp's C cast


class HashGrid:
    def __init__(self, dim_x, dim_y, dim_z, device=None):
        self.dims = (int(dim_x), int(dim_y), int(dim_z))
        self.id = id(self)
        _grids[self.id] = self
        self.point_ids = np.zeros(0, np.int32)
        self.cell_starts = np.zeros(self.dims[0] * self.dims[1] * self.dims[2], np.int32)
        self.cell_ends = np.zeros_like(self.cell_starts)
        self.inv = f32(1.0)

    def reserve(self, n):
        pass

    def phys(self, x, y, z):
        dx, dy, dz = self.dims
        o = 1 << 20
        x, y, z = builtins_max(0, x + o), builtins_max(0, y + o), builtins_max(0, z + o)
        return (z % dz) * (dx * dy) + (y % dy) * dx + (x % dx)

    def build(self, points, radius):
        self.inv = f32(1.0) / f32(radius)
        p = points.data
        keys = np.array([self.phys(_to_cell(q[0] * self.inv), _to_cell(q[1] * self.inv),
                                   _to_cell(q[2] * self.inv)) for q in p], dtype=np.int64)
        order = np.argsort(keys, kind="stable").astype(np.int32)
        self.point_ids = order
        sk = keys[order]
        self.cell_starts[:] = 0
        self.cell_ends[:] = 0
        for s in range(len(sk)):
            c = sk[s]
            if s == 0 or sk[s - 1] != c:
                self.cell_starts[c] = s
            if s == len(sk) - 1 or sk[s + 1] != c:
                self.cell_ends[c] = s + 1

    def query(self, pos, r):
        r = f32(r)
        inv = self.inv
        x0 = _to_cell((pos[0] - r) * inv)
        y0 = _to_cell((pos[1] - r) * inv)
        z0 = _to_cell((pos[2] - r) * inv)
        x1 = builtins_min(_to_cell((pos[0] + r) * inv), x0 + self.dims[0] - 1)
        y1 = builtins_min(_to_cell((pos[1] + r) * inv), y0 + self.dims[1] - 1)
        z1 = builtins_min(_to_cell((pos[2] + r) * inv), z0 + self.dims[2] - 1)
        out = []
        for z in range(z0, z1 + 1):
            for y in range(y0, y1 + 1):
                for x in range(x0, x1 + 1):
                    c = self.phys(x, y, z)
                    out.extend(int(j) for j in self.point_ids[self.cell_starts[c]:self.cell_ends[c]])
        return out


import builtins as _b  # noqa: E402

builtins_max = _b.max
builtins_min = _b.min


def hash_grid_point_id(grid_id, index):
    return int(_grids[int(grid_id)].point_ids[index])


def hash_grid_query(grid_id, pos, radius):
    return iter(_grids[int(grid_id)].query(pos, radius))


# ---------------------------------------------------------------- newton ----
def make_newton_module():
    newton = types.ModuleType("newton")

    class ParticleFlags(enum.IntFlag):
        ACTIVE = 1

    class Model:
        class AttributeFrequency(enum.Enum):
            PARTICLE = 1

        class AttributeAssignment(enum.Enum):
            MODEL = 1
            STATE = 2

    class ModelBuilder:
        class CustomAttribute:
            def __init__(self, name, frequency, assignment, dtype, default, namespace=None):
                self.name, self.frequency, self.assignment = name, frequency, assignment
                self.dtype, self.default, self.namespace = dtype, default, namespace

        def __init__(self):
            self.custom_attributes = []

        def add_custom_attribute(self, attr):
            self.custom_attributes.append(attr)

    class State:
        pass

    class Control:
        pass

    class Contacts:
        pass

    class SolverBase:
        def __init__(self, model):
            self.model = model

    solvers = types.ModuleType("newton.solvers")
    solvers.SolverBase = SolverBase
    newton.ParticleFlags = ParticleFlags
    newton.Model = Model
    newton.ModelBuilder = ModelBuilder
    newton.State = State
    newton.Control = Control
    newton.Contacts = Contacts
    newton.solvers = solvers
    return newton, solvers


def install():
    """Register the substitute modules as ``warp``, ``newton``, ``newton.solvers``."""
    wp = sys.modules[__name__]
    newton, solvers = make_newton_module()
    sys.modules["warp"] = wp
    sys.modules["newton"] = newton
    sys.modules["newton.solvers"] = solvers
    return wp, newton
