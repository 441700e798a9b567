"""Drop-in boundary (CPU): the C ABI and the reference-facing Python surface.

* every function declared in include/fluid_b200.h is exported by the
  library and bound by the ctypes layer;
* the solver classes register the same custom attributes (name, frequency,
  assignment, dtype, default, namespace) and carry the same config fields and
  defaults as the reference solvers (recorded from the reference's own
  register_custom_attributes / dataclasses in tests/golden/attributes.json);
* the dam-break scene generator reproduces the reference's scenes bit for bit
  (SHA-256 of the positions recorded in tests/golden/scenes.json) and the
  spec pins of unit_test_dam_break.py:19-27.
"""

import ctypes
import dataclasses
import json
import os
import re

import numpy as np
import pytest

from fluid_simulation_b200 import _lib
from fluid_simulation_b200.newton_shim import Model, ModelBuilder, vec3
from fluid_simulation_b200.scene import make_scene
from fluid_simulation_b200.solver import SolverDFSPH, SolverPBF, SolverWCSPH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def header_functions():
    src = open(os.path.join(ROOT, "include", "fluid_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|int64_t|const char\*)\s+(fs_[a-z0-9_]+)\s*\(", src, re.M)))


def test_library_exports_every_declared_function():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} not bound in _lib.SIGNATURES"
    assert set(_lib.SIGNATURES) == set(names)


def test_library_version_and_error_string():
    lib = _lib.load()
    assert b"sm_100a" in lib.fs_version()
    assert isinstance(lib.fs_last_error_string(), bytes)


def test_invalid_arguments_fail_without_a_gpu():
    lib = _lib.load()
    ctx = ctypes.c_void_p()
    bad = _lib.GridConfig(0, 128, 128, 0)
    assert lib.fs_context_create(ctypes.byref(ctx), 10, ctypes.byref(bad), 0) == _lib.FS_ERR_INVALID
    assert b"bad arguments" in lib.fs_last_error_string()
    assert lib.fs_grid_build(None, None, 0, 0.1, None) == _lib.FS_ERR_INVALID


def _registered(cls):
    b = ModelBuilder()
    cls.register_custom_attributes(b)
    out = []
    for a in b.custom_attributes.values():
        dtype = {int: "int32", float: "float32", vec3: "vec3"}[a.dtype]
        default = list(a.default) if a.dtype is vec3 else a.default
        out.append(dict(name=a.name, frequency=a.frequency.name, assignment=a.assignment.name, dtype=dtype,
                        default=default, namespace=a.namespace))
    return out


@pytest.mark.parametrize("kind,cls", [("wcsph", SolverWCSPH), ("dfsph", SolverDFSPH), ("pbf", SolverPBF)])
def test_custom_attributes_match_reference(kind, cls):
    ref = json.load(open(os.path.join(GOLDEN, "attributes.json")))
    assert _registered(cls) == ref[kind]


@pytest.mark.parametrize("kind,cfg", [("wcsph", SolverWCSPH.SphConfig), ("dfsph", SolverDFSPH.SphConfig),
                                      ("pbf", SolverPBF.PbfConfig)])
def test_config_defaults_match_reference(kind, cfg):
    ref = json.load(open(os.path.join(GOLDEN, "attributes.json")))[kind + "_config_defaults"]
    assert dataclasses.asdict(cfg()) == ref


def test_solvers_need_cuda_and_fail_loudly_on_cpu():
    from fluid_simulation_b200.newton_shim import model_from_arrays
    x = np.zeros((4, 3), np.float32)
    m = model_from_arrays(x, x, 1.0, device="cpu", solver_cls=SolverWCSPH)
    with pytest.raises(RuntimeError, match="CUDA"):
        SolverWCSPH(m, SolverWCSPH.SphConfig())


def test_smoothing_length_property():
    m = Model(device="cpu")
    s = SolverPBF.__new__(SolverPBF)
    s.config = SolverPBF.PbfConfig(particle_length=0.01, smoothing_length_coff=2.0)
    assert s.smoothing_length == pytest.approx(0.02)
    del m


def test_scene_generator_reproduces_reference_scenes():
    import hashlib
    ref = json.load(open(os.path.join(GOLDEN, "scenes.json")))
    for target, r in ref.items():
        s = make_scene(int(target))
        assert s.count == r["count"]
        assert s.spacing == r["spacing"] and s.radius == r["radius"]
        assert hashlib.sha256(s.positions.tobytes()).hexdigest() == r["sha256"]


def test_default_scene_spec_pins():
    # unit_test_dam_break.py:19-27
    scene = make_scene()
    assert scene.count == 401856
    assert scene.report()["lattice_resolution"] == [78, 56, 92]
    np.testing.assert_allclose(scene.positions.min(axis=0), [-1.17, -0.25, 0.03], atol=1e-6)
    np.testing.assert_allclose(scene.positions.max(axis=0), [-0.468, 0.25, 0.8508], atol=1e-6)
    assert scene.radius * 2.0 == scene.spacing
    assert scene.mass == scene.spec.density * scene.volume
    assert scene.ideal_height == pytest.approx(scene.count * scene.mass / 1000.0 / 1.344)
