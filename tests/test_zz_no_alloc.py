"""The allocation-free WCSPH density entry point (fs_wcsph_density_noalloc).

It exists for callers that cannot allocate device memory (an allocator that
forbids cudaMalloc, a plugin inside a runtime owning all device memory): it
keeps its scratch in a fixed area compiled into the library.  This file is
collected last so that a run stopping at the first failure has run every
other test first.  The test calls the entry point through the C ABI twice
in a row, on two different particle sets, and
checks density and pressure against the context-based entry points
(fs_grid_build + fs_wcsph_density) within the 1e-5 norm-relative tolerance
of the other GPU tests; the second call also shows that the scratch left by
the first call does not leak into the result.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from fluid_simulation_b200 import _lib
from fluid_simulation_b200.newton_shim import HashGrid
from fluid_simulation_b200.solver import _common as cm
from fluid_simulation_b200.newton_shim import model_from_arrays
from fluid_simulation_b200.solver import SolverWCSPH
from golden_io import rel_err

pytestmark = pytest.mark.gpu


def compressed_block(n_side, spacing, seed):
    """Jittered lattice squeezed to 95 % spacing: clearly positive pressure."""
    rng = np.random.default_rng(seed)
    g = np.arange(n_side) * spacing * 0.95
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = x + rng.uniform(-0.02, 0.02, x.shape) * spacing - 0.5 * g[-1] + np.array([0.0, 0.0, 0.5])
    return x.astype(np.float32)


def run_both(x, spacing, dev, expect_rc=0):
    n = len(x)
    h = np.float32(2.0 * spacing)
    flags = np.ones(n, np.int32)
    flags[::97] = 0  # a few inactive particles
    m = model_from_arrays(x, np.zeros_like(x), 1000.0 * spacing ** 3, device=dev, flags=flags,
                          attributes=dict(rest_density=1000.0, surface_tension=0.0, viscosity=1e-6, stiffness=2.5e5,
                                          exponent=7.0, particle_mask=0), solver_cls=SolverWCSPH)
    ms = cm.model_struct(m, wcsph=True)
    xt = m.particle_q
    stream = torch.cuda.current_stream(dev).cuda_stream
    lib = _lib.load()
    rho_a = torch.zeros(n, device=dev)
    p_a = torch.zeros(n, device=dev)
    grid = HashGrid(device=dev)
    grid.build(xt, float(h))
    _lib.check(lib.fs_wcsph_density(grid._ctx, C.byref(ms), xt.data_ptr(), float(h), 1, rho_a.data_ptr(),
                                    p_a.data_ptr(), stream), "fs_wcsph_density")
    rho_b = torch.full((n,), -1.0, device=dev)
    p_b = torch.full((n,), -1.0, device=dev)
    rc = lib.fs_wcsph_density_noalloc(C.byref(ms), xt.data_ptr(), float(h), 1, rho_b.data_ptr(), p_b.data_ptr(),
                                      stream)
    assert rc == expect_rc, lib.fs_last_error_string()
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in (rho_a, p_a, rho_b, p_b)]


def test_noalloc_density_matches_context_entry_on_two_calls(cuda_device):
    lib = _lib.load()
    cap = lib.fs_noalloc_max_particles()
    assert cap >= 4096
    for seed, (side, spacing) in enumerate([(20, 0.01), (16, 0.013)]):
        x = compressed_block(side, spacing, seed)
        assert len(x) <= cap
        rho_a, p_a, rho_b, p_b = run_both(x, spacing, cuda_device)
        assert rel_err(rho_b, rho_a) <= 1e-5
        assert rel_err(p_b, p_a) <= 1e-5
        assert np.all(rho_b[::97] == 0.0) and np.all(p_b[::97] == 0.0)
        assert p_a.max() > 1e4  # the comparison exercises a real pressure field


def test_noalloc_rejects_more_particles_than_its_scratch(cuda_device):
    lib = _lib.load()
    cap = lib.fs_noalloc_max_particles()
    ms = _lib.Model()
    ms.n = cap + 1
    rc = lib.fs_wcsph_density_noalloc(C.byref(ms), None, 0.1, 1, None, None, None)
    assert rc == _lib.FS_ERR_CAPACITY
    assert b"exceed" in lib.fs_last_error_string()


def test_noalloc_crowded_cell_and_nonfinite_positions(cuda_device):
    """A cell of ~5,000 particles (ordered by the crowded-cell radix sort)
    next to an ordinary block, and a few non-finite positions: the call
    returns FS_ERR_NONFINITE, the non-finite particles get density 0, and
    every finite particle matches the context entry points, which bin the
    non-finite positions apart in the same way."""
    rng = np.random.default_rng(7)
    spacing = 0.01
    x = compressed_block(16, spacing, 3)
    crowd = rng.uniform(0.3, 0.3 + 1.9 * spacing, (5000, 3)).astype(np.float32)  # one cell of width 2 spacing
    x = np.concatenate([x, crowd])
    x[[5, 777, 3000], [0, 1, 2]] = [np.nan, np.inf, -np.inf]
    rho_a, p_a, rho_b, p_b = run_both(x, spacing, cuda_device, expect_rc=_lib.FS_ERR_NONFINITE)
    assert b"not finite" in _lib.load().fs_last_error_string()
    ok = np.isfinite(x).all(1)
    assert rel_err(rho_b[ok], rho_a[ok]) <= 1e-5
    assert rel_err(p_b[ok], p_a[ok]) <= 1e-5
    assert np.all(rho_b[~ok] == 0.0)
    assert rho_a[len(x) - 1] > 100 * np.median(rho_a[:4096])  # the crowd is dense
