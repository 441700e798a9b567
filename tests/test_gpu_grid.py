"""Hash-grid build and query on the GPU against the oracle's restatement of
warp's wp.HashGrid: sort order (point_ids), sorted cell keys, cell ranges of
every occupied cell and complete candidate lists must be bit-identical."""

import numpy as np
import pytest
import torch

import oracle
from fluid_simulation_b200.newton_shim import HashGrid
from fluid_simulation_b200.scene import make_scene, stress_lattice

pytestmark = pytest.mark.gpu


def point_sets():
    rng = np.random.default_rng(11)
    yield "dam540", make_scene(512).positions, 2.0 * make_scene(512).spacing, (128, 128, 128), 0
    s = make_scene(10000)
    yield "dam9936", s.positions, 2.0 * s.spacing, (128, 128, 128), 0
    # x extent of 2.4 m at h = 0.018 spans more than 128 cells: buckets alias
    yield "aliasing", rng.uniform([-1.2, -0.28, 0.0], [1.2, 0.28, 1.2], (20000, 3)).astype(np.float32), 0.018, \
        (128, 128, 128), 0
    yield "negative_floor", rng.uniform(-0.5, 0.5, (8000, 3)).astype(np.float32), 0.05, (128, 128, 128), 1
    yield "small_dims", rng.uniform(-0.3, 0.7, (5000, 3)).astype(np.float32), 0.04, (7, 5, 3), 0
    x, _, sp = stress_lattice(cells=20, box=0.25)
    yield "bcc_lattice", x, 2.0 * sp, (128, 128, 128), 0
    yield "single_cell", np.full((37, 3), 0.01, np.float32), 0.1, (128, 128, 128), 0


@pytest.mark.parametrize("case", list(point_sets()), ids=lambda c: c[0])
def test_grid_tables_bit_exact(case, cuda_device):
    name, x, h, dims, rounding = case
    ref = oracle.grid_build(x, h, dims, rounding)
    g = HashGrid(*dims, device=cuda_device, rounding=rounding)
    g.reserve(len(x))
    g.build(torch.as_tensor(x, device=cuda_device), h)
    ids, cells, starts, ends = [t.cpu().numpy() for t in g.tables()]
    np.testing.assert_array_equal(ids, ref["point_ids"])
    np.testing.assert_array_equal(cells, ref["point_cells"])
    occ = ref["cell_ends"] > ref["cell_starts"]
    np.testing.assert_array_equal(starts[occ], ref["cell_starts"][occ])
    np.testing.assert_array_equal(ends[occ], ref["cell_ends"][occ])
    assert np.all(starts[~occ] == ends[~occ])  # empty cells give empty ranges
    assert g.status() == 0


@pytest.mark.parametrize("case", list(point_sets()), ids=lambda c: c[0])
def test_grid_candidates_bit_exact(case, cuda_device):
    name, x, h, dims, rounding = case
    rng = np.random.default_rng(5)
    q = np.concatenate([x[: min(len(x), 3000)],
                        x[rng.integers(0, len(x), 500)] + rng.normal(0, h, (500, 3)).astype(np.float32)])
    off_ref, cand_ref = oracle.grid_candidates(x, h, q, h, dims, rounding)
    g = HashGrid(*dims, device=cuda_device, rounding=rounding)
    g.build(torch.as_tensor(x, device=cuda_device), h)
    off, cand = g.candidates(torch.as_tensor(q, device=cuda_device), h)
    np.testing.assert_array_equal(off.cpu().numpy(), off_ref)
    np.testing.assert_array_equal(cand.cpu().numpy(), cand_ref)


@pytest.mark.parametrize("dims,rounding", [((128, 128, 128), 0), ((7, 5, 3), 1)])
def test_far_queries_bit_exact(dims, rounding, cuda_device):
    """Queries millions of cells away (and at +-3e38, whose scaled
    coordinates overflow to infinity): cell coordinates clamp and wrap as in
    warp's hash grid, including the per-cell walk of x runs that start below
    the shifted range."""
    rng = np.random.default_rng(2)
    x = rng.uniform(-0.5, 0.5, (3000, 3)).astype(np.float32)
    h = 0.05
    q = np.array([[-1e7, 0, 0], [1e7, 0, 0], [0, -1e7, 0], [0, 0, 1e7], [-3e38, 0.1, 0.1], [3e38, -3e38, 0.0],
                  [-2.0e5, 0.0, 0.0], [-5.3e4, 0.2, -0.2], [0.1, 0.1, 0.1]], np.float32)
    off_ref, cand_ref = oracle.grid_candidates(x, h, q, h, dims, rounding)
    g = HashGrid(*dims, device=cuda_device, rounding=rounding)
    g.build(torch.as_tensor(x, device=cuda_device), h)
    off, cand = g.candidates(torch.as_tensor(q, device=cuda_device), h)
    np.testing.assert_array_equal(off.cpu().numpy(), off_ref)
    np.testing.assert_array_equal(cand.cpu().numpy(), cand_ref)


def test_neighbour_sets_match_brute_force(cuda_device):
    """Within-h neighbour sets from the GPU candidates equal an O(N^2) search."""
    rng = np.random.default_rng(3)
    x = rng.uniform(-0.2, 0.2, (3000, 3)).astype(np.float32)
    h = np.float32(0.03)
    g = HashGrid(device=cuda_device)
    g.build(torch.as_tensor(x, device=cuda_device), float(h))
    off, cand = (t.cpu().numpy() for t in g.candidates(torch.as_tensor(x, device=cuda_device), float(h)))
    d = x[:, None, :] - x[None, :, :]
    r = np.sqrt(np.sum(d * d, axis=-1, dtype=np.float32), dtype=np.float32)
    for i in range(0, len(x), 7):
        c = cand[off[i]:off[i + 1]]
        got = set(int(j) for j in c if r[i, j] < h)
        want = set(np.nonzero(r[i] < h)[0].tolist())
        assert got == want


def test_nonfinite_position_sets_status(cuda_device):
    x = np.zeros((64, 3), np.float32)
    x[:, 0] = np.linspace(0, 1, 64)
    x[5, 1] = np.nan
    g = HashGrid(device=cuda_device)
    g.build(torch.as_tensor(x, device=cuda_device), 0.1)
    assert g.status() & 1  # FS_STATUS_NONFINITE
    g.clear_status()
    assert g.status() == 0
