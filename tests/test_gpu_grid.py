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
    # crowded cells: above 64 particles a cell is sorted by one block (bitonic
    # up to 4,096 particles, radix above), and the order must stay the same
    crowd = rng.uniform(-1.0, 1.0, (20000, 3)).astype(np.float32)
    crowd[-5000:] = rng.uniform(0.2, 0.2499, (5000, 3))  # one cell of ~5,000 (radix)
    crowd[-5300:-5000] = rng.uniform(0.5, 0.5499, (300, 3))  # one of ~300 (bitonic)
    rng.shuffle(crowd)
    yield "crowded_cells", crowd, 0.05, (128, 128, 128), 0


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
    q = np.concatenate([x[: min(len(x), 3000)] if name != "crowded_cells" else x[np.all(x < 0.15, 1)][:3000],
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


def test_one_cell_of_200000_particles_builds_in_milliseconds(cuda_device):
    """200,000 particles in one cell: the in-cell order is sorted by a radix
    sort in O(N) (not by k^2 comparisons), still bit-identical to the
    stable order, and a build takes milliseconds."""
    rng = np.random.default_rng(12)
    x = rng.uniform(0.0, 0.0499, (200000, 3)).astype(np.float32)
    g = HashGrid(device=cuda_device)
    g.reserve(len(x))
    xt = torch.as_tensor(x, device=cuda_device)
    g.build(xt, 0.05)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(3):
        g.build(xt, 0.05)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / 3
    ids, cells, starts, ends = [t.cpu().numpy() for t in g.tables()]
    np.testing.assert_array_equal(ids, np.arange(len(x)))  # one cell: ascending ids
    ref = oracle.grid_build(x, 0.05)
    np.testing.assert_array_equal(cells, ref["point_cells"])
    assert ms < 50.0, f"grid build of one crowded cell took {ms:.1f} ms"


def test_nonfinite_positions_are_binned_apart(cuda_device):
    """Non-finite positions raise the status, take a bucket after every cell
    (no query visits it; their ids ascend there), and leave the finite
    particles' tables as the grid of the finite particles alone gives them."""
    rng = np.random.default_rng(13)
    x = rng.uniform(-0.2, 0.2, (6000, 3)).astype(np.float32)
    bad = rng.choice(len(x), 500, replace=False)
    x[bad[:200], 0] = np.nan
    x[bad[200:400], 1] = np.inf
    x[bad[400:], 2] = -np.inf
    finite = np.setdiff1d(np.arange(len(x)), bad)
    ref = oracle.grid_build(x[finite], 0.03)
    g = HashGrid(device=cuda_device)
    g.build(torch.as_tensor(x, device=cuda_device), 0.03)
    assert g.status() & 1
    ids, cells, starts, ends = [t.cpu().numpy() for t in g.tables()]
    nf = len(finite)
    np.testing.assert_array_equal(ids[:nf], finite[ref["point_ids"]])
    np.testing.assert_array_equal(cells[:nf], ref["point_cells"])
    np.testing.assert_array_equal(ids[nf:], np.sort(bad))
    assert np.all(cells[nf:] == 128 ** 3)
    occ = ref["cell_ends"] > ref["cell_starts"]
    np.testing.assert_array_equal(starts[occ], ref["cell_starts"][occ])
    np.testing.assert_array_equal(ends[occ], ref["cell_ends"][occ])
    # a query from anywhere never returns a non-finite particle
    off, cand = g.candidates(torch.as_tensor(x[finite[:500]], device=cuda_device), 0.03)
    assert not np.isin(cand.cpu().numpy(), bad).any()
