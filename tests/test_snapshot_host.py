"""On-disk snapshots (fluid_simulation_b200.snapshot, batch.save_batch):
round trips, the reference's initial-position digest, and refusal of files
whose positions do not match their digests."""

import json
import types

import numpy as np
import pytest
import torch

from fluid_simulation_b200 import snapshot
from fluid_simulation_b200.batch import load_batch, make_batch, save_batch, scene_table
from fluid_simulation_b200.scene import make_scene


def test_digest_is_the_scene_report_digest():
    s = make_scene(10000)
    assert snapshot.positions_sha256(s.positions) == s.report()["initial_position_sha256"]


def test_round_trip_keeps_every_bit(tmp_path):
    s = make_scene(10000)
    rng = np.random.default_rng(0)
    x = s.positions + rng.normal(size=s.positions.shape).astype(np.float32) * 1e-3
    v = rng.normal(size=x.shape).astype(np.float32)
    rho = rng.uniform(900, 1100, len(x)).astype(np.float32)
    path = tmp_path / "frame_0007"
    info = snapshot.save(path, x, torch.as_tensor(v), rho, initial_positions=s.positions, frame=7, solver="pbf")
    assert info["initial_position_sha256"] == s.report()["initial_position_sha256"]
    snap = snapshot.load(path)  # no suffix added to the path
    assert np.array_equal(snap.particle_q, x) and np.array_equal(snap.particle_qd, v)
    assert np.array_equal(snap.rho, rho) and snap.particle_world is None
    assert snap.meta["frame"] == 7 and snap.meta["solver"] == "pbf" and snap.count == len(x)
    assert snap.matches(s.positions) and not snap.matches(x)
    # readable with numpy alone
    with np.load(path) as z:
        assert json.loads(str(z["meta"]))["format"] == snapshot.FORMAT


def test_save_needs_the_initial_condition(tmp_path):
    x = np.zeros((4, 3), np.float32)
    with pytest.raises(ValueError, match="initial"):
        snapshot.save(tmp_path / "a.npz", x, x)
    with pytest.raises(ValueError, match="do not match"):
        snapshot.save(tmp_path / "a.npz", x, x, initial_positions=x, initial_position_sha256="0" * 64)
    with pytest.raises(ValueError, match="rows"):
        snapshot.save(tmp_path / "a.npz", x, x, np.zeros(3, np.float32), initial_positions=x)


def test_restore_state_copies_into_a_state():
    x = np.arange(12, dtype=np.float32).reshape(4, 3)
    snap = snapshot.Snapshot(particle_q=x, particle_qd=-x, rho=np.full(4, 2.0, np.float32))
    st = types.SimpleNamespace(particle_q=torch.zeros(4, 3), particle_qd=torch.zeros(4, 3),
                               sph=types.SimpleNamespace(rho=torch.zeros(4)))
    snapshot.restore_state(snap, st)
    assert torch.equal(st.particle_q, torch.as_tensor(x)) and torch.equal(st.particle_qd, torch.as_tensor(-x))
    assert torch.equal(st.sph.rho, torch.full((4,), 2.0))
    with pytest.raises(ValueError, match="particles"):
        snapshot.restore_state(snap, types.SimpleNamespace(particle_q=torch.zeros(5, 3)))


def test_batch_round_trip(tmp_path):
    b = make_batch(n_scenes=12, seed=4, n_lo=500, n_hi=3000)
    path = tmp_path / "batch.npz"
    info = save_batch(path, b)
    assert info["scenes"] == 12 and info["particle_count"] == b.total
    b2, snap = load_batch(path)
    assert np.array_equal(b2.positions(), b.positions())
    assert np.array_equal(snap.particle_world, b.world())
    assert b2.boxes() == b.boxes() and b2.spacing == b.spacing
    for k, v in scene_table(b).items():
        assert np.array_equal(scene_table(b2)[k], v), k


def test_batch_with_altered_positions_is_refused(tmp_path):
    b = make_batch(n_scenes=3, seed=5, n_lo=500, n_hi=1000)
    path = tmp_path / "batch.npz"
    save_batch(path, b)
    with np.load(path) as z:
        arrays = {k: z[k] for k in z.files}
    arrays["particle_q"] = arrays["particle_q"].copy()
    arrays["particle_q"][b.starts[1], 0] += np.float32(1e-3)  # first particle of scene 1
    with open(path, "wb") as f:
        np.savez(f, **arrays)
    with pytest.raises(ValueError, match="scene 1"):
        load_batch(path)
