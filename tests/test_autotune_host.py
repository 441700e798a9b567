"""Candidate lists and selection rule of the launch autotuner (no GPU)."""

from fluid_simulation_b200.autotune import DEFAULT, Tuning, candidates, choose


def test_candidates_cover_the_knobs_with_the_default_first():
    for kind in ("pbf", "dfsph"):
        c = candidates(kind)
        assert c[0] == Tuning(*DEFAULT) and len(c) == 9 and len(set(c)) == 9
        assert all(t.cell_ratio == 1.0 for t in c)
    w = candidates("wcsph")
    assert w[0] == Tuning(*DEFAULT) and len(w) == 18
    assert {t.cell_ratio for t in w} == {1.0, 0.5}
    # batched contexts bin in cells of width h
    assert all(t.cell_ratio == 1.0 for t in candidates("wcsph", batched=True))


def test_choose_takes_the_fastest_and_the_first_of_equals():
    a, b, c = Tuning(128, 1, 1.0), Tuning(64, 2, 1.0), Tuning(256, 1, 1.0)
    assert choose({a: 2.0, b: 1.5, c: 1.7}) == b
    assert choose({a: 1.0, b: 1.0, c: 1.0}) == a
