"""Autotuner search logic (no GPU): every candidate is timed once and the
fastest is chosen; the candidate grid covers every tuning axis."""
from mkf_b200 import autotune


def test_candidate_grid():
    c = autotune.candidates()
    assert len(c) == 2 * 3 * 3
    assert {x["fuse_ip"] for x in c} == {0, 1}
    assert {x["ip_block"] for x in c} == {128, 256, 512}
    assert {x["modup_chunk"] for x in c} == {8, 12, 24}


def test_search_picks_the_fastest():
    seen = []

    def fake(cnd):
        seen.append(cnd)
        return 10.0 - cnd["fuse_ip"] * 3 + abs(cnd["ip_block"] - 256) / 100 + cnd["modup_chunk"] / 100

    best, table = autotune.search(autotune.candidates(), fake)
    assert best == {"fuse_ip": 1, "ip_block": 256, "modup_chunk": 8}
    assert len(table) == 18 and len(seen) == 36  # two sweeps


def test_search_keeps_each_candidates_best_time():
    times = iter([5.0, 1.0, 9.0, 2.0])  # sweep 1: a=5, b=1; sweep 2: a=9, b=2
    best, table = autotune.search([{"x": 0}, {"x": 1}], lambda c: next(times))
    assert best == {"x": 1} and table['{"x": 0}'] == 5.0 and table['{"x": 1}'] == 1.0
