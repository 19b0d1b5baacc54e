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
    assert len(seen) == len(table) == 18
