"""Autotuner search logic (no GPU): the grid search times every candidate and
keeps the fastest; the coordinate descent over the tuning axes finds the
optimum of a separable cost while timing far fewer points than the grid."""
from mkf_b200 import autotune

SMALL = {"fuse_ip": (0, 1), "ip_block": (128, 256, 512), "modup_chunk": (8, 12, 24)}


def test_candidate_grid():
    c = autotune.candidates()
    assert len(c) == 2 * 3 * 3 * 4 * 2
    assert {x["fuse_ip"] for x in c} == {0, 1}
    assert {x["ip_block"] for x in c} == {128, 256, 512}
    assert {x["modup_chunk"] for x in c} == {8, 12, 24}
    assert {x["col_split"] for x in c} == {1, 2, 4, 8}
    assert {x["ip_width"] for x in c} == {1, 2}


def test_search_picks_the_fastest():
    seen = []

    def fake(cnd):
        seen.append(cnd)
        return 10.0 - cnd["fuse_ip"] * 3 + abs(cnd["ip_block"] - 256) / 100 + cnd["modup_chunk"] / 100

    best, table = autotune.search(autotune.candidates(SMALL), fake)
    assert best == {"fuse_ip": 1, "ip_block": 256, "modup_chunk": 8}
    assert len(table) == 18 and len(seen) == 36  # two sweeps


def test_descent_finds_the_separable_optimum():
    seen = []

    def fake(c):
        seen.append(dict(c))
        return (10.0 - 3 * c["fuse_ip"] + abs(c["ip_block"] - 256) / 100 + c["modup_chunk"] / 100
                + abs(c["col_split"] - 2) / 10 + (0.05 if c["ip_width"] == 1 else 0.0))

    start = {"fuse_ip": 0, "ip_block": 128, "modup_chunk": 24, "col_split": 8, "ip_width": 1}
    best, table = autotune.descend(autotune.AXES, fake, start)
    assert best == {"fuse_ip": 1, "ip_block": 256, "modup_chunk": 8, "col_split": 2,
                    "ip_width": 2}
    assert len(seen) == 2 * sum(len(v) for v in autotune.AXES.values())
    assert len(table) < len(autotune.candidates())


def test_search_keeps_each_candidates_best_time():
    times = iter([5.0, 1.0, 9.0, 2.0])  # sweep 1: a=5, b=1; sweep 2: a=9, b=2
    best, table = autotune.search([{"x": 0}, {"x": 1}], lambda c: next(times))
    assert best == {"x": 1} and table['{"x": 0}'] == 5.0 and table['{"x": 1}'] == 1.0


def test_split_options_are_the_built_phase_pairs():
    """The NTT splits the kernels are built for: the default (ceil(logN/2)
    row stages) first, then the other split where one exists."""
    assert autotune.split_options(12) == []
    assert autotune.split_options(13) == [7]
    assert autotune.split_options(14) == [7, 8]
    assert autotune.split_options(15) == [8, 7]
    assert autotune.split_options(16) == [8]
    for log_n in (13, 14, 15, 16):
        for rl in autotune.split_options(log_n):
            assert 6 <= log_n - rl <= 8 and 7 <= rl <= 8
