"""CPU tests of the autotuner's search logic and tables (no GPU: synthetic
cost functions; the library's tuning entry points need no device)."""
import json

import pytest

from uaamg_b200 import autotune


def test_search_finds_the_optimum_of_a_separable_cost():
    target = {"a": 3, "b": 20, "c": 1}
    space = {"a": [1, 2, 3, 4], "b": [10, 20, 30], "c": [0, 1]}

    def cost(s):
        return 1.0 + (s["a"] - 3) ** 2 + abs(s["b"] - 20) / 10 + (1 - s["c"]) * 0.5

    log = []
    best, c = autotune.search(cost, space, {"a": 1, "b": 30, "c": 0}, log=log)
    assert best == target and c == 1.0
    # no setting is measured twice
    keys = [tuple(sorted(t["setting"].items())) for t in log]
    assert len(keys) == len(set(keys))


def test_search_needs_a_real_gain_to_move():
    """Candidates within min_gain of the incumbent do not replace it (timing
    noise must not churn the table)."""
    space = {"a": [0, 1, 2]}
    best, c = autotune.search(lambda s: {0: 1.0, 1: 0.995, 2: 1.2}[s["a"]], space, {"a": 0}, min_gain=0.01)
    assert best == {"a": 0} and c == 1.0
    best, _ = autotune.search(lambda s: {0: 1.0, 1: 0.9, 2: 1.2}[s["a"]], space, {"a": 0}, min_gain=0.01)
    assert best == {"a": 1}


def test_search_rounds_continue_until_nothing_improves():
    """With coupled knobs one pass can stop short; later rounds continue
    from the improved setting until a round improves nothing."""
    space = {"y": [0, 1, 2], "x": [0, 1, 2]}  # y is visited before x

    def cost(s):  # y only pays off once x has moved
        return abs(s["y"] - s["x"]) + 2 * abs(s["x"] - 2)

    best, c = autotune.search(cost, space, {"x": 0, "y": 0}, max_rounds=1, min_gain=0.0)
    assert best == {"x": 2, "y": 0} and c == 2
    best, c = autotune.search(cost, space, {"x": 0, "y": 0}, max_rounds=4, min_gain=0.0)
    assert best == {"x": 2, "y": 2} and c == 0


def test_table_round_trip_and_key(tmp_path):
    path = autotune.table_path("NVIDIA B200", 148, str(tmp_path))
    assert path.endswith("NVIDIA_B200_148sm.json")
    table = {"gpu": "NVIDIA B200", "sm_count": 148,
             "tuning": {"staged_min_leaves": 32, "split_min_leaves": 2048, "pipe_min_leaves": 8192,
                        "elem_ctas_per_sm": 8, "bottom_cycle": 1}}
    with open(path, "w") as f:
        json.dump(table, f)
    assert autotune.load(path)["tuning"]["split_min_leaves"] == 2048
    bad = tmp_path / "bad.json"
    bad.write_text(json.dumps({"tuning": {"staged_min_leaves": 1}}))
    with pytest.raises(ValueError):
        autotune.load(str(bad))


def test_library_tuning_set_get_and_validation():
    from uaamg_b200 import build
    build.build()
    old = autotune.get()
    try:
        autotune.set({"staged_min_leaves": 32, "split_min_leaves": 4096, "elem_ctas_per_sm": 8, "bottom_cycle": 0})
        t = autotune.get()
        assert t["staged_min_leaves"] == 32 and t["split_min_leaves"] == 4096
        assert t["elem_ctas_per_sm"] == 8 and t["bottom_cycle"] == 0
        with pytest.raises(Exception):
            autotune.set({"elem_ctas_per_sm": 0})
        with pytest.raises(Exception):
            autotune.set({"bottom_cycle": 2})
        assert autotune.get() == t  # a rejected setting changes nothing
    finally:
        autotune.set(old)
    assert autotune.get() == old


def test_committed_tables_are_valid():
    import os
    if not os.path.isdir(autotune.TABLE_DIR):
        pytest.skip("no tuning tables")
    for fn in os.listdir(autotune.TABLE_DIR):
        if fn.endswith(".json"):
            t = autotune.load(os.path.join(autotune.TABLE_DIR, fn))
            assert fn == os.path.basename(autotune.table_path(t["gpu"], t["sm_count"]))
            for k, vals in autotune.SPACE.items():
                assert t["tuning"][k] in vals
