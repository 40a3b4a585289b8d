"""Host logic of the batch autotuner (cholesky_gpu_b200/tune.py): size
classes, cache keys, the choice among measured candidates and the table
round trip.  The measurements themselves run on the GPU
(tests/test_gpu_batch.py)."""
import pytest

from cholesky_gpu_b200 import tune


def test_size_classes_cover_every_order_once():
    bounds = tune.SIZE_CLASSES
    assert bounds[0][0] == 1
    for (lo0, hi0), (lo1, hi1) in zip(bounds, bounds[1:]):
        assert lo1 == hi0 + 1
    assert tune.size_class(64) == 0 and tune.size_class(256) == 0
    assert tune.size_class(257) == 1 and tune.size_class(2048) == 3
    with pytest.raises(ValueError):
        tune.size_class(0)


def test_group_by_class_keeps_caller_order():
    ns = [2000, 70, 600, 300, 90, 1500]
    g = tune.group_by_class(ns)
    assert g == {3: [0, 5], 0: [1, 4], 2: [2], 1: [3]}
    assert tune.table_key(ns, 4) == "classes=0,1,2,3;rhs=4"


def test_pick_ignores_failed_and_unconverged_candidates():
    res = {"a": {"ms": 5.0, "converged": False}, "b": {"ms": 7.0, "converged": True},
           "c": {"ms": None, "converged": False, "status": 2}, "d": {"ms": 6.5, "converged": True}}
    assert tune.pick(res) == ("d", 6.5)
    assert tune.pick({"a": {"ms": 1.0, "converged": False}}) is None


def test_plan_from_table_and_round_trip(tmp_path):
    ns = [100, 400, 1800]
    assert tune.plan_for(ns, 4, {}) == {"mode": "whole", "config": tune.DEFAULT}
    key = tune.table_key(ns, 4)
    split = {key: {"mode": "split", "classes": {"0": {"block_size": 64, "precision": "fp16x2"},
                                                "1": {"block_size": 128, "precision": "fp16x2"},
                                                "3": {"block_size": 256, "precision": "fp16x2"}}}}
    p = tune.save_table(split, tmp_path / "t.json")
    plan = tune.plan_for(ns, 4, tune.load_table(p))
    assert plan["mode"] == "split" and plan["classes"][0]["block_size"] == 64
    whole = {key: {"mode": "whole", "config": {"block_size": 128, "precision": "fp16"}}}
    assert tune.plan_for(ns, 4, whole)["config"]["precision"] == "fp16"
    # another rhs count is another shape
    assert tune.plan_for(ns, 2, whole) == {"mode": "whole", "config": tune.DEFAULT}


def test_shipped_table_is_valid_json_with_known_configs():
    table = tune.load_table()
    names = {tune.config_name(c) for c in tune.CANDIDATES}
    for key, ent in table.items():
        assert key.startswith("classes=") and ent["mode"] in ("whole", "split")
        cfgs = [ent["config"]] if ent["mode"] == "whole" else list(ent["classes"].values())
        for c in cfgs:
            assert tune.config_name(c) in names
