"""Host logic of the autotuner front end: cache keys and the JSON store."""
from agentray import autotune


def test_cache_key_separates_workloads():
    st = {"num_triangles": 1000, "num_instances": 3}
    a = autotune.cache_key("B200", st, "pt", 256, 256, 4)
    assert a != autotune.cache_key("B200", st, "bdpt", 256, 256, 4)
    assert a != autotune.cache_key("B200", st, "pt", 512, 512, 4)
    assert a != autotune.cache_key("B200", dict(st, num_triangles=1001), "pt", 256, 256, 4)


def test_cache_round_trip(tmp_path):
    p = str(tmp_path / "sub" / "tune.json")
    assert autotune.load_cache(p) == {}
    entry = {"tuning": {"path_capacity": 1 << 20, "traversal_blocks_per_sm": 6, "shade_block": 128,
                        "bdpt_batch_mib": 1536},
             "accel": {"max_leaf_size": 2, "sah_bins": 32, "build_threads": 0, "bvh_width": 8},
             "default_ms": 2.0, "best_ms": 1.5, "candidates": 12}
    autotune.store_cache(p, {"k": entry})
    assert autotune.load_cache(p) == {"k": entry}
