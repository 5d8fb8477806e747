"""Host side of the launch-shape autotuner: buckets, the cache file, the
candidate stages (no GPU)."""
import json
import os

from qlatanneal_b200 import autotune


def test_bucket_rounds_up_to_powers_of_two():
    assert autotune.bucket("dense", 512, 32, 256) == "dense|n512|P32|rings256"
    assert autotune.bucket("sparse", 513, 16, 1000) == "sparse|n1024|P16|rings1024"
    assert autotune.bucket("hubo", 1, 1, 1) == "hubo|n1|P1|rings1"


def test_cache_lookup(tmp_path):
    path = os.path.join(tmp_path, "t.json")
    key = autotune.bucket("dense", 512, 32, 256)
    with open(path, "w") as f:
        json.dump({key: {"tuning": {"warps_per_ring": 8, "rotate": 1, "rot_steps": 50, "rot_group": 2},
                         "ms": 1.0}}, f)
    autotune.use_cache(path)
    try:
        assert autotune.lookup("dense", 500, 32, 200) == {"warps_per_ring": 8, "rotate": 1, "rot_steps": 50,
                                                          "rot_group": 2}
        assert autotune.lookup("dense", 512, 16, 256) is None
    finally:
        autotune.use_cache(None)
    assert autotune.lookup("dense", 512, 32, 256) is None


def test_candidate_stages():
    base = dict(autotune.AUTO)
    warps = autotune._candidates_stage("warps", base, "dense", 32, 256, 148)
    assert sorted(c["warps_per_ring"] for c in warps) == [8, 16, 32]
    assert [c["field_form"] for c in autotune._candidates_stage("form", base, "dense", 32, 256, 148)] == [-1, 0, 1, 2]
    assert autotune._candidates_stage("form", base, "sparse", 16, 256, 148) == []
    rot = autotune._candidates_stage("rotation", base, "dense", 32, 256, 148)
    assert rot[0]["rotate"] == 0 and len(rot) == 10
    assert len(autotune._candidates_stage("rotation", base, "dense", 32, 100, 148)) == 1


def test_chi_buckets_and_forms():
    """SQA-Chi has buckets of its own; its dense models get the ring-state forms."""
    assert autotune.bucket("dense-chi", 1024, 64, 512) == "dense-chi|n1024|P64|rings512"
    base = dict(autotune.AUTO)
    assert len(autotune._candidates_stage("form", base, "dense-chi", 64, 512, 148)) == 4
    assert autotune._candidates_stage("form", base, "sparse-chi", 64, 512, 148) == []


def test_apply_is_suspended_while_tuning(tmp_path):
    """A run that a tuning times keeps the candidate shape even when a cache
    with an entry for its bucket is active."""
    path = os.path.join(tmp_path, "t.json")
    key = autotune.bucket("dense", 64, 8, 16)
    with open(path, "w") as f:
        json.dump({key: {"tuning": {"warps_per_ring": 2}, "ms": 1.0}}, f)
    seen = []

    class FakeEngine:
        pass

    orig = autotune.set_tuning
    autotune.set_tuning = lambda eng, t: seen.append(t)
    autotune.use_cache(path)
    try:
        autotune.apply(FakeEngine(), "dense", 64, 8, 16)
        assert seen == [{"warps_per_ring": 2}]
        autotune._suspend.on = True
        autotune.apply(FakeEngine(), "dense", 64, 8, 16)
        assert seen == [{"warps_per_ring": 2}]
    finally:
        autotune._suspend.on = False
        autotune.set_tuning = orig
        autotune.use_cache(None)
