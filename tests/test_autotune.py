"""Autotuner logic on the CPU: choice per bucket, table round trip, bucket mapping."""
import json

from b200dft import autotune


def test_pick_fastest_per_bucket_ties_to_fewer_tiles():
    times = {0: {1: 2.0, 2: 1.5, 4: 1.5}, 3: {8: 0.9, 16: 1.2}, 4: {}}
    assert autotune.pick(times) == {0: 2, 3: 8}


def test_bucket_of_matches_kernel_grouping():
    assert [autotune.bucket_of(n) for n in (1, 16, 17, 32, 48, 49, 64, 65, 80)] == [0, 0, 1, 1, 2, 3, 3, 4, 4]
    a = autotune.tiles_array({1: 4, 3: 16})
    assert list(a) == [0, 4, 0, 16, 0] and a.dtype.name == "int32"


def test_table_round_trip(tmp_path):
    p = str(tmp_path / "tuned.json")
    autotune.save({2: 8}, {2: {4: 1.25, 8: 1.0}}, "NVIDIA B200", path=p, workload="w")
    d = json.load(open(p))
    assert d["NVIDIA B200"]["xc_tiles"] == {"2": 8}
    assert autotune.load(p)["NVIDIA B200"]["xc_ms"]["2"]["8"] == 1.0
