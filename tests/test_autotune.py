"""The autotuner's host logic (CPU): shape classes, candidates, a
deterministic choice from given timings, and the cache file's round trip."""
from __future__ import annotations

import json

from pageflow_b200 import autotune as T


def test_shape_class_rounds_sizes_up_to_powers_of_two():
    a = T.shape_class("B200", 150_000_000, 600_000_000, 1_500_000)
    assert a == "B200|join_aggregate|b28|p30|g21"
    assert T.shape_class("B200", 1 << 27, 1, 1) == "B200|join_aggregate|b27|p0|g0"
    assert T.shape_class("B200", (1 << 27) + 1, 1, 1).split("|")[2] == "b28"


def test_fanout_candidates_are_the_seed_and_its_neighbours():
    assert T.b_candidates(256) == [256, 128, 512]
    assert T.b_candidates(1) == [1, 2]
    assert T.b_candidates(4096) == [4096, 2048]


def _timer(table):
    calls = []

    def time_of(c):
        calls.append(c.label())
        return table.get(c.label(), 100.0)
    return time_of, calls


def test_search_is_coordinate_wise_and_deterministic():
    times = {"B=256,table=0,sub_rows=1365": 20.0, "B=512,table=0,sub_rows=1365": 18.0,
             "B=128,table=0,sub_rows=1365": 25.0, "B=512,table=1,sub_rows=1365": 17.0,
             "B=512,table=1,sub_rows=682": 17.0}
    f, calls = _timer(times)
    r = T.search(256, f)
    # B first, then the table at the best B, then sub_rows; a tie keeps the
    # earlier candidate
    assert r.choice == T.Choice(512, 1, 1365)
    assert calls == ["B=256,table=0,sub_rows=1365", "B=128,table=0,sub_rows=1365",
                     "B=512,table=0,sub_rows=1365", "B=512,table=1,sub_rows=1365",
                     "B=512,table=1,sub_rows=682", "B=512,table=1,sub_rows=1365,counted=1"]
    f2, _ = _timer(times)
    assert T.search(256, f2).choice == r.choice
    assert r.times_ms == {k: times.get(k, 100.0) for k in calls}


def test_cache_round_trip_skips_the_search(tmp_path):
    path = tmp_path / "tune.json"
    f, calls = _timer({"B=128,table=0,sub_rows=1365": 1.0})
    first = T.tune("k", 256, f, path)
    assert not first.cached and first.choice.B == 128
    n = len(calls)
    again = T.tune("k", 256, f, path)
    assert again.cached and again.choice == first.choice and len(calls) == n
    data = json.loads(path.read_text())
    assert data["k"]["choice"] == {"B": 128, "table": 0, "sub_rows": 1365, "counted": 0}
    # another shape class searches on its own and keeps the first entry
    T.tune("k2", 64, _timer({})[0], path)
    assert set(json.loads(path.read_text())) == {"k", "k2"}


def test_counting_first_wins_where_the_regions_overflow():
    """A skewed shape class, where scattering into regions overflows and is
    run again, picks the counted passes; a cache entry without the counted
    field reads as regions."""
    times = {"B=256,table=0,sub_rows=1365": 30.0, "B=256,table=0,sub_rows=1365,counted=1": 21.0}
    f, calls = _timer(times)
    r = T.search(256, f)
    assert r.choice == T.Choice(256, 0, 1365, 1)
    assert calls[-1] == "B=256,table=0,sub_rows=1365,counted=1"


def test_old_cache_entries_read_as_regions(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"k": {"choice": {"B": 64, "table": 1, "sub_rows": 682}}}))
    hit = T.lookup("k", path)
    assert hit.cached and hit.choice == T.Choice(64, 1, 682, 0)
