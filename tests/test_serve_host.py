"""The serving loop's admission rule (warpjq_b200/serve.py), without a GPU:
a free slot takes the longest prefix of the waiting requests that fits the
device-memory budget beside what is in flight, in arrival order."""

from warpjq_b200.serve import admit_count, footprint


def test_admits_the_prefix_that_fits():
    assert admit_count([10, 20, 30], 0, 100) == 3
    assert admit_count([10, 20, 30], 50, 100) == 2
    assert admit_count([10, 20, 30], 95, 100) == 0
    assert admit_count([], 0, 100) == 0


def test_no_overtaking_behind_a_request_that_waits():
    # the 60 does not fit beside 50 in flight; the 5 behind it waits too
    assert admit_count([60, 5], 50, 100) == 0
    assert admit_count([40, 60, 5], 0, 100) == 2


def test_footprints_grow_with_size_and_csv():
    assert footprint(0, "ndjson") == 1 << 20
    assert footprint(1000, "csv") > footprint(1000, "ndjson") > 1000
