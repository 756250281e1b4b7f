"""Host logic of the batch's lane choice and the autotuner's table lookup (no GPU): the
16-bit window of lanes_for_voters at its boundaries, the size buckets, and how a tuning table
overrides the defaults."""
from scalingelections_b200 import LANES_U16, LANES_U32
from scalingelections_b200.autotune import BUCKETS, bucket_of, choose
from scalingelections_b200.batch import lanes_for_voters


def test_sixteen_bit_window_holds_every_kept_count():
    """A kept count of a complete tally lies in (V/2, V]. Stored minus the offset it must be a
    nonzero 16-bit value (0 means no edge)."""
    for V in (1, 2, 3, 65534, 65535, 65536, 65537, 100001, 131069, 131070):
        lanes, off = lanes_for_voters(V)
        assert lanes == LANES_U16, V
        lo, hi = V // 2 + 1, V  # the smallest and largest kept counts
        assert 1 <= lo - off and hi - off <= 0xFFFF, (V, off)
        if V < 65536:
            assert off == 0
    for V in (131071, 131072, 10**6):
        assert lanes_for_voters(V) == (LANES_U32, 0)


def test_buckets_cover_sizes_in_order():
    assert BUCKETS[0][0] == 1
    for (lo0, hi0), (lo1, hi1) in zip(BUCKETS, BUCKETS[1:]):
        assert lo1 == hi0 + 1 and lo0 <= hi0
    for b, (lo, hi) in enumerate(BUCKETS):
        assert bucket_of(lo) == b and bucket_of(hi) == b
    assert bucket_of(BUCKETS[-1][1] + 1) == len(BUCKETS) - 1  # larger elections share the last bucket


def test_choose_without_a_table():
    lanes, order, ctas = choose(None, [8, 300, 2048], [50, 70000, 200000])
    assert lanes == [(LANES_U16, 0), (LANES_U16, 35000), (LANES_U32, 0)]
    assert (order, ctas) == (0, 0)


def test_choose_with_a_table():
    table = {"buckets": {str(bucket_of(300)): {"lanes": 32}, str(bucket_of(8)): {"lanes": 16}},
             "order": 1, "ctas_per_sm": 2}
    lanes, order, ctas = choose(table, [8, 300, 1000], [50, 70000, 70000])
    assert lanes == [(LANES_U16, 0), (LANES_U32, 0), (LANES_U16, 35000)]
    assert (order, ctas) == (1, 2)


def test_choose_micro_tiles():
    from scalingelections_b200.autotune import choose_micro_tiles

    table = {"buckets": {str(bucket_of(300)): {"lanes": 16, "micro_tile": 4},
                         str(bucket_of(1000)): {"lanes": 16, "micro_tile": 8}}}
    lanes = [(LANES_U16, 0), (LANES_U16, 0), (LANES_U32, 0), (LANES_U16, 35000)]
    assert choose_micro_tiles(table, [300, 1000, 300, 300], lanes) == [4, 8, 8, 4]
    assert choose_micro_tiles(None, [300], [(LANES_U16, 0)]) == [8]
    assert choose_micro_tiles({"buckets": {str(bucket_of(8)): {"lanes": 16}}}, [8], [LANES_U16]) == [8]
