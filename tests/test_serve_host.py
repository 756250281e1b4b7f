"""Host-side admission logic of the server: the HBM arena allocator (no GPU needed)."""
import random

from scalingelections_b200.serve import ALIGN, Arena


def test_arena_first_fit_and_coalescing():
    a = Arena(10 * ALIGN)
    x = a.alloc(1)
    y = a.alloc(3 * ALIGN)
    z = a.alloc(ALIGN + 1)
    assert (x, y, z) == (0, ALIGN, 4 * ALIGN)
    assert a.alloc(5 * ALIGN) is None  # only 4 blocks left
    a.free(y, 3 * ALIGN)
    assert a.alloc(3 * ALIGN) == ALIGN  # reuses the hole
    a.free(x, 1)
    a.free(ALIGN, 3 * ALIGN)
    a.free(z, ALIGN + 1)
    assert a.used == 0 and a.alloc(10 * ALIGN) == 0


def test_arena_random_workload_never_overlaps():
    rng = random.Random(0)
    a = Arena(1 << 20)
    live = {}
    for step in range(3000):
        if live and (rng.random() < 0.45 or len(live) > 60):
            off = rng.choice(list(live))
            a.free(off, live.pop(off))
        else:
            n = rng.randint(1, 40000)
            off = a.alloc(n)
            if off is not None:
                assert off % ALIGN == 0
                end = off + n
                for o, m in live.items():
                    assert end <= o or o + m <= off, "overlap"
                assert end <= a.capacity
                live[off] = n
    for off, n in list(live.items()):
        a.free(off, n)
    assert a.used == 0 and a.alloc(a.capacity) == 0
