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


def _host_server(priority, max_slots=100, free_bytes=1 << 40, fits=lambda t: True):
    """A Server with only its admission state (no engine, no GPU): try_submit records the
    order and admits what `fits` accepts."""
    from scalingelections_b200 import serve

    srv = object.__new__(serve.Server)
    srv.priority, srv.by_slot, srv.max_slots = priority, {}, max_slots

    class _Arena:
        pass

    srv.arena = _Arena()
    srv.arena.free_bytes = free_bytes
    srv.order = []

    def try_submit(t, ballots):
        if not fits(t):
            return False
        srv.order.append(t.rid)
        t.slot = len(srv.by_slot)
        srv.by_slot[t.slot] = t
        return True

    srv.try_submit = try_submit
    return srv


def _tickets(Cs, arrivals=None):
    from scalingelections_b200.serve import Ticket

    arrivals = arrivals or [0.0] * len(Cs)
    return [Ticket(rid=i, V=100, C=C, arrival=a) for i, (C, a) in enumerate(zip(Cs, arrivals))]


def test_admission_priority_orders_a_burst():
    for priority, expect in (("arrival", [0, 1, 2, 3]), ("largest", [3, 1, 2, 0])):
        srv = _host_server(priority)
        pending = _tickets([10, 300, 50, 2000])
        assert srv.admit(pending, lambda t: None, now=0.0) == 4
        assert pending == [] and srv.order == expect, priority


def test_admission_priority_keeps_what_does_not_fit_and_no_starvation():
    # Largest first, but C = 2000 does not fit: the others pass it while it is young ...
    srv = _host_server("largest", fits=lambda t: t.C != 2000)
    pending = _tickets([10, 2000, 300])
    assert srv.admit(pending, lambda t: None, now=0.0) == 2
    assert srv.order == [2, 0] and [t.rid for t in pending] == [1]
    # ... and once the oldest has waited past the bypass limit, nothing passes it.
    srv = _host_server("largest", fits=lambda t: t.C != 2000)
    pending = _tickets([2000, 10, 300])
    assert srv.admit(pending, lambda t: None, now=1.0, max_bypass_s=0.25) == 0
    assert [t.rid for t in pending] == [0, 1, 2]


def test_cancel_drops_a_waiting_request_before_admission():
    srv = _host_server("arrival")
    ts = _tickets([64, 128, 256])
    assert srv.cancel(ts[1]) is True  # still waiting: nothing of it will run
    pending = list(ts)
    srv.admit(pending, lambda t: None, now=0.0)
    assert srv.order == [0, 2] and pending == []
    assert srv.cancel(ts[0]) is False  # admitted: in flight


def test_cancelled_request_in_flight_is_not_returned_but_its_memory_is():
    """poll() frees a cancelled request's memory when the engine finishes it, and does not
    hand it out. The engine is faked: it reports slot 0 tallied, then done."""
    import ctypes

    from scalingelections_b200 import serve

    srv = object.__new__(serve.Server)
    srv.arena = Arena(1 << 20)
    srv.by_slot = {}
    srv.max_slots = 4
    srv._poll_slots = (ctypes.c_int * 4)()
    srv._poll_status = (ctypes.c_uint32 * 4)()
    srv.engine = None

    class FakeLib:
        def se_engine_poll_tallied(self, engine, slots, cap, n):
            slots[0] = 0
            ctypes.cast(n, ctypes.POINTER(ctypes.c_int))[0] = 1
            return 0

        def se_engine_poll(self, engine, slots, status, cap, n):
            slots[0], status[0] = 0, 0
            ctypes.cast(n, ctypes.POINTER(ctypes.c_int))[0] = 1
            return 0

    srv.L = FakeLib()
    t = _tickets([64])[0]
    t.offset, t.nbytes = srv.arena.alloc(4096), 4096
    t.pos_offset, t.pos_nbytes = srv.arena.alloc(8192), 8192
    t.ids_offset, t.ids_nbytes = srv.arena.alloc(1024), 1024
    t.slot = 0
    srv.by_slot[0] = t
    assert srv.cancel(t) is False  # in flight
    assert srv.poll() == []
    assert srv.arena.used == 0 and srv.by_slot == {}
    assert srv.cancel(t) is False  # already finished
