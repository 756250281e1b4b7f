"""The dataflow closure's task order (the compiled se_closure_flow_task, no GPU needed):
every round's tasks appear exactly once, and every task comes after all the tasks it waits
for, so the persistent grid can never wait on a task nobody has taken."""
import ctypes

import pytest

from scalingelections_b200 import _lib


def order(R):
    L = _lib.lib()
    out = []
    v = [ctypes.c_int() for _ in range(4)]
    for t in range(R ** 3):
        _lib.check(L.se_closure_flow_task(t, R, *[ctypes.byref(x) for x in v]))
        out.append(tuple(x.value for x in v))
    return out


def prerequisites(task, R):
    kind, k, i, j = task
    pre = []
    panels = lambda kk: [(1, kk, kk, x) for x in range(R) if x != kk] + [(2, kk, x, kk) for x in range(R) if x != kk]
    rem = lambda kk: [(3, kk, a, b) for a in range(R) for b in range(R) if a != kk and b != kk]
    if kind == 0:
        if k > 0:
            pre.append((3, k - 1, k, k))  # the tile at version k
        if k >= 2:
            pre += panels(k - 2)  # readers of dT[k % 2]
        return pre
    pre.append((0, k, k, k))
    if k > 0:  # the task's own tile at version k: whoever wrote it in round k-1
        pre.append((0, k - 1, i, j) if i == j == k - 1 else (1, k - 1, i, j) if i == k - 1
                   else (2, k - 1, i, j) if j == k - 1 else (3, k - 1, i, j))
    if kind == 2 and k >= 2:
        pre += rem(k - 2)  # readers of AT[k % 2]
    if kind == 3:
        pre += [(1, k, k, j), (2, k, i, k)]
    if i == k - 1 and kind >= 2:  # overwrites a row-panel tile (or the pivot) of round k-1
        pre += panels(k - 1) + rem(k - 1)
    return pre


@pytest.mark.parametrize("R", list(range(2, 15)))
def test_flow_order_is_complete_and_topological(R):
    seq = order(R)
    expected = set()
    for k in range(R):
        expected |= {(0, k, k, k)} | {(1, k, k, j) for j in range(R) if j != k}
        expected |= {(2, k, i, k) for i in range(R) if i != k}
        expected |= {(3, k, i, j) for i in range(R) for j in range(R) if i != k and j != k}
    assert len(seq) == len(expected) and set(seq) == expected
    pos = {task: n for n, task in enumerate(seq)}
    for n, task in enumerate(seq):
        for pre in prerequisites(task, R):
            assert pos[pre] < n, (task, pre)
