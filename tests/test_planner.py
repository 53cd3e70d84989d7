"""Scheduling policy of the request server (host only, no GPU): FIFO
admission into contiguous runs of table-pool slots, launches of at most
max_batch points drawn oldest-first, slot release on completion."""
import ctypes as C

import numpy as np
import pytest

from y3_cluster_cpp_b200 import _capi as A

BUDGET = 6  # Y3B_ERR_BUDGET


class Planner:
    def __init__(self, pool, max_batch):
        self.L = A.lib()
        h = C.c_void_p()
        A.check(self.L.y3b_planner_create(pool, max_batch, C.byref(h)))
        self.h = h

    def submit(self, rid, n):
        return self.L.y3b_planner_submit(self.h, rid, n)

    def admit(self):
        ids = (C.c_longlong * 256)()
        slots = (C.c_int * 256)()
        n = C.c_int()
        A.check(self.L.y3b_planner_admit(self.h, ids, slots, 256, C.byref(n)))
        return [(ids[i], slots[i]) for i in range(n.value)]

    def batch(self, cap=256):
        ids = (C.c_longlong * cap)()
        first, count, slot = (C.c_int * cap)(), (C.c_int * cap)(), (C.c_int * cap)()
        nc, npt = C.c_int(), C.c_int()
        A.check(self.L.y3b_planner_next_batch(self.h, ids, first, count, slot, cap,
                                              C.byref(nc), C.byref(npt)))
        return [(ids[i], first[i], count[i], slot[i]) for i in range(nc.value)], npt.value

    def complete(self, rid, count):
        f = C.c_int()
        A.check(self.L.y3b_planner_complete(self.h, rid, count, C.byref(f)))
        return f.value

    def cancel(self, rid):
        f = C.c_int()
        A.check(self.L.y3b_planner_cancel(self.h, rid, C.byref(f)))
        return f.value

    def free(self):
        return self.L.y3b_planner_free_points(self.h)

    def close(self):
        self.L.y3b_planner_destroy(self.h)


def test_fifo_admission_and_split_batches():
    p = Planner(pool=100, max_batch=32)
    assert p.submit(1, 40) == 0 and p.submit(2, 50) == 0 and p.submit(3, 30) == 0
    assert p.admit() == [(1, 0), (2, 40)]     # 3 waits: 10 slots left
    assert p.free() == 10
    chunks, n = p.batch()
    assert n == 32 and chunks == [(1, 0, 32, 0)]
    chunks, n = p.batch()
    assert n == 32 and chunks == [(1, 32, 8, 32), (2, 0, 24, 40)]
    # request 1 done -> its 40 slots return; 3 is admitted at the front of the pool
    assert p.complete(1, 32) == 0
    assert p.complete(1, 8) == 1
    assert p.admit() == [(3, 0)]
    chunks, n = p.batch()
    assert chunks == [(2, 24, 26, 64), (3, 0, 6, 0)] and n == 32
    chunks, n = p.batch()
    assert chunks == [(3, 6, 24, 6)] and n == 24
    assert p.batch() == ([], 0)
    assert p.complete(2, 24) == 0 and p.complete(2, 26) == 1
    assert p.complete(3, 6) == 0 and p.complete(3, 24) == 1
    assert p.free() == 100
    p.close()


def test_head_of_line_is_not_overtaken():
    p = Planner(pool=64, max_batch=64)
    p.submit(1, 40)
    p.submit(2, 40)   # does not fit while 1 holds the pool
    p.submit(3, 8)    # would fit, but must not overtake 2
    assert p.admit() == [(1, 0)]
    p.batch()
    assert p.complete(1, 40) == 1
    assert p.admit() == [(2, 0), (3, 40)]
    p.close()


def test_rejections_and_fragmentation():
    p = Planner(pool=64, max_batch=16)
    assert p.submit(1, 65) == BUDGET
    assert p.submit(2, 0) == BUDGET
    assert p.submit(3, 16) == 0
    assert p.submit(3, 16) == BUDGET                          # duplicate id
    for rid in (4, 5, 6):
        assert p.submit(rid, 16) == 0
    assert [s for _, s in p.admit()] == [0, 16, 32, 48]
    for _ in range(4):
        p.batch()
    # free 3 and 5 (non-adjacent), then a 32-point request cannot fit until 4 returns
    assert p.complete(3, 16) == 1 and p.complete(5, 16) == 1
    assert p.free() == 32
    p.submit(7, 32)
    assert p.admit() == []
    assert p.complete(4, 16) == 1
    assert p.admit() == [(7, 0)]   # runs 0..47 merged, first fit at 0
    # completing more than was scheduled is an error
    f = C.c_int()
    assert p.L.y3b_planner_complete(p.h, 7, 1, C.byref(f)) == 1
    p.close()


def test_random_stream_conserves_slots():
    rng = np.random.default_rng(5)
    pool, mb = 300, 64
    p = Planner(pool, mb)
    sizes = {i: int(rng.integers(1, 120)) for i in range(1, 201)}
    outstanding = []           # chunks in flight
    returned = {i: 0 for i in sizes}
    nxt = 1
    done = set()
    for step in range(5000):
        if nxt <= 200 and rng.random() < 0.5:
            assert p.submit(nxt, sizes[nxt]) == 0
            nxt += 1
        for rid, s in p.admit():
            assert 0 <= s and s + sizes[rid] <= pool
        chunks, n = p.batch()
        assert n <= mb and n == sum(c[2] for c in chunks)
        outstanding += chunks
        if outstanding and rng.random() < 0.7:
            rid, first, cnt, slot = outstanding.pop(0)
            returned[rid] += cnt
            if p.complete(rid, cnt):
                assert returned[rid] == sizes[rid]
                done.add(rid)
        if len(done) == 200:
            break
    assert len(done) == 200
    assert p.free() == pool
    p.close()


def test_cancel_waiting_admitted_and_inflight_requests():
    """Cancellation (host-side injection, no device): a waiting request leaves
    the queue; an admitted one gets nothing more scheduled and frees its slots
    once its launched points are back; others are unaffected."""
    p = Planner(pool=64, max_batch=16)
    for rid, n in ((1, 40), (2, 40), (3, 8)):
        assert p.submit(rid, n) == 0
    assert p.admit() == [(1, 0)]
    assert p.cancel(2) == 1                  # waiting: gone at once
    assert p.admit() == [(3, 40)]            # 3 no longer blocked behind 2
    chunks, n = p.batch()
    assert chunks == [(1, 0, 16, 0)]
    assert p.cancel(1) == 0                  # 16 points still out
    chunks, n = p.batch()
    assert chunks == [(3, 0, 8, 40)] and n == 8   # nothing more of 1
    assert p.free() == 16
    assert p.complete(1, 16) == 1            # its slots return now
    assert p.free() == 56
    assert p.complete(3, 8) == 1 and p.free() == 64
    with pytest.raises(A.Y3BError):
        p.cancel(7)
    p.close()


def test_cancel_before_any_launch_frees_slots_immediately():
    p = Planner(pool=32, max_batch=8)
    assert p.submit(1, 20) == 0
    assert p.admit() == [(1, 0)]
    assert p.cancel(1) == 1 and p.free() == 32
    assert p.batch() == ([], 0)
    p.close()
