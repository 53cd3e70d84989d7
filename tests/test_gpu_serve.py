"""Request server on the GPU: each request's result is the same alone, in a
mix of requests of other sizes and grid densities, split across launches,
and as a direct engine evaluation of its points.  The per-point work and the
fixed-order reductions do not depend on what else is in a launch, so the
results are expected to be bitwise identical; the tests allow 1e-12
relative."""
import numpy as np
import pytest

from y3_cluster_cpp_b200 import _capi as A
from y3_cluster_cpp_b200 import engine as E
from y3_cluster_cpp_b200 import serve, synthetic

pytestmark = pytest.mark.gpu
TOL = 1e-12
GRID_OF = {1: 0, 2: 1}


def _engine(max_points=64, shear=None):
    grids = [synthetic.grid(1), synthetic.grid(2)]
    t0 = synthetic.fiducial().tables
    pz, pc = synthetic.plob_baseline()
    return E.Engine(grids, len(t0["hmf_m_h"]), len(t0["hmf_z"]), len(t0["dist_z"]), (pz, pc),
                    max_points=max_points, n_sci=len(t0["sci_z"]), shear=shear)


def _requests(eng, sizes, seed):
    pool = synthetic.walkers(16, seed=seed, densities=(1, 2))
    rng = np.random.default_rng(seed)
    reqs = []
    for n in sizes:
        pts = [pool[i] for i in rng.integers(0, len(pool), n)]
        reqs.append((eng.points_array(pts, grid_of=lambda p: GRID_OF[p.density]),
                     np.ascontiguousarray(eng.pack(pts))))
    return reqs


def _direct(eng, reqs, precision):
    out = []
    for pts, tab in reqs:
        n = len(pts)
        counts = np.empty((n, eng.n_bins))
        sh = np.empty((n, eng.n_bins, eng.n_R)) if eng.n_R else None
        E.check(E.lib().y3b_engine_eval(eng.handle, precision, n, pts, A.ptr(tab),
                                        A.ptr(counts), A.ptr(sh)))
        out.append((counts, sh))
    return out


def _close(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)) <= TOL


def test_alone_equals_mix(gpu):
    sh = synthetic.shear_opts(n_theta=16, n_s=32, n_R=4)
    eng = _engine(max_points=64, shear=sh)
    sizes = [5, 17, 3, 30, 9, 11, 22, 1, 14, 8]
    X = 5                                   # the request checked alone and in the mix
    reqs = _requests(eng, sizes, seed=21)
    ref = _direct(eng, reqs, E.MIXED)
    with serve.Server(eng, pool_points=256, max_batch=24) as srv:
        alone = srv.wait(srv.submit(*reqs[X]))
        tickets = [srv.submit(p, t) for p, t in reqs]          # back to back: they mix
        mixed = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert _close(alone["counts"], ref[X][0]) and _close(alone["shear"], ref[X][1])
    assert _close(mixed[X]["counts"], alone["counts"])
    assert _close(mixed[X]["shear"], alone["shear"])
    for r, (c, s) in zip(mixed, ref):
        assert _close(r["counts"], c) and _close(r["shear"], s)
        assert r["latency_s"] > 0
    assert st["points_done"] == sum(sizes) + sizes[X]
    assert st["requests_done"] == len(sizes) + 1
    assert st["max_launch_points"] <= 24
    assert st["launches"] >= (sum(sizes) + 23) // 24
    assert st["pool_free_points"] == 256 and st["waiting"] == 0
    eng.close()


def test_admission_under_a_small_pool_and_fp64(gpu):
    eng = _engine(max_points=32)
    sizes = [20, 20, 20, 5, 31, 2]
    reqs = _requests(eng, sizes, seed=22)
    ref_mx = _direct(eng, reqs, E.MIXED)
    ref_64 = _direct(eng, reqs[:2], E.FP64)
    with serve.Server(eng, pool_points=32, max_batch=16) as srv:
        tickets = [srv.submit(p, t) for p, t in reqs]    # more than the pool holds at once
        res = [srv.wait(t) for t in tickets]
        big = _requests(eng, [40], seed=23)[0]
        with pytest.raises(A.Y3BError) as e:
            srv.submit(*big)
        assert e.value.status == 6                       # BUDGET: never fits the pool
    for r, (c, _) in zip(res, ref_mx):
        assert _close(r["counts"], c)
    with serve.Server(eng, pool_points=64, max_batch=32, precision=E.FP64) as srv:
        res64 = [srv.wait(srv.submit(p, t)) for p, t in reqs[:2]]
    for r, (c, _) in zip(res64, ref_64):
        assert _close(r["counts"], c)
    eng.close()


def test_submit_checks_tables_and_points(gpu):
    eng = _engine(max_points=8)
    (pts, tab), = _requests(eng, [3], seed=24)
    bad = tab.copy()
    o = eng.offsets[3]
    nd = eng.shapes[2]
    bad[1, o:o + nd] *= 0.3                              # distances/z ends at 0.6 < z_t nodes
    with serve.Server(eng, pool_points=16, max_batch=8) as srv:
        with pytest.raises(A.Y3BError) as e:
            srv.submit(pts, bad)
        assert e.value.status == 2
        g0 = pts[0].grid
        pts[0].grid = 7
        with pytest.raises(A.Y3BError) as e:
            srv.submit(pts, tab)
        assert e.value.status == 1
        pts[0].grid = g0
        r = srv.wait(srv.submit(pts, tab))                # the server still works
        assert np.all(np.isfinite(r["counts"]))
    eng.close()


def test_cancel_and_memory_stats(gpu):
    """Cancellation through the server (host-side injection): a request
    cancelled while it waits behind a full pool completes with CANCELLED and
    writes nothing; the others finish unchanged; the stats report the HBM the
    server holds and every pool slot comes back.  (Whether the request is
    still waiting when cancel() arrives depends on timing: eight launches are
    queued ahead of it, and the scenario is repeated until a cancel lands.)"""
    eng = _engine(max_points=16)
    sizes = [16, 16, 12, 4]
    reqs = _requests(eng, sizes, seed=25)
    ref = _direct(eng, reqs, E.MIXED)
    cancelled = 0
    with serve.Server(eng, pool_points=32, max_batch=4, max_inflight=1) as srv:
        for _ in range(3):
            tickets = [srv.submit(p, t) for p, t in reqs]
            srv.cancel(tickets[2])
            try:
                r2 = srv.wait(tickets[2])
            except A.Y3BError as e:
                assert e.status == A.ERR_CANCELLED
                cancelled += 1
            else:                                # it had finished first: untouched
                assert _close(r2["counts"], ref[2][0])
            for i in (0, 1, 3):
                assert _close(srv.wait(tickets[i])["counts"], ref[i][0])
            if cancelled:
                break
        st = srv.stats()
        with pytest.raises(A.Y3BError) as e:
            srv.cancel(tickets[0])              # already collected
        assert e.value.status == A.ERR_INVALID
    assert cancelled == 1 and st["requests_cancelled"] == 1
    assert st["device_bytes"] >= eng.device_bytes() + 32 * eng.stride * 8
    assert st["pool_bytes_in_use"] == 0 and st["pool_free_points"] == 32
    eng.close()
