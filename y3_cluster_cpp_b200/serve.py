"""Serving form: likelihood-evaluation requests from a running sampler,
continuously batched on one GPU (the ``y3b_server_*`` C ABI).

A request is a group of parameter points, each with its own packed table
block (:meth:`Engine.pack` layout).  The native server copies a request's
tables once into a device-resident pool when the pool has room (arrival
order, bounded by the HBM budget), builds every launch from the points of all
admitted requests (oldest first, large requests split across launches) and
keeps up to ``max_inflight`` launches queued on the device, so requests that
arrive while the GPU is busy join the next launch.  Each request's latency is
measured by the server from submission to the moment its last point is back
on the host.

The reference evaluates one point per CosmoSIS ``execute`` call and has no
request server; :func:`run_stream` drives the server with the Poisson request
stream of the serving workload and reports throughput and p50/p99 latency.
"""
from __future__ import annotations

import ctypes as C
import threading
import time

import numpy as np

from . import _capi as A
from ._capi import check, lib
from .engine import MIXED


class Server:
    """Continuous-batching server over an :class:`Engine` (which it owns
    while it exists: do not call ``engine.eval`` meanwhile)."""

    def __init__(self, engine, pool_points=0, max_batch=0, precision=MIXED, with_shear=None,
                 hbm_budget=0, max_inflight=2):
        self.engine = engine
        cfg = A.ServerConfig()
        cfg.pool_points = pool_points
        cfg.hbm_budget = hbm_budget
        cfg.max_batch = max_batch
        cfg.precision = precision
        self.with_shear = bool(engine.n_R) if with_shear is None else bool(with_shear)
        cfg.with_shear = 1 if self.with_shear else 0
        cfg.max_inflight = max_inflight
        h = C.c_void_p()
        check(lib().y3b_server_create(engine.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        self._live = {}
        self._lock = threading.Lock()

    def submit(self, points, tables):
        """Queue a request; returns its ticket at once.  points: ctypes array
        of ``Point`` (see :meth:`Engine.points_array`); tables: float64
        C-contiguous [n, stride] (pinned memory uploads fastest)."""
        n = len(points)
        tables = np.asarray(tables)
        if tables.dtype != np.float64 or not tables.flags["C_CONTIGUOUS"] or \
                tables.shape != (n, self.engine.stride):
            raise ValueError(f"tables must be float64 C-contiguous [{n}, {self.engine.stride}]")
        counts = np.empty((n, self.engine.n_bins))
        shear = np.empty((n, self.engine.n_bins, self.engine.n_R)) if self.with_shear else None
        t = C.c_longlong()
        check(lib().y3b_server_submit(
            self._h, n, C.cast(points, C.c_void_p), C.c_void_p(tables.ctypes.data),
            C.c_void_p(counts.ctypes.data),
            C.c_void_p(shear.ctypes.data) if shear is not None else None, C.byref(t)))
        with self._lock:
            # the native side reads these buffers until the request completes
            self._live[t.value] = (points, tables, counts, shear)
        return t.value

    def wait(self, ticket, timeout=None):
        """Blocks until the request is complete; returns {"counts", "shear"?,
        "latency_s"}.  Raises Y3BError on failure (or TIMEOUT)."""
        lat = C.c_double()
        rc = lib().y3b_server_wait(self._h, ticket, -1.0 if timeout is None else float(timeout),
                                   C.byref(lat))
        if rc == 5:  # still running: keep the buffers alive
            check(rc)
        with self._lock:
            _, _, counts, shear = self._live.pop(ticket, (None, None, None, None))
        check(rc)
        out = {"counts": counts, "latency_s": lat.value}
        if shear is not None:
            out["shear"] = shear
        return out

    def cancel(self, ticket):
        """Stops launching the request's points; its wait() then raises
        Y3BError with status CANCELLED once the points already on the device
        are back (their results are not written)."""
        check(lib().y3b_server_cancel(self._h, ticket))

    def stats(self):
        s = A.ServerStats()
        check(lib().y3b_server_stats_read(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in A.ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().y3b_server_destroy(self._h)
            self._h = None
            self._live.clear()

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def request_sizes(n, seed=2, max_points=1024):
    """Request sizes round(exp(U[0, ln max_points])), i.e. log-uniform 1..max."""
    rng = np.random.default_rng(seed)
    return np.maximum(1, np.rint(np.exp(rng.uniform(0.0, np.log(max_points), n)))).astype(int)


def poisson_arrivals(n, mean_gap_s=0.002, seed=2):
    """Arrival offsets [s] of a Poisson stream (exponential gaps)."""
    rng = np.random.default_rng(seed + 1)
    return np.cumsum(rng.exponential(mean_gap_s, n))


def run_stream(server, requests, arrivals):
    """Submits requests[i] = (points, tables) at arrivals[i] seconds after
    the start (a submitting thread) and collects every result.  Returns
    {"results", "latency_s", "wall_s", "points"}."""
    n = len(requests)
    tickets = [None] * n
    errors = []

    def submitter():
        t0 = time.perf_counter()
        for i, (pts, tab) in enumerate(requests):
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            try:
                tickets[i] = server.submit(pts, tab)
            except Exception as e:  # noqa: BLE001 -- reported after the join
                errors.append((i, e))
                tickets[i] = -1

    start = time.perf_counter()
    th = threading.Thread(target=submitter)
    th.start()
    results = [None] * n
    lat = np.zeros(n)
    for i in range(n):
        while tickets[i] is None:
            time.sleep(1e-4)
        if tickets[i] < 0:
            continue
        r = server.wait(tickets[i])
        results[i] = r
        lat[i] = r["latency_s"]
    th.join()
    wall = time.perf_counter() - start
    if errors:
        raise RuntimeError(f"{len(errors)} submissions failed; first: {errors[0]}")
    return {"results": results, "latency_s": lat, "wall_s": wall,
            "points": int(sum(len(p) for p, _ in requests))}


def run_closed_loop(server, requests, outstanding=16):
    """Saturating stream: keeps `outstanding` requests submitted at all times,
    submitting the next as soon as the oldest has completed (requests complete
    in order: admission and batching are oldest first).  Measures what the
    server sustains when requests never wait for an arrival.  Returns
    {"results", "latency_s", "wall_s", "points"}."""
    n = len(requests)
    tickets = {}
    results = [None] * n
    lat = np.zeros(n)
    start = time.perf_counter()
    for i in range(min(outstanding, n)):
        tickets[i] = server.submit(*requests[i])
    for i in range(n):
        r = server.wait(tickets.pop(i))
        results[i] = r
        lat[i] = r["latency_s"]
        j = i + outstanding
        if j < n:
            tickets[j] = server.submit(*requests[j])
    wall = time.perf_counter() - start
    return {"results": results, "latency_s": lat, "wall_s": wall,
            "points": int(sum(len(p) for p, _ in requests))}


def percentiles_ms(lat_s):
    lat = np.asarray(lat_s) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()), "mean_ms": float(lat.mean())}
