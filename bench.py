#!/usr/bin/env python
"""Benchmark: parameter-point evaluations per second of the cluster
number-count integral N(lambda_obs bin, z_obs bin) at the 4x node density
(256 lnM x 128 z_t x 256 lambda_t x 256 lambda_obs/bin x 64 z_obs/bin),
mixed precision (FP32 integrands, split-BF16 tcgen05 contraction, FP64 final
sums), on batches of walkers drawn from the batched-config prior, each point
with its own HMF / dV/dz / Sigma_crit tables (seeded synthetic data).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on rank 0.  `value` is device-timed with inputs resident in
HBM (L2 flushed between steps); `e2e` goes through the C ABI with pinned host
buffers, host<->device copies inside the timed region.  Under torchrun every
rank evaluates its own batch (weak scaling, no data-path collective) and the
time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "param-point evals/sec at <=1e-4 rel err vs FP64 (counts, 4x nodes)"
UNIT = "points/s"
WORKLOAD = ("number counts N(lambda_obs, z_obs), 12 bins, 4x nodes 256 lnM x 128 z_t x 256 "
            "lam_t x 256 lam_o/bin x 64 z_o/bin, walkers from the batched-config prior")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=2048, help="points per step per GPU")
    ap.add_argument("--unique", type=int, default=256, help="distinct walker tables per batch")
    ap.add_argument("--density", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=8,
                    help="points in the CPU baseline sample (reference chain)")
    ap.add_argument("--cpu-port-sample", type=int, default=2,
                    help="points of the FP64 direct-quadrature port timed beside it")
    ap.add_argument("--no-extra-workloads", dest="extra_workloads", action="store_false",
                    help="skip the batched-uneven and DeltaSigma measurements")
    ap.add_argument("--serve-requests", type=int, default=256,
                    help="requests in the serving stream (0: skip the serving measurement)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("bf16_tflops", 1590.0), d.get("hbm_gbs", 6650.0), "measured"
    return 1590.0, 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML queried every 2 ms from a background thread (read-only), or
    nvidia-smi at 100 ms when NVML is not importable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.thread = None
        self.proc = None
        self.path = None
        self.running = False

    def start(self):
        try:
            import threading

            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByUUID(self.gpu) if isinstance(self.gpu, str) \
                else pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            masks = [(n, getattr(pynvml, a, 0)) for n, a in self.REASONS]

            def poll():
                while self.running:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append((sm, [n for n, m in masks if m and (r & m)]))
                    time.sleep(0.002)

            self.running = True
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:  # noqa: BLE001 -- fall back to nvidia-smi
            self.thread = None
        fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={fields}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.running = False
            self.thread.join(timeout=2)
            rows = self.rows
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["no samples"],
                        "samples": 0, "source": "nvml"}
            sm = [r[0] for r in rows]
            loaded = [x for x in sm if x > 0.5 * self.smax] or sm
            reasons = sorted({n for _, rs in rows for n in rs})
            return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": self.smax,
                    "reasons": reasons, "samples": len(rows), "source": "nvml, 2 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi, 100 ms"}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# The reference's production resolution for this path: sel_function.py on the
# des_y3.ini grid (192 lnM x 64 z x 32 lam_t nodes per cell), then
# NumCountsSelGL with its defaults (96 lnM x 64 z GL nodes).
REF_SEL_GRID = dict(n_lnm=192, n_z=64, n_q=32)


def _ref_chain_setup():
    import numpy as np

    import oracle
    from oracle import ref as R
    from y3_cluster_cpp_b200 import synthetic
    g = synthetic.grid(1)
    le, ze = g["lam_edges"], g["zob_edges"]
    cfg = dict(lam_min=np.tile(le[:-1], 3), lam_max=np.tile(le[1:], 3),
               zob_min=np.repeat(ze[:-1], 4), zob_max=np.repeat(ze[1:], 4),
               sigma_z=np.full(12, 0.0145), zt_low=g["zt_lo"], zt_high=g["zt_hi"],
               lnm_low=g["lnm_lo"], lnm_high=g["lnm_hi"], **REF_SEL_GRID)
    selgl = dict(zt_low=g["zt_lo"], zt_high=g["zt_hi"], lnm_low=g["lnm_lo"],
                 lnm_high=g["lnm_hi"])
    oracle.lib()
    return cfg, selgl, R.available()


def _ref_chain_point(p, cfg, selgl, have_ref):
    """One parameter point through the reference chain: the S_stack
    tabulation of sel_function.py (its C restatement, pinned to the
    reference's Python at 1e-13; Python cannot run on the GPU host) and
    NumCountsSelGL, the reference's own C++ compiled from its sources (the
    oracle's bit-identical restatement where that build is absent)."""
    import oracle
    from oracle import ref as R
    from y3_cluster_cpp_b200 import synthetic
    pz, pc = synthetic.plob_baseline()
    mor = [p.A, p.B, p.C, p.sigma, p.Mpiv, 1.0, 1000.0]
    sel = oracle.sel_function(cfg, oracle.MOR_LOGNORMAL, mor, pz, pc)
    if have_ref:
        cosmo = dict(omega_m=p.om, omega_nu=0.0, omega_lambda=1.0 - p.om, omega_k=0.0,
                     h0=p.h0, hmf_s=0.0, hmf_q=1.0)
        return R.numcounts(selgl, cosmo, p.tables, sel)
    return oracle.selgl_weights(96, 64, selgl["zt_low"], selgl["zt_high"], selgl["lnm_low"],
                                selgl["lnm_high"], oracle.cosmo(p.om, p.h0), p.tables, sel)[1]


def _ref_worker(seed):
    from y3_cluster_cpp_b200 import synthetic
    cfg, selgl, have_ref = _ref_chain_setup()
    p = synthetic.walkers(1, seed=seed, densities=(1,), with_sci=False)[0]
    _ref_chain_point(p, cfg, selgl, have_ref)
    return 1


def _ref_kind(have_ref):
    return "reference" if have_ref else "port"


def _ref_sample(have_ref):
    what = ("NumCountsSelGL: the reference's C++ compiled from its sources"
            if have_ref else "NumCountsSelGL: the oracle's restatement")
    return (f"reference chain per point: sel_function S_stack at "
            f"{REF_SEL_GRID['n_lnm']} lnM x {REF_SEL_GRID['n_z']} z x {REF_SEL_GRID['n_q']} "
            f"lam_t (C restatement of sel_function.py, pinned to it at 1e-13), then {what} "
            f"(96 lnM x 64 z); walkers' own tables")


def cpu_baseline(n_points, density, n_port):
    """The reference chain on the host, one thread, on a bounded sample of
    walkers; beside it the FP64 direct quadrature (the oracle port) at the
    bench's node density."""
    from y3_cluster_cpp_b200 import synthetic
    cfg, selgl, have_ref = _ref_chain_setup()
    pts = synthetic.walkers(n_points, seed=11, densities=(1,), with_sci=False)
    _ref_chain_point(pts[0], cfg, selgl, have_ref)
    t0 = time.perf_counter()
    for p in pts:
        _ref_chain_point(p, cfg, selgl, have_ref)
    dt = time.perf_counter() - t0
    out = {"value": n_points / dt, "unit": UNIT, "cores": 1, "kind": _ref_kind(have_ref),
           "sample": f"{n_points} points, {_ref_sample(have_ref)}; 1 thread, {dt:.2f} s",
           "ms_per_point": 1e3 * dt / n_points, "cpu_model": cpu_model(),
           "nproc": os.cpu_count()}
    if n_port > 0:
        import oracle
        g = synthetic.grid(density)
        pz, pc = synthetic.plob_baseline()
        pp = synthetic.walkers(n_port, seed=11, densities=(density,), with_sci=False)
        t0 = time.perf_counter()
        for p in pp:
            oracle.direct_eval(g, pz, pc, p.mor, oracle.cosmo(p.om, p.h0), p.tables)
        dt = time.perf_counter() - t0
        out["port_direct_quadrature"] = {
            "value": n_port / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n_port} points, FP64 direct nested GL at {density}x nodes (C), 1 thread"}
    return out


def run_reference(a):
    """Reference arm: the reference chain on all host cores (one point per
    worker process per step; the reference evaluates one point per CosmoSIS
    execute, single-threaded)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    import oracle
    oracle.build()
    _, _, have_ref = _ref_chain_setup()
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        for w in range(a.warmup):
            pool.map(_ref_worker, [100 + w * cores + i for i in range(cores)])
        t0 = time.perf_counter()
        for s in range(a.steps):
            pool.map(_ref_worker, [1000 + s * cores + i for i in range(cores)])
        dt = time.perf_counter() - t0
    value = a.steps * cores / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * dt / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded walkers, HMF/dV/dz tables)",
            "config": {"workload": WORKLOAD, "points_per_step": cores,
                       "reference_resolution": "sel_function 192x64x32, SelGL 96x64 (its "
                                               "tabulation differs from the converged "
                                               "integral by ~4e-4)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                             "kind": _ref_kind(have_ref),
                             "sample": f"{cores} points per step, one per core; "
                                       + _ref_sample(have_ref),
                             "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _device_batch(eng, pts, grid_of, dev):
    """Packed device buffers (points, tables) of a walker list."""
    import torch
    parr = eng.points_array(pts, grid_of=grid_of)
    ph = torch.empty(C.sizeof(parr), dtype=torch.uint8, pin_memory=True)
    C.memmove(ph.data_ptr(), C.addressof(parr), C.sizeof(parr))
    return ph.to(dev), torch.tensor(eng.pack(pts)).to(dev)


def workload_run(name, grids, dens, n_points, shear, steps, dev):
    """One evaluation per step of `n_points` walkers (each with its own HMF,
    dV/dz and Sigma_crit tables) over `grids`, counts and, with `shear`, the
    stacked miscentred DeltaSigma; mixed form, device-resident inputs, L2
    flushed between steps, one CUDA-graph replay per step.  The FP64 form on
    the same batch gives the relative errors."""
    import numpy as np
    import torch

    from y3_cluster_cpp_b200 import engine, synthetic

    gi = {d: i for i, d in enumerate(dens)}
    pts = synthetic.walkers(n_points, seed=1, densities=dens)
    t0 = pts[0].tables
    pz, pc = synthetic.plob_baseline()
    eng = engine.Engine(grids, len(t0["hmf_m_h"]), len(t0["hmf_z"]), len(t0["dist_z"]),
                        (pz, pc), max_points=n_points, n_sci=len(t0["sci_z"]), shear=shear)
    pd, td = _device_batch(eng, pts, lambda p: gi[p.density], dev)
    nb, nr = eng.n_bins, eng.n_R
    cd = torch.empty((n_points, nb), dtype=torch.float64, device=dev)
    sd = torch.empty((n_points, nb, max(nr, 1)), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step(prec):
        eng.eval_device(prec, n_points, pd.data_ptr(), td.data_ptr(), cd.data_ptr(),
                        sd.data_ptr() if nr else 0, sp)

    tuning = eng.autotune(n_points, pd.data_ptr(), td.data_ptr(), cd.data_ptr())
    step(engine.FP64)
    eng.sync(sp)
    c64, s64 = cd.cpu().numpy().copy(), sd.cpu().numpy().copy()
    step(engine.MIXED)
    eng.sync(sp)
    cmx, smx = cd.cpu().numpy().copy(), sd.cpu().numpy().copy()
    err_c = float(np.max(np.abs(cmx / c64 - 1)))
    err_s = float(np.max(np.abs(smx / s64 - 1))) if nr else None
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(3):
        flush.zero_()
        step(engine.MIXED)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    torch.cuda.synchronize(dev)
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        step(engine.MIXED)
        e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / steps
    eng.profile(True)
    for _ in range(3):
        flush.zero_()
        step(engine.MIXED)
    prof = eng.profile_read()
    eng.profile(False)
    eng.sync(sp)
    tot = sum(prof[k] for k in ("prep", "contraction", "shear", "final"))
    eng.close()
    return {"workload": name, "points_per_step": n_points, "value": n_points / (ms / 1e3),
            "unit": UNIT, "ms_per_step": ms, "steps": steps,
            "max_rel_err_counts_vs_fp64": err_c, "max_rel_err_delta_sigma_vs_fp64": err_s,
            "stage_share": {k: prof[k] / tot for k in ("prep", "contraction", "shear", "final")},
            "tuning": tuning, "l2": "flushed between steps", "cuda_graph": True}


def module_latency(n_calls=40):
    """Per-sample latency of the drop-in module: NumCountsFastMass.so with
    engine = fused, setup once, then execute() on a CosmoSIS-style DataBlock
    per parameter point (the whole integral, S_stack stage included), as
    CosmoSIS calls it; median wall time per execute after warm-up, one point
    per call, for the configs' 1x and 4x node densities."""
    import numpy as np

    from y3_cluster_cpp_b200 import prj_params, synthetic
    from y3_cluster_cpp_b200.cosmosis import DataBlock, Module

    out = {}
    p = synthetic.fiducial()
    pz, pc = synthetic.plob_baseline()
    lab = "NumCountsFastMass"
    for name, dens in (("1x (64 lnM x 32 z_t x 64 lam_t x 64 lam_o x 16 z_o)", 1),
                       ("4x (256 x 128 x 256 x 256 x 64)", 4)):
        g = synthetic.grid(dens)
        res = {}
        for prec in ("mixed", "fp64"):
            o = DataBlock()
            o[lab, "engine"] = "fused"
            o[lab, "precision"] = prec
            o[lab, "bin_index"] = np.arange(12)
            le, ze = g["lam_edges"], g["zob_edges"]
            o[lab, "lam_min"], o[lab, "lam_max"] = np.tile(le[:-1], 3), np.tile(le[1:], 3)
            o[lab, "zob_min"], o[lab, "zob_max"] = np.repeat(ze[:-1], 4), np.repeat(ze[1:], 4)
            o[lab, "sigma_z"] = np.zeros(12)
            o[lab, "sz0"] = 0.01
            for k in ("zt_lo", "zt_hi", "lnm_lo", "lnm_hi"):
                o[lab, {"zt_lo": "zt_low", "zt_hi": "zt_high", "lnm_lo": "lnm_low",
                        "lnm_hi": "lnm_high"}[k]] = float(g[k])
            o[lab, "n_lnm"], o[lab, "n_z"], o[lab, "n_lt"] = g["n_m"], g["n_z"], g["n_t"]
            o[lab, "n_lo"], o[lab, "n_zo"] = g["n_o"], g["n_zo"]
            b = DataBlock()
            b["cosmological_parameters", "omega_M"] = p.om
            b["cosmological_parameters", "omega_lambda"] = 1 - p.om
            b["cosmological_parameters", "omega_k"] = 0.0
            b["cosmological_parameters", "h0"] = p.h0
            b["cosmological_parameters", "omega_nu"] = 0.0
            b["cluster_abundance", "hmf_s"] = 0.0
            b["cluster_abundance", "hmf_q"] = 1.0
            t = p.tables
            b["mass_function", "m_h"], b["mass_function", "z"] = t["hmf_m_h"], t["hmf_z"]
            b["mass_function", "dndlnmh"] = t["dndlnmh"]
            b["distances", "z"], b["distances", "d_a"] = t["dist_z"], t["dist_da"]
            for k, v in dict(A=p.A, B=p.B, C=p.C, sigma_intr=p.sigma, M_pivot=p.Mpiv).items():
                b["cluster_mor", k] = v
            b["plob_ltr_params", "z"] = pz
            for k, row in zip(prj_params.COEFF_NAMES, pc):
                b["plob_ltr_params", k] = row
            m = Module(lab)
            if not m.setup(o):
                raise RuntimeError("fused module setup failed")
            for _ in range(3):
                if m.execute(b) != 0:
                    raise RuntimeError("fused module execute failed")
            ts = []
            for _ in range(n_calls):
                t0 = time.perf_counter()
                m.execute(b)
                ts.append(time.perf_counter() - t0)
            m.cleanup()
            res[prec + "_ms"] = 1e3 * statistics.median(ts)
        out[name] = res
    return {"module": "NumCountsFastMass.so, engine = fused (whole integral per execute)",
            "calls": n_calls, "per_sample": out,
            "reference_published_ms": {
                "NumCountsFastMass/NumCountsSel execute (S_stack given)": 6.0,
                "number-count module page figure": 22.0,
                "sel_function S_stack tabulation (upstream module)": 215.0}}


def prj_latency(n_calls=30):
    """Per-sample latency of the frozen-physics projection shear
    (y3b_prj_eval: host grids, table upload, device sums, 12 slices x 10
    radii, default options, direct single-kernel quadrature), next to the
    reference's published 82 ms per sample."""
    import numpy as np

    from y3_cluster_cpp_b200 import engine, synthetic
    p = synthetic.fiducial()
    prj = synthetic.prj_tables(p)
    R10 = np.logspace(np.log10(0.2), np.log10(5.0), 10)
    grid = dict(lambda_bin=np.repeat(np.tile(np.arange(4), 3), 10),
                zo_low=np.repeat(np.repeat([0.2, 0.35, 0.5], 4), 10),
                zo_high=np.repeat(np.repeat([0.35, 0.5, 0.65], 4), 10), radii=np.tile(R10, 12))
    h = engine.PrjShear(grid)
    cz = engine.cosmo(p.om, p.h0)
    for _ in range(3):
        h.eval(cz, p.tables, prj)
    ts = []
    for _ in range(n_calls):
        t0 = time.perf_counter()
        h.eval(cz, p.tables, prj)
        ts.append(time.perf_counter() - t0)
    h.close()
    return {"observable": "ShearPrjFrozenPhysics, 12 slices x 10 radii, 24 lnM nodes",
            "ms_per_sample": 1e3 * statistics.median(ts), "calls": n_calls,
            "reference_published_ms": 82.0}


def bsel_run(n_calls=30, n_batch=256):
    """The selection-bias operators P1, I1, J (y3b_bsel_eval; 12 (z_obs bin,
    richness bin) points, default nodes: 60 lam_t x 24 lnM x up to 80 z x 10
    theta, 80 reference z nodes): per-sample latency through the host-buffer
    call, batched throughput over seeded walkers, and the reference's own
    P_operator (compiled from its sources, where present) timed on one host
    core on the same samples, next to the reference's published 66-74 ms."""
    import numpy as np

    from oracle import ref as R
    from y3_cluster_cpp_b200 import engine, synthetic
    grid = dict(zo_low=np.repeat([0.2, 0.35, 0.5], 4), zo_high=np.repeat([0.35, 0.5, 0.65], 4),
                lambda_bin=np.tile(np.arange(4), 3))
    lo, hi = np.log(1e13), np.log(10 ** 15.5)
    hod = dict(log10_Mmin=11.7, log10_M1=12.9, alpha=0.85, epsilon=0.2, sigma_lambda=0.2)
    pts = synthetic.walkers(n_batch, seed=3, densities=(1,), with_sci=False)
    prj0 = synthetic.prj_tables(pts[0], n_r=120)
    samples = [(engine.cosmo(p.om, p.h0), p.tables, synthetic.prj_tables(p, n_r=120),
                dict(hod, alpha=0.8 + 0.1 * (i % 4) / 3)) for i, p in enumerate(pts)]
    h1 = engine.BselMarg(grid, lo, hi, max_samples=1)
    for _ in range(3):
        h1.eval(samples[:1])
    ts = []
    for _ in range(n_calls):
        t0 = time.perf_counter()
        h1.eval(samples[:1])
        ts.append(time.perf_counter() - t0)
    h1.close()
    hb = engine.BselMarg(grid, lo, hi, max_samples=n_batch)
    hb.eval(samples)
    tb, tk = [], []
    for _ in range(5):
        t0 = time.perf_counter()
        out = hb.eval(samples)
        tb.append(time.perf_counter() - t0)
        tk.append(hb.kernel_ms())
    hb.close()
    res = {"observable": "P_operator (b_sel_marg): P1, I1, J on 12 (z_obs bin, richness bin) "
                         "points, 60 lam_t x 24 lnM x <=80 z x 10 theta",
           "ms_per_sample": 1e3 * statistics.median(ts), "calls": n_calls,
           "batched": {"samples": n_batch, "samples_per_s": n_batch / statistics.median(tb),
                       "ms_per_call": 1e3 * statistics.median(tb),
                       "kernel_ms_per_call": statistics.median(tk),
                       "device_samples_per_s": n_batch / (1e-3 * statistics.median(tk)),
                       "note": "ms_per_call includes the Python-side sample structs, host "
                               "packing into pinned memory and the copies"},
           "reference_published_ms": [66.0, 74.0]}
    del prj0
    if R.available():
        n_ref = 4
        t0 = time.perf_counter()
        refs = []
        for p, smp in zip(pts[:n_ref], samples[:n_ref]):
            cz = dict(omega_m=p.om, omega_nu=0.0, omega_lambda=1.0 - p.om, omega_k=0.0,
                      h0=p.h0, hmf_s=0.0, hmf_q=1.0)
            refs.append(R.bsel_marg(dict(lnm_low=lo, lnm_high=hi), cz, p.tables, smp[2], smp[3],
                                    grid))
        dt = (time.perf_counter() - t0) / n_ref
        refs = np.stack(refs)
        scale = np.max(np.abs(refs), axis=(0, 1))
        res["reference_cpu"] = {"ms_per_sample": 1e3 * dt, "cores": 1, "kind": "reference",
                                "sample": f"{n_ref} walkers, the reference's P_operator "
                                          "compiled from its sources, 1 thread"}
        res["max_abs_diff_vs_reference_over_scale"] = float(
            np.max(np.abs(out[:n_ref] - refs) / scale))
    return res


def serving_run(a, rank, dev):
    """Serving workload: a Poisson request stream (mean gap 2 ms) of requests
    of 1..1024 points (log-uniform), points from the batched-config prior at
    mixed 1x/2x/4x densities, each with its own tables; counts at 1e-4.
    Runs the stream through the continuous-batching server and, for
    comparison, the plain per-request FP64 form (each request evaluated by
    itself in arrival order, queueing included).  Latency = completion -
    arrival."""
    import numpy as np
    import torch

    from y3_cluster_cpp_b200 import _capi, engine, serve, synthetic

    n_req = a.serve_requests
    dens = (1, 2, 4)
    grids = [synthetic.grid(d) for d in dens]
    gi = {d: i for i, d in enumerate(dens)}
    pool = synthetic.walkers(96, seed=2 + 1000 * rank, densities=dens)
    t0 = pool[0].tables
    pz, pc = synthetic.plob_baseline()
    eng = engine.Engine(grids, len(t0["hmf_m_h"]), len(t0["hmf_z"]), len(t0["dist_z"]),
                        (pz, pc), max_points=2048, n_sci=len(t0["sci_z"]))
    tab_pool = eng.pack(pool)
    sizes = serve.request_sizes(n_req, seed=2 + rank)
    arrivals = serve.poisson_arrivals(n_req, 0.002, seed=2 + rank)
    rng = np.random.default_rng(3 + rank)
    total = int(sizes.sum())
    tables_h = torch.empty((total, eng.stride), dtype=torch.float64, pin_memory=True).numpy()
    # The same requests with the HMF grid in FP32 in the packed tables (the
    # mixed form's wire format: fewer host-to-device bytes per point).
    eng32 = engine.Engine(grids, len(t0["hmf_m_h"]), len(t0["hmf_z"]), len(t0["dist_z"]),
                          (pz, pc), max_points=2048, n_sci=len(t0["sci_z"]), hmf_fp32=True)
    tab_pool32 = eng32.pack(pool)
    tables32_h = torch.empty((total, eng32.stride), dtype=torch.float64, pin_memory=True).numpy()
    reqs, reqs32, o = [], [], 0
    for n in sizes:
        idx = rng.integers(0, len(pool), n)
        tables_h[o:o + n] = tab_pool[idx]
        tables32_h[o:o + n] = tab_pool32[idx]
        pts = eng.points_array([pool[i] for i in idx], grid_of=lambda p: gi[p.density])
        reqs.append((pts, tables_h[o:o + n]))
        reqs32.append((pts, tables32_h[o:o + n]))
        o += n

    # plain per-request FP64 GPU form, in arrival order (one request at a time)
    lib = engine.lib()
    fp64_counts, finish, lat64, busy = [], 0.0, [], 0.0
    for (pts, tab), t_arr in zip(reqs, arrivals):
        out = np.empty((len(pts), eng.n_bins))
        t_s = time.perf_counter()
        engine.check(lib.y3b_engine_eval(eng.handle, engine.FP64, len(pts), pts,
                                         _capi.ptr(tab), _capi.ptr(out), None))
        svc = time.perf_counter() - t_s
        busy += svc
        finish = max(finish, t_arr) + svc
        lat64.append(finish - t_arr)
        fp64_counts.append(out)
    fp64_tp = total / finish
    fp64_capacity = total / busy     # back to back, no arrival gaps

    # warm the server path once, then the timed stream, then the same
    # requests kept `outstanding` at a time (saturated: no arrival gaps)
    outstanding = 16
    with serve.Server(eng, pool_points=8192, max_batch=2048, precision=engine.MIXED) as srv:
        srv.wait(srv.submit(*reqs[0]))
        s0 = srv.stats()
        run = serve.run_stream(srv, reqs, arrivals)
        s1 = srv.stats()
        sat = serve.run_closed_loop(srv, reqs, outstanding)
        s2 = srv.stats()
    eng.close()
    with serve.Server(eng32, pool_points=8192, max_batch=2048, precision=engine.MIXED) as srv:
        srv.wait(srv.submit(*reqs32[0]))
        s3 = srv.stats()
        sat32 = serve.run_closed_loop(srv, reqs32, outstanding)
        s4 = srv.stats()
    eng32.close()
    err = max(float(np.max(np.abs(r["counts"] / c - 1)))
              for rr in (run, sat, sat32) for r, c in zip(rr["results"], fp64_counts))
    sat32_tp = total / sat32["wall_s"]
    sat32_launches = s4["launches"] - s3["launches"]
    launches = s1["launches"] - s0["launches"]
    sat_launches = s2["launches"] - s1["launches"]
    sat_tp = total / sat["wall_s"]
    return {"requests": n_req, "points": total,
            "arrivals": "Poisson, mean gap 2 ms", "sizes": "round(exp(U[0, ln 1024]))",
            "densities": "1x/2x/4x in thirds per point", "tables": "per point, pinned host",
            "throughput": total / run["wall_s"], "unit": UNIT,
            **serve.percentiles_ms(run["latency_s"]),
            "launches": launches, "mean_launch_points": total / max(launches, 1),
            "max_launch_points": s1["max_launch_points"],
            "max_rel_err_vs_fp64": err,
            "fp64_per_request": {"throughput": fp64_tp, "unit": UNIT,
                                 **serve.percentiles_ms(np.asarray(lat64)),
                                 "capacity": fp64_capacity,
                                 "form": "FP64 direct nested GL (one exp per lnM, z_t, lam_t "
                                         "node, no factorisation), one engine call per "
                                         "request, host tables"},
            "saturated": {"outstanding_requests": outstanding, "throughput": sat_tp,
                          "unit": UNIT, **serve.percentiles_ms(sat["latency_s"]),
                          "launches": sat_launches,
                          "mean_launch_points": total / max(sat_launches, 1),
                          "speedup_vs_fp64_per_request": sat_tp / fp64_capacity,
                          "host_table_bytes_per_point": eng.stride * 8},
            "saturated_fp32_hmf_tables": {
                "outstanding_requests": outstanding, "throughput": sat32_tp, "unit": UNIT,
                **serve.percentiles_ms(sat32["latency_s"]),
                "launches": sat32_launches,
                "mean_launch_points": total / max(sat32_launches, 1),
                "speedup_vs_fp64_per_request": sat32_tp / fp64_capacity,
                "host_table_bytes_per_point": eng32.stride * 8}}


def run_ours(a):
    import numpy as np
    import torch

    from y3_cluster_cpp_b200 import _capi, engine, sharding, synthetic

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    engine.check(engine.lib().y3b_device_init(local))
    dev = torch.device("cuda", local)

    # ---- inputs: B points, `unique` distinct walker tables (seed + rank) ----
    B = a.batch
    uniq = synthetic.walkers(min(a.unique, B), seed=1 + 1000 * rank, densities=(a.density,))
    pts = [uniq[i % len(uniq)] for i in range(B)]
    g = synthetic.grid(a.density)
    t0 = uniq[0].tables
    pz, pc = synthetic.plob_baseline()
    # Two engines on the same points: `eng32` is the mixed form with the HMF
    # grid in FP32 in its packed tables (the form's wire format: it rounds
    # that grid to FP32 on the device anyway, so its counts equal those from
    # FP64 tables); `eng` takes FP64 tables and gives the FP64 reference.
    eng = engine.Engine([g], len(t0["hmf_m_h"]), len(t0["hmf_z"]), len(t0["dist_z"]), (pz, pc),
                        max_points=B, n_sci=len(t0["sci_z"]))
    eng32 = engine.Engine([g], len(t0["hmf_m_h"]), len(t0["hmf_z"]), len(t0["dist_z"]),
                          (pz, pc), max_points=B, n_sci=len(t0["sci_z"]), hmf_fp32=True)
    n_bins = eng.n_bins
    tab_u = eng.pack(uniq)
    tables_h = torch.empty((B, eng.stride), dtype=torch.float64, pin_memory=True)
    tables_h.numpy()[:] = tab_u[np.arange(B) % len(uniq)]
    tab32 = eng32.pack(uniq)
    tables32_h = torch.empty((B, eng32.stride), dtype=torch.float64, pin_memory=True)
    tables32_h.numpy()[:] = tab32[np.arange(B) % len(uniq)]
    parr = eng.points_array(pts, grid_of=lambda _: 0)
    pts_h = torch.empty(C.sizeof(parr), dtype=torch.uint8, pin_memory=True)
    C.memmove(pts_h.data_ptr(), C.addressof(parr), C.sizeof(parr))
    counts_h = torch.empty((B, n_bins), dtype=torch.float64, pin_memory=True)
    tables_d = tables_h.to(dev)
    tables32_d = tables32_h.to(dev)
    pts_d = pts_h.to(dev)
    counts_d = torch.empty((B, n_bins), dtype=torch.float64, device=dev)
    # A dedicated (non-default) stream: the library launches on it and the
    # CUDA events below are recorded on it.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream

    def step(prec, n=B):
        if prec == engine.FP64:
            eng.eval_device(prec, n, pts_d.data_ptr(), tables_d.data_ptr(), counts_d.data_ptr(),
                            0, sp)
        else:
            eng32.eval_device(prec, n, pts_d.data_ptr(), tables32_d.data_ptr(),
                              counts_d.data_ptr(), 0, sp)

    # ---- autotuner: ring depth and bins per tile, on this batch (untimed) ----
    tuning = eng32.autotune(B, pts_d.data_ptr(), tables32_d.data_ptr(), counts_d.data_ptr())
    eng.autotune(B, pts_d.data_ptr(), tables_d.data_ptr(), counts_d.data_ptr())

    # ---- accuracy of the mixed form vs FP64 on this batch (untimed) ----
    step(engine.FP64)
    eng.sync(sp)
    c64 = counts_d.double().cpu().numpy().copy()
    step(engine.MIXED)
    eng.sync(sp)
    cmx = counts_d.double().cpu().numpy().copy()
    max_rel = float(np.max(np.abs(cmx / c64 - 1)))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)


    # ---- device-resident timed region ----
    for _ in range(a.warmup):
        flush.zero_()
        step(engine.MIXED)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    # NVML enumerates every GPU of the host: find ours by UUID.
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:  # noqa: BLE001
        gpu_id = local
    clocks = ClockSampler(gpu_id)
    clocks.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    launches0 = engine.launch_count()
    torch.cuda.synchronize(dev)
    for s in range(a.steps):
        flush.zero_()
        starts[s].record(stream)
        step(engine.MIXED)          # a replayed CUDA graph of the whole evaluation
        ends[s].record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    launches = engine.launch_count() - launches0
    eng32.sync(sp)
    clk = clocks.stop()
    # Stage times (CUDA events the library records around each stage on the
    # same stream; plain launches, as stage timing bypasses the graph).
    eng32.profile(True)
    for _ in range(max(3, a.steps // 2)):
        flush.zero_()
        step(engine.MIXED)
    prof = eng32.profile_read()
    eng32.profile(False)
    step_ms = [st.elapsed_time(en) for st, en in zip(starts, ends)]
    total_ms = sharding.max_over_ranks(sum(step_ms), dev)
    value = world * B * a.steps / (total_ms / 1e3)

    # ---- roofline of the dominant kernel (the tcgen05 contraction) ----
    gemm_ms = prof["contraction"] / max(prof["evals"], 1)
    flops_alg = 2.0 * g["n_m"] * (len(g["lam_edges"]) - 1) * g["n_z"] * g["n_t"] * B
    peak_tf, peak_gbs, peak_kind = measured_peaks()
    achieved_tf = flops_alg / (gemm_ms / 1e3) / 1e12
    # The contraction skips lam_t stages where the MOR density of every
    # (lnM, z) pair of a tile is below 4e-6 of its peak; the tensor pipe
    # issues this fraction of the dense stages.
    torch.cuda.synchronize(dev)
    st_ex, st_dn = eng32.stage_count()
    issued = st_ex / max(st_dn, 1)
    stage_share = {k: prof[k] / max(sum(prof[x] for x in ("prep", "contraction", "shear",
                                                             "final")), 1e-12)
                   for k in ("prep", "contraction", "final")}

    # ---- plain FP64 GPU form: one point per call (the metric's denominator) ----
    n_plain = 16
    for _ in range(3):
        step(engine.FP64, 1)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(n_plain):
        step(engine.FP64, 1)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    plain_fp64 = n_plain / (e0.elapsed_time(e1) / 1e3)
    # batched FP64 on the same batch, for context
    flush.zero_()
    e0.record(stream)
    step(engine.FP64)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    fp64_batched = B / (e0.elapsed_time(e1) / 1e3)

    # ---- end to end through the C ABI with pinned host buffers ----
    lib = engine.lib()
    PPt = C.cast(C.c_void_p(pts_h.data_ptr()), C.POINTER(_capi.Point))
    TPt = C.cast(C.c_void_p(tables_h.data_ptr()), _capi.PD)
    CPt = C.cast(C.c_void_p(counts_h.data_ptr()), _capi.PD)
    for _ in range(2):
        engine.check(lib.y3b_engine_eval(eng.handle, engine.MIXED, B, PPt, TPt, CPt, None))
    e2e_t = []
    for _ in range(max(3, a.steps // 2)):
        t_0 = time.perf_counter()
        engine.check(lib.y3b_engine_eval(eng.handle, engine.MIXED, B, PPt, TPt, CPt, None))
        e2e_t.append(time.perf_counter() - t_0)
    e2e_total = sharding.max_over_ranks(sum(e2e_t), dev)
    e2e64_value = world * B * len(e2e_t) / e2e_total
    h2d64 = B * (C.sizeof(_capi.Point) + eng.stride * 8)
    d2h = B * n_bins * 8
    # The same through the engine whose packed tables carry the HMF grid in
    # FP32 (the headline e2e): its counts equal those above up to the
    # autotuner's choice of tile, which changes FP32 rounding only, for about
    # half the bytes per point.
    counts32_h = torch.empty((B, n_bins), dtype=torch.float64, pin_memory=True)
    TPt32 = C.cast(C.c_void_p(tables32_h.data_ptr()), _capi.PD)
    CPt32 = C.cast(C.c_void_p(counts32_h.data_ptr()), _capi.PD)
    for _ in range(2):
        engine.check(lib.y3b_engine_eval(eng32.handle, engine.MIXED, B, PPt, TPt32, CPt32, None))
    diff32 = float(np.max(np.abs(counts32_h.numpy() / counts_h.numpy() - 1)))
    e2e_t = []
    for _ in range(max(3, a.steps // 2)):
        t_0 = time.perf_counter()
        engine.check(lib.y3b_engine_eval(eng32.handle, engine.MIXED, B, PPt, TPt32, CPt32, None))
        e2e_t.append(time.perf_counter() - t_0)
    e2e_total = sharding.max_over_ranks(sum(e2e_t), dev)
    e2e_value = world * B * len(e2e_t) / e2e_total
    h2d = B * (C.sizeof(_capi.Point) + eng32.stride * 8)
    eng32.close()

    eng.close()
    serving = None
    if a.serve_requests > 0:
        serving = serving_run(a, rank, dev)
    modlat = module_latency() if a.extra_workloads else None
    prjlat = prj_latency() if a.extra_workloads else None
    bsel = bsel_run() if a.extra_workloads else None
    extra = None
    if a.extra_workloads:
        from y3_cluster_cpp_b200 import synthetic as _syn
        sh15 = _syn.shear_opts(n_theta=64, n_s=128, n_R=15)
        extra = [
            workload_run("batched: 256 walkers, 1x/2x/4x grids in thirds, counts + stacked "
                         "miscentred DeltaSigma (15 R)",
                         [_syn.grid(1), _syn.grid(2), _syn.grid(4)], (1, 2, 4), 256, sh15,
                         a.steps, dev),
            workload_run("DeltaSigma: stacked miscentred NFW one-halo, 12 bins x 15 R "
                         "(64 theta x 128 R_mis x 64 lnM x 32 z_t x 64 lam_t), 2048 walkers",
                         [_syn.grid(1)], (1,), 2048, sh15, a.steps, dev),
        ]

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a.cpu_sample, a.density, a.cpu_port_sample)

    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/bf16x3 (f64 final sums)",
            "data": "synthetic (seeded walkers; per-point HMF, dV/dz, Sigma_crit tables)",
            "config": {"workload": WORKLOAD, "points_per_step_per_gpu": B,
                       "distinct_walker_tables": len(uniq), "density": a.density,
                       "l2": "flushed between timed steps (256 MB write)",
                       "tables": "device-resident packed tables, HMF grid in FP32 (hmf_fp32)",
                       "tuning": tuning, "cuda_graph": True,
                       "parallelism": f"walker-sharded x{world}"},
            "max_rel_err_vs_fp64": max_rel,
            "plain_fp64": {"value": plain_fp64, "unit": UNIT,
                           "mode": "FP64 direct quadrature, one point per call"},
            "fp64_batched": {"value": fp64_batched, "unit": UNIT},
            "speedup_vs_plain_fp64": value / world / plain_fp64,
            "roofline": {"bound": "tensor", "achieved": achieved_tf, "peak": peak_tf,
                         "unit": "TFLOP/s", "frac": achieved_tf / peak_tf,
                         "traffic": ncu_traffic(a.density, B),
                         "kernel": "contract_kernel",
                         "algorithmic_flops_per_launch": flops_alg,
                         "issued_stage_fraction": issued,
                         "tensor_pipe_flops_per_launch": 3 * flops_alg * issued,
                         "tensor_pipe_tflops": 3 * achieved_tf * issued,
                         "peak_source": f"bf16_tflops ({peak_kind})",
                         "avg_launch_ms": gemm_ms},
            "stage_share": stage_share,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "tables": "per point, HMF grid in FP32 (hmf_fp32), pinned host",
                    "max_rel_diff_vs_fp64_tables": diff32},
            "e2e_fp64_tables": {"value": e2e64_value, "unit": UNIT, "h2d_bytes_per_step": h2d64,
                                "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if serving is not None:
            line["serving"] = serving
        if modlat is not None:
            line["module_execute"] = modlat
        if prjlat is not None:
            line["projection_shear"] = prjlat
        if bsel is not None:
            line["selection_bias"] = bsel
        if extra is not None:
            line["other_workloads"] = extra
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


# DRAM bytes (read + write) per point of one contraction launch at 4x nodes,
# from one ncu capture of the small case:
#   ncu --set full --clock-control none -k regex:contract_kernel -s 2 -c 1 \
#       python bench.py --steps 3 --warmup 3 --batch 256 --no-cpu-baseline \
#       --serve-requests 0 --no-extra-workloads
# (73.32 MB read + 3.07 MB written over 256 points).  Traffic grows with the
# points (each reads its own operand blocks), so a launch of B points moves
# B times this.
CONTRACT_TRAFFIC_BYTES_PER_POINT_4X = 298426.0


def ncu_traffic(density, points):
    return CONTRACT_TRAFFIC_BYTES_PER_POINT_4X * points if density == 4 else None


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
