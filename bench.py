"""Benchmark: FP64 spherical-harmonic synthesis + analysis round trip on a
Gauss--Legendre grid (CHarm's charm_shs_point + charm_sha_point), nmax 2190,
grid 2191 x 4382, Kaula-decay coefficients (seed 2000), r = R.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--nmax N]
                    [--impl ours|reference]

One step = one SHS + SHA round trip.  "value" is seconds per round trip with
the coefficients and the grid resident in HBM (device-timed with CUDA
events on the library's stream, L2 flushed between steps by a 256 MiB
write); "e2e" is the same round trip through the C ABI with pinned host
buffers, host<->device copies included (with, measured after the timed
region, each host-array call alone, the pinned copy bandwidths and the
time the round trip's copies alone take at them).  With --gpus N > 1
(torchrun) every
rank runs its own round trips (replicas, no collective on the data path);
value = max-over-ranks time / (N * K).

--impl reference times CHarm 0.4.9 itself on the host cores: its own
sources compiled by oracle/build_ref.py (OpenMP, AVX-512 or AVX2, -O3
-ffast-math, FFTW replaced by the FFTW-API shim of oracle/fftw_shim), every
step the full round trip of the same workload through charm_shs_point and
charm_sha_point.  It loads nothing of the charm_b200 package's library.
"""
import argparse
import ctypes as ct
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("SHS+SHA s at nmax 2190/10800: plain FP64 vs batched split-prec, "
          "% FP64 peak")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--nmax", type=int, default=2190)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch-i8", action="store_true",
                    help="skip the batched split-precision section")
    ap.add_argument("--no-n10800", action="store_true",
                    help="skip the nmax 10800 round trip")
    ap.add_argument("--workload", default="roundtrip",
                    choices=["roundtrip", "sctr-cg", "batch", "cells"],
                    help="sctr-cg: scattered synthesis + adjoint + CGLS fit "
                         "(nmax 2160); batch: 64 coefficient sets with ten "
                         "quantities each on DH grids; cells: block-mean "
                         "synthesis and analysis on 2191 x 4382 cells; "
                         "instead of the grid round trip")
    ap.add_argument("--npoint", type=int, default=10_000_000)
    ap.add_argument("--cg-iters", type=int, default=20)
    ap.add_argument("--no-batch-dh", action="store_true",
                    help="skip the 64-set DH section")
    ap.add_argument("--no-sctr", action="store_true",
                    help="skip the scattered-point section")
    ap.add_argument("--sctr-points", type=int, default=1_000_000,
                    help="points of the scattered section of the default "
                         "line (the full workload: --workload sctr-cg)")
    ap.add_argument("--sctr-iters", type=int, default=2)
    ap.add_argument("--no-cells", action="store_true",
                    help="skip the block-mean (cell) synthesis and analysis")
    ap.add_argument("--no-gfm", action="store_true",
                    help="skip the global gravity forward modelling section")
    return ap.parse_args()


def dist_env():
    from charm_b200.replicas import dist_env as env
    return env()


# ---------------------------------------------------------------------------
# Clocks sampling during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    # A timed region of a few milliseconds is shorter than the sampling
    # interval: the caller runs the same work untimed for SETTLE_S just
    # before it and keeps the samples of [settle start, region end], a
    # window in which the GPU does nothing else.
    SETTLE_S = 0.3

    def __init__(self, index):
        self.index = index
        self.rows = []             # (host time, fields)
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
            return
        # nvidia-smi is running once its first line has arrived
        t = time.perf_counter()
        while not self.rows and time.perf_counter() - t < 5.0:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(),
                              [x.strip() for x in line.split(",")]))

    def mark(self, t0, t1):
        self.t0, self.t1 = t0, t1

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.th.join(timeout=2)
        rows = [r for t, r in self.rows
                if self.t0 is None or self.t0 <= t <= self.t1]
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows),
                "window_s": ((self.t1 - self.t0)
                             if self.t0 is not None else None),
                "interval_ms": 50}


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    import charm_b200 as cb
    from charm_b200._lib import _libcharm
    from charm_b200.replicas import job_seconds_per_transform, max_over_ranks
    from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula

    L = _libcharm
    L.charm_b200_shs_point_dev.argtypes = [
        ct.c_void_p, ct.c_ulong, ct.c_double, ct.c_double, ct.c_void_p,
        ct.c_void_p, ct.c_ulong, ct.c_int, ct.c_uint, ct.c_uint, ct.c_uint,
        ct.c_void_p, ct.c_void_p]
    L.charm_b200_sha_point_dev.argtypes = [
        ct.c_void_p, ct.c_void_p, ct.c_ulong, ct.c_double, ct.c_double,
        ct.c_ulong, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.charm_b200_stream.restype = ct.c_void_p
    L.charm_b200_timing.argtypes = [ct.c_int]
    L.charm_b200_timing_read.argtypes = [
        ct.POINTER(ct.c_double), ct.POINTER(ct.c_ulonglong), ct.c_int,
        ct.POINTER(ct.c_ulonglong), ct.POINTER(ct.c_ulonglong)]
    L.charm_b200_fp64_peak_tflops.restype = ct.c_double

    N = args.nmax
    c, s = kaula(N, 2000)
    pnt = cb.PointGridGL(N, R_EARTH)
    nlat, nlon = pnt.lat.size, pnt.lon.size
    T = c.size
    dev = torch.device("cuda", torch.cuda.current_device())
    d_c = torch.from_numpy(c).to(dev)
    d_s = torch.from_numpy(s).to(dev)
    d_f = torch.empty(nlat * nlon, dtype=torch.float64, device=dev)
    d_c2 = torch.empty(T, dtype=torch.float64, device=dev)
    d_s2 = torch.empty(T, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    sptr = L.charm_b200_stream()
    stream = torch.cuda.ExternalStream(sptr)
    err = L.charm_err_init()

    def check():
        if not L.charm_err_isempty(err):
            msg = ct.string_at(err.contents.msg).decode()
            raise RuntimeError(msg)

    def step_dev():
        L.charm_b200_shs_point_dev(ct.cast(pnt._Point, ct.c_void_p), N, GM,
                                   R_EARTH, d_c.data_ptr(), d_s.data_ptr(), N,
                                   0, 0, 0, 0, d_f.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        check()
        L.charm_b200_sha_point_dev(ct.cast(pnt._Point, ct.c_void_p),
                                   d_f.data_ptr(), N, GM, R_EARTH, N,
                                   d_c2.data_ptr(), d_s2.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        check()

    # warm-up (plans, tables, buffers)
    for _ in range(args.warmup):
        step_dev()
    torch.cuda.synchronize()
    rt = coef_rel_rms(d_c2.cpu().numpy(), d_s2.cpu().numpy(), c, s)

    peak = L.charm_b200_fp64_peak_tflops()

    # ---- device-resident timed region --------------------------------
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    # the same round trip, untimed, so that the clock samples see this load
    t_region0 = time.perf_counter()
    while time.perf_counter() - t_region0 < Clocks.SETTLE_S:
        step_dev()
        torch.cuda.synchronize()
    L.charm_b200_timing(1)
    per_step = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)           # L2 flush, outside the step's events
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        step_dev()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        per_step.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    ms = (ct.c_double * 7)()
    cnt = (ct.c_ulonglong * 7)()
    kl = ct.c_ulonglong()
    fe = ct.c_ulonglong()
    L.charm_b200_timing_read(ms, cnt, 7, ct.byref(kl), ct.byref(fe))
    L.charm_b200_timing(0)
    clocks.mark(t_region0, time.perf_counter())
    clk = clocks.stop()
    total_ms = max_over_ranks(float(sum(per_step)), dev)
    if dist is not None:
        dist.barrier()

    # ---- end to end through the C ABI with pinned host buffers -------
    hc = torch.from_numpy(c).pin_memory()
    hs = torch.from_numpy(s).pin_memory()
    hf = torch.empty(nlat * nlon, dtype=torch.float64).pin_memory()
    oc = torch.empty(T, dtype=torch.float64).pin_memory()
    os_ = torch.empty(T, dtype=torch.float64).pin_memory()
    P = ct.POINTER(ct.c_double)
    shc_in = L.charm_shc_init(N, GM, R_EARTH, ct.cast(hc.data_ptr(), P),
                              ct.cast(hs.data_ptr(), P))
    shc_out = L.charm_shc_init(N, GM, R_EARTH, ct.cast(oc.data_ptr(), P),
                               ct.cast(os_.data_ptr(), P))

    def step_e2e():
        L.charm_shs_point(pnt._Point, shc_in, N, ct.cast(hf.data_ptr(), P), err)
        check()
        L.charm_sha_point(pnt._Point, ct.cast(hf.data_ptr(), P), N, shc_out,
                          err)
        check()

    for _ in range(max(1, args.warmup)):
        step_e2e()
    e2e_steps = max(2, min(args.steps, 5))
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    with torch.cuda.stream(stream):
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        step_e2e()
    wall = time.perf_counter() - t0
    with torch.cuda.stream(stream):
        f1.record(stream)
    f1.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), dev)
    rt_e2e = coef_rel_rms(oc.numpy(), os_.numpy(), c, s)

    # where the end-to-end time goes (after the timed region): each
    # host-array call alone (they return with their streams idle) and the
    # pinned copy bandwidths that bound them
    def call_ms(fn, reps=5):
        ts = []
        for _ in range(reps):
            t1 = time.perf_counter()
            fn()
            check()
            ts.append(time.perf_counter() - t1)
        return 1e3 * float(np.median(ts))
    shs_call_ms = call_ms(lambda: L.charm_shs_point(
        pnt._Point, shc_in, N, ct.cast(hf.data_ptr(), P), err))
    sha_call_ms = call_ms(lambda: L.charm_sha_point(
        pnt._Point, ct.cast(hf.data_ptr(), P), N, shc_out, err))
    d_tmp = torch.empty(nlat * nlon, dtype=torch.float64, device=dev)
    copy_gbs = {}
    for name, fn in (("h2d", lambda: d_tmp.copy_(hf, non_blocking=True)),
                     ("d2h", lambda: hf.copy_(d_tmp, non_blocking=True))):
        fn()
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record()
        for _ in range(5):
            fn()
        c1.record()
        c1.synchronize()
        copy_gbs[name] = 5 * 8 * nlat * nlon / (c0.elapsed_time(c1) * 1e-3) / 1e9
    del d_tmp
    # synthesis: coefficients up, then the grid down; analysis: the grid
    # up, then the coefficients down (neither pair can overlap)
    coef_b, grid_b = 16 * T, 8 * nlat * nlon
    copy_bound_ms = 1e3 * ((coef_b + grid_b) / (copy_gbs["h2d"] * 1e9) +
                           (grid_b + coef_b) / (copy_gbs["d2h"] * 1e9))

    # the same round trip with pageable host arrays (numpy), as PyHarm
    # passes them: the library stages the copies itself
    pc_, ps_ = np.ascontiguousarray(c), np.ascontiguousarray(s)
    pf_ = np.empty(nlat * nlon)
    pc2, ps2 = np.empty(T), np.empty(T)
    shc_pin = L.charm_shc_init(N, GM, R_EARTH, pc_.ctypes.data_as(P),
                               ps_.ctypes.data_as(P))
    shc_pout = L.charm_shc_init(N, GM, R_EARTH, pc2.ctypes.data_as(P),
                                ps2.ctypes.data_as(P))

    def step_pageable():
        L.charm_shs_point(pnt._Point, shc_pin, N, pf_.ctypes.data_as(P), err)
        check()
        L.charm_sha_point(pnt._Point, pf_.ctypes.data_as(P), N, shc_pout, err)
        check()

    step_pageable()
    tpg = []
    for _ in range(3):
        t1 = time.perf_counter()
        step_pageable()
        tpg.append(time.perf_counter() - t1)
    e2e_pageable = {"value": float(np.median(tpg)), "unit": "s",
                    "round_trip_rel_rms": coef_rel_rms(pc2, ps2, c, s),
                    "note": "numpy (pageable) host arrays, wall clock, "
                            "median of 3 after one untimed call"}
    L.charm_shc_free(shc_pin)
    L.charm_shc_free(shc_pout)

    f32 = single_precision(L, err, pnt, N, c, s, d_f, stream, flush,
                           args.steps)
    bi8 = None if args.no_batch_i8 else batched_split_precision(
        L, err, pnt, N, dev, peak, args.steps)
    hi = None if args.no_n10800 else ultra_high_degree(L, err, dev, stream,
                                                        flush, peak)
    n360 = nmax360_round_trip()
    bdh = None if args.no_batch_dh else batch_dh(single_calls=False)
    sct = None if args.no_sctr else scattered(args.sctr_points, args.sctr_iters)
    cel = None if args.no_cells else cells()
    gfmr = None if args.no_gfm else gfm()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel ------------------------------
    # Algorithmic work of the reference algorithm per (n, m, latitude pair)
    # unit: synthesis 12 flops (recurrence 2 mul + 1 FMA, four FMA
    # accumulations), analysis 8 flops (recurrence, two FMA).  The kernels
    # execute fewer FP64 instructions per unit (rescaled recurrence 1 DMUL +
    # 1 DFMA, even/odd lumped sums 2 DFMA), reported as fp64_instr_per_unit.
    P_pairs = (nlat + 1) // 2
    units = T * P_pairs
    shs_ms = ms[0] / max(cnt[0], 1)
    sha_ms = ms[1] / max(cnt[1], 1)
    kern = {
        "shs_grid": {"ms": shs_ms, "flops_per_unit": 12.0,
                     "fp64_instr_per_unit": 4.0},
        "sha_grid": {"ms": sha_ms, "flops_per_unit": 8.0,
                     "fp64_instr_per_unit": 4.0},
    }
    for k in kern.values():
        k["achieved_tflops"] = units * k["flops_per_unit"] / (k["ms"] * 1e-3) / 1e12
        k["frac"] = k["achieved_tflops"] / peak if peak > 0 else None
        # FP64 pipe: one warp instruction per 2 cycles per scheduler, i.e.
        # peak/2 thread instructions per second
        k["fp64_pipe_frac"] = (units * k["fp64_instr_per_unit"] /
                               (k["ms"] * 1e-3) / (peak * 1e12 / 2.0)
                               if peak > 0 else None)
    dom = max(kern, key=lambda n: kern[n]["ms"])
    traffic = profiled_traffic(dom, N)
    step_s = total_ms / 1e3 / args.steps
    value = job_seconds_per_transform(total_ms / 1e3, args.steps, ws)
    h2d = 16 * T + 8 * nlat * nlon
    d2h = 8 * nlat * nlon + 16 * T
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_s * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (Kaula-decay coefficients, seed 2000)",
        "config": workload_config(N, nlat, nlon, ws),
        "round_trip_rel_rms": rt,
        "kernel_ms": {"shs_grid": shs_ms, "sha_grid": sha_ms,
                      "fft_total_per_step": ms[3] / args.steps,
                      "prep_total_per_step": ms[5] / args.steps},
        "roofline": {
            "bound": "fp64",
            "kernel": dom,
            "achieved": kern[dom]["achieved_tflops"],
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": kern[dom]["frac"],
            "peak_source": "measured live: FP64 FMA-chain probe "
                           "(charm_b200_fp64_peak_tflops) on this GPU; the "
                           "driver's peak file has no FP64 figure",
            "flops_per_unit": kern[dom]["flops_per_unit"],
            "units_per_launch": units,
            "traffic": traffic,
            "kernels": kern,
        },
        "e2e": {"value": job_seconds_per_transform(e2e_ms / 1e3, e2e_steps, ws),
                "unit": "s",
                "wall_s": wall / e2e_steps,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "round_trip_rel_rms": rt_e2e,
                "shs_call_ms": shs_call_ms, "sha_call_ms": sha_call_ms,
                "pinned_copy_gbs": copy_gbs,
                "copy_bound_ms": copy_bound_ms,
                "pageable": e2e_pageable},
        "gpu_launches": int(kl.value),
        "fft_execs": int(fe.value),
        "clocks": clk,
    }
    line["f32"] = f32
    if bi8 is not None:
        line["batch_i8"] = bi8
    # the synthesis autotuner's choices (tile of latitude pairs per lane)
    L.charm_b200_autotune_report.restype = ct.c_size_t
    L.charm_b200_autotune_report.argtypes = [ct.c_char_p, ct.c_size_t]
    rbuf = ct.create_string_buffer(8192)
    L.charm_b200_autotune_report(rbuf, 8192)
    line["autotune"] = rbuf.value.decode().splitlines()
    if hi is not None:
        line["nmax10800"] = hi
    line["nmax360"] = n360
    if bdh is not None:
        line["batch_dh"] = bdh
    if sct is not None:
        line["scattered"] = sct
    if cel is not None:
        line["cells"] = cel
    if gfmr is not None:
        line["gfm"] = gfmr
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(N, c, s)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU oracle (reference arm and cpu_baseline leg)
# ---------------------------------------------------------------------------
def single_precision(L, err, pnt, N, c, s, d_f64, stream, flush, steps):
    """The same round trip in the single-precision mode (FP32 Legendre
    recurrence and sums, FP64 row transforms, float inputs and outputs),
    device resident; its field is compared with the FP64 path's d_f64."""
    import torch
    from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, rel_rms
    P = ct.c_void_p
    L.charm_b200_shs_point_dev_f32.argtypes = [
        P, ct.c_ulong, ct.c_double, ct.c_double, P, P, ct.c_ulong, P, P]
    L.charm_b200_sha_point_dev_f32.argtypes = [
        P, P, ct.c_ulong, ct.c_double, ct.c_double, ct.c_ulong, P, P, P]
    dev = d_f64.device
    d_c = torch.from_numpy(c.astype(np.float32)).to(dev)
    d_s = torch.from_numpy(s.astype(np.float32)).to(dev)
    d_f = torch.empty(d_f64.numel(), dtype=torch.float32, device=dev)
    o_c = torch.empty_like(d_c)
    o_s = torch.empty_like(d_s)

    def check():
        if not L.charm_err_isempty(err):
            raise RuntimeError(ct.string_at(err.contents.msg).decode())

    def step():
        L.charm_b200_shs_point_dev_f32(ct.cast(pnt._Point, P), N, GM, R_EARTH,
                                       d_c.data_ptr(), d_s.data_ptr(), N,
                                       d_f.data_ptr(), ct.cast(err, P))
        check()
        L.charm_b200_sha_point_dev_f32(ct.cast(pnt._Point, P), d_f.data_ptr(),
                                       N, GM, R_EARTH, N, o_c.data_ptr(),
                                       o_s.data_ptr(), ct.cast(err, P))
        check()

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e_field = rel_rms(d_f.cpu().numpy().astype(np.float64),
                      d_f64.cpu().numpy())
    e_rt = coef_rel_rms(o_c.cpu().numpy().astype(np.float64),
                        o_s.cpu().numpy().astype(np.float64), c, s)
    L.charm_b200_timing(1)
    total = 0.0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        step()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    ms = (ct.c_double * 7)()
    cnt = (ct.c_ulonglong * 7)()
    L.charm_b200_timing_read(ms, cnt, 7, None, None)
    L.charm_b200_timing(0)
    return {"workload": "GL-grid SHS+SHA round trip, single-precision mode, "
                        "nmax %d" % N,
            "ms_per_round_trip": total / steps, "steps": steps,
            "kernel_ms": {"shs_grid_f32": ms[0] / max(cnt[0], 1),
                          "sha_grid_f32": ms[1] / max(cnt[1], 1),
                          "fft_total_per_step": ms[3] / steps},
            "field_rel_rms_vs_fp64": e_field,
            "round_trip_rel_rms": e_rt}


def batched_split_precision(L, err, pnt, N, dev, peak, steps, nsets=16):
    """Synthesis of nsets Kaula coefficient sets of degree N on the GL grid:
    the FP64 batched path (charm_b200_shs_point_batch_dev, the plain FP64
    kernels) against the split-precision one (..._batch_i8_dev: INT8 digit
    products on the tensor cores, FP64 recombination), same inputs, device
    resident.  Reports per-call and per-kernel times, sets/s, the largest
    per-set relative RMS difference, the INT8 tensor-core rate (ops per MMA
    as issued: 2 x 128 x 2176 x 32 per 64-degree chunk and latitude tile)
    and the FP64-equivalent rate (12 flops per (n, m, latitude pair) unit
    and set, as the synthesis roofline)."""
    import torch
    from charm_b200.workloads import GM, R_EARTH, kaula, rel_rms
    P = ct.c_void_p
    for f in (L.charm_b200_shs_point_batch_dev,
              L.charm_b200_shs_point_batch_i8_dev):
        f.argtypes = [P, ct.c_size_t, ct.POINTER(ct.c_ulong),
                      ct.POINTER(ct.c_ulong), ct.POINTER(ct.c_double),
                      ct.c_double, ct.POINTER(ct.c_void_p),
                      ct.POINTER(ct.c_void_p), ct.c_int,
                      ct.POINTER(ct.c_void_p), P]
    npts = pnt.lat.size * pnt.lon.size
    cs = [kaula(N, 6000 + j) for j in range(nsets)]
    dc = [torch.from_numpy(c).to(dev) for c, _ in cs]
    ds = [torch.from_numpy(s).to(dev) for _, s in cs]
    o64 = [torch.empty(npts, dtype=torch.float64, device=dev)
           for _ in range(nsets)]
    o8 = [torch.empty(npts, dtype=torch.float64, device=dev)
          for _ in range(nsets)]
    nm = (ct.c_ulong * nsets)(*([N] * nsets))
    mu = (ct.c_double * nsets)(*([GM] * nsets))
    pc = (ct.c_void_p * nsets)(*[t.data_ptr() for t in dc])
    ps = (ct.c_void_p * nsets)(*[t.data_ptr() for t in ds])

    def run(fn, outs):
        pf = (ct.c_void_p * nsets)(*[t.data_ptr() for t in outs])
        fn(ct.cast(pnt._Point, P), nsets, nm, nm, mu, R_EARTH, pc, ps, 0, pf,
           ct.cast(err, P))
        if not L.charm_err_isempty(err):
            raise RuntimeError(ct.string_at(err.contents.msg).decode())

    res = {}
    for name, fn, outs in (("fp64", L.charm_b200_shs_point_batch_dev, o64),
                           ("i8", L.charm_b200_shs_point_batch_i8_dev, o8)):
        run(fn, outs)               # tables, buffers
        torch.cuda.synchronize()
        L.charm_b200_timing(1)
        t0 = time.perf_counter()
        for _ in range(steps):
            run(fn, outs)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) / steps
        ms = (ct.c_double * 7)()
        cnt = (ct.c_ulonglong * 7)()
        L.charm_b200_timing_read(ms, cnt, 7, None, None)
        L.charm_b200_timing(0)
        res[name] = {"s_per_batch": wall, "sets_per_s": nsets / wall,
                     "legendre_kernel_ms": ms[0] / steps,
                     "row_transforms_ms": ms[3] / steps,
                     "prep_ms": ms[5] / steps}
    worst = max(rel_rms(a.cpu().numpy(), b.cpu().numpy())
                for a, b in zip(o8, o64))
    np_ = (pnt.lat.size + 1) // 2
    ntiles = (np_ + 127) // 128
    chunks = sum((N - m + 64) // 64 for m in range(N + 1))
    int8_ops = 2.0 * 128 * 2176 * 32 * chunks * ntiles
    units = (N + 1) * (N + 2) / 2 * np_ * nsets
    k8 = res["i8"]["legendre_kernel_ms"] * 1e-3
    k64 = res["fp64"]["legendre_kernel_ms"] * 1e-3
    out = {
        "workload": "%d Kaula sets of nmax %d, potential on the GL grid "
                    "(%d x %d), r = R" % (nsets, N, pnt.lat.size,
                                          pnt.lon.size),
        "fp64_batch": res["fp64"], "i8_batch": res["i8"],
        "speedup_sets_per_s": res["fp64"]["s_per_batch"] /
        res["i8"]["s_per_batch"],
        "speedup_legendre_kernel": k64 / k8,
        "max_set_rel_rms_vs_fp64": worst,
        "tensor_int8_tops": int8_ops / k8 / 1e12,
        "tensor_int8_frac_of_nominal_4500": int8_ops / k8 / 1e12 / 4500.0,
        "fp64_equivalent_tflops": units * 12.0 / k8 / 1e12,
        "fp64_equivalent_frac_of_fp64_peak": (units * 12.0 / k8 / 1e12 / peak
                                              if peak > 0 else None),
    }
    del dc, ds, o64, o8
    torch.cuda.empty_cache()
    return out


def ultra_high_degree(L, err, dev, stream, flush, peak, steps=2):
    """The nmax 10800 GL round trip (10801 x 21602 grid, Kaula decay
    1e-5 n^-2, seed 3000), device resident: one untimed round trip, then
    `steps` timed ones (CUDA events on the library stream, L2 flushed
    between them).  Returns its summary for the JSON line."""
    import torch
    import charm_b200 as cb
    from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula
    N = 10800
    c, s = kaula(N, 3000, sqrt_scaling=False)
    pnt = cb.PointGridGL(N, R_EARTH)
    nlat, nlon = pnt.lat.size, pnt.lon.size
    d_c = torch.from_numpy(c).to(dev)
    d_s = torch.from_numpy(s).to(dev)
    d_f = torch.empty(nlat * nlon, dtype=torch.float64, device=dev)
    o_c = torch.empty_like(d_c)
    o_s = torch.empty_like(d_s)

    def check():
        if not L.charm_err_isempty(err):
            raise RuntimeError(ct.string_at(err.contents.msg).decode())

    def step():
        L.charm_b200_shs_point_dev(ct.cast(pnt._Point, ct.c_void_p), N, GM,
                                   R_EARTH, d_c.data_ptr(), d_s.data_ptr(), N,
                                   0, 0, 0, 0, d_f.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        check()
        L.charm_b200_sha_point_dev(ct.cast(pnt._Point, ct.c_void_p),
                                   d_f.data_ptr(), N, GM, R_EARTH, N,
                                   o_c.data_ptr(), o_s.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        check()

    step()
    torch.cuda.synchronize()
    rt = coef_rel_rms(o_c.cpu().numpy(), o_s.cpu().numpy(), c, s)
    L.charm_b200_timing(1)
    total = 0.0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        step()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    ms = (ct.c_double * 7)()
    cnt = (ct.c_ulonglong * 7)()
    L.charm_b200_timing_read(ms, cnt, 7, None, None)
    L.charm_b200_timing(0)
    T = c.size
    units = T * ((nlat + 1) // 2)
    shs = ms[0] / max(cnt[0], 1)
    sha = ms[1] / max(cnt[1], 1)
    leg_tflops = units * 20.0 / ((shs + sha) * 1e-3) / 1e12
    del d_c, d_s, d_f, o_c, o_s
    torch.cuda.empty_cache()
    return {"workload": "GL-grid SHS+SHA round trip, plain FP64, nmax 10800, "
                        "grid %dx%d, Kaula 1e-5 n^-2 (seed 3000)" % (nlat, nlon),
            "ms_per_round_trip": total / steps, "steps": steps,
            "round_trip_rel_rms": rt,
            "kernel_ms": {"shs_grid": shs, "sha_grid": sha,
                          "fft_total_per_step": ms[3] / steps},
            "legendre_tflops": leg_tflops,
            "legendre_frac_of_fp64_peak": leg_tflops / peak if peak > 0 else None}


def profiled_traffic(kernel, N):
    """DRAM bytes (read + write) per launch of `kernel` at this nmax from
    the committed ncu summary profiles/<kernel>_gl<N>.md (its line
    'traffic_bytes_per_launch: B'), or None."""
    path = os.path.join(ROOT, "profiles", "k_%s_gl%d.md" % (kernel, N))
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def host_cores():
    """Host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def workload_config(N, nlat, nlon, ws):
    """The config object of the round-trip workload, shared by both arms."""
    from charm_b200.workloads import GM, R_EARTH
    return {
        "workload": "GL-grid SHS+SHA round trip, plain FP64",
        "nmax": N, "grid": "%dx%d" % (nlat, nlon), "r": "R",
        "GM": GM, "R": R_EARTH,
        "coefficients": "Kaula 1e-5 n^-2 / sqrt(2n+1), seed 2000",
        "l2": "flushed between GPU steps (256 MiB write outside the timed "
              "events); the grid (76.8 MB) and triangles exceed the host "
              "caches",
        "parallelism": "replicas" if ws > 1 else "single device",
    }


def charm_round_trips(N, c, s, steps, warmup, fft_share=True):
    """Times CHarm 0.4.9 itself -- charm_shs_point then charm_sha_point of
    the double-precision build in oracle/_ref (its own sources compiled with
    OpenMP and AVX-512, or AVX2 where the host lacks AVX-512, -O3
    -ffast-math), on the full GL grid of degree N at r = R, `warmup`
    untimed and `steps` timed round trips, wall clock, all host threads.
    Also times, once, the row FFTs CHarm makes in a round trip through the
    same library's FFTW-API shim (analysis: one r2c per row in one thread,
    as sha_point.c runs them; synthesis: one c2r per row, spread over the
    threads by CHarm), so that the shim's share can be read off."""
    cores = host_cores()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    from charm_b200.workloads import GM, R_EARTH, coef_rel_rms
    from oracle import charm_ref
    C = charm_ref.Charm("d")
    pnt, lat, lon, w = C.grid(charm_ref.GL, N, R_EARTH)
    shc = C.shc(N, GM, R_EARTH, c, s)
    npt = lat.size * lon.size
    shs_t, sha_t = [], []
    c2 = s2 = None
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        f = C.shs_point(pnt, shc, N, npt)
        t1 = time.perf_counter()
        c2, s2 = C.sha_point(pnt, f, N, GM, R_EARTH)
        t2 = time.perf_counter()
        if i >= warmup:
            shs_t.append(t1 - t0)
            sha_t.append(t2 - t1)
    rt = coef_rel_rms(c2, s2, c, s)
    out = {"cores": cores, "lib": os.path.relpath(C.path, ROOT),
           "avx512": charm_ref.cpu_has_avx512(),
           "shs_s": float(np.mean(shs_t)), "sha_s": float(np.mean(sha_t)),
           "round_trip_s": [a + b for a, b in zip(shs_t, sha_t)],
           "round_trip_rel_rms": rt}
    if fft_share:
        L = C.L
        vp = ct.c_void_p
        for nm_, at in (("fftw_plan_dft_r2c_1d", [ct.c_int, vp, vp, ct.c_uint]),
                        ("fftw_plan_dft_c2r_1d", [ct.c_int, vp, vp, ct.c_uint])):
            getattr(L, nm_).argtypes = at
            getattr(L, nm_).restype = vp
        for nm_ in ("fftw_execute_dft_r2c", "fftw_execute_dft_c2r"):
            getattr(L, nm_).argtypes = [vp, vp, vp]
            getattr(L, nm_).restype = None
        L.fftw_destroy_plan.argtypes = [vp]
        nlon = lon.size
        x = np.random.default_rng(0).standard_normal(nlon)
        X = np.zeros(nlon // 2 + 1, np.complex128)
        pr = L.fftw_plan_dft_r2c_1d(nlon, None, None, 1 << 6)
        pc = L.fftw_plan_dft_c2r_1d(nlon, None, None, 1 << 6)
        t0 = time.perf_counter()
        for _ in range(lat.size):
            L.fftw_execute_dft_r2c(pr, x.ctypes.data, X.ctypes.data)
        t_r2c = time.perf_counter() - t0
        t0 = time.perf_counter()
        for _ in range(lat.size):
            L.fftw_execute_dft_c2r(pc, X.ctypes.data, x.ctypes.data)
        t_c2r = time.perf_counter() - t0
        L.fftw_destroy_plan(pr)
        L.fftw_destroy_plan(pc)
        out["fft_shim_s"] = {"sha_r2c_serial": t_r2c,
                             "shs_c2r_one_thread": t_c2r,
                             "shs_c2r_spread_over_threads": t_c2r / cores}
    return out


def cpu_baseline(N, c, s):
    """The cpu_baseline object: CHarm itself on the same round trip (one
    warm-up, three timed round trips, their median)."""
    r = charm_round_trips(N, c, s, steps=3, warmup=1)
    v = float(np.median(r["round_trip_s"]))
    return {"value": v, "unit": "s", "cores": r["cores"], "kind": "reference",
            "sample": "the full round trip (nmax %d GL grid), 1 warm-up + 3 "
                      "timed, median" % N,
            "detail": r}


def run_reference(args):
    """The reference arm: CHarm 0.4.9 (oracle/_ref) on the host cores,
    every step the full round trip of the GPU arm's workload.  Under
    torchrun only rank 0 runs and prints; the others exit."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from charm_b200.workloads import kaula
    N = args.nmax
    c, s = kaula(N, 2000)
    r = charm_round_trips(N, c, s, steps=args.steps, warmup=args.warmup)
    v = float(np.mean(r["round_trip_s"]))
    line = {
        "impl": "reference",
        "metric": METRIC, "value": v, "unit": "s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (Kaula-decay coefficients, seed 2000)",
        "config": workload_config(N, N + 1, 2 * (N + 1), ws),
        "round_trip_rel_rms": r["round_trip_rel_rms"],
        "cpu_baseline": {"value": v, "unit": "s", "cores": r["cores"],
                         "kind": "reference",
                         "sample": "every step the full round trip: "
                                   "charm_shs_point + charm_sha_point of "
                                   "CHarm 0.4.9 (%s), wall clock" % r["lib"]},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference": r,
    }
    print(json.dumps(line), flush=True)


def scattered(npt=10_000_000, cg_iters=20):
    """Scattered points: nmax 2160 Kaula coefficients (seed 5000), `npt`
    points uniform on the sphere with heights 0-9000 m (seed 5001),
    observations A c + N(0, (1e-3 rms)^2) (seed 5002); times one synthesis,
    one adjoint (with its dot-product identity <A c, y> = <c, A^T y>) and a
    CGLS fit from zero of `cg_iters` iterations, and reports the fit's
    misfit and coefficient error.  Returns a dict."""
    import torch
    import charm_b200 as cb
    from charm_b200 import autograd as ag
    from charm_b200.workloads import GM, R_EARTH, kaula
    N = 2160
    rng = np.random.default_rng(5001)
    lat = np.arcsin(rng.uniform(-1.0, 1.0, npt))
    lon = rng.uniform(0.0, 2.0 * np.pi, npt)
    r = R_EARTH + rng.uniform(0.0, 9000.0, npt)
    p = cb.PointSctr(lat, lon, r)
    c, s = kaula(N, 5000)
    dc = torch.from_numpy(c).cuda()
    ds = torch.from_numpy(s).cuda()

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    ag._synthesis(dc, ds, p, N, GM, R_EARTH)    # tables, buffers
    truth, t_fwd = timed(lambda: ag._synthesis(dc, ds, p, N, GM, R_EARTH))
    rms = float(torch.sqrt(torch.mean(truth * truth)))
    noise = np.random.default_rng(5002).standard_normal(npt) * (1e-3 * rms)
    obs = truth + torch.from_numpy(noise).cuda()
    (gc, gs), t_adj = timed(lambda: ag._adjoint(obs, p, N, GM, R_EARTH))
    lhs = float(torch.dot(truth, obs))
    rhs = float(torch.dot(dc, gc) + torch.dot(ds, gs))
    out = {
        "workload": "scattered synthesis + adjoint + CGLS, nmax %d, %d points "
                    "(heights 0-9000 m), %d iterations" % (N, npt, cg_iters),
        "forward_s": t_fwd, "adjoint_s": t_adj,
        "forward_tflops_alg": c.size * npt * 8.0 / t_fwd / 1e12,
        "adjoint_tflops_alg": c.size * npt * 8.0 / t_adj / 1e12,
        "flops_per_unit": "8 per (n, m, point): recurrence 2 mul + 1 FMA, "
                          "two FMA (src/shs/shs_point_sctr.c)",
        "dot_product_rel": abs(lhs - rhs) / abs(lhs),
        "dtype": "f64", "data": "synthetic (seeds 5000, 5001, 5002)",
    }
    if cg_iters > 0:
        (xc, xs, hist), t_cg = timed(
            lambda: ag.cgls(p, obs, N, GM, R_EARTH, iters=cg_iters))
        num = torch.linalg.norm(torch.cat([xc - dc, xs - ds]))
        den = torch.linalg.norm(torch.cat([dc, ds]))
        out.update({"cgls_s": t_cg,
                    "misfit_first_last": [hist[0], hist[-1]],
                    "noise_norm": float(np.linalg.norm(noise)),
                    "coef_rel_error": float(num / den)})
    return out


def run_sctr_cg(args):
    """The scattered workload alone; prints one JSON line.  One GPU."""
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(scattered(args.npoint, args.cg_iters)), flush=True)


def nmax360_round_trip(steps=10):
    """The nmax 360 GL round trip (361 x 722 grid, seed 1000): device time
    per round trip through the device entry points and CHarm's own time on
    the host cores for the same round trip."""
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula
    N = 360
    c, s = kaula(N, 1000)
    pnt = cb.PointGridGL(N, R_EARTH)
    dev = torch.device("cuda", torch.cuda.current_device())
    d_c = torch.from_numpy(c).to(dev)
    d_s = torch.from_numpy(s).to(dev)
    d_f = torch.empty(pnt.lat.size * pnt.lon.size, dtype=torch.float64,
                      device=dev)
    o_c = torch.empty_like(d_c)
    o_s = torch.empty_like(d_s)
    err = L.charm_err_init()
    stream = torch.cuda.ExternalStream(L.charm_b200_stream())

    def step():
        L.charm_b200_shs_point_dev(ct.cast(pnt._Point, ct.c_void_p), N, GM,
                                   R_EARTH, d_c.data_ptr(), d_s.data_ptr(), N,
                                   0, 0, 0, 0, d_f.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        L.charm_b200_sha_point_dev(ct.cast(pnt._Point, ct.c_void_p),
                                   d_f.data_ptr(), N, GM, R_EARTH, N,
                                   o_c.data_ptr(), o_s.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        if not L.charm_err_isempty(err):
            raise RuntimeError(ct.string_at(err.contents.msg).decode())

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    for _ in range(steps):
        step()
    with torch.cuda.stream(stream):
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    rt = coef_rel_rms(o_c.cpu().numpy(), o_s.cpu().numpy(), c, s)
    L.charm_err_free(err)
    out = {"workload": "GL-grid SHS+SHA round trip, plain FP64, nmax 360, "
                       "grid 361x722 (seed 1000)",
           "ms_per_round_trip": ms, "steps": steps,
           "round_trip_rel_rms": rt}
    try:
        r = charm_round_trips(N, c, s, steps=5, warmup=1, fft_share=False)
        out["charm_cpu_ms_per_round_trip"] = 1e3 * float(
            np.median(r["round_trip_s"]))
        out["charm_cpu_cores"] = r["cores"]
    except (OSError, RuntimeError) as e:
        out["charm_cpu"] = "unavailable: %s" % e
    return out


def cells(steps=5, oracle_rows=3):
    """Block means on the whole-sphere grid of 2191 x 4382 cells at nmax
    2190 (the cells of the GL round trip's resolution, r = R, Kaula seed
    2000): cell synthesis and approximate-quadrature analysis through the
    device entry points, per-kernel times, FP64 pipe fractions, the
    synthesis against the oracle on a few rows, and CHarm's own time and
    coefficients for the same calls on the host cores."""
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms
    from oracle import charm_ref, orc
    N = 2190
    nlat, nlon = N + 1, 2 * (N + 1)
    lat_e = np.linspace(np.pi / 2, -np.pi / 2, nlat + 1)
    lat_e[0], lat_e[-1] = np.pi / 2, -np.pi / 2
    lon_e = np.arange(nlon + 1) * (2.0 * np.pi / nlon)
    args = (lat_e[1:], lat_e[:-1], lon_e[:-1], lon_e[1:], np.full(nlat, R_EARTH))
    cl = cb.CellGrid(*args)
    c, s = kaula(N, 2000)
    T = c.size
    dev = torch.device("cuda", torch.cuda.current_device())
    d_c = torch.from_numpy(c).to(dev)
    d_s = torch.from_numpy(s).to(dev)
    d_f = torch.empty(nlat * nlon, dtype=torch.float64, device=dev)
    o_c = torch.empty_like(d_c)
    o_s = torch.empty_like(d_s)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    P = ct.c_void_p
    L.charm_b200_shs_cell_dev.argtypes = [P, ct.c_ulong, ct.c_double,
                                          ct.c_double, P, P, ct.c_ulong, P, P]
    L.charm_b200_sha_cell_dev.argtypes = [P, P, ct.c_ulong, ct.c_double,
                                          ct.c_double, ct.c_ulong, P, P, P]
    L.charm_b200_stream.restype = ct.c_void_p
    L.charm_b200_timing.argtypes = [ct.c_int]
    L.charm_b200_timing_read.argtypes = [
        ct.POINTER(ct.c_double), ct.POINTER(ct.c_ulonglong), ct.c_int,
        ct.POINTER(ct.c_ulonglong), ct.POINTER(ct.c_ulonglong)]
    L.charm_b200_fp64_peak_tflops.restype = ct.c_double
    err = L.charm_err_init()
    stream = torch.cuda.ExternalStream(L.charm_b200_stream())

    def check():
        if not L.charm_err_isempty(err):
            raise RuntimeError(ct.string_at(err.contents.msg).decode())

    def shs():
        L.charm_b200_shs_cell_dev(ct.cast(cl._Cell, P), N, GM, R_EARTH,
                                  d_c.data_ptr(), d_s.data_ptr(), N,
                                  d_f.data_ptr(), ct.cast(err, P))
        check()

    def sha():
        L.charm_b200_sha_cell_dev(ct.cast(cl._Cell, P), d_f.data_ptr(), N, GM,
                                  R_EARTH, N, o_c.data_ptr(), o_s.data_ptr(),
                                  ct.cast(err, P))
        check()

    for _ in range(2):
        shs()
        sha()
    torch.cuda.synchronize()
    res = {}
    for name, fn in (("shs_cell", shs), ("sha_cell", sha)):
        L.charm_b200_timing(1)
        tot = 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            fn()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        ms = (ct.c_double * 7)()
        cnt = (ct.c_ulonglong * 7)()
        kl = ct.c_ulonglong()
        fe = ct.c_ulonglong()
        L.charm_b200_timing_read(ms, cnt, 7, ct.byref(kl), ct.byref(fe))
        L.charm_b200_timing(0)
        res[name] = {"ms_per_call": tot / steps,
                     "legendre_ms": (ms[0] + ms[1]) / steps,
                     "fft_ms": ms[3] / steps,
                     "prep_ms": ms[5] / steps}
    f = d_f.cpu().numpy().reshape(nlat, nlon)
    cg, sg = o_c.cpu().numpy(), o_s.cpu().numpy()
    L.charm_err_free(err)
    peak = L.charm_b200_fp64_peak_tflops()
    units = T * ((nlat + 1) // 2)
    # FP64 instructions per (n, m, cell-row pair) as ncu counts them at
    # nmax 2190: the boundary recurrences (DMUL + DFMA each; two adjacent
    # rows share one), the integral (2 DMUL + 2 DFMA; h_n beta_n comes
    # staged) and two DFMA sums; the analysis adds the reduction of the
    # lane sums
    for name, ipu in (("shs_cell", 9.2), ("sha_cell", 10.4)):
        k = res[name]
        k["fp64_instr_per_unit"] = ipu
        k["fp64_pipe_frac"] = (units * ipu / (k["legendre_ms"] * 1e-3) /
                               (peak * 1e12 / 2.0)) if peak > 0 else None
    # the synthesis against the oracle on a few rows (a grid of those rows)
    rows = np.linspace(0, nlat - 1, oracle_rows).astype(int)
    sub = (args[0][rows], args[1][rows], args[2], args[3], args[4][rows])
    fo = orc.shs_cell(orc.Cell(orc.CELL_GRID, *sub), orc.Shc(N, GM, R_EARTH, c, s),
                      N).reshape(rows.size, nlon)
    f00 = GM / R_EARTH
    out = {"workload": "block means on 2191 x 4382 whole-sphere cells, "
                       "nmax 2190, r = R, Kaula seed 2000",
           "steps": steps, "units_n_m_pair": units,
           "shs_cell": res["shs_cell"], "sha_cell": res["sha_cell"],
           "shs_rel_rms_vs_oracle_rows": rel_rms(f[rows], fo),
           "shs_signal_rel_rms_vs_oracle_rows": rel_rms(f[rows] - f00, fo - f00),
           "oracle_rows": [int(r) for r in rows],
           "aq_round_trip_rel_rms_vs_truth": coef_rel_rms(cg, sg, c, s),
           "dtype": "f64", "data": "synthetic (seed 2000)"}
    try:
        C = charm_ref.Charm("d")
        cc = C.cell(orc.CELL_GRID, *args)
        shc = C.shc(N, GM, R_EARTH, c, s)
        t0 = time.perf_counter()
        fr = C.shs_cell(cc, shc, N, nlat * nlon)
        t1 = time.perf_counter()
        cr, sr = C.sha_cell(cc, np.ravel(f), N, GM, R_EARTH)
        t2 = time.perf_counter()
        out["charm_cpu"] = {"shs_cell_s": t1 - t0, "sha_cell_s": t2 - t1,
                            "cores": host_cores(), "lib": os.path.relpath(
                                charm_ref.lib_path("d"), ROOT)}
        out["shs_rel_rms_vs_charm"] = rel_rms(np.ravel(f), fr)
        out["sha_rel_rms_vs_charm"] = coef_rel_rms(cg, sg, cr, sr)
    except (OSError, RuntimeError) as e:
        out["charm_cpu"] = "unavailable: %s" % e
    return out


def gfm(steps=2):
    """Global spectral gravity forward modelling of a synthetic body:
    shape of degree 360 (lunar radius, Kaula-like relief), a density
    polynomial of order 1 (coefficients of degree 180 and 90), topography
    powers 1..5, potential to degree 720 (Gauss--Legendre grids up to nmax
    1980).  GPU time per call (wall clock, the call returns after its
    streams are idle), the potential's agreement with CHarm's own
    charm_gfm_global_density_3d, and CHarm's time on the host cores."""
    import torch
    import charm_b200 as cb
    from charm_b200.workloads import coef_rel_rms
    from oracle import charm_ref
    R = 1728000.0
    G, M = 6.67430e-11, 7.346e22

    def body(nmax, seed, relief, c00):
        rng = np.random.default_rng(seed)
        T = (nmax + 1) * (nmax + 2) // 2
        n = np.concatenate([np.arange(m, nmax + 1) for m in range(nmax + 1)])
        sig = relief / (1.0 + n) ** 2
        c = rng.standard_normal(T) * sig
        s = rng.standard_normal(T) * sig
        s[:nmax + 1] = 0.0
        c[0] = c00
        return c, s
    shape = body(360, 61, 3000.0, R + 1700.0)
    dens = [body(180, 62, 80.0, 2500.0), body(90, 63, 1e-6, -2e-5)]
    args_s = (360, 1.0, 1.0) + shape
    sh = cb.Shc(*args_s)
    ds = [cb.Shc(180, 1.0, 1.0, *dens[0]), cb.Shc(90, 1.0, 1.0, *dens[1])]

    def call():
        return cb.gfm_global_density_3d(sh, 360, R, ds, [180, 90], 1, G, M, 1,
                                        5, 720)
    pot = call()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        pot = call()
        ts.append(time.perf_counter() - t0)
    out = {"workload": "global gravity forward modelling: shape nmax 360, "
                       "density order 1 (nmax 180, 90), powers 1..5, "
                       "potential nmax 720 (GL grids up to nmax 1980)",
           "gpu_s": float(np.median(ts)), "steps": steps,
           "data": "synthetic (seeds 61-63)"}
    try:
        C = charm_ref.Charm("d")
        P = ct.POINTER
        fn = C.fn("gfm_global_density_3d")
        fn.argtypes = [P(C.Shc), ct.c_ulong, ct.c_double, P(P(C.Shc)),
                       P(ct.c_ulong), ct.c_uint, ct.c_double, ct.c_double,
                       ct.c_uint, ct.c_uint, ct.c_ulong, ct.c_char_p,
                       ct.c_char_p, ct.c_char_p, P(C.Shc), P(C.Err)]
        fn.restype = None
        csh = C.shc(*args_s)
        cds = [C.shc(180, 1.0, 1.0, *dens[0]), C.shc(90, 1.0, 1.0, *dens[1])]
        arr = (P(C.Shc) * 2)(*[d.ptr for d in cds])
        nm = (ct.c_ulong * 2)(180, 90)
        T = 721 * 722 // 2
        cpot = C.shc(720, 1.0, 1.0, np.zeros(T), np.zeros(T))
        t0 = time.perf_counter()
        fn(csh.ptr, 360, R, arr, nm, 1, G, M, 1, 5, 720, None, None, None,
           cpot.ptr, C.err)
        t1 = time.perf_counter()
        C.check()
        out["charm_cpu"] = {"s": t1 - t0, "cores": host_cores(),
                            "lib": os.path.relpath(charm_ref.lib_path("d"),
                                                   ROOT)}
        out["potential_rel_rms_vs_charm"] = coef_rel_rms(
            pot.c, pot.s, cpot.keep[0], cpot.keep[1])
    except (OSError, RuntimeError, AttributeError) as e:
        out["charm_cpu"] = "unavailable: %s" % e
    return out


def batch_dh(single_calls=True, oracle_rows=6):
    """64 coefficient sets, nmax_j uniform in 90..2160 (numpy default_rng
    4999), Kaula coefficients (seeds 4000 + j), synthesised at r = R + 250 km
    with the potential, grad1 and grad2 (ten quantities): even sets on the
    DH1 grid and odd sets on the DH2 grid of their largest degree.  Times
    the batched FP64 entry point (groups of 8 sets per call, bounded by the
    output memory), optionally one call per set and derivative kind, and the
    potential of all 64 sets through the FP64 batch and the split-precision
    batch (tensor cores).  Errors per component: the batched FP64 output of
    the lowest-degree set of each grid against the CPU oracle on
    `oracle_rows` of its rows, and the split-precision potential against the
    FP64 batch (all sets) and the oracle (those rows).  Returns a dict."""
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    from charm_b200.workloads import GM, R_EARTH, kaula, rel_rms
    from oracle import orc
    P = ct.c_void_p
    L.charm_b200_shs_point_batch_dev.argtypes = [
        P, ct.c_size_t, ct.POINTER(ct.c_ulong), ct.POINTER(ct.c_ulong),
        ct.POINTER(ct.c_double), ct.c_double, ct.POINTER(ct.c_void_p),
        ct.POINTER(ct.c_void_p), ct.c_int, ct.POINTER(ct.c_void_p), P]
    L.charm_b200_shs_point_batch_i8_dev.argtypes = \
        L.charm_b200_shs_point_batch_dev.argtypes
    L.charm_b200_shs_point_dev.argtypes = [
        P, ct.c_ulong, ct.c_double, ct.c_double, P, P, ct.c_ulong, ct.c_int,
        ct.c_uint, ct.c_uint, ct.c_uint, P, P]
    nm = np.random.default_rng(4999).integers(90, 2161, size=64)
    err = L.charm_err_init()

    def check():
        if not L.charm_err_isempty(err):
            raise RuntimeError(ct.string_at(err.contents.msg).decode())

    # where the batched calls' time goes: one more call of each with the
    # library's per-kernel event timing (not part of the timed calls)
    L.charm_b200_timing.argtypes = [ct.c_int]
    L.charm_b200_timing_read.argtypes = [
        ct.POINTER(ct.c_double), ct.POINTER(ct.c_ulonglong), ct.c_int,
        ct.POINTER(ct.c_ulonglong), ct.POINTER(ct.c_ulonglong)]
    split_ms = {"fp64": [0.0] * 7, "split": [0.0] * 7}

    def kernel_times(kind, call):
        L.charm_b200_timing(1)
        call()
        torch.cuda.synchronize()
        ms_ = (ct.c_double * 7)()
        cnt_ = (ct.c_ulonglong * 7)()
        kl_, fe_ = ct.c_ulonglong(), ct.c_ulonglong()
        L.charm_b200_timing_read(ms_, cnt_, 7, ct.byref(kl_), ct.byref(fe_))
        L.charm_b200_timing(0)
        for i_ in range(7):
            split_ms[kind][i_] += ms_[i_]

    h = 250e3
    names = ["V", "Vx", "Vy", "Vz", "Vxx", "Vxy", "Vxz", "Vyy", "Vyz", "Vzz"]
    groups = []
    for parity, ctor in ((0, cb.PointGridDH1), (1, cb.PointGridDH2)):
        idx = [j for j in range(64) if j % 2 == parity]
        Ng = int(max(nm[j] for j in idx))
        groups.append((ctor(Ng, R_EARTH + h), idx))
    coefs = {j: kaula(int(nm[j]), 4000 + j) for j in range(64)}
    total_units = 0.0
    t_batch = 0.0
    t_single = 0.0
    G = 8
    probe = {}     # set -> (grid, rows, [10 x (rows, nlon)]) of the FP64 batch
    probe8 = {}    # the same of the split-precision batch
    worst8 = {}    # component -> largest relative RMS split vs FP64
    t_batch8 = 0.0
    for pnt, idx in groups:
        npts = pnt.lat.size * pnt.lon.size
        jmin = min(idx, key=lambda j: nm[j])
        rows = np.linspace(1, pnt.lat.size - 2, oracle_rows).astype(int)
        for g0 in range(0, len(idx), G):
            sel = idx[g0:g0 + G]
            n = len(sel)
            dc = [torch.from_numpy(coefs[j][0]).cuda() for j in sel]
            ds = [torch.from_numpy(coefs[j][1]).cuda() for j in sel]
            out = [torch.empty(10 * npts, dtype=torch.float64, device="cuda")
                   for _ in sel]
            nmv = (ct.c_ulong * n)(*[int(nm[j]) for j in sel])
            muv = (ct.c_double * n)(*([GM] * n))
            pc = (ct.c_void_p * n)(*[t.data_ptr() for t in dc])
            ps = (ct.c_void_p * n)(*[t.data_ptr() for t in ds])
            pf = (ct.c_void_p * n)(*[t.data_ptr() for t in out])
            for rep in range(2):   # first call warms tables and buffers
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                L.charm_b200_shs_point_batch_dev(ct.cast(pnt._Point, P), n,
                                                 nmv, nmv, muv, R_EARTH, pc,
                                                 ps, 3, pf, ct.cast(err, P))
                check()
                torch.cuda.synchronize()
                if rep == 1:
                    t_batch += time.perf_counter() - t0
            kernel_times("fp64", lambda: (L.charm_b200_shs_point_batch_dev(
                ct.cast(pnt._Point, P), n, nmv, nmv, muv, R_EARTH, pc, ps, 3,
                pf, ct.cast(err, P)), check()))
            if jmin in sel:
                o = out[sel.index(jmin)].view(10, pnt.lat.size, pnt.lon.size)
                probe[jmin] = (pnt, rows, o[:, rows, :].cpu().numpy())
            # the same ten quantities with the degree sums on the tensor
            # cores (split precision, 3 sets per launch), compared per
            # component off the poles (x / y components are singular there)
            out8 = [torch.empty(10 * npts, dtype=torch.float64, device="cuda")
                    for _ in sel]
            pf8 = (ct.c_void_p * n)(*[t.data_ptr() for t in out8])
            for rep in range(2):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                L.charm_b200_shs_point_batch_i8_dev(
                    ct.cast(pnt._Point, P), n, nmv, nmv, muv, R_EARTH, pc, ps,
                    3, pf8, ct.cast(err, P))
                check()
                torch.cuda.synchronize()
                if rep == 1:
                    t_batch8 += time.perf_counter() - t0
            kernel_times("split", lambda: (L.charm_b200_shs_point_batch_i8_dev(
                ct.cast(pnt._Point, P), n, nmv, nmv, muv, R_EARTH, pc, ps, 3,
                pf8, ct.cast(err, P)), check()))
            keep = torch.from_numpy(np.cos(pnt.lat) > 1e-8).cuda()
            for b in range(n):
                a8 = out8[b].view(10, pnt.lat.size, pnt.lon.size)
                a64 = out[b].view(10, pnt.lat.size, pnt.lon.size)
                for q, nm_ in enumerate(names):
                    d = (a8[q][keep] - a64[q][keep]).double()
                    r_ = a64[q][keep].double()
                    e = float(torch.sqrt(torch.mean(d * d)) /
                              torch.sqrt(torch.mean(r_ * r_)))
                    worst8[nm_] = max(worst8.get(nm_, 0.0), e)
            if jmin in sel:
                o8 = out8[sel.index(jmin)].view(10, pnt.lat.size, pnt.lon.size)
                probe8[jmin] = o8[:, rows, :].cpu().numpy()
            del out8
            if single_calls:
                # one call per set and kind (potential, grad1, grad2); the
                # first pass, untimed, takes each shape's one-time costs
                # (tables, the synthesis autotuner), as the batched call's
                # warm-up does
                for rep in range(2):
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    for b, j in enumerate(sel):
                        for kg, d, off in ((0, 0, 0), (1, 1, 1), (2, 2, 4)):
                            L.charm_b200_shs_point_dev(
                                ct.cast(pnt._Point, P), int(nm[j]), GM,
                                R_EARTH, dc[b].data_ptr(), ds[b].data_ptr(),
                                int(nm[j]), kg, d, d, d,
                                out[b].data_ptr() + off * npts * 8,
                                ct.cast(err, P))
                            check()
                    torch.cuda.synchronize()
                    if rep == 1:
                        t_single += time.perf_counter() - t0
            for j in sel:
                T = (int(nm[j]) + 1) * (int(nm[j]) + 2) / 2
                total_units += T * (pnt.lat.size // 2 + 1)
            del dc, ds, out
            torch.cuda.empty_cache()
    # the potential of the same 64 sets: FP64 batch against the
    # split-precision batch (tensor cores), each parity group in one call
    pot = {"fp64_s": 0.0, "i8_s": 0.0, "worst_rel_rms_vs_fp64": 0.0}
    i8_probe = {}
    for pnt, idx in groups:
        npts = pnt.lat.size * pnt.lon.size
        n = len(idx)
        dc = [torch.from_numpy(coefs[j][0]).cuda() for j in idx]
        ds = [torch.from_numpy(coefs[j][1]).cuda() for j in idx]
        nmv = (ct.c_ulong * n)(*[int(nm[j]) for j in idx])
        muv = (ct.c_double * n)(*([GM] * n))
        pc = (ct.c_void_p * n)(*[t.data_ptr() for t in dc])
        ps = (ct.c_void_p * n)(*[t.data_ptr() for t in ds])
        outs = {}
        for name, fn in (("fp64", L.charm_b200_shs_point_batch_dev),
                         ("i8", L.charm_b200_shs_point_batch_i8_dev)):
            out = [torch.empty(npts, dtype=torch.float64, device="cuda")
                   for _ in idx]
            pf = (ct.c_void_p * n)(*[t.data_ptr() for t in out])
            for rep in range(2):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                fn(ct.cast(pnt._Point, P), n, nmv, nmv, muv, R_EARTH, pc, ps,
                   0, pf, ct.cast(err, P))
                check()
                torch.cuda.synchronize()
                if rep == 1:
                    pot[name + "_s"] += time.perf_counter() - t0
            outs[name] = out
        for a, b in zip(outs["i8"], outs["fp64"]):
            pot["worst_rel_rms_vs_fp64"] = max(
                pot["worst_rel_rms_vs_fp64"],
                rel_rms(a.cpu().numpy(), b.cpu().numpy()))
        for j in idx:
            if j in probe:
                rows = probe[j][1]
                o = outs["i8"][idx.index(j)].view(pnt.lat.size, pnt.lon.size)
                i8_probe[j] = o[rows, :].cpu().numpy()
        del dc, ds, outs
        torch.cuda.empty_cache()
    pot["speedup"] = pot["fp64_s"] / pot["i8_s"]
    pot["i8_sets_per_s"] = 64.0 / pot["i8_s"]
    pot["fp64_sets_per_s"] = 64.0 / pot["fp64_s"]
    # per-component errors against the oracle
    comp = {}
    for j, (pnt, rows, vals) in probe.items():
        c, s = coefs[j]
        po = orc.Point(orc.GRID, pnt.lat[rows], pnt.lon,
                       np.full(rows.size, R_EARTH + h))
        shc = orc.Shc(int(nm[j]), GM, R_EARTH, c, s)
        ref = (orc.shs_point(po, shc, int(nm[j]), "pot") +
               orc.shs_point(po, shc, int(nm[j]), "grad1") +
               orc.shs_point(po, shc, int(nm[j]), "grad2"))
        e = {nm_: rel_rms(vals[q], ref[q]) for q, nm_ in enumerate(names)}
        e["split_precision"] = {nm_: rel_rms(probe8[j][q], ref[q])
                                for q, nm_ in enumerate(names)}
        comp["set%d_nmax%d_%s" % (j, int(nm[j]),
                                  "dh1" if j % 2 == 0 else "dh2")] = e
    L.charm_err_free(err)
    out = {
        "workload": "64 coefficient sets, nmax U(90, 2160) (rng 4999), "
                    "potential + grad1 + grad2 (10 quantities) at r = R + "
                    "250 km, DH1 / DH2 grids of the largest degree",
        "fp64_batched_10q_s": t_batch,
        "fp64_batched_10q_sets_per_s": 64.0 / t_batch,
        "split_precision_batched_10q_s": t_batch8,
        "split_precision_batched_10q_sets_per_s": 64.0 / t_batch8,
        "split_precision_speedup_10q": t_batch / t_batch8,
        "split_vs_fp64_rel_rms_per_component_off_poles": worst8,
        # summed device time of the library's kernels in one more call of
        # each batched form (events per kernel): Legendre kernels, row
        # transforms, tables / seeds / digit preparation
        "kernel_ms_10q": {
            k: {"legendre": v[0], "row_transforms": v[3], "prep": v[5],
                "tables": v[6]} for k, v in split_ms.items()},
        "units_n_m_pair": total_units,
        "potential_fp64_vs_split_precision": pot,
        "rel_rms_vs_oracle_per_component": comp,
        "oracle_rows_per_set": oracle_rows,
        "dtype": "f64", "data": "synthetic (seeds 4999, 4000 + j)",
    }
    if single_calls:
        out["single_calls_10q_s"] = t_single
        out["single_calls_10q_sets_per_s"] = 64.0 / t_single
        out["batched_speedup_over_single_calls"] = t_single / t_batch
    return out


def run_batch(args):
    """The batched DH workload alone (batch_dh with single calls); prints
    one JSON line.  One GPU."""
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(batch_dh(single_calls=True)), flush=True)


def run_cells(args):
    """The cell workload alone (cells()); prints one JSON line.  One GPU."""
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(cells(steps=args.steps)), flush=True)


def main():
    args = parse()
    if args.workload == "batch":
        run_batch(args)
    elif args.workload == "cells":
        run_cells(args)
    elif args.workload == "sctr-cg":
        run_sctr_cg(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
