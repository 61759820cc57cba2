#!/usr/bin/env python
"""Throughput of the pseudospectral temporal-jet step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 512] [--precision fp64|mixed] [--scalars 2] [--scheme cnab2|rk3if]

Headline workload (default): one 512^3 periodic temporal jet in FP64 carrying the
reference's field set u, v, w, s, c (the reference's solver_ps always advances both
scalars; here c is a second passive scalar, alpha 0), Re 5000, Sc = Sc_c = 0.7,
dt 2.5e-4, 2/3 dealiasing, the reference's Euler/AB2 + Crank-Nicolson scheme; state
resident on the device.  A step is one full time step (nonlinear term, projection,
dealiasing, update).  Metric: Mpoint-steps/s = N^3 * steps / s / 1e6, summed over
GPUs (each GPU advances its own jet: replicas, no collective).  The same field set,
grid, precision and scheme run in the reference arm, so the two values compare like
for like.

Legs beside the headline (each can be switched off): the mixed-precision form
(FP32 transforms and storage, FP64 update coefficients and statistics) with one
scalar at 512^3 against the FP64 step of the same field set, and its error against
FP64 after 100 steps; the IF-RK3 scheme; the batched ensemble; the served stream
(three runs); the reference program relinked against this library (drop-in shim).

Rank 0 prints one JSON line.  Inputs (>= 0.5 GB per field) exceed L2 (126 MB), so no
flush is needed between steps.  --impl reference runs the reference's own CUDA step
(oracle/_ref/c512/refdrv built from the unmodified sources) on the same grid.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "gnss-1_b200"))

METRIC = "Mpoint-steps/s at 512^3, FP64, fields u v w s c (the reference's field set); mixed precision alongside"
UNIT = "Mpoint-steps/s"
RE, SC, SC_C, DT, NOISE_K, AMP = 5000.0, 0.7, 0.7, 2.5e-4, 8.0, 0.05
E2E_STEPS_PER_CALL = 20


# ------------------------------------------------------------------ utilities
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if gpu_index < len(ids):
                gpu_index = ids[gpu_index]
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.out.flush()
        rows = []
        try:
            with open(self.out.name) as fp:
                for line in fp:
                    p = [x.strip() for x in line.split(",")]
                    if len(p) >= 9:
                        rows.append(p)
        finally:
            os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def max_over_ranks(x: float) -> float:
    """Max of a per-rank scalar over the process group (identity without one).
    Times are the slowest rank's: every rank advances its own jet (replicas)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    dev = f"cuda:{torch.cuda.current_device()}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    """Sum of a per-rank scalar over the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    dev = f"cuda:{torch.cuda.current_device()}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_value(points: float, ms_max: float, world: int) -> float:
    """Whole-job Mpoint-steps/s: every rank advanced `points` per step in ms_max."""
    return world * points / (ms_max * 1e-3) / 1e6


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# ------------------------------------------------------------------ our arm
VARIANTS = {"auto": 0, "register": 1, "staged": 2, "warpspec": 3, "tensor": 4}
ZNAMES = tuple(VARIANTS)   # variant names by value


def run_leg(G, torch, n, precision, scheme, steps, warmup, dev, profile_steps=4, barrier=None, variants=None,
            n_scalars=1):
    """Time `steps` steps of one jet resident on `dev`; returns a dict."""
    cdt = np.complex128 if precision == G.GNSS_FP64 else np.complex64
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    init = G.jet_initial_state(nx, ny, nz, n_scalars=n_scalars, seed=0, noise_kmax=NOISE_K, amp=AMP)
    ctx = G.Context(nx=nx, ny=ny, nz=nz, re=RE, sc=SC, sc_c=SC_C, dt=DT, n_scalars=n_scalars, precision=precision,
                    scheme=scheme, device=dev)
    if variants:
        ctx.set_option(G.GNSS_OPT_ZVARIANT, VARIANTS[variants[0]])
        ctx.set_option(G.GNSS_OPT_PVARIANT, VARIANTS[variants[1]])
    st = [torch.from_numpy(a.astype(cdt)).to(f"cuda:{dev}") for a in init]
    del init
    hi = [torch.zeros_like(st[0]) for _ in st] if scheme == G.GNSS_SCHEME_CNAB2 else None
    ctx.de_alias(st)
    for s in range(warmup):
        ctx.solver_ps(st, hi, euler=(s == 0))
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if barrier:
        barrier()
    torch.cuda.synchronize(dev)
    l0 = ctx.launch_count()
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for s in range(steps):
            ctx.solver_ps(st, hi, euler=(warmup == 0 and s == 0))
        e1.record(stream)
        torch.cuda.synchronize(dev)
    if barrier:
        barrier()
    launches = ctx.launch_count() - l0
    ms = e0.elapsed_time(e1) / steps
    ctx.check()
    stats = ctx.stats(st)
    # per-stage device times (separate profiled steps of the same workload)
    ctx.profile(True)
    for s in range(profile_steps):
        ctx.solver_ps(st, hi, euler=False)
    prof = ctx.profile_read()
    ctx.profile(False)
    out = dict(ms=ms, launches=launches, clocks=clk.summary(), stats=stats, profile=prof,
               field_bytes=ctx.field_bytes(), stage_bytes=ctx.stage_bytes())
    del st, hi
    ctx.close()
    torch.cuda.empty_cache()
    return out


def stage_table(leg) -> dict:
    """Per-stage device ms per launch and algorithmic GB/s of a leg's profiled steps."""
    prof = leg["profile"]
    return {"stages_ms_per_launch": {k: round(v[0] / max(v[1], 1), 4) for k, v in prof.items()},
            "stages_gbs": {k: round(leg["stage_bytes"][k] / (v[0] / max(v[1], 1) * 1e-3) / 1e9, 1)
                           for k, v in prof.items() if v[1]}}


def run_e2e(G, torch, n, precision, scheme, calls, dev, n_scalars=1):
    """Public host-buffer API: pinned state in, E2E_STEPS_PER_CALL steps, state and statistics out."""
    cdt = np.complex128 if precision == G.GNSS_FP64 else np.complex64
    init = [a.astype(cdt) for a in G.jet_initial_state(n, n_scalars=n_scalars, seed=0, noise_kmax=NOISE_K,
                                                       amp=AMP)]
    ctx = G.Context(n, re=RE, sc=SC, sc_c=SC_C, dt=DT, n_scalars=n_scalars, precision=precision, scheme=scheme,
                    device=dev)
    host_in = torch.from_numpy(G.pack_state(init)).pin_memory()
    del init
    host_out = torch.empty_like(host_in).pin_memory()
    stats = np.zeros((E2E_STEPS_PER_CALL, G.GNSS_NSTATS))
    ctx.run_host(host_in, host_out, E2E_STEPS_PER_CALL, True, stats)   # warm-up call
    stream = torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(calls):
        ctx.run_host(host_in, host_out, E2E_STEPS_PER_CALL, True, stats)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_call = e0.elapsed_time(e1) / calls
    h2d, d2h = ctx.run_host_bytes()    # the kept box of each field in, the whole state out
    ctx.close()
    del host_in, host_out
    return dict(ms_call=ms_call, h2d=h2d / E2E_STEPS_PER_CALL,
                d2h=(d2h + E2E_STEPS_PER_CALL * 6 * 8) / E2E_STEPS_PER_CALL)   # + six double sums per step


def run_error_vs_fp64(G, torch, n, steps, dev) -> dict:
    """Per-field relative L2 of the mixed-precision state against the FP64 state
    after `steps` steps from the same initial state (both on the device)."""
    init = G.jet_initial_state(n, n_scalars=1, seed=0, noise_kmax=NOISE_K, amp=AMP)
    res = {}
    for prec in (G.GNSS_FP64, G.GNSS_FP32):
        cdt = np.complex128 if prec == G.GNSS_FP64 else np.complex64
        with G.Context(n, re=RE, sc=SC, dt=DT, n_scalars=1, precision=prec, device=dev) as ctx:
            st = [torch.from_numpy(a.astype(cdt)).to(f"cuda:{dev}") for a in init]
            hi = [torch.zeros_like(st[0]) for _ in st]
            ctx.de_alias(st)
            for k in range(steps):
                ctx.solver_ps(st, hi, euler=(k == 0))
            ctx.check()
            res[prec] = st
            del hi
    ref, got = res[G.GNSS_FP64], res[G.GNSS_FP32]
    errs = [float((g.to(torch.complex128) - r).norm() / r.norm()) for g, r in zip(got, ref)]
    # the mean profiles (kx = kz = 0 line of u and s, statistics.cu:1936-2003)
    prof = [float((got[q][:, 0, 0].to(torch.complex128) - ref[q][:, 0, 0]).norm() / ref[q][:, 0, 0].norm())
            for q in (0, 3)]
    del res, ref, got
    torch.cuda.empty_cache()
    return {"steps": steps, "rel_l2_per_field": dict(zip(("u", "v", "w", "s"), [float(f"{e:.3e}") for e in errs])),
            "mean_profile_rel_l2": {"u": float(f"{prof[0]:.3e}"), "s": float(f"{prof[1]:.3e}")},
            "max": float(f"{max(errs):.3e}"), "tolerance": 1e-5}


def run_rk3(G, torch, n, precision, steps, dev) -> dict:
    """The IF-RK3 scheme (three nonlinear evaluations per step) at n^3, one scalar."""
    leg = run_leg(G, torch, n, precision, G.GNSS_SCHEME_RK3IF, steps, 3, dev, profile_steps=2)
    pts = float(n) ** 3
    step_bytes = 3.0 * sum(leg["stage_bytes"].values())
    ms = leg["ms"]
    peaks = measured_peaks()
    out = {"value": round(pts / (ms * 1e-3) / 1e6, 3), "unit": UNIT, "ms_per_step": round(ms, 4),
           "steps": steps, "precision": "fp32" if precision == G.GNSS_FP32 else "fp64",
           "launches_per_step": leg["launches"] / steps,
           "workload": f"temporal jet {n}^3, 1 scalar, Re {RE:g}, Sc {SC}, dt {DT:g}, rk3if (3 substeps)",
           "bytes_per_point_step": round(step_bytes / pts, 1),
           "step_gbs": round(step_bytes / (ms * 1e-3) / 1e9, 1),
           "step_frac_of_measured_hbm": round(step_bytes / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4),
           "clocks": leg["clocks"]}
    out.update(stage_table(leg))
    return out


def run_dropin(n, steps, warmup) -> dict | None:
    """The reference's own driver relinked against this library through the
    reference-ABI shim (oracle/_ref/c<n>/refdrv_gnss): the speed a user of the
    reference's functions gets without changing their code."""
    exe = ROOT / "oracle" / "_ref" / f"c{n}" / "refdrv_gnss"
    if not exe.exists():
        return None
    r = subprocess.run([str(exe), "time", str(steps), str(warmup)], capture_output=True, text=True, timeout=1200)
    if r.returncode != 0:
        return {"error": r.stderr.strip()[-300:]}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    ms = float(d["ms_per_step"])
    return {"value": round(float(n) ** 3 / (ms * 1e-3) / 1e6, 3), "unit": UNIT, "ms_per_step": round(ms, 4),
            "steps": steps, "warmup": warmup,
            "program": "reference driver + reference initialize/statistics/iofuncs objects, solver.o and "
                       "fftfuncs.o replaced by refabi.cu over libgnss_b200.so; FP64, fields u v w s c"}


# the batched ensemble workload: 16 x 64^3, 8 x 96^3, 6 x 128^3, 2 x 192^3
ENSEMBLE_SIZES = [64] * 16 + [96] * 8 + [128] * 6 + [192] * 2


def run_ensemble(G, torch, dev, steps, branches=8) -> dict:
    rng = np.random.default_rng(4)
    res = rng.uniform(500.0, 4000.0, len(ENSEMBLE_SIZES))
    scs = rng.choice([0.7, 1.0, 2.0], len(ENSEMBLE_SIZES))
    cfgs = [G.make_config(n, re=float(r), sc=float(sc), dt=1e-3, precision=G.GNSS_FP32, device=dev)
            for n, r, sc in zip(ENSEMBLE_SIZES, res, scs)]
    points = float(sum(n ** 3 for n in ENSEMBLE_SIZES))
    with G.Ensemble(cfgs, n_branches=branches) as ens:
        t0 = time.perf_counter()
        choices = ens.autotune(3)
        t_tune = time.perf_counter() - t0
        for i, n in enumerate(ENSEMBLE_SIZES):
            f = G.jet_initial_state(n, n_scalars=1, seed=i, noise_kmax=NOISE_K, amp=AMP, dtype=np.complex64)
            ens.upload(i, G.pack_state(f))
        stream = torch.cuda.current_stream(dev)
        chunk = 50
        ens.step(1 + chunk)        # first (Euler) step and graph capture, untimed
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clk:
            e0.record(stream)
            for _ in range(steps // chunk):
                ens.step(chunk)
            e1.record(stream)
            torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / (steps // chunk * chunk)
        lps = ens.launches_per_step()
        batched = {n: ens.batched(ENSEMBLE_SIZES.index(n)) for n in set(ENSEMBLE_SIZES)}
        ke = [ens.stats(i)["ke"] for i in (0, 16, 24, 30)]
    assert all(math.isfinite(k) for k in ke)
    return {"value": round(points / (ms * 1e-3) / 1e6, 3), "unit": UNIT, "ms_per_step": round(ms, 4),
            "steps": steps // chunk * chunk, "members": len(cfgs), "points_per_step": int(points),
            "workload": "16x64^3 + 8x96^3 + 6x128^3 + 2x192^3 jets, Re ~ U[500,4000], Sc in {0.7,1,2}, seeds 0-31, "
                        "FP32, dt 1e-3, cnab2",
            "graph": f"{chunk} steps of all 32 members per CUDA graph launch, {branches} branches; each size group "
                     f"member by member or as batched launches, as the autotuner measured faster",
            "gpu_launches_per_step": lps, "autotune_s": round(t_tune, 2),
            "autotune_choices": {str(n): {"z": ZNAMES[choices[ENSEMBLE_SIZES.index(n)] & 3],
                                          "pass": ZNAMES[choices[ENSEMBLE_SIZES.index(n)] >> 2],
                                          "batched": batched[n]}
                                 for n in sorted(set(ENSEMBLE_SIZES))},
            "clocks": clk.summary()}


SERVE_SIZES = (64, 96, 128, 192, 256)


def run_serving(G, dev, duration_s=15.0, rate=4.0) -> dict:
    """Poisson arrivals of jet runs into the continuous-batching server; latency
    is submission to completion on the server's clock."""
    rng = np.random.default_rng(5)
    pool = {}
    for n in SERVE_SIZES:
        for ns in (1, 2):
            f = G.jet_initial_state(n, n_scalars=ns, seed=n + ns, noise_kmax=NOISE_K, amp=AMP, dtype=np.complex64)
            pool[(n, ns)] = G.pack_state(f)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration_s:
            break
        arrivals.append(t)
    reqs = []
    for a in arrivals:
        n = int(rng.choice(SERVE_SIZES))
        ns = int(rng.integers(1, 3))
        re = float(rng.uniform(500.0, 5000.0))
        steps = int(rng.integers(100, 2001))
        reqs.append((a, G.make_config(n, re=re, sc=0.7, sc_c=1.0, dt=5e-4, n_scalars=ns, precision=G.GNSS_FP32,
                                      device=dev), pool[(n, ns)], steps))
    budget = 150 << 30
    # untimed warm-up on a server of its own: one short request per (size, scalars), so that the timed stream
    # does not pay the first launch of each kernel
    with G.Server(budget_bytes=budget, max_active=16, steps_per_launch=25, device=dev) as srv:
        wids = [srv.submit(G.make_config(n, re=1000.0, sc=0.7, sc_c=1.0, dt=5e-4, n_scalars=ns,
                                         precision=G.GNSS_FP32, device=dev), st, 26)
                for (n, ns), st in pool.items()]
        for rid in wids:
            srv.wait(rid, timeout=600.0)
            srv.result(rid)
    ids = []
    with G.Server(budget_bytes=budget, max_active=16, steps_per_launch=25, device=dev) as srv:
        t0 = time.perf_counter()
        for a, cfg, st, steps in reqs:
            d = t0 + a - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(cfg, st, steps))
        lat, first, last = [], None, 0.0
        for rid in ids:
            srv.wait(rid, timeout=1800.0)
            _, _, tm = srv.result(rid)
            lat.append(tm[2] - tm[0])
            first = tm[0] if first is None else min(first, tm[0])
            last = max(last, tm[2])
        rep = srv.report()
    lat = np.array(lat)
    return {"requests": len(ids), "arrival_rate_per_s": rate, "arrival_window_s": duration_s,
            "p50_s": round(float(np.percentile(lat, 50)), 3), "p99_s": round(float(np.percentile(lat, 99)), 3),
            "mean_s": round(float(lat.mean()), 3),
            "value": round(rep["point_steps"] / (last - first) / 1e6, 3), "unit": UNIT,
            "completed": rep["completed"], "failed": rep["failed"], "active_max": rep["active_max"],
            "budget_gb": budget / 2 ** 30, "reserved_max_gb": round(rep["bytes_reserved_max"] / 2 ** 30, 2),
            "workload": "Poisson arrivals, N in {64,96,128,192,256}^3, Re ~ U[500,5000], 100-2000 steps, "
                        "1-2 scalars, FP32, dt 5e-4; 25 steps per graph launch, 16 slots, 150 GB budget; "
                        "after an untimed warm-up request per (size, scalars)"}


def run_serving_repeated(G, dev, runs=3, duration_s=15.0) -> dict:
    """The served stream `runs` times (same seeded arrivals); the median run and the spread."""
    outs = [run_serving(G, dev, duration_s) for _ in range(runs)]
    order = sorted(range(runs), key=lambda i: outs[i]["p50_s"])
    med = dict(outs[order[runs // 2]])
    med["runs"] = [{k: o[k] for k in ("p50_s", "p99_s", "value", "completed", "failed")} for o in outs]
    med["spread"] = {k: [min(o[k] for o in outs), max(o[k] for o in outs)] for k in ("p50_s", "p99_s", "value")}
    med["reported"] = f"median run of {runs} by p50"
    return med


def cpu_baseline(n_sample=256, steps=2) -> dict:
    """The CPU oracle (same scheme and parameters) on all host cores, bounded sample."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    import gnss_b200 as G
    O.build()
    cores = os.cpu_count() or 1
    oc = O.cfg(n_sample, re=RE, sc=SC, sc_c=SC_C, dt=DT, nthreads=cores)
    f = G.jet_initial_state(n_sample, n_scalars=2, seed=0, noise_kmax=NOISE_K, amp=AMP)
    r = [np.zeros_like(f[0]) for _ in range(5)]
    t0 = time.perf_counter()
    for s in range(steps):
        O.step_cnab2(oc, f, r, euler=(s == 0))
    dt = time.perf_counter() - t0
    return {"value": round(n_sample ** 3 * steps / dt / 1e6, 3), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} FP64 steps of the reference scheme (29 transforms/step, the reference's own "
                      f"sequence, solver.cu:700-765) at {n_sample}^3 with the same parameters and fields "
                      f"u v w s c, {dt:.1f} s on {cores} threads"}


def headline_config(args, ws: int) -> dict:
    """The `config` object of the headline line; both arms print the same one."""
    prec = "fp64" if args.precision == "fp64" else "mixed"
    shape = args.grid or f"{args.n}^3"
    fields = "u v w s" + (" c" if args.scalars > 1 else "")
    return {"workload": f"temporal jet {shape}, {prec}, fields {fields}"
                        f"{' (c a second passive scalar, alpha 0)' if args.scalars > 1 else ''}, "
                        f"Re {RE:g}, Sc {SC}{f', Sc_c {SC_C}' if args.scalars > 1 else ''}, dt {DT:g}, "
                        f"2/3 dealias, {args.scheme}",
            "grid": args.grid or args.n, "precision": prec, "scheme": args.scheme, "scalars": args.scalars,
            "parallelism": f"replicas x{ws}",
            "l2": "inputs larger than L2 (>= 0.5 GB per field); no flush"}


def ours(args):
    import torch
    import gnss_b200 as G
    ws, rank, local = dist_env()
    dev = local
    torch.cuda.set_device(dev)
    barrier = None
    red = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{dev}"))
        barrier = dist.barrier
        red = max_over_ranks
    prec = G.GNSS_FP32 if args.precision == "mixed" else G.GNSS_FP64
    scheme = G.GNSS_SCHEME_CNAB2 if args.scheme == "cnab2" else G.GNSS_SCHEME_RK3IF
    n = args.n
    shape = tuple(int(v) for v in args.grid.split("x")) if args.grid else (n, n, n)
    var = (args.z_variant, args.pass_variant)
    full = not args.grid
    leg = run_leg(G, torch, shape, prec, scheme, args.steps, args.warmup, dev, barrier=barrier, variants=var,
                  n_scalars=args.scalars)
    ms = leg["ms"] if red is None else red(leg["ms"])
    pts = float(shape[0] * shape[1] * shape[2])
    value = replica_value(pts, ms, ws)
    e2e = None
    if not args.no_e2e and full:
        e = run_e2e(G, torch, n, prec, scheme, args.e2e_calls, dev, n_scalars=args.scalars)
        ms_call = e["ms_call"] if red is None else red(e["ms_call"])
        e2e = {"value": round(replica_value(pts * E2E_STEPS_PER_CALL, ms_call, ws), 3), "unit": UNIT,
               "h2d_bytes_per_step": int(e["h2d"]), "d2h_bytes_per_step": int(e["d2h"]),
               "steps_per_call": E2E_STEPS_PER_CALL,
               "call": "gnss_run_host: pinned host state in, steps, per-step statistics and state out"}
    # roofline of the dominant kernel (stage of the fused step with the largest device time);
    # algorithmic bytes per launch come from the library's own layout (gnss_stage_bytes)
    prof = leg["profile"]
    dom = max(prof, key=lambda k: prof[k][0])
    t_ms, nl = prof[dom]
    alg = leg["stage_bytes"][dom]
    peaks = measured_peaks()
    achieved = alg / (t_ms / nl * 1e-3) / 1e9
    tr_file = ROOT / "profiles" / "traffic.json"
    traffic_meas = None
    if tr_file.exists():
        tj = json.loads(tr_file.read_text())
        key = f"{args.precision}:{args.scalars}:{args.grid or n}:{dom}"
        if key in tj:
            traffic_meas = tj[key]["bytes_per_launch"]
    roofline = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic_meas,
                "algorithmic_bytes": int(alg), "peak_source": peaks["source"] + " (burst copy)"}
    roofline.update(stage_table(leg))
    # the mixed-precision form (one scalar, FP32 transforms) against the FP64 step of the same field set
    mixed = None
    if prec == G.GNSS_FP64 and not args.no_mixed_leg:
        l32 = run_leg(G, torch, shape, G.GNSS_FP32, scheme, max(args.steps, 10), 3, dev, barrier=barrier,
                      variants=var, n_scalars=1)
        l64 = run_leg(G, torch, shape, G.GNSS_FP64, scheme, max(3, min(args.steps, 10)), 3, dev, barrier=barrier,
                      variants=var, n_scalars=1)
        ms32 = l32["ms"] if red is None else red(l32["ms"])
        ms64 = l64["ms"] if red is None else red(l64["ms"])
        mixed = {"value": round(replica_value(pts, ms32, ws), 3), "unit": UNIT, "ms_per_step": round(ms32, 4),
                 "dtype": "f32", "fields": "u v w s",
                 "fp64_same_fields": {"value": round(replica_value(pts, ms64, ws), 3), "ms_per_step": round(ms64, 4)},
                 "mixed_over_fp64": round(ms64 / ms32, 3), "clocks": l32["clocks"]}
        mixed.update(stage_table(l32))
        mixed["fp64_same_fields"].update(stage_table(l64))
        dom32 = max(l32["profile"], key=lambda k: l32["profile"][k][0])
        t32, n32 = l32["profile"][dom32]
        a32 = l32["stage_bytes"][dom32] / (t32 / n32 * 1e-3) / 1e9
        mixed["roofline"] = {"kernel": dom32, "achieved": round(a32, 1), "frac": round(a32 / peaks["hbm_gbs"], 4)}
        if full and not args.no_error_check:
            mixed["error_vs_fp64"] = run_error_vs_fp64(G, torch, n, args.error_steps, dev)
    rk3 = None
    if full and not args.no_rk3:
        rk3 = run_rk3(G, torch, n, G.GNSS_FP32, args.rk3_steps, dev)
    ens = None
    if not args.no_ensemble and full:
        ens = run_ensemble(G, torch, dev, args.ensemble_steps, args.ensemble_branches)
        if red is not None:
            ens["value"] = round(ws * ens["points_per_step"] / (red(ens["ms_per_step"]) * 1e-3) / 1e6, 3)
    serve = None
    if not args.no_serve and full:
        serve = run_serving_repeated(G, dev, args.serve_runs, args.serve_seconds)
        # the same stream at a rate below the GPU's capacity: latency without the queueing of the 4/s stream
        light = run_serving(G, dev, args.serve_seconds, rate=args.serve_light_rate)
        serve["below_capacity"] = {k: light[k] for k in ("arrival_rate_per_s", "requests", "p50_s", "p99_s", "mean_s",
                                                         "value", "completed", "failed", "active_max")}
        if red is not None:   # whole-job throughput: every rank served its own stream
            serve["value"] = round(sum_over_ranks(serve["value"]), 3)
            serve["p50_s"] = red(serve["p50_s"])
            serve["p99_s"] = red(serve["p99_s"])
    dropin = None
    if rank == 0 and ws == 1 and full and not args.no_dropin:
        dropin = run_dropin(n, max(3, min(args.steps, 10)), 2)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if prec == G.GNSS_FP32 else "f64", "data": "synthetic",
        "config": headline_config(args, ws),
        "initial_state": f"seeded solenoidal noise |k|<={NOISE_K:g} rms {AMP} on the tanh jet profiles",
        "kernels": {"z": args.z_variant, "pass": args.pass_variant},
        "gpu_launches": leg["launches"], "clocks": leg["clocks"], "e2e": e2e, "roofline": roofline,
        "cpu_baseline": cpu, "mixed": mixed, "rk3if": rk3, "ensemble": ens, "serving": serve, "dropin": dropin,
        "stats_after": {k: leg["stats"][k] for k in ("ke", "eps", "chi_s", "var_s")},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ reference arm
def reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return
    exe = ROOT / "oracle" / "_ref" / f"c{args.n}" / "refdrv"
    if not exe.exists():
        print(json.dumps({"impl": "reference", "unavailable": f"reference build {exe} missing "
                                                             f"(oracle/build_ref.sh)"}))
        return
    r = subprocess.run([str(exe), "time", str(args.steps), str(args.warmup)], capture_output=True, text=True,
                       timeout=3600, env=dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get(
                           "CUDA_VISIBLE_DEVICES", str(local))))
    if r.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": f"refdrv failed: {r.stderr.strip()[-200:]}"}))
        return
    d = json.loads(r.stdout.strip().splitlines()[-1])
    ms = float(d["ms_per_step"])
    value = float(args.n) ** 3 / (ms * 1e-3) / 1e6
    line = {
        "metric": METRIC, "impl": "reference", "value": round(value, 3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(argparse.Namespace(**{**vars(args), "precision": "fp64", "scalars": 2}), 1),
        "initial_state": "the reference's jet profiles (initializeVelocity / initializeScalar), no noise",
        "program": "the reference's solver_ps (cuFFT; it always advances u v w s c) from the unmodified "
                   "sources built -O3 for sm_100a",
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the reference's own CUDA step (cuFFT, sm_100a build of the unmodified "
                                   "sources, one host thread driving the GPU); the reference has no CPU "
                                   f"implementation of this path; {args.steps} timed steps after "
                                   f"{args.warmup} warm-up"},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--grid", default=None, help="NXxNYxNZ instead of n^3 (profiling workloads; no e2e leg)")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--scalars", type=int, choices=(1, 2), default=2)
    ap.add_argument("--scheme", choices=("cnab2", "rk3if"), default="cnab2")
    ap.add_argument("--e2e-calls", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed-leg", action="store_true")
    ap.add_argument("--no-rk3", action="store_true")
    ap.add_argument("--rk3-steps", type=int, default=5)
    ap.add_argument("--no-dropin", action="store_true")
    ap.add_argument("--serve-runs", type=int, default=3)
    ap.add_argument("--serve-light-rate", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--z-variant", choices=tuple(VARIANTS), default="auto")
    ap.add_argument("--pass-variant", choices=("auto", "register", "staged", "tensor"), default="auto")
    ap.add_argument("--no-error-check", action="store_true")
    ap.add_argument("--error-steps", type=int, default=100)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--ensemble-branches", type=int, default=8)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("bench.py: at least 3 warm-up steps are required", file=sys.stderr)
        args.warmup = 3
    if args.impl == "reference":
        reference(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
