"""Benchmark: chem+property cell-updates/s of UNICORN's species sweep on B200.

One step = one species sweep over the 601x301 (180,901-cell) heptane field
(fuel=11, T peak 2300 K, seed 0): Y clip + mixture-averaged transport, cp and
h, the 544 rate coefficients, omega_k and d(omega_k)/dY_k, then the
point-implicit update of SOLVESP with the reference's input-card settings
(up to 100 passes, relaxation 0.99, tolerance 1e-8) at dt = 1e-5 s.
A cell-update = one cell through one such sweep.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``value`` is device-resident throughput (fields already on the GPU);
``e2e`` is the same sweep through the C ABI with the step's inputs copied
from pinned host memory and its outputs copied back, inside the timed
region. ``--impl reference`` times the reference's own routines (translated
to C, oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "chem+property cell-updates/s: FP64 vs mixed vs MLP+fallback at stated ω error"
UNIT = "cell-updates/s"
DT = 1e-3            # non-dimensional: 1e-5 s / TMSTR (0.01 s)
ISOR, RELX, TOL = 100, 0.99, 1e-8     # docs/input.uni:25-27
NZ, NR, FUEL, TPEAK = 601, 301, 11, 2300.0


def workload_config(n_gpus, extra=None):
    c = {"workload": "C2: 601x301 heptane jet field (fuel=11, T_peak 2300 K, seed 0), one species sweep per step "
                     "(props, cp/h, rates, omega, domega/dY, point-implicit update isor=100 relx=0.99 tol=1e-8, dt=1e-5 s)",
         "cells": NZ * NR, "precision": "fp64", "l2": "working set > L2 (RC plane 787 MB written and read every step)",
         "parallelism": f"cell-sharded x{n_gpus} (independent fields per rank)"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index: int):
        self.index, self.samples, self._stop = index, [], threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
            "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for nm, v in zip(names, s[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------- our arm
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline_port(f, scales_src):
    """The oracle (a faithful FP64 C restatement) on one host core, bounded sample."""
    from oracle.oracle import Oracle
    from unicorn_b200.fields import nondimensional
    o = Oracle()
    ns = 1024
    tk, rho = nondimensional(f, o.scales, o.wm)
    tk, rho, y = tk[:ns].copy(), rho[:ns].copy(), np.ascontiguousarray(f.y[:, :ns])
    t0 = time.perf_counter()
    yc, mu, lam, dk, _ = o.props(tk, y)
    cp = o.cp(tk, yc)
    h = o.enthalpy(tk, yc)
    q = o.omega(tk, rho, yc)
    rc, sour = o.rates(tk, rho, yc)
    yn, s, passes = o.species_update(rho, yc, rc, sour, DT, isor=ISOR, relx=RELX, tol=TOL)
    dt = time.perf_counter() - t0
    return {"value": ns / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"first {ns} cells of the C2 field, one full sweep (oracle/unichem_oracle.c, -O2, 1 thread; "
                      f"{passes} update passes), {dt:.2f} s"}


def run_ours(args, rank, world, dev):
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import jet_field, nondimensional
    f = jet_field(NZ, NR, fuel=FUEL, t_peak=TPEAK, seed=rank)
    if args.cells:
        f.T, f.p, f.y = f.T[:args.cells].copy(), f.p[:args.cells].copy(), np.ascontiguousarray(f.y[:, :args.cells])
    n = f.n
    u = unichem.UniChem(n, device=dev)
    tk, rho = nondimensional(f, u.scales, u.wm)
    view = unichem_view(u)
    ext = torch.cuda.ExternalStream(view["stream"], device=dev)
    # pinned host buffers for the end-to-end path
    pin = lambda *s: torch.empty(s, dtype=torch.float64, pin_memory=True).numpy()
    h_tk, h_rho, h_y = pin(n), pin(n), pin(52, n)
    h_tk[:], h_rho[:], h_y[:] = tk, rho, f.y
    outs = dict(qdsp=pin(52, n), qdot=pin(n), domega_dy=pin(52, n), vmu=pin(n), vtc=pin(n), vdf=pin(52, n),
                cp=pin(n), h=pin(n))
    h_yout = pin(52, n)

    def reset():
        u.upload(h_tk, h_rho, h_y)

    prec = unichem.MIXED if args.precision == "mixed" else unichem.FP64

    def step_device():
        return u.sweep(DT, precision=prec, isor=args.isor, relx=RELX, tol=TOL)

    passes_seen = []
    reset()
    for _ in range(args.warmup):
        passes_seen.append(step_device())
    # ---------------- device-resident timing
    reset()
    torch.cuda.synchronize(dev)
    barrier(world)
    u.profile(True)
    with torch.cuda.stream(ext):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev if world == 1 else dev) as clk:
            e0.record(ext)
            for _ in range(args.steps):
                passes_seen.append(step_device())
            e1.record(ext)
            torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    kt = u.profile_read()
    u.profile(False)
    ms = max_over_ranks(ms, world)
    # ---------------- end-to-end through the C ABI (host buffers)
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        u.upload(h_tk, h_rho, h_y)
        u.sweep(DT, precision=prec, isor=args.isor, relx=RELX, tol=TOL)
        u.download_outputs(outs)
        u.lib.uc_download_fields(u._h, None, None, unichem._p(h_yout), None, None)
    u.sync()
    e2e_s = max_over_ranks((time.perf_counter() - t0) * 1e3, world) / 1e3
    h2d = (2 + 52) * 8 * n
    d2h = (52 * 4 + 5) * 8 * n
    res = {"ms_per_step": ms / args.steps, "value": world * n * args.steps / (ms / 1e3),
           "e2e": {"value": world * n * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h},
           "kernel_ms": kt, "passes": passes_seen, "clocks": clk.summary(), "n": n,
           "gpu_launches": sum(c for _, c in kt.values())}
    u.close()
    return res, f


def unichem_view(u):
    import ctypes

    class View(ctypes.Structure):
        _fields_ = [(k, ctypes.c_void_p) for k in ("tk", "rho", "fsp", "fsp_old", "stmf", "stnd", "rc", "qdsp", "qdot",
                                                    "domega_dy", "vmu", "vtc", "vdf", "cp", "h")] + \
                   [("n", ctypes.c_int), ("npad", ctypes.c_int), ("stream", ctypes.c_void_p)]
    v = View()
    u.lib.uc_device_view_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(View)]
    u._ck(u.lib.uc_device_view_get(u._h, ctypes.byref(v)))
    return {"stream": v.stream or 0, "npad": v.npad}


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def roofline(res, n, steps, mixed=False, isor=ISOR):
    """Dominant kernel of the step and its achieved rate against the measured HBM copy bandwidth."""
    kt = res["kernel_ms"]
    name = max(kt, key=lambda k: kt[k][0])
    ms, cnt = kt[name]
    hbm, src = peaks()
    npad = (n + 31) // 32 * 32
    # passes run per step (the reported count is isor + 1 when the tolerance was not met)
    passes = sum(min(p, isor) for p in res["passes"][-steps:]) / max(1, steps)
    # algorithmic bytes per launch: per-cell figures x cells
    traffic = None
    if name == "update" and mixed:
        per_cell = passes * (544 * 4 + (52 + 52 + 6 + 2 + 2) * 8) + (52 + 2) * 8
        unit_note = (f"per cell and launch: {passes:.1f} passes x (RC 544 x 4 B of the FP32 plane + (Y 52 in + 52 out "
                     "+ SOUR 6 + soot 4) x 8 B)")
    elif name == "update":
        per_cell = passes * (544 + 52 + 52 + 6 + 2 + 2) * 8 + (52 + 2) * 8
        unit_note = f"per cell and launch: {passes:.1f} passes x (RC 544 + Y 52 in + 52 out + SOUR 6 + soot 4) x 8 B"
        # DRAM read + write of one launch of the FP64 update (Y in place, 14 warps per SM) under ncu
        # (65,536 C2 cells, 5 passes: 3.723 GB + 0.193 GB), per cell and pass, scaled to this launch
        # by cells x passes run
        traffic = round(11951.0 * n * passes)
    elif name == "chem":
        per_cell = (52 + 4) * 8 + (544 + 52 + 52 + 1 + 6) * 8
        unit_note = "per cell: read T, rho, soot, Y (56 x 8 B); write RC 544, QDSP 52, dw/dY 52, QDOT, SOUR 6"
    else:
        per_cell = (54 + 54) * 8
        unit_note = "per cell: 54 inputs + 54 outputs x 8 B"
    bytes_per_launch = per_cell * n
    achieved = bytes_per_launch / (ms / cnt / 1e3) / 1e9
    return {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "peak_source": src,
            "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": traffic, "bytes_per_launch": bytes_per_launch,
            "avg_launch_ms": ms / cnt, "bytes_rule": unit_note}


def main_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res, f = run_ours(args, rank, world, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(f, None)
    if rank == 0:
        line = {"metric": METRIC, "value": round(res["value"], 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(res["ms_per_step"], 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded C2 generator; the reference ships no benchmark data)",
                "config": workload_config(world, {"update_passes_per_step": res["passes"][-args.steps:],
                                                  "precision": args.precision}),
                "e2e": res["e2e"], "gpu_launches": res["gpu_launches"] * world, "clocks": res["clocks"],
                "roofline": roofline(res, res["n"], args.steps, args.precision == "mixed", args.isor),
                "kernel_ms": {k: round(v[0], 3) for k, v in res["kernel_ms"].items()}}
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- reference arm
def _ref_worker(args_tuple):
    """One host process: the reference's own routines on a chunk of cells."""
    tk, rho, y, isor = args_tuple
    from oracle.ref import RefUnicorn
    r = _ref_worker.r if hasattr(_ref_worker, "r") else None
    if r is None:
        r = _ref_worker.r = RefUnicorn()
    t0 = time.perf_counter()
    yc, mu, lam, vdf = r.props(tk, y)
    cp = r.cp(tk, yc)
    q = r.omega(tk, rho, yc)
    yn, s1, s2, passes = r.species_update(tk, rho, yc, DT, isor=isor, relx=RELX, tol=TOL)
    return len(tk), time.perf_counter() - t0, passes


def main_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference routines translated to C) "
                          "is not built: run python -c 'import __graft_entry__ as g; g.build()' where the reference "
                          "checkout exists"}))
        return
    import multiprocessing as mp
    from unicorn_b200.fields import jet_field, nondimensional
    r0 = R.RefUnicorn()
    f = jet_field(NZ, NR, fuel=FUEL, t_peak=TPEAK, seed=0)
    tk, rho = nondimensional(f, r0.scales, r0.wm)
    chunk = r0.chunk
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        def one_step(step):
            jobs = []
            for w in range(cores):
                a = ((step * cores + w) * chunk) % (f.n - chunk)
                jobs.append((tk[a:a + chunk].copy(), rho[a:a + chunk].copy(),
                             np.ascontiguousarray(f.y[:, a:a + chunk]), ISOR))
            t0 = time.perf_counter()
            out = pool.map(_ref_worker, jobs)
            return sum(o[0] for o in out), time.perf_counter() - t0, [o[2] for o in out]
        for w in range(args.warmup):
            one_step(w)
        cells, secs, passes = 0, 0.0, []
        for s in range(args.steps):
            c, t, p = one_step(args.warmup + s)
            cells += c
            secs += t
            passes += p
    v = cells / secs
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(secs / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded C2 generator)",
        "config": workload_config(1, {"update_passes_per_chunk": passes[:8]}),
        "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{cores} chunks of {chunk} cells of the C2 field per step, one process per core, "
                                   "each running the reference's PROPS/CKRATES/SOLVESP/SOLVEH-rate code "
                                   "(translated from its Fortran, gcc -O2)"},
        "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


# ---------------------------------------------------------------- C3: batched stiff integration
C3_CELLS = 1 << 20


def cpu_baseline_c3(f, ncells=2048):
    """The oracle's batched integration (orc_integrate, OpenMP over cells) on a bounded sample."""
    from oracle.oracle import Oracle
    from unicorn_b200.fields import nondimensional
    o = Oracle()
    tk, rho = nondimensional(f, o.scales, o.wm)
    sl = slice(0, ncells)
    y = np.ascontiguousarray(f.y[:, sl])
    pnd = f.p[sl] / o.scales["PSTR"]
    t0 = time.perf_counter()
    q = o.omega(tk[sl], rho[sl], y)[0]
    ns, _ = o.nsub(rho[sl], y, q, DT)
    o.integrate(tk[sl], rho[sl], y, pnd, ns, DT)
    dt = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    return {"value": ncells / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {ncells} cells of the C3 batch (mean n_sub {ns.mean():.1f}), oracle/unichem_oracle.c "
                      f"orc_integrate, -O2, OpenMP over cells, {dt:.2f} s"}


def main_c3(args):
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import batch_cells, nondimensional
    n = args.cells or C3_CELLS
    f = batch_cells(n, seed=0)
    prec = unichem.FP64
    opts = dict(isor=args.isor, relx=RELX, tol=TOL)
    u = unichem.UniChem(n)
    tk, rho = nondimensional(f, u.scales, u.wm)
    pnd = f.p / u.scales["PSTR"]
    pin = lambda *s: torch.empty(s, dtype=torch.float64, pin_memory=True).numpy()
    h_tk, h_rho, h_y, h_p = pin(n), pin(n), pin(52, n), pin(n)
    h_tk[:], h_rho[:], h_y[:], h_p[:] = tk, rho, f.y, pnd
    o_tk, o_rho, o_y = pin(n), pin(n), pin(52, n)
    u.set_pressure(h_p)
    u.upload(h_tk, h_rho, h_y)
    tune = u.integrate_tune(DT, precision=prec, **opts)
    for _ in range(args.warmup):
        u.upload(h_tk, h_rho, h_y)
        u.integrate(DT, precision=prec, **opts)
    u.sync()
    # device time of the integration graph only (each step restarts from the same state, uploaded before it)
    u.profile(True)
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            u.upload(h_tk, h_rho, h_y)
            u.integrate(DT, precision=prec, **opts)
        kt = u.profile_read()
    u.profile(False)
    ms = kt["integrate"][0]
    ns, pa = u.integrate_counts()
    # end to end through the C ABI: inputs from pinned host memory, state back to the host
    u.sync()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        u.upload(h_tk, h_rho, h_y)
        u.integrate(DT, precision=prec, **opts)
        u.lib.uc_download_fields(u._h, unichem._p(o_tk), unichem._p(o_rho), unichem._p(o_y), None, None)
    u.sync()
    e2e = time.perf_counter() - t0
    u.close()
    substeps = float(ns.sum())
    per_sub_flop = 9.0e3 + 470 + 2 * 2189 * float(pa.sum()) / substeps
    achieved = per_sub_flop * substeps / (ms / args.steps / 1e3) / 1e12
    line = {"metric": "batched stiff integration cell-updates/s (one cell over dt = 1e-5 s)",
            "value": round(n * args.steps / (ms / 1e3), 1), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded C3 generator)",
            "config": {"workload": f"C3: {n} independent heptane-generator cells, T~U[300,2400] K, p~U[0.8,1.2] atm, "
                                   "dt=1e-5 s, n_sub=clamp(ceil(max_k dt|w_k|/Y_k over Y_k>1e-3), 1, 200), "
                                   f"update passes to 1e-8 per sub-step (<={args.isor})",
                       "cells": n, "precision": "fp64", "tuned": tune,
                       "nsub": {"mean": round(float(ns.mean()), 2), "min": int(ns.min()), "max": int(ns.max()),
                                "frac_1": round(float((ns == 1).mean()), 4),
                                "frac_max": round(float((ns == ns.max()).mean()), 4)},
                       "passes_per_substep": round(float(pa.sum()) / substeps, 2),
                       "l2": "state 470 MB > L2; all sub-step work on chip"},
            "e2e": {"value": round(n * args.steps / e2e, 1), "unit": UNIT, "h2d_bytes_per_step": (2 + 52) * 8 * n,
                    "d2h_bytes_per_step": (2 + 52) * 8 * n},
            "gpu_launches": kt["integrate"][1] * (6 if tune["int_sorted"] else 3),
            "clocks": clk.summary(),
            "roofline": {"kernel": "integrate", "bound": "fp64", "achieved": round(achieved, 3), "peak": 37.0,
                         "peak_source": "nominal B200 FP64 (no measured FP64 peak on this pool)", "unit": "TFLOP/s",
                         "frac": round(achieved / 37.0, 4), "traffic": None,
                         "flops_rule": "per cell and sub-step: 9e3 rate flops + 470 transcendentals (1 op each) + "
                                       "2 flops x 2189 update terms x passes"}}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_c3(f)
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- C4: learned surrogate
C4_TRAIN, C4_FIELD = 4 << 20, 1 << 20
MLP_FLOP_PER_CELL = 2 * (64 * 256 + 3 * 256 * 256 + 256 * 64)     # padded GEMM shapes, multiply-add = 2 flops


def main_c4(args):
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import batch_cells, nondimensional
    from unicorn_b200.surrogate import Surrogate, raw_features
    ntrain = args.cells * 4 if args.cells else C4_TRAIN
    nfield = args.cells or C4_FIELD
    chunk = min(ntrain, 1 << 20)
    steps = args.train_steps
    # ---- training set: exact FP64 omega of C3-distribution states, in chunks
    t0 = time.perf_counter()
    s = Surrogate(capacity=ntrain, seed=1)
    u = unichem.UniChem(chunk)
    hull_lo, hull_hi, norm = None, None, None
    for c in range(ntrain // chunk):
        f = batch_cells(chunk, seed=100 + c)
        tk, rho = nondimensional(f, u.scales, u.wm)
        pref = u.scales["PBACK"] * u.scales["PSTR"]
        u.upload(tk, rho, f.y)
        u.set_pressure(f.p / u.scales["PSTR"])
        feats = raw_features(f.T, f.p / pref, f.y)
        if norm is None:
            sub = np.arange(0, chunk, max(1, chunk // 65536))
            q = u.omega().qdsp
            norm = Surrogate.norm_from_sample(feats[:, sub], q[:, sub])
            s.set_norm(**norm)
        lo, hi = feats.min(axis=1), feats.max(axis=1)
        hull_lo = lo if hull_lo is None else np.minimum(hull_lo, lo)
        hull_hi = hi if hull_hi is None else np.maximum(hull_hi, hi)
        s.add_data(u)
    u.close()
    norm.update(hull_lo=hull_lo, hull_hi=hull_hi)
    s.set_norm(**norm)
    t_data = time.perf_counter() - t0
    # ---- training (device time of the whole run, graph per step)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = s.train(steps=steps, batch=8192, lr=1e-3, seed=3)
    t_train = time.perf_counter() - t0
    # ---- inference on a fresh field: exact FP64 omega vs surrogate + fallback
    f = batch_cells(nfield, seed=7)
    u = unichem.UniChem(nfield)
    tk, rho = nondimensional(f, u.scales, u.wm)
    u.upload(tk, rho, f.y)
    u.set_pressure(f.p / u.scales["PSTR"])
    view = unichem_view(u)
    ext = torch.cuda.ExternalStream(view["stream"])
    out = {"qdsp": np.empty((52, nfield))}

    def timed(fn, reps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(reps):
            r = fn()
        e1.record(ext)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, r

    ms_exact, _ = timed(lambda: u.omega(download=False), args.steps)
    u.download_outputs(out)
    exact = out["qdsp"].copy()
    res = {}
    with ClockSampler(0) as clk:
        for tol in (1e-3, 1e-1, 1e300, float("inf")):
            ms, _ = timed(lambda: s.omega(u, tol=tol, stats=False), args.steps)
            st = s.omega(u, tol=tol)
            u.download_outputs(out)
            q = out["qdsp"]
            wmax = np.abs(exact).max(axis=0)
            r = np.abs(q - exact) / np.maximum(np.abs(exact), 1e-6 * wmax + 1e-300)
            r[f.y <= 1e-8] = 0.0
            err = r.max(axis=0)
            res["tol=%g" % tol] = {"ms": round(ms, 3), "cell_updates_per_s": round(nfield / (ms / 1e3), 1),
                                  "speedup_vs_fp64": round(ms_exact / ms, 3), "tiles_exact": round(st["tiles_exact"], 4),
                                  "cells_outside_hull": round(st["cells_outside_hull"], 5),
                                  "median_sampled_residual": st["median_residual"],
                                  "err_vs_fp64_p50": float(np.median(err)), "err_vs_fp64_p99": float(np.quantile(err, 0.99)),
                                  "frac_cells_err_le_1e-3": round(float((err <= 1e-3).mean()), 4)}
    u.close()
    s.close()
    pure = res["tol=inf"]          # the network alone: features, 5 tensor-core layers, decode
    tflops = MLP_FLOP_PER_CELL * nfield / (pure["ms"] / 1e3) / 1e12
    line = {"metric": "omega cell-updates/s: learned surrogate + per-tile FP64 fallback at the stated error",
            "value": res["tol=0.001"]["cell_updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["tol=0.001"]["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network / f64 fallback", "data": "synthetic (seeded C3/C4 generators)",
            "config": {"workload": f"C4: network 54-256x4-52 GELU, Adam lr 1e-3 batch 8192, {steps} steps on {ntrain} "
                                   f"exact-FP64 states of the C3 distribution; inference on a fresh {nfield}-cell field "
                                   "with fallback per 32-cell tile (training hull, one sampled residual per tile)",
                       "fp64_omega_ms": round(ms_exact, 3),
                       "fp64_omega_cell_updates_per_s": round(nfield / (ms_exact / 1e3), 1),
                       "by_tolerance": res, "train_s": round(t_train, 2), "data_s": round(t_data, 2),
                       "train_samples_per_s": round(steps * 8192 / t_train, 1),
                       "loss_first": float(loss[:10].mean()), "loss_last": float(loss[-50:].mean())},
            "e2e": None, "gpu_launches": None, "clocks": clk.summary(),
            "roofline": {"kernel": "surrogate forward (features, 5 tensor-core layers, decode; tol=inf)", "bound": "tensor",
                         "achieved": round(tflops, 2), "peak": 1693.5, "peak_source": "measured (bf16 burst)",
                         "unit": "TFLOP/s", "frac": round(tflops / 1693.5, 4), "traffic": None,
                         "flops_rule": f"{MLP_FLOP_PER_CELL} flop per cell (padded 64-256x4-64 layers) / forward time"}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- C5: in-loop sweeps
def main_c5(args):
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import jet_field, nondimensional
    from unicorn_b200.inloop import frozen_faces, omega_error
    from unicorn_b200.surrogate import Surrogate, raw_features
    f = jet_field(NZ, NR, fuel=FUEL, t_peak=TPEAK, seed=0)
    n = f.n
    checkpoints = sorted({c for c in (100, 500, 1000, args.sweeps) if c <= args.sweeps})
    # ---- surrogate trained on four other seeded fields of the same generator
    s = Surrogate(capacity=4 * n, seed=1)
    u = unichem.UniChem(n)
    pref = u.scales["PBACK"] * u.scales["PSTR"]
    norm = None
    for seed in (11, 12, 13, 14):
        g = jet_field(NZ, NR, fuel=FUEL, t_peak=TPEAK, seed=seed)
        tk, rho = nondimensional(g, u.scales, u.wm)
        u.upload(tk, rho, g.y)
        u.set_pressure(g.p / u.scales["PSTR"])
        if norm is None:
            norm = Surrogate.norm_from_sample(raw_features(g.T, g.p / pref, g.y), u.omega().qdsp)
            s.set_norm(**norm)
        s.add_data(u)
    u.close()
    loss = s.train(steps=args.train_steps, batch=8192, lr=1e-3, seed=3)
    # ---- the in-loop runs
    report = {}
    timing = {}
    ref_states = {}
    probe = unichem.UniChem(n)
    for name, prec in (("fp64", unichem.FP64), ("mixed", unichem.MIXED)):
        u = unichem.UniChem(n)
        tk, rho = nondimensional(f, u.scales, u.wm)
        u.upload(tk, rho, f.y)
        u.set_pressure(f.p / u.scales["PSTR"])
        if name == "fp64":
            vdf = u.props()[2]
            _, _, yc, _, _ = u.download()
            fs, fn = frozen_faces((NZ, NR), vdf, yc, DT)
            u.upload(tk, rho, f.y)
        u.hold_enthalpy()
        view = unichem_view(u)
        ext = torch.cuda.ExternalStream(view["stream"])
        rep = {}
        ms_total, passes = 0.0, []
        for sw in range(1, args.sweeps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            passes.append(u.sweep(DT, precision=prec, isor=ISOR, relx=RELX, tol=TOL, face_sum=fs, face_nbr=fn))
            u.temperature_from_held()
            e1.record(ext)
            e1.synchronize()
            ms_total += e0.elapsed_time(e1)
            if sw in checkpoints:
                tk1, rho1, y1, s1, _ = u.download()
                T1 = tk1 * u.scales["TSTR"]
                free = T1 < 5000.0 - 1e-6          # cells not held at the T clamp of solveh.f
                entry = {"peak_T": round(float(T1.max()), 3), "peak_T_drift": round(float(T1.max() - f.T.max()), 3),
                         "peak_T_below_clamp": round(float(T1[free].max()), 3), "mean_T": round(float(T1.mean()), 3),
                         "cells_at_5000K": int((~free).sum()),
                         "sumY_drift_max": float(np.abs(y1.sum(0) + s1 - 1.0).max()),
                         "mean_passes": round(float(np.mean(passes[-100:])), 2)}
                if name == "fp64":
                    ref_states[sw] = (T1.copy(), y1.copy())
                else:
                    Tr, yr = ref_states[sw]
                    entry.update({"vs_fp64_max_dT": float(np.abs(T1 - Tr).max()), "vs_fp64_max_dY": float(np.abs(y1 - yr).max()),
                                  "vs_fp64_p99_dT": float(np.quantile(np.abs(T1 - Tr), 0.99))})
                # omega of this state: FP64 kernel, mixed kernel, surrogate (no fallback / with fallback at 1e-3)
                probe.upload(tk1, rho1, y1, s1, None)
                probe.set_pressure(f.p / u.scales["PSTR"])
                ex = probe.omega(unichem.FP64).qdsp
                mx = probe.omega(unichem.MIXED).qdsp
                s.omega(probe, tol=float("inf"), stats=False)
                out = {"qdsp": np.empty((52, n))}
                probe.download_outputs(out)
                e_mx, e_ml = omega_error(mx, ex, y1), omega_error(out["qdsp"], ex, y1)
                fb = s.omega(probe, tol=1e-3)
                entry.update({"omega_err_mixed_p50": float(np.median(e_mx)), "omega_err_mixed_p99": float(np.quantile(e_mx, 0.99)),
                              "omega_mixed_frac_le_1e-3": round(float((e_mx <= 1e-3).mean()), 4),
                              "omega_err_mlp_p50": float(np.median(e_ml)), "omega_err_mlp_p99": float(np.quantile(e_ml, 0.99)),
                              "mlp_tiles_exact_at_1e-3": round(fb["tiles_exact"], 4)})
                rep[f"sweep_{sw}"] = entry
        timing[name] = {"ms_per_sweep": round(ms_total / args.sweeps, 3),
                        "cell_updates_per_s": round(n * args.sweeps / (ms_total / 1e3), 1)}
        report[name] = rep
        u.close()
    probe.close()
    s.close()
    line = {"metric": "in-loop heptane sweeps: peak-T drift, sum-Y drift and omega error at sweeps 100/500/1000",
            "value": timing["fp64"]["cell_updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.sweeps, "warmup": 0,
            "ms_per_step": timing["fp64"]["ms_per_sweep"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (and mixed)", "data": "synthetic (seeded C2 generator)",
            "config": {"workload": f"C5: 601x301 heptane field, {args.sweeps} sweeps of dt=1e-5 s, transport frozen "
                                   "(diffusion faces from the initial field), T from held enthalpy each sweep",
                       "timing": timing, "report": report,
                       "surrogate": {"train_steps": args.train_steps, "train_states": 4 * n,
                                     "loss_first": float(loss[:10].mean()), "loss_last": float(loss[-50:].mean())}}}
    print(json.dumps(line), flush=True)


def cpu_baseline_enthalpy(u, fl, ht, ncols=61):
    """The oracle's enthalpy step (rates, EKT/Z, RHSZ, Gauss-Seidel relaxation, T) on one host core for
    the first ncols columns of the device's current field, as a bounded sample."""
    from oracle.oracle import Oracle
    o = Oracle()
    tk, rho, y, s1, _ = u.download()
    nr = fl["lj"]
    m = nr * ncols
    sl = slice(0, m)
    yc, _, vtc, vdf, _ = o.props(tk[sl], np.ascontiguousarray(y[:, sl]))
    t0 = time.perf_counter()
    r = o.enthalpy_solve(nr, ncols, tk[sl], rho[sl], yc, yc, ht[sl], s1[sl], vtc, vdf, fl["u"][sl], fl["v"][sl],
                         fl["tmu"][sl], fl["yr"][sl], fl["xxs"][:ncols], fl["xxc"][:ncols], fl["yys"], fl["yyc"],
                         dt=DT, isor=ISOR, relx=RELX, tol=TOL)
    dt = time.perf_counter() - t0
    return {"value": m / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"enthalpy step only (oracle/unichem_oracle.c, -O2, 1 thread) on the first {ncols} columns "
                      f"({m} cells) of the field after the pre-sweeps, {r['passes']} relaxation passes, {dt:.2f} s"}


def main_c5_live(args):
    """In-loop sweeps with live transport: the species faces assembled on the device from the state of
    each sweep (SPGSOLV's coefficients), then the enthalpy equation (SOLVEH: heat release, species
    enthalpy diffusion, radiation, Gauss-Seidel relaxation, T from FPZ) and the density at PBACK."""
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import jet_field, jet_flow, nondimensional, sensible_enthalpy
    f = jet_field(NZ, NR, fuel=FUEL, t_peak=TPEAK, seed=0)
    fl = jet_flow(NZ, NR, seed=0)
    n = f.n
    prec = unichem.MIXED if args.precision == "mixed" else unichem.FP64
    u = unichem.UniChem(n)
    sc = u.scales
    tk, rho = nondimensional(f, sc, u.wm)
    u.upload(tk, rho, f.y)
    u.set_grid(fl["lj"], fl["li"], fl["xxs"], fl["xxc"], fl["yys"], fl["yyc"], fl["yr"], isym=1)
    u.set_flow(fl["u"], fl["v"], fl["tmu"], 0.9)
    with open(Path(__file__).resolve().parent / "unicorn_b200" / "mech" / "sandiego52.json") as fh:
        poly = np.array(json.load(fh)["poly"])
    ht = sensible_enthalpy(f.T, f.y, poly, u.wm, u.hfo, sc) + 0.5 * (fl["u"] ** 2 + fl["v"] ** 2)
    # the generator puts radicals (1e-10..1e-3) into cold cells as well; species-only sweeps at held
    # enthalpy first let the chemistry consume them, as the frozen in-loop run does, before the
    # enthalpy equation couples the heat release to T
    import warnings
    if args.presweeps > 0:
        u.set_pressure(f.p / sc["PSTR"])
        u.hold_enthalpy()
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            for _ in range(args.presweeps):
                u.sweep(DT, precision=prec, isor=ISOR, relx=RELX, tol=TOL)
                u.temperature_from_held()
        tk0, _, y0, _, _ = u.download()
        T0 = tk0 * sc["TSTR"]
        ht = sensible_enthalpy(T0, y0, poly, u.wm, u.hfo, sc) + 0.5 * (fl["u"] ** 2 + fl["v"] ** 2)
    else:
        T0 = f.T
    u.set_enthalpy(ht)
    cpu = None if args.no_cpu_baseline else cpu_baseline_enthalpy(u, fl, ht)
    view = unichem_view(u)
    ext = torch.cuda.ExternalStream(view["stream"])
    sweeps = args.sweeps
    sp_passes, h_passes, resdh = [], [], []
    ms, ms_split = 0.0, {}
    for sw in range(args.warmup + sweeps):
        timed = sw >= args.warmup
        if timed:
            u.profile(True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            p1 = u.sweep(DT, precision=prec, isor=ISOR, relx=RELX, tol=TOL)
            p2, r = u.enthalpy_update(DT, isor=ISOR, relx=RELX, tol=TOL, sigh=0.9)
        u.density()
        if timed:
            e1.record(ext)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            for k, (t, c) in u.profile_read().items():
                ms_split[k] = ms_split.get(k, 0.0) + t
            u.profile(False)
            sp_passes.append(p1)
            h_passes.append(p2)
            resdh.append(r)
    tk1, rho1, y1, s1, _ = u.download()
    T1 = tk1 * sc["TSTR"]
    inner = np.zeros((NZ, NR), dtype=bool)
    inner[1:-1, 1:-1] = True
    inner = inner.reshape(-1)
    report = {"peak_T": round(float(T1.max()), 3), "mean_T": round(float(T1[inner].mean()), 3),
              "mean_T_start": round(float(T0[inner].mean()), 3), "presweeps": args.presweeps,
              "cells_at_5000K": int((T1 >= 5000.0 - 1e-6).sum()), "cells_at_TKDMIN": int((T1 <= sc["TSTR"] - 1 + 1e-6).sum()),
              "sumY_drift_max": float(np.abs(y1.sum(0) + s1 - 1.0).max()),
              "rho_range": [float(rho1.min()), float(rho1.max())],
              "species_passes": sp_passes[:5] + sp_passes[-3:], "enthalpy_passes": h_passes[:5] + h_passes[-3:],
              "resdh_first_last": [resdh[0], resdh[-1]] if resdh else None,
              "ms_per_sweep_by_kind": {k: round(v / max(sweeps, 1), 3) for k, v in ms_split.items() if v > 0}}
    u.close()
    line = {"metric": "in-loop sweeps with live transport and the enthalpy equation", "value": round(n * sweeps / (ms / 1e3), 1),
            "unit": UNIT, "n_gpus": 1, "steps": sweeps, "warmup": args.warmup, "ms_per_step": round(ms / sweeps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
            "data": "synthetic (seeded C2 generator and jet flow)",
            "config": {"workload": f"C5 with live transport: 601x301 heptane field, {sweeps} sweeps of dt=1e-5 s; "
                                   "each sweep = uc_sweep (faces assembled on the device) + uc_enthalpy_update "
                                   "(SOLVEH) + uc_density", "report": report}}
    if cpu is not None:
        line["cpu_baseline_enthalpy_step"] = cpu
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cells", type=int, default=0, help="use only the first N cells (profiling runs)")
    ap.add_argument("--isor", type=int, default=ISOR, help="update passes cap (profiling runs)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "c5", "c5-live"],
                    help="c2: the species sweep of the 601x301 heptane field (headline); c3: batched stiff "
                         "integration; c4: learned surrogate with fallback; c5: in-loop sweeps; c5-live: in-loop "
                         "sweeps with live transport faces and the enthalpy equation")
    ap.add_argument("--sweeps", type=int, default=1000, help="c5: sweeps")
    ap.add_argument("--presweeps", type=int, default=200, help="c5-live: species-only sweeps before the live ones")
    ap.add_argument("--train-steps", type=int, default=2000, help="c4: Adam steps")
    args = ap.parse_args()
    if args.workload == "c3":
        main_c3(args)
    elif args.workload == "c4":
        main_c4(args)
    elif args.workload == "c5":
        main_c5(args)
    elif args.workload == "c5-live":
        main_c5_live(args)
    elif args.impl == "reference":
        main_reference(args)
    else:
        main_ours(args)


if __name__ == "__main__":
    main()
