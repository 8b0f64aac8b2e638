"""Benchmark: chem+property cell-updates/s of UNICORN's species sweep on B200,
FP64 against the mixed-precision form and the learned surrogate with fallback.

Headline workload (default): the 1M-cell heptane field -- 1,048,576 cells of
the heptane generator (fuel=11) with T ~ U[300, 2400] K and p ~ U[0.8, 1.2]
atm, seed 7. One step = one species sweep of the field from its seeded state:
Y clip + mixture-averaged transport, cp and h, the 544 rate coefficients,
omega_k and d(omega_k)/dY_k, then the point-implicit update of SOLVESP with
the reference's input-card settings (up to 100 passes, relaxation 0.99,
tolerance 1e-8) at dt = 1e-5 s. A cell-update = one cell through one such
sweep. Every step starts from the same seeded state (a device-to-device copy
inside the step), so every step does the same work, and the reference arm
runs the same sweep on chunks of the same field.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``value`` is device-resident FP64 throughput (fields already on the GPU);
``e2e`` is the same sweep through the C ABI (uc_sweep_host) with the step's
inputs copied from pinned host memory and its outputs copied back, inside
the timed region; the outputs of the properties and rates are copied while
the species update runs. ``forms`` compares, on the same field, the FP64 form with the mixed
form and with the learned surrogate plus per-cell fallback, with the error
of each against FP64; ``c2`` is the FP64 sweep of the 601x301 heptane jet
field. ``--impl reference`` times the reference's own routines (translated
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
C5_HEAD_SWEEPS = 100   # in-loop sweeps reported in the headline line (the full run: --workload c5)
HEAD_CELLS, HEAD_SEED = 1 << 20, 7
TRAIN_STATES, TRAIN_STEPS = 4 << 20, 6000
MLP_TOLS = (1e-3, 1e-2, 1e-1)


def head_field(n=HEAD_CELLS, seed=HEAD_SEED):
    from unicorn_b200.fields import batch_cells
    return batch_cells(n, seed=seed)


def head_config(n, n_gpus, extra=None):
    c = {"workload": f"{n}-cell heptane field (fuel=11, T~U[300,2400] K, p~U[0.8,1.2] atm, seed {HEAD_SEED}), one "
                     "species sweep per step from the seeded state (props, cp/h, rates, omega, domega/dY, "
                     "point-implicit update isor=100 relx=0.99 tol=1e-8, dt=1e-5 s)",
         "cells": n, "precision": "fp64",
         "l2": "inputs larger than L2 (state 453 MB, RC plane 4.6 GB at 1M cells)",
         "parallelism": f"cell-sharded x{n_gpus} (an independent field per rank)"}
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


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass


# ---------------------------------------------------------------- helpers
def peaks():
    """Measured HBM copy bandwidth and bf16 tensor throughput of this pool's B200s."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])),
                "source": "measured (MEASURED_PEAKS.json)"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback (no MEASURED_PEAKS.json)"}


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
    """The largest x over the ranks (a device tensor under NCCL, a host one under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def omega_rel_error(q, exact, y):
    """Relative error of QDSP per (cell, species) on species above 1e-8 mass fraction, with a floor of
    1e-6 x the cell's largest |omega| (a stated near-zero net); the flat array of those pairs."""
    wmax = np.abs(exact).max(axis=0)
    r = np.abs(q - exact) / np.maximum(np.abs(exact), 1e-6 * wmax + 1e-300)
    return r[y > 1e-8]


def err_summary(r, tol=1e-3):
    return {"p50": float(np.median(r)), "p99": float(np.quantile(r, 0.99)), "max": float(r.max()),
            "frac_le_1e-3": round(float((r <= tol).mean()), 6)}


class DeviceState:
    """The seeded state of a field kept on the device; restore() loads it into a context (asynchronous,
    on the context's stream)."""

    def __init__(self, u, tk, rho, y, dev):
        import torch
        self.t = {"tk": torch.from_numpy(np.ascontiguousarray(tk)).to(dev),
                  "rho": torch.from_numpy(np.ascontiguousarray(rho)).to(dev),
                  "y": torch.from_numpy(np.ascontiguousarray(y)).to(dev)}
        torch.cuda.synchronize(dev)
        self.u = u

    def restore(self):
        t = self.t
        self.u.upload_device(t["tk"].data_ptr(), t["rho"].data_ptr(), t["y"].data_ptr(), None, None, self.u.n)


def time_sweeps(u, st, ext, prec, steps, warmup, isor=ISOR, clocks=None):
    """K sweeps, each from the seeded state, bracketed by CUDA events on the context's stream."""
    import torch
    for _ in range(warmup):
        st.restore()
        u.sweep(DT, precision=prec, isor=isor, relx=RELX, tol=TOL)
    u.sync()
    u.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    passes = []
    with (clocks if clocks is not None else _Null()):
        e0.record(ext)
        for _ in range(steps):
            st.restore()
            passes.append(u.sweep(DT, precision=prec, isor=isor, relx=RELX, tol=TOL))
        e1.record(ext)
        e1.synchronize()
    kt = u.profile_read()
    u.profile(False)
    return e0.elapsed_time(e1), passes, kt


def time_calls(fn, ext, reps, warmup):
    """Mean device time (ms) of fn() over reps calls after warmup calls."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(reps):
        fn()
    e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def fp64_fma_peak(dev):
    """FP64 FMA throughput of this GPU, measured: an elementwise kernel of four independent chains of 256
    fused multiply-adds per element over 2^26 doubles (torch's jiterator compiles it), best of 5, CUDA
    events. TFLOP/s, counting an FMA as two operations; None if the kernel cannot be built."""
    try:
        import torch
        code = ("template <typename T> T fma_loop(T x, T a, T b) {"
                " T y0 = x, y1 = x + T(1), y2 = x + T(2), y3 = x + T(3);"
                " for (int i = 0; i < 256; ++i) { y0 = y0 * a + b; y1 = y1 * a + b; y2 = y2 * a + b; y3 = y3 * a + b; }"
                " return y0 + y1 + y2 + y3; }")
        fn = torch.cuda.jiterator._create_jit_fn(code)
        x = torch.rand(1 << 26, dtype=torch.float64, device=dev)
        a = torch.full_like(x, 0.999)
        b = torch.full_like(x, 1e-3)
        fn(x, a, b)
        torch.cuda.synchronize(dev)
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn(x, a, b)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return (1 << 26) * 4 * 256 * 2 / (best / 1e3) / 1e12
    except Exception:
        return None


# DRAM read + write of one launch of the tile-resident update under ncu (65,536 cells of the benchmark
# field, 16 passes: 367 MB + 412 MB), per cell and pass; scaled to a launch by cells x passes run
UPDATE_DRAM_PER_CELL_PASS = (367.4e6 + 412.3e6) / (65536 * 16)


def roofline(kt, n, passes_run, pk, flops_per_cell_pass, fp64_peak):
    """Dominant kernel of the FP64 sweep and its achieved rate against its bound: the species update
    holds each tile's RC block on chip across passes and is bound by the FP64 pipe, the others by HBM."""
    name = max(kt, key=lambda k: kt[k][0])
    ms, cnt = kt[name]
    if name == "update":
        flops = flops_per_cell_pass * passes_run * n
        achieved = flops / (ms / cnt / 1e3) / 1e12
        peak = fp64_peak if fp64_peak else 37.0
        return {"kernel": name, "bound": "fp64", "achieved": round(achieved, 3), "peak": round(peak, 2),
                "peak_source": "measured in this run: FP64 FMA loop (bench.py fp64_fma_peak)" if fp64_peak else
                "nominal B200 FP64 (the measurement did not run)", "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4), "traffic": round(UPDATE_DRAM_PER_CELL_PASS * n * passes_run),
                "flops_per_launch": flops, "avg_launch_ms": round(ms / cnt, 4),
                "flops_rule": f"{flops_per_cell_pass} operations per cell and pass (each multiplication, addition "
                              f"and division of the update program one) x {passes_run:.1f} passes x {n} cells"}
    if name == "chem":
        per_cell = (52 + 4) * 8 + (544 + 52 + 52 + 1 + 6) * 8
        rule = "per cell: read T, rho, soot, Y (56 x 8 B); write RC 544, QDSP 52, dw/dY 52, QDOT, SOUR 6"
    else:
        per_cell = (54 + 54) * 8
        rule = "per cell: 54 inputs + 54 outputs x 8 B"
    achieved = per_cell * n / (ms / cnt / 1e3) / 1e9
    return {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"],
            "peak_source": pk["source"], "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4),
            "traffic": None, "bytes_per_launch": per_cell * n, "avg_launch_ms": round(ms / cnt, 4),
            "bytes_rule": rule}


# ---------------------------------------------------------------- CPU baselines
def cpu_baseline_port(tk, rho, y, ns=1024):
    """The oracle (a faithful FP64 C restatement) on one host core, bounded sample."""
    from oracle.oracle import Oracle
    o = Oracle()
    tk, rho, y = tk[:ns].copy(), rho[:ns].copy(), np.ascontiguousarray(y[:, :ns])
    t0 = time.perf_counter()
    yc, mu, lam, dk, _ = o.props(tk, y)
    o.cp(tk, yc)
    o.enthalpy(tk, yc)
    o.omega(tk, rho, yc)
    rc, sour = o.rates(tk, rho, yc)
    yn, s, passes = o.species_update(rho, yc, rc, sour, DT, isor=ISOR, relx=RELX, tol=TOL)
    dt = time.perf_counter() - t0
    return {"value": round(ns / dt, 1), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"first {ns} cells of the field, one full sweep (oracle/unichem_oracle.c, -O2, 1 thread; "
                      f"{passes} update passes), {dt:.2f} s"}


def cpu_baseline_reference(tk, rho, y):
    """The reference's own routines (translated to C, oracle/_ref) on one host core: one chunk of the
    field through one full sweep (props, cp, omega, rates and the point-implicit update). Falls back to
    the oracle port where the translation is not built."""
    from oracle import ref as R
    if not R.available():
        return cpu_baseline_port(tk, rho, y)
    r = R.RefUnicorn()
    ns = r.chunk
    tk, rho, y = tk[:ns].copy(), rho[:ns].copy(), np.ascontiguousarray(y[:, :ns])
    t0 = time.perf_counter()
    yc, mu, lam, vdf = r.props(tk, y)
    r.cp(tk, yc)
    r.omega(tk, rho, yc)
    yn, s1, s2, passes = r.species_update(tk, rho, yc, DT, isor=ISOR, relx=RELX, tol=TOL)
    dt = time.perf_counter() - t0
    return {"value": round(ns / dt, 1), "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"first {ns} cells of the field, one full sweep (the reference's routines translated to C, "
                      f"oracle/_ref, 1 thread; {passes} update passes), {dt:.2f} s"}


def _ref_worker(args_tuple):
    """One host process: the reference's own routines on a chunk of cells (one full sweep)."""
    tk, rho, y, isor = args_tuple
    from oracle.ref import RefUnicorn
    r = _ref_worker.r if hasattr(_ref_worker, "r") else None
    if r is None:
        r = _ref_worker.r = RefUnicorn()
    t0 = time.perf_counter()
    yc, mu, lam, vdf = r.props(tk, y)
    r.cp(tk, yc)
    r.omega(tk, rho, yc)
    yn, s1, s2, passes = r.species_update(tk, rho, yc, DT, isor=isor, relx=RELX, tol=TOL)
    return len(tk), time.perf_counter() - t0, passes


def reference_steps(tk, rho, y, steps, warmup, cores=None):
    """The reference's routines on all host cores, one process per core, each step one chunk per core
    (consecutive chunks of the field); returns (cells, seconds, passes per chunk)."""
    import multiprocessing as mp
    from oracle import ref as R
    chunk = R.RefUnicorn().chunk
    cores = cores or os.cpu_count() or 1
    n = len(tk)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        def one_step(step):
            jobs = []
            for w in range(cores):
                a = ((step * cores + w) * chunk) % (n - chunk)
                jobs.append((tk[a:a + chunk].copy(), rho[a:a + chunk].copy(), np.ascontiguousarray(y[:, a:a + chunk]),
                             ISOR))
            t0 = time.perf_counter()
            out = pool.map(_ref_worker, jobs)
            return sum(o[0] for o in out), time.perf_counter() - t0, [o[2] for o in out]
        pool.map(_ref_worker, [(tk[:64].copy(), rho[:64].copy(), np.ascontiguousarray(y[:, :64]), 1)] * cores)
        for w in range(warmup):
            one_step(w)
        cells, secs, passes = 0, 0.0, []
        for s in range(steps):
            c, t, p = one_step(warmup + s)
            cells += c
            secs += t
            passes += p
    return cells, secs, passes, chunk, cores


# ---------------------------------------------------------------- surrogate
def train_surrogate(ntrain, steps, chunk=1 << 20, seed0=100):
    """Training set of exact FP64 omega on states of the C3/C4 distribution (seeds seed0..), then Adam."""
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import batch_cells, nondimensional
    from unicorn_b200.surrogate import Surrogate, raw_features
    chunk = min(ntrain, chunk)
    t0 = time.perf_counter()
    s = Surrogate(capacity=ntrain, seed=1)
    u = unichem.UniChem(chunk)
    hull_lo, hull_hi, norm = None, None, None
    for c in range(ntrain // chunk):
        f = batch_cells(chunk, seed=seed0 + c)
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
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = s.train(steps=steps, batch=8192, lr=1e-3, seed=3)
    t_train = time.perf_counter() - t0
    info = {"train_states": ntrain, "train_steps": steps, "batch": 8192, "lr": 1e-3, "train_s": round(t_train, 2),
            "data_s": round(t_data, 2), "train_samples_per_s": round(steps * 8192 / t_train, 1),
            "loss_first": float(loss[:10].mean()), "loss_last": float(loss[-50:].mean())}
    return s, info


# ---------------------------------------------------------------- our arm
def run_c2(args, dev, pk):
    """The FP64 sweep of the 601x301 heptane jet field, each step from the seeded state."""
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import jet_field, nondimensional
    f = jet_field(NZ, NR, fuel=FUEL, t_peak=TPEAK, seed=0)
    u = unichem.UniChem(f.n, device=dev)
    tk, rho = nondimensional(f, u.scales, u.wm)
    st = DeviceState(u, tk, rho, f.y, dev)
    ext = torch.cuda.ExternalStream(unichem_view(u)["stream"], device=dev)
    ms, passes, kt = time_sweeps(u, st, ext, unichem.FP64, args.steps, args.warmup)
    u.close()
    return {"workload": "601x301 heptane jet field (fuel=11, T_peak 2300 K, seed 0), FP64 sweep from the seeded state",
            "cells": f.n, "value": round(f.n * args.steps / (ms / 1e3), 1), "ms_per_step": round(ms / args.steps, 3),
            "update_passes_per_step": passes,
            "kernel_ms_per_step": {k: round(v[0] / args.steps, 3) for k, v in kt.items() if v[1]}}


def run_forms(args, u, st, ext, f, tk, rho, fp64_sweep_ms, dev, pk):
    """FP64 against the mixed form and the surrogate with per-cell fallback on the same field:
    sweep and omega+property throughput and the error of each against FP64."""
    from unicorn_b200 import unichem
    n = f.n
    res = {}
    # mixed sweep
    ms_mx, passes_mx, kt_mx = time_sweeps(u, st, ext, unichem.MIXED, args.steps, args.warmup)
    fp64_tiles = u.stat("mixed_fp64_tiles") / u.stat("tiles")
    # omega and properties of the seeded state, FP64 and mixed (outputs compared on the host)
    out, evals = {}, {}
    for name, prec in (("fp64", unichem.FP64), ("mixed", unichem.MIXED)):
        st.restore()
        evals[name] = time_calls(lambda prec=prec: u.chem_props(prec), ext, args.steps, args.warmup)
        st.restore()
        u.chem_props(prec)
        d = {k: np.empty((52, n)) if k in ("qdsp", "vdf") else np.empty(n) for k in ("qdsp", "vmu", "vtc", "vdf", "cp", "h")}
        u.download_outputs(d)
        out[name] = d
    ex, mx = out["fp64"], out["mixed"]
    r_mx = omega_rel_error(mx["qdsp"], ex["qdsp"], f.y)
    prop_err = {k: float((np.abs(mx[k] - ex[k]) / np.abs(ex[k])).max()) for k in ("vmu", "vtc", "vdf", "cp")}
    big = np.abs(ex["h"]) > 1e-3 * np.abs(ex["h"]).max()
    prop_err["h"] = float((np.abs(mx["h"] - ex["h"])[big] / np.abs(ex["h"][big])).max())
    res["fp64"] = {"sweep_cell_updates_per_s": round(n * args.steps / (fp64_sweep_ms / 1e3), 1),
                   "omega_props_ms": round(evals["fp64"], 3),
                   "omega_props_cell_updates_per_s": round(n / (evals["fp64"] / 1e3), 1)}
    res["mixed"] = {"sweep_cell_updates_per_s": round(n * args.steps / (ms_mx / 1e3), 1),
                    "sweep_speedup_vs_fp64": round(fp64_sweep_ms / ms_mx, 3),
                    "update_passes_per_step": passes_mx, "fp64_fallback_tiles": round(fp64_tiles, 4),
                    "omega_props_ms": round(evals["mixed"], 3),
                    "omega_props_cell_updates_per_s": round(n / (evals["mixed"] / 1e3), 1),
                    "omega_props_speedup_vs_fp64": round(evals["fp64"] / evals["mixed"], 3),
                    "omega_err_vs_fp64": err_summary(r_mx), "props_max_rel_err_vs_fp64": prop_err,
                    "kernel_ms_per_step": {k: round(v[0] / args.steps, 3) for k, v in kt_mx.items() if v[1]}}
    # surrogate with per-cell fallback
    if args.no_mlp:
        return res
    try:
        s, info = train_surrogate(args.train_states, args.train_steps)
        u.set_pressure(f.p / u.scales["PSTR"])
        ml = {"training": info}
        for tol in MLP_TOLS + (float("inf"),):
            def ev(tol=tol):
                u.props(download=False)
                u.cp_h(download=False)
                s.omega(u, tol=tol, stats=False)
            st.restore()
            ms = time_calls(ev, ext, args.steps, args.warmup)
            st.restore()
            u.props(download=False)
            stt = s.omega(u, tol=tol)
            q = {"qdsp": np.empty((52, n))}
            u.download_outputs(q)
            r = omega_rel_error(q["qdsp"], ex["qdsp"], f.y)
            key = "network_alone" if tol == float("inf") else f"tol={tol:g}"
            ml[key] = {"omega_props_ms": round(ms, 3), "omega_props_cell_updates_per_s": round(n / (ms / 1e3), 1),
                       "omega_props_speedup_vs_fp64": round(evals["fp64"] / ms, 3), "fallback": stt,
                       "omega_err_vs_fp64": err_summary(r)}
        s.close()
        res["mlp_fallback"] = ml
    except Exception as e:          # the headline stands; the failure is reported in the line
        res["mlp_fallback"] = {"error": f"{type(e).__name__}: {e}"}
    return res


def main_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(dev)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from unicorn_b200 import unichem
    from unicorn_b200.fields import nondimensional
    pk = peaks()
    f = head_field(args.cells or HEAD_CELLS, seed=HEAD_SEED + rank)
    n = f.n
    u = unichem.UniChem(n, device=dev)
    tk, rho = nondimensional(f, u.scales, u.wm)
    st = DeviceState(u, tk, rho, f.y, dev)
    ext = torch.cuda.ExternalStream(unichem_view(u)["stream"], device=dev)
    # ---------------- device-resident FP64 sweeps (the headline)
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = ClockSampler(dev)
    ms, passes, kt = time_sweeps(u, st, ext, unichem.FP64, args.steps, args.warmup, isor=args.isor, clocks=clk)
    ms = max_over_ranks(ms, world)
    # ---------------- end to end through the C ABI (pinned host buffers in and out)
    pin = lambda *s: torch.empty(s, dtype=torch.float64, pin_memory=True).numpy()
    h_tk, h_rho, h_y = pin(n), pin(n), pin(52, n)
    h_tk[:], h_rho[:], h_y[:] = tk, rho, f.y
    outs = dict(qdsp=pin(52, n), qdot=pin(n), domega_dy=pin(52, n), vmu=pin(n), vtc=pin(n), vdf=pin(52, n),
                cp=pin(n), h=pin(n))
    h_yout = pin(52, n)
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    e2e_passes = []
    for _ in range(args.steps):
        # uc_sweep_host: upload, sweep, outputs copied back while the species update runs, updated Y
        e2e_passes.append(u.sweep_host(h_tk, h_rho, h_y, out=outs, y_out=h_yout, dt=DT, precision=unichem.FP64,
                                       isor=args.isor, relx=RELX, tol=TOL))
    u.sync()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    passes_run = float(np.mean([min(p, args.isor) for p in passes]))
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": round(world * n * args.steps / (ms / 1e3), 1), "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded heptane-generator field; the reference ships no benchmark data)",
                "config": head_config(n, world, {"update_passes_per_step": passes, "e2e_update_passes": e2e_passes}),
                "e2e": {"value": round(world * n * args.steps / e2e_s, 1), "unit": UNIT,
                        "h2d_bytes_per_step": (2 + 52) * 8 * n, "d2h_bytes_per_step": (52 * 4 + 5) * 8 * n},
                "gpu_launches": world * sum(c for _, c in kt.values()), "clocks": clk.summary(),
                "roofline": roofline(kt, n, passes_run, pk, u.stat("update_flops_per_cell_pass"), fp64_fma_peak(dev)),
                "kernel_ms_per_step": {k: round(v[0] / args.steps, 3) for k, v in kt.items() if v[1]}}
    # ---------------- the three forms and the C2 field (rank 0 of a one-GPU run)
    if rank == 0 and world == 1:
        if not args.no_forms:
            line["forms"] = run_forms(args, u, st, ext, f, tk, rho, ms, dev, pk)
        u.close()
        if not args.no_c2:
            line["c2"] = run_c2(args, dev, pk)
        if not args.no_c5:
            line["c5"] = run_c5(args, C5_HEAD_SWEEPS)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_reference(tk, rho, f.y)
        print(json.dumps(line), flush=True)
    else:
        u.close()
        if rank == 0:
            print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- reference arm
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
    from unicorn_b200.fields import nondimensional
    r0 = R.RefUnicorn()
    f = head_field(args.cells or HEAD_CELLS)
    tk, rho = nondimensional(f, r0.scales, r0.wm)
    cells, secs, passes, chunk, cores = reference_steps(tk, rho, f.y, args.steps, args.warmup)
    v = cells / secs
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(secs / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded heptane-generator field)",
        "config": head_config(f.n, 1, {"update_passes_per_chunk": passes}),
        "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": cores, "kind": "reference",
                         "per_core": round(v / cores, 1),
                         "sample": f"{cores} chunks of {chunk} cells of the field per step, one process per core, "
                                   "each running the reference's property block, TCP, CKRATES, SOLVEH rates and "
                                   "SOLVESP (translated from its Fortran, gcc -O2)"},
        "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


# ---------------------------------------------------------------- C3: batched stiff integration
C3_CELLS = 1 << 20
NSUB_MAX = 200                       # the sub-step cap of the C3 options (UniChem.integrate default)


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
    prec = unichem.MIXED if args.precision == "mixed" else unichem.FP64
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
    fp64_m = fp64_fma_peak(0)
    fp64 = fp64_m or 37.0
    substeps = float(ns.sum())
    per_sub_flop = 9.0e3 + 470 + 2 * 2189 * float(pa.sum()) / substeps
    achieved = per_sub_flop * substeps / (ms / args.steps / 1e3) / 1e12
    line = {"metric": "batched stiff integration cell-updates/s (one cell over dt = 1e-5 s)",
            "value": round(n * args.steps / (ms / 1e3), 1), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == unichem.FP64 else "f32 rates / f64 update", "data": "synthetic (seeded C3 generator)",
            "config": {"workload": f"C3: {n} independent heptane-generator cells, T~U[300,2400] K, p~U[0.8,1.2] atm, "
                                   "dt=1e-5 s, n_sub=clamp(ceil(max_k dt|w_k|/Y_k over Y_k>1e-3), 1, 200), "
                                   f"update passes to 1e-8 per sub-step (<={args.isor})",
                       "cells": n, "precision": args.precision, "tuned": tune,
                       "nsub": {"mean": round(float(ns.mean()), 2), "min": int(ns.min()), "max": int(ns.max()),
                                "frac_1": round(float((ns == 1).mean()), 4),
                                "frac_max": round(float((ns == ns.max()).mean()), 4)},
                       "passes_per_substep": round(float(pa.sum()) / substeps, 2),
                       "shape": ("rounds form (field kernels per sub-step round; cells in n_sub order, "
                                 "re-sorted by the passes of their last sub-step between rounds)"
                                 if tune["int_warps"] == 3 else
                                 f"persistent work-queue kernel, {int(tune['int_warps'])} warps"),
                       "l2": ("state 470 MB > L2; RC plane 4.6 GB written and read back per round"
                              if tune["int_warps"] == 3 else "state 470 MB > L2; all sub-step work on chip")},
            "e2e": {"value": round(n * args.steps / e2e, 1), "unit": UNIT, "h2d_bytes_per_step": (2 + 52) * 8 * n,
                    "d2h_bytes_per_step": (2 + 52) * 8 * n},
            # per step: rates of the start state, n_sub, the sort (3), then the persistent kernel, or the round
            # counts, gather, held enthalpy, 3 kernels per round (one round per possible sub-step), 5 for the
            # re-sort between rounds, and the scatter
            "gpu_launches": kt["integrate"][1] * ((4 + 8 * NSUB_MAX) if tune["int_warps"] == 3 else
                                                  (6 if tune["int_sorted"] else 3)),
            "clocks": clk.summary(),
            "roofline": {"kernel": "integrate", "bound": "fp64", "achieved": round(achieved, 3), "peak": round(fp64, 2),
                         "peak_source": "measured in this run: FP64 FMA loop (bench.py fp64_fma_peak)" if fp64_m else
                         "nominal B200 FP64 (the measurement did not run)", "unit": "TFLOP/s",
                         "frac": round(achieved / fp64, 4), "traffic": None,
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
    ntrain = args.cells * 4 if args.cells else args.train_states
    nfield = args.cells or C4_FIELD
    steps = args.train_steps
    s, tinfo = train_surrogate(ntrain, steps)
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

    pk = peaks()
    ms_exact, _ = timed(lambda: u.omega(download=False), args.steps)
    u.download_outputs(out)
    exact = out["qdsp"].copy()
    res = {}
    with ClockSampler(0) as clk:
        for tol in MLP_TOLS + (float("inf"),):
            ms, _ = timed(lambda: s.omega(u, tol=tol, stats=False), args.steps)
            stt = s.omega(u, tol=tol)
            u.download_outputs(out)
            r = omega_rel_error(out["qdsp"], exact, f.y)
            key = "network_alone" if tol == float("inf") else f"tol={tol:g}"
            res[key] = {"ms": round(ms, 3), "cell_updates_per_s": round(nfield / (ms / 1e3), 1),
                        "speedup_vs_fp64": round(ms_exact / ms, 3), "fallback": stt,
                        "omega_err_vs_fp64": err_summary(r)}
    u.close()
    s.close()
    pure = res["network_alone"]          # features, 5 tensor-core layers, decode
    tflops = MLP_FLOP_PER_CELL * nfield / (pure["ms"] / 1e3) / 1e12
    line = {"metric": "omega cell-updates/s: learned surrogate + per-cell FP64 fallback at the stated error",
            "value": res["tol=0.001"]["cell_updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["tol=0.001"]["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network / f64 fallback", "data": "synthetic (seeded C3/C4 generators)",
            "config": {"workload": f"C4: network 54-256x4-52 GELU, Adam batch 8192, {steps} steps on {ntrain} "
                                   f"exact-FP64 states of the C3 distribution; inference on a fresh {nfield}-cell field "
                                   "with per-cell fallback to the exact FP64 kernel",
                       "fp64_omega_ms": round(ms_exact, 3),
                       "fp64_omega_cell_updates_per_s": round(nfield / (ms_exact / 1e3), 1),
                       "by_tolerance": res, "training": tinfo},
            "e2e": None, "gpu_launches": None, "clocks": clk.summary(),
            "roofline": {"kernel": "surrogate forward (features, 5 tensor-core layers, decode; network alone)",
                         "bound": "tensor", "achieved": round(tflops, 2), "peak": pk["bf16_tflops"],
                         "peak_source": pk["source"] + ", bf16 burst", "unit": "TFLOP/s",
                         "frac": round(tflops / pk["bf16_tflops"], 4), "traffic": None,
                         "flops_rule": f"{MLP_FLOP_PER_CELL} flop per cell (padded 64-256x4-64 layers) / forward time"}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- C5: in-loop sweeps
def run_c5(args, sweeps):
    """The in-loop C5 run over `sweeps` sweeps: timing and checkpoint report of the FP64 and mixed forms
    (with the omega errors of the mixed kernel and the surrogate at the checkpoints)."""
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import jet_field, nondimensional
    from unicorn_b200.inloop import frozen_faces, omega_error
    from unicorn_b200.surrogate import Surrogate, raw_features
    f = jet_field(NZ, NR, fuel=FUEL, t_peak=TPEAK, seed=0)
    n = f.n
    checkpoints = sorted({c for c in (100, 500, 1000, sweeps) if c <= sweeps})
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
        for sw in range(1, sweeps + 1):
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
                              "mlp_cells_exact_at_1e-3": round(fb["cells_exact"], 4)})
                rep[f"sweep_{sw}"] = entry
        timing[name] = {"ms_per_sweep": round(ms_total / sweeps, 3),
                        "cell_updates_per_s": round(n * sweeps / (ms_total / 1e3), 1)}
        report[name] = rep
        u.close()
    probe.close()
    s.close()
    return {"workload": f"C5: 601x301 heptane field, {sweeps} sweeps of dt=1e-5 s, transport frozen "
                        "(diffusion faces from the initial field), T from held enthalpy each sweep",
            "timing": timing, "report": report,
            "surrogate": {"train_steps": args.train_steps, "train_states": 4 * n,
                          "loss_first": float(loss[:10].mean()), "loss_last": float(loss[-50:].mean())}}


def main_c5(args):
    c5 = run_c5(args, args.sweeps)
    fp = c5["timing"]["fp64"]
    line = {"metric": "in-loop heptane sweeps: peak-T drift, sum-Y drift and omega error at sweeps 100/500/1000",
            "value": fp["cell_updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.sweeps, "warmup": 0,
            "ms_per_step": fp["ms_per_sweep"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (and mixed)", "data": "synthetic (seeded C2 generator)", "config": c5}
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
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"], help="c3, c5-live: precision")
    ap.add_argument("--workload", default="head", choices=["head", "c3", "c4", "c5", "c5-live"],
                    help="head: the species sweep of the 1M-cell heptane field with the FP64 / mixed / surrogate "
                         "comparison and the 601x301 field (headline); c3: batched stiff integration; c4: learned "
                         "surrogate with fallback; c5: in-loop sweeps; c5-live: in-loop sweeps with live transport "
                         "faces and the enthalpy equation")
    ap.add_argument("--sweeps", type=int, default=1000, help="c5: sweeps")
    ap.add_argument("--presweeps", type=int, default=200, help="c5-live: species-only sweeps before the live ones")
    ap.add_argument("--train-steps", type=int, default=TRAIN_STEPS, help="surrogate: Adam steps")
    ap.add_argument("--train-states", type=int, default=TRAIN_STATES, help="surrogate: training states")
    ap.add_argument("--no-forms", action="store_true", help="head: skip the mixed / surrogate comparison")
    ap.add_argument("--no-mlp", action="store_true", help="head: skip the surrogate")
    ap.add_argument("--no-c2", action="store_true", help="head: skip the 601x301 field")
    ap.add_argument("--no-c5", action="store_true", help="head: skip the in-loop sweeps of the 601x301 field")
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
