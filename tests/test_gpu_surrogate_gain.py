"""The learned surrogate with per-cell fallback against the method without it:
the exact FP64 omega kernel alone (uc_omega), on a fresh 262,144-cell field of
the heptane distribution the network was trained on (1,048,576 states of four
other seeds, 3,000 Adam steps of 8,192).

For each tolerance the test times both paths with CUDA events on the
context's stream, measures the error of the result against the exact omega
on every cell (max over species with Y_k > 1e-8 of the error relative to
max(|omega_k|, 1e-6 max_j |omega_j|)), and prints the fallback fraction, the
speed-up and the error. It asserts what holds at every tolerance -- recomputed
cells carry the exact kernel's omega bit for bit, accepted cells the network's
-- and that the path is faster than the exact kernel once the checks accept
most cells."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOLS = (1e-3, 1e-2, 1e-1, 1.0)


def _err(q, e, y):
    wmax = np.abs(e).max(axis=0)
    r = np.abs(q - e) / np.maximum(np.abs(e), 1e-6 * wmax + 1e-300)
    r[y <= 1e-8] = 0.0
    return r.max(axis=0)


def _timed(fn, ext, reps=5):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(reps):
        fn()
    e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def test_surrogate_with_fallback_against_the_exact_kernel():
    import torch
    from unicorn_b200 import unichem
    from unicorn_b200.fields import batch_cells, nondimensional
    from unicorn_b200.surrogate import Surrogate, raw_features
    chunk, nchunk = 1 << 18, 4
    s = Surrogate(capacity=chunk * nchunk, seed=1)
    u = unichem.UniChem(chunk)
    pref = u.scales["PBACK"] * u.scales["PSTR"]
    norm, lo, hi = None, None, None
    for c in range(nchunk):
        f = batch_cells(chunk, seed=300 + c)
        tk, rho = nondimensional(f, u.scales, u.wm)
        u.upload(tk, rho, f.y)
        u.set_pressure(f.p / u.scales["PSTR"])
        feats = raw_features(f.T, f.p / pref, f.y)
        if norm is None:
            norm = Surrogate.norm_from_sample(feats, u.omega().qdsp)
            s.set_norm(**norm)
        lo = feats.min(axis=1) if lo is None else np.minimum(lo, feats.min(axis=1))
        hi = feats.max(axis=1) if hi is None else np.maximum(hi, feats.max(axis=1))
        s.add_data(u)
    norm.update(hull_lo=lo, hull_hi=hi)
    s.set_norm(**norm)
    loss = s.train(steps=3000, batch=8192, lr=1e-3, seed=3)
    assert loss[-100:].mean() < 0.1 * loss[:10].mean()
    # a fresh field of the same distribution
    f = batch_cells(chunk, seed=310)
    tk, rho = nondimensional(f, u.scales, u.wm)
    u.upload(tk, rho, f.y)
    u.set_pressure(f.p / u.scales["PSTR"])
    import ctypes

    class View(ctypes.Structure):
        _fields_ = [(k, ctypes.c_void_p) for k in ("tk", "rho", "fsp", "fsp_old", "stmf", "stnd", "rc", "qdsp", "qdot",
                                                    "domega_dy", "vmu", "vtc", "vdf", "cp", "h")] + \
                   [("n", ctypes.c_int), ("npad", ctypes.c_int), ("stream", ctypes.c_void_p)]
    v = View()
    u.lib.uc_device_view_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(View)]
    u.lib.uc_device_view_get(u._h, ctypes.byref(v))
    ext = torch.cuda.ExternalStream(v.stream)
    out = {"qdsp": np.empty((52, chunk))}
    ms_exact = _timed(lambda: u.omega(download=False), ext)
    exact = u.omega().qdsp.copy()
    s.omega(u, tol=float("inf"))
    u.download_outputs(out)
    net = out["qdsp"].copy()
    rows = []
    for tol in TOLS:
        ms = _timed(lambda: s.omega(u, tol=tol, stats=False), ext)
        st = s.omega(u, tol=tol)
        u.download_outputs(out)
        q = out["qdsp"]
        rec = np.all(q == exact, axis=0)
        assert np.all(rec | np.all(q == net, axis=0))
        e = _err(q, exact, f.y)
        acc = ~rec
        rows.append((tol, ms_exact / ms, st["cells_exact"], float(np.median(e[acc])) if acc.any() else 0.0,
                     float(np.quantile(e[acc], 0.99)) if acc.any() else 0.0,
                     float((e <= tol).mean()), st["sample_accepted_within_tol"]))
    print("\n  tol     speed-up  recomputed  accepted err p50  p99       cells within tol  (sampled estimate)")
    for r in rows:
        print(f"  {r[0]:<7g} {r[1]:8.3f}  {r[2]:10.4f}  {r[3]:16.3e}  {r[4]:9.3e}  {r[5]:16.4f}  ({r[6]:.4f})")
    loosest = rows[-1]
    assert loosest[2] < 0.2 and loosest[1] > 1.5, "with most cells accepted the surrogate path must beat the exact kernel"
    s.close()
    u.close()
