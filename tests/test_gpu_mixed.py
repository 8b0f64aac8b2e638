"""Mixed-precision form (UC_MIXED) against the FP64 oracle, at the stated accuracy.

Stated accuracy of the mixed form: omega_k within 1e-3 relative on every
(cell, species) with Y_k > 1e-8, where the only floor is the stated
near-zero net: |omega_k| below 1e-6 of the cell's largest |omega_j| is
measured against that 1e-6 max|omega_j|; the transport properties, cp and h
within 1e-6 relative on every cell.
"""
import numpy as np
import pytest

from unicorn_b200.fields import batch_cells, jet_field, nondimensional

pytestmark = pytest.mark.gpu


def omega_bound_ok(q, exact, y, tol=1e-3):
    """|q - exact| <= tol * max(|exact|, 1e-6 max_j |exact_j|) on species above 1e-8; (ok mask, rel)."""
    wmax = np.abs(exact).max(axis=0, keepdims=True)
    rel = np.abs(q - exact) / np.maximum(np.abs(exact), 1e-6 * wmax + 1e-300)
    mask = y > 1e-8
    return rel[mask], mask


@pytest.fixture(scope="module")
def c2_slice(oracle):
    f = jet_field(601, 301, fuel=11, t_peak=2300.0, seed=0)     # C2 generator; every 23rd cell
    sel = np.arange(0, f.n, 23)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    return tk[sel].copy(), rho[sel].copy(), np.ascontiguousarray(f.y[:, sel])


def test_mixed_omega_error(oracle, c2_slice):
    from unicorn_b200 import unichem
    tk, rho, y = c2_slice
    with unichem.UniChem(len(tk)) as u:
        u.upload(tk, rho, y)
        om = u.omega(precision=unichem.MIXED)
        fp64_tiles = u.stat("mixed_fp64_tiles") / u.stat("tiles")
        rc32 = u.ckrates(precision=unichem.MIXED, return_rc=True)
    assert np.isfinite(om.qdsp).all() and np.isfinite(om.domega_dy).all() and np.isfinite(rc32).all()
    q, qd, h, d = oracle.omega(tk, rho, y)
    rel, mask = omega_bound_ok(om.qdsp, q, y)
    print(f"\nmixed omega on the C2 slice: {mask.sum()} (cell, species) pairs with Y>1e-8; max rel {rel.max():.2e}, "
          f"median {np.median(rel):.2e}; tiles recomputed in FP64 {100 * fp64_tiles:.1f}%")
    assert rel.max() <= 1e-3
    # diagonal linearisation: all-positive sums
    assert np.allclose(om.domega_dy, d, rtol=1e-4, atol=0)
    rc64, _ = oracle.rates(tk, rho, y)
    big = np.abs(rc64) > 1e-30
    assert np.allclose(rc32[big], rc64[big], rtol=1e-5, atol=0)


def test_mixed_omega_and_properties_on_the_1m_field():
    """The mixed form against the FP64 form (itself pinned to the oracle at 1e-11) on every 4th cell of
    the 1M-cell heptane benchmark field: omega and every property at the stated bounds."""
    from unicorn_b200 import unichem
    f = batch_cells(1 << 20, seed=7)
    sel = np.arange(0, f.n, 4)
    out = {}
    with unichem.UniChem(len(sel)) as u:
        tk, rho = nondimensional(f, u.scales, u.wm)
        tk, rho, y = tk[sel].copy(), rho[sel].copy(), np.ascontiguousarray(f.y[:, sel])
        for prec in (unichem.FP64, unichem.MIXED):
            u.upload(tk, rho, y)
            u.chem_props(prec)
            d = {k: np.empty((52, len(sel))) if k in ("qdsp", "vdf") else np.empty(len(sel))
                 for k in ("qdsp", "vmu", "vtc", "vdf", "cp", "h")}
            u.download_outputs(d)
            out[prec] = d
        fp64_tiles = u.stat("mixed_fp64_tiles") / u.stat("tiles")
    ex, mx = out[unichem.FP64], out[unichem.MIXED]
    rel, mask = omega_bound_ok(mx["qdsp"], ex["qdsp"], y)
    print(f"\n1M field (every 4th cell): omega max rel {rel.max():.2e}; tiles recomputed in FP64 {100 * fp64_tiles:.1f}%")
    assert rel.max() <= 1e-3
    for k in ("vmu", "vtc", "vdf", "cp", "h"):
        r = np.abs(mx[k] - ex[k]) / np.abs(ex[k])
        print(f"  {k}: max rel {r.max():.2e}")
        assert r.max() <= 1e-6, (k, r.max())


def test_mixed_sweep_vs_fp64_sweep(oracle, c2_slice):
    """The whole sweep in mixed form (FP32 RC plane, FP64 update) against the FP64 sweep."""
    from unicorn_b200 import unichem
    tk, rho, y = c2_slice
    out = {}
    for prec in (unichem.FP64, unichem.MIXED):
        with unichem.UniChem(len(tk)) as u:
            u.upload(tk, rho, y)
            passes = u.sweep(1e-3, precision=prec, isor=30, tol=0.0)
            _, _, yn, _, _ = u.download()
            out[prec] = (yn, passes)
    y64, y32 = out[unichem.FP64][0], out[unichem.MIXED][0]
    assert out[unichem.FP64][1] == out[unichem.MIXED][1] == 31
    mask = y64 > 1e-8
    rel = np.abs(y32 - y64)[mask] / y64[mask]
    print(f"\nmixed sweep: Y after 30 passes, median rel {np.median(rel):.2e}, max rel {rel.max():.2e}")
    assert np.all(rel <= 1e-3)


def test_mixed_properties_vs_oracle(oracle, c2_slice):
    """Mixed-form properties (FP32 per-pair terms of the transport sums; polynomials, sums, cp and h in
    FP64) against the FP64 oracle: every cell within 1e-6 relative. The mixture enthalpy h = sum Y_k h_k
    is a signed sum (formation enthalpies); it is compared against |h| where |h| is above 1e-3 of the
    field's largest, and against the scale sum |Y_k h_k| everywhere."""
    from unicorn_b200 import unichem
    tk, rho, y = c2_slice
    with unichem.UniChem(len(tk)) as u:
        u.upload(tk, rho, y)
        u.sweep(1e-3, precision=unichem.MIXED, isor=1, tol=0.0)
        out = {k: np.empty((52, len(tk))) if k == "vdf" else np.empty(len(tk)) for k in ("vmu", "vtc", "vdf", "cp", "h")}
        u.download_outputs(out)
    yc, mu, lam, dk, _ = oracle.props(tk, y)
    cp = oracle.cp(tk, yc)
    hk, hm = oracle.enthalpy(tk, yc)
    stats = {}
    for name, a, b in (("mu", out["vmu"], mu), ("lambda", out["vtc"], lam), ("D_k", out["vdf"], dk), ("cp", out["cp"], cp)):
        rel = np.abs(a - b) / np.abs(b)
        stats[name] = (np.median(rel), rel.max())
    big = np.abs(hm) > 1e-3 * np.abs(hm).max()
    rel_h = np.abs(out["h"] - hm)[big] / np.abs(hm[big])
    stats["h"] = (np.median(rel_h), rel_h.max())
    print("\nmixed properties (median, max rel): " + ", ".join(f"{k} {v[0]:.1e}/{v[1]:.1e}" for k, v in stats.items()))
    for name, (med, mx) in stats.items():
        assert mx <= 1e-6, (name, mx)
    hscale = (np.abs(yc * hk)).sum(0)
    assert (np.abs(out["h"] - hm) / hscale).max() <= 1e-6
