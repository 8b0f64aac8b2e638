"""Mixed-precision form (UC_MIXED) against the FP64 oracle.

The stated accuracy of the mixed form: omega_k within 1e-3 relative on
species above 1e-8 mass fraction. Where omega_k is a near-cancelling net of
large gross rates, FP32 rate terms cannot meet a relative bound on the net,
so the bound used is |d omega| <= 1e-3 * max(|omega|, 1e-4 * gross) -- the
reported statistics give the plain relative figure as well.
"""
import numpy as np
import pytest

from test_gpu_parity import gross
from unicorn_b200.fields import jet_field, nondimensional

pytestmark = pytest.mark.gpu


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
        rc32 = u.ckrates(precision=unichem.MIXED, return_rc=True)
    assert np.isfinite(om.qdsp).all() and np.isfinite(om.domega_dy).all() and np.isfinite(rc32).all()
    q, qd, h, d = oracle.omega(tk, rho, y)
    g = gross(oracle, tk, rho, y)
    mask = y > 1e-8
    err = np.abs(om.qdsp - q)
    rel = err / np.maximum(np.abs(q), 1e-300)
    frac_rel = np.mean(rel[mask] <= 1e-3)
    bound = 1e-3 * np.maximum(np.abs(q), 1e-4 * g)
    print(f"\nmixed omega: {mask.sum()} (cell,species) pairs with Y>1e-8; "
          f"{100 * frac_rel:.3f}% within 1e-3 relative; median rel {np.median(rel[mask]):.2e}; "
          f"max err/gross {np.max(err[mask] / np.maximum(g[mask], 1e-300)):.2e}")
    assert np.all(err[mask] <= bound[mask])
    assert frac_rel > 0.99
    # diagonal linearisation: all-positive sums
    assert np.allclose(om.domega_dy, d, rtol=1e-4, atol=0)
    rc64, _ = oracle.rates(tk, rho, y)
    big = np.abs(rc64) > 1e-30
    assert np.allclose(rc32[big], rc64[big], rtol=1e-5, atol=0)


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
    """Mixed-form properties (FP32 polynomials, square roots and sums) against the FP64 oracle.

    mu, lambda, D_k and cp are sums of positive terms. The median relative
    error is at most 1e-6 (the stated property accuracy); the largest is
    bounded by 1e-5 for mu, lambda and cp (FP32 rounding of the polynomials in
    T up to T^5 and of the sums over the sub-mixture) and by 3e-5 for D_k,
    whose collision integral is a quartic in T* = T/eps_ij with
    alternating-sign coefficients (main:944-952), evaluated in FP32. The
    mixture enthalpy h = sum Y_k h_k is a signed sum (formation enthalpies),
    so it is compared against the scale sum |Y_k h_k|."""
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
    print("\nmixed properties (median, max rel): " + ", ".join(f"{k} {v[0]:.1e}/{v[1]:.1e}" for k, v in stats.items()))
    for name, (med, mx) in stats.items():
        assert med <= 1e-6, (name, med)
        assert mx <= (3e-5 if name == "D_k" else 1e-5), (name, mx)
    hscale = (np.abs(yc * hk)).sum(0)
    rel_h = np.abs(out["h"] - hm) / hscale
    stats["h"] = (np.median(rel_h), rel_h.max())
    print(f"mixed h (median, max rel to sum |Y_k h_k|): {stats['h'][0]:.1e}/{stats['h'][1]:.1e}")
    assert rel_h.max() <= 1e-5
