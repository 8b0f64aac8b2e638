"""CUDA path (libunichem.so through its C ABI) against the FP64 oracle.

Tolerances (FP64 kernels; the GPU's exp/log/pow differ from the host libm by
an ulp or so, and nvcc contracts multiply-adds into FMAs):
  RC, d(omega)/dY, cp, h, mu, lambda, D_k    relative 1e-11
  QDSP (net rates) and QDOT                  1e-11 of the gross rate
                                             (sum of |terms|), since the net
                                             value can cancel to ~0
  species update (fixed pass count)          1e-9 relative, 1e-18 absolute
  T from h                                   2e-3 K (the Newton stopping rule)
"""
import numpy as np
import pytest

from conftest import random_state
from unicorn_b200.fields import batch_cells, jet_field, nondimensional, sensible_enthalpy

pytestmark = pytest.mark.gpu

RTOL = 1e-11


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


def gross(oracle, tk, rho, y):
    """Per species and cell: RCONV*W_k*sum |terms| of its PRD list (scale of QDSP)."""
    rc, _ = oracle.rates(tk, rho, y)
    m = oracle.mech
    ra = np.zeros_like(rc)
    for key, sps in m["ra"].items():
        r = int(key) - 1
        if sps is None:
            continue
        v = rc[r].copy()
        for s in sps:
            v = v * y[s - 1]
        ra[r] = v
    g = np.zeros((52, len(tk)))
    for key, terms in m["prd"].items():
        k = int(key) - 1
        if not terms:
            continue
        for s, fac in terms:
            for f in fac:
                if f[0] == "RA":
                    g[k] += np.abs(ra[f[1] - 1])
    sc = oracle.scales
    rconv = sc["VSTR"] / sc["WMSTR"] / sc["ALSTR"] * 1e-6
    return rconv * oracle.wm[:, None] * g


def assert_rel(a, b, rtol, atol=0.0, what=""):
    err = np.abs(a - b)
    lim = rtol * np.abs(b) + atol
    bad = err > lim
    assert not bad.any(), f"{what}: {bad.sum()} values out of tolerance; worst {np.max(err / np.maximum(lim, 1e-300)):.3g}x"


@pytest.fixture(scope="module")
def c1(oracle):
    f = jet_field(101, 61, fuel=2, t_peak=2200.0, seed=0)        # C1: 101x61 CH4/air
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    return tk, rho, f.y


@pytest.fixture(scope="module")
def mixed_states(oracle):
    return random_state(oracle, 3000, 5, 300, 3000)


def test_scales_match_oracle(cuda, oracle):
    with cuda.UniChem(10) as u:
        for k, v in oracle.scales.items():
            if k in u.scales:
                assert u.scales[k] == v, k
        assert np.array_equal(u.wm, oracle.wm) and np.array_equal(u.hfo, oracle.hfo)


@pytest.mark.parametrize("which", ["c1", "mixed_states"])
def test_rates_plane(cuda, oracle, request, which):
    tk, rho, y = request.getfixturevalue(which)
    with cuda.UniChem(len(tk)) as u:
        u.upload(tk, rho, y)
        rc = u.ckrates(return_rc=True)
    rc_o, _ = oracle.rates(tk, rho, y)
    assert_rel(rc, rc_o, RTOL, 1e-300, "RC")


@pytest.mark.parametrize("which", ["c1", "mixed_states"])
def test_omega(cuda, oracle, request, which):
    tk, rho, y = request.getfixturevalue(which)
    with cuda.UniChem(len(tk)) as u:
        u.upload(tk, rho, y)
        om = u.omega()
    q, qd, h, d = oracle.omega(tk, rho, y)
    g = gross(oracle, tk, rho, y)
    assert_rel(om.qdsp, q, 0.0, RTOL * g + 1e-300, "QDSP")
    assert_rel(om.domega_dy, d, RTOL, 1e-300, "domega/dY")
    hs = (g * np.abs(h)).sum(0)          # gross scale of the heat-release sum
    assert_rel(om.qdot, qd, 0.0, RTOL * hs + 1e-300, "QDOT")


@pytest.mark.parametrize("which", ["c1", "mixed_states"])
def test_props_cp_h(cuda, oracle, request, which):
    tk, rho, y = request.getfixturevalue(which)
    with cuda.UniChem(len(tk)) as u:
        u.upload(tk, rho, y)
        cp, h = u.cp_h()
        mu, lam, dk = u.props()
        _, _, yc, _, _ = u.download()
    assert_rel(cp, oracle.cp(tk, y), RTOL, 0, "cp")
    _, hm = oracle.enthalpy(tk, y)
    assert_rel(h, hm, 1e-10, 1e-12 * np.abs(hm).max(), "h")
    yc_o, mu_o, lam_o, d_o, nsub = oracle.props(tk, y)
    assert np.array_equal(yc, yc_o)
    assert_rel(mu, mu_o, RTOL, 0, "mu")
    assert_rel(lam, lam_o, RTOL, 0, "lambda")
    assert_rel(dk, d_o, RTOL, 0, "D_k")


@pytest.mark.parametrize("isor,tol", [(1, 1e-8), (5, 0.0)])
def test_species_update(cuda, oracle, c1, isor, tol):
    tk, rho, y = c1
    n = len(tk)
    with cuda.UniChem(n) as u:
        u.upload(tk, rho, y)
        u.ckrates()
        passes = u.solvesp(1e-3, isor=isor, relx=0.99, tol=tol)
        _, _, yg, s1, s2 = u.download()
    rc, sour = oracle.rates(tk, rho, y)
    yo, so, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=isor, tol=tol)
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y after update")
    assert_rel(s1, so[0], 1e-9, 1e-30, "soot mass fraction")


def test_species_update_converges_like_oracle(cuda, oracle):
    f = batch_cells(4096, seed=2)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    with cuda.UniChem(f.n) as u:
        u.upload(tk, rho, f.y)
        u.ckrates()
        passes = u.solvesp(1e-3, isor=100, relx=0.99, tol=1e-8)
        _, _, yg, _, _ = u.download()
    rc, sour = oracle.rates(tk, rho, f.y)
    yo, _, po = oracle.species_update(rho, f.y, rc, sour, 1e-3, isor=100, tol=1e-8)
    assert abs(passes - po) <= 1
    assert_rel(yg, yo, 1e-7, 1e-16, "Y after converged update")


def test_frozen_transport_terms(cuda, oracle, c1):
    tk, rho, y = c1
    n = len(tk)
    rng = np.random.default_rng(4)
    fs = rng.uniform(-0.02, 0.0, (51, n)) * rho          # E+W+N+S (negative, like the reference's)
    fn = fs * y[:51] * rng.uniform(0.9, 1.1, (51, n))    # coefficients times frozen neighbour values
    with cuda.UniChem(n) as u:
        u.upload(tk, rho, y)
        u.ckrates()
        passes = u.solvesp(1e-3, isor=3, tol=0.0, face_sum=fs, face_nbr=fn)
        _, _, yg, _, _ = u.download()
    rc, sour = oracle.rates(tk, rho, y)
    yo, _, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=3, tol=0.0, face_sum=fs, face_nbr=fn)
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y with frozen transport")


def test_temperature_from_h(cuda, oracle, mixed_states):
    tk, rho, y = mixed_states
    T = tk * oracle.scales["TSTR"]
    ht = sensible_enthalpy(T, y, np.array(oracle.mech["poly"]), oracle.wm, oracle.hfo, oracle.scales)
    guess = np.full_like(tk, 1200.0 / oracle.scales["TSTR"])
    with cuda.UniChem(len(tk)) as u:
        u.upload(guess, rho, y)
        u.temperature(ht)
        tg, _, _, _, _ = u.download()
    to = oracle.temperature(guess, y, ht)
    assert np.abs(tg - to).max() * oracle.scales["TSTR"] <= 2e-3


def test_edge_sizes(cuda, oracle):
    """One cell, a non-multiple of the 32-cell tile, and a pure-N2 cell."""
    for n in (1, 33):
        tk, rho, y = random_state(oracle, n, 9)
        y[:, 0] = 0.0
        y[51, 0] = 1.0
        with cuda.UniChem(n) as u:
            u.upload(tk, rho, y)
            om = u.omega()
            mu, lam, dk = u.props()
        q, qd, h, d = oracle.omega(tk, rho, y)
        assert np.isfinite(om.qdsp).all()
        g = gross(oracle, tk, rho, y)
        assert_rel(om.qdsp, q, 0.0, RTOL * g + 1e-300, "QDSP")
        _, mu_o, lam_o, d_o, _ = oracle.props(tk, y)
        assert_rel(mu, mu_o, RTOL, 0, "mu")
        assert_rel(dk, d_o, RTOL, 0, "D_k")


def test_errors_are_reported(cuda):
    u = cuda.UniChem(8)
    with pytest.raises(cuda.UniChemError) as e:
        u.solvesp(1e-3)                 # no RC plane yet
    assert e.value.code == -3
    with pytest.raises(ValueError):
        u.upload(np.ones(7), np.ones(8), np.ones((52, 8)))
    u.close()


def test_soot_sources_and_update_with_soot(cuda, oracle):
    """Non-zero soot (STMF, STND): the soot source terms of ckrates.f:1337-1352 enter the rate kernel's
    SOUR and the species update of H2, O2, H, O, OH, CO and C2H2 and the two soot scalars
    (solvesp.f:415,529,697,851,1005,1343-1344,1969, 2807-2832)."""
    tk, rho, y = random_state(oracle, 3000, 17, 900, 2600)
    rng = np.random.default_rng(17)
    stmf = rng.uniform(0.0, 1e-3, 3000)
    stnd = 10 ** rng.uniform(-1, 14, 3000)
    with cuda.UniChem(3000) as u:
        u.upload(tk, rho, y, stmf, stnd)
        rc = u.ckrates(return_rc=True)
        passes = u.solvesp(1e-3, isor=4, relx=0.99, tol=0.0)
        _, _, yg, s1, s2 = u.download()
    rc_o, sour_o = oracle.rates(tk, rho, y, stmf, stnd)
    assert np.abs(sour_o[2:5]).max() > 0                      # the surface-growth and oxidation terms are live
    assert_rel(rc, rc_o, RTOL, 1e-300, "RC with soot")
    yo, so, po = oracle.species_update(rho, y, rc_o, sour_o, 1e-3, isor=4, tol=0.0,
                                       soot0=np.vstack([stmf, stnd]))
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y with soot sources")
    assert_rel(s1, so[0], 1e-9, 1e-30, "soot mass fraction")
    assert_rel(s2, so[1], 1e-9, 1e-30, "soot number density")


def test_c2_slice_sweep_converged(cuda, oracle):
    """The FP64 sweep with the reference's card settings (isor 100, relaxation 0.99, tolerance 1e-8) on
    2,056 cells of the 601x301 heptane field (every 88th): the pass count the reference reports and Y."""
    f = jet_field(601, 301, fuel=11, t_peak=2300.0, seed=0)
    sel = np.arange(0, f.n, 88)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    tk, rho, y = tk[sel].copy(), rho[sel].copy(), np.ascontiguousarray(f.y[:, sel])
    with cuda.UniChem(len(sel)) as u:
        u.upload(tk, rho, y)
        passes = u.sweep(1e-3, isor=100, relx=0.99, tol=1e-8)
        _, _, yg, _, _ = u.download()
    yc = oracle.props(tk, y)[0]
    rc, sour = oracle.rates(tk, rho, yc)
    yo, _, po = oracle.species_update(rho, yc, rc, sour, 1e-3, isor=100, relx=0.99, tol=1e-8)
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y after the converged C2 sweep")
