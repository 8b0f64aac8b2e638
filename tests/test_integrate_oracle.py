"""Oracle of the batched stiff integration (orc_nsub, orc_integrate): the
sub-step rule and the invariants of a step, on the CPU."""
import numpy as np
import pytest

from unicorn_b200.fields import batch_cells, nondimensional, sensible_enthalpy

DT = 1e-3


@pytest.fixture(scope="module")
def c3(oracle):
    f = batch_cells(96, seed=3)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    return f, tk, rho, f.p / oracle.scales["PSTR"]


def test_nsub_rule(oracle, c3):
    f, tk, rho, _ = c3
    q = oracle.omega(tk, rho, f.y)[0]
    ns, x = oracle.nsub(rho, f.y, q, DT, c_tau=1.0, y_tau=1e-3, nsub_max=200)
    sc = oracle.scales
    rconv = sc["VSTR"] / sc["WMSTR"] / sc["ALSTR"] * 1e-6
    with np.errstate(divide="ignore", invalid="ignore"):
        v = np.where(f.y > 1e-3, DT * np.abs(q) / (rconv * rho * f.y), 0.0)
    assert np.allclose(x, v.max(0), rtol=1e-14, atol=0)
    want = np.clip(np.ceil(v.max(0)), 1, 200).astype(int)
    assert np.array_equal(ns, want)
    assert ns.min() == 1 and ns.max() == 200          # the distribution spans the whole range


def test_integrate_invariants(oracle, c3):
    f, tk, rho, pnd = c3
    q = oracle.omega(tk, rho, f.y)[0]
    ns, _ = oracle.nsub(rho, f.y, q, DT)
    tk1, rho1, y1, s1, passes = oracle.integrate(tk, rho, f.y, pnd, ns, DT)
    # closure: species + soot mass sum to one (N2 takes the rest, or renormalisation)
    assert np.abs(y1.sum(0) + s1[0] - 1.0).max() < 1e-12
    assert (y1 >= 0).all()
    # constant total enthalpy: h(T1, Y1) matches h(T0, Y0) to the Newton step tolerance (1e-3 K)
    poly = np.array(oracle.mech["poly"])
    sc = oracle.scales
    T0, T1 = tk * sc["TSTR"], tk1 * sc["TSTR"]
    h0 = sensible_enthalpy(T0, f.y, poly, oracle.wm, oracle.hfo, sc) + (f.y * oracle.hfo[:, None]).sum(0)
    h1 = sensible_enthalpy(T1, y1, poly, oracle.wm, oracle.hfo, sc) + (y1 * oracle.hfo[:, None]).sum(0)
    cp = oracle.cp(tk1, y1)
    free = (T1 > sc["TSTR"] - 1.0 + 1e-6) & (T1 < 5000.0 - 1e-6)   # not held at the clamp of solveh.f:1232-1233
    assert free.sum() >= len(T1) // 2
    assert (np.abs(h1 - h0) / (cp * sc["TSTR"]))[free].max() < 1e-2     # in K
    # ideal gas at the cell pressure
    rbar = (y1 / oracle.wm[:, None]).sum(0)
    assert np.allclose(rho1, pnd / (sc["BETA1"] * tk1 * rbar), rtol=1e-14)
    assert (passes >= ns).all() and (passes <= 100 * ns).all()


def test_one_substep_is_the_reference_chain(oracle, c3):
    """n_sub = 1: rates -> species update of a one-cell field (SPNORM 51), cell by cell."""
    f, tk, rho, pnd = c3
    idx = np.arange(0, 96, 7)
    ns = np.ones(len(idx), dtype=np.int32)
    tk1, rho1, y1, s1, passes = oracle.integrate(tk[idx], rho[idx], f.y[:, idx], pnd[idx], ns, DT)
    for j, c in enumerate(idx):
        rc, sour = oracle.rates(tk[c:c + 1], rho[c:c + 1], f.y[:, c:c + 1])
        yn, sn, p = oracle.species_update(rho[c:c + 1], f.y[:, c:c + 1], rc, sour, DT, spnorm=51.0)
        assert np.array_equal(yn[:, 0], y1[:, j]) and np.array_equal(sn[:, 0], s1[:, j])
        assert min(p, 100) == passes[j]


def test_cells_integrate_independently_of_their_order(oracle, c3):
    """The batched integration advances each cell as a one-cell field: a cell's result does not depend on
    the other cells of the batch or on their order. The device's rounds form relies on this when it
    gathers the cells in sub-step order and re-orders them between rounds."""
    f, tk, rho, pnd = c3
    q = oracle.omega(tk, rho, f.y)[0]
    ns, _ = oracle.nsub(rho, f.y, q, DT)
    a = oracle.integrate(tk, rho, f.y, pnd, ns, DT)
    perm = np.random.default_rng(5).permutation(len(tk))
    b = oracle.integrate(tk[perm], rho[perm], f.y[:, perm], pnd[perm], ns[perm], DT)
    inv = np.argsort(perm)
    for u, v in zip(a, b):
        assert np.array_equal(u, v[..., inv])
    half = perm[: len(perm) // 2]                     # and a cell alone in a smaller batch
    c = oracle.integrate(tk[half], rho[half], f.y[:, half], pnd[half], ns[half], DT)
    for u, v in zip(a, c):
        assert np.array_equal(u[..., half], v)
