"""ISKIP on the device (uc_set_iskip) against the oracle's ISKIP wrappers, which
are pinned bit for bit to the translated reference (tests/test_oracle_pin.py).

A 40x50 heptane field with a block of injection cells (ISKIP = 3), body cells
(10 and 11) and cells whose flags skip nothing here (1, 2): skipped cells keep
their (zero) RC, omega and QDOT and their Y, T and soot, bit for bit; the other
cells match the oracle at the tolerances of the FP64 parity tests (RC 1e-11,
omega 1e-11 of the gross rate, Y 1e-9) with the oracle's pass count, for the
tile-resident and the per-pass update kernels."""
import numpy as np
import pytest

from test_gpu_parity import assert_rel, gross
from unicorn_b200.fields import jet_field, nondimensional, sensible_enthalpy

pytestmark = pytest.mark.gpu


def iskip_field(oracle):
    f = jet_field(40, 50, fuel=11, t_peak=2300.0, seed=3)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    iskip = np.zeros(f.n, dtype=np.int32)
    iskip[100:180] = 3
    iskip[500:520] = 10
    iskip[900:905] = 11
    iskip[1200:1210] = 1
    iskip[1300:1310] = 2
    return tk, rho, f.y, iskip


@pytest.mark.parametrize("kind", ["resident", "inplace"])
@pytest.mark.parametrize("isor,tol", [(3, 0.0), (100, 1e-8)])
def test_iskip_rates_omega_update(oracle, monkeypatch, kind, isor, tol):
    from unicorn_b200 import unichem
    monkeypatch.setenv("UNICHEM_UPDATE", kind)
    tk, rho, y, iskip = iskip_field(oracle)
    skipped = iskip >= 3
    with unichem.UniChem(len(tk)) as u:
        u.set_iskip(iskip)
        u.upload(tk, rho, y)
        rc = u.ckrates(return_rc=True)
        om = u.omega()
        u.upload(tk, rho, y)
        u.ckrates()
        passes = u.solvesp(1e-3, isor=isor, relx=0.99, tol=tol)
        _, _, yg, s1, _ = u.download()
    rc_o, sour_o = oracle.rates_iskip(tk, rho, y, iskip)
    assert not rc[:, skipped].any()
    assert_rel(rc[:, ~skipped], rc_o[:, ~skipped], 1e-11, 0.0, "RC")
    q_o, qd_o, _, d_o = oracle.omega_iskip(tk, rho, y, iskip)
    assert not om.qdsp[:, skipped].any() and not om.qdot[skipped].any() and not om.domega_dy[:, skipped].any()
    g = gross(oracle, tk, rho, y)
    err = np.abs(om.qdsp - q_o)[:, ~skipped]
    assert np.all(err <= 1e-11 * g[:, ~skipped] + 1e-300)
    yo, so, po = oracle.species_update_iskip(rho, y, rc_o, sour_o, 1e-3, iskip, isor=isor, relx=0.99, tol=tol)
    assert passes == po
    assert np.array_equal(yg[:, skipped], y[:, skipped])                      # kept, N2 included
    assert not s1[skipped].any()
    assert_rel(yg[:, ~skipped], yo[:, ~skipped], 1e-9, 1e-18, "Y of the computed cells")


def test_iskip_temperature(oracle):
    from unicorn_b200 import unichem
    tk, rho, y, iskip = iskip_field(oracle)
    T = tk * oracle.scales["TSTR"]
    ht = sensible_enthalpy(T + 50.0, y, np.array(oracle.mech["poly"]), oracle.wm, oracle.hfo, oracle.scales)
    with unichem.UniChem(len(tk)) as u:
        u.set_iskip(iskip)
        u.upload(tk, rho, y)
        u.temperature(ht)
        tg = u.download()[0]
    to = oracle.temperature_iskip(tk, y, ht, iskip)
    skipped = iskip >= 3
    assert np.array_equal(tg[skipped], tk[skipped])
    assert np.abs(tg - to).max() * oracle.scales["TSTR"] < 2e-3
    assert np.abs(tg[~skipped] - tk[~skipped]).min() * oracle.scales["TSTR"] > 10.0   # the others moved
