"""The in-loop pieces on the CPU: the frozen diffusion faces of
unicorn_b200/inloop.py and the oracle's held-enthalpy T step.

The faces form a conservative diffusion operator: a uniform field has no net
exchange (face_nbr = face_sum * Y), and for any field the exchanges sum to
zero over the grid. The oracle's T step (orc_enthalpy_total +
orc_temperature_held) composed with its rates and species update on one cell
is, bit for bit, the one-sub-step batched integration (orc_integrate), which
the reference's per-cell chain pins."""
import numpy as np

from unicorn_b200.fields import batch_cells, jet_field, nondimensional
from unicorn_b200.inloop import frozen_faces

DT = 1e-3


def test_faces_uniform_field_exchanges_nothing():
    nz, nr = 7, 5
    rng = np.random.default_rng(1)
    vdf = rng.uniform(1e-3, 1e-2, (52, nz * nr))
    y = np.tile(rng.dirichlet(np.ones(52))[:, None], (1, nz * nr))
    fs, fn = frozen_faces((nz, nr), vdf, y, DT)
    assert fs.shape == fn.shape == (51, nz * nr)
    assert (fs < 0).all()
    assert np.allclose(fn, fs * y[:51], rtol=1e-14, atol=0)


def test_faces_conserve_mass_over_the_grid():
    nz, nr = 9, 6
    f = jet_field(nz, nr, fuel=11, seed=2)
    vdf = np.random.default_rng(3).uniform(1e-3, 1e-2, (52, nz * nr))
    fs, fn = frozen_faces((nz, nr), vdf, f.y, DT)
    net = fn - fs * f.y[:51]           # -DT * sum_f a_f (Y_nbr - Y_c) per cell
    scale = np.abs(fn).sum(axis=1)
    assert (np.abs(net.sum(axis=1)) <= 1e-12 * scale).all()


def test_held_temperature_step_is_the_integration_step(oracle):
    f = batch_cells(6, seed=5)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    pnd = f.p / oracle.scales["PSTR"]
    tk1, rho1, y1, s1, _ = oracle.integrate(tk, rho, f.y, pnd, np.ones(6, dtype=np.int32), DT)
    enth = oracle.enthalpy_total(tk, f.y)
    for c in range(6):
        sl = slice(c, c + 1)
        rc, sour = oracle.rates(tk[sl], rho[sl], f.y[:, sl])
        yn, sn, _ = oracle.species_update(rho[sl], f.y[:, sl], rc, sour, DT, spnorm=51.0)
        t, r = oracle.temperature_held(tk[sl], yn, pnd[sl], enth[sl])
        assert np.array_equal(yn[:, 0], y1[:, c]) and np.array_equal(sn[:, 0], s1[:, c])
        assert t[0] == tk1[c] and r[0] == rho1[c]
