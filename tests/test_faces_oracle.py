"""E/W/N/S coefficients of the species equations: the oracle's restatement
(orc_faces) against the reference's own assembly (lib/spgsolv.f:98-1290,
translated), bit for bit on the interior cells."""
import numpy as np
import pytest

from unicorn_b200.fields import jet_field, nondimensional


def grid_case(oracle, LJ, LI, seed):
    rng = np.random.default_rng(seed)
    f = jet_field(LI, LJ, fuel=11, t_peak=2300.0, seed=seed)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    n = LJ * LI
    # stretched grid spacings, a radial coordinate from the axis, random velocities / eddy viscosity
    xxs = 1.0 / (LJ - 2) * rng.uniform(0.8, 1.2, LI)
    xxc = 1.0 / (LJ - 2) * rng.uniform(0.8, 1.2, LI)
    yys = 1.0 / (LJ - 2) * rng.uniform(0.8, 1.2, LJ)
    yyc = 1.0 / (LJ - 2) * rng.uniform(0.8, 1.2, LJ)
    yr = np.tile(np.cumsum(yyc) - 0.5 * yyc[0], LI)
    u, v = rng.uniform(-2, 2, n), rng.uniform(-1, 1, n)
    tmu = 10 ** rng.uniform(-5, -2, n)
    vdf = 10 ** rng.uniform(-4, -1, (52, n))
    return dict(tk=tk, rho=rho, y=f.y, u=u, v=v, tmu=tmu, vdf=vdf, xxs=xxs, xxc=xxc, yys=yys, yyc=yyc, yr=yr)


@pytest.mark.parametrize("isym,seed", [(1, 0), (0, 1)])
def test_faces_bitwise_vs_reference(oracle, ref, isym, seed):
    LJ, LI = ref.LJ, ref.LI
    g = grid_case(oracle, LJ, LI, seed)
    n = LJ * LI
    r = ref.spgsolv_coefficients(g["tk"], g["rho"], g["y"], np.full(n, 1e-3), g["vdf"], g["u"], g["v"], g["tmu"],
                                 np.zeros(n), g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=isym, dt=1e-3,
                                 sigsp=0.7)
    o = oracle.faces(LJ, LI, g["rho"], g["vdf"], g["u"], g["v"], g["tmu"], g["yr"], g["xxs"], g["xxc"], g["yys"],
                     g["yyc"], isym=isym, dt=1e-3, sigsp=0.7)
    J, I = np.meshgrid(np.arange(LJ), np.arange(LI), indexing="ij")
    interior = ((J > 0) & (J < LJ - 1) & (I > 0) & (I < LI - 1)).reshape(-1, order="F")
    for a, b in zip(r, o):
        assert np.array_equal(a[:, interior], b[:, interior])
