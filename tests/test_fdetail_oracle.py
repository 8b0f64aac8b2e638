"""FDETAIL fields (lib/stdata.f:26-118): the oracle's restatement
(orc_fdetail) against the reference's own routine (translated), bit for bit."""
import numpy as np

from unicorn_b200.fields import jet_field, nondimensional


def fd_case(oracle, LJ, LI, seed):
    rng = np.random.default_rng(seed)
    f = jet_field(LI, LJ, fuel=11, t_peak=2300.0, seed=seed)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    n = LJ * LI
    xs = np.cumsum(rng.uniform(0.5, 1.5, LI)) / LJ
    ys = np.cumsum(rng.uniform(0.5, 1.5, LJ)) / LJ
    x = np.tile(xs[None, :], (LJ, 1)).reshape(-1, order="F")
    y = np.tile(ys[:, None], (1, LI)).reshape(-1, order="F")
    return dict(x=x, y=y, rho=rho, u=rng.uniform(-1, 1, n), v=rng.uniform(-1, 1, n), tk=tk,
                qdot=rng.standard_normal(n), vmu=10 ** rng.uniform(-3, -1, n), vtc=10 ** rng.uniform(-3, -1, n),
                fsp=f.y, vdf=10 ** rng.uniform(-4, -1, (52, n)), qdsp=rng.standard_normal((52, n)))


def test_fdetail_bitwise_vs_reference(oracle, ref):
    LJ, LI = ref.LJ, ref.LI
    g = fd_case(oracle, LJ, LI, 3)
    args = [g[k] for k in ("x", "y", "rho", "u", "v", "tk", "qdot", "vmu", "vtc", "fsp", "vdf", "qdsp")]
    r = ref.stdata_fields(*args)
    o = oracle.fdetail(LJ, LI, *args)
    assert r.shape == o.shape == (218, LJ * LI)
    assert np.array_equal(r, o)
