"""Enthalpy equation on the GPU (uc_enthalpy_relax, uc_enthalpy_update) against
the oracle's restatement, itself pinned bit for bit to the reference's SOLVEH
(tests/test_enthalpy_oracle.py).

* The relaxation alone on the oracle's own coefficients: FPZ bit for bit and
  the same pass count (the device runs the reference's lexicographic
  Gauss-Seidel order and rounds every operation as written), converged or
  not, with the ring of pass buffers full and capped at 2 and 3 slots, on the
  C1 grid, on the reference's 131 x 711 grid, and on edge grids (one interior
  row, one interior column, one interior cell, 1024 interior rows) and the
  whole C2 grid (301 x 601), where the converged FPZ also satisfies the
  discrete enthalpy equation; more rows than one pass takes are refused.
* The whole update after a sweep, against the oracle given the device's rate
  plane, properties and cp of the start state (their own parity is covered by
  tests/test_gpu_parity.py): ZE..ZS to 1e-12 of the cell's largest
  coefficient; RHSZ to 1e-10 of the gross size of its terms (RHO HT, the
  diffusion sums, the radiation, DT times the gross heat release); QDSP and
  QDOT to 1e-10 of their gross sizes; FPZ bit for bit against the oracle's
  relaxation of the device's coefficients; T to 2e-3 K (the Newton step
  tolerance of solveh.f:1211 is 1e-3 K). The same after a mixed-precision
  sweep, whose FP32 rate plane (with FP64 tiles for the cold cells) the
  heat release reads."""
import numpy as np
import pytest

from test_enthalpy_oracle import enthalpy_case

pytestmark = pytest.mark.gpu
LJ, LI = 61, 101          # the C1 grid: 101 (z) x 61 (r)


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


def interior(lj, li):
    J, I = np.meshgrid(np.arange(lj), np.arange(li), indexing="ij")
    return ((J > 0) & (J < lj - 1) & (I > 0) & (I < li - 1)).reshape(-1, order="F")


def consistent_ht(oracle, g, w=None):
    """HT of each cell's own temperature and composition plus its kinetic energy, so that T stays
    near the start temperature (solveh.f:1170-1200), perturbed by a few per cent."""
    from unicorn_b200.fields import sensible_enthalpy
    sc = oracle.scales
    T = g["tk"] * sc["TSTR"]
    ht = sensible_enthalpy(T, g["y"], np.array(oracle.mech["poly"]), oracle.wm, oracle.hfo, sc)
    ke = 0.5 * (g["u"] ** 2 + g["v"] ** 2 + (0.0 if w is None else w ** 2))
    rng = np.random.default_rng(31)
    return ht * (1.0 + 0.005 * rng.uniform(-1, 1, ht.shape)) + ke


def oracle_coefficients(oracle, lj, li, seed):
    g = enthalpy_case(oracle, lj, li, seed)
    o = oracle.enthalpy_solve(lj, li, g["tk"], g["rho"], g["y"], g["y_new"], g["ht"], g["stmf"], g["vtc"], g["vdf"],
                              g["u"], g["v"], g["tmu"], g["yr"], g["xxs"], g["xxc"], g["yys"], g["yyc"], isor=1, tol=0.0)
    return g, o


# tol < 0 never converges (at tol = 0 the passes reach a fixed point of exactly zero residual)
@pytest.mark.parametrize("isor,tol,ring", [(100, 1e-8, None), (6, -1.0, None), (100, 1e-8, 2), (40, -1.0, 3),
                                           (40, 0.0, None)])
def test_relax_bitwise(cuda, oracle, monkeypatch, isor, tol, ring):
    if ring is not None:
        monkeypatch.setenv("UNICHEM_RELAX_RING", str(ring))
    g, o = oracle_coefficients(oracle, LJ, LI, 6)
    fpz_o, passes_o = oracle.enthalpy_relax(LJ, LI, g["rho"], o["rhsz"], o["z"], g["ht"], isor=isor, tol=tol)
    fpz_g, passes_g = cuda.enthalpy_relax(LJ, LI, g["rho"], o["rhsz"], o["z"], g["ht"], isor=isor, tol=tol)
    assert passes_g == passes_o
    if tol < 0.0:
        assert passes_g == isor + 1
    else:
        assert 1 < passes_g <= isor
    assert np.array_equal(fpz_g, fpz_o)
    assert np.abs(fpz_g - g["ht"])[interior(LJ, LI)].max() > 1e-6


def test_relax_bitwise_reference_grid(cuda, oracle):
    """The reference's compile-time grid, LJ = 131 rows by LI = 711 columns, 100 passes at most."""
    lj, li = 131, 711
    g, o = oracle_coefficients(oracle, lj, li, 7)
    fpz_o, passes_o = oracle.enthalpy_relax(lj, li, g["rho"], o["rhsz"], o["z"], g["ht"], isor=100, tol=1e-8)
    fpz_g, passes_g = cuda.enthalpy_relax(lj, li, g["rho"], o["rhsz"], o["z"], g["ht"], isor=100, tol=1e-8)
    assert passes_g == passes_o
    assert np.array_equal(fpz_g, fpz_o)


def test_relax_zero_passes(cuda, oracle):
    g, o = oracle_coefficients(oracle, 8, 9, 8)
    fpz_g, passes_g = cuda.enthalpy_relax(8, 9, g["rho"], o["rhsz"], o["z"], g["ht"], isor=0)
    assert passes_g == 1 and np.array_equal(fpz_g, g["ht"])


@pytest.mark.parametrize("dt", [1e-7, 1e-3])
def test_enthalpy_update_matches_oracle(cuda, oracle, dt):
    """At DT = 1e-3 (1e-5 s) the heat release of the synthetic compositions, far from equilibrium,
    drives T of many cells to the limits of solveh.f:1229-1230, where the Newton of solveh.f:1211 does
    not converge; T is compared at DT = 1e-7, where no cell reaches a limit."""
    from test_gpu_parity import gross
    g = enthalpy_case(oracle, LJ, LI, 5)
    n = LJ * LI
    rng = np.random.default_rng(77)
    w = rng.uniform(-0.3, 0.3, n)
    ht = consistent_ht(oracle, g, w)
    inner = interior(LJ, LI)
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"], stmf=g["stmf"])
        u.set_grid(LJ, LI, g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=1)
        u.set_flow(g["u"], g["v"], g["tmu"], 0.9)
        u.set_enthalpy(ht, w)
        u.sweep(dt, isor=4, tol=0.0)
        _, _, y_new, _, _ = u.download()
        passes, resdh = u.enthalpy_update(dt, isor=100, relx=0.99, tol=1e-8, sigh=0.9)
        tk_g, _, y_after, _, _ = u.download()
        ht_g, rhsz_g, ze_g, zw_g, zn_g, zs_g = u.enthalpy_get()
        out = u.download_outputs()
    assert np.array_equal(y_after, y_new)
    # start state of the device: clipped Y, rate plane, properties, cp
    with cuda.UniChem(n) as u2:
        u2.upload(g["tk"], g["rho"], g["y"], stmf=g["stmf"])
        _, vtc, vdf = u2.props()
        cp, _ = u2.cp_h()
        rc = u2.ckrates(return_rc=True)
        _, _, y_start, _, _ = u2.download()
    z_o, ekt = oracle.zfaces(LJ, LI, g["rho"], cp, vtc, g["tmu"], g["u"], g["v"], g["yr"], g["xxs"], g["xxc"],
                             g["yys"], g["yyc"], isym=1, dt=dt, sigh=0.9)
    zmax = np.max(np.abs(np.stack(z_o)), axis=0)
    for a, b in zip((ze_g, zw_g, zn_g, zs_g), z_o):
        assert np.all(np.abs(a - b)[inner] <= 1e-12 * zmax[inner] + 1e-300)
    rhsz_o, qdsp_o, qdot_o = oracle.enthalpy_rhs(LJ, LI, g["tk"], g["rho"], y_new, ht, g["stmf"], vdf, g["tmu"], ekt,
                                                 rc, g["yr"], g["xxs"], g["xxc"], g["yys"], g["yyc"], isym=1, dt=dt,
                                                 sigsp=0.9)
    gq = gross(oracle, g["tk"], g["rho"], y_new)                     # RCONV W_k sum|terms| per species
    sc = oracle.scales
    rconv = sc["VSTR"] / sc["WMSTR"] / sc["ALSTR"] * 1e-6
    gprod = (gq * np.abs(oracle.hfo)[:, None]).sum(0) / rconv          # gross size of PROD
    scale = np.abs(g["rho"] * ht) + np.abs(rhsz_o) + dt * gprod + 1e-300
    err = np.abs(rhsz_g - rhsz_o)[inner] / scale[inner]
    assert err.max() <= 1e-10, err.max()
    assert np.all(np.abs(out["qdsp"] - qdsp_o)[:, inner] <= 1e-10 * gq[:, inner] + 1e-300)
    hscale = (gq * np.abs(oracle.hfo)[:, None]).sum(0) * 10.0           # gross heat release (|h_k| <~ 10 |HFO|)
    assert np.all(np.abs(out["qdot"] - qdot_o)[inner] <= 1e-10 * hscale[inner] + 1e-300)
    # the relaxation of the device's own coefficients, bit for bit, and its pass count
    fpz_o, passes_o = oracle.enthalpy_relax(LJ, LI, g["rho"], rhsz_g, (ze_g, zw_g, zn_g, zs_g), ht, isor=100,
                                            tol=1e-8)
    assert passes == passes_o and 1 < passes <= 100
    assert np.array_equal(ht_g[inner], fpz_o[inner])
    assert np.array_equal(ht_g[~inner], ht[~inner])                   # boundary HT is held
    assert np.array_equal(tk_g[~inner], g["tk"][~inner])
    resdh_o = np.abs(fpz_o - ht)[inner].sum() / (LJ * LI)           # spgsolv.f:1304,1415
    assert abs(resdh - resdh_o) <= 1e-12 * resdh_o
    if dt > 1e-6:
        return
    tk_o = oracle.temperature_ke(LJ, LI, g["tk"], y_new, fpz_o, g["u"], g["v"], w)
    To = tk_o[inner] * sc["TSTR"]
    assert To.min() > sc["TSTR"] - 1.0 + 1e-6 and To.max() < 5000.0 - 1e-6        # no cell at a limit
    dT = np.abs(tk_g - tk_o)[inner] * sc["TSTR"]
    assert dT.max() <= 2e-3, dT.max()
    # the update moved T
    assert np.abs(tk_g - g["tk"])[inner].max() * sc["TSTR"] > 1e-3


def test_enthalpy_update_needs_a_sweep(cuda, oracle):
    g = enthalpy_case(oracle, 8, 9, 9)
    n = 8 * 9
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"])
        u.set_grid(8, 9, g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=1)
        u.set_flow(g["u"], g["v"], g["tmu"], 0.9)
        u.set_enthalpy(g["ht"])
        with pytest.raises(RuntimeError):
            u.enthalpy_update(1e-3)
        u.sweep(1e-3, isor=2, tol=0.0)
        u.enthalpy_update(1e-3, isor=5)
        with pytest.raises(RuntimeError):        # the rate plane belongs to the state before the update
            u.enthalpy_update(1e-3, isor=5)


def test_density_matches_oracle(cuda, oracle):
    g = enthalpy_case(oracle, LJ, LI, 12)
    n = LJ * LI
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y_new"])
        u.set_grid(LJ, LI, g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=1)
        u.density()
        _, rho_g, _, _, _ = u.download()
    rho_o = oracle.density(LJ, LI, g["tk"], g["y_new"])
    assert np.array_equal(rho_g, rho_o)


@pytest.mark.parametrize("lj,li", [(3, 9), (9, 3), (3, 3), (1026, 5)])
def test_relax_edge_grids(cuda, oracle, lj, li):
    """One interior row, one interior column, a single interior cell, and the most rows one pass
    takes (1024 interior rows, one thread each): bit for bit with the oracle."""
    g, o = oracle_coefficients(oracle, lj, li, 13)
    fpz_o, passes_o = oracle.enthalpy_relax(lj, li, g["rho"], o["rhsz"], o["z"], g["ht"], isor=30, tol=1e-10)
    fpz_g, passes_g = cuda.enthalpy_relax(lj, li, g["rho"], o["rhsz"], o["z"], g["ht"], isor=30, tol=1e-10)
    assert passes_g == passes_o
    assert np.array_equal(fpz_g, fpz_o)


def test_relax_rejects_too_many_rows(cuda, oracle):
    """1025 interior rows exceed one thread per row: a clear error, no launch."""
    lj, li = 1027, 4
    n = lj * li
    z = tuple(np.zeros(n) for _ in range(4))
    with pytest.raises(RuntimeError):
        cuda.enthalpy_relax(lj, li, np.ones(n), np.zeros(n), z, np.zeros(n), isor=3)


def test_enthalpy_update_after_mixed_sweep(cuda, oracle):
    """The heat release read from the mixed form's rate plane (FP32, with the tiles sent to FP64 read
    from the FP64 plane): against the oracle given that same plane and the sweep's own properties."""
    from test_gpu_parity import gross
    g = enthalpy_case(oracle, LJ, LI, 14)
    n = LJ * LI
    g["tk"][:10 * LJ] = 300.0 / oracle.scales["TSTR"]      # cold columns: their rates leave the FP32 range
    ht = consistent_ht(oracle, g)
    dt = 1e-7
    inner = interior(LJ, LI)
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"], stmf=g["stmf"])
        u.set_grid(LJ, LI, g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=1)
        u.set_flow(g["u"], g["v"], g["tmu"], 0.9)
        u.set_enthalpy(ht)
        u.sweep(dt, precision=cuda.MIXED, isor=4, tol=0.0)
        _, _, y_new, _, _ = u.download()
        start = u.download_outputs()                        # properties and cp of the start state
        u.enthalpy_update(dt, isor=100, relx=0.99, tol=1e-8, sigh=0.9)
        ht_g, rhsz_g, ze_g, zw_g, zn_g, zs_g = u.enthalpy_get()
        out = u.download_outputs()
    with cuda.UniChem(n) as u2:
        u2.upload(g["tk"], g["rho"], g["y"], stmf=g["stmf"])
        u2.props()
        rc = u2.ckrates(precision=cuda.MIXED, return_rc=True)
        assert u2.stat("mixed_fp64_tiles") > 0
    z_o, ekt = oracle.zfaces(LJ, LI, g["rho"], start["cp"], start["vtc"], g["tmu"], g["u"], g["v"], g["yr"], g["xxs"],
                             g["xxc"], g["yys"], g["yyc"], isym=1, dt=dt, sigh=0.9)
    zmax = np.max(np.abs(np.stack(z_o)), axis=0)
    for a, b in zip((ze_g, zw_g, zn_g, zs_g), z_o):
        assert np.all(np.abs(a - b)[inner] <= 1e-12 * zmax[inner] + 1e-300)
    rhsz_o, qdsp_o, qdot_o = oracle.enthalpy_rhs(LJ, LI, g["tk"], g["rho"], y_new, ht, g["stmf"], start["vdf"],
                                                 g["tmu"], ekt, rc, g["yr"], g["xxs"], g["xxc"], g["yys"], g["yyc"],
                                                 isym=1, dt=dt, sigsp=0.9)
    gq = gross(oracle, g["tk"], g["rho"], y_new)
    sc = oracle.scales
    rconv = sc["VSTR"] / sc["WMSTR"] / sc["ALSTR"] * 1e-6
    scale = np.abs(g["rho"] * ht) + np.abs(rhsz_o) + dt * (gq * np.abs(oracle.hfo)[:, None]).sum(0) / rconv + 1e-300
    assert (np.abs(rhsz_g - rhsz_o)[inner] / scale[inner]).max() <= 1e-10
    assert np.all(np.abs(out["qdsp"] - qdsp_o)[:, inner] <= 1e-10 * gq[:, inner] + 1e-300)
    fpz_o, _ = oracle.enthalpy_relax(LJ, LI, g["rho"], rhsz_g, (ze_g, zw_g, zn_g, zs_g), ht, isor=100, tol=1e-8)
    assert np.array_equal(ht_g[inner], fpz_o[inner])


def test_relax_full_c2_grid(cuda, oracle):
    """The C2 grid (301 rows x 601 columns, 180,901 cells): bit for bit with the oracle, and the
    converged FPZ satisfies the discrete enthalpy equation PPP F = RHSZ - (ZE F_E + ZW F_W + ZN F_N
    + ZS F_S) on the interior to the relaxation's tolerance."""
    lj, li = 301, 601
    g, o = oracle_coefficients(oracle, lj, li, 15)
    fpz_o, passes_o = oracle.enthalpy_relax(lj, li, g["rho"], o["rhsz"], o["z"], g["ht"], isor=100, tol=1e-10)
    fpz_g, passes_g = cuda.enthalpy_relax(lj, li, g["rho"], o["rhsz"], o["z"], g["ht"], isor=100, tol=1e-10)
    assert passes_g == passes_o and passes_g <= 100
    assert np.array_equal(fpz_g, fpz_o)
    F = fpz_g.reshape(li, lj)
    ze, zw, zn, zs = (z.reshape(li, lj) for z in o["z"])
    rho, rhsz = g["rho"].reshape(li, lj), o["rhsz"].reshape(li, lj)
    c = (slice(1, -1), slice(1, -1))
    ppp = rho[c] - (ze[c] + zw[c] + zn[c] + zs[c])
    nb = ze[c] * F[2:, 1:-1] + zw[c] * F[:-2, 1:-1] + zn[c] * F[1:-1, 2:] + zs[c] * F[1:-1, :-2]
    res = np.abs(ppp * F[c] - (rhsz[c] - nb)) / (np.abs(rhsz[c]) + np.abs(ppp * F[c]) + 1e-300)
    assert np.median(res) < 1e-9 and res.max() < 1e-6, (np.median(res), res.max())


def test_relaxation_wait_limit_gives_up_cleanly(cuda, oracle, monkeypatch):
    """Failure detection without a fault: with the wait limit between relaxation passes set to zero the
    passes give up at their first wait, the call reports UC_E_TIMEOUT and leaves T and HT as they were;
    the context stays usable and the next call (default limit) succeeds."""
    g = enthalpy_case(oracle, LJ, LI, 5)
    n = LJ * LI
    ht = consistent_ht(oracle, g)
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"], stmf=g["stmf"])
        u.set_grid(LJ, LI, g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=1)
        u.set_flow(g["u"], g["v"], g["tmu"], 0.9)
        u.set_enthalpy(ht)
        u.sweep(1e-7, isor=4, tol=0.0)
        tk0 = u.download()[0]
        monkeypatch.setenv("UNICHEM_RELAX_WAIT_NS", "0")
        with pytest.raises(cuda.UniChemError) as ei:
            u.enthalpy_update(1e-7, isor=50, relx=0.99, tol=-1.0, sigh=0.9)
        assert ei.value.code == -4
        assert np.array_equal(u.download()[0], tk0)
        assert np.array_equal(u.enthalpy_get()[0], ht)
        monkeypatch.delenv("UNICHEM_RELAX_WAIT_NS")
        u.sweep(1e-7, isor=4, tol=0.0)                    # an enthalpy update follows a species sweep
        passes, _ = u.enthalpy_update(1e-7, isor=50, relx=0.99, tol=-1.0, sigh=0.9)
        assert passes == 51
