"""Species-equation faces assembled on the GPU (uc_set_grid / uc_set_flow /
uc_assemble_faces) against the oracle's restatement (itself pinned bit for
bit to the reference's assembly, tests/test_faces_oracle.py), and a sweep
that uses them against the oracle's update with the same faces.

Tolerances: the coefficients to 1e-10 of the largest |coefficient| of the
cell and species (the hybrid form takes max(|rho u|, D), so an ulp in D can
change which branch holds; the coefficients themselves are differences of
O(1) terms); the swept Y to 1e-9 relative (the FP64 update tolerance)."""
import numpy as np
import pytest

from test_faces_oracle import grid_case

pytestmark = pytest.mark.gpu
LJ, LI = 61, 101          # the C1 grid: 101 (z) x 61 (r)


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


@pytest.fixture(scope="module")
def case(oracle):
    return grid_case(oracle, LJ, LI, 4)


def interior_mask():
    J, I = np.meshgrid(np.arange(LJ), np.arange(LI), indexing="ij")
    return ((J > 0) & (J < LJ - 1) & (I > 0) & (I < LI - 1)).reshape(-1, order="F")


def test_faces_match_oracle(cuda, oracle, case):
    g = case
    n = LJ * LI
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"])
        u.props()
        u.set_grid(LJ, LI, g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=1)
        u.set_flow(g["u"], g["v"], g["tmu"], 0.7)
        faces = u.assemble_faces(1e-3)
    yc, mu, lam, vdf, _ = oracle.props(g["tk"], g["y"])
    ref = oracle.faces(LJ, LI, g["rho"], vdf, g["u"], g["v"], g["tmu"], g["yr"], g["xxs"], g["xxc"], g["yys"],
                       g["yyc"], isym=1, dt=1e-3, sigsp=0.7)
    inside = interior_mask()
    scale = np.max(np.abs(np.stack(ref)), axis=0)
    for a, b in zip(faces, ref):
        assert np.all(np.abs(a - b)[:, inside] <= 1e-10 * scale[:, inside] + 1e-300)
        assert np.all(a[:, ~inside] == 0.0)


def test_sweep_with_faces_matches_oracle(cuda, oracle, case):
    g = case
    n = LJ * LI
    dt = 1e-3
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"])
        u.set_grid(LJ, LI, g["xxs"], g["xxc"], g["yys"], g["yyc"], g["yr"], isym=1)
        u.set_flow(g["u"], g["v"], g["tmu"], 0.7)
        u.sweep(dt, isor=4, tol=0.0)
        _, _, y_gpu, _, _ = u.download()
    yc, mu, lam, vdf, _ = oracle.props(g["tk"], g["y"])
    e, w, nn, s = oracle.faces(LJ, LI, g["rho"], vdf, g["u"], g["v"], g["tmu"], g["yr"], g["xxs"], g["xxc"],
                               g["yys"], g["yyc"], isym=1, dt=dt, sigsp=0.7)
    inside = interior_mask()
    Y = yc[:51]
    fsum = np.where(inside, e + w + nn + s, 0.0)
    fnbr = np.zeros_like(fsum)
    idx = np.nonzero(inside)[0]
    fnbr[:, idx] = (nn[:, idx] * Y[:, idx + 1] + s[:, idx] * Y[:, idx - 1] + e[:, idx] * Y[:, idx + LJ]
                    + w[:, idx] * Y[:, idx - LJ])
    rc, sour = oracle.rates(g["tk"], g["rho"], yc)
    y_o, _, _ = oracle.species_update(g["rho"], yc, rc, sour, dt, isor=4, tol=0.0, face_sum=fsum, face_nbr=fnbr)
    err = np.abs(y_gpu - y_o)[:, inside] - (1e-9 * np.abs(y_o[:, inside]) + 1e-18)
    assert (err <= 0).all(), err.max()
    assert np.array_equal(y_gpu[:, ~inside], yc[:, ~inside])        # boundary cells are held
    # the faces move the interior: the same sweep without them differs
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"])
        u.sweep(dt, isor=4, tol=0.0)
        _, _, y_nf, _, _ = u.download()
    assert np.abs(y_nf - y_gpu)[:, inside].max() > 1e-6


def test_fdetail_fields_match_oracle(cuda, oracle, case, tmp_path):
    """uc_fdetail (regular-grid fields of stdata.f:26-118) after a sweep, against the oracle on
    the same device state, and the file the writer makes of them."""
    from unicorn_b200.fdetail import read_fdetail, write_fdetail
    g = case
    n = LJ * LI
    rng = np.random.default_rng(9)
    xs, ys = np.cumsum(rng.uniform(0.5, 1.5, LI)) / LJ, np.cumsum(rng.uniform(0.5, 1.5, LJ)) / LJ
    x = np.tile(xs[None, :], (LJ, 1)).reshape(-1, order="F")
    y = np.tile(ys[:, None], (1, LI)).reshape(-1, order="F")
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"])
        u.sweep(1e-3, isor=2, tol=0.0)
        tk, rho, yy, _, _ = u.download()
        out = {k: np.empty((52, n)) if k in ("qdsp", "vdf") else np.empty(n) for k in ("qdsp", "qdot", "vmu", "vtc", "vdf")}
        u.download_outputs(out)
        fd = u.fdetail(LJ, LI, x, y, g["u"], g["v"])
    ref = oracle.fdetail(LJ, LI, x, y, rho, g["u"], g["v"], tk, out["qdot"], out["vmu"], out["vtc"], yy, out["vdf"],
                         out["qdsp"])
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.all(np.abs(fd - ref) <= 1e-12 * np.abs(ref) + 1e-14 * scale)
    p = tmp_path / "FDETAIL"
    write_fdetail(p, fd, LJ, LI, itr=1, ttime=1e-5)
    _, _, _, back = read_fdetail(p)
    assert np.allclose(back, fd, rtol=5.1e-7, atol=0)


def test_restart_round_trip_resumes(cuda, oracle, case, tmp_path):
    """A device state saved in the reference's restart layout and loaded into a fresh context
    gives the same next sweep (to the 8 digits the file keeps)."""
    g = case
    n = LJ * LI
    flow = dict(X=np.zeros(n), Y=g["yr"], U=g["u"], V=g["v"], W=np.zeros(n), P=np.zeros(n))
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"])
        u.sweep(1e-3, isor=3, tol=0.0)
        u.save_restart(tmp_path / "FLAMEA", LJ, LI, flow, infuel=11, itr=1)
        tk_s, rho_s, y_s, _, _ = u.download()
        y_saved = (tk_s, rho_s, y_s)
        u.sweep(1e-3, isor=3, tol=0.0)
        _, _, y_a, _, _ = u.download()
    with cuda.UniChem(n) as u2:
        h, f = u2.load_restart(tmp_path / "FLAMEA")
        assert (h["LJ"], h["LI"]) == (LJ, LI) and np.allclose(f["U"], g["u"], rtol=5.1e-8)
        tk_l, rho_l, y_l, _, _ = u2.download()
        assert np.allclose(tk_l, y_saved[0], rtol=5.1e-8, atol=0) and np.allclose(rho_l, y_saved[1], rtol=5.1e-8, atol=0)
        assert np.allclose(y_l[:51], y_saved[2][:51], rtol=5.1e-8, atol=0)
        u2.sweep(1e-3, isor=3, tol=0.0)
        _, _, y_b, _, _ = u2.download()
    # the continuation from the 8-digit state: almost every value to 1e-6 relative; values near
    # zero can land on either side of the update's clip at 0, so the bound for all is absolute
    big = y_a > 1e-10
    rel = np.abs(y_b - y_a)[big] / y_a[big]
    assert np.mean(rel <= 1e-6) > 0.999, np.mean(rel <= 1e-6)
    assert np.abs(y_b - y_a).max() <= 1e-6
