"""The FP64 species update through the shared-memory RC ring
(update_staged_kernel, selected with UNICHEM_UPDATE=staged at uc_init)
against the oracle and against the register-fed update_kernel: the same pass
counts, Y within 1e-9 of the oracle (the tolerance of the FP64 update
tests), on the C1 field, a many-tile batch that runs several rounds and
passes per warp (so the row stream crosses tiles and passes), frozen
transport terms and held boundary cells."""
import numpy as np
import pytest

from test_gpu_parity import assert_rel, c1  # noqa: F401  (c1: the 101x61 CH4 field)
from unicorn_b200.fields import batch_cells, nondimensional

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


def run_update(cuda, monkeypatch, kind, tk, rho, y, **kw):
    monkeypatch.setenv("UNICHEM_UPDATE", kind)
    with cuda.UniChem(len(tk)) as u:
        assert u.stat("update_staged") == (1.0 if kind == "staged" else 0.0)
        u.upload(tk, rho, y)
        u.ckrates()
        passes = u.solvesp(1e-3, **kw)
        _, _, yg, s1, _ = u.download()
    return passes, yg, s1


@pytest.mark.parametrize("isor,tol", [(1, 1e-8), (5, 0.0)])
def test_staged_matches_oracle(cuda, oracle, monkeypatch, c1, isor, tol):
    tk, rho, y = c1
    passes, yg, s1 = run_update(cuda, monkeypatch, "staged", tk, rho, y, isor=isor, relx=0.99, tol=tol)
    rc, sour = oracle.rates(tk, rho, y)
    yo, so, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=isor, tol=tol)
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y after update")
    assert_rel(s1, so[0], 1e-9, 1e-30, "soot mass fraction")


def test_staged_many_rounds_matches_plain(cuda, oracle, monkeypatch):
    """65,536 cells: 2,048 tiles, several rounds per warp, converged passes."""
    f = batch_cells(65536, seed=5)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    pa, ya, sa = run_update(cuda, monkeypatch, "plain", tk, rho, f.y, isor=100, relx=0.99, tol=1e-8)
    pb, yb, sb = run_update(cuda, monkeypatch, "staged", tk, rho, f.y, isor=100, relx=0.99, tol=1e-8)
    assert pa == pb and pa > 3
    assert_rel(yb, ya, 1e-9, 1e-18, "Y staged vs plain")             # FMA contraction differs between the two
    # against the oracle at the tolerance of the converged-update test of the register-fed kernel
    sl = slice(0, 2048)
    rc, sour = oracle.rates(tk[sl], rho[sl], f.y[:, sl])
    yo, _, _ = oracle.species_update(rho[sl], f.y[:, sl], rc, sour, 1e-3, isor=pa, tol=0.0)
    err_a = np.max(np.abs(ya[:, sl] - yo) / (1e-7 * np.abs(yo) + 1e-16))
    err_b = np.max(np.abs(yb[:, sl] - yo) / (1e-7 * np.abs(yo) + 1e-16))
    assert err_b <= max(1.0, 2.0 * err_a), (err_a, err_b)


def test_staged_frozen_transport(cuda, oracle, monkeypatch, c1):
    tk, rho, y = c1
    n = len(tk)
    rng = np.random.default_rng(4)
    fs = rng.uniform(-0.02, 0.0, (51, n)) * rho
    fn = fs * y[:51] * rng.uniform(0.9, 1.1, (51, n))
    passes, yg, _ = run_update(cuda, monkeypatch, "staged", tk, rho, y, isor=3, tol=0.0, face_sum=fs, face_nbr=fn)
    rc, sour = oracle.rates(tk, rho, y)
    yo, _, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=3, tol=0.0, face_sum=fs, face_nbr=fn)
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y with frozen transport")
