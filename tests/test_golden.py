"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py
from the reference's own routines) against the CPU oracle, bit for bit, and
against the CUDA path through the C ABI within the FP64 parity tolerances."""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    return dict(np.load(GOLD / name))


# ----------------------------------------------------------------- oracle (CPU)

def test_oracle_rates_omega(oracle):
    g = load("rates_omega.npz")
    rc, sour = oracle.rates(g["tk"], g["rho"], g["y"], g["stmf"], g["stnd"])
    assert np.array_equal(rc, g["rc"]) and np.array_equal(sour, g["sour"])
    q, qd, h, _ = oracle.omega(g["tk"], g["rho"], g["y"], g["stmf"], g["stnd"])
    assert np.array_equal(q, g["qdsp"]) and np.array_equal(qd, g["qdot"]) and np.array_equal(h, g["henth"])


def test_oracle_cp_props(oracle):
    g = load("cp_props.npz")
    assert np.array_equal(oracle.cp(g["tk"], g["y"]), g["tcp"])
    yc, mu, lam, d, _ = oracle.props(g["tk"], g["y"])
    for a, k in ((yc, "yc"), (mu, "vmu"), (lam, "vtc"), (d, "vdf")):
        assert np.array_equal(a, g[k]), k


@pytest.mark.parametrize("tag", ["a", "b"])
def test_oracle_update(oracle, tag):
    g = load("update.npz")
    rc, sour = oracle.rates(g["tk"], g["rho"], g["y"])
    y, soot, passes = oracle.species_update(g["rho"], g["y"], rc, sour, float(g["dt"]),
                                            isor=int(g[f"isor_{tag}"]), relx=float(g["relx"]),
                                            tol=float(g[f"tol_{tag}"]), spnorm=float(g["spnorm"]))
    assert passes == int(g[f"passes_{tag}"])
    assert np.array_equal(y, g[f"y_{tag}"])
    assert np.array_equal(soot[0], g[f"stmf_{tag}"]) and np.array_equal(soot[1], g[f"stnd_{tag}"])


def test_oracle_temperature(oracle):
    g = load("temperature.npz")
    assert np.array_equal(oracle.temperature(g["guess"], g["y"], g["ht"]), g["tk"])


# ----------------------------------------------------------------- CUDA path

@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


def rel_ok(a, b, rtol, atol):
    return np.all(np.abs(a - b) <= rtol * np.abs(b) + atol)


@pytest.mark.gpu
def test_cuda_rates_omega(cuda, oracle):
    from test_gpu_parity import gross
    g = load("rates_omega.npz")
    n = len(g["tk"])
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"], g["stmf"], g["stnd"])
        rc = u.ckrates(return_rc=True)
        om = u.omega()
    assert rel_ok(rc, g["rc"], 1e-11, 1e-300)
    gr = gross(oracle, g["tk"], g["rho"], g["y"])
    assert np.all(np.abs(om.qdsp - g["qdsp"]) <= 1e-11 * gr + 1e-300)


@pytest.mark.gpu
def test_cuda_props(cuda):
    g = load("cp_props.npz")
    n = len(g["tk"])
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], np.ones(n), g["y"])
        cp, _ = u.cp_h()
        mu, lam, dk = u.props()
    assert rel_ok(cp, g["tcp"], 1e-11, 0)
    assert rel_ok(mu, g["vmu"], 1e-11, 0) and rel_ok(lam, g["vtc"], 1e-11, 0)
    assert rel_ok(dk, g["vdf"], 1e-11, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["a", "b"])
def test_cuda_update(cuda, tag):
    g = load("update.npz")
    n = len(g["tk"])
    with cuda.UniChem(n) as u:
        u.upload(g["tk"], g["rho"], g["y"])
        u.ckrates()
        passes = u.solvesp(dt=float(g["dt"]), isor=int(g[f"isor_{tag}"]), relx=float(g["relx"]),
                           tol=float(g[f"tol_{tag}"]), spnorm=float(g["spnorm"]))
        _, _, y, stmf, stnd = u.download()
    assert passes == int(g[f"passes_{tag}"])
    assert rel_ok(y, g[f"y_{tag}"], 1e-9, 1e-18)
