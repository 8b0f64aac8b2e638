import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libunichem.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    """The reference's own routines, translated to C (oracle/_ref)."""
    from oracle import ref as R
    if not R.available():
        from unicorn_b200.refsrc import reference_root
        src = str(reference_root())
        if Path(src).exists():
            from oracle.build_ref import build
            build(src, 34, 66)
    if not R.available():
        pytest.skip("oracle/_ref (the translated reference) is not built on this host")
    return R.RefUnicorn()


def random_state(o, n, seed, tlo=300.0, thi=2600.0):
    """Random but physical cells: O2/N2/fuel majors plus log-uniform minors."""
    rng = np.random.default_rng(seed)
    y = 10 ** rng.uniform(-10, -3, (52, n))
    y[1] = rng.uniform(0.05, 0.23, n)
    y[51] = 0.7
    y[12] = rng.uniform(0.0, 0.1, n)
    y[46] = rng.uniform(0.0, 0.05, n)
    y /= y.sum(0)
    T = rng.uniform(tlo, thi, n)
    tk = T / o.scales["TSTR"]
    rho = o.scales["PBACK"] / (o.scales["BETA1"] * tk * (y / o.wm[:, None]).sum(0))
    return tk, rho, y
