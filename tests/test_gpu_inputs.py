"""Inputs at the C ABI: invalid arguments are refused with UC_E_ARG before anything runs, and a cell with
non-finite inputs stays its own (the reference has no input checks; a NaN cell gives NaN results for that
cell, and its NaN residual keeps the update from meeting any tolerance, as SOLVESP's test
RSD/SPNORM <= TOLRSP, solvesp.f:2833, is then false)."""
import ctypes

import numpy as np
import pytest

from conftest import random_state

pytestmark = pytest.mark.gpu


def test_invalid_arguments_are_refused(oracle):
    from unicorn_b200 import unichem
    tk, rho, y = random_state(oracle, 256, 3)
    with unichem.UniChem(256) as u:
        with pytest.raises(unichem.UniChemError) as e:
            u.solvesp(1e-3)                                   # no rate plane yet
        assert e.value.code == -3
        u.upload(tk, rho, y)
        u.ckrates()
        for kw in (dict(isor=0), dict(relx=0.0), dict(relx=float("nan"))):
            with pytest.raises(unichem.UniChemError) as e:
                u.solvesp(1e-3, **kw)
            assert e.value.code == -1, kw
        with pytest.raises(unichem.UniChemError) as e:
            u.solvesp(-1.0)
        assert e.value.code == -1
        with pytest.raises(unichem.UniChemError) as e:
            u.sweep(1e-3, precision=7)
        assert e.value.code == -1
        assert u.lib.uc_upload_fields_device(u._h, 1, 1, 1, None, None, 255) == -1      # row stride below n
        assert u.lib.uc_upload_fields(u._h, None, None, None, None, None) == -1
        assert u.lib.uc_stat(u._h, b"no such statistic", unichem._p(np.zeros(1))) == -1
    bad = unichem.Inputs(**{**unichem.DEFAULT_INPUTS, "rtot": 0.0})
    h = ctypes.c_void_p()
    assert unichem.load_library().uc_init(ctypes.byref(bad), 10, 0, ctypes.byref(h)) == -1 and not h.value


def test_nan_cell_stays_its_own(oracle):
    from unicorn_b200 import unichem
    tk, rho, y = random_state(oracle, 4096, 4, 900, 2500)
    bad = 1000
    tk_nan = tk.copy()
    tk_nan[bad] = np.nan
    out = {}
    for name, t in (("clean", tk), ("nan", tk_nan)):
        with unichem.UniChem(4096) as u:
            u.upload(t, rho, y)
            om = u.omega()
            mu, lam, dk = u.props()
            u.upload(t, rho, y)
            u.ckrates()
            passes = u.solvesp(1e-3, isor=5, tol=1e-30)
            yn = u.download()[2]
            out[name] = (om.qdsp, mu, dk, passes, yn)
    c, n = out["clean"], out["nan"]
    others = np.arange(4096) != bad
    assert np.isnan(n[0][:, bad]).any()
    for i in (0, 1, 2, 4):
        assert np.array_equal(n[i][..., others], c[i][..., others])
    assert n[3] == 6 and c[3] == 6               # tol 1e-30 is not met in 5 passes either way
