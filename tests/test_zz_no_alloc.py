"""uc_species_update_noalloc against the regular uc_species_update, through the C ABI.

Why the entry point exists: some hosts cannot let a library allocate device
memory -- all their device arrays come from their own allocator or pool (a
Fortran code with CUDA Fortran or OpenACC device arrays, a solver held to a
fixed memory budget). uc_species_update_noalloc works only on the caller's
device arrays and keeps its one piece of scratch (the residual partial sums
and the pass counter) in a fixed array inside the library.

The file name makes pytest collect it last; it also passes on its own in a
fresh process. Tolerance: that of the other species-update tests
(1e-9 relative, 1e-18 absolute).
"""
import ctypes

import numpy as np
import pytest

from unicorn_b200.fields import jet_field, nondimensional

pytestmark = pytest.mark.gpu


class UpdateArrays(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("npad", ctypes.c_int)] + \
               [(k, ctypes.c_void_p) for k in ("rc", "sour", "rho", "y0", "soot0", "face_sum", "face_nbr", "y", "soot")]


def _padded(torch, host_rows, npad):
    """A caller-owned [rows][npad] device array; padding cells copy the last cell."""
    rows, n = host_rows.shape
    a = np.empty((rows, npad))
    a[:, :n] = host_rows
    a[:, n:] = host_rows[:, n - 1:n]
    return torch.from_numpy(a).to("cuda")


def test_noalloc_update_matches_regular_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from oracle.oracle import Oracle
    from unicorn_b200 import unichem
    lib = unichem.load_library()
    lib.uc_species_update_noalloc.argtypes = [ctypes.c_void_p, ctypes.POINTER(UpdateArrays), ctypes.c_double,
                                             ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.POINTER(ctypes.c_int)]
    f = jet_field(61, 43, fuel=11, t_peak=2300.0, seed=12)        # 2,623 cells: not a multiple of 32
    n = f.n
    npad = (n + 31) // 32 * 32
    u = unichem.UniChem(n)
    tk, rho = nondimensional(f, u.scales, u.wm)
    _, sour = Oracle().rates(tk, rho, f.y)            # soot source terms of this state (host libm; ~1 ulp)
    for call, (isor, tol) in enumerate([(3, 0.0), (40, 1e-8)]):
        # regular entry point: the context's own device arrays
        u.upload(tk, rho, f.y)
        rc_host = u.ckrates(return_rc=True)
        p_regular = u.solvesp(1e-3, isor=isor, relx=0.99, tol=tol)
        _, _, y_regular, s1_regular, s2_regular = u.download()
        # no-allocation entry point: the caller's device arrays, same state
        d_rc = _padded(torch, rc_host, npad)
        d_sour = _padded(torch, sour, npad)
        d_rho = _padded(torch, rho[None, :], npad)
        d_y0 = _padded(torch, f.y, npad)
        d_soot0 = torch.zeros((2, npad), dtype=torch.float64, device="cuda")
        d_y = d_y0.clone()
        d_soot = d_soot0.clone()
        arr = UpdateArrays(n, npad, d_rc.data_ptr(), d_sour.data_ptr(), d_rho.data_ptr(), d_y0.data_ptr(),
                           d_soot0.data_ptr(), None, None, d_y.data_ptr(), d_soot.data_ptr())
        # the arrays were filled on torch's stream; the call runs on the context's own
        # stream, which is not ordered after it
        torch.cuda.synchronize()
        passes = ctypes.c_int(-1)
        rc = lib.uc_species_update_noalloc(u._h, ctypes.byref(arr), 1e-3, isor, 0.99, tol, 0.0,
                                           ctypes.byref(passes))
        assert rc == 0, lib.uc_last_error(u._h).decode()
        assert passes.value == p_regular, f"call {call}: {passes.value} passes, regular entry point {p_regular}"
        y_noalloc = d_y.cpu().numpy()[:, :n]
        soot = d_soot.cpu().numpy()[:, :n]
        err = np.abs(y_noalloc - y_regular)
        assert np.all(err <= 1e-9 * np.abs(y_regular) + 1e-18), f"call {call}: max error {err.max():.3g}"
        assert np.all(np.abs(soot[0] - s1_regular) <= 1e-9 * np.abs(s1_regular) + 1e-30)
        assert np.all(np.abs(soot[1] - s2_regular) <= 1e-9 * np.abs(s2_regular) + 1e-30)
    # a row stride that is not a multiple of 32 is refused before anything runs
    bad = UpdateArrays(n, npad + 1, d_rc.data_ptr(), d_sour.data_ptr(), d_rho.data_ptr(), d_y0.data_ptr(),
                       d_soot0.data_ptr(), None, None, d_y.data_ptr(), d_soot.data_ptr())
    assert lib.uc_species_update_noalloc(u._h, ctypes.byref(bad), 1e-3, 1, 0.99, 0.0, 0.0, None) == -1
    assert b"multiple of 32" in lib.uc_last_error(u._h)
    u.close()
