"""uc_sweep_host (one sweep on host buffers, the output copies overlapping the
species update) against the same sweep through uc_upload_fields, uc_sweep,
uc_download_outputs and uc_download_fields: bit for bit, with pageable and
with pinned host buffers, repeated calls on one context and soot given."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("qdsp", "qdot", "domega_dy", "vmu", "vtc", "vdf", "cp", "h")


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


def _outs(n, alloc):
    return {k: alloc((52, n)) if k in ("qdsp", "domega_dy", "vdf") else alloc((n,)) for k in KEYS}


def _sequential(u, tk, rho, y, soot):
    u.upload(tk, rho, y, stmf=soot[0], stnd=soot[1])
    passes = u.sweep(1e-5)
    out = u.download_outputs()
    _, _, y1, s1, s2 = u.download()
    return passes, out, y1, (s1, s2)


@pytest.mark.parametrize("pinned", [False, True])
def test_sweep_host_matches_the_call_sequence(cuda, pinned):
    import torch
    from unicorn_b200.fields import batch_cells, nondimensional
    n = 5000
    f = batch_cells(n, seed=3)
    if pinned:
        alloc = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    else:
        alloc = lambda shape: np.empty(shape)
    with cuda.UniChem(n) as u:
        tk, rho = nondimensional(f, u.scales, u.wm)
        rng = np.random.default_rng(4)
        soot = (rng.uniform(0, 1e-6, n), rng.uniform(0, 1e-3, n))
        ref = _sequential(u, tk, rho, f.y, soot)
        h_tk, h_rho, h_y = alloc((n,)), alloc((n,)), alloc((52, n))
        h_tk[:], h_rho[:], h_y[:] = tk, rho, f.y
        h_s = (alloc((n,)), alloc((n,)))
        h_s[0][:], h_s[1][:] = soot
        for _ in range(2):                       # the second call reuses the side stream
            outs, y_out, s_out = _outs(n, alloc), alloc((52, n)), (alloc((n,)), alloc((n,)))
            passes = u.sweep_host(h_tk, h_rho, h_y, out=outs, y_out=y_out, soot=h_s, soot_out=s_out, dt=1e-5)
            assert passes == ref[0]
            for k in KEYS:
                assert np.array_equal(outs[k], ref[1][k]), k
            assert np.array_equal(y_out, ref[2])
            assert np.array_equal(s_out[0], ref[3][0]) and np.array_equal(s_out[1], ref[3][1])


def test_sweep_host_partial_outputs_and_bad_arrays(cuda):
    from unicorn_b200.fields import batch_cells, nondimensional
    n = 700
    f = batch_cells(n, seed=5)
    with cuda.UniChem(n) as u:
        tk, rho = nondimensional(f, u.scales, u.wm)
        ref = _sequential(u, tk, rho, f.y, (np.zeros(n), np.zeros(n)))
        q = np.empty((52, n))
        y_out = np.empty((52, n))
        passes = u.sweep_host(np.ascontiguousarray(tk), np.ascontiguousarray(rho), np.ascontiguousarray(f.y),
                              out={"qdsp": q}, y_out=y_out)
        assert passes == ref[0]
        assert np.array_equal(q, ref[1]["qdsp"]) and np.array_equal(y_out, ref[2])
        with pytest.raises(ValueError):
            u.sweep_host(tk, rho, f.y.astype(np.float32), out={"qdsp": q})
        with pytest.raises(ValueError):
            u.sweep_host(tk, rho, f.y, out={"qdsp": np.empty((51, n))})
