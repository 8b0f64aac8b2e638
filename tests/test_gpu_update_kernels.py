"""The FP64 species-update kernels against each other and the oracle: the
default tile-resident one (update_tr_kernel: RC blocks on chip across a chunk
of passes), the per-pass one with Y in place (UNICHEM_UPDATE=inplace,
update_kernel<double, 14, true>) and the per-pass two-Y-set one
(UNICHEM_UPDATE=twoset, 8 warps per SM), selected at uc_init.
Same pass counts, Y within 1e-9 of the oracle (the tolerance of the FP64
update tests), on the C1 field, a many-tile batch that runs several rounds per
warp, frozen transport terms, and stopping passes inside and at the end of a
chunk of the tile-resident kernel."""
import numpy as np
import pytest

from conftest import random_state
from test_gpu_parity import assert_rel, c1  # noqa: F401  (c1: the 101x61 CH4 field)
from unicorn_b200.fields import batch_cells, nondimensional

pytestmark = pytest.mark.gpu
KINDS = ["resident", "inplace", "twoset"]
KIND_ID = {"resident": 0, "inplace": 1, "twoset": 2}


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


def run_update(cuda, monkeypatch, kind, tk, rho, y, chunk=None, **kw):
    monkeypatch.setenv("UNICHEM_UPDATE", kind)
    if chunk is not None:
        monkeypatch.setenv("UNICHEM_TR_CHUNK", str(chunk))
    with cuda.UniChem(len(tk)) as u:
        assert u.stat("update_kind") == KIND_ID[kind]
        u.upload(tk, rho, y)
        u.ckrates()
        passes = u.solvesp(1e-3, **kw)
        _, _, yg, s1, _ = u.download()
    return passes, yg, s1


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("isor,tol", [(1, 1e-8), (5, 0.0)])
def test_inplace_matches_oracle(cuda, oracle, monkeypatch, c1, kind, isor, tol):
    tk, rho, y = c1
    passes, yg, s1 = run_update(cuda, monkeypatch, kind, tk, rho, y, isor=isor, relx=0.99, tol=tol)
    rc, sour = oracle.rates(tk, rho, y)
    yo, so, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=isor, tol=tol)
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y after update")
    assert_rel(s1, so[0], 1e-9, 1e-30, "soot mass fraction")


def test_inplace_many_rounds_matches_twoset(cuda, oracle, monkeypatch):
    """65,536 cells: 2,048 tiles, several rounds per warp, converged passes."""
    f = batch_cells(65536, seed=5)
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    pa, ya, _ = run_update(cuda, monkeypatch, "twoset", tk, rho, f.y, isor=100, relx=0.99, tol=1e-8)
    pb, yb, _ = run_update(cuda, monkeypatch, "inplace", tk, rho, f.y, isor=100, relx=0.99, tol=1e-8)
    pc, yc, _ = run_update(cuda, monkeypatch, "resident", tk, rho, f.y, isor=100, relx=0.99, tol=1e-8)
    assert pa == pb == pc and pa > 3
    assert_rel(yb, ya, 1e-9, 1e-18, "Y in place vs two Y sets")
    assert_rel(yc, ya, 1e-9, 1e-18, "Y tile-resident vs two Y sets")


@pytest.mark.parametrize("chunk", [1, 3, 8, 16])
def test_resident_chunks_stop_where_the_per_pass_kernel_stops(cuda, oracle, monkeypatch, chunk):
    """The converging pass falls inside a chunk, at its end or in a later chunk depending on the
    chunk length; pass count and Y equal those of the per-pass kernel."""
    # 2,000 random cells at 1000-2000 K (which converge at 1e-3 in 39 passes on the oracle) repeated
    # 32 times: 2,000 tiles, several per warp, with the same mean residual per pass
    tk1, rho1, y1 = random_state(oracle, 2000, 4, 1000, 2000)
    tk, rho, y = np.tile(tk1, 32), np.tile(rho1, 32), np.tile(y1, (1, 32))
    pa, ya, sa = run_update(cuda, monkeypatch, "inplace", tk, rho, y, isor=100, relx=0.99, tol=1e-3)
    pc, yc, sc = run_update(cuda, monkeypatch, "resident", tk, rho, y, chunk=chunk, isor=100, relx=0.99, tol=1e-3)
    assert 5 <= pa <= 60, pa
    assert pc == pa
    print(f"\nchunk {chunk}: {pc} passes; Y values differing from the per-pass kernel: {(yc != ya).sum()}")
    assert_rel(yc, ya, 1e-12, 1e-30, "Y tile-resident vs in place")      # the same arithmetic in the same order
    assert_rel(sc, sa, 1e-12, 1e-30, "soot tile-resident vs in place")


@pytest.mark.parametrize("kind", KINDS)
def test_inplace_frozen_transport(cuda, oracle, monkeypatch, c1, kind):
    tk, rho, y = c1
    n = len(tk)
    rng = np.random.default_rng(4)
    fs = rng.uniform(-0.02, 0.0, (51, n)) * rho
    fn = fs * y[:51] * rng.uniform(0.9, 1.1, (51, n))
    passes, yg, _ = run_update(cuda, monkeypatch, kind, tk, rho, y, isor=3, tol=0.0, face_sum=fs, face_nbr=fn)
    rc, sour = oracle.rates(tk, rho, y)
    yo, _, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=3, tol=0.0, face_sum=fs, face_nbr=fn)
    assert passes == po
    assert_rel(yg, yo, 1e-9, 1e-18, "Y with frozen transport")


def test_inplace_mixed_matches_twoset(cuda, oracle, monkeypatch, c1):
    """The mixed form (FP32 RC plane, flagged tiles from the FP64 plane) through both kernels."""
    tk, rho, y = c1
    out = {}
    for kind in ("twoset", "inplace"):
        monkeypatch.setenv("UNICHEM_UPDATE", kind)
        with cuda.UniChem(len(tk)) as u:
            u.upload(tk, rho, y)
            passes = u.sweep(1e-3, precision=cuda.MIXED, isor=100, relx=0.99, tol=1e-8)
            assert u.stat("mixed_fp64_tiles") > 0            # both planes are read
            out[kind] = (passes, u.download()[2])
    assert out["twoset"][0] == out["inplace"][0]
    assert_rel(out["inplace"][1], out["twoset"][1], 1e-9, 1e-18, "mixed Y in place vs two Y sets")


def test_resident_chunk_schedule_from_the_last_call(cuda, oracle, monkeypatch):
    """By default the tile-resident update lengthens its chunks (up to 32 passes) while the previous
    call's pass count says more passes are to come; UNICHEM_TR_CHUNK fixes them. The schedule changes
    only which passes run beyond the stopping one, so two runs of the same call sequence -- a converging
    update, a second one from its result, and two that run every pass -- agree bit for bit."""
    tk1, rho1, y1 = random_state(oracle, 2000, 4, 1000, 2000)
    tk, rho, y = np.tile(tk1, 32), np.tile(rho1, 32), np.tile(y1, (1, 32))

    def run(fixed):
        monkeypatch.setenv("UNICHEM_UPDATE", "resident")
        if fixed:
            monkeypatch.setenv("UNICHEM_TR_CHUNK", "16")
        else:
            monkeypatch.delenv("UNICHEM_TR_CHUNK", raising=False)
        out = []
        with cuda.UniChem(len(tk)) as u:
            u.upload(tk, rho, y)
            for isor, tol in ((100, 1e-3), (100, 1e-3), (100, 0.0), (100, 0.0)):
                u.ckrates()
                p = u.solvesp(1e-3, isor=isor, relx=0.99, tol=tol)
                _, _, yg, s1, _ = u.download()
                out.append((p, yg, s1))
        return out

    a, b = run(True), run(False)
    print("\npasses per call:", [x[0] for x in a])
    assert a[2][0] == a[3][0] == 101 and 5 <= a[0][0] <= 60
    for (pa, ya, sa), (pb, yb, sb) in zip(a, b):
        assert pa == pb
        assert np.array_equal(ya, yb) and np.array_equal(sa, sb)
