"""The CPU oracle of the surrogate network (oracle/mlp_oracle.py): with the
BF16 rounding switched off its gradient must match central differences of
its own loss, which pins the backward formulas the GPU kernels are checked
against."""
import numpy as np

from oracle import mlp_oracle as mo


def test_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(mo, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(0)
    n = sum(o * i + o for i, o in zip(mo.IN, mo.OUT))
    w = rng.uniform(-0.1, 0.1, n)
    x = np.zeros((8, 64))
    x[:, :54] = rng.standard_normal((8, 54))
    t = np.zeros((8, 64))
    t[:, :52] = rng.standard_normal((8, 52))
    loss, g = mo.forward_backward(w, x, t)
    # a few parameters of every layer, including biases
    offs, off = [], 0
    for i, o in zip(mo.IN, mo.OUT):
        offs += [off + 3, off + o * i // 2, off + o * i + 1]
        off += o * i + o
    for p in offs:
        if p >= off:
            continue
        wp, wm = w.copy(), w.copy()
        h = 1e-6
        wp[p] += h
        wm[p] -= h
        num = (mo.forward_backward(wp, x, t)[0] - mo.forward_backward(wm, x, t)[0]) / (2 * h)
        assert abs(num - g[p]) <= 1e-6 * max(1.0, abs(g[p])) + 1e-9, (p, num, g[p])


def test_padded_outputs_carry_no_gradient():
    rng = np.random.default_rng(1)
    n = sum(o * i + o for i, o in zip(mo.IN, mo.OUT))
    w = rng.uniform(-0.1, 0.1, n)
    x = mo.bf16(rng.standard_normal((64, 64)))
    t = rng.standard_normal((64, 64))
    _, g = mo.forward_backward(w, x, t)
    W4, b4 = mo.unpack(g)[4]
    assert np.all(W4[52:] == 0) and np.all(b4[52:] == 0)
