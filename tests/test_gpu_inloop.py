"""In-loop sweeps (the C5 form) on the GPU against the oracle, sweep by sweep.

A 41 x 21 heptane jet field with frozen diffusion faces (unicorn_b200/inloop.py)
is advanced three sweeps on the device: uc_sweep with the faces (properties
with the Y clip, cp/h, rates, the point-implicit update to 1e-8 over the whole
field, closure) and uc_temperature_from_held (T at the held total enthalpy,
rho at the cell pressure). Each sweep is recomputed by the oracle from the
device's state before it (so differences do not compound): oracle props (the
clip), rates, species update with the same faces, held-enthalpy T step.

Tolerances: pass counts equal; Y to 1e-9 relative and 1e-18 absolute (the
FP64 kernels differ from the host libm by an ulp and contract multiply-adds);
T to 2e-3 K (the Newton stops on a step of 1e-3 K); rho to 1e-6 relative
(it follows T). Cells on the reference's T clamp, or whose T Newton did not
meet its step rule in 100 steps (the reference prints a message and carries
on; where such a Newton stops depends on the last ulp), are counted, not
compared: at most 5 % (observed at most 39 of 861: ambient cells whose
enthalpy falls below h(TSTR - 1), and a few above 5000 K). The closure of the device
state: sum Y + soot = 1 to 1e-14. (The held enthalpy is not an exact
invariant of the reference's T step: the Newton picks its polynomial range by
its own test, not by T > TPOL1.)"""
import numpy as np
import pytest

from unicorn_b200.fields import jet_field, nondimensional
from unicorn_b200.inloop import frozen_faces

pytestmark = pytest.mark.gpu

DT = 1e-3
NZ, NR = 41, 21


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from unicorn_b200 import unichem
    return unichem


def test_inloop_sweeps_match_the_oracle(cuda, oracle):
    f = jet_field(NZ, NR, fuel=11, t_peak=2300.0, seed=0)
    n = f.n
    with cuda.UniChem(n) as u:
        tk, rho = nondimensional(f, u.scales, u.wm)
        pnd = f.p / u.scales["PSTR"]
        u.upload(tk, rho, f.y)
        u.set_pressure(pnd)
        vdf = u.props()[2]
        _, _, yc, _, _ = u.download()
        fs, fn = frozen_faces((NZ, NR), vdf, yc, DT)
        u.upload(tk, rho, f.y)
        enth = oracle.enthalpy_total(tk, f.y)
        u.hold_enthalpy()
        for sweep in range(3):
            tk_b, rho_b, y_b, s1_b, s2_b = u.download()
            passes = u.sweep(DT, face_sum=fs, face_nbr=fn)
            u.temperature_from_held()
            tk_a, rho_a, y_a, s1_a, s2_a = u.download()
            # the oracle's sweep from the same state
            soot_b = np.stack([s1_b, s2_b])
            yc_o = oracle.props(tk_b, y_b)[0]
            rc, sour = oracle.rates(tk_b, rho_b, yc_o, s1_b, s2_b)
            y_o, s_o, p_o = oracle.species_update(rho_b, yc_o, rc, sour, DT, soot0=soot_b, face_sum=fs, face_nbr=fn)
            tk_o, rho_o, conv_o = oracle.temperature_held(tk_b, y_o, pnd, enth, with_conv=True)
            assert passes == p_o, f"sweep {sweep}: passes {passes} vs {p_o}"
            err = np.abs(y_a - y_o) - (1e-9 * np.abs(y_o) + 1e-18)
            assert (err <= 0).all(), f"sweep {sweep}: worst Y excess {err.max():.3g}"
            assert np.abs(s1_a - s_o[0]).max() <= 1e-9 * np.abs(s_o[0]).max() + 1e-18
            # cells whose T ends on a bound of the reference's clamp [TSTR-1, 5000 K] have left the model
            # (their Newton does not converge; where it stops depends on the last ulp): counted, not compared
            T_a, T_o = tk_a * u.scales["TSTR"], tk_o * u.scales["TSTR"]
            lo, hi = u.scales["TSTR"] - 1.0 + 1e-6, 5000.0 - 1e-6
            # the device's Newton met its rule where the oracle's Newton started from its result stays put
            tk_chk, _, conv_chk = oracle.temperature_held(tk_a, y_a, pnd, enth, with_conv=True)
            conv_a = conv_chk & (np.abs(tk_chk - tk_a) * u.scales["TSTR"] <= 2e-3)
            free = (T_a > lo) & (T_a < hi) & (T_o > lo) & (T_o < hi) & conv_o & conv_a
            print(f"sweep {sweep}: {passes} passes; cells not compared: {(~free).sum()} of {n} (T clamp below "
                  f"{(T_a <= lo).sum()}, above {(T_a >= hi).sum()}; Newton not converged: oracle {(~conv_o).sum()}, device {(~conv_a).sum()})")
            assert (~free).sum() <= 0.05 * n                 # observed: at most 39 of 861
            assert np.abs(T_a - T_o)[free].max() <= 2e-3
            assert np.allclose(rho_a[free], rho_o[free], rtol=1e-6, atol=0)
            # the closure of the device state
            assert np.abs(y_a.sum(axis=0) + s1_a - 1.0).max() <= 1e-14
