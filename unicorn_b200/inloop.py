"""In-loop use of the hot path: a field advanced sweep after sweep.

Each sweep is the species sweep of the reference's time step (uc_sweep:
properties, cp/h, rates, omega, the point-implicit update) followed by the
T update at constant total enthalpy per cell and rho at the cell pressure
(uc_temperature_from_held). Transport is frozen: the face coefficients of
the species equations and the neighbours' mass fractions are those of the
initial field, built here as a plain diffusion operator on the (z, r) grid
(the reference assembles them in SPGSOLV, src/lib/spgsolv.f:233-1290, which
is outside this library): between neighbouring cells a face carries
a = Gamma_f / Delta^2 with Gamma_f the mean of the two cells' VDFSP_k and
Delta = 1/(nr-1) (the radius is the length scale), so that

    face_sum_k = -DT * sum_f a_f,    face_nbr_k = -DT * sum_f a_f * Y_k(neighbour),

the sign convention of SOLVESP (PPP = RHO - face_sum, RHS1 - face_nbr).
"""
from __future__ import annotations

import numpy as np

LSP = 52


def frozen_faces(shape, vdf: np.ndarray, y: np.ndarray, dt: float):
    """face_sum, face_nbr [51, n] for a (nz, nr) field with r fastest."""
    nz, nr = shape
    n = nz * nr
    delta = 1.0 / (nr - 1)
    G = vdf[:LSP - 1].reshape(LSP - 1, nz, nr)
    Y = y[:LSP - 1].reshape(LSP - 1, nz, nr)
    fs = np.zeros_like(G)
    fn = np.zeros_like(G)
    for axis in (1, 2):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis] = slice(0, -1)
        hi[axis] = slice(1, None)
        lo, hi = tuple(lo), tuple(hi)
        a = 0.5 * (G[lo] + G[hi]) / delta ** 2
        fs[lo] += a
        fs[hi] += a
        fn[lo] += a * Y[hi]
        fn[hi] += a * Y[lo]
    return (-dt * fs).reshape(LSP - 1, n), (-dt * fn).reshape(LSP - 1, n)


def omega_error(q: np.ndarray, exact: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Per cell: max over species with Y > 1e-8 of |q - exact| / max(|exact|, 1e-6 max_j |exact_j|)."""
    wmax = np.abs(exact).max(axis=0)
    r = np.abs(q - exact) / np.maximum(np.abs(exact), 1e-6 * wmax + 1e-300)
    r[y <= 1e-8] = 0.0
    return r.max(axis=0)
