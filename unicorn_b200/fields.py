"""Seeded synthetic fields of the benchmark configurations.

The reference ships no benchmark data, so the workloads are generated:

* ``jet_field(nz, nr, fuel, t_peak, seed)``: a jet-like mixture-fraction field
  on a (z, r) grid in grid units,
  (1) Z = exp(-(r/(0.2+0.02 z))^2) + N(0, 0.02^2) noise, clipped to [0, 1];
  (2) T = 300 + (t_peak-300) exp(-((Z-0.055)/0.08)^2) K;
  (3) fuel, O2, N2 by linear fuel/air mixing in Z (fuel stream pure fuel,
      air Y_O2 = 0.233, Y_N2 = 0.767; CO2 and H2O are zero in both streams
      and so stay 0);
  (4) the other 47 species log-uniform in [1e-10, 1e-3]; then all 52 are
      renormalised so that sum Y = 1.
  Cells are ordered like the reference's arrays: r (J) fastest.
* ``jet_flow(nz, nr, seed)``: geometry and a synthetic flow for that grid
  (uniform spacing 1/(nr-1), cell-centre radius, a spreading round jet with
  co-flow, seeded radial noise, an eddy viscosity that follows the jet).
* ``batch_cells(n, seed)``: n independent cells with compositions of the
  heptane generator, T ~ U[300, 2400] K and p ~ U[0.8, 1.2] atm.

Fuel numbers follow the reference (src/unicornd-mild-sd-5.f:301-317):
2 = CH4 (species 13), 11 = C7H16 (species 47).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

LSP = 52
ATM = 1.01325e5
FUEL_SPECIES = {1: 1, 2: 13, 3: 30, 4: 22, 5: 17, 6: 20, 7: 41, 8: 40, 9: 12, 10: 9, 11: 47}
O2, N2, CO2, H2O = 2, 52, 10, 6


@dataclass
class Field:
    T: np.ndarray        # [n] K
    p: np.ndarray        # [n] Pa
    y: np.ndarray        # [52, n] mass fractions
    shape: tuple         # (nz, nr) or (n,)
    seed: int
    fuel: int

    @property
    def n(self) -> int:
        return self.T.shape[0]


def _compose(Z: np.ndarray, fuel: int, rng: np.random.Generator) -> np.ndarray:
    n = Z.shape[0]
    kf = FUEL_SPECIES[fuel]
    y = np.zeros((LSP, n))
    majors = {kf, O2, N2, CO2, H2O}
    minors = [k for k in range(1, LSP + 1) if k not in majors]
    y[np.array(minors) - 1] = 10.0 ** rng.uniform(-10.0, -3.0, size=(len(minors), n))
    y[kf - 1] = Z
    y[O2 - 1] = (1.0 - Z) * 0.233
    y[N2 - 1] = (1.0 - Z) * 0.767
    y /= y.sum(axis=0, keepdims=True)
    return y


def jet_field(nz: int, nr: int, fuel: int = 2, t_peak: float = 2200.0, p_atm: float = 1.0,
              seed: int = 0) -> Field:
    rng = np.random.default_rng(seed)
    z = np.arange(nz, dtype=np.float64)[:, None]
    r = np.arange(nr, dtype=np.float64)[None, :]
    Z = np.exp(-(r / (0.2 + 0.02 * z)) ** 2) + rng.normal(0.0, 0.02, size=(nz, nr))
    Z = np.clip(Z, 0.0, 1.0).reshape(-1)              # r fastest, like FSP(LJ,LI)
    T = 300.0 + (t_peak - 300.0) * np.exp(-((Z - 0.055) / 0.08) ** 2)
    y = _compose(Z, fuel, rng)
    p = np.full(Z.shape[0], p_atm * ATM)
    return Field(T, p, y, (nz, nr), seed, fuel)


def batch_cells(n: int, seed: int = 0, fuel: int = 11) -> Field:
    """Independent cells: heptane-generator compositions, T~U[300,2400] K, p~U[0.8,1.2] atm."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(np.sqrt(n)))
    z = rng.uniform(0.0, side, size=n)
    r = rng.uniform(0.0, 0.25 * side, size=n)
    Z = np.clip(np.exp(-(r / (0.2 + 0.02 * z)) ** 2) + rng.normal(0.0, 0.02, size=n), 0.0, 1.0)
    y = _compose(Z, fuel, rng)
    T = rng.uniform(300.0, 2400.0, size=n)
    p = rng.uniform(0.8, 1.2, size=n) * ATM
    return Field(T, p, y, (n,), seed, fuel)


def nondimensional(f: Field, scales: dict, wm: np.ndarray):
    """(tk, rho) in the reference's units: TK = T/TSTR and rho from the ideal
    gas at the cell pressure, RHO = (p/PSTR)/(BETA1*TK*sum Y/W)
    (src/unicornd-mild-sd-5.f:1056-1062 with a per-cell pressure)."""
    tk = f.T / scales["TSTR"]
    rbar = (f.y / wm[:, None]).sum(axis=0)
    rho = (f.p / scales["PSTR"]) / (scales["BETA1"] * tk * rbar)
    return tk, rho


def sensible_enthalpy(T: np.ndarray, y: np.ndarray, poly: np.ndarray, wm: np.ndarray, hfo: np.ndarray,
                      scales: dict) -> np.ndarray:
    """Non-dimensional sensible enthalpy HT consistent with the reference's
    T-from-h relation (src/lib/solveh.f:1170-1200): the total h of the NASA
    polynomials minus sum Y_k HFO_k, divided by HSTR."""
    hi = T > 1000.0
    out = np.empty_like(T)
    for sel, off in ((~hi, 0), (hi, 7)):
        if not sel.any():
            continue
        t = T[sel][None, :]
        a = poly[:, off:off + 7][:, :, None]
        hk = a[:, 0] * t + a[:, 1] * t ** 2 / 2 + a[:, 2] * t ** 3 / 3 + a[:, 3] * t ** 4 / 4 + a[:, 4] * t ** 5 / 5 + a[:, 5]
        out[sel] = (y[:, sel] / wm[:, None] * hk).sum(axis=0) * scales["GASC"] / scales["WMSTR"]
    return out / scales["HSTR"] - (y * hfo[:, None]).sum(axis=0)


def jet_flow(nz: int, nr: int, seed: int = 0, u_jet: float = 1.0, tmu: float = 1e-3) -> dict:
    """Geometry and flow of the (z, r) grid of ``jet_field`` (r fastest, LJ = nr rows, LI = nz columns),
    non-dimensional: spacing 1/(nr-1) in both directions (XXS, XXC, YYS, YYC), radius of the cell
    centres (j + 1/2)/(nr-1), axial velocity u = u_jet exp(-(r/(0.2+0.02 z))^2) + 0.05 (r, z in grid
    units, the spreading of the mixture fraction), radial velocity N(0, 0.01^2), eddy viscosity
    tmu (0.1 + u/u_jet)."""
    rng = np.random.default_rng(seed)
    d = 1.0 / (nr - 1)
    z = np.arange(nz, dtype=np.float64)[:, None]
    r = np.arange(nr, dtype=np.float64)[None, :]
    u = (u_jet * np.exp(-(r / (0.2 + 0.02 * z)) ** 2) + 0.05).reshape(-1)
    v = rng.normal(0.0, 0.01, size=nz * nr)
    return dict(lj=nr, li=nz, xxs=np.full(nz, d), xxc=np.full(nz, d), yys=np.full(nr, d), yyc=np.full(nr, d),
                yr=np.tile((np.arange(nr) + 0.5) * d, nz), u=u, v=v, tmu=tmu * (0.1 + u / u_jet))
