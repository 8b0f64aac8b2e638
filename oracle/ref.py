"""ctypes driver for the reference's own routines (``oracle/_ref``).

ORACLE INFRASTRUCTURE (test-only): imported by tests, the golden-fixture
script and the reference arm of ``bench.py``; never by the product.

The library is the reference Fortran translated to C by
``oracle/build_ref.py``. This driver plays the role of the reference's main
program: it fills the COMMON blocks the way ``src/unicornd-mild-sd-5.f``
does (reference scales from ``docs/input.uni:5``), runs the set-up block
(``src/unicornd-mild-sd-5.f:327-483``) and then calls the translated
routines on fields placed in the interior cells (J=2..LJ-1, I=2..LI-1) of
the compile-time grid, chunk by chunk.

Field convention (the reference's own, non-dimensional):
  tk[n]      = T / TSTR            rho[n] = rho / RSTR
  y[52, n]   mass fractions (species order of ``src/lib/DATA.f``)
  stmf[n], stnd[n]  soot mass fraction / number density (zero by default)
"""
from __future__ import annotations

import ctypes
import json
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / "_ref"
LSP, LRX = 52, 544

NP_T = {"real8": np.float64, "int": np.int32, "real4": np.float32, "logical": np.int32}
C_T = {"real8": ctypes.c_double, "int": ctypes.c_int, "real4": ctypes.c_float}

# reference-case inputs: docs/input.uni:4-5 (RTIN,RTOT; VREF,TREF,PREF,RREF,AK,EPS,FO2IN)
DEFAULT_INPUTS = dict(RTIN=0.0, RTOT=0.100, VREF=10.0, TREF=294.0, PREF=1.0133e5, RREF=1.225,
                      FO2IN=0.233)


def available() -> bool:
    return (REF_DIR / "libunicorn_ref.so").exists() and (REF_DIR / "layout.json").exists()


class RefUnicorn:
    def __init__(self, lib_dir: Path = REF_DIR, inputs: dict | None = None):
        self.lib = ctypes.CDLL(str(lib_dir / "libunicorn_ref.so"))
        self.lay = json.loads((lib_dir / "layout.json").read_text())
        self.LJ, self.LI = self.lay["LJ"], self.lay["LI"]
        self.LE = self.LJ * self.LI
        self.nj, self.ni = self.LJ - 2, self.LI - 2
        self.chunk = self.nj * self.ni
        self._blocks = {}
        inp = dict(DEFAULT_INPUTS)
        inp.update(inputs or {})
        self._setup(inp)

    # -------------------------------------------------------------- memory
    def _block(self, blk: str) -> np.ndarray:
        if blk not in self._blocks:
            size = ctypes.c_long.in_dll(self.lib, f"F77C_{blk}_size").value
            raw = (ctypes.c_ubyte * size).in_dll(self.lib, f"F77C_{blk}")
            self._blocks[blk] = np.ctypeslib.as_array(raw)
        return self._blocks[blk]

    def var(self, unit: str, name: str) -> np.ndarray:
        """numpy view (Fortran order) of a COMMON variable as ``unit`` declares it."""
        d = self.lay["units"][unit][name]
        b = self._block(d["block"])
        dt = NP_T[d["type"]]
        n = 1
        shape = []
        for lo, hi in (d["dims"] or []):
            n *= hi - lo + 1
            shape.append(hi - lo + 1)
        a = b[d["offset"]: d["offset"] + n * np.dtype(dt).itemsize].view(dt)
        return a.reshape(shape, order="F") if shape else a

    def scalar(self, unit: str, name: str, value=None):
        a = self.var(unit, name)
        if value is not None:
            a[0] = value
        return a[0]

    def mlocal(self, name: str, value=None):
        d = self.lay["main_locals"][name]
        if d["dims"]:
            n = int(np.prod([hi - lo + 1 for lo, hi in d["dims"]]))
            raw = (C_T[d["type"]] * n).in_dll(self.lib, f"MAIN_{name}")
            a = np.ctypeslib.as_array(raw)
            if value is not None:
                a[:] = value
            return a
        c = C_T[d["type"]].in_dll(self.lib, f"MAIN_{name}")
        if value is not None:
            c.value = value
        return c.value

    # -------------------------------------------------------------- set-up
    def _setup(self, inp: dict):
        self.lib.f77_blockdata()
        self.lib.f77_main_data()
        M = "UNICORN"
        for k in ("VREF", "TREF", "PREF", "RREF"):
            self.scalar(M, k, inp[k])
        for k in ("RTIN", "RTOT", "FO2IN"):
            self.mlocal(k, inp[k])
        self.mlocal("IRSW", 1)          # docs/input.uni:30 "10000*1": every reaction on
        self.mlocal("ISECS", 0)
        self.mlocal("IPROP", 1)
        self.mlocal("EAG", 1000.0)
        self.scalar(M, "IGRAV", 0)
        self.scalar(M, "ISYM", 1)
        self.scalar(M, "ICHEM", 1)
        self.scalar(M, "ITHRM", 1)
        self.scalar(M, "IFLOW", 1)
        self.lib.f77_main_setup()
        s = {}
        for k in ("ALSTR", "VSTR", "RSTR", "PSTR", "TSTR", "TMSTR", "AMSTR", "ACSTR", "DSTR",
                  "HSTR", "CPSTR", "AKSTR", "EPSTR", "WMSTR", "GASC", "BETA1", "BETA2",
                  "BETA3", "BETA4", "REI"):
            s[k] = float(self.scalar(M, k))
        s["PBACK"] = float(self.mlocal("PBACK"))
        self.scales = s
        self.wm = self.var(M, "WM").copy()
        self.hfo = self.var(M, "HFO").copy()

    def set_dt(self, dt: float):
        self.scalar("UNICORN", "DT", dt)

    # -------------------------------------------------------------- fields
    def _ij(self, n: int):
        c = np.arange(n)
        j = 1 + c % self.nj          # 0-based J index of interior cells
        i = 1 + c // self.nj
        return j, i

    def _load(self, tk, rho, y, stmf, stnd, iskip=None):
        n = len(tk)
        M = "UNICORN"
        TK = self.var(M, "TK").reshape(self.LJ, self.LI, order="F")
        RHO = self.var(M, "RHO").reshape(self.LJ, self.LI, order="F")
        FSP = self.var(M, "FSP").reshape(self.LJ, self.LI, LSP, order="F")
        STMF = self.var(M, "STMF").reshape(self.LJ, self.LI, order="F")
        STND = self.var(M, "STND").reshape(self.LJ, self.LI, order="F")
        ISKIP = self.var(M, "ISKIP")
        ISKIP[:] = 0
        # every cell (boundary ones too) gets a valid state: the first cell's
        TK[:] = tk[0]
        RHO[:] = rho[0]
        FSP[:] = y[:, 0]
        STMF[:] = stmf[0]
        STND[:] = stnd[0]
        j, i = self._ij(n)
        TK[j, i] = tk
        RHO[j, i] = rho
        FSP[j, i, :] = y.T
        STMF[j, i] = stmf
        STND[j, i] = stnd
        if iskip is not None:
            # ISKIP of /CB01/ (lib/skipdf.f); the arrays a skipped cell keeps start at zero, as the
            # COMMON blocks do in a fresh run
            ISKIP.reshape(self.LJ, self.LI, order="F")[j, i] = iskip
            for unit, nm in (("SOLVESP", "RC"), ("CKRATES", "SOUR"), ("SOLVEH", "QDSP"), ("SOLVEH", "QDOT")):
                self.var(unit, nm)[:] = 0.0
        return j, i

    def _chunks(self, n):
        for a in range(0, n, self.chunk):
            yield a, min(n, a + self.chunk)

    @staticmethod
    def _soot(n, stmf, stnd):
        return (np.zeros(n) if stmf is None else np.asarray(stmf, float),
                np.zeros(n) if stnd is None else np.asarray(stnd, float))

    def ckrates(self, tk, rho, y, stmf=None, stnd=None, iskip=None):
        """CKRATES (lib/ckrates.f:1-1363): returns RC[544,n] and SOUR[6,n]. With iskip, cells
        with ISKIP >= 3 keep the zero RC and SOUR of a fresh run (ckrates.f:94)."""
        n = len(tk)
        stmf, stnd = self._soot(n, stmf, stnd)
        rc = np.empty((LRX, n))
        sour = np.empty((6, n))
        for a, b in self._chunks(n):
            j, i = self._load(tk[a:b], rho[a:b], y[:, a:b], stmf[a:b], stnd[a:b],
                              None if iskip is None else iskip[a:b])
            self.lib.f77_ckrates()
            RC = self.var("SOLVESP", "RC")
            SOUR = self.var("CKRATES", "SOUR")
            rc[:, a:b] = RC[j, i, :].T
            sour[:, a:b] = SOUR[j, i, :].T
        return rc, sour

    def omega(self, tk, rho, y, stmf=None, stnd=None, iskip=None):
        """CKRATES then SOLVEH's rate part (lib/solveh.f:34-57,116-1145).

        Returns QDSP[52,n] (the reference's per-species rate, = -omega),
        QDOT[n] and HENTH[52,n] (species enthalpies)."""
        n = len(tk)
        stmf, stnd = self._soot(n, stmf, stnd)
        qdsp = np.empty((LSP, n))
        qdot = np.empty(n)
        henth = np.empty((LSP, n))
        for a, b in self._chunks(n):
            j, i = self._load(tk[a:b], rho[a:b], y[:, a:b], stmf[a:b], stnd[a:b],
                              None if iskip is None else iskip[a:b])
            self.lib.f77_ckrates()
            SSP = self.var("SOLVEH", "SSP").reshape(self.LJ, self.LI, LSP, order="F")
            FSP = self.var("UNICORN", "FSP").reshape(self.LJ, self.LI, LSP, order="F")
            SSP[:] = FSP
            self.lib.f77_solveh_omega()
            Q = self.var("SOLVEH", "QDSP")
            QD = self.var("SOLVEH", "QDOT")
            H = self.var("SOLVEH", "HENTH")
            qdsp[:, a:b] = Q[j, i, :].T
            qdot[a:b] = QD[j, i]
            henth[:, a:b] = H[j, i, :].T
        return qdsp, qdot, henth

    def cp(self, tk, y):
        """Mixture cp TCP of SPGSOLV (lib/spgsolv.f:102-173), non-dimensional."""
        n = len(tk)
        out = np.empty(n)
        tcp = np.ctypeslib.as_array((ctypes.c_double * self.LE).in_dll(self.lib, "F77P_TCP"))
        for a, b in self._chunks(n):
            j, i = self._load(tk[a:b], np.ones(b - a), y[:, a:b], np.zeros(b - a), np.zeros(b - a))
            self.lib.f77_spgsolv_cp()
            out[a:b] = tcp.reshape(self.LJ, self.LI, order="F")[j, i]
        return out

    def props(self, tk, y):
        """Y clip/N2 closure and mixture-averaged transport (main:821-1006).

        Returns (y_clipped[52,n], VMU[n], VTC[n], VDFSP[52,n]), non-dimensional."""
        n = len(tk)
        vmu = np.empty(n)
        vtc = np.empty(n)
        vdf = np.empty((LSP, n))
        yc = np.empty((LSP, n))
        M = "UNICORN"
        for a, b in self._chunks(n):
            j, i = self._load(tk[a:b], np.ones(b - a), y[:, a:b], np.zeros(b - a), np.zeros(b - a))
            self.lib.f77_main_props()
            VMU = self.var(M, "VMU").reshape(self.LJ, self.LI, order="F")
            VTC = self.var(M, "VTC").reshape(self.LJ, self.LI, order="F")
            VDF = self.var(M, "VDFSP").reshape(self.LJ, self.LI, LSP, order="F")
            FSP = self.var(M, "FSP").reshape(self.LJ, self.LI, LSP, order="F")
            vmu[a:b] = VMU[j, i]
            vtc[a:b] = VTC[j, i]
            vdf[:, a:b] = VDF[j, i, :].T
            yc[:, a:b] = FSP[j, i, :].T
        return yc, vmu, vtc, vdf

    def species_update(self, tk, rho, y0, dt, isor=100, relx=0.99, tol=1e-8, y_start=None,
                       stmf=None, stnd=None, spnorm=None, iskip=None):
        """CKRATES then SOLVESP (lib/solvesp.f) with zero face coefficients.

        One chunk only (the pass count is a property of the whole field).
        Returns (y_new[52,n], soot_mf[n], soot_nd[n], passes)."""
        n = len(tk)
        if n > self.chunk:
            raise ValueError(f"species_update handles at most {self.chunk} cells per call")
        stmf, stnd = self._soot(n, stmf, stnd)
        self.set_dt(dt)
        j, i = self._load(tk, rho, y0, stmf, stnd, iskip)
        self.lib.f77_ckrates()
        for blk in ("DUMMY", "DUM0", "DUMX"):
            self._block(blk)[:] = 0
        for nm in ("STE", "STW", "STN", "STS"):          # soot face coefficients (no transport here)
            self.var("SOLVESP", nm)[:] = 0.0
        SSP = self.var("SOLVEH", "SSP").reshape(self.LJ, self.LI, LSP, order="F")
        FSP = self.var("UNICORN", "FSP").reshape(self.LJ, self.LI, LSP, order="F")
        SSP[:] = FSP
        if y_start is not None:
            SSP[j, i, :] = y_start.T
        DUMS = "SOLVESP"
        self.var(DUMS, "SST1")[:] = self.var("UNICORN", "STMF").reshape(self.LJ, self.LI, order="F")
        self.var(DUMS, "SST2")[:] = self.var("UNICORN", "STND").reshape(self.LJ, self.LI, order="F")
        ii = ctypes.c_int(isor)
        r = ctypes.c_double(relx)
        t = ctypes.c_double(tol)
        sp = ctypes.c_double(float(self.LE * (LSP - 1)) if spnorm is None else spnorm)
        self.lib.f77_solvesp(ctypes.byref(ii), ctypes.byref(r), ctypes.byref(t), ctypes.byref(sp))
        ynew = SSP[j, i, :].T.copy()
        ynew[LSP - 1] = FSP[j, i, LSP - 1]
        sst1 = self.var(DUMS, "SST1")[j, i].copy()
        sst2 = self.var(DUMS, "SST2")[j, i].copy()
        return ynew, sst1, sst2, ii.value

    def temperature(self, tk_guess, y, ht, u=None, v=None, w=None):
        """T from h by Newton (lib/solveh.f:1170-1234); returns tk[n]."""
        n = len(tk_guess)
        out = np.empty(n)
        for a, b in self._chunks(n):
            j, i = self._load(tk_guess[a:b], np.ones(b - a), y[:, a:b], np.zeros(b - a), np.zeros(b - a))
            SSP = self.var("SOLVEH", "SSP").reshape(self.LJ, self.LI, LSP, order="F")
            FSP = self.var("UNICORN", "FSP").reshape(self.LJ, self.LI, LSP, order="F")
            SSP[:] = FSP
            FPZ = self.var("SOLVEH", "FPZ")
            FPZ[:] = ht[a]
            FPZ[j, i] = ht[a:b]
            for nm in ("U", "V", "W"):
                self.var("UNICORN", nm)[:] = 0.0
            self.lib.f77_solveh_temperature()
            out[a:b] = self.var("UNICORN", "TK").reshape(self.LJ, self.LI, order="F")[j, i]
        return out

    # -------------------------------------------------------------- SPGSOLV coefficients
    SPECIES_SUFFIX = [f"{a}{b}" for a in "ABC" for b in "0123456789ABCDEFGHIJ"][:LSP - 1]

    def spgsolv_coefficients(self, tk, rho, y, vtc, vdf, u, v, tmu, stdf, xxs, xxc, yys, yyc, yr,
                             isym=1, dt=1e-3, sigsp=0.7, sigh=0.7):
        """The E/W/N/S coefficients of the species equations (lib/spgsolv.f:98-1290) on the whole
        compile-time grid (fields [LJ*LI], J fastest; vdf, y [52][LJ*LI]; geometry XXS/XXC [LI],
        YYS/YYC [LJ], Y(J,I) radial coordinate [LJ*LI]). Returns e, w, n, s [51][LJ*LI] for the
        interior cells (boundary entries as the routine leaves them)."""
        LJ, LI = self.LJ, self.LI
        S = "SPGSOLV"
        sh = lambda a: np.asarray(a, dtype=np.float64).reshape(LJ, LI, order="F")
        self.var(S, "TK")[:] = sh(tk)
        self.var(S, "RHO")[:] = sh(rho)
        for k in range(LSP):
            nm = "F" + (self.SPECIES_SUFFIX[k] if k < LSP - 1 else "CB")
            self.var(S, nm)[:] = sh(y[k])
        self.var(S, "VTC")[:] = sh(vtc)
        VDF = self.var(S, "VDF")
        for k in range(LSP):
            VDF[:, :, k] = sh(vdf[k])
        for nm, a in (("U", u), ("V", v), ("TMU", tmu), ("STDF", stdf), ("Y", yr)):
            self.var(S, nm)[:] = sh(a)
        self.var(S, "XXS")[:] = xxs
        self.var(S, "XXC")[:] = xxc
        self.var(S, "YYS")[:] = yys
        self.var(S, "YYC")[:] = yyc
        self.var(S, "ISKIP")[:] = 0
        self.scalar(S, "ISYM", isym)
        self.scalar(S, "DT", dt)
        ctypes.c_double.in_dll(self.lib, "F77A_SPGSOLV_SIGSP").value = sigsp
        ctypes.c_double.in_dll(self.lib, "F77A_SPGSOLV_SIGH").value = sigh
        self.lib.f77_spgsolv_coef()
        out = []
        for face in "EWPQ":
            out.append(np.stack([self.var(S, face + self.SPECIES_SUFFIX[k]).reshape(-1, order="F")
                                 for k in range(LSP - 1)]))
        return tuple(o.copy() for o in out)

    # -------------------------------------------------------------- FDETAIL fields
    FD_NAMES = ["XRG", "YRG", "RHORG", "URG", "VRG", "TKRG", "QRG", "VMURG", "VTCRG", "CP"]

    def stdata_fields(self, x, y, rho, u, v, tk, qdot, vmu, vtc, fsp, vdf, qdsp):
        """lib/stdata.f:26-118 on the whole compile-time grid: returns [10 + 4*52, LJ*LI] in the
        order of the FDETAIL record (10 scalars, then Y, D, QDSP, h of every species)."""
        LJ, LI = self.LJ, self.LI
        S = "STDATA"
        sh = lambda a: np.asarray(a, dtype=np.float64).reshape(LJ, LI, order="F")
        for nm, a in (("X", x), ("Y", y), ("RHO", rho), ("U", u), ("V", v), ("TK", tk), ("QDOT", qdot),
                      ("VMU", vmu), ("VTC", vtc)):
            self.var(S, nm)[:] = sh(a)
        F, VD, Q = self.var(S, "FSP"), self.var(S, "VDF"), self.var(S, "QDSP")
        for k in range(LSP):
            F[:, :, k] = sh(fsp[k])
            VD[:, :, k] = sh(vdf[k])
            Q[:, :, k] = sh(qdsp[k])
        self.lib.f77_stdata_rg()
        rows = [self.var(S, nm).reshape(-1, order="F").copy() for nm in self.FD_NAMES]
        FR, VR, QR, EN = (self.var(S, nm) for nm in ("FSPRG", "VDFRG", "QSPRG", "ENTH"))
        for k in range(LSP):
            for A in (FR, VR, QR, EN):
                rows.append(A[:, :, k].reshape(-1, order="F").copy())
        return np.stack(rows)

    # -------------------------------------------------------------- SOLVEH enthalpy equation
    def enthalpy_rhs(self, tk, rho, y_start, y_new, ht, stmf, vtc, vdf, u, v, tmu, xxs, xxc, yys, yyc, yr,
                     isym=1, dt=1e-3, sigsp=0.9, sigh=0.9):
        """SPGSOLV's assembly (spgsolv.f:98-1290: EKT, EMU and the enthalpy coefficients ZE..ZS),
        CKRATES at the start state, then lib/solveh.f:34-1145 with SSP = y_new: returns
        (rhsz, (ze, zw, zn, zs), qdsp [52], qdot) on the whole compile-time grid."""
        n = self.LJ * self.LI
        self.spgsolv_coefficients(tk, rho, y_start, vtc, vdf, u, v, tmu, np.zeros(n), xxs, xxc, yys, yyc, yr,
                                  isym=isym, dt=dt, sigsp=sigsp, sigh=sigh)
        z = tuple(self.var("SPGSOLV", nm).reshape(-1, order="F").copy() for nm in ("ZE", "ZW", "ZN", "ZS"))
        self.lib.f77_ckrates()
        H = "SOLVEH"
        SSP = self.var(H, "SSP")
        SSP[:, :] = np.asarray(y_new, dtype=np.float64).T
        self.var(H, "HT")[:] = np.asarray(ht, dtype=np.float64).reshape(self.LJ, self.LI, order="F")
        self.var(H, "STMF")[:] = np.asarray(stmf, dtype=np.float64).reshape(self.LJ, self.LI, order="F")
        self.scalar(H, "RSOOT", 1.9e3)
        self.var(H, "ISKIP")[:] = 0
        ctypes.c_double.in_dll(self.lib, "F77A_SOLVEH_SIGSP").value = sigsp
        self.lib.f77_solveh_rhs()
        rhsz = self.var(H, "RHSZ").reshape(-1, order="F").copy()
        q = self.var(H, "QDSP")
        qdsp = np.stack([q[:, :, k].reshape(-1, order="F") for k in range(LSP)])
        qdot = self.var(H, "QDOT").reshape(-1, order="F").copy()
        return rhsz, z, qdsp, qdot

    def enthalpy_solve(self, tk, rho, y_start, y_new, ht, stmf, vtc, vdf, u, v, tmu, xxs, xxc, yys, yyc, yr,
                       w=None, isym=1, dt=1e-3, sigsp=0.9, sigh=0.9, isor=100, relx=0.99, tol=1e-8, hnorm=None):
        """SPGSOLV's assembly with FPZ = HT (spgsolv.f:98-1290), CKRATES at the start state, then the
        whole of SOLVEH (lib/solveh.f:34-1234) with SSP = y_new. Returns a dict with fpz, tk, passes
        (ISOR2 on return), rhsz, qdsp, qdot on the whole compile-time grid."""
        n = self.LJ * self.LI
        sh = lambda a: np.asarray(a, dtype=np.float64).reshape(self.LJ, self.LI, order="F")
        S = "SPGSOLV"
        self.var(S, "HT")[:] = sh(ht)
        self.var(S, "W")[:] = sh(np.zeros(n) if w is None else w)
        self.spgsolv_coefficients(tk, rho, y_start, vtc, vdf, u, v, tmu, np.zeros(n), xxs, xxc, yys, yyc, yr,
                                  isym=isym, dt=dt, sigsp=sigsp, sigh=sigh)
        self.lib.f77_ckrates()
        H = "SOLVEH"
        self.var(H, "SSP")[:, :] = np.asarray(y_new, dtype=np.float64).T
        self.var(H, "STMF")[:] = sh(stmf)
        self.scalar(H, "RSOOT", 1.9e3)
        self.var(H, "ISKIP")[:] = 0
        ctypes.c_double.in_dll(self.lib, "F77A_SOLVEH_SIGSP").value = sigsp
        ctypes.c_double.in_dll(self.lib, "F77A_SOLVEH_RELXH").value = relx
        ctypes.c_double.in_dll(self.lib, "F77A_SOLVEH_TOLRH").value = tol
        ctypes.c_double.in_dll(self.lib, "F77A_SOLVEH_HNORM").value = float(n) if hnorm is None else hnorm
        ctypes.c_int.in_dll(self.lib, "F77A_SOLVEH_ISOR2").value = isor
        self.lib.f77_solveh_full()
        flat = lambda nm: self.var(H, nm).reshape(-1, order="F").copy()
        q = self.var(H, "QDSP")
        return dict(fpz=flat("FPZ"), tk=flat("TK"), passes=ctypes.c_int.in_dll(self.lib, "F77A_SOLVEH_ISOR2").value,
                    rhsz=flat("RHSZ"), qdsp=np.stack([q[:, :, k].reshape(-1, order="F") for k in range(LSP)]),
                    qdot=flat("QDOT"))

    # -------------------------------------------------------------- density after SPGSOLV
    def density(self, tk, y):
        """main:1056-1068 on the whole compile-time grid: RHONP = PBACK/(BETA1 TK RBAR), the last
        column extrapolated linearly, the first row copied from the second. Returns RHONP [LJ*LI]."""
        M = "UNICORN"
        n = self.LJ * self.LI
        self.var(M, "TK")[:] = np.asarray(tk, dtype=np.float64)          # main's view: TK(LE), FSP(LE,LSP)
        self.var(M, "FSP")[:, :] = np.asarray(y, dtype=np.float64).T
        self.lib.f77_main_density()
        return self.var(M, "RHONP").reshape(-1, order="F").copy()
