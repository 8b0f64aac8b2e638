"""Python host interface to ``libunichem.so`` (the C ABI of include/unichem.h).

Mirrors the reference's hot-path routines by name and argument meaning:

=======================  =====================================================
``UniChem.ckrates``      CALL CKRATES (src/lib/ckrates.f) -> RC plane
``UniChem.omega``        rate part of CALL SOLVEH (src/lib/solveh.f:116-1145)
``UniChem.solvesp``      CALL SOLVESP(ISOR1,RELXSP,TOLRSP,SPNORM)
``UniChem.props``        property block of PROGRAM UNICORN (main:821-1006)
``UniChem.cp_h``         TCP of SPGSOLV (spgsolv.f:102-173) and HENTH sums
``UniChem.temperature``  T from h (src/lib/solveh.f:1170-1234)
=======================  =====================================================

Arrays are numpy float64, species-major ``[52, n]`` (the Fortran layout
``FSP(LJ,LI,LSP)`` flattened), non-dimensional as in the reference. There is
no CPU fallback: without the CUDA library or a GPU every call raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LSP, LRX = 52, 544
FP64, MIXED = 0, 1
import os

LIB_PATH = Path(os.environ.get("UNICHEM_LIB", str(Path(__file__).resolve().parent / "libunichem.so")))

UC_ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "call order", -4: "device timeout",
             -5: "no convergence", -6: "out of device memory"}


class UniChemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"unichem error {code} ({UC_ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Inputs(ctypes.Structure):
    """Input-card values (docs/input.uni:4-5 of the reference)."""
    _fields_ = [(k, ctypes.c_double) for k in ("rtin", "rtot", "vref", "tref", "pref", "rref", "fo2in")]


SCALE_FIELDS = ["alstr", "vstr", "rstr", "pstr", "tstr", "tmstr", "amstr", "acstr", "dstr", "hstr", "cpstr",
                "akstr", "epstr", "wmstr", "gasc", "beta1", "beta2", "beta3", "beta4", "rei", "pback", "hconv",
                "convrc", "convrm", "convrd"]


class Scales(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in SCALE_FIELDS]


DEFAULT_INPUTS = dict(rtin=0.0, rtot=0.100, vref=10.0, tref=294.0, pref=1.0133e5, rref=1.225, fo2in=0.233)

_lib = None


class Grid(ctypes.Structure):
    """uc_grid: the lj x li grid of the species-equation faces."""
    _fields_ = [("lj", ctypes.c_int), ("li", ctypes.c_int), ("isym", ctypes.c_int)] + \
               [(k, ctypes.POINTER(ctypes.c_double)) for k in ("xxs", "xxc", "yys", "yyc", "yr")]


class IntegrateOpts(ctypes.Structure):
    """uc_integrate_opts: batched stiff integration settings."""
    _fields_ = [("dt", ctypes.c_double), ("isor", ctypes.c_int), ("relx", ctypes.c_double), ("tol", ctypes.c_double),
                ("c_tau", ctypes.c_double), ("y_tau", ctypes.c_double), ("nsub_max", ctypes.c_int)]


class EnthalpyOpts(ctypes.Structure):
    """uc_enthalpy_opts: settings of the enthalpy equation (SOLVEH)."""
    _fields_ = [("dt", ctypes.c_double), ("isor", ctypes.c_int), ("relx", ctypes.c_double), ("tol", ctypes.c_double),
                ("hnorm", ctypes.c_double), ("sigh", ctypes.c_double)]


class HostIO(ctypes.Structure):
    """uc_host_io: the host buffers of one uc_sweep_host call (NULL = not copied)."""
    _fields_ = [(k, ctypes.POINTER(ctypes.c_double)) for k in
                ("tk", "rho", "fsp", "stmf", "stnd", "qdsp", "qdot", "domega_dy", "vmu", "vtc", "vdf", "cp", "h",
                 "fsp_out", "stmf_out", "stnd_out")]


def load_library(path: Path = LIB_PATH) -> ctypes.CDLL:
    """Load libunichem.so; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not Path(path).exists():
        raise UniChemError(-2, f"{path} not found: build it with `python -m unicorn_b200.build`")
    lib = ctypes.CDLL(str(path))
    P = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    lib.uc_init.argtypes = [ctypes.POINTER(Inputs), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    lib.uc_get_scales.argtypes = [vp, ctypes.POINTER(Scales), P, P]
    lib.uc_upload_fields.argtypes = [vp, P, P, P, P, P]
    lib.uc_download_fields.argtypes = [vp, P, P, P, P, P]
    lib.uc_upload_fields_device.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int]
    lib.uc_rates.argtypes = [vp, ctypes.c_int, P]
    lib.uc_omega.argtypes = [vp, ctypes.c_int, P, P, P]
    lib.uc_props.argtypes = [vp, P, P, P]
    lib.uc_cp_h.argtypes = [vp, P, P]
    lib.uc_species_update.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, P, P, ctypes.POINTER(ctypes.c_int)]
    lib.uc_temperature_from_h.argtypes = [vp, P]
    lib.uc_sweep.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, P, P, ctypes.POINTER(ctypes.c_int)]
    lib.uc_download_outputs.argtypes = [vp, P, P, P, P, P, P, P, P]
    lib.uc_sweep_host.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, P, P, ctypes.POINTER(HostIO), ctypes.POINTER(ctypes.c_int)]
    lib.uc_chem_props.argtypes = [vp, ctypes.c_int]
    lib.uc_set_iskip.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    lib.uc_profile.argtypes = [vp, ctypes.c_int]
    lib.uc_profile_read.argtypes = [vp, P, ctypes.POINTER(ctypes.c_int)]
    lib.uc_stat.argtypes = [vp, ctypes.c_char_p, P]
    lib.uc_sync.argtypes = [vp]
    lib.uc_last_error.argtypes = [vp]
    lib.uc_last_error.restype = ctypes.c_char_p
    lib.uc_destroy.argtypes = [vp]
    lib.uc_destroy.restype = None
    IP = ctypes.POINTER(ctypes.c_int)
    lib.uc_set_pressure.argtypes = [vp, P]
    lib.uc_set_grid.argtypes = [vp, ctypes.POINTER(Grid)]
    lib.uc_set_flow.argtypes = [vp, P, P, P, ctypes.c_double]
    lib.uc_assemble_faces.argtypes = [vp, ctypes.c_double, P, P, P, P]
    lib.uc_fdetail.argtypes = [vp, ctypes.c_int, ctypes.c_int, P, P, P, P, P]
    lib.uc_hold_enthalpy.argtypes = [vp]
    lib.uc_temperature_from_held.argtypes = [vp]
    lib.uc_integrate.argtypes = [vp, ctypes.c_int, ctypes.POINTER(IntegrateOpts)]
    lib.uc_integrate_tune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(IntegrateOpts)]
    lib.uc_integrate_counts.argtypes = [vp, IP, IP]
    lib.uc_set_enthalpy.argtypes = [vp, P, P]
    lib.uc_enthalpy_update.argtypes = [vp, ctypes.POINTER(EnthalpyOpts), IP, P]
    lib.uc_enthalpy_get.argtypes = [vp, P, P, P, P, P, P]
    lib.uc_density.argtypes = [vp]
    lib.uc_enthalpy_relax.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P, P, P, P, P, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, IP]
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _host(a, shape):
    """A host array used in place by a call (no copy): float64, C-contiguous, of the given shape."""
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != shape:
        raise ValueError(f"expected a C-contiguous float64 array of shape {shape}")
    return a


def _in(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


@dataclass
class Omega:
    qdsp: np.ndarray        # [52, n] the reference's QDSP (= -omega)
    qdot: np.ndarray        # [n]
    domega_dy: np.ndarray   # [52, n]

    @property
    def omega(self) -> np.ndarray:
        return -self.qdsp


class UniChem:
    """A device-resident field of n cells and the chemistry/property calls on it."""

    def __init__(self, n: int, inputs: dict | None = None, device: int = 0):
        self.lib = load_library()
        inp = dict(DEFAULT_INPUTS)
        inp.update(inputs or {})
        self.inputs = inp
        self.n = int(n)
        h = ctypes.c_void_p()
        rc = self.lib.uc_init(ctypes.byref(Inputs(**inp)), self.n, device, ctypes.byref(h))
        if rc != 0:
            raise UniChemError(rc, "uc_init failed (see stderr)")
        self._h = h
        sc = Scales()
        self.wm = np.zeros(LSP)
        self.hfo = np.zeros(LSP)
        self._ck(self.lib.uc_get_scales(h, ctypes.byref(sc), _p(self.wm), _p(self.hfo)))
        self.scales = {k.upper(): getattr(sc, k) for k in SCALE_FIELDS}

    # ------------------------------------------------------------ plumbing
    def _ck(self, rc: int):
        # UC_E_NOCONV (-5): a T Newton ran out of steps in some cell, recorded by an asynchronous
        # kernel and reported at the next synchronising call, whose own work has completed; the
        # reference prints a message and carries on, so it is a warning here
        if rc == -5:
            import warnings
            warnings.warn(self.lib.uc_last_error(self._h).decode())
        elif rc != 0:
            raise UniChemError(rc, self.lib.uc_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self.lib.uc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ state
    def upload(self, tk, rho, y, stmf=None, stnd=None):
        n = self.n
        tk, rho, y = _in(tk, (n,)), _in(rho, (n,)), _in(y, (LSP, n))
        stmf, stnd = _in(stmf, (n,)), _in(stnd, (n,))
        self._ck(self.lib.uc_upload_fields(self._h, _p(tk), _p(rho), _p(y), _p(stmf), _p(stnd)))

    def upload_device(self, tk, rho, y, stmf=None, stnd=None, ld=None):
        """State from device memory: integer device addresses (e.g. torch's data_ptr()) of
        tk, rho [ld], y [52][ld], stmf, stnd [ld] (or None); asynchronous on the context's stream."""
        self._ck(self.lib.uc_upload_fields_device(self._h, tk, rho, y, stmf, stnd, int(ld if ld is not None else self.n)))

    def set_iskip(self, iskip=None):
        """The reference's ISKIP per cell (int [n]); None clears it."""
        if iskip is None:
            self._ck(self.lib.uc_set_iskip(self._h, None))
            return
        a = np.ascontiguousarray(iskip, dtype=np.int32)
        if a.shape != (self.n,):
            raise ValueError(f"expected shape ({self.n},), got {a.shape}")
        self._ck(self.lib.uc_set_iskip(self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    def download(self):
        n = self.n
        tk, rho, y, s1, s2 = np.empty(n), np.empty(n), np.empty((LSP, n)), np.empty(n), np.empty(n)
        self._ck(self.lib.uc_download_fields(self._h, _p(tk), _p(rho), _p(y), _p(s1), _p(s2)))
        return tk, rho, y, s1, s2

    def sync(self):
        """Wait for the context's stream; a T Newton that ran out of steps is a warning
        (the reference prints one and carries on), every other error raises."""
        self._ck_warn(self.lib.uc_sync(self._h))

    def _ck_warn(self, rc: int):
        if rc == -5:
            import warnings
            warnings.warn(self.lib.uc_last_error(self._h).decode())
        else:
            self._ck(rc)

    # ------------------------------------------------------------ hot path
    def ckrates(self, precision: int = FP64, return_rc: bool = False):
        rc = np.empty((LRX, self.n)) if return_rc else None
        self._ck(self.lib.uc_rates(self._h, precision, _p(rc)))
        return rc

    def omega(self, precision: int = FP64, download: bool = True):
        if not download:
            self._ck(self.lib.uc_omega(self._h, precision, None, None, None))
            return None
        q, qd, d = np.empty((LSP, self.n)), np.empty(self.n), np.empty((LSP, self.n))
        self._ck(self.lib.uc_omega(self._h, precision, _p(q), _p(qd), _p(d)))
        return Omega(q, qd, d)

    def props(self, download: bool = True):
        if not download:
            self._ck(self.lib.uc_props(self._h, None, None, None))
            return None
        mu, lam, d = np.empty(self.n), np.empty(self.n), np.empty((LSP, self.n))
        self._ck(self.lib.uc_props(self._h, _p(mu), _p(lam), _p(d)))
        return mu, lam, d

    def cp_h(self, download: bool = True):
        if not download:
            self._ck(self.lib.uc_cp_h(self._h, None, None))
            return None
        cp, h = np.empty(self.n), np.empty(self.n)
        self._ck(self.lib.uc_cp_h(self._h, _p(cp), _p(h)))
        return cp, h

    def solvesp(self, dt: float, isor: int = 100, relx: float = 0.99, tol: float = 1e-8, spnorm: float = 0.0,
                face_sum=None, face_nbr=None) -> int:
        fs = _in(face_sum, (LSP - 1, self.n))
        fn = _in(face_nbr, (LSP - 1, self.n))
        passes = ctypes.c_int(0)
        self._ck_warn(self.lib.uc_species_update(self._h, dt, int(isor), relx, tol, spnorm, _p(fs), _p(fn),
                                                 ctypes.byref(passes)))
        return passes.value

    def sweep(self, dt: float, precision: int = FP64, isor: int = 100, relx: float = 0.99, tol: float = 1e-8,
              spnorm: float = 0.0, face_sum=None, face_nbr=None) -> int:
        """One species sweep: props, cp/h, rates + omega, point-implicit update. A T Newton of an
        earlier asynchronous call that ran out of steps (reported when this call synchronises) is a
        warning, as the reference prints one and carries on; the sweep itself has completed."""
        fs = _in(face_sum, (LSP - 1, self.n))
        fn = _in(face_nbr, (LSP - 1, self.n))
        passes = ctypes.c_int(0)
        self._ck_warn(self.lib.uc_sweep(self._h, precision, dt, int(isor), relx, tol, spnorm, _p(fs), _p(fn),
                                        ctypes.byref(passes)))
        return passes.value

    def sweep_host(self, tk, rho, y, out: dict | None = None, y_out=None, soot=None, soot_out=None, dt: float = 1e-5,
                   precision: int = FP64, isor: int = 100, relx: float = 0.99, tol: float = 1e-8, spnorm: float = 0.0,
                   face_sum=None, face_nbr=None) -> int:
        """uc_sweep_host: upload (tk, rho, y[, soot = (stmf, stnd)]), one sweep, and the outputs (keys of
        download_outputs) and the updated Y (and soot) into the given host arrays; the output copies
        overlap the species update. The arrays are used in place (pinned ones make the copies
        asynchronous): float64, C-contiguous, of the shapes of upload/download_outputs."""
        n = self.n
        chk = lambda a, shape: None if a is None else _host(a, shape)
        io = HostIO()
        io.tk, io.rho, io.fsp = _p(chk(tk, (n,))), _p(chk(rho, (n,))), _p(chk(y, (LSP, n)))
        if soot is not None:
            io.stmf, io.stnd = _p(chk(soot[0], (n,))), _p(chk(soot[1], (n,)))
        out = out or {}
        shapes = dict(qdsp=(LSP, n), qdot=(n,), domega_dy=(LSP, n), vmu=(n,), vtc=(n,), vdf=(LSP, n), cp=(n,), h=(n,))
        for k, shape in shapes.items():
            setattr(io, k, _p(chk(out.get(k), shape)))
        io.fsp_out = _p(chk(y_out, (LSP, n)))
        if soot_out is not None:
            io.stmf_out, io.stnd_out = _p(chk(soot_out[0], (n,))), _p(chk(soot_out[1], (n,)))
        fs = _in(face_sum, (LSP - 1, n))
        fn = _in(face_nbr, (LSP - 1, n))
        passes = ctypes.c_int(0)
        self._ck(self.lib.uc_sweep_host(self._h, precision, dt, int(isor), relx, tol, spnorm, _p(fs), _p(fn),
                                        ctypes.byref(io), ctypes.byref(passes)))
        return passes.value

    def chem_props(self, precision: int = FP64):
        """Y clip + transport, cp/h, omega and d(omega)/dY of the device state (no update); asynchronous."""
        self._ck(self.lib.uc_chem_props(self._h, precision))

    def download_outputs(self, out: dict | None = None) -> dict:
        """Copy omega, d(omega)/dY, QDOT, transport, cp and h of the last sweep to host arrays."""
        n = self.n
        if out is None:
            out = dict(qdsp=np.empty((LSP, n)), qdot=np.empty(n), domega_dy=np.empty((LSP, n)), vmu=np.empty(n),
                       vtc=np.empty(n), vdf=np.empty((LSP, n)), cp=np.empty(n), h=np.empty(n))
        self._ck(self.lib.uc_download_outputs(self._h, *[_p(out.get(k)) for k in
                                                         ("qdsp", "qdot", "domega_dy", "vmu", "vtc", "vdf", "cp", "h")]))
        return out

    def stat(self, name: str) -> float:
        v = np.zeros(1)
        self._ck(self.lib.uc_stat(self._h, name.encode(), _p(v)))
        return float(v[0])

    def profile(self, on: bool = True):
        self._ck(self.lib.uc_profile(self._h, int(on)))

    def profile_read(self) -> dict:
        """Device time (ms) and launches per kernel kind since the last read."""
        ms = np.zeros(7)
        cnt = (ctypes.c_int * 7)()
        self._ck(self.lib.uc_profile_read(self._h, _p(ms), cnt))
        names = ["chem", "update", "props", "cp_h", "temperature", "integrate", "enthalpy"]
        return {nm: (float(ms[i]), int(cnt[i])) for i, nm in enumerate(names)}

    # ------------------------------------------------------------ species-equation faces
    def set_grid(self, lj: int, li: int, xxs, xxc, yys, yyc, yr, isym: int = 1):
        """Grid of the face assembly (SPGSOLV geometry); the context's cells are the lj x li grid."""
        arrs = [_in(a) for a in (xxs, xxc, yys, yyc, yr)]
        self._grid_keep = arrs
        g = Grid(int(lj), int(li), int(isym), *[_p(a) for a in arrs])
        self._ck(self.lib.uc_set_grid(self._h, ctypes.byref(g)))

    def clear_grid(self):
        self._ck(self.lib.uc_set_grid(self._h, None))

    def set_flow(self, u, v, tmu, sigsp: float = 0.7):
        n = self.n
        self._ck(self.lib.uc_set_flow(self._h, _p(_in(u, (n,))), _p(_in(v, (n,))), _p(_in(tmu, (n,))), sigsp))

    def assemble_faces(self, dt: float):
        """E, W, N, S [51, n] of the current state (uc_props must have run)."""
        out = [np.empty((LSP - 1, self.n)) for _ in range(4)]
        self._ck(self.lib.uc_assemble_faces(self._h, dt, *[_p(o) for o in out]))
        return tuple(out)

    def fdetail(self, lj: int, li: int, x, y, u, v) -> np.ndarray:
        """FDETAIL fields [218, n] of the current state (uc_fdetail)."""
        n = self.n
        out = np.empty((218, n))
        self._ck(self.lib.uc_fdetail(self._h, int(lj), int(li), _p(_in(x, (n,))), _p(_in(y, (n,))),
                                     _p(_in(u, (n,))), _p(_in(v, (n,))), _p(out)))
        return out

    # ------------------------------------------------------------ enthalpy equation
    def set_enthalpy(self, ht, w=None):
        """HT [n] (non-dimensional FPZ) and the swirl velocity W [n] (None: no swirl)."""
        n = self.n
        self._ck(self.lib.uc_set_enthalpy(self._h, _p(_in(ht, (n,))), _p(_in(w, (n,)))))

    def enthalpy_update(self, dt: float, isor: int = 100, relx: float = 0.99, tol: float = 1e-8,
                        hnorm: float = 0.0, sigh: float = 0.9):
        """SOLVEH after a uc_sweep: returns (passes as ISOR2 reports it, RESDH). T and HT are updated
        on the device; QDSP/QDOT of the interior cells become SOLVEH's."""
        o = EnthalpyOpts(float(dt), int(isor), float(relx), float(tol), float(hnorm), float(sigh))
        passes = ctypes.c_int(0)
        resdh = np.zeros(1)
        self._ck_warn(self.lib.uc_enthalpy_update(self._h, ctypes.byref(o), ctypes.byref(passes), _p(resdh)))
        return passes.value, float(resdh[0])

    def density(self):
        """RHO of every cell from the gas law at PBACK with the grid's edge rules (main:1056-1073)."""
        self._ck(self.lib.uc_density(self._h))

    def enthalpy_get(self):
        """(HT, RHSZ, ZE, ZW, ZN, ZS) [n] each, after an enthalpy update."""
        out = [np.empty(self.n) for _ in range(6)]
        self._ck(self.lib.uc_enthalpy_get(self._h, *[_p(o) for o in out]))
        return tuple(out)

    # ------------------------------------------------------------ restart files
    def save_restart(self, path, lj: int, li: int, flow: dict, **header):
        """Write the device state (RHO, FSP, TK, QDOT, STMF, STND) with the host's grid and flow
        fields (flow: X, Y, U, V, W, P and, with iflow=2, AK, EPS) as a restart file."""
        from .restart import write_restart
        tk, rho, y, s1, s2 = self.download()
        qd = np.zeros(self.n)
        if self.lib.uc_download_outputs(self._h, None, _p(qd), None, None, None, None, None, None) != 0:
            qd[:] = 0.0                      # no omega computed yet: QDOT is written as zero
        f = dict(flow, RHO=rho, FSP=y, TK=tk, QDOT=qd, STMF=s1, STND=s2)
        write_restart(path, f, self.scales, lj, li, **header)

    def load_restart(self, path) -> tuple[dict, dict]:
        """Read a restart file, upload its state (TK, RHO, FSP, STMF, STND); returns (header, fields)."""
        from .restart import read_restart
        h, f = read_restart(path)
        if h["LI"] * h["LJ"] != self.n:
            raise ValueError(f"restart grid {h['LJ']}x{h['LI']} does not match {self.n} cells")
        self.upload(f["TK"], f["RHO"], f["FSP"], f["STMF"], f["STND"])
        return h, f

    # ------------------------------------------------------------ batched integration
    @staticmethod
    def integrate_opts(dt: float, isor: int = 100, relx: float = 0.99, tol: float = 1e-8, c_tau: float = 1.0,
                       y_tau: float = 1e-3, nsub_max: int = 200) -> IntegrateOpts:
        return IntegrateOpts(dt, int(isor), relx, tol, c_tau, y_tau, int(nsub_max))

    def set_pressure(self, pnd):
        """Cell pressures p/PSTR (the reference's non-dimensional pressure)."""
        self._ck(self.lib.uc_set_pressure(self._h, _p(_in(pnd, (self.n,)))))

    def hold_enthalpy(self):
        """Record each cell's total enthalpy (the in-loop T update keeps it)."""
        self._ck(self.lib.uc_hold_enthalpy(self._h))

    def temperature_from_held(self):
        """T from the held enthalpy for the current Y, then rho at the cell pressure."""
        self._ck(self.lib.uc_temperature_from_held(self._h))

    def integrate(self, dt: float, precision: int = FP64, **kw):
        """Advance every cell over dt (uc_integrate); the state stays on the device."""
        o = self.integrate_opts(dt, **kw)
        self._ck(self.lib.uc_integrate(self._h, precision, ctypes.byref(o)))

    def integrate_tune(self, dt: float, precision: int = FP64, **kw) -> dict:
        o = self.integrate_opts(dt, **kw)
        self._ck(self.lib.uc_integrate_tune(self._h, precision, ctypes.byref(o)))
        return {k: self.stat(k) for k in ("int_warps", "int_sorted", "int_tune_best_ms", "int_tune_worst_ms")}

    def integrate_counts(self):
        """(n_sub[n], update passes[n]) of the last integration."""
        ns = np.empty(self.n, dtype=np.int32)
        pa = np.empty(self.n, dtype=np.int32)
        IP = ctypes.POINTER(ctypes.c_int)
        # a T-from-h Newton that ran out of steps in some cell is a warning: the
        # reference prints one and carries on with the clamped value, and so does the integration
        self._ck_warn(self.lib.uc_integrate_counts(self._h, ns.ctypes.data_as(IP), pa.ctypes.data_as(IP)))
        return ns, pa

    def temperature(self, ht):
        """T from h; a cell whose Newton iteration ran out of steps is reported
        as a warning, as the reference prints one and carries on."""
        import warnings
        ht = _in(ht, (self.n,))
        rc = self.lib.uc_temperature_from_h(self._h, _p(ht))
        if rc == -5:
            warnings.warn(self.lib.uc_last_error(self._h).decode())
        else:
            self._ck(rc)


def enthalpy_relax(lj: int, li: int, rho, rhsz, z, ht, isor: int = 100, relx: float = 0.99, tol: float = 1e-8,
                   hnorm: float = 0.0, device: int = 0):
    """The relaxation of solveh.f:1146-1167 alone on the device: z = (ze, zw, zn, zs); returns (FPZ, passes)."""
    lib = load_library()
    n = lj * li
    fpz = np.array(ht, dtype=np.float64, copy=True).reshape(n)
    passes = ctypes.c_int(0)
    arrs = [_in(a, (n,)) for a in (rho, rhsz, *z)]
    rc = lib.uc_enthalpy_relax(int(device), int(lj), int(li), *[_p(a) for a in arrs], _p(fpz), int(isor),
                               float(relx), float(tol), float(hnorm), ctypes.byref(passes))
    if rc != 0:
        raise RuntimeError(f"uc_enthalpy_relax failed ({rc})")
    return fpz, passes.value
