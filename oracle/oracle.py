"""ctypes wrapper of the FP64 CPU restatement ``oracle/unichem_oracle.c``.

ORACLE INFRASTRUCTURE (test-only): imported by tests/, the golden-fixture
script, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg as the
checker; the product never imports it.

The mechanism tables come from ``unicorn_b200/mech/sandiego52.json`` (read as
data) and are packed here into the flat arrays the C code walks.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
MECH = HERE.parent / "unicorn_b200" / "mech" / "sandiego52.json"
LSP, LRX = 52, 544

FK = {"num": 0, "A": 1, "RC": 2, "Y": 3, "Y0": 4, "SOUR": 5, "RA": 6, "SRA": 7}
SCALE_NAMES = ["ALSTR", "VSTR", "RSTR", "PSTR", "TSTR", "TMSTR", "AMSTR", "ACSTR", "DSTR", "HSTR",
               "CPSTR", "AKSTR", "EPSTR", "WMSTR", "GASC", "BETA1", "BETA2", "BETA3", "BETA4", "REI",
               "PBACK", "HCONV", "CONVRC", "CONVRM", "CONVRD"]
DEFAULT_INPUTS = dict(RTIN=0.0, RTOT=0.100, VREF=10.0, TREF=294.0, PREF=1.0133e5, RREF=1.225,
                      FO2IN=0.233)

_TABLE_FIELDS = [
    "wsp", "cdia", "tlj", "poly", "om22", "ci11", "tpol1", "tpol2",
    "akf", "alf", "exaf", "aklow", "allow", "ealow", "troe",
    "rev_has", "rev_rut", "rev_off", "rev_len", "rev_op", "rev_sp",
    "tb_off", "tb_len", "tb_sign", "tb_sp", "tb_coef", "tb_hascoef",
    "dmole_grp",
    "rc_has", "rc_order", "rc_tb", "rc_off", "rc_len", "rc_op", "rc_kind", "rc_idx",
    "ra_has", "ra_off", "ra_len", "ra_sp",
    "prd_has", "prd_off", "prd_len",
    "term_sign", "term_foff", "term_flen",
    "fac_kind", "fac_idx", "fac_val",
    "blk_rec_off", "blk_rec_len", "rec_r", "rec_foff", "rec_flen",
    "blk_prod_has", "blk_prod_off", "blk_prod_len",
    "blk_extra_off", "blk_extra_len",
    "blk_loss_has", "blk_loss_off", "blk_loss_len",
    "blk_mul_off", "blk_mul_len", "mul_r",
]
_DOUBLE_FIELDS = {"wsp", "cdia", "tlj", "poly", "om22", "ci11", "akf", "alf", "exaf", "aklow",
                  "allow", "ealow", "troe", "tb_coef", "fac_val"}


_f = []
for name in _TABLE_FIELDS:
    if name in ("tpol1", "tpol2"):
        _f.append((name, ctypes.c_double))
    elif name in _DOUBLE_FIELDS:
        _f.append((name, ctypes.POINTER(ctypes.c_double)))
    else:
        _f.append((name, ctypes.POINTER(ctypes.c_int)))


class _Tables(ctypes.Structure):
    _fields_ = _f     # same order as orc_tables in unichem_oracle.c


class _Inputs(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("RTIN", "RTOT", "VREF", "TREF", "PREF", "RREF", "FO2IN")]


def build_lib() -> Path:
    LIB.parent.mkdir(parents=True, exist_ok=True)
    src = HERE / "unichem_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
                        "-fopenmp", "-o", str(LIB), str(src), "-lm"], check=True)
    return LIB


class _Pack:
    """Flat term/factor store shared by all product chains."""

    def __init__(self):
        self.term_sign, self.term_foff, self.term_flen = [], [], []
        self.fac_kind, self.fac_idx, self.fac_val = [], [], []

    def chain(self, factors) -> tuple[int, int]:
        off = len(self.fac_kind)
        for f in factors:
            kind = f[0]
            self.fac_kind.append(FK[kind])
            if kind == "num":
                self.fac_idx.append(0)
                self.fac_val.append(float(f[1]))
            elif kind == "A":
                self.fac_idx.append(int(f[1]))       # A-terms keep their 1-based number
                self.fac_val.append(0.0)
            else:
                self.fac_idx.append(int(f[1]) - 1)
                self.fac_val.append(0.0)
        return off, len(factors)

    def terms(self, terms) -> tuple[int, int]:
        off = len(self.term_sign)
        for s, factors in terms:
            fo, fl = self.chain(factors)
            self.term_sign.append(int(s))
            self.term_foff.append(fo)
            self.term_flen.append(fl)
        return off, len(terms)


def pack_tables(mech: dict) -> dict:
    t: dict[str, object] = {}
    t["wsp"] = mech["wsp"]
    t["cdia"] = mech["cdia"]
    t["tlj"] = mech["tlj"]
    t["poly"] = [v for row in mech["poly"] for v in row]
    t["om22"] = [v for row in mech["omega22"] for v in row]
    t["ci11"] = [v for row in mech["ci11"] for v in row]
    t["tpol1"], t["tpol2"] = mech["tpol"]
    R = mech["reactions"]
    for k in ("akf", "alf", "exaf", "aklow", "allow", "ealow"):
        t[k] = [x[k] for x in R]
    t["troe"] = [v for x in R for v in x["troe"]]
    # reverse formulas
    has, rut, off, ln, op, sp = [0] * LRX, [0] * LRX, [0] * LRX, [0] * LRX, [], []
    for key, rv in mech["reverse"].items():
        r = int(key) - 1
        has[r], rut[r], off[r], ln[r] = 1, rv["rut"], len(sp), len(rv["q"])
        for o, s in rv["q"]:
            op.append(ord(o))
            sp.append(s - 1)
    t.update(rev_has=has, rev_rut=rut, rev_off=off, rev_len=ln, rev_op=op, rev_sp=sp)
    # third bodies: group 0 = TBODY (its 52 terms must be species 1..52 in order)
    tbody = mech["tb"]["TBODY"]
    assert [x[1] for x in tbody] == list(range(1, LSP + 1))
    toff, tlen, tsign, tsp, tcoef, thas = [0] * 11, [0] * 11, [], [], [], []
    for g in range(1, 11):
        terms = mech["tb"][f"TB{g:03d}"]
        assert terms[0] == [1, "TBODY"]
        toff[g], tlen[g] = len(tsp), len(terms) - 1
        for s, k, c in terms[1:]:
            tsign.append(s)
            tsp.append(k - 1)
            tcoef.append(0.0 if c is None else c)
            thas.append(0 if c is None else 1)
    t.update(tb_off=toff, tb_len=tlen, tb_sign=tsign, tb_sp=tsp, tb_coef=tcoef, tb_hascoef=thas)
    dm = [0] * LRX
    for key, g in mech["dmole"].items():
        dm[int(key) - 1] = int(g[2:])
    t["dmole_grp"] = dm
    # RC assembly
    rh, ro, rt, roff, rl, rop, rk, ri = [0] * LRX, [0] * LRX, [-1] * LRX, [0] * LRX, [0] * LRX, [], [], []
    for key, rc in mech["rc"].items():
        r = int(key) - 1
        rh[r], ro[r] = 1, rc["order"]
        rt[r] = -1 if rc["tb"] is None else (0 if rc["tb"] == "TBODY" else int(rc["tb"][2:]))
        roff[r], rl[r] = len(rop), len(rc["post"])
        for o, kind, idx in rc["post"]:
            rop.append(ord(o))
            rk.append(FK["Y"] if kind == "Y" else 99)
            ri.append(idx - 1)
    t.update(rc_has=rh, rc_order=ro, rc_tb=rt, rc_off=roff, rc_len=rl, rc_op=rop, rc_kind=rk, rc_idx=ri)
    # RA reactants
    ah, aoff, al, asp = [0] * LRX, [0] * LRX, [0] * LRX, []
    for key, sps in mech["ra"].items():
        r = int(key) - 1
        if sps is None:
            continue
        ah[r], aoff[r], al[r] = 1, len(asp), len(sps)
        asp.extend(s - 1 for s in sps)
    t.update(ra_has=ah, ra_off=aoff, ra_len=al, ra_sp=asp)
    P = _Pack()
    ph, po, pl = [0] * LSP, [0] * LSP, [0] * LSP
    for key, terms in mech["prd"].items():
        k = int(key) - 1
        if not terms:
            continue
        ph[k] = 1
        po[k], pl[k] = P.terms(terms)
    t.update(prd_has=ph, prd_off=po, prd_len=pl)
    # update blocks
    B = mech["update"]["blocks"]
    ro_, rl_, rr, rfo, rfl = [], [], [], [], []
    pho, poo, plo, eo, el, lh, lo, ll, mo, ml, mr = [], [], [], [], [], [], [], [], [], [], []
    for b in B:
        ro_.append(len(rr))
        rl_.append(len(b["recompute"]))
        for r, fac in b["recompute"]:
            fo, fl = P.chain(fac)
            rr.append(r)
            rfo.append(fo)
            rfl.append(fl)
        if b["prod"] is None:
            pho.append(0); poo.append(0); plo.append(0)
        else:
            o, n = P.terms(b["prod"])
            pho.append(1); poo.append(o); plo.append(n)
        o, n = P.terms(b["extra"])
        eo.append(o); el.append(n)
        if b["loss"] is None:
            lh.append(0); lo.append(0); ll.append(0)
        else:
            o, n = P.terms(b["loss"])
            lh.append(1); lo.append(o); ll.append(n)
        mo.append(len(mr))
        ml.append(len(b["multiply"]))
        mr.extend(b["multiply"])
    t.update(blk_rec_off=ro_, blk_rec_len=rl_, rec_r=rr, rec_foff=rfo, rec_flen=rfl,
             blk_prod_has=pho, blk_prod_off=poo, blk_prod_len=plo,
             blk_extra_off=eo, blk_extra_len=el,
             blk_loss_has=lh, blk_loss_off=lo, blk_loss_len=ll,
             blk_mul_off=mo, blk_mul_len=ml, mul_r=mr)
    t.update(term_sign=P.term_sign, term_foff=P.term_foff, term_flen=P.term_flen,
             fac_kind=P.fac_kind, fac_idx=P.fac_idx, fac_val=P.fac_val)
    return t


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


class Oracle:
    """FP64 CPU restatement; all field arrays are SoA: y[52, n]."""

    def __init__(self, inputs: dict | None = None, mech_path: Path = MECH):
        self.lib = ctypes.CDLL(str(build_lib()))
        self.mech = json.loads(Path(mech_path).read_text())
        packed = pack_tables(self.mech)
        self._keep = {}
        tab = _Tables()
        for name in _TABLE_FIELDS:
            v = packed[name]
            if name in ("tpol1", "tpol2"):
                setattr(tab, name, float(v))
                continue
            if name in _DOUBLE_FIELDS:
                a = np.ascontiguousarray(v if len(v) else [0.0], dtype=np.float64)
                setattr(tab, name, _dptr(a))
            else:
                a = np.ascontiguousarray(v if len(v) else [0], dtype=np.int32)
                setattr(tab, name, _iptr(a))
            self._keep[name] = a
        self._tab = tab
        inp = dict(DEFAULT_INPUTS)
        inp.update(inputs or {})
        self.inputs = inp
        ci = _Inputs(**inp)
        sc = np.zeros(len(SCALE_NAMES))
        self.lib.orc_setup(ctypes.byref(tab), ctypes.byref(ci), _dptr(sc))
        self.scales = dict(zip(SCALE_NAMES, sc.tolist()))
        self.wm = np.zeros(LSP)
        self.hfo = np.zeros(LSP)
        akf, exaf, ealow = np.zeros(LRX), np.zeros(LRX), np.zeros(LRX)
        self.pair = np.zeros((7, LSP, LSP))
        self.lib.orc_get_tables(_dptr(self.wm), _dptr(self.hfo), _dptr(akf), _dptr(exaf),
                                _dptr(ealow), _dptr(self.pair))
        self.akf, self.exaf, self.ealow = akf, exaf, ealow
        self.lib.orc_species_update.restype = ctypes.c_int

    # ---------------------------------------------------------------- API
    def rates(self, tk, rho, y, stmf=None, stnd=None):
        n = len(tk)
        rc = np.empty((LRX, n))
        sour = np.empty((6, n))
        tk, rho, y = _c(tk), _c(rho), _c(y)
        sm = _c(np.zeros(n) if stmf is None else stmf)
        sn = _c(np.zeros(n) if stnd is None else stnd)
        self.lib.orc_rates(n, _dptr(tk), _dptr(rho), _dptr(y), _dptr(sm), _dptr(sn), _dptr(rc), _dptr(sour))
        return rc, sour

    def omega(self, tk, rho, y, stmf=None, stnd=None):
        """Returns (qdsp[52,n], qdot[n], henth[52,n], domega_dy[52,n])."""
        n = len(tk)
        q, qd, h, d = np.empty((LSP, n)), np.empty(n), np.empty((LSP, n)), np.empty((LSP, n))
        tk, rho, y = _c(tk), _c(rho), _c(y)
        sm = _c(np.zeros(n) if stmf is None else stmf)
        sn = _c(np.zeros(n) if stnd is None else stnd)
        self.lib.orc_omega(n, _dptr(tk), _dptr(rho), _dptr(y), _dptr(sm), _dptr(sn), _dptr(q),
                           _dptr(qd), _dptr(h), _dptr(d))
        return q, qd, h, d

    def cp(self, tk, y):
        n = len(tk)
        out = np.empty(n)
        self.lib.orc_cp(n, _dptr(_c(tk)), _dptr(_c(y)), _dptr(out))
        return out

    def enthalpy(self, tk, y):
        n = len(tk)
        h, hm = np.empty((LSP, n)), np.empty(n)
        self.lib.orc_enthalpy(n, _dptr(_c(tk)), _dptr(_c(y)), _dptr(h), _dptr(hm))
        return h, hm

    def props(self, tk, y):
        """Returns (y_clipped, vmu, vtc, vdf[52,n], nsub)."""
        n = len(tk)
        yc = np.array(y, dtype=np.float64, order="C", copy=True)
        vmu, vtc, vdf = np.empty(n), np.empty(n), np.empty((LSP, n))
        nsub = np.empty(n, dtype=np.int32)
        self.lib.orc_props(n, _dptr(_c(tk)), _dptr(yc), _dptr(vmu), _dptr(vtc), _dptr(vdf), _iptr(nsub))
        return yc, vmu, vtc, vdf, nsub

    def species_update(self, rho, y0, rc, sour, dt, isor=100, relx=0.99, tol=1e-8, y_start=None,
                       soot0=None, spnorm=None, face_sum=None, face_nbr=None):
        """Returns (y_new[52,n], soot[2,n], passes)."""
        n = y0.shape[1]
        y = np.array(y0 if y_start is None else y_start, dtype=np.float64, order="C", copy=True)
        s0 = _c(np.zeros((2, n)) if soot0 is None else soot0)
        s = s0.copy()
        sp = float(n * (LSP - 1)) if spnorm is None else float(spnorm)
        fs = _dptr(_c(face_sum)) if face_sum is not None else None
        fn = _dptr(_c(face_nbr)) if face_nbr is not None else None
        keep = (face_sum, face_nbr)
        passes = self.lib.orc_species_update(
            n, _dptr(_c(rho)), _dptr(_c(y0)), _dptr(y), _dptr(_c(rc)), _dptr(_c(sour)), _dptr(s0),
            _dptr(s), fs, fn, ctypes.c_double(dt), isor, ctypes.c_double(relx),
            ctypes.c_double(tol), ctypes.c_double(sp))
        del keep
        return y, s, passes

    # ---------------------------------------------------------------- ISKIP
    # The reference skips cells with ISKIP >= 3 in CKRATES (ckrates.f:94), SOLVESP (solvesp.f:89,2842)
    # and the T Newton (solveh.f:1173), and cells with ISKIP >= 10 in SOLVEH's rates (solveh.f:119).
    # A skipped cell keeps what its arrays hold; in a fresh run that is zero (the COMMON blocks), and
    # a cell with 3 <= ISKIP < 10 gets its omega from that zero RC, i.e. zero. The per-cell routines
    # above are unchanged; these wrappers apply the skips around them.
    @staticmethod
    def _skipped(iskip, level):
        return np.asarray(iskip) >= level

    def rates_iskip(self, tk, rho, y, iskip, stmf=None, stnd=None):
        rc, sour = self.rates(tk, rho, y, stmf, stnd)
        s = self._skipped(iskip, 3)
        rc[:, s] = 0.0
        sour[:, s] = 0.0
        return rc, sour

    def omega_iskip(self, tk, rho, y, iskip, stmf=None, stnd=None):
        q, qd, h, d = self.omega(tk, rho, y, stmf, stnd)
        s = self._skipped(iskip, 3)
        q[:, s] = 0.0
        qd[s] = 0.0
        d[:, s] = 0.0
        return q, qd, h, d

    def species_update_iskip(self, rho, y0, rc, sour, dt, iskip, **kw):
        """The update of the cells with ISKIP < 3 (in their order, the residual over them only, the
        spnorm of the whole field); skipped cells keep Y and soot."""
        n = y0.shape[1]
        act = ~self._skipped(iskip, 3)
        kw.setdefault("spnorm", float(n * (LSP - 1)))
        sub = lambda a: None if a is None else np.ascontiguousarray(a[..., act])
        y_start = kw.pop("y_start", None)
        soot0 = kw.pop("soot0", None)
        ya, sa, passes = self.species_update(rho[act], sub(y0), sub(rc), sub(sour), dt, y_start=sub(y_start),
                                             soot0=sub(soot0), **kw)
        y = np.array(y0 if y_start is None else y_start, dtype=np.float64, copy=True)
        soot = np.zeros((2, n)) if soot0 is None else np.array(soot0, dtype=np.float64, copy=True)
        y[:, act] = ya
        soot[:, act] = sa
        return y, soot, passes

    def temperature_iskip(self, tk_guess, y, ht, iskip):
        t = self.temperature(tk_guess, y, ht)
        s = self._skipped(iskip, 3)
        t[s] = np.asarray(tk_guess)[s]
        return t

    def nsub(self, rho, y, qdsp, dt, c_tau=1.0, y_tau=1e-3, nsub_max=200):
        """Per-cell sub-step counts of the batched integration and the ratio x they come from."""
        n = len(rho)
        ns, x = np.empty(n, dtype=np.int32), np.empty(n)
        self.lib.orc_nsub(n, _dptr(_c(rho)), _dptr(_c(y)), _dptr(_c(qdsp)), ctypes.c_double(dt),
                          ctypes.c_double(c_tau), ctypes.c_double(y_tau), int(nsub_max), _iptr(ns), _dptr(x))
        return ns, x

    def integrate(self, tk, rho, y, pnd, nsub, dt, soot=None, isor=100, relx=0.99, tol=1e-8):
        """Batched stiff integration over dt; returns (tk, rho, y, soot, passes) after the step."""
        n = len(tk)
        tk, rho = np.array(tk, dtype=np.float64), np.array(rho, dtype=np.float64)
        y = np.array(y, dtype=np.float64, order="C", copy=True)
        s = np.array(np.zeros((2, n)) if soot is None else soot, dtype=np.float64, order="C", copy=True)
        passes = np.empty(n, dtype=np.int32)
        self.lib.orc_integrate(n, _dptr(tk), _dptr(rho), _dptr(y), _dptr(s), _dptr(_c(pnd)),
                               _iptr(_c(nsub, np.int32)), ctypes.c_double(dt), int(isor), ctypes.c_double(relx),
                               ctypes.c_double(tol), _iptr(passes))
        return tk, rho, y, s, passes

    def faces(self, lj, li, rho, vdf, u, v, tmu, yr, xxs, xxc, yys, yyc, isym=1, dt=1e-3, sigsp=0.7):
        """E/W/N/S species coefficients [51][lj*li] of the interior cells (zero elsewhere)."""
        ne = lj * li
        out = [np.zeros((LSP - 1, ne)) for _ in range(4)]
        self.lib.orc_faces(lj, li, _dptr(_c(rho)), _dptr(_c(vdf)), _dptr(_c(u)), _dptr(_c(v)), _dptr(_c(tmu)),
                           _dptr(_c(yr)), _dptr(_c(xxs)), _dptr(_c(xxc)), _dptr(_c(yys)), _dptr(_c(yyc)), int(isym),
                           ctypes.c_double(dt), ctypes.c_double(sigsp), *[_dptr(o) for o in out])
        return tuple(out)

    def zfaces(self, lj, li, rho, tcp, vtc, tmu, u, v, yr, xxs, xxc, yys, yyc, isym=1, dt=1e-3, sigh=0.9):
        """Enthalpy-equation coefficients (ze, zw, zn, zs) [lj*li] of the interior cells and EKT [lj*li]."""
        ne = lj * li
        out = [np.zeros(ne) for _ in range(5)]
        self.lib.orc_zfaces(lj, li, *[_dptr(_c(a)) for a in (rho, tcp, vtc, tmu, u, v, yr, xxs, xxc, yys, yyc)],
                            int(isym), ctypes.c_double(dt), ctypes.c_double(sigh), *[_dptr(o) for o in out])
        return tuple(out[:4]), out[4]

    def enthalpy_rhs(self, lj, li, tk, rho, y_new, ht, stmf, vdf, tmu, ekt, rc, yr, xxs, xxc, yys, yyc, isym=1,
                     dt=1e-3, sigsp=0.9):
        """Enthalpy right-hand side RHSZ [lj*li], QDSP [52][lj*li] and QDOT [lj*li] of the interior cells
        (zero elsewhere); rc [544][lj*li] is the start-state rate table."""
        ne = lj * li
        rhsz, qdsp, qdot = np.zeros(ne), np.zeros((LSP, ne)), np.zeros(ne)
        self.lib.orc_enthalpy_rhs(lj, li, *[_dptr(_c(a)) for a in (tk, rho, y_new, ht, stmf, vdf, tmu, ekt, rc, yr,
                                                                    xxs, xxc, yys, yyc)],
                                  int(isym), ctypes.c_double(dt), ctypes.c_double(sigsp), _dptr(rhsz), _dptr(qdsp),
                                  _dptr(qdot))
        return rhsz, qdsp, qdot

    def enthalpy_relax(self, lj, li, rho, rhsz, z, ht, isor=100, relx=0.99, tol=1e-8, hnorm=None):
        """FPZ after the point relaxation (starting from ht) and the pass count the reference reports."""
        fpz = np.array(ht, dtype=np.float64, copy=True)
        self.lib.orc_enthalpy_relax.restype = ctypes.c_int
        passes = self.lib.orc_enthalpy_relax(lj, li, *[_dptr(_c(a)) for a in (rho, rhsz, *z)], _dptr(fpz), int(isor),
                                             ctypes.c_double(relx), ctypes.c_double(tol),
                                             ctypes.c_double(float(lj * li) if hnorm is None else hnorm))
        return fpz, passes

    def temperature_ke(self, lj, li, tk, y, fpz, u, v, w=None):
        """Temperature of the interior cells from FPZ less the kinetic energy (guess: tk)."""
        t = np.array(tk, dtype=np.float64, copy=True)
        self.lib.orc_temperature_ke(lj, li, _dptr(t), _dptr(_c(y)), _dptr(_c(fpz)), _dptr(_c(u)), _dptr(_c(v)),
                                    None if w is None else _dptr(_c(w)))
        return t

    def enthalpy_solve(self, lj, li, tk, rho, y_start, y_new, ht, stmf, vtc, vdf, u, v, tmu, yr, xxs, xxc, yys, yyc,
                       w=None, isym=1, dt=1e-3, sigsp=0.9, sigh=0.9, isor=100, relx=0.99, tol=1e-8, hnorm=None):
        """The whole enthalpy step (SPGSOLV's EKT and Z, SOLVEH): returns a dict with fpz, tk, passes,
        rhsz, z, qdsp, qdot. Start state: tk, rho, y_start (rates, cp); y_new: after the species update."""
        tcp = self.cp(tk, y_start)
        z, ekt = self.zfaces(lj, li, rho, tcp, vtc, tmu, u, v, yr, xxs, xxc, yys, yyc, isym=isym, dt=dt, sigh=sigh)
        rc, _ = self.rates(tk, rho, y_start)
        rhsz, qdsp, qdot = self.enthalpy_rhs(lj, li, tk, rho, y_new, ht, stmf, vdf, tmu, ekt, rc, yr, xxs, xxc, yys,
                                             yyc, isym=isym, dt=dt, sigsp=sigsp)
        fpz, passes = self.enthalpy_relax(lj, li, rho, rhsz, z, ht, isor=isor, relx=relx, tol=tol, hnorm=hnorm)
        tk_new = self.temperature_ke(lj, li, tk, y_new, fpz, u, v, w)
        return dict(fpz=fpz, tk=tk_new, passes=passes, rhsz=rhsz, z=z, qdsp=qdsp, qdot=qdot, ekt=ekt)

    def density(self, lj, li, tk, y):
        """RHONP [lj*li] of the gas law at PBACK with the grid's edge rules (main:1056-1068)."""
        out = np.empty(lj * li)
        self.lib.orc_density(lj, li, _dptr(_c(tk)), _dptr(_c(y)), _dptr(out))
        return out

    def fdetail(self, lj, li, x, y, rho, u, v, tk, qdot, vmu, vtc, fsp, vdf, qdsp):
        """FDETAIL fields [10 + 4*52, lj*li] (stdata.f:26-118)."""
        out = np.zeros((10 + 4 * LSP, lj * li))
        self.lib.orc_fdetail(lj, li, *[_dptr(_c(a)) for a in (x, y, rho, u, v, tk, qdot, vmu, vtc, fsp, vdf, qdsp)],
                             _dptr(out))
        return out

    def enthalpy_total(self, tk, y):
        """Total enthalpy per cell at its own T (the quantity uc_hold_enthalpy holds)."""
        enth = np.empty(len(tk))
        self.lib.orc_enthalpy_total(len(tk), _dptr(_c(tk)), _dptr(_c(y)), _dptr(enth))
        return enth

    def temperature_held(self, tk_guess, y, pnd, enth, with_conv=False):
        """(tk, rho) from the held total enthalpy and new Y, rho at the cell pressure; with_conv adds
        per cell whether the Newton met its step rule."""
        tk = np.array(tk_guess, dtype=np.float64, copy=True)
        rho = np.empty(len(tk))
        conv = np.zeros(len(tk), dtype=np.int32)
        self.lib.orc_temperature_held(len(tk), _dptr(tk), _dptr(rho), _dptr(_c(y)), _dptr(_c(pnd)), _dptr(_c(enth)),
                                      _iptr(conv))
        return (tk, rho, conv.astype(bool)) if with_conv else (tk, rho)

    def temperature(self, tk_guess, y, ht):
        tk = np.array(tk_guess, dtype=np.float64, copy=True)
        self.lib.orc_temperature(len(tk), _dptr(tk), _dptr(_c(y)), _dptr(_c(ht)))
        return tk
