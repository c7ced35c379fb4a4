"""ctypes access to the checker libraries (TEST INFRASTRUCTURE ONLY).

  Oracle  : oracle/_build/liboracle.so, the CPU restatement (peec_oracle.c). Built from
            committed sources with gcc on demand, so it is available wherever the repo is.
  RefLib  : oracle/_ref/libpeecref.so, the reference's own sources + ref_harness.c.
            Only exists where the reference checkout was available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from openpeec_b200.abi import (CELL_DTYPE, LUMP_DTYPE, MUT_DTYPE, PORT_DTYPE,
                               problem_struct, PbProblem)
from openpeec_b200.problem import Problem

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpeecref.so")
REF_BIN = os.path.join(HERE, "_ref", "peec")
_vp = C.c_void_p


def build_oracle():
    src = os.path.join(HERE, "peec_oracle.c")
    if (not os.path.exists(ORACLE_SO)
            or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src)):
        subprocess.run(["make", "-C", HERE, "oracle"], check=True,
                       stdout=subprocess.DEVNULL)
    return ORACLE_SO


def ref_available():
    return os.path.exists(REF_SO)


def reference_root():
    """The reference checkout, where one is present: $PEEC_REFERENCE, else a directory
    named `reference` beside the repository. None when neither exists (e.g. on a machine
    that only has the prebuilt oracle/_ref files)."""
    env = os.environ.get("PEEC_REFERENCE")
    cand = env if env else os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
    return cand if os.path.isdir(os.path.join(cand, "src")) else None


class Oracle:
    """CPU restatement of the reference hot path on a Problem."""
    _L = None

    @classmethod
    def lib(cls):
        if cls._L is None:
            L = C.CDLL(build_oracle())
            L.or_create.restype = _vp
            L.or_create.argtypes = [C.POINTER(PbProblem)]
            L.or_destroy.argtypes = [_vp]
            L.or_sizes.argtypes = [_vp, _vp]
            L.or_cellmap.argtypes = [_vp, _vp, _vp, _vp]
            for f in ("or_lp_entry", "or_pot_entry"):
                getattr(L, f).argtypes = [_vp, C.c_int, C.c_int, C.c_double, _vp]
            L.or_pair_k.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.c_double, _vp]
            L.or_lp_fill.argtypes = [_vp, C.c_double, _vp]
            L.or_pot_fill.argtypes = [_vp, C.c_double, _vp]
            L.or_mna_assemble.argtypes = [_vp, C.c_double, _vp, _vp, _vp]
            L.or_lu_decomp.argtypes = [C.c_int, _vp, _vp]
            L.or_lu_decomp.restype = C.c_int
            L.or_lu_solve.argtypes = [C.c_int, _vp, _vp, _vp]
            L.or_sweep.argtypes = [_vp, C.c_int, _vp, _vp, C.c_int]
            L.or_sweep.restype = C.c_int
            L.or_planewave.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp]
            L.or_planewave.restype = C.c_int
            L.or_zint.argtypes = [_vp, C.c_int, C.c_double, _vp]
            cls._L = L
        return cls._L

    def __init__(self, prob: Problem):
        self.prob = prob
        self._s = problem_struct(prob)
        self.h = self.lib().or_create(C.byref(self._s))
        sz = np.zeros(9, np.int32)
        self.lib().or_sizes(self.h, sz.ctypes.data)
        (self.nseg, self.nchg, self.ncell, self.nnode, self.nunknown, self.offS,
         self.refnode, self.offL, self.offV) = [int(v) for v in sz]

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().or_destroy(self.h)
            self.h = None

    def cellmap(self):
        cid = np.zeros(max(self.ncell, 1), np.int32)
        cof = np.zeros(max(self.nchg, 1), np.int32)
        car = np.zeros(max(self.ncell, 1))
        self.lib().or_cellmap(self.h, cid.ctypes.data, cof.ctypes.data, car.ctypes.data)
        return cid[:self.ncell], cof[:self.nchg], car[:self.ncell]

    def lp_entry(self, i, j, kw):
        o = np.zeros(2)
        self.lib().or_lp_entry(self.h, i, j, kw, o.ctypes.data)
        return complex(o[0], o[1])

    def pot_entry(self, i, j, kw):
        o = np.zeros(2)
        self.lib().or_pot_entry(self.h, i, j, kw, o.ctypes.data)
        return complex(o[0], o[1])

    def pair_k(self, i, j, mirror, kw):
        o = np.zeros(2)
        self.lib().or_pair_k(self.h, i, j, int(mirror), kw, o.ctypes.data)
        return complex(o[0], o[1])

    def lp_fill(self, kw):
        out = np.zeros((self.nseg, self.nseg), np.complex128)
        self.lib().or_lp_fill(self.h, kw, out.ctypes.data)
        return out

    def pot_fill(self, kw):
        out = np.zeros((self.ncell, self.ncell), np.complex128)
        self.lib().or_pot_fill(self.h, kw, out.ctypes.data)
        return out

    def zint(self, k, f):
        o = np.zeros(2)
        self.lib().or_zint(self.h, k, f, o.ctypes.data)
        return complex(o[0], o[1])

    def mna_assemble(self, f, lp, cmat):
        a = np.zeros((self.nunknown, self.nunknown), np.complex128)
        lp = np.ascontiguousarray(lp, np.complex128)
        cm = None if cmat is None else np.ascontiguousarray(cmat, np.complex128)
        self.lib().or_mna_assemble(self.h, f, lp.ctypes.data,
                                   None if cm is None else cm.ctypes.data, a.ctypes.data)
        return a

    def sweep(self, freqs, nthreads=0):
        freqs = np.ascontiguousarray(freqs, np.float64)
        npt = len(self.prob.port)
        z = np.zeros((len(freqs), npt, npt), np.complex128)
        r = self.lib().or_sweep(self.h, len(freqs), freqs.ctypes.data, z.ctypes.data,
                                nthreads)
        if r != 0:
            raise RuntimeError("oracle sweep failed (%d)" % r)
        return z

    def planewave(self, freqs, pw):
        """Plane-wave sweep (mna.c:434-468, solve.c:372-389): pw = (theta_deg, phi_deg,
        pol, amp, phase_deg). Returns (voc [nport, nfreq], segipw [nfreq, nseg])."""
        freqs = np.ascontiguousarray(freqs, np.float64)
        pwp = np.array(pw, np.float64)
        voc = np.zeros((len(self.prob.port), len(freqs)), np.complex128)
        segipw = np.zeros((len(freqs), len(self.prob.seg)), np.complex128)
        r = self.lib().or_planewave(self.h, len(freqs), freqs.ctypes.data, pwp.ctypes.data,
                                    voc.ctypes.data, segipw.ctypes.data)
        if r != 0:
            raise RuntimeError("oracle plane-wave sweep failed (%d)" % r)
        return voc, segipw

    @classmethod
    def lu_decomp(cls, a):
        a = np.ascontiguousarray(a, np.complex128).copy()
        piv = np.zeros(a.shape[0], np.int32)
        r = cls.lib().or_lu_decomp(a.shape[0], a.ctypes.data, piv.ctypes.data)
        return r, a, piv


class RefLib:
    """The reference's own implementation (compiled from its sources into oracle/_ref)."""
    _L = None

    @classmethod
    def lib(cls):
        if cls._L is None:
            if not ref_available():
                raise RuntimeError("oracle/_ref/libpeecref.so not built")
            L = C.CDLL(REF_SO)
            L.rh_load.restype = _vp
            L.rh_load.argtypes = [C.c_char_p]
            L.rh_load_light.restype = _vp
            L.rh_load_light.argtypes = [C.c_char_p]
            L.rh_free.argtypes = [_vp]
            L.rh_info.argtypes = [_vp, _vp]
            L.rh_infod.argtypes = [_vp, _vp]
            L.rh_freq.argtypes = [_vp, C.c_int]
            L.rh_freq.restype = C.c_double
            L.rh_npv.argtypes = [_vp, C.c_int]
            L.rh_cells.argtypes = [_vp, C.c_int, _vp, _vp, C.c_int, _vp]
            L.rh_ports.argtypes = [_vp, _vp]
            L.rh_lumps.argtypes = [_vp, _vp, _vp]
            for f in ("rh_lp_entry", "rh_pot_entry"):
                getattr(L, f).argtypes = [_vp, C.c_int, C.c_int, C.c_double, _vp]
            L.rh_lp_fill.argtypes = [_vp, C.c_double, _vp]
            L.rh_pot_fill.argtypes = [_vp, C.c_double, _vp]
            L.rh_cellmap.argtypes = [_vp, _vp, _vp, _vp]
            L.rh_nodemap.argtypes = [_vp, _vp]
            L.rh_mna_assemble.argtypes = [_vp, C.c_double, _vp]
            L.rh_solve.argtypes = [_vp, _vp]
            L.rh_voc.argtypes = [_vp, _vp, _vp, _vp]
            L.rh_voc.restype = C.c_int
            L.rh_results.argtypes = [_vp, _vp, _vp, _vp]
            L.rh_results.restype = C.c_int
            L.rh_output_far.argtypes = [_vp, C.c_char_p]
            L.rh_output_tran.argtypes = [_vp, C.c_char_p]
            L.rh_vnode.argtypes = [_vp, C.c_double, _vp]
            L.rh_vnode.restype = C.c_int
            L.rh_set_freqs.argtypes = [_vp, C.c_double, C.c_double, C.c_int, C.c_int]
            L.rh_lu_decomp.argtypes = [C.c_int, _vp, _vp]
            L.rh_lu_solve.argtypes = [C.c_int, _vp, _vp, _vp]
            L.rh_set_threads.argtypes = [C.c_int]
            cls._L = L
        return cls._L

    def __init__(self, path, light=False):
        self.h = (self.lib().rh_load_light if light else self.lib().rh_load)(path.encode())
        if not self.h:
            raise RuntimeError("reference failed to load " + path)
        info = np.zeros(20, np.int32)
        self.lib().rh_info(self.h, info.ctypes.data)
        self.info = info
        (self.nseg, self.nchg, self.ncell, self.nnode, self.nunknown, self.offS,
         self.refnode, self.maxid, self.nport, self.nfreq) = [int(v) for v in info[:10]]
        d = np.zeros(4)
        self.lib().rh_infod(self.h, d.ctypes.data)
        self.gpz, self.f0, self.f1, self.gmin = d

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().rh_free(self.h)
            self.h = None

    def problem(self):
        """Export the reference's discretisation as a Problem."""
        L = self.lib()
        nps, npc = L.rh_npv(self.h, 0), L.rh_npv(self.h, 1)
        seg = np.zeros(self.nseg, CELL_DTYPE)
        chg = np.zeros(self.nchg, CELL_DTYPE)
        pv = np.zeros(3 * (nps + npc))
        chgnode = np.zeros(self.nchg, np.int32)
        L.rh_cells(self.h, 0, seg.ctypes.data if self.nseg else None,
                   pv.ctypes.data if nps + npc else None, 0, None)
        L.rh_cells(self.h, 1, chg.ctypes.data if self.nchg else None,
                   pv[3 * nps:].ctypes.data if npc else None, nps,
                   chgnode.ctypes.data if self.nchg else None)
        port = np.zeros(self.nport, PORT_DTYPE)
        L.rh_ports(self.h, port.ctypes.data)
        lump = np.zeros(int(self.info[16]) + 1, LUMP_DTYPE)
        mut = np.zeros(int(self.info[17]) + 1, MUT_DTYPE)
        nl = L.rh_lumps(self.h, lump.ctypes.data, mut.ctypes.data)
        i = self.info
        return Problem(seg, chg, chgnode, pv, self.maxid, port, lump[:nl],
                       mut[:int(i[17])], capacitance=i[10], retardation=i[11], skin=i[12],
                       gp=i[13], gpz=self.gpz, gmin=self.gmin, f0=self.f0, f1=self.f1,
                       nfreq=self.nfreq, flog=i[15])

    def lp_entry(self, i, j, kw):
        o = np.zeros(2)
        self.lib().rh_lp_entry(self.h, i, j, kw, o.ctypes.data)
        return complex(o[0], o[1])

    def pot_entry(self, i, j, kw):
        o = np.zeros(2)
        self.lib().rh_pot_entry(self.h, i, j, kw, o.ctypes.data)
        return complex(o[0], o[1])

    def lp_fill(self, f):
        out = np.zeros((self.nseg, self.nseg), np.complex128)
        self.lib().rh_lp_fill(self.h, f, out.ctypes.data)
        return out

    def pot_fill(self, f):
        out = np.zeros((self.ncell, self.ncell), np.complex128)
        if self.lib().rh_pot_fill(self.h, f, out.ctypes.data):
            raise RuntimeError("reference pot_fill failed")
        return out

    def cellmap(self):
        cid = np.zeros(self.ncell, np.int32)
        cof = np.zeros(self.nchg, np.int32)
        car = np.zeros(self.ncell)
        self.lib().rh_cellmap(self.h, cid.ctypes.data, cof.ctypes.data, car.ctypes.data)
        return cid, cof, car

    def nodemap(self):
        m = np.zeros(self.maxid + 1, np.int32)
        self.lib().rh_nodemap(self.h, m.ctypes.data)
        return m

    def mna_assemble(self, f):
        a = np.zeros((self.nunknown, self.nunknown), np.complex128)
        self.lib().rh_mna_assemble(self.h, f, a.ctypes.data)
        return a

    def freqs(self):
        return np.array([self.lib().rh_freq(self.h, i) for i in range(self.nfreq)])

    def set_freqs(self, f0, f1, nfreq, flog=0):
        self.lib().rh_set_freqs(self.h, f0, f1, nfreq, flog)
        self.nfreq = nfreq

    def solve(self):
        z = np.zeros((self.nfreq, self.nport, self.nport), np.complex128)
        if self.lib().rh_solve(self.h, z.ctypes.data) != 0:
            raise RuntimeError("reference solve failed")
        return z

    def voc(self):
        """Plane-wave results of the last solve(): (voc [nport, nfreq], segipw [nfreq, nseg]
        or None, pw parameters) or None when the input has no plane wave."""
        voc = np.zeros((self.nport, self.nfreq), np.complex128)
        seg = np.zeros((self.nfreq, self.nseg), np.complex128)
        pwp = np.zeros(5)
        r = self.lib().rh_voc(self.h, voc.ctypes.data, seg.ctypes.data, pwp.ctypes.data)
        if r == 0:
            return None
        return voc, (seg if r == 2 else None), pwp

    def results(self):
        """(zin [nport, nfreq], segi [nfreq, nport, nseg] or None, smat [nfreq, nport, nport])
        of the last solve()."""
        zin = np.zeros((self.nport, self.nfreq), np.complex128)
        segi = np.zeros((self.nfreq, self.nport, self.nseg), np.complex128)
        smat = np.zeros((self.nfreq, self.nport, self.nport), np.complex128)
        r = self.lib().rh_results(self.h, zin.ctypes.data, segi.ctypes.data, smat.ctypes.data)
        if r == 0:
            raise RuntimeError("no results: solve() first")
        return zin, (segi if r == 2 else None), smat

    def output_csv(self, which, path):
        """Run the reference's output_far ('far') or output_tran ('tran') into path."""
        f = self.lib().rh_output_far if which == "far" else self.lib().rh_output_tran
        if f(self.h, path.encode()) != 0:
            raise RuntimeError("reference output_%s failed" % which)

    def vnode(self, f):
        """Node voltages [maxid+1] of the independent-source excitation at f (rh_vnode:
        the reference's own fill, MNA, mna_rhs_sources and LU)."""
        out = np.zeros(self.maxid + 1, np.complex128)
        r = self.lib().rh_vnode(self.h, float(f), out.ctypes.data)
        if r != -1:
            raise RuntimeError("rh_vnode status %d" % r)
        return out

    @classmethod
    def set_threads(cls, n):
        return cls.lib().rh_set_threads(n)

    @classmethod
    def lu_decomp(cls, a):
        a = np.ascontiguousarray(a, np.complex128).copy()
        piv = np.zeros(a.shape[0], np.int32)
        r = cls.lib().rh_lu_decomp(a.shape[0], a.ctypes.data, piv.ctypes.data)
        return r, a, piv
