"""Discretised problem container: the arrays handed to pb_create().

A Problem holds the current cells, charge sub-cells (with their node ids), the polygon
vertex pool, ports, lumped elements and the sweep flags of one structure. It is what
the reference keeps in peec_t after wire_build() (include/peec.h:138-231), reduced to
what the frequency-sweep hot path reads.
"""
import math

import numpy as np

from .abi import CELL_DTYPE, LUMP_DTYPE, MUT_DTYPE, PORT_DTYPE

C0 = 2.99792458e8
PI = 4.0 * math.atan(1.0)


class Problem:
    def __init__(self, seg, chg, chgnode, pv, maxid, port, lump=None, mut=None,
                 capacitance=0, retardation=0, skin=0, gp=0, gpz=0.0, gmin=0.0,
                 f0=0.0, f1=0.0, nfreq=1, flog=0, title="", planewave=None, compress=0, ctol=0.0,
                 accel=0, sources=None):
        self.seg = np.ascontiguousarray(seg, dtype=CELL_DTYPE)
        self.chg = np.ascontiguousarray(chg, dtype=CELL_DTYPE)
        self.chgnode = np.ascontiguousarray(chgnode, dtype=np.int32)
        self.pv = np.ascontiguousarray(pv, dtype=np.float64).reshape(-1)
        self.maxid = int(maxid)
        self.port = np.ascontiguousarray(port, dtype=PORT_DTYPE)
        self.lump = np.ascontiguousarray(lump if lump is not None else
                                         np.zeros(0, LUMP_DTYPE), dtype=LUMP_DTYPE)
        self.mut = np.ascontiguousarray(mut if mut is not None else
                                        np.zeros(0, MUT_DTYPE), dtype=MUT_DTYPE)
        self.capacitance, self.retardation = int(capacitance), int(retardation)
        self.skin, self.gp = int(skin), int(gp)
        self.gpz, self.gmin = float(gpz), float(gmin)
        self.f0, self.f1, self.nfreq, self.flog = float(f0), float(f1), int(nfreq), int(flog)
        self.title = title
        self.planewave = tuple(planewave) if planewave is not None else None
        # solver keys of the .peec file (compression = 1 [tol], acceleration = 1)
        self.compress, self.ctol, self.accel = int(compress), float(ctol), int(accel)
        # independent sources (isvsrc, n1, n2, amp, phase_deg) in file order (src_t)
        self.sources = [tuple(x) for x in sources] if sources is not None else []

    # include/peec.h:241-248
    def freq_at(self, i):
        if self.nfreq <= 1:
            return self.f0
        if self.flog:
            return self.f0 * math.pow(self.f1 / self.f0, i / (self.nfreq - 1))
        return self.f0 + (self.f1 - self.f0) * i / (self.nfreq - 1)

    def freqs(self):
        return np.array([self.freq_at(i) for i in range(self.nfreq)], dtype=np.float64)

    def kw(self, f):
        return 2 * PI * f / C0 if self.retardation else 0.0

    def save(self, path):
        np.savez_compressed(
            path, seg=self.seg.view(np.uint8), chg=self.chg.view(np.uint8),
            chgnode=self.chgnode, pv=self.pv, port=self.port.view(np.uint8),
            lump=self.lump.view(np.uint8), mut=self.mut.view(np.uint8),
            scal=np.array([self.maxid, self.capacitance, self.retardation, self.skin,
                           self.gp, self.nfreq, self.flog], dtype=np.int64),
            scald=np.array([self.gpz, self.gmin, self.f0, self.f1]),
            title=np.array(self.title))

    @classmethod
    def load(cls, path):
        z = np.load(path)
        s, d = z["scal"], z["scald"]
        return cls(z["seg"].view(CELL_DTYPE), z["chg"].view(CELL_DTYPE), z["chgnode"],
                   z["pv"], int(s[0]), z["port"].view(PORT_DTYPE),
                   z["lump"].view(LUMP_DTYPE), z["mut"].view(MUT_DTYPE),
                   capacitance=s[1], retardation=s[2], skin=s[3], gp=s[4],
                   gpz=d[0], gmin=d[1], f0=d[2], f1=d[3], nfreq=s[5], flog=s[6],
                   title=str(z["title"]))
