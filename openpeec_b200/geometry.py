"""Reader for the .peec input format and geometry builder (host side).

Covers the keys the sweep hot path needs for thin-wire / bar / plate structures:
title, node, wire, bar, plate (incl. the volume layers of ndiv_t >= 2), port,
resistor, capacitor, inductor, vsource, isource, frequency, nodetol, skineffect, capacitance,
retardation, groundplane, gmin, grading. Unknown keys are ignored (as the reference's
parser does, src/input_data.c:555). quad / disk / dielectric / planewave structures are
not built here (their cells come from the reference's own builder in the fixtures).

The discretisation reproduces the reference's wire_build (src/wire.c:348-913, the
wire and plate parts :420-611): same node matching within nodetol, the same
automatic node numbering, the same cell order and fields. tests/test_geometry.py checks
it field by field against the reference.
"""
import math

import numpy as np

from .abi import CELL_DTYPE, LUMP_DTYPE, PORT_DTYPE, PB_LUMP_C, PB_LUMP_L, PB_LUMP_R, PB_LUMP_V
from .problem import Problem

PI = 4.0 * math.atan(1.0)
SHAPE_ROUND, SHAPE_BAR, SHAPE_PLATE = 0, 1, 2


class PeecInput:
    def __init__(self):
        self.title = ""
        self.nodes = []          # (id, xyz)
        self.wires = []          # dict
        self.plates = []
        self.ports = []          # (n1, n2, z0)
        self.lumps = []          # (kind, n1, n2, val)
        self.f0 = self.f1 = 0.0
        self.nfreq = 0
        self.flog = 0
        self.nodetol = 1e-8
        self.skin = self.capacitance = self.retardation = self.gp = self.grading = 0
        self.gpz = 0.0
        self.gmin = 0.0
        self.maxid = 0
        self.planewave = None    # (theta_deg, phi_deg, pol, amp, phase_deg)
        self.compress, self.ctol, self.accel = 0, 0.0, 0
        self.sources = []        # (isvsrc, n1, n2, amp, phase_deg), file order
        self.unsupported = []


def parse_peec(text):
    """Parse .peec text (src/input_data.c:38-602, subset)."""
    p = PeecInput()
    first = True
    for raw in text.splitlines():
        line = raw.rstrip("\r\n")
        if len(line) < 1 or line.startswith("#"):
            continue
        if line.startswith("end"):
            break
        tok = line.split()
        if first:
            if not tok or tok[0] != "OpenPEEC":
                raise ValueError("not OpenPEEC data")
            first = False
            continue
        if len(tok) < 3 or tok[1] != "=":
            continue
        key, a = tok[0], tok[2:]
        if key == "title":
            p.title = line.split("=", 1)[1].strip()
        elif key == "node":
            nid = int(a[0])
            p.nodes.append((nid, [float(v) for v in a[1:4]]))
            p.maxid = max(p.maxid, nid)
        elif key in ("wire", "bar"):
            w = {"x1": [float(v) for v in a[0:3]], "x2": [float(v) for v in a[3:6]]}
            if key == "bar":
                w.update(shape=SHAPE_BAR, width=float(a[6]), thick=float(a[7]),
                         sigma=float(a[8]), ndiv=int(a[9]), radius=0.0)
            else:
                w.update(shape=SHAPE_ROUND, radius=float(a[6]), sigma=float(a[7]),
                         ndiv=int(a[8]), width=0.0, thick=0.0)
            p.wires.append(w)
        elif key == "plate":
            v = [float(x) for x in a[0:11]]
            p.plates.append({"org": v[0:3], "ea": v[3:6], "eb": v[6:9], "thick": v[9],
                             "sigma": v[10], "na": int(a[11]), "nb": int(a[12]),
                             "nt": int(a[13]) if len(a) >= 14 else 1})
        elif key == "port":
            n1, n2 = int(a[0]), int(a[1])
            p.ports.append((n1, n2, float(a[2])))
            p.maxid = max(p.maxid, n1, n2)
        elif key in ("resistor", "capacitor"):
            n1, n2 = int(a[0]), int(a[1])
            p.lumps.append((PB_LUMP_R if key == "resistor" else PB_LUMP_C, n1, n2, float(a[2])))
            p.maxid = max(p.maxid, n1, n2)
        elif key == "inductor":            # inductor = name n1 n2 L
            n1, n2 = int(a[1]), int(a[2])
            p.lumps.append((PB_LUMP_L, n1, n2, float(a[3])))
            p.maxid = max(p.maxid, n1, n2)
        elif key in ("vsource", "isource"):  # n1 n2 amp [phase_deg] (input_data.c:175-192)
            n1, n2 = int(a[0]), int(a[1])
            amp, ph = float(a[2]), float(a[3]) if len(a) > 3 else 0.0
            if key == "vsource":
                p.lumps.append((PB_LUMP_V, n1, n2, amp))
            p.sources.append((1 if key == "vsource" else 0, n1, n2, amp, ph))
            p.maxid = max(p.maxid, n1, n2)
        elif key == "frequency":
            p.f0, p.f1 = float(a[0]), float(a[1])
            p.nfreq = int(a[2]) + 1
            p.flog = 1 if (len(a) > 3 and a[3] == "log") else 0
        elif key == "nodetol":
            p.nodetol = float(a[0])
        elif key == "skineffect":
            p.skin = int(a[0])
        elif key == "capacitance":
            p.capacitance = int(a[0])
        elif key == "retardation":
            p.retardation = int(a[0])
        elif key == "groundplane":
            p.gp, p.gpz = 1, float(a[0])
        elif key == "gmin":
            p.gmin = float(a[0])
        elif key == "grading":
            p.grading = int(a[0])
        elif key == "planewave":           # planewave = theta phi pol amp [phase] (input_data.c:501-519)
            pol, amp = int(a[2]), float(a[3])
            if pol not in (1, 2) or amp <= 0:
                raise ValueError("planewave: polarisation 1/2 and amplitude > 0")
            p.planewave = (float(a[0]), float(a[1]), pol, amp, float(a[4]) if len(a) > 4 else 0.0)
        elif key == "compression":         # compression = 1 [tol] (input_data.c, solve.c:251-294)
            p.compress = int(a[0])
            p.ctol = float(a[1]) if len(a) > 1 else 0.0
        elif key == "acceleration":        # acceleration = 1 (solve.c:47-64)
            p.accel = int(a[0])
        elif key in ("quad", "disk", "dielectric", "mutual"):
            p.unsupported.append(key)
    return p


def _dist(a, b):
    return math.sqrt((a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2 + (a[2] - b[2]) ** 2)


class _Nodes:
    """Coordinate -> node id table with the reference's matching rule (wire.c:36-63)."""

    def __init__(self, tol, autoid):
        self.tol, self.autoid = tol, autoid
        self.xyz, self.ids = [], []

    def find(self, x):
        for i, y in enumerate(self.xyz):
            if _dist(y, x) <= self.tol:
                return i
        return -1

    def add(self, nid, x):
        self.ids.append(nid)
        self.xyz.append(list(x))

    def at(self, x):
        i = self.find(x)
        if i >= 0:
            return self.ids[i]
        self.autoid += 1
        self.add(self.autoid, x)
        return self.autoid


class _FastNodes(_Nodes):
    """Same rule, with a spatial hash so large plates build in O(n)."""

    def __init__(self, tol, autoid):
        super().__init__(tol, autoid)
        self.cell = max(tol * 4, 1e-12)
        self.grid = {}

    def _key(self, x):
        return tuple(int(math.floor(v / self.cell)) for v in x)

    def find(self, x):
        k = self._key(x)
        best = -1
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for i in self.grid.get((k[0] + dx, k[1] + dy, k[2] + dz), ()):
                        if _dist(self.xyz[i], x) <= self.tol and (best < 0 or i < best):
                            best = i
        return best

    def add(self, nid, x):
        super().add(nid, x)
        self.grid.setdefault(self._key(x), []).append(len(self.xyz) - 1)


def build(p: PeecInput) -> Problem:
    """Discretise wires, bars and plates like src/wire.c:348-611 and return a Problem."""
    if p.unsupported:
        raise NotImplementedError("geometry builder does not handle: " + ", ".join(sorted(set(p.unsupported))))
    nodes = _FastNodes(p.nodetol, p.maxid)
    for nid, x in p.nodes:                       # wire.c:404-412
        if nodes.find(x) >= 0:
            continue
        nodes.add(nid, x)
    segs, chgs, chgnode = [], [], []

    def newcell():
        return np.zeros(1, CELL_DTYPE)[0]

    for w in p.wires:                             # wire.c:420-477
        nd = w["ndiv"]
        x1, x2 = w["x1"], w["x2"]
        prev = -1
        for k in range(nd + 1):
            x = [x1[c] + (x2[c] - x1[c]) * k / nd for c in range(3)]
            nid = nodes.at(x)
            if k > 0:
                s = newcell()
                s["n1"], s["n2"] = prev, nid
                s["x1"] = [x1[c] + (x2[c] - x1[c]) * (k - 1) / nd for c in range(3)]
                s["x2"] = x
                s["len"] = _dist(s["x1"], s["x2"])
                s["shape"], s["radius"], s["sigma"] = w["shape"], w["radius"], w["sigma"]
                s["thick"] = w["thick"]
                if w["shape"] == SHAPE_BAR:
                    wt = w["width"] + w["thick"]
                    s["aL"], s["aP"] = 0.2235 * wt, 0.25 * wt
                    s["area"], s["perim"] = w["width"] * w["thick"], 2 * wt
                else:
                    s["aL"] = s["aP"] = w["radius"]
                    s["area"] = PI * w["radius"] * w["radius"]
                    s["perim"] = 2 * PI * w["radius"]
                s["res"] = s["len"] / (w["sigma"] * s["area"]) if w["sigma"] > 0 else 0.0
                mid = [0.5 * (s["x1"][c] + s["x2"][c]) for c in range(3)]
                for (a, b, nn) in ((s["x1"], mid, s["n1"]), (mid, s["x2"], s["n2"])):
                    c = s.copy()
                    c["x1"], c["x2"], c["wv"] = a, b, (0, 0, 0)
                    c["len"] = _dist(a, b)
                    c["wid"] = 0.0
                    chgs.append(c)
                    chgnode.append(nn)
                segs.append(s)
            prev = nid

    for pl in p.plates:                           # wire.c:480-611
        na, nb = pl["na"], pl["nb"]
        ea, eb, org = pl["ea"], pl["eb"], pl["org"]
        la = math.sqrt(sum(v * v for v in ea))
        lb = math.sqrt(sum(v * v for v in eb))
        ha, hb = la / na, lb / nb
        ta = [v / la for v in ea]
        tb = [v / lb for v in eb]
        xa = [0.5 * la * (1 - math.cos(PI * i / na)) if p.grading else i * ha for i in range(na + 1)]
        xb = [0.5 * lb * (1 - math.cos(PI * i / nb)) if p.grading else i * hb for i in range(nb + 1)]
        nid = [[0] * (nb + 1) for _ in range(na + 1)]
        for ia in range(na + 1):
            for ib in range(nb + 1):
                x = [org[c] + xa[ia] * ta[c] + xb[ib] * tb[c] for c in range(3)]
                nid[ia][ib] = nodes.at(x)
        nt = pl["nt"] if pl["nt"] > 1 else 1
        tl = pl["thick"] / nt
        nv = [ta[1] * tb[2] - ta[2] * tb[1], ta[2] * tb[0] - ta[0] * tb[2], ta[0] * tb[1] - ta[1] * tb[0]]
        last_wid = 0.0
        for it in range(nt):
            zoff = (it - 0.5 * (nt - 1)) * tl
            for d in range(2):
                n1, n2 = (nb, na) if d else (na, nb)
                x1a, x2a = (xb, xa) if d else (xa, xb)
                t1, t2 = (tb, ta) if d else (ta, tb)
                for j in range(n2 + 1):
                    lo = x2a[0] if j == 0 else 0.5 * (x2a[j - 1] + x2a[j])
                    hi = x2a[n2] if j == n2 else 0.5 * (x2a[j] + x2a[j + 1])
                    wid = hi - lo
                    last_wid = wid
                    cen = 0.5 * (lo + hi)
                    for k in range(n1):
                        s = newcell()
                        s["shape"], s["sigma"] = SHAPE_PLATE, pl["sigma"]
                        s["wid"] = wid
                        ia1, ib1 = (j, k) if d else (k, j)
                        ia2, ib2 = (j, k + 1) if d else (k + 1, j)
                        s["n1"], s["n2"] = nid[ia1][ib1], nid[ia2][ib2]
                        base = [org[c] + cen * t2[c] + zoff * nv[c] for c in range(3)]
                        s["x1"] = [base[c] + x1a[k] * t1[c] for c in range(3)]
                        s["x2"] = [base[c] + x1a[k + 1] * t1[c] for c in range(3)]
                        s["wv"] = t2
                        s["len"] = x1a[k + 1] - x1a[k]
                        s["vol"] = 1 if nt > 1 else 0
                        s["thick"] = tl if nt > 1 else pl["thick"]
                        s["area"] = wid * s["thick"]
                        s["perim"] = 2 * (wid + s["thick"])
                        s["aL"] = 0.2235 * (wid + s["thick"])
                        s["aP"] = 0.25 * (wid + s["thick"])
                        s["res"] = s["len"] / (pl["sigma"] * s["area"]) if pl["sigma"] > 0 else 0.0
                        segs.append(s)
        for ia in range(na + 1):                  # dual rectangles, wire.c:592-606
            for ib in range(nb + 1):
                loa = xa[0] if ia == 0 else 0.5 * (xa[ia - 1] + xa[ia])
                hia = xa[na] if ia == na else 0.5 * (xa[ia] + xa[ia + 1])
                lob = xb[0] if ib == 0 else 0.5 * (xb[ib - 1] + xb[ib])
                hib = xb[nb] if ib == nb else 0.5 * (xb[ib] + xb[ib + 1])
                c0 = [org[c] + 0.5 * (loa + hia) * ta[c] + 0.5 * (lob + hib) * tb[c] for c in range(3)]
                c = newcell()
                c["shape"], c["thick"], c["sigma"] = SHAPE_PLATE, pl["thick"], pl["sigma"]
                c["x1"] = [c0[q] - 0.5 * (hia - loa) * ta[q] for q in range(3)]
                c["x2"] = [c0[q] + 0.5 * (hia - loa) * ta[q] for q in range(3)]
                c["wv"] = tb
                c["len"] = _dist(c["x1"], c["x2"])
                c["wid"] = hib - lob
                chgs.append(c)
                chgnode.append(nid[ia][ib])
        del last_wid

    maxid = nodes.autoid
    port = np.array([(a, b, z) for a, b, z in p.ports], dtype=PORT_DTYPE)
    lump = np.zeros(len(p.lumps), LUMP_DTYPE)
    # stamping order of the reference: resistors, capacitors, inductors, vsources
    for i, (k, a, b, v) in enumerate(sorted(p.lumps, key=lambda t: t[0])):
        lump[i]["kind"], lump[i]["n1"], lump[i]["n2"], lump[i]["val"] = k, a, b, v
    return Problem(np.array(segs, dtype=CELL_DTYPE).reshape(-1),
                   np.array(chgs, dtype=CELL_DTYPE).reshape(-1),
                   np.array(chgnode, dtype=np.int32), np.zeros(0), maxid, port, lump,
                   capacitance=p.capacitance, retardation=p.retardation, skin=p.skin,
                   gp=p.gp, gpz=p.gpz, gmin=p.gmin, f0=p.f0, f1=p.f1, nfreq=p.nfreq,
                   flog=p.flog, title=p.title, planewave=p.planewave, compress=p.compress,
                   ctol=p.ctol, accel=p.accel, sources=p.sources)


def load_peec(path) -> Problem:
    with open(path) as f:
        return build(parse_peec(f.read()))
