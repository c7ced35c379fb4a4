"""The benchmark workloads as .peec text (seeded, synthetic; no external data).

cfg1  straight thin-wire dipole, 0.5 m, r = 1 mm, 2 arms x 32 segments, centre 1 A port,
      capacitance = 1, quasi-static, 100 log frequencies 10 MHz - 1 GHz
cfg2  copper plate 100 x 50 mm (35 um, 64 x 32 grid) 5 mm over a ground plane fed by a
      5 mm vertical wire at the corner; capacitance, retardation, skin effect;
      512 frequencies, df = 5 MHz
cfg3  batch of random thin-wire polylines: per instance numpy.random.default_rng(seed+i),
      20-400 segments random-walked in a 10 cm cube (steps 2-8 mm), radius 0.1-2 mm, port
      across a gap cut into the first segment; capacitance, retardation,
      64 log frequencies 50 MHz - 3 GHz
cfg4  volume-cell bar stack for the compressed (H-matrix + GMRES) path: copper plate
      40 x 40 mm, 0.2 mm thick, 96 x 96 grid x 4 layers (74,496 current cells), retardation,
      32 log frequencies 1 MHz - 2 GHz, ACA tolerance 1e-6; fed across the diagonal
      (node 1 at one corner, node 2 at the opposite one, as the compressed plate sample)
cfg5  mixed conductor / dielectric full-wave structure above a ground plane (z = 0):
      6 disks (r = 10 mm, 8 rings x 32 sectors) and 4 convex quads (sides 20-40 mm,
      24 x 24 grid) at seeded positions in a 60 mm box, one horizontal panel per height
      level so that none intersects another, and a dielectric brick 30 x 30 x 1.6 mm,
      epsr 4.4, 30 x 30 x 2 cells, 2 mm above the ground plane (every charge cell strictly
      above z = 0); capacitance, retardation; plane wave theta 30, phi 45 deg, 1 V/m, plus
      a port between the centres of the first two disks; 256 frequencies, df = 10 MHz
Scaled-down variants of cfg2 (plate grid na x nb) serve the parity tests.
"""
import numpy as np

CFG1 = """OpenPEEC 1 0
title = thin-wire dipole 0.5 m, 2x32 segments, quasi-static, 100 log frequencies
capacitance = 1
retardation = 0
node = 1 0 0 -0.0005
node = 2 0 0 0.0005
wire = 0 0 -0.25 0 0 -0.0005 1e-3 5.8e7 32
wire = 0 0 0.0005 0 0 0.25 1e-3 5.8e7 32
port = 1 2 50
frequency = 1e7 1e9 99 log
end
"""


def cfg2(na=64, nb=32, nfreq=512, f0=5e6, df=5e6):
    f1 = f0 + df * (nfreq - 1)
    return f"""OpenPEEC 1 0
title = plate 100x50 mm {na}x{nb} over groundplane fed by 5 mm wire
capacitance = 1
retardation = 1
skineffect = 1
groundplane = 0
node = 1 0 0 0
plate = 0 0 0.005  0.1 0 0  0 0.05 0  35e-6 5.8e7 {na} {nb}
wire = 0 0 0 0 0 0.005 0.5e-3 5.8e7 4
port = 1 0 50
frequency = {f0:.10g} {f1:.10g} {nfreq - 1}
end
"""


CFG2 = cfg2()


def cfg3_instance(seed, i, nmin=20, nmax=400, nfreq=64):
    """One random polyline of the config-3 batch as .peec text."""
    rng = np.random.default_rng(seed + i)
    n = int(rng.integers(nmin, nmax + 1))
    p = rng.uniform(0.02, 0.08, 3)
    pts = [p.copy()]
    while len(pts) < n + 1:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        step = rng.uniform(2e-3, 8e-3)
        q = pts[-1] + step * d
        if np.all(q >= 0) and np.all(q <= 0.1):
            pts.append(q)
    radius = rng.uniform(0.1e-3, 2e-3)
    a, b = pts[0], pts[1]
    g0, g1 = a + 0.45 * (b - a), a + 0.55 * (b - a)
    f = lambda v: " ".join("%.12g" % x for x in v)
    lines = ["OpenPEEC 1 0", f"title = random wire seed {seed} instance {i}, {n} segments",
             "capacitance = 1", "retardation = 1",
             f"node = 1 {f(g0)}", f"node = 2 {f(g1)}",
             f"wire = {f(a)} {f(g0)} {radius:.12g} 5.8e7 1",
             f"wire = {f(g1)} {f(b)} {radius:.12g} 5.8e7 1"]
    for k in range(1, n):
        lines.append(f"wire = {f(pts[k])} {f(pts[k + 1])} {radius:.12g} 5.8e7 1")
    lines += ["port = 1 2 50", f"frequency = 5e7 3e9 {nfreq - 1} log", "end", ""]
    return "\n".join(lines)


def cfg4(nx=96, ny=96, nz=4, nfreq=32, L=0.04, W=0.04, t=2e-4):
    return f"""OpenPEEC 1 0
title = bar stack {L * 1e3:g}x{W * 1e3:g} mm, {t * 1e3:g} mm thick, {nx}x{ny}x{nz} cells
compression = 1 1e-6
retardation = 1
plate = 0 0 0  {L:.10g} 0 0  0 {W:.10g} 0  {t:.10g} 5.8e7 {nx} {ny} {nz}
node = 1 0 0 0
node = 2 {L:.10g} {W:.10g} 0
port = 1 2 50
frequency = 1e6 2e9 {nfreq - 1} log
end
"""


def cfg5(seed=0, ndisk=6, nquad=4, disk_grid=(8, 32), quad_grid=24, brick=(30, 30, 2),
         nfreq=256, f0=1e7, df=1e7):
    """Config 5 as .peec text; smaller counts and grids give the scaled-down variants
    (ndisk >= 2: the port joins the centres of the first two disks)."""
    rng = np.random.default_rng(seed)
    f = lambda v: " ".join("%.9g" % x for x in v)
    box = 0.06
    # brick 30 x 30 x 1.6 mm centred in the box, 2 mm above the ground plane
    bx = by = 0.5 * (box - 0.03)
    lines = ["OpenPEEC 1 0",
             f"title = cfg5 seed {seed}: {ndisk} disks, {nquad} quads, dielectric brick over ground",
             "capacitance = 1", "retardation = 1", "groundplane = 0",
             f"dielectric = {bx:.9g} {by:.9g} 0.002  0.03 0 0  0 0.03 0  0.0016 4.4 "
             f"{brick[0]} {brick[1]} {brick[2]}"]
    # one panel per height level between 6 mm and 58 mm, in a shuffled order
    kinds = ["disk"] * ndisk + ["quad"] * nquad
    levels = np.linspace(0.006, 0.058, len(kinds))
    order = rng.permutation(len(kinds))
    disks = []
    for lev, kidx in zip(levels, order):
        if kinds[kidx] == "disk":
            c = np.array([rng.uniform(0.012, box - 0.012), rng.uniform(0.012, box - 0.012), lev])
            disks.append(c)
            lines.append(f"disk = {f(c)}  0 0 1  0.01 3.5e-5 5.8e7 {disk_grid[0]} {disk_grid[1]}")
        else:
            # a convex quadrilateral: an a x b rectangle (sides 20-40 mm) with each corner
            # moved by less than 15 % of the shorter side, inside the box
            a, b = rng.uniform(0.02, 0.04, 2)
            jit = 0.15 * min(a, b) * rng.uniform(-1, 1, (4, 2))
            x0, y0 = rng.uniform(0, box - a), rng.uniform(0, box - b)
            v = np.array([[0, 0], [a, 0], [a, b], [0, b]]) + jit
            v[:, 0] = np.clip(v[:, 0] + x0, 0, box)
            v[:, 1] = np.clip(v[:, 1] + y0, 0, box)
            pts = " ".join(f(np.array([p[0], p[1], lev])) for p in v)
            lines.append(f"quad = {pts}  3.5e-5 5.8e7 {quad_grid} {quad_grid}")
    lines += [f"node = 1 {f(disks[0])}", f"node = 2 {f(disks[1])}", "port = 1 2 50",
              "planewave = 30 45 1 1.0",
              f"frequency = {f0:.10g} {f0 + (nfreq - 1) * df:.10g} {nfreq - 1}", "end", ""]
    return "\n".join(lines)
