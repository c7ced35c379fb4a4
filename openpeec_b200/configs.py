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
