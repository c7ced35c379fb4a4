"""Write the golden fixtures of the parity tests from the reference implementation.

Runs only where the reference checkout is available (it builds oracle/_ref from the
reference's own sources with oracle/Makefile). For every case it stores:
  * the discretised problem exactly as the reference's wire_build produced it,
  * sampled partial-inductance / potential-coefficient entries from the reference's
    lp_entry / pot_entry (src/partial.c:371-424, src/potential.c:124-150),
  * the Z matrix of the reference's own sweep (solve(), src/solve.c:171-430) at the
    listed frequencies.

    python tests/golden/make_golden.py            # all small cases (about a minute)
    python tests/golden/make_golden.py --cfg2     # + the full 64x32 plate at 2 frequencies
    python tests/golden/make_golden.py --pw-only  # only the plane-wave cases (tests/golden/pw)
    python tests/golden/make_golden.py --comp-only  # only the compressed-path cases (tests/golden/comp)
    python tests/golden/make_golden.py --dropin-only  # the reference CLI's output files (tests/golden/dropin)
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from openpeec_b200 import configs  # noqa: E402
from oracle.pyoracle import RefLib, reference_root  # noqa: E402

REF = reference_root()
if REF is None:
    sys.exit("make_golden.py needs the reference checkout: set PEEC_REFERENCE")
C0 = 2.99792458e8


def sample_pairs(n, count, rng):
    if n == 0:
        return np.zeros((0, 2), np.int32)
    diag = np.arange(min(n, 16))
    pairs = [np.stack([diag, diag], 1)]
    near = rng.integers(0, n, count // 2)
    pairs.append(np.stack([near, np.clip(near + rng.integers(-3, 4, len(near)), 0, n - 1)], 1))
    pairs.append(rng.integers(0, n, (count // 2, 2)))
    return np.concatenate(pairs).astype(np.int32)


def make_case(name, peec_text, freqs, count=300, threads=8):
    with tempfile.NamedTemporaryFile("w", suffix=".peec", delete=False) as f:
        f.write(peec_text)
        path = f.name
    RefLib.set_threads(threads)
    r = RefLib(path)
    prob = r.problem()
    rng = np.random.default_rng(1234)
    kws = [0.0, 2 * np.pi * max(freqs) / C0]
    lp = sample_pairs(r.nseg, count, rng)
    lp_v = np.array([[r.lp_entry(int(i), int(j), kw) for (i, j) in lp] for kw in kws])
    pp = sample_pairs(r.ncell, count // 2, rng) if r.ncell > 0 else np.zeros((0, 2), np.int32)
    p_v = np.array([[r.pot_entry(int(i), int(j), kw) for (i, j) in pp] for kw in kws]) \
        if len(pp) else np.zeros((2, 0), complex)
    zs = []
    for f in freqs:
        r.set_freqs(f, f, 1, 0)
        zs.append(r.solve()[0])
    os.unlink(path)
    out = os.path.join(HERE, name + ".npz")
    tmp = os.path.join(HERE, name + "_prob.npz")
    prob.save(tmp)
    pz = dict(np.load(tmp))
    os.unlink(tmp)
    np.savez_compressed(out, **{"prob_" + k: v for k, v in pz.items()}, freqs=np.array(freqs),
                        z=np.array(zs), kws=np.array(kws), lp_ij=lp, lp_v=lp_v, p_ij=pp, p_v=p_v,
                        peec=np.array(peec_text))
    print(name, "nseg", r.nseg, "ncell", r.ncell, "nunknown", r.nunknown, "->", out)


def make_pw_case(name, peec_text, freqs, threads=8):
    """Plane-wave case: the reference's open-circuit port voltages (p->voc) and, when the
    input asks for distributions, the induced segment currents (p->segipw), one solve per
    frequency (solve.c:372-389). Written to tests/golden/pw/."""
    with tempfile.NamedTemporaryFile("w", suffix=".peec", delete=False) as f:
        f.write(peec_text)
        path = f.name
    RefLib.set_threads(threads)
    r = RefLib(path)
    prob = r.problem()
    vocs, segs, pwp = [], [], None
    for fr in freqs:
        r.set_freqs(fr, fr, 1, 0)
        r.solve()
        voc, seg, pwp = r.voc()
        vocs.append(voc[:, 0])
        segs.append(seg[0] if seg is not None else np.zeros(r.nseg, complex))
    os.unlink(path)
    os.makedirs(os.path.join(HERE, "pw"), exist_ok=True)
    out = os.path.join(HERE, "pw", name + ".npz")
    tmp = os.path.join(HERE, name + "_prob.npz")
    prob.save(tmp)
    pz = dict(np.load(tmp))
    os.unlink(tmp)
    np.savez_compressed(out, **{"prob_" + k: v for k, v in pz.items()}, freqs=np.array(freqs),
                        voc=np.array(vocs).T, segipw=np.array(segs), pw=pwp,
                        has_segi=np.array(seg is not None), peec=np.array(peec_text))
    print(name, "nseg", r.nseg, "voc", np.array(vocs).T.ravel()[:2], "->", out)


def make_src_case(name, peec_text, freqs, threads=8):
    """Independent-source case: the node voltages of the reference's source solve
    (mna_rhs_sources through its dense MNA, solve.c:392-396) at each frequency, and the
    source list as the package's parser reads it. Written to tests/golden/src/."""
    from openpeec_b200 import geometry
    with tempfile.NamedTemporaryFile("w", suffix=".peec", delete=False) as f:
        f.write(peec_text)
        path = f.name
    RefLib.set_threads(threads)
    r = RefLib(path)
    prob = r.problem()
    vn = np.array([r.vnode(fr) for fr in freqs])
    srcs = np.array(geometry.parse_peec(peec_text).sources, dtype=np.float64).reshape(-1, 5)
    os.unlink(path)
    os.makedirs(os.path.join(HERE, "src"), exist_ok=True)
    out = os.path.join(HERE, "src", name + ".npz")
    tmp = os.path.join(HERE, name + "_prob.npz")
    prob.save(tmp)
    pz = dict(np.load(tmp))
    os.unlink(tmp)
    np.savez_compressed(out, **{"prob_" + k: v for k, v in pz.items()}, freqs=np.array(freqs),
                        vnode=vn, sources=srcs, peec=np.array(peec_text))
    print(name, "nseg", r.nseg, "vnode", vn[0, :3], "->", out)


def make_post_case(name, peec_text, which):
    """Post-processing case: the reference's sweep, then its own output_far or output_tran
    writer (parsed back from the CSV, 10 significant digits), together with the inputs
    the writer read (port-1 segment currents, Zin, S, Voc). Written to tests/golden/post/."""
    import csv
    with tempfile.NamedTemporaryFile("w", suffix=".peec", delete=False) as f:
        f.write(peec_text)
        path = f.name
    r = RefLib(path)
    prob = r.problem()
    r.solve()
    zin, segi, smat = r.results()
    pw = r.voc()
    out = path + ".csv"
    r.output_csv(which, out)
    rows = list(csv.reader(open(out)))[1:]
    os.unlink(out)
    os.unlink(path)
    extra = {}
    if which == "far":
        a = np.array([[float(v) for v in row] for row in rows])
        extra = dict(ff_freq=a[:, 0], ff_th=a[:, 1], ff_ph=a[:, 2], et=a[:, 3] + 1j * a[:, 4],
                     ep=a[:, 5] + 1j * a[:, 6], d_dbi=a[:, 7], g_dbi=a[:, 8])
    else:
        extra = dict(tr_type=np.array([row[0] for row in rows]), tr_i=np.array([int(row[1]) for row in rows]),
                     tr_j=np.array([int(row[2]) for row in rows]), tr_t=np.array([float(row[3]) for row in rows]),
                     tr_y=np.array([float(row[4]) for row in rows]))
    os.makedirs(os.path.join(HERE, "post"), exist_ok=True)
    dst = os.path.join(HERE, "post", name + ".npz")
    tmp = os.path.join(HERE, name + "_prob.npz")
    prob.save(tmp)
    pz = dict(np.load(tmp))
    os.unlink(tmp)
    np.savez_compressed(dst, **{"prob_" + k: v for k, v in pz.items()}, freqs=np.array(r.freqs()), zin=zin,
                        segi=segi if segi is not None else np.zeros(0), smat=smat,
                        voc=pw[0] if pw is not None else np.zeros(0), peec=np.array(peec_text), **extra)
    print(name, which, len(rows), "rows ->", dst)


def post_cases():
    make_post_case("ff_dipole", sample("dipole_ff.peec"), "far")
    mono = sample("monopole_gp.peec").replace("groundplane = 0", "groundplane = 0\nfarfield = 12 16")
    mono = "\n".join(l for l in mono.splitlines() if not l.startswith("frequency")).replace(
        "\nend", "\nfrequency = 1.3e8 1.6e8 1\nend")
    make_post_case("ff_monopole_gp", mono, "far")
    plate = configs.cfg2(16, 8, 2, 6.4e8, 6.4e8).replace("capacitance = 1", "capacitance = 1\nfarfield = 8 12")
    make_post_case("ff_plate_gp", plate, "far")
    make_post_case("tran_tdr", sample("tdr_resistor.peec"), "tran")
    make_post_case("tran_loop_pw", sample("loop_tran.peec"), "tran")
    twop = configs.cfg2(16, 8, 32, 8e7, 8e7).replace("capacitance = 1", "capacitance = 1\ntransient = 1 60")
    make_post_case("tran_plate", twop, "tran")


def src_cases():
    rlc = sample("rlc_series.peec")
    make_src_case("rlc_isource", rlc.replace("end", "isource = 0 1 1.0 30\nend"), [5.0329212e6, 1.0065842e7])
    make_src_case("rlc_vsource", rlc.replace("end", "vsource = 1 0 2.0 0\nend"), [5.0329212e6, 1.0065842e7])
    dip = sample("dipole_halfwave.peec")
    make_src_case("dipole_isource", dip.replace("\nend", "\nisource = 2 1 1.0 0\nend"), [2.93e8, 6.0e8])
    make_src_case("cfg2_isource", configs.cfg2(16, 8, 512).replace("\nend", "\nisource = 0 1 0.5 -45\nend"),
                  [5e6, 6.4e8])


def make_comp_case(name, peec_text, freqs, threads=16):
    """Compressed-path case: Z of the reference's compression = 1 solve (H-matrix + ACA,
    leaf-Schur preconditioner, GMRES) and Z of its dense solve of the same input with the
    compression key removed. Written to tests/golden/comp/."""
    dense_text = "\n".join(l for l in peec_text.splitlines() if not l.startswith("compression"))
    zs = {}
    prob = None
    for tag, text in (("z", peec_text), ("z_dense", dense_text)):
        with tempfile.NamedTemporaryFile("w", suffix=".peec", delete=False) as f:
            f.write(text + "\n")
            path = f.name
        RefLib.set_threads(threads)
        r = RefLib(path)
        if prob is None:
            prob = r.problem()
        out = []
        for fr in freqs:
            r.set_freqs(fr, fr, 1, 0)
            out.append(r.solve()[0])
        zs[tag] = np.array(out)
        os.unlink(path)
    os.makedirs(os.path.join(HERE, "comp"), exist_ok=True)
    out = os.path.join(HERE, "comp", name + ".npz")
    tmp = os.path.join(HERE, name + "_prob.npz")
    prob.save(tmp)
    pz = dict(np.load(tmp))
    os.unlink(tmp)
    np.savez_compressed(out, **{"prob_" + k: v for k, v in pz.items()}, freqs=np.array(freqs),
                        peec=np.array(peec_text), **zs)
    print(name, "nseg", len(prob.seg), "z", zs["z"].ravel()[:1], "dense", zs["z_dense"].ravel()[:1], "->", out)


def make_cfg4_full(freq=1e8, threads=8):
    """Config 4 at full size (the 96 x 96 x 4 volume-bar stack, 74 496 cells) through the
    reference's own CLI on its compressed path (compression = 1 1e-6) at one frequency:
    its Zin (zin.csv, 10 significant digits) and the H-matrix / GMRES statistics of
    peec.log. About five minutes on 8 cores. The geometry is not stored: the tests
    rebuild it from the stored .peec text (plates are within the package's builder)."""
    import re
    import shutil
    text = re.sub(r"frequency\s*=.*", "frequency = %.10g %.10g 0" % (freq, freq), configs.cfg4())
    work = tempfile.mkdtemp(prefix="cfg4_")
    open(os.path.join(work, "cfg4.peec"), "w").write(text)
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "peec"), "-n", str(threads), "cfg4.peec"],
                   cwd=work, check=True, stdout=subprocess.DEVNULL)
    log = open(os.path.join(work, "peec.log")).read()
    row = open(os.path.join(work, "zin.csv")).read().splitlines()[1].split(",")
    z = complex(float(row[2]), float(row[3]))
    m = re.search(r"compression Lp : (\d+) cells, (\d+) far blocks \+ (\d+) near blocks", log)
    g = re.search(r"GMRES solves \(avg ([0-9.]+) iterations\)", log)
    t = re.search(r"solve ([0-9.]+) s", log)
    out = os.path.join(HERE, "comp", "cfg4_full.npz")
    np.savez_compressed(out, freqs=np.array([float(row[1])]), z=np.array([[[z]]]),
                        ncell=np.array(int(m.group(1))), far=np.array(int(m.group(2))),
                        near=np.array(int(m.group(3))), gmres_its=np.array(float(g.group(1))),
                        ref_solve_s=np.array(float(t.group(1))), threads=np.array(threads),
                        peec=np.array(text))
    shutil.rmtree(work, ignore_errors=True)
    print("cfg4_full", z, m.groups(), g.group(1), "->", out)


def cfg5_cases():
    """Scaled-down config 5 (two disks, one quad and a 6 x 6 x 2 dielectric brick over the
    ground plane): the reference's port Z and sampled entries (make_case), and its
    plane-wave open-circuit voltage (make_pw_case), at three frequencies of the sweep."""
    text = configs.cfg5(0, ndisk=2, nquad=1, disk_grid=(4, 16), quad_grid=8, brick=(6, 6, 2), nfreq=3,
                        f0=1e7, df=1.275e9)
    make_case("cfg5_small", text, [1e7, 1.285e9, 2.56e9])
    make_pw_case("cfg5_small_pw", text, [1e7, 1.285e9, 2.56e9])


def make_cfg5_full_ref(freq=1e9, threads=6):
    """Full config 5 (15 374 current cells, 6 925 charge cells) at one frequency through the
    reference's own CLI: port S11 (Touchstone, 10 digits), Z derived from it and the
    plane-wave open-circuit voltage (pw.csv). The dense reference solve takes about
    50 minutes on 6 threads (setup 15 minutes)."""
    text = configs.cfg5(0)
    fs = ("%.6g" % freq).replace("e+0", "e").replace("e+", "e")
    text = "\n".join(("frequency = %s %s 0" % (fs, fs)) if l.startswith("frequency") else l
                      for l in text.splitlines()) + "\n"
    out = run_cli(text, threads=threads)
    s1p = [l.split() for l in out["peec.s1p"].splitlines() if l.strip() and l[0] not in "!#"]
    s11 = complex(float(s1p[0][1]), float(s1p[0][2]))
    pw = out["pw.csv"].splitlines()[1].split(",")
    voc = complex(float(pw[2]), float(pw[3]))
    z = 50.0 * (1 + s11) / (1 - s11)
    np.savez_compressed(os.path.join(HERE, "geom", "cfg5_full_ref.npz"), freq=np.array([freq]), s11=np.array([s11]),
                        z=np.array([z]), voc=np.array([voc]), peec=np.array(text), s1p=np.array(out["peec.s1p"]),
                        pw_csv=np.array(out["pw.csv"]))
    print("cfg5 full reference: Z", z, "Voc", voc)


def comp_cases():
    make_comp_case("compress_wire", sample("compress_wire.peec"), [1e6])
    make_comp_case("compress_plate", sample("compress_plate.peec"), [1e8])
    bars = """OpenPEEC 1 0
title = volume-cell bar stack (reduced)
compression = 1 1e-6
retardation = 1
plate = 0 0 0  0.04 0 0  0 0.04 0  2e-4 5.8e7 12 12 4
node = 1 0 0 0
node = 2 0.04 0.04 0
port = 1 2 50
frequency = 1e6 2e9 1 log
end
"""
    make_comp_case("bars_small", bars, [1e6, 2e9])
    make_comp_case("compress_cap", sample("compress_cap.peec"), [1e6])
    make_comp_case("cap_retarded", configs.cfg2(16, 8, 512).replace("capacitance = 1", "capacitance = 1\ncompression = 1 1e-6"),
                   [3.2e8, 1.28e9])


def pw_cases():
    loop_load = sample("loop_pw.peec").replace("planewave = 90 0 2 1.0",
                                               "planewave = 90 0 2 1.0\ndistribution = 1\nresistor = 1 5 50")
    mono = sample("monopole_gp.peec").replace("groundplane = 0", "groundplane = 0\nplanewave = 60 0 1 1.0")
    make_pw_case("dipole_pw", sample("dipole_pw.peec"), [1.4376e8, 3.0e8])
    make_pw_case("bent_pw", sample("bent_pw.peec"), [1.5e8])
    make_pw_case("loop_pw", sample("loop_pw.peec"), [1e7])
    make_pw_case("loop_pw_load", loop_load, [1e7, 1e8])
    make_pw_case("mono_pw", mono, [1.3e8, 1.45e8, 1.6e8])


def run_cli(peec_text, threads=8):
    """The reference's own CLI (oracle/_ref/peec, built from its sources) on one input:
    its output files, as text."""
    exe = os.path.join(ROOT, "oracle", "_ref", "peec")
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "case.peec"), "w") as f:
            f.write(peec_text)
        subprocess.run([exe, "-n", str(threads), "case.peec"], cwd=d, check=True, stdout=subprocess.DEVNULL)
        out = {}
        for fn in sorted(os.listdir(d)):
            if fn == "case.peec":
                continue
            with open(os.path.join(d, fn)) as f:
                out[fn] = f.read()
    log = out.pop("peec.log")
    assert "normal end" in log, log[-400:]
    out["captotal"] = "\n".join(l for l in log.splitlines() if "total capacitance" in l)
    return out


def with_key(text, line):
    """Insert a key line after the title (as the reference's checks build their variants)."""
    return "\n".join(l + ("\n" + line if l.startswith("title = ") else "") for l in text.splitlines()) + "\n"


def skin_hf(text):
    """skineffect = 1 before the title and a single frequency of 1 GHz."""
    out = []
    for l in text.splitlines():
        if l.startswith("title = "):
            out.append("skineffect = 1")
        out.append("frequency = 1e9 1e9 0" if l.startswith("frequency = ") else l)
    return "\n".join(out) + "\n"


def dropin_cases():
    """Reference CLI outputs (zin.csv, dist.csv, pw.csv, far.csv, tran.csv, Touchstone, the
    total-capacitance log line) of the sample inputs on the hot path, for the drop-in
    binary peec_gpu (openpeec_b200/dropin)."""
    out = os.path.join(HERE, "dropin")
    os.makedirs(out, exist_ok=True)
    wd = sample("wire_dist.peec")
    cases = {
        "rlc_series": sample("rlc_series.peec"),
        "dipole_halfwave": sample("dipole_halfwave.peec"),
        "dipole_hw_accel": with_key(sample("dipole_halfwave.peec"), "acceleration = 1"),
        "dipole_full": sample("dipole_full.peec"),
        "monopole_gp": sample("monopole_gp.peec"),
        "plate_cap": sample("plate_cap.peec"),
        "disk_cap": sample("disk_cap.peec"),
        "quad_square": sample("quad_square.peec"),
        "bar_skin": sample("bar_skin.peec"),
        "wire_skin_hf": sample("wire_skin_hf.peec"),
        "diel_pp": sample("diel_pp.peec"),
        "diel_debye": sample("diel_debye.peec"),
        "strip_dipole_ret": sample("strip_dipole_ret.peec"),
        "compress_wire": sample("compress_wire.peec"),
        "compress_plate": sample("compress_plate.peec"),
        "compress_cap": sample("compress_cap.peec"),
        "wire_dist": wd,
        "wire_dist_cap": "\n".join(("capacitance = 1\n" + l) if l.startswith("distribution = 1") else l
                                   for l in wd.splitlines()) + "\n",
        "twoport_dist": sample("twoport_dist.peec"),
        "tnetwork_l_spara": sample("tnetwork_l_spara.peec"),
        "loop_pw": sample("loop_pw.peec"),
        "bent_pw": sample("bent_pw.peec"),
        "dipole_ff": sample("dipole_ff.peec"),
        "loop_tran": sample("loop_tran.peec"),
        "tdr_resistor": sample("tdr_resistor.peec"),
        # the sheet at 1 GHz with skin effect (the reference's "quad sheet R vs plate" pair):
        # R is 6e-5 of |Z| behind 1e-9 ohm bus resistors, cond(A) ~ 4e13
        "sk_plate_hf": skin_hf(sample("quad_square_ref.peec")),
        "sk_quad_hf": skin_hf(sample("quad_square.peec")),
    }
    for name, text in cases.items():
        files = run_cli(text)
        np.savez_compressed(os.path.join(out, name + ".npz"), peec=np.array(text),
                            names=np.array(sorted(files)), **{"f_" + k: np.array(v) for k, v in files.items()})
        print(name, sorted(files))


def sample(fn):
    with open(os.path.join(REF, "data", "sample", fn)) as f:
        return f.read()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cfg2", action="store_true")
    ap.add_argument("--pw-only", action="store_true", help="only the plane-wave cases")
    ap.add_argument("--comp-only", action="store_true", help="only the compressed-path cases")
    ap.add_argument("--src-only", action="store_true", help="only the independent-source cases")
    ap.add_argument("--post-only", action="store_true", help="only the far-field / transient cases")
    ap.add_argument("--cfg4-only", action="store_true", help="only config 4 at full size (minutes)")
    ap.add_argument("--cfg5-only", action="store_true", help="only the scaled-down config-5 cases")
    ap.add_argument("--dropin-only", action="store_true", help="only the reference-CLI outputs (tests/golden/dropin)")
    ap.add_argument("--cfg5-full", action="store_true", help="full config 5 at 1 GHz through the reference CLI (~1 h)")
    a = ap.parse_args()
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True,
                   stdout=subprocess.DEVNULL)
    if a.dropin_only:
        dropin_cases()
        return
    if a.cfg5_full:
        make_cfg5_full_ref()
        return
    if a.cfg4_only:
        make_cfg4_full()
        return
    if a.cfg5_only:
        cfg5_cases()
        return
    if a.src_only:
        src_cases()
        return
    if a.post_only:
        post_cases()
        return
    if not a.comp_only:
        pw_cases()
    comp_cases()
    if a.pw_only or a.comp_only:
        return
    f1 = [1e7 * (100.0 ** (i / 99.0)) for i in range(100)]
    make_case("cfg1_dipole_qs", configs.CFG1, f1[::9] + [f1[-1]])
    make_case("dipole_halfwave", sample("dipole_halfwave.peec"), [2.8e8, 2.93e8, 3.0e8, 6.0e8])
    make_case("monopole_gp", sample("monopole_gp.peec"), [2.8e8, 2.93e8, 3.0e8, 6.0e8])
    make_case("strip_dipole_ret", sample("strip_dipole_ret.peec"), [1e8, 2.8e8, 5e8])
    make_case("plate_thick", sample("plate_thick.peec"), [1e6, 1e8])
    make_case("quad_square", sample("quad_square.peec"), [1e6, 1e8])
    make_case("disk_cap", sample("disk_cap.peec"), [1e7, 3e8])
    make_case("plate_cap", sample("plate_cap.peec"), [1e7, 3e8])
    make_case("rlc_series", sample("rlc_series.peec"), [1e5, 1e6, 1e7])
    make_case("cfg2_small", configs.cfg2(16, 8, 512), [5e6, 3.2e8, 6.4e8, 1.28e9, 2.56e9])
    for i in range(3):
        make_case("cfg3_small_%d" % i, configs.cfg3_instance(0, i, 20, 80),
                  [5e7, 3.3e8, 1.1e9, 3e9])
    if a.cfg2:
        make_case("cfg2_full", configs.CFG2, [5e6, 1.28e9], count=200, threads=os.cpu_count())


if __name__ == "__main__":
    main()
