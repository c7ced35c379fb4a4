"""The drop-in binary peec_gpu: the reference's own CLI (main.c, input_data.c, wire.c,
output.c, farfield.c, transient.c, skin.c, utils.c, compiled unchanged) linked with
openpeec_b200/dropin/peec_shim.c, which supplies the hot-path entry points of
include/peec.h (solve, lp_fill, pot_fill, mna_numbering, lu_decomp, lu_solve, poly_area,
hmat_free) on libpeec_b200.

Fixtures: tests/golden/dropin/*.npz (make_golden.py --dropin-only), the output files of the
reference's CLI on sample inputs on the hot path: zin.csv, the Touchstone file, dist.csv
(current and charge distribution), pw.csv (plane wave), far.csv, tran.csv and the
total-capacitance log line.

CPU: the binary links against libpeec_b200.so, defines the shim's entry points and none of
the reference's hot-path internals, and without a GPU stops with the library's error (no
host fall back). GPU: every output file matches the reference's: port impedances within
1e-6 relative (1e-5 on the compressed path, whose ACA differs from the reference's within
its tolerance), distributions within 1e-6 of their largest entry.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
EXE = os.path.join(ROOT, "openpeec_b200", "dropin", "_build", "peec_gpu")
GOLD = os.path.join(HERE, "golden", "dropin")
CASES = sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLD, "*.npz")))
SHIM = ["solve", "lp_fill", "pot_fill", "mna_numbering", "lu_decomp", "lu_solve", "poly_area", "hmat_free"]
# functions of the replaced reference files that must not be in the binary
REPLACED = ["lp_entry", "pot_entry", "mna_assemble", "mna_sparse", "hmat_build", "gmres_solve", "pc_build",
            "neumann_pair_k", "poly_static", "ribbon_static", "bar_pair", "pot_cells"]


def need_exe():
    if not os.path.exists(EXE):
        pytest.skip("peec_gpu not built (it needs the reference checkout: make -C openpeec_b200/dropin)")


def run(name, workdir):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    with open(os.path.join(workdir, "case.peec"), "w") as f:
        f.write(str(g["peec"]))
    r = subprocess.run([EXE, "-n", "2", "case.peec"], cwd=workdir, capture_output=True, text=True, timeout=600)
    return g, r


def rows(text):
    lines = [l for l in text.splitlines() if l.strip()]
    return [l.split(",") for l in lines[1:]]


def cmp_zin(out, ref, tol, rtol=None):
    """|dZ| / |Z| per row; rtol: also the resistance on its own, |dR| <= rtol |R| + 1e-7 |Z|
    (the reference's own checks compare R of inductive structures to 0.1 %)."""
    a, b = rows(out), rows(ref)
    assert len(a) == len(b)
    err = 0.0
    for x, y in zip(a, b):
        assert x[0] == y[0] and float(x[1]) == float(y[1])
        za, zb = complex(float(x[2]), float(x[3])), complex(float(y[2]), float(y[3]))
        err = max(err, abs(za - zb) / abs(zb))
        if rtol is not None:
            assert abs(za.real - zb.real) <= rtol * abs(zb.real) + 1e-7 * abs(zb), (x, y)
    assert err <= tol, err
    return err


def cmp_groups(out, ref, key, val, tol, exact=()):
    """Rows grouped by the key columns; complex (or real) value columns compared relative to
    the group's largest reference entry; the exact columns (positions) must agree."""
    a, b = rows(out), rows(ref)
    assert len(a) == len(b)
    groups = {}
    for x, y in zip(a, b):
        assert [x[k] for k in key] == [y[k] for k in key]
        for k in exact:
            assert abs(float(x[k]) - float(y[k])) <= 1e-12 * max(1.0, abs(float(y[k])))
        va = np.array([float(x[k]) for k in val])
        vb = np.array([float(y[k]) for k in val])
        g = groups.setdefault(tuple(y[k] for k in key), [0.0, 0.0])
        g[0] = max(g[0], float(np.max(np.abs(va - vb))))
        g[1] = max(g[1], float(np.sqrt(np.sum(vb * vb))))
    err = max(d / m if m > 0 else d for d, m in groups.values())
    assert err <= tol, err
    return err


def cmp_touchstone(out, ref, tol):
    num = lambda t: [list(map(float, l.split())) for l in t.splitlines() if l.strip() and l[0] not in "!#"]
    a, b = np.array(num(out)), np.array(num(ref))
    assert a.shape == b.shape
    assert np.array_equal(a[:, 0], b[:, 0])
    err = float(np.max(np.abs(a[:, 1:] - b[:, 1:])))
    assert err <= tol, err
    return err


def cmp_far(out, ref, tol):
    a = np.array([list(map(float, r)) for r in rows(out)])
    b = np.array([list(map(float, r)) for r in rows(ref)])
    assert a.shape == b.shape and np.array_equal(a[:, :3], b[:, :3])
    err = 0.0
    for f in np.unique(b[:, 0]):
        m = b[:, 0] == f
        err = max(err, float(np.max(np.abs(a[m, 3:7] - b[m, 3:7])) / np.max(np.abs(b[m, 3:7]))))
        live = b[m, 7] > np.max(b[m, 7]) - 40          # dB columns printed to 1e-4 dB
        assert np.max(np.abs(a[m, 7:9][live] - b[m, 7:9][live])) <= 2e-3
    assert err <= tol, err
    return err


def cmp_captotal(out, ref):
    va = [float(l.split()[-2]) for l in out.splitlines() if "total capacitance" in l]
    vb = [float(l.split()[-2]) for l in ref.splitlines() if "total capacitance" in l]
    assert len(va) == len(vb)
    for x, y in zip(va, vb):
        assert abs(x - y) <= 2e-6 * abs(y), (x, y)


# ---------------------------------------------------------------- CPU
def test_dropin_fixtures_present():
    assert len(CASES) >= 20
    for c in CASES:
        g = np.load(os.path.join(GOLD, c + ".npz"))
        assert "zin.csv" in list(g["names"])


def test_dropin_binary_links_and_defines_the_entry_points():
    need_exe()
    lib = os.path.join(ROOT, "openpeec_b200", "libpeec_b200.so")
    ld = subprocess.run(["ldd", EXE], capture_output=True, text=True).stdout
    line = [l for l in ld.splitlines() if "libpeec_b200.so" in l]
    assert line and "not found" not in line[0], ld
    assert os.path.samefile(line[0].split("=>")[1].split("(")[0].strip(), lib)
    syms = subprocess.run(["nm", EXE], capture_output=True, text=True, check=True).stdout.split("\n")
    defined = {l.split()[-1] for l in syms if len(l.split()) == 3 and l.split()[1] in "TtDdBb"}
    undefined = {l.split()[-1] for l in syms if len(l.split()) == 2 and l.split()[0] == "U"}
    for s in SHIM:
        assert s in defined, s
    for s in REPLACED:
        assert s not in defined, s
    for s in ("pb_create", "pb_sweep_dist", "pb_lp_fill", "pb_pot_fill", "pb_lu_decomp", "pb_planewave"):
        assert s in undefined, s
    for s in ("input_data", "wire_build", "output_csv", "output_far", "output_tran", "zint_seg"):
        assert s in defined, s


def test_dropin_without_gpu_fails_loudly(tmp_path):
    need_exe()
    from openpeec_b200 import abi
    if abi.lib().pb_device_count() > 0:
        pytest.skip("a GPU is present")
    g, r = run("dipole_halfwave", str(tmp_path))
    assert r.returncode == 1
    assert "no host fallback" in r.stdout
    assert not (tmp_path / "zin.csv").exists()


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_dropin_matches_reference_cli(name, tmp_path):
    need_exe()
    g, r = run(name, str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:]
    log = (tmp_path / "peec.log").read_text()
    assert "normal end" in log
    comp = name.startswith("compress")
    tz = 1e-5 if comp else 1e-6
    report = {}
    for fn in [str(x) for x in g["names"]]:
        ref = str(g["f_" + fn])
        if fn == "captotal":
            cmp_captotal(log, ref)
            continue
        out = (tmp_path / fn).read_text()
        if fn == "zin.csv":
            report[fn] = cmp_zin(out, ref, tz, None if comp else 1e-3)
        elif fn.startswith("peec.s"):
            report[fn] = cmp_touchstone(out, ref, tz)
        elif fn == "pw.csv":
            report[fn] = cmp_zin(out, ref, tz)        # Voc real/imag in columns 2, 3
        elif fn == "dist.csv":
            report[fn] = cmp_groups(out, ref, key=(0, 1, 3), val=(7, 8), tol=tz, exact=(4, 5, 6))
        elif fn == "tran.csv":
            report[fn] = cmp_groups(out, ref, key=(0, 1, 2), val=(4,), tol=tz, exact=(3,))
        elif fn == "far.csv":
            report[fn] = cmp_far(out, ref, tz)
    print(name, report)
