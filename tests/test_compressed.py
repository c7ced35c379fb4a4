"""Compressed sweep (the reference's compression = 1): H-matrix with ACA far blocks,
leaf-block + circuit-Schur preconditioner, matrix-free GMRES (hmatrix.c, precond.c,
iterative.c:285-354, solve.c:251-294).

Fixtures: tests/golden/comp/*.npz, written by tests/golden/make_golden.py from the
reference's own compressed solve and its dense solve of the same input (compression key
removed): the sample compress_wire (200-segment wire) and compress_plate (16 x 16 sheet
with mixed cell orientations, the case that needs ACA's restarts from unrepresented
rows), a 12 x 12 x 4 volume-bar stack with retardation at 1 MHz and 2 GHz, the sample
compress_cap (capacitive sheet: charge unknowns, H-matrices of Lp and P, two-block
preconditioner) and the 16 x 8 plate + wire over ground with capacitance, retardation and
skin effect.

Bar: Z within 1e-5 of the reference's compressed Z (the same algorithm on entries equal
to ~1e-15, so the same blocks and nearly the same low-rank factors), and within the
reference's own compression error plus 2e-5 of its dense Z (the reference's ACA at tol 1e-6
leaves 2.7e-7 on the plate but 1.6e-3 on the bar stack). Known answers as the
reference's checks (peec_check.sh, compress wire): L = 1.320380e-6 H within 0.1 %,
R = 5.48810e-3 ohm within 0.5 %.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu
CASES = ["compress_wire", "compress_plate", "bars_small", "compress_cap", "cap_retarded"]


def rel(a, b):
    return np.abs(a - b).reshape(len(a), -1).max(1) / np.abs(b).reshape(len(b), -1).max(1)


@pytest.mark.parametrize("name", CASES)
def test_compressed_matches_reference(name):
    from openpeec_b200 import abi, api
    prob, fx = load_golden(name, "comp")
    with api.Context(prob) as ctx:
        z, st = ctx.sweep(fx["freqs"], fill_prec=abi.PREC_FP64, lu=abi.LU_FP64, compress=1)
    assert st["hmat_far"] + st["hmat_near"] > 0
    e_ref = rel(z, fx["z"])
    e_den = rel(z, fx["z_dense"])
    ref_err = rel(fx["z"], fx["z_dense"])
    assert np.all(e_ref <= 1e-5), (name, e_ref, st)
    # triangle inequality: within the reference's own compression error plus the 1e-5 bar
    assert np.all(e_den <= ref_err + 2e-5), (name, e_den, ref_err)


@pytest.mark.parametrize("name,prec", [("compress_plate", "fp64"), ("bars_small", "mixed"),
                                       ("cap_retarded", "mixed"), ("compress_wire", "fp64")])
def test_on_demand_aca_equals_dense_fill(name, prec):
    """ACA with entries evaluated on demand (rows, columns and dense blocks from the geometry,
    no N x N fill) against the dense fill followed by ACA over it: the entries are the same
    bits, so the blocks, ranks and Z agree to rounding; the on-demand build evaluates a
    fraction of the N^2 entries per frequency."""
    from openpeec_b200 import abi, api
    prob, fx = load_golden(name, "comp")
    fp = abi.PREC_FP64 if prec == "fp64" else abi.PREC_MIXED
    with api.Context(prob) as ctx:
        zd, sd = ctx.sweep(fx["freqs"], fill_prec=fp, compress=1, aca_dense=1)
        zo, so = ctx.sweep(fx["freqs"], fill_prec=fp, compress=1, aca_dense=0)
    n, nf = len(prob.seg), len(fx["freqs"])
    for k in ("hmat_far", "hmat_near", "hmat_max_rank", "hmat_dense_far"):
        assert sd[k] == so[k], (k, sd[k], so[k])
    # dense: N^2 per fill (once without retardation, else per frequency)
    assert float(n) * n <= sd["hmat_entries"] <= float(n) * n * nf
    assert so["hmat_entries"] > 0
    assert np.all(rel(zo, zd) <= 1e-12), rel(zo, zd)
    print(name, prec, "on-demand entries %.3g of %.3g dense" % (so["hmat_entries"], sd["hmat_entries"]))


def test_compressed_mixed_fill_agrees():
    from openpeec_b200 import abi, api
    prob, fx = load_golden("compress_plate", "comp")
    with api.Context(prob) as ctx:
        z64, _ = ctx.sweep(fx["freqs"], fill_prec=abi.PREC_FP64, compress=1)
        zmx, _ = ctx.sweep(fx["freqs"], fill_prec=abi.PREC_MIXED, compress=1)
    assert np.all(rel(zmx, z64) <= 1e-6)


def test_compressed_wire_known_answer():
    from openpeec_b200 import api
    prob, fx = load_golden("compress_wire", "comp")
    with api.Context(prob) as ctx:
        z, _ = ctx.sweep(fx["freqs"], compress=1)
    w = 2 * np.pi * fx["freqs"][0]
    assert abs(z[0, 0, 0].imag / w / 1.320380e-6 - 1) <= 1e-3
    assert abs(z[0, 0, 0].real / 5.48810e-3 - 1) <= 5e-3


def test_compressed_capacitive_exact_at_small_scale(golden):
    """With every block near (no approximation at this size) the charge formulation of the
    compressed path is the dense system itself: Z equals the dense sweep to round-off
    (the reference's 'compress cap exact' check, peec_check.sh:754-771)."""
    from openpeec_b200 import abi, api
    prob, fx = golden("dipole_halfwave")
    with api.Context(prob) as ctx:
        zc, st = ctx.sweep(fx["freqs"], fill_prec=abi.PREC_FP64, lu=abi.LU_FP64, compress=1)
        zd, _ = ctx.sweep(fx["freqs"], fill_prec=abi.PREC_FP64, lu=abi.LU_FP64)
    assert st["hmat_far"] == 0
    assert np.all(rel(zc, zd) <= 1e-9), rel(zc, zd)


def test_compressed_large_circuit_schur():
    """A sheet with more than 1024 circuit unknowns (32 x 32 x 1: 1089 nodes) applies the
    circuit Schur complement as an explicit inverse (one matrix-vector product per GMRES
    step). GMRES must converge in the first cycle as with the substitution, and Z must agree
    with the dense sweep of the same structure within the compression error (ACA tolerance
    1e-6)."""
    from openpeec_b200 import abi, api, configs, geometry
    prob = geometry.build(geometry.parse_peec(configs.cfg4(32, 32, 1, 2)))
    with api.Context(prob) as ctx:
        assert ctx.nnode > 1024
        zc, st = ctx.sweep([1e6, 1e9], fill_prec=abi.PREC_FP64, compress=1)
        zd, _ = ctx.sweep([1e6, 1e9], fill_prec=abi.PREC_FP64, lu=abi.LU_FP64, compress=0)
    assert 0 < st["gmres_its_max"] <= 60, st["gmres_its_max"]
    assert np.all(rel(zc, zd) <= 1e-4), rel(zc, zd)


@pytest.mark.parametrize("name", ["compress_plate", "bars_small", "compress_cap"])
def test_two_level_matches_reference(name):
    """The two-level preconditioner changes the iteration count, never the answer: Z within
    1e-5 of the reference's compressed Z, as with the plain preconditioner."""
    from openpeec_b200 import abi, api
    prob, fx = load_golden(name, "comp")
    with api.Context(prob) as ctx:
        z, st = ctx.sweep(fx["freqs"], fill_prec=abi.PREC_FP64, lu=abi.LU_FP64, compress=1, pc_coarse=1)
    assert st["pc_coarse_n"] > 0
    assert np.all(rel(z, fx["z"]) <= 1e-5), (name, rel(z, fx["z"]), st)


def test_two_level_cuts_iterations():
    """Bar stack 20 x 12 x 4 (config-4 family): the coarse correction over divergence-free
    leaf currents at least halves the GMRES iterations of the plain leaf + Schur
    preconditioner (measured 23 -> 12 and 30 -> 15), with Z unchanged at the GMRES
    tolerance."""
    from openpeec_b200 import api, configs, geometry
    prob = geometry.build(geometry.parse_peec(configs.cfg4(20, 12, 4, 2)))
    with api.Context(prob) as ctx:
        for f in (1e6, 1e9):
            z0, s0 = ctx.sweep([f], compress=1)
            z1, s1 = ctx.sweep([f], compress=1, pc_coarse=1)
            assert np.abs(z1 - z0).max() <= 1e-8 * np.abs(z0).max()
            assert 2 * s1["gmres_its_max"] <= s0["gmres_its_max"] + 1, (f, s0["gmres_its_max"], s1["gmres_its_max"])


def test_two_level_large_circuit():
    """A sheet with 1089 nodes: the coarse set-up then applies the explicit inverse of the
    circuit Schur complement as one matrix product per batch of coarse vectors. Same Z as
    the plain preconditioner, fewer iterations."""
    from openpeec_b200 import api, configs, geometry
    prob = geometry.build(geometry.parse_peec(configs.cfg4(32, 32, 1, 2)))
    with api.Context(prob) as ctx:
        assert ctx.nnode > 1024
        z0, s0 = ctx.sweep([1e9], compress=1)
        z1, s1 = ctx.sweep([1e9], compress=1, pc_coarse=1)
    assert np.abs(z1 - z0).max() <= 1e-8 * np.abs(z0).max()
    assert s1["gmres_its_max"] < s0["gmres_its_max"], (s0["gmres_its_max"], s1["gmres_its_max"])


def test_config4_full_size_matches_reference():
    """Config 4 at full size (96 x 96 x 4 bar stack, 74 496 current cells) at 100 MHz on the
    compressed path against the reference's own compressed solve of the same input
    (golden comp/cfg4_full.npz: Zin to 10 digits, its block counts and GMRES iterations;
    make_golden.py --cfg4-only). Same cluster tree and admissibility, so the same block
    partition; Z within 1e-5 as for the smaller compressed cases."""
    import os
    from openpeec_b200 import abi, api, geometry
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "comp", "cfg4_full.npz"))
    prob = geometry.build(geometry.parse_peec(str(g["peec"])))
    assert len(prob.seg) == int(g["ncell"])
    with api.Context(prob) as ctx:
        z, st = ctx.sweep(g["freqs"], fill_prec=abi.PREC_MIXED, compress=1, ctol=1e-6)
    e = float(np.max(np.abs(z - g["z"]) / np.abs(g["z"])))
    print("cfg4 full: Z", z.ravel(), "reference", g["z"].ravel(), "rel", e, "GMRES", st["gmres_its_max"],
          "reference GMRES", float(g["gmres_its"]), "blocks", st["hmat_far"], st["hmat_near"])
    assert (st["hmat_far"], st["hmat_near"]) == (int(g["far"]), int(g["near"]))
    assert e <= 1e-5, e
    # entries on demand: well under the N^2 of a dense fill
    assert 0 < st["hmat_entries"] < 0.25 * float(len(prob.seg)) ** 2 * len(g["freqs"]), st["hmat_entries"]
