"""Parity of the CUDA partial-element fill (Lp, P) with the oracle and the reference.

Tolerances (per entry, relative to |entry|):
  FP64 path  (static + correction in FP64)            : 1e-9
  mixed path (FP64 static, FP32 retardation correction): 1e-5  (the stated Lp/P bar)
The FP64 bar is round-off: CUDA's asinh / atan2 / log differ from the host libm in the
last bit, and the closed forms (rectangle potential, Hoer-Love, Wilton edge sums) cancel
up to ~6 digits, so identical formulas agree to ~1e-10, not to the last bit.
"""
import numpy as np
import pytest

from conftest import golden_names, relerr
from openpeec_b200 import abi, api
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu
CASES = [n for n in golden_names() if n not in ("cfg2_full", "rlc_series")]
C0 = 2.99792458e8


def entry_err(got, ref, prec=abi.PREC_FP64):
    """Relative error per entry. FP64 path: entries below 1e-9 of the matrix scale are
    compared absolutely. Mixed path: entries below 1e-4 of the matrix scale are compared
    normwise (relative to 1e-4 of the scale): such entries are the near-cancellation of
    the direct and ground-plane-image terms (e.g. P between distant cells 5 mm above the
    ground), and each term carries its own ~1e-7 FP32 error, so their relative error is
    not a property of the fill but of the cancellation."""
    scale = np.max(np.abs(ref)) if ref.size else 1.0
    return relerr(got, ref, (1e-9 if prec == abi.PREC_FP64 else 1e-4) * scale)


@pytest.mark.parametrize("name", CASES)
def test_lp_matches_oracle(name, golden):
    prob, fx = golden(name)
    o = Oracle(prob)
    with api.Context(prob) as ctx:
        for kw in fx["kws"]:
            ref = o.lp_fill(kw)
            assert entry_err(ctx.lp_fill(kw, abi.PREC_FP64), ref) <= 1e-9, (name, kw)
            assert entry_err(ctx.lp_fill(kw, abi.PREC_MIXED), ref, abi.PREC_MIXED) <= 1e-5, (name, kw)


@pytest.mark.parametrize("name", [n for n in CASES if n not in ("plate_thick", "quad_square")])
def test_pot_matches_oracle(name, golden):
    prob, fx = golden(name)
    if not prob.capacitance:
        pytest.skip("no capacitive cells")
    o = Oracle(prob)
    with api.Context(prob) as ctx:
        for kw in fx["kws"]:
            ref = o.pot_fill(kw)
            assert entry_err(ctx.pot_fill(kw, abi.PREC_FP64), ref) <= 1e-9, (name, kw)
            assert entry_err(ctx.pot_fill(kw, abi.PREC_MIXED), ref, abi.PREC_MIXED) <= 1e-5, (name, kw)


@pytest.mark.parametrize("name", CASES)
def test_entries_match_reference_golden(name, golden):
    prob, fx = golden(name)
    with api.Context(prob) as ctx:
        for ik, kw in enumerate(fx["kws"]):
            lp = ctx.lp_fill(kw, abi.PREC_MIXED)
            got = np.array([lp[i, j] for i, j in fx["lp_ij"]])
            scale = np.max(np.abs(lp))
            assert relerr(got, fx["lp_v"][ik], 1e-4 * scale) <= 1e-5, name
            if prob.capacitance and len(fx["p_ij"]):
                pm = ctx.pot_fill(kw, abi.PREC_MIXED)
                got = np.array([pm[i, j] for i, j in fx["p_ij"]])
                assert relerr(got, fx["p_v"][ik], 1e-4 * np.max(np.abs(pm))) <= 1e-5, name


def test_mixed_fill_normwise_error(golden):
    """Normwise entry error of the mixed fill: max |dL| / max |L| <= 1e-7 (same for P)."""
    prob, fx = golden("cfg2_small")
    o = Oracle(prob)
    kw = fx["kws"][1]
    with api.Context(prob) as ctx:
        for got, ref in ((ctx.lp_fill(kw), o.lp_fill(kw)), (ctx.pot_fill(kw), o.pot_fill(kw))):
            assert np.max(np.abs(got - ref)) <= 1e-7 * np.max(np.abs(ref))


def test_fill_is_deterministic(golden):
    prob, fx = golden("cfg2_small")
    kw = fx["kws"][1]
    with api.Context(prob) as ctx:
        a = ctx.lp_fill(kw, abi.PREC_MIXED)
        b = ctx.lp_fill(kw, abi.PREC_MIXED)
    assert a.tobytes() == b.tobytes()


def test_lp_symmetric_and_positive_self(golden):
    prob, _ = golden("cfg2_small")
    with api.Context(prob) as ctx:
        lp = ctx.lp_fill(2 * np.pi * 1e9 / C0, abi.PREC_MIXED)
    assert np.array_equal(lp, lp.T)
    assert np.all(np.diag(lp).real > 0)
