"""Pin the CPU oracle (oracle/peec_oracle.c) against the reference's own numbers.

The golden fixtures were written by tests/golden/make_golden.py from the reference's
lp_entry / pot_entry / solve. The oracle must reproduce them (it follows the same
algorithms in the same summation order), so the tolerances are round-off only.
"""
import numpy as np
import pytest

from conftest import golden_names, relerr
from oracle.pyoracle import Oracle, RefLib, ref_available

CASES = [n for n in golden_names() if n != "cfg2_full"]


@pytest.mark.parametrize("name", CASES)
def test_entries_match_reference(name, golden):
    prob, fx = golden(name)
    o = Oracle(prob)
    for ik, kw in enumerate(fx["kws"]):
        got = np.array([o.lp_entry(int(i), int(j), kw) for i, j in fx["lp_ij"]])
        assert relerr(got, fx["lp_v"][ik], 1e-300) <= 1e-13, name
        if len(fx["p_ij"]) and prob.capacitance:
            got = np.array([o.pot_entry(int(i), int(j), kw) for i, j in fx["p_ij"]])
            assert relerr(got, fx["p_v"][ik], 1e-300) <= 1e-13, name


@pytest.mark.parametrize("name", CASES)
def test_sweep_matches_reference(name, golden):
    prob, fx = golden(name)
    z = Oracle(prob).sweep(fx["freqs"])
    assert relerr(z, fx["z"], 1e-300) <= 1e-9, name


def test_oracle_lu_rule():
    """Pivot rule of lu.c:19-30: max |re|+|im|, first index on ties; zero pivot row."""
    a = np.array([[1, 2], [2, 4]], complex)
    r, lu, piv = Oracle.lu_decomp(a)
    assert r == 1 and piv[0] == 1
    a = np.array([[1 + 1j, 2], [-2j, 1]], complex)
    r, lu, piv = Oracle.lu_decomp(a)
    assert r == -1 and piv[0] == 0          # |1+1j| measure 2 == |-2j| measure 2 -> first


@pytest.mark.skipif(not ref_available(), reason="reference build not present")
@pytest.mark.parametrize("fn", ["wire_gp.peec", "plate_strip.peec", "twowire_cap.peec",
                                "loop_square.peec", "plate_skin_layers.peec"])
def test_oracle_vs_live_reference(fn):
    import os
    from oracle.pyoracle import reference_root
    root = reference_root()
    path = os.path.join(root, "data", "sample", fn) if root else ""
    if not root or not os.path.exists(path):
        pytest.skip("reference samples not present")
    r = RefLib(path)
    prob = r.problem()
    o = Oracle(prob)
    kw = 2 * np.pi * 1e9 / 2.99792458e8
    rng = np.random.default_rng(0)
    for _ in range(50):
        i, j = (int(v) for v in rng.integers(0, r.nseg, 2))
        assert o.lp_entry(i, j, kw) == r.lp_entry(i, j, kw)
    f = r.freqs()[:3]
    r.set_freqs(f[0], f[-1], len(f))
    assert relerr(o.sweep(r.freqs()), r.solve(), 1e-300) <= 1e-12
