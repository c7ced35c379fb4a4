"""Independent sources (vsource / isource): the extra solve of solve.c:392-396 with the
right-hand side of mna_rhs_sources (src/mna.c:471-489), reported as node voltages the way
print_vnode (src/solve.c:102-112) prints them.

Fixtures: tests/golden/src/*.npz, written by tests/golden/make_golden.py (--src-only) from
the reference's own lp_fill / pot_fill / mna_assemble / mna_rhs_sources / lu_decomp /
lu_solve (oracle/ref_harness.c rh_vnode): the series RLC sample with a 1 A / 30 deg current
source and with a 2 V voltage source, the half-wave dipole sample driven by a 1 A current
source across its gap, and the 16 x 8 plate + wire over ground (capacitance, retardation,
skin effect) with a 0.5 A / -45 deg current source.
"""
import numpy as np
import pytest

from conftest import load_golden

CASES = ["rlc_isource", "rlc_vsource", "dipole_isource", "cfg2_isource"]


def _src(fx):
    return [(int(v), int(a), int(b), amp, ph) for v, a, b, amp, ph in fx["sources"]]


def _rel(a, b):
    return np.abs(a - b).max(axis=1) / np.abs(b).max(axis=1)


def test_parser_reads_sources():
    from openpeec_b200 import abi, geometry
    p = geometry.parse_peec("OpenPEEC 1 0\nresistor = 1 0 50\nvsource = 1 0 2.0 15\n"
                            "isource = 0 1 0.5\nport = 1 0 50\nfrequency = 1e6 1e6 0\nend\n")
    assert p.sources == [(1, 1, 0, 2.0, 15.0), (0, 0, 1, 0.5, 0.0)]
    assert [l[0] for l in p.lumps] == [abi.PB_LUMP_R, abi.PB_LUMP_V]


def test_fixtures_known_answers():
    """The reference's node voltages obey the circuit's own answers: at the series
    resonance the RLC input is 50 ohm, so 1 A at 30 deg gives V1 = 50 V at 30 deg; an ideal
    2 V source fixes V1 = 2 V; 1 A across the dipole gap gives V1 - V2 = Z11 of the
    reference's own port sweep."""
    _, fx = load_golden("rlc_isource", "src")
    assert abs(fx["vnode"][0, 1] - 50 * np.exp(1j * np.pi / 6)) <= 1e-6 * 50
    _, fx = load_golden("rlc_vsource", "src")
    assert np.allclose(fx["vnode"][:, 1], 2.0, rtol=0, atol=1e-12)
    _, fx = load_golden("dipole_isource", "src")
    _, zf = load_golden("dipole_halfwave")
    for q, f in enumerate(fx["freqs"]):
        k = int(np.argmin(np.abs(zf["freqs"] - f)))
        assert zf["freqs"][k] == f
        z = zf["z"].reshape(len(zf["freqs"]), -1)[k, 0]
        assert abs((fx["vnode"][q, 1] - fx["vnode"][q, 2]) - z) <= 1e-9 * abs(z)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_sources_match_reference_fp64(name):
    from openpeec_b200 import abi, api
    prob, fx = load_golden(name, "src")
    with api.Context(prob) as ctx:
        vn, st = ctx.sources(fx["freqs"], sources=_src(fx), fill_prec=abi.PREC_FP64, lu=abi.LU_FP64)
    assert np.all(_rel(vn, fx["vnode"]) <= 1e-9), (_rel(vn, fx["vnode"]), st)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_sources_match_reference_mixed(name):
    """FP32 correction fill and tensor-core LU with FP64 refinement: 1e-6, the Zin bar."""
    from openpeec_b200 import abi, api
    prob, fx = load_golden(name, "src")
    with api.Context(prob) as ctx:
        vn, _ = ctx.sources(fx["freqs"], sources=_src(fx), fill_prec=abi.PREC_MIXED, lu=abi.LU_TC)
    assert np.all(_rel(vn, fx["vnode"]) <= 1e-6), _rel(vn, fx["vnode"])


@pytest.mark.gpu
def test_sources_reject_unmatched_voltage_source():
    """A voltage source must be the k-th PB_LUMP_V element of the problem (its branch row)."""
    from openpeec_b200 import abi, api
    prob, fx = load_golden("rlc_vsource", "src")
    with api.Context(prob) as ctx:
        with pytest.raises(api.PbError) as e:
            ctx.sources(fx["freqs"], sources=[(1, 2, 0, 1.0, 0.0)])
        assert e.value.code == abi.PB_ERR_ARG
        with pytest.raises(api.PbError) as e:
            ctx.sources(fx["freqs"], sources=[(0, 0, 1, 1.0, 0.0)])   # the V branch has no source
        assert e.value.code == abi.PB_ERR_ARG
