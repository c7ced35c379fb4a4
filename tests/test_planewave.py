"""Plane-wave incidence (the reference's planewave key): mna_rhs_planewave / pw_emf
(src/mna.c:408-468) and the open-circuit port voltages of solve() (src/solve.c:372-389).

Fixtures: tests/golden/pw/*.npz, written by tests/golden/make_golden.py from the
reference's own solve() on its sample inputs (dipole_pw, bent_pw, loop_pw, a loaded loop
with distribution = 1, and monopole_gp with a plane wave, for the ground-plane
reflection). Known answers follow the reference's checks:
  * half-wave dipole at resonance: receiving effective length |Voc|/E0 = lambda/pi
    (0.663793 m) within 1 %;
  * small loop, magnetic coupling: |Voc| = k E0 A = 8.383380e-3 V within 0.5 %, and Voc
    nearly imaginary (|Re Voc| / |Voc| <= 0.05).
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle.pyoracle import Oracle

PW = ["dipole_pw", "bent_pw", "loop_pw", "loop_pw_load", "mono_pw", "cfg5_small_pw"]
C0 = 2.99792458e8


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("name", PW)
def test_oracle_planewave_matches_reference(name):
    prob, fx = load_golden(name, "pw")
    voc, seg = Oracle(prob).planewave(fx["freqs"], fx["pw"])
    assert rel(voc, fx["voc"]) <= 1e-9, (name, rel(voc, fx["voc"]))
    if bool(fx["has_segi"]):
        assert rel(seg, fx["segipw"]) <= 1e-9


def test_oracle_dipole_effective_length():
    prob, fx = load_golden("dipole_pw", "pw")
    voc, _ = Oracle(prob).planewave(fx["freqs"][:1], fx["pw"])
    lam = C0 / fx["freqs"][0]
    assert abs(abs(voc[0, 0]) / fx["pw"][3] / (lam / np.pi) - 1) <= 0.01


def test_oracle_loop_faraday():
    prob, fx = load_golden("loop_pw", "pw")
    voc, _ = Oracle(prob).planewave(fx["freqs"], fx["pw"])
    v = voc[0, 0]
    assert abs(abs(v) / 8.383380e-3 - 1) <= 0.005
    assert abs(v.real) / abs(v) <= 0.05


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("name", PW)
def test_gpu_planewave_matches_reference(name):
    """FP64 path to round-off, mixed path (FP32 correction + tensor-core LU + FP64
    refinement) within 1e-6 of the reference's open-circuit voltages."""
    from openpeec_b200 import abi, api
    prob, fx = load_golden(name, "pw")
    with api.Context(prob) as ctx:
        v64, s64, st = ctx.planewave(fx["freqs"], fx["pw"], fill_prec=abi.PREC_FP64, lu=abi.LU_FP64,
                                     want_segi=True)
        vmx, smx, _ = ctx.planewave(fx["freqs"], fx["pw"], want_segi=True)
    assert rel(v64, fx["voc"]) <= 1e-9, (name, rel(v64, fx["voc"]), st)
    assert rel(vmx, fx["voc"]) <= 1e-6, (name, rel(vmx, fx["voc"]))
    if bool(fx["has_segi"]):
        assert rel(s64, fx["segipw"]) <= 1e-9
        assert rel(smx, fx["segipw"]) <= 1e-6


@pytest.mark.gpu
def test_gpu_planewave_known_answers():
    from openpeec_b200 import api
    prob, fx = load_golden("dipole_pw", "pw")
    with api.Context(prob) as ctx:
        voc, _ = ctx.planewave(fx["freqs"][:1], fx["pw"])
    lam = C0 / fx["freqs"][0]
    assert abs(abs(voc[0, 0]) / fx["pw"][3] / (lam / np.pi) - 1) <= 0.01
    prob, fx = load_golden("loop_pw", "pw")
    with api.Context(prob) as ctx:
        voc, _ = ctx.planewave(fx["freqs"], fx["pw"])
    assert abs(abs(voc[0, 0]) / 8.383380e-3 - 1) <= 0.005
    assert abs(voc[0, 0].real) / abs(voc[0, 0]) <= 0.05
