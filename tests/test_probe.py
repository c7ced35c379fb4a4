"""Conditioning probe of the mixed-precision solve (pb_sweep_stats.probe_fallbacks).

A refined solution at FP64 backward error is not accurate when the system is
ill-conditioned. The reference's "quad sheet R vs plate (HF)" pair is such a case: a
0.2 m copper sheet between 1e-9 ohm bus resistors at 1 GHz with skin effect, where the
port resistance is 6e-5 of |Z| and cond(A) ~ 4e13. FP32 LU + FP64 refinement converges
(backward error 7e-15) to R = 0.00514 ohm; the reference's FP64 elimination gives
0.0205640 ohm, as does the same structure meshed with quad panels. The probe perturbs each
refined system by its remaining backward error and sends frequencies whose port voltages
move by more than 2.5e-7 relative to the FP64 factorisation, whose pivot order is the
reference's.

Fixtures: tests/golden/dropin/sk_plate_hf.npz and dipole_halfwave.npz (the reference
CLI's zin.csv and the input text).
"""
import os

import numpy as np
import pytest

from openpeec_b200 import geometry

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "dropin")


def case(name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    prob = geometry.build(geometry.parse_peec(str(g["peec"])))
    rows = [l.split(",") for l in str(g["f_zin.csv"]).splitlines()[1:] if l.strip()]
    f = np.array([float(r[1]) for r in rows])
    z = np.array([complex(float(r[2]), float(r[3])) for r in rows])
    return prob, f, z


def test_probe_fixture_builds_on_cpu():
    prob, f, z = case("sk_plate_hf")
    assert prob.skin == 1 and len(prob.seg) == 144 and f[0] == 1e9
    assert abs(z[0].real / abs(z[0])) < 1e-4          # R is a tiny part of |Z|


@pytest.mark.gpu
def test_probe_sends_ill_conditioned_sheet_to_fp64():
    from openpeec_b200 import abi, api
    prob, f, zref = case("sk_plate_hf")
    with api.Context(prob) as ctx:
        zm, st = ctx.sweep(f, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC)
        zp, _ = ctx.sweep(f, fill_prec=abi.PREC_FP64, lu=abi.LU_FP64)
    print("probe", st["probe_max"], st["probe_fallbacks"], zm.ravel(), zref)
    assert st["probe_fallbacks"] == 1 and st["fp64_fallbacks"] >= 1
    assert st["probe_max"] > 2.5e-7
    assert abs(zm[0, 0, 0] - zp[0, 0, 0]) <= 1e-9 * abs(zp[0, 0, 0])
    assert abs(zm[0, 0, 0].real - zref[0].real) <= 1e-3 * abs(zref[0].real)


@pytest.mark.gpu
def test_probe_quiet_on_well_conditioned_sweep():
    from openpeec_b200 import abi, api
    prob, f, zref = case("dipole_halfwave")
    with api.Context(prob) as ctx:
        zm, st = ctx.sweep(f, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC)
    print("probe", st["probe_max"], st["probe_fallbacks"])
    assert st["probe_fallbacks"] == 0 and st["probe_max"] < 2.5e-7
    assert np.max(np.abs(zm[:, 0, 0] - zref) / np.abs(zref)) <= 1e-6
