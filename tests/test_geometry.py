"""The host-side .peec reader + geometry builder against the reference's wire_build."""
import numpy as np
import pytest

from conftest import golden_names
from openpeec_b200 import configs, geometry

TEXT_CASES = ["cfg1_dipole_qs", "cfg2_small", "cfg3_small_0", "cfg3_small_1", "cfg3_small_2",
              "dipole_halfwave", "monopole_gp", "strip_dipole_ret", "plate_thick", "plate_cap"]


@pytest.mark.parametrize("name", [n for n in TEXT_CASES if n in golden_names()])
def test_builder_matches_reference(name, golden):
    ref, fx = golden(name)
    got = geometry.build(geometry.parse_peec(str(fx["peec"])))
    for fld in ("seg", "chg"):
        a, b = getattr(got, fld), getattr(ref, fld)
        assert len(a) == len(b)
        for f in a.dtype.names:
            if f != "pad_":
                assert np.array_equal(a[f], b[f]), (name, fld, f)
    assert np.array_equal(got.chgnode, ref.chgnode)
    assert got.maxid == ref.maxid
    assert got.port.tobytes() == ref.port.tobytes()
    assert (got.capacitance, got.retardation, got.skin, got.gp, got.gpz) == \
        (ref.capacitance, ref.retardation, ref.skin, ref.gp, ref.gpz)


def test_cfg2_sizes():
    p = geometry.build(geometry.parse_peec(configs.CFG2))
    assert (len(p.seg), len(p.chg)) == (4196, 2153)
    assert p.nfreq == 512 and abs(p.freq_at(511) - 2.56e9) < 1


def test_cfg3_instance_is_seeded():
    a, b = configs.cfg3_instance(7, 3), configs.cfg3_instance(7, 3)
    assert a == b
    p = geometry.build(geometry.parse_peec(a))
    assert 20 <= len(p.seg) - 1 <= 400 and p.nfreq == 64


def test_freq_at_log_and_linear():
    p = geometry.build(geometry.parse_peec(configs.CFG1))
    f = p.freqs()
    assert len(f) == 100 and f[0] == 1e7 and abs(f[-1] / 1e9 - 1) < 1e-14
    assert np.allclose(np.diff(np.log(f)), np.log(100) / 99)


def test_problem_roundtrip(tmp_path):
    p = geometry.build(geometry.parse_peec(configs.cfg2(8, 4, 4)))
    p.save(tmp_path / "p.npz")
    q = type(p).load(tmp_path / "p.npz")
    assert q.seg.tobytes() == p.seg.tobytes() and q.chg.tobytes() == p.chg.tobytes()
    assert (q.gp, q.gpz, q.nfreq, q.f1) == (p.gp, p.gpz, p.nfreq, p.f1)


def test_unsupported_keys_raise():
    with pytest.raises(NotImplementedError):
        geometry.build(geometry.parse_peec("OpenPEEC\ndisk = 0 0 0 0 0 1 0.01 1e-4 5.8e7 4 8\nport = 1 0 50\nend\n"))
