"""Config 5: the mixed conductor / dielectric full-wave structure over a ground plane with
a plane-wave excitation. Disks and quads take the Wilton polygon kernels, the dielectric
brick the dielectric branch impedance (src/mna.c:128-138) and its volume cells, the wave
the right-hand side of mna_rhs_planewave (src/mna.c:434-468); dense and compressed paths.

Fixtures (tests/golden/make_golden.py --cfg5-only, from the reference's own solve()):
  cfg5_small.npz, pw/cfg5_small_pw.npz   the scaled-down config 5 (two disks, one quad,
      a 6 x 6 x 2 brick; 750 current cells, N = 1108) at 10 MHz, 1.285 GHz and 2.56 GHz:
      port Z, sampled entries, plane-wave open-circuit voltage
  geom/cfg5_full.npz                     the reference builder's discretisation of the full
      config 5 (15 374 current cells, 6 925 charge cells; N = 22 299 in the reference's
      MNA), for the full-size runs
  geom/cfg5_full_ref.npz                 the reference CLI's port S11 (Z) and plane-wave Voc
      of the full config 5 at 1 GHz (make_golden.py --cfg5-full)
The dense Z and Voc of the small case against the reference are part of test_gpu_sweep.py
and test_planewave.py (golden lists); here the compressed path is held to them, and at
full size the two paths to each other.
"""
import os

import numpy as np
import pytest

from conftest import load_golden

HERE = os.path.dirname(os.path.abspath(__file__))

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


def test_small_compressed_port_z_matches_reference():
    from openpeec_b200 import abi, api
    prob, fx = load_golden("cfg5_small")
    with api.Context(prob) as ctx:
        z, st = ctx.sweep(fx["freqs"], fill_prec=abi.PREC_MIXED, compress=1, ctol=1e-6)
    assert st["hmat_far"] + st["hmat_near"] > 0
    e = rel(z, fx["z"])
    print("cfg5_small compressed Z vs reference", e, "GMRES its", st["gmres_its_max"])
    assert e <= 2e-5, e


def test_small_compressed_planewave_matches_reference():
    """The plane wave on the compressed path. Voc is a small difference of node potentials
    that the incident field drives in common, so it carries the ACA error amplified
    (1.7e-5 at the reference's tolerance 1e-6, where the port Z is at 2e-7); a tighter ACA
    tolerance takes it to the dense answer (2.4e-7 at 1e-8). The branch currents stay
    within ~2e-4 of their maximum at either tolerance: GMRES stops on the normwise residual
    of the full system (1e-10), which the charge rows (P ~ 1e10) dominate."""
    from openpeec_b200 import abi, api
    prob, fx = load_golden("cfg5_small_pw", "pw")
    with api.Context(prob) as ctx:
        voc_d, seg_d, _ = ctx.planewave(fx["freqs"], fx["pw"], fill_prec=abi.PREC_MIXED, want_segi=True)
        res = {}
        for tol in (1e-6, 1e-8):
            voc_c, seg_c, st = ctx.planewave(fx["freqs"], fx["pw"], fill_prec=abi.PREC_MIXED, compress=1,
                                             ctol=tol, want_segi=True)
            res[tol] = (rel(voc_c, fx["voc"]), rel(voc_c, voc_d), rel(seg_c, seg_d))
    print("cfg5_small compressed Voc (vs reference, vs dense, segment currents vs dense):", res)
    assert rel(voc_d, fx["voc"]) <= 1e-6
    assert max(res[1e-6][:2]) <= 5e-5 and res[1e-6][2] <= 5e-4, res
    assert max(res[1e-8][:2]) <= 2e-6 and res[1e-8][2] <= 5e-4, res


def test_full_size_dense_sweep_and_planewave():
    """Full config 5 (15 374 current cells, 6 925 charge cells) at 1 GHz on the dense
    batched mixed-precision path against the reference's own CLI on the same input
    (geom/cfg5_full_ref.npz: S11 to 10 digits, Z derived from it, Voc; a 50-minute dense
    reference solve): the port Z and the plane-wave Voc within 1e-6, refined to FP64
    backward error without any FP64 fall-back, and the plain FP64 path the same."""
    from openpeec_b200 import abi, api
    prob, _ = load_golden("cfg5_full", "geom")
    ref = np.load(os.path.join(HERE, "golden", "geom", "cfg5_full_ref.npz"))
    f = ref["freq"]
    pw = (30.0, 45.0, 1, 1.0, 0.0)
    with api.Context(prob) as ctx:
        zm, stm = ctx.sweep(f, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC)
        vm, _ = ctx.planewave(f, pw, fill_prec=abi.PREC_MIXED)
        zp, _ = ctx.sweep(f, fill_prec=abi.PREC_FP64, lu=abi.LU_FP64)
    print("cfg5 full 1 GHz: Z mixed", zm.ravel(), "plain", zp.ravel(), "reference", ref["z"], "Voc", vm.ravel(),
          "reference", ref["voc"], stm)
    assert stm["n_system"] == 15374 and stm["fp64_fallbacks"] == 0
    assert rel(zm.ravel(), ref["z"]) <= 1e-6 and rel(zp.ravel(), ref["z"]) <= 1e-6
    assert rel(vm.ravel(), ref["voc"]) <= 1e-6
    assert rel(zm, zp) <= 1e-6
