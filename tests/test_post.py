"""Post-processing of the sweep: far field (output_far, src/farfield.c:42-182) and transient
synthesis (tran_synth / output_tran, src/transient.c:73-177).

Fixtures: tests/golden/post/*.npz, written by tests/golden/make_golden.py (--post-only):
the reference's sweep followed by its own writers, parsed back from far.csv / tran.csv
(10 significant digits), with the inputs those writers read (port-1 currents, Zin, S,
Voc). Far field: the half-wave dipole sample dipole_ff (36 x 24 directions), the monopole
over ground (upper hemisphere with image currents) and the 16 x 8 plate + wire over
ground. Transient: the resistor TDR sample, the plane-wave loop sample (Voc waveform) and
the plate + wire over ground on a 32-point k*df sweep (S11 waveform, 60 dB pulse).

CPU: the numpy oracle (oracle/post_oracle.py) against those writers, and the samples' own
known answers (dipole directivity 2.117 dBi and efficiency 1; TDR y = S11 x; the pulse is
the analytic Gaussian). GPU: pb_farfield and pb_transient against the same fixtures, and
the far field of the library's own sweep currents against the reference's pattern.
"""
import os
import sys

import numpy as np
import pytest

from conftest import load_golden

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import post_oracle as po  # noqa: E402

FF = ["ff_dipole", "ff_monopole_gp", "ff_plate_gp"]
TR = ["tran_tdr", "tran_loop_pw", "tran_plate"]


def _ff_ref(fx):
    nf = len(fx["freqs"])
    nth = len(np.unique(fx["ff_th"])) - 1
    nph = len(np.unique(fx["ff_ph"]))
    r = lambda k: fx[k].reshape(nf, (nth + 1) * nph)
    return nth, nph, r("et"), r("ep"), r("d_dbi"), r("g_dbi")


def _ff_inputs(fx):
    return fx["segi"][:, 0, :], fx["zin"][0]


def _check_ff(fx, et, ep, d, g, tol):
    _, _, ret, rep, rd, rg = _ff_ref(fx)
    for q in range(len(fx["freqs"])):
        scale = max(np.abs(ret[q]).max(), np.abs(rep[q]).max())
        assert np.abs(et[q] - ret[q]).max() <= tol * scale
        assert np.abs(ep[q] - rep[q]).max() <= tol * scale
        live = rd[q] > -100
        assert np.abs(d[q][live] - rd[q][live]).max() <= 1e-3
        assert np.abs(g[q][live] - rg[q][live]).max() <= 1e-3


def _att(fx):
    for line in str(fx["peec"]).splitlines():
        if line.startswith("transient"):
            a = line.split("=")[1].split()
            return float(a[1]) if len(a) > 1 else 40.0
    raise ValueError("no transient key")


def _tr_signals(fx):
    """(reference waveforms per label, responses h per label) in the writer's order."""
    typ, ii, jj, y = fx["tr_type"], fx["tr_i"], fx["tr_j"], fx["tr_y"]
    labels, ref, h = [], {}, {}
    for t, i, j in zip(typ, ii, jj):
        key = (str(t), int(i), int(j))
        if key not in ref:
            labels.append(key)
            ref[key] = []
    for t, i, j, v in zip(typ, ii, jj, y):
        ref[(str(t), int(i), int(j))].append(v)
    for t, i, j in labels:
        if t == "S":
            h[(t, i, j)] = fx["smat"][:, i - 1, j - 1]
        elif t == "V":
            h[(t, i, j)] = fx["voc"][i - 1]
    return labels, {k: np.array(v) for k, v in ref.items()}, h


@pytest.mark.parametrize("name", FF)
def test_farfield_oracle_pinned(name):
    prob, fx = load_golden(name, "post")
    nth, nph, *_ = _ff_ref(fx)
    segi, zin = _ff_inputs(fx)
    o = po.farfield(prob.seg, fx["freqs"], segi, zin, nth, nph, prob.gp, prob.gpz)
    _check_ff(fx, o["et"], o["ep"], o["d_dbi"], o["g_dbi"], 5e-9)


def test_farfield_dipole_known_answers():
    """dipole_ff.peec: directivity of the near-sinusoidal current 1.628 (2.117 dBi) within
    1.5 %, radiation efficiency Prad / Pin = 1 within 0.5 % (copper loss 4e-5 of Rin)."""
    prob, fx = load_golden("ff_dipole", "post")
    nth, nph, _, _, rd, _ = _ff_ref(fx)
    assert abs(10 ** (rd.max() / 10) / 1.628 - 1) <= 0.015
    segi, zin = _ff_inputs(fx)
    o = po.farfield(prob.seg, fx["freqs"], segi, zin, nth, nph)
    assert abs(o["prad"][0] / o["pin"][0] - 1) <= 0.005


@pytest.mark.parametrize("name", TR)
def test_transient_oracle_pinned(name):
    prob, fx = load_golden(name, "post")
    f = fx["freqs"]
    labels, ref, h = _tr_signals(fx)
    x, y, dt = po.transient(f[0], f[-1], len(f), _att(fx), [h[k] for k in labels if k[0] != "X"])
    assert np.allclose(ref[("X", 0, 0)], x, rtol=0, atol=2e-9 * np.abs(x).max())
    for k, yy in zip([k for k in labels if k[0] != "X"], y):
        assert np.abs(ref[k] - yy).max() <= 2e-9 * max(np.abs(ref[k]).max(), 1e-300) + 1e-12, k


def test_transient_tdr_known_answers():
    """tdr_resistor.peec (R = 150 ohm on a 50 ohm port): S11 = 0.5 at every frequency, so
    y(t) = 0.5 x(t) exactly; the pulse is the analytic Gaussian (peak 1) within 5e-3."""
    _, fx = load_golden("tran_tdr", "post")
    labels, ref, _ = _tr_signals(fx)
    x, y = ref[("X", 0, 0)], ref[("S", 1, 1)]
    assert np.abs(y - 0.5 * x).max() <= 1e-9
    f1 = fx["freqs"][-1]
    sigma = np.sqrt(40 * np.log(10.0) / (20 * 2 * np.pi ** 2)) / f1
    t = np.arange(len(x)) / (2 * f1)
    assert np.abs(x - np.exp(-(t - 4 * sigma) ** 2 / (2 * sigma ** 2))).max() <= 5e-3


@pytest.mark.gpu
@pytest.mark.parametrize("name", FF)
def test_farfield_gpu_matches_reference(name):
    from openpeec_b200 import api
    prob, fx = load_golden(name, "post")
    nth, nph, *_ = _ff_ref(fx)
    segi, zin = _ff_inputs(fx)
    with api.Context(prob) as ctx:
        o = ctx.farfield(fx["freqs"], segi, zin, nth, nph)
    _check_ff(fx, o["et"], o["ep"], o["d_dbi"], o["g_dbi"], 5e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ff_dipole", "ff_plate_gp"])
def test_farfield_of_own_sweep(name):
    """End to end: the library's own mixed-precision sweep currents through pb_farfield
    give the reference's pattern (D, G within 1e-3 dB; E within 1e-5)."""
    from openpeec_b200 import api
    prob, fx = load_golden(name, "post")
    nth, nph, *_ = _ff_ref(fx)
    with api.Context(prob) as ctx:
        z, segi, _ = ctx.sweep(fx["freqs"], want_segi=True)
        o = ctx.farfield(fx["freqs"], segi, z[:, 0, 0], nth, nph)
    _, _, ret, rep, rd, rg = _ff_ref(fx)
    for q in range(len(fx["freqs"])):
        scale = np.abs(ret[q]).max()
        assert np.abs(o["et"][q] - ret[q]).max() <= 1e-5 * scale
        live = rd[q] > -100
        assert np.abs(o["d_dbi"][q][live] - rd[q][live]).max() <= 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("name", TR)
def test_transient_gpu_matches_reference(name):
    from openpeec_b200 import api
    _, fx = load_golden(name, "post")
    f = fx["freqs"]
    labels, ref, h = _tr_signals(fx)
    sig = [k for k in labels if k[0] != "X"]
    x, y, dt = api.transient(f[0], f[-1], len(f), [h[k] for k in sig], _att(fx))
    assert abs(dt - 1 / (2 * f[-1])) <= 1e-25
    assert np.abs(ref[("X", 0, 0)] - x).max() <= 2e-9 * np.abs(x).max()
    for k, yy in zip(sig, y):
        assert np.abs(ref[k] - yy).max() <= 2e-9 * max(np.abs(ref[k]).max(), 1e-300) + 1e-12, k


def test_transient_rejects_log_sweep():
    """tran_check (transient.c:40-66): the sweep must be f_k = k df; checked before any
    device work, so this runs without a GPU."""
    from openpeec_b200 import abi, api
    with pytest.raises(api.PbError) as e:
        api.transient(1e6, 1e9, 16, np.ones((1, 16)))
    assert e.value.code == abi.PB_ERR_ARG
