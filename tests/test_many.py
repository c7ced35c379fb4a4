"""Many structures in one call (pb_sweep_many): config-3 style random thin-wire
structures of uneven size, each with its own frequency list, run concurrently on their
own streams from a size-ordered work queue. Each instance must give exactly what its own
pb_sweep gives (same kernels, same order), and the reference's Z on the config-3 golden
instances (tests/golden/cfg3_small_*.npz, from the reference's solve)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _instances(k, nmin=20, nmax=160):
    from openpeec_b200 import configs, geometry
    return [geometry.build(geometry.parse_peec(configs.cfg3_instance(7, i, nmin, nmax, nfreq=8))) for i in range(k)]


def test_many_equals_one_by_one():
    from openpeec_b200 import api
    probs = _instances(6)
    ctxs = [api.Context(p) for p in probs]
    try:
        freqs = [p.freqs()[i % 3::2] for i, p in enumerate(probs)]      # uneven lists
        zs = api.sweep_many(ctxs, freqs, nthreads=4)
        for c, f, z in zip(ctxs, freqs, zs):
            z1, _ = c.sweep(f)
            assert np.array_equal(z, z1)
    finally:
        for c in ctxs:
            c.close()


def test_many_matches_reference(golden):
    from openpeec_b200 import api
    cases = [golden("cfg3_small_%d" % i) for i in range(3)]
    ctxs = [api.Context(p) for p, _ in cases]
    try:
        zs = api.sweep_many(ctxs, [fx["freqs"] for _, fx in cases])
        for z, (_, fx) in zip(zs, cases):
            ref = fx["z"].reshape(z.shape)
            assert np.abs(z - ref).max() <= 1e-6 * np.abs(ref).max()
    finally:
        for c in ctxs:
            c.close()


def test_many_rejects_repeated_context():
    from openpeec_b200 import abi, api
    p = _instances(1)[0]
    with api.Context(p) as c:
        with pytest.raises(api.PbError) as e:
            api.sweep_many([c, c], [p.freqs()[:2], p.freqs()[:2]])
        assert e.value.code == abi.PB_ERR_ARG


@pytest.mark.parametrize("inst", [0, 7, 11])
def test_config3_instance_mixed_matches_fp64(inst):
    """Full config-3 instances (64 log frequencies 50 MHz-3 GHz): the mixed path (FP32
    correction, with the 4 x 8 rule on separated wire pairs, FP32 factorisation, FP64
    refinement) against the plain FP64 path (the reference's 8 x 8 rule, FP64 LU): Z within
    1e-6 at every frequency."""
    from openpeec_b200 import abi, api, configs, geometry
    prob = geometry.build(geometry.parse_peec(configs.cfg3_instance(0, inst)))
    f = prob.freqs()
    with api.Context(prob) as c:
        z64, _ = c.sweep(f, fill_prec=abi.PREC_FP64, lu=abi.LU_FP64)
        zmx, st = c.sweep(f, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC)
    e = np.abs(zmx - z64).reshape(len(f), -1).max(1) / np.abs(z64).reshape(len(f), -1).max(1)
    print("instance", inst, len(prob.seg), "segments, worst", e.max())
    assert e.max() <= 1e-6, (e.max(), int(e.argmax()))

