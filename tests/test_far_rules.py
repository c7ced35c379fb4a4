"""Accuracy of the lower-order product rules that the FP32 correction path takes for
separated ribbon pairs (CPU, numpy).

The reference integrates the retardation term (e^{-jkR} - 1)/R of a ribbon pair with the
4-point Gauss-Legendre rule in each of the four in-plane coordinates (ribbon_corr,
src/surface.c:134-178). The FP32 path replaces it by the 3-point rule where the centre
distance is >= 3 lmax and by the 2-point rule where it is >= 10 lmax, both only where
k lmax <= 0.1 (lmax: the pair's largest cell dimension). This test evaluates all three
rules on pairs of the benchmark plate (100 x 50 mm, 64 x 32 cells, 5 mm over the ground
plane), direct and image, at k lmax = 0.1, and checks the difference against the
reference's rule relative to |static| + |correction| of the entry: <= 1e-7 for the
2-point rule and <= 1e-8 for the 3-point rule, below the FP32 rounding of the
correction (~6e-8 of its own size).
"""
import numpy as np
import pytest

from openpeec_b200 import configs, geometry

RATIO2, RATIO3, KL = 10.0, 3.0, 0.1


def _plate():
    prob = geometry.build(geometry.parse_peec(configs.cfg2(64, 32, 2)))
    seg = prob.seg
    rib = np.where(np.asarray(seg["wid"]) > 0)[0]
    return seg, rib, float(prob.gpz)


def _frame(seg, i, mirror, gpz):
    a, b, w = (np.array(seg[k][i], float) for k in ("x1", "x2", "wv"))
    if mirror:
        a[2], b[2], w[2] = 2 * gpz - a[2], 2 * gpz - b[2], -w[2]
    ln = float(seg["len"][i])
    return (b - a) / ln, w / np.linalg.norm(w), 0.5 * (a + b)


def _corr(seg, i, j, mirror, gpz, kw, n):
    """L1 L2 / 16 * sum of W (e^{-jkR}-1)/R over the n^4 product rule (weights sum to 16)."""
    xg, wg = np.polynomial.legendre.leggauss(n)
    t1, w1, c1 = _frame(seg, i, False, gpz)
    t2, w2, c2 = _frame(seg, j, mirror, gpz)
    L1, W1, L2, W2 = (float(seg[k][q]) for q, k in ((i, "len"), (i, "wid"), (j, "len"), (j, "wid")))
    p1 = c1 + (0.5 * L1 * xg)[:, None, None] * t1 + (0.5 * W1 * xg)[None, :, None] * w1
    p2 = c2 + (0.5 * L2 * xg)[:, None, None] * t2 + (0.5 * W2 * xg)[None, :, None] * w2
    r = np.sqrt(((p2[None, None] - p1[:, :, None, None]) ** 2).sum(-1))
    W = np.einsum("a,b,c,d->abcd", wg, wg, wg, wg)
    return L1 * L2 / 16 * (W * (np.exp(-1j * kw * r) - 1) / r).sum()


def _pairs(seg, rib, gpz, lo, hi, count, seed):
    """Parallel ribbon pairs (direct or image) whose centre distance / lmax is in [lo, hi)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(20000):
        i, j = rng.choice(rib, 2, replace=False)
        mirror = bool(rng.integers(2))
        t1, _, c1 = _frame(seg, i, False, gpz)
        t2, _, c2 = _frame(seg, j, mirror, gpz)
        if abs(t1 @ t2) < 0.5:
            continue
        lmax = max(seg["len"][i], seg["len"][j], seg["wid"][i], seg["wid"][j])
        if lo <= np.linalg.norm(c2 - c1) / lmax < hi:
            out.append((i, j, mirror, float(lmax)))
            if len(out) == count:
                break
    return out


@pytest.mark.parametrize("n,lo,hi,tol", [(2, RATIO2, 14.0, 1e-7), (3, RATIO3, 5.0, 1e-8),
                                         (3, 5.0, RATIO2, 1e-8)])
def test_lower_order_rule_matches_reference_rule(n, lo, hi, tol):
    seg, rib, gpz = _plate()
    pairs = _pairs(seg, rib, gpz, lo, hi, 40, seed=n * 100 + int(lo))
    assert len(pairs) == 40
    worst = 0.0
    for i, j, mirror, lmax in pairs:
        kw = KL / lmax
        c4 = _corr(seg, i, j, mirror, gpz, kw, 4)
        cn = _corr(seg, i, j, mirror, gpz, kw, n)
        _, _, c1 = _frame(seg, i, False, gpz)
        _, _, c2 = _frame(seg, j, mirror, gpz)
        static = seg["len"][i] * seg["len"][j] / np.linalg.norm(c2 - c1)
        worst = max(worst, abs(cn - c4) / (abs(static) + abs(c4)))
    assert worst <= tol, worst


def test_two_point_rule_needs_the_wavenumber_bound():
    """Without k lmax <= 0.1 the 2-point rule is not good enough: at k lmax = 0.5 its error
    on the same far pairs exceeds 1e-7, which is why the FP32 path checks the bound."""
    seg, rib, gpz = _plate()
    worst = 0.0
    for i, j, mirror, lmax in _pairs(seg, rib, gpz, RATIO2, 14.0, 20, seed=7):
        kw = 0.5 / lmax
        c4 = _corr(seg, i, j, mirror, gpz, kw, 4)
        c2 = _corr(seg, i, j, mirror, gpz, kw, 2)
        _, _, a = _frame(seg, i, False, gpz)
        _, _, b = _frame(seg, j, mirror, gpz)
        worst = max(worst, abs(c2 - c4) / (abs(seg["len"][i] * seg["len"][j] / np.linalg.norm(b - a)) + abs(c4)))
    assert worst > 1e-7, worst
