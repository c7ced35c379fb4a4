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


# ---------------------------------------------------------------- thin wires
# The reference integrates the retardation term of a wire pair over nsub = 2 + k lmax
# sub-intervals of each segment with the 8-point rule in each (gauss_kernel mode 1,
# src/partial.c:61-99, 166-173), R = sqrt(|p2 - p1|^2 + a^2) with the pair's mean radius
# a. The FP32 path takes 4 points along the whole first segment and 8 along the whole
# second where the centre distance is >= 3 lmax and k lmax <= 0.5.
WRATIO, WKL = 3.0, 0.5


def _wire_corr(x1, x2, y1, y2, a, kw, n1, n2, nsub=1):
    """len1 len2 / (4 nsub^2) * sum of W (e^{-jkR}-1)/R over the composite n1 x n2
    Gauss-Legendre rule on nsub x nsub sub-intervals."""
    g1, w1 = np.polynomial.legendre.leggauss(n1)
    g2, w2 = np.polynomial.legendre.leggauss(n2)
    u = ((np.arange(nsub)[:, None] + 0.5 * (1 + g1)) / nsub).ravel()
    v = ((np.arange(nsub)[:, None] + 0.5 * (1 + g2)) / nsub).ravel()
    wu, wv = np.tile(w1, nsub), np.tile(w2, nsub)
    p1 = x1 + u[:, None] * (x2 - x1)
    p2 = y1 + v[:, None] * (y2 - y1)
    r = np.sqrt(((p2[None] - p1[:, None]) ** 2).sum(-1) + a * a)
    l1, l2 = np.linalg.norm(x2 - x1), np.linalg.norm(y2 - y1)
    return l1 * l2 / (4 * nsub * nsub) * (np.outer(wu, wv) * (np.exp(-1j * kw * r) - 1) / r).sum()


def test_wire_far_rule_matches_reference_rule():
    """Segment pairs of config-3 random polylines (2-8 mm steps, radius 0.1-2 mm) at centre
    distance 3-40 lmax, k lmax = 0.5 (the bound): the 4 x 8 rule agrees with the
    reference's 2 x 2 sub-intervals of 8 x 8 points to < 1e-9 of |static| + |correction|,
    far below the FP32 rounding (~6e-8)."""
    from openpeec_b200 import configs, geometry
    worst, n = 0.0, 0
    for inst in range(4):
        prob = geometry.build(geometry.parse_peec(configs.cfg3_instance(3, inst, 60, 120, nfreq=2)))
        seg = prob.seg
        x1, x2 = np.asarray(seg["x1"], float), np.asarray(seg["x2"], float)
        ln = np.asarray(seg["len"], float)
        rad = np.asarray(seg["aL"], float) if "aL" in seg.dtype.names else np.full(len(ln), 1e-3)
        rng = np.random.default_rng(inst)
        for _ in range(3000):
            i, j = rng.choice(len(ln), 2, replace=False)
            lmax = max(ln[i], ln[j])
            d = np.linalg.norm(0.5 * (x1[j] + x2[j]) - 0.5 * (x1[i] + x2[i]))
            if not (WRATIO <= d / lmax < 40):
                continue
            kw = WKL / lmax
            a = 0.5 * (rad[i] + rad[j])
            c88 = _wire_corr(x1[i], x2[i], x1[j], x2[j], a, kw, 8, 8, nsub=2 + int(kw * lmax))
            c48 = _wire_corr(x1[i], x2[i], x1[j], x2[j], a, kw, 4, 8)
            static = ln[i] * ln[j] / d
            worst = max(worst, abs(c48 - c88) / (static + abs(c88)))
            n += 1
    assert n > 1000, n
    assert worst <= 1e-9, worst
