"""CPU oracle of the sweep's post-processing (test infrastructure only: imported by tests/,
never by the library). A float64 numpy restatement of

* output_far (src/farfield.c:42-182): radiation vector
  N(r^) = sum_m I_m len_m t_m sinc(k len_m (r^.t_m)/2) exp(+j k r^.r_cm), image cells with
  -I over a ground plane (t' = (tx, ty, -tz), z' = 2 gpz - z), transverse far field
  r E = -j (omega mu0 / 4 pi) [N - (N.r^) r^], radiated power by the theta trapezoid and
  periodic phi rectangle rules, directivity and gain in dBi (-600 below 1e-30);
* tran_synth / output_tran (src/transient.c:73-177): Gaussian pulse att dB down at f_max,
  y(t_n) = df [H(0) X(0) + 2 Re sum_k H(f_k) X(f_k) e^{j 2 pi f_k t_n}], t_n = n/(2 f_max),
  H(0) = 2 Re H(f_1) - Re H(f_2), 2N samples.

It is pinned against the reference's own writers (tests/golden/post/*.npz).
"""
import numpy as np

PI = 4.0 * np.arctan(1.0)
C0 = 2.99792458e8
MU0 = 4.0 * PI * 1e-7


def _sinc(x):
    out = np.ones_like(x)
    big = np.abs(x) >= 1e-8
    out[big] = np.sin(x[big]) / x[big]
    return out


def farfield(seg, freqs, segi, zin, nth, nph, gp=0, gpz=0.0):
    """seg: structured cells (x1, x2, len); segi [nfreq, nseg] port-1 currents; zin [nfreq].
    Returns dict(et, ep [nfreq, ndir], d_dbi, g_dbi [nfreq, ndir], prad, pin [nfreq])."""
    x1 = np.asarray(seg["x1"], float)
    x2 = np.asarray(seg["x2"], float)
    ln = np.asarray(seg["len"], float)
    tv = (x2 - x1) / ln[:, None]
    rc = 0.5 * (x1 + x2)
    thmax = PI / 2 if gp else PI
    it = np.repeat(np.arange(nth + 1), nph)
    ip = np.tile(np.arange(nph), nth + 1)
    th = thmax * it / nth
    ph = 2 * PI * ip / nph
    st, ct, sp, cp = np.sin(th), np.cos(th), np.sin(ph), np.cos(ph)
    rh = np.stack([st * cp, st * sp, ct], 1)
    thh = np.stack([ct * cp, ct * sp, -st], 1)
    phh = np.stack([-sp, cp, np.zeros_like(sp)], 1)
    passes = [(tv, rc, 1.0)]
    if gp:
        tvi = tv * np.array([1, 1, -1.0])
        rci = rc.copy()
        rci[:, 2] = 2 * gpz - rci[:, 2]
        passes.append((tvi, rci, -1.0))
    eta0 = MU0 * C0
    out = {k: [] for k in ("et", "ep", "d_dbi", "g_dbi", "prad", "pin")}
    for q, f in enumerate(freqs):
        kw = 2 * PI * f / C0
        coef = 2 * PI * f * MU0 / (4 * PI)
        nv = np.zeros((len(th), 3), complex)
        for t_, r_, sgn in passes:
            rt = rh @ t_.T                      # [ndir, nseg]
            rr = rh @ r_.T
            amp = sgn * ln[None, :] * _sinc(0.5 * kw * ln[None, :] * rt)
            w = amp * segi[q][None, :] * np.exp(1j * kw * rr)
            nv += w @ t_
        nt = np.sum(thh * nv, 1)
        npp = np.sum(phh * nv, 1)
        et = coef * nt.imag - 1j * coef * nt.real
        ep = coef * npp.imag - 1j * coef * npp.real
        uu = (np.abs(et) ** 2 + np.abs(ep) ** 2) / (2 * eta0)
        wt = np.where((it == 0) | (it == nth), 0.5, 1.0)
        prad = np.sum(wt * np.sin(thmax * it / nth) * uu) * (thmax / nth) * (2 * PI / nph)
        pin = 0.5 * zin[q].real
        d = 4 * PI * uu / prad if prad > 0 else np.zeros_like(uu)
        g = 4 * PI * uu / pin if pin > 0 else np.zeros_like(uu)
        out["et"].append(et)
        out["ep"].append(ep)
        out["d_dbi"].append(np.where(d > 1e-30, 10 * np.log10(np.maximum(d, 1e-300)), -600.0))
        out["g_dbi"].append(np.where(g > 1e-30, 10 * np.log10(np.maximum(g, 1e-300)), -600.0))
        out["prad"].append(prad)
        out["pin"].append(pin)
    return {k: np.array(v) for k, v in out.items()}


def transient(f0, f1, nfreq, att_db, h):
    """h [nsig, nfreq] responses. Returns (x [2 nfreq] pulse, y [nsig, 2 nfreq], dt)."""
    df = (f1 - f0) / (nfreq - 1)
    m = 2 * nfreq
    dt = 1 / (2 * f1)
    sigma = np.sqrt(att_db * np.log(10.0) / (20 * 2 * PI * PI)) / f1
    t0 = 4 * sigma
    x0 = sigma * np.sqrt(2 * PI)
    k = np.arange(nfreq)
    fk = f0 + (f1 - f0) * k / (nfreq - 1)
    xs = x0 * np.exp(-2 * PI * PI * sigma * sigma * fk * fk) * np.exp(-1j * 2 * PI * fk * t0)
    t = np.arange(m) * dt
    ph = np.exp(1j * 2 * PI * np.outer(t, fk))          # [m, nfreq]

    def synth(g, g0):
        return df * (g0 + 2 * (ph @ g).real)
    x = synth(xs, x0)
    h = np.atleast_2d(np.asarray(h, complex))
    y = np.array([synth(hh * xs, (2 * hh[0].real - hh[1].real) * x0) for hh in h]) if h.size else np.zeros((0, m))
    return x, y, dt
