"""Python binding of the batched core of libpeec_b200.so (include/peec_b200.h).

    from openpeec_b200 import geometry, api
    prob = geometry.load_peec("dipole.peec")
    with api.Context(prob) as ctx:
        z, stats = ctx.sweep(prob.freqs())           # Z matrices per frequency

Every compute call runs on the GPU; a missing library or device raises.
"""
import ctypes as C

import numpy as np

from . import abi


class PbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("libpeec_b200 error %d: %s" % (code, msg))
        self.code = code


def _check(code):
    if code != abi.PB_OK:
        raise PbError(code, abi.last_error())


class Context:
    """Device-resident discretisation of one structure (pb_create / pb_destroy)."""

    def __init__(self, prob):
        self.prob = prob
        self._s = abi.problem_struct(prob)
        h = C.c_void_p()
        _check(abi.lib().pb_create(C.byref(self._s), C.byref(h)))
        self.h = h
        ns, nh, nc, nn, nu = (C.c_int() for _ in range(5))
        _check(abi.lib().pb_sizes(self.h, C.byref(ns), C.byref(nh), C.byref(nc), C.byref(nn),
                                  C.byref(nu)))
        self.nseg, self.nchg, self.ncell = ns.value, nh.value, nc.value
        self.nnode, self.nunknown = nn.value, nu.value

    def close(self):
        if getattr(self, "h", None):
            abi.lib().pb_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def lp_fill(self, kw, prec=abi.PREC_MIXED):
        out = np.zeros((self.nseg, self.nseg), np.complex128)
        _check(abi.lib().pb_lp_fill(self.h, float(kw), int(prec), out.ctypes.data))
        return out

    def pot_fill(self, kw, prec=abi.PREC_MIXED):
        out = np.zeros((self.ncell, self.ncell), np.complex128)
        _check(abi.lib().pb_pot_fill(self.h, float(kw), int(prec), out.ctypes.data))
        return out

    def sweep(self, freqs, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC, form=abi.FORM_AUTO,
              batch=0, refine_tol=0.0, refine_maxit=0, want_segi=False, zmat_out=None,
              corr_freqs=0, verbose=0, accel=None, compress=None, ctol=None, pc_mlp=None, pc_coarse=0,
              want_cellq=False, pc_exact_leaf=0, aca_dense=0):
        """pb_sweep. accel / compress / ctol = None take the .peec file's acceleration and
        compression keys. want_cellq (pb_sweep_dist) adds the cell charges
        [nfreq, nport, ncell] of every port excitation after the segment currents."""
        accel = getattr(self.prob, "accel", 0) if accel is None else accel
        compress = getattr(self.prob, "compress", 0) if compress is None else compress
        ctol = getattr(self.prob, "ctol", 0.0) if ctol is None else ctol
        freqs = np.ascontiguousarray(freqs, np.float64)
        npt = len(self.prob.port)
        z = zmat_out if zmat_out is not None else np.zeros((len(freqs), npt, npt), np.complex128)
        segi = np.zeros((len(freqs), npt, self.nseg), np.complex128) if want_segi else None
        o = abi.PbSweepOpts(int(fill_prec), int(lu), int(form), int(batch), float(refine_tol),
                            int(refine_maxit), int(verbose), int(corr_freqs), int(accel),
                            int(compress), 0, float(ctol))
        if pc_mlp is not None:
            pc_mlp = np.ascontiguousarray(pc_mlp, np.float32)
            o.pc_mlp = pc_mlp.ctypes.data
        o.pc_coarse = int(pc_coarse)
        o.pc_exact_leaf = int(pc_exact_leaf)
        o.aca_dense = int(aca_dense)
        st = abi.PbSweepStats()
        if want_cellq:
            q = np.zeros((len(freqs), npt, self.ncell), np.complex128)
            _check(abi.lib().pb_sweep_dist(self.h, len(freqs), freqs.ctypes.data, C.byref(o),
                                           z.ctypes.data, None if segi is None else segi.ctypes.data,
                                           q.ctypes.data, C.byref(st)))
            if want_segi:
                return z, segi, q, st.as_dict()
            return z, q, st.as_dict()
        _check(abi.lib().pb_sweep(self.h, len(freqs), freqs.ctypes.data, C.byref(o),
                                  z.ctypes.data, None if segi is None else segi.ctypes.data,
                                  C.byref(st)))
        if want_segi:
            return z, segi, st.as_dict()
        return z, st.as_dict()


    def planewave(self, freqs, pw, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC, form=abi.FORM_AUTO,
                  batch=0, accel=0, want_segi=False, compress=0, ctol=0.0):
        """Plane-wave incidence (pb_planewave): pw = (theta_deg, phi_deg, pol, amp,
        phase_deg). Returns voc [nport, nfreq] (open-circuit port voltages), the induced
        segment currents [nfreq, nseg] when want_segi, and the stats. compress = 1 solves
        on the compressed path (H-matrix + GMRES)."""
        freqs = np.ascontiguousarray(freqs, np.float64)
        npt = len(self.prob.port)
        voc = np.zeros((npt, len(freqs)), np.complex128)
        seg = np.zeros((len(freqs), self.nseg), np.complex128) if want_segi else None
        o = abi.PbSweepOpts(int(fill_prec), int(lu), int(form), int(batch), 0.0, 0, 0, 0, int(accel),
                            int(compress), 0, float(ctol), None)
        w = abi.PbPlanewave(float(pw[0]), float(pw[1]), int(pw[2]), 0, float(pw[3]),
                            float(pw[4]) if len(pw) > 4 else 0.0)
        st = abi.PbSweepStats()
        _check(abi.lib().pb_planewave(self.h, len(freqs), freqs.ctypes.data, C.byref(o), C.byref(w),
                                      voc.ctypes.data, None if seg is None else seg.ctypes.data,
                                      C.byref(st)))
        if want_segi:
            return voc, seg, st.as_dict()
        return voc, st.as_dict()


    def sources(self, freqs, sources=None, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC, batch=0):
        """Independent-source excitation (pb_sources): node voltages [nfreq, maxid+1] as
        the reference's print_vnode reports them, and the stats. sources: (isvsrc, n1, n2,
        amp, phase_deg) tuples; None takes the problem's own vsource/isource list."""
        src = self.prob.sources if sources is None else sources
        arr = (abi.PbSource * len(src))(*[abi.PbSource(int(n1), int(n2), int(v), 0, float(a), float(ph))
                                          for v, n1, n2, a, ph in src])
        freqs = np.ascontiguousarray(freqs, np.float64)
        vn = np.zeros((len(freqs), self.prob.maxid + 1), np.complex128)
        o = abi.PbSweepOpts(int(fill_prec), int(lu), int(abi.FORM_FULL), int(batch), 0.0, 0, 0, 0, 0, 0, 0, 0.0,
                            None)
        st = abi.PbSweepStats()
        _check(abi.lib().pb_sources(self.h, len(freqs), freqs.ctypes.data, C.byref(o), len(src),
                                    C.cast(arr, C.c_void_p), vn.ctypes.data, C.byref(st)))
        return vn, st.as_dict()

    def farfield(self, freqs, segi, zin, nth, nph):
        """Far field of port-1 currents segi [nfreq, nseg] (or [nfreq, nport, nseg]: port 1
        is taken) with input impedance zin [nfreq] (pb_farfield). Returns a dict of et, ep,
        d_dbi, g_dbi [nfreq, (nth+1)*nph], prad, pin [nfreq]."""
        freqs = np.ascontiguousarray(freqs, np.float64)
        segi = np.ascontiguousarray(segi, np.complex128)
        stride = segi.shape[-1] * (segi.shape[1] if segi.ndim == 3 else 1)
        zin = np.ascontiguousarray(zin, np.complex128)
        nf, nd = len(freqs), (nth + 1) * nph
        out = {k: np.zeros((nf, nd), np.complex128) for k in ("et", "ep")}
        out.update({k: np.zeros((nf, nd)) for k in ("d_dbi", "g_dbi")})
        out.update({k: np.zeros(nf) for k in ("prad", "pin")})
        _check(abi.lib().pb_farfield(self.h, nf, freqs.ctypes.data, segi.ctypes.data, stride, zin.ctypes.data,
                                     int(nth), int(nph), out["et"].ctypes.data, out["ep"].ctypes.data,
                                     out["d_dbi"].ctypes.data, out["g_dbi"].ctypes.data, out["prad"].ctypes.data,
                                     out["pin"].ctypes.data))
        return out

    def pc_samples(self, freq, fill_prec=abi.PREC_MIXED, ctol=0.0):
        """Training samples of the learned preconditioner correction at one frequency:
        (features [nseg, 12], targets [nseg, 2]) (pb_pc_samples)."""
        x = np.zeros((self.nseg, 12), np.float32)
        t = np.zeros((self.nseg, 2), np.float32)
        o = abi.PbSweepOpts(int(fill_prec), int(abi.LU_FP64), 0, 0, 0.0, 0, 0, 0, 0, 1, 0, float(ctol))
        _check(abi.lib().pb_pc_samples(self.h, float(freq), C.byref(o), x.ctypes.data, t.ctypes.data))
        return x, t


def sweep_many(ctxs, freqs, fill_prec=abi.PREC_MIXED, lu=abi.LU_TC, nthreads=0, want_stats=False):
    """pb_sweep_many: every context sweeps its own frequency list (freqs: one list per
    context) concurrently. Returns the Z matrices [nfreq_k, nport_k, nport_k] per context
    (and the per-instance stats)."""
    n = len(ctxs)
    fl = [np.ascontiguousarray(f, np.float64) for f in freqs]
    zs = [np.zeros((len(f), len(c.prob.port), len(c.prob.port)), np.complex128) for c, f in zip(ctxs, fl)]
    hs = (C.c_void_p * n)(*[c.h for c in ctxs])
    nf = (C.c_int * n)(*[len(f) for f in fl])
    fp = (C.c_void_p * n)(*[f.ctypes.data for f in fl])
    zp = (C.c_void_p * n)(*[z.ctypes.data for z in zs])
    st = (abi.PbSweepStats * n)()
    o = abi.PbSweepOpts(int(fill_prec), int(lu), 0, 0, 0.0, 0, 0, 0, 0, 0, 0, 0.0, None)
    _check(abi.lib().pb_sweep_many(n, C.cast(hs, C.c_void_p), C.cast(nf, C.c_void_p), C.cast(fp, C.c_void_p),
                                   C.byref(o), C.cast(zp, C.c_void_p), C.cast(st, C.c_void_p), int(nthreads)))
    return (zs, [s.as_dict() for s in st]) if want_stats else zs


def transient(f0, f1, nfreq, h, att_db=40.0):
    """Transient synthesis (pb_transient) of responses h [nsig, nfreq] on the sweep
    f_k = k df: (x pulse [2 nfreq], y [nsig, 2 nfreq], dt)."""
    h = np.ascontiguousarray(np.atleast_2d(h), np.complex128)
    nsig = h.shape[0] if h.size else 0
    x = np.zeros(2 * nfreq)
    y = np.zeros((nsig, 2 * nfreq))
    dt = C.c_double()
    _check(abi.lib().pb_transient(int(nfreq), float(f0), float(f1), float(att_db), nsig,
                                  h.ctypes.data if nsig else None, x.ctypes.data,
                                  y.ctypes.data if nsig else None, C.byref(dt)))
    return x, y, dt.value


MLP_IN, MLP_H, MLP_OUT = 12, 128, 2


def mlp_nparam():
    return abi.lib().pb_mlp_nparam()


def mlp_init(seed=0):
    """Initial weights (uniform +-1/sqrt(fan_in), biases 0) in the library's layout."""
    rng = np.random.default_rng(seed)
    parts = []
    for fin, fout in ((MLP_IN, MLP_H), (MLP_H, MLP_H), (MLP_H, MLP_OUT)):
        parts.append(rng.uniform(-1, 1, (fout, fin)).astype(np.float32).ravel() / np.float32(np.sqrt(fin)))
        parts.append(np.zeros(fout, np.float32))
    w = np.concatenate(parts).astype(np.float32)
    assert w.size == mlp_nparam()
    return w


def mlp_train(w, x, t, steps=2000, lr=1e-3, want_loss=False):
    w = np.ascontiguousarray(w, np.float32).copy()
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    hist = np.zeros(steps, np.float32) if want_loss else None
    _check(abi.lib().pb_mlp_train(w.ctypes.data, len(x), x.ctypes.data, t.ctypes.data, int(steps),
                                  float(lr), None if hist is None else hist.ctypes.data))
    return (w, hist) if want_loss else w


def mlp_grad(w, x, t):
    w = np.ascontiguousarray(w, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    g = np.zeros(mlp_nparam(), np.float32)
    loss = C.c_float()
    _check(abi.lib().pb_mlp_grad(w.ctypes.data, len(x), x.ctypes.data, t.ctypes.data, g.ctypes.data,
                                 C.byref(loss)))
    return float(loss.value), g


def mlp_predict(w, x):
    w = np.ascontiguousarray(w, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros((len(x), MLP_OUT), np.float32)
    _check(abi.lib().pb_mlp_predict(w.ctypes.data, len(x), x.ctypes.data, y.ctypes.data))
    return y


def lu_decomp(a):
    """GPU LU with the reference's contract (src/lu.c:16-66): returns (info, LU, piv)."""
    a = np.ascontiguousarray(a, np.complex128).copy()
    piv = np.zeros(a.shape[0], np.int32)
    r = abi.lib().pb_lu_decomp(a.shape[0], a.ctypes.data, piv.ctypes.data)
    if r == -2:
        raise PbError(abi.PB_ERR_CUDA, abi.last_error())
    return r, a, piv


def lu_solve(lu, piv, b):
    b = np.ascontiguousarray(b, np.complex128).copy()
    _check(abi.lib().pb_lu_solve(lu.shape[0], np.ascontiguousarray(lu).ctypes.data,
                                 np.ascontiguousarray(piv, np.int32).ctypes.data, b.ctypes.data))
    return b
