"""ctypes mirror of include/peec_b200.h and the loader of libpeec_b200.so.

The shared library is built in-tree (openpeec_b200/libpeec_b200.so) by
openpeec_b200/build.py. Loading fails loudly when it is missing: there is no host
fallback for any compute entry point.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpeec_b200.so")

# pb_cell_t (include/peec_b200.h): 28 doubles followed by 8 ints, 256 bytes.
CELL_DTYPE = np.dtype([
    ("x1", "<f8", 3), ("x2", "<f8", 3), ("len", "<f8"), ("wid", "<f8"), ("thick", "<f8"),
    ("wv", "<f8", 3), ("papex", "<f8", 3), ("aL", "<f8"), ("aP", "<f8"), ("radius", "<f8"),
    ("area", "<f8"), ("perim", "<f8"), ("sigma", "<f8"), ("res", "<f8"),
    ("cexc", "<f8"), ("gexc", "<f8"), ("gfac", "<f8"), ("epss", "<f8"), ("epsinf", "<f8"),
    ("frelax", "<f8"),
    ("n1", "<i4"), ("n2", "<i4"), ("shape", "<i4"), ("vol", "<i4"), ("diel", "<i4"),
    ("npv", "<i4"), ("pvoff", "<i4"), ("pad_", "<i4"),
])
assert CELL_DTYPE.itemsize == 256

PORT_DTYPE = np.dtype([("n1", "<i4"), ("n2", "<i4"), ("z0", "<f8")])
LUMP_DTYPE = np.dtype([("kind", "<i4"), ("n1", "<i4"), ("n2", "<i4"), ("pad", "<i4"),
                       ("val", "<f8")])
MUT_DTYPE = np.dtype([("l1", "<i4"), ("l2", "<i4"), ("k", "<f8")])

PB_LUMP_R, PB_LUMP_C, PB_LUMP_L, PB_LUMP_V = 0, 1, 2, 3
PB_OK, PB_ERR_ARG, PB_ERR_CUDA, PB_ERR_SINGULAR, PB_ERR_NOCONV, PB_ERR_UNSUP = range(6)
PREC_FP64, PREC_MIXED = 0, 1
LU_FP64, LU_FP32, LU_TC, LU_TC_CUBLAS, LU_TC_PIVOTED, LU_LDLT = 0, 1, 2, 3, 4, 5
FORM_AUTO, FORM_FULL, FORM_REDUCED = 0, 1, 2

_vp = C.c_void_p


class PbProblem(C.Structure):
    _fields_ = [
        ("nseg", C.c_int), ("seg", _vp),
        ("nchg", C.c_int), ("chg", _vp), ("chgnode", _vp),
        ("npv", C.c_int), ("pv", _vp),
        ("maxid", C.c_int),
        ("nport", C.c_int), ("port", _vp),
        ("nlump", C.c_int), ("lump", _vp),
        ("nmut", C.c_int), ("mut", _vp),
        ("capacitance", C.c_int), ("retardation", C.c_int), ("skin", C.c_int),
        ("gp", C.c_int), ("gpz", C.c_double), ("gmin", C.c_double),
    ]


class PbSweepOpts(C.Structure):
    _fields_ = [
        ("fill_prec", C.c_int), ("lu", C.c_int), ("form", C.c_int), ("batch", C.c_int),
        ("refine_tol", C.c_double), ("refine_maxit", C.c_int), ("verbose", C.c_int),
        ("corr_freqs", C.c_int), ("accel", C.c_int), ("compress", C.c_int), ("aca_dense", C.c_int),
        ("ctol", C.c_double), ("pc_mlp", C.c_void_p), ("pc_coarse", C.c_int), ("pc_exact_leaf", C.c_int),
    ]


class PbSweepStats(C.Structure):
    _fields_ = [
        ("t_static_ms", C.c_double), ("t_corr_ms", C.c_double),
        ("t_assemble_ms", C.c_double), ("t_lu_ms", C.c_double),
        ("t_refine_ms", C.c_double), ("t_total_ms", C.c_double),
        ("corr_samples", C.c_double), ("lu_flops", C.c_double),
        ("max_resid", C.c_double), ("max_iters", C.c_int), ("form_used", C.c_int),
        ("n_system", C.c_int), ("static_refreshes", C.c_int),
        ("kernel_launches", C.c_int), ("fp64_fallbacks", C.c_int),
        ("fp64_direct", C.c_int), ("fp64_max_hz", C.c_double),
        ("lu_count", C.c_int), ("gmres_solves", C.c_int), ("gmres_its_max", C.c_int),
        ("gmres_refactored", C.c_int), ("gmres_its_avg", C.c_double),
        ("hmat_far", C.c_int), ("hmat_near", C.c_int), ("hmat_max_rank", C.c_int),
        ("hmat_dense_far", C.c_int), ("hmat_mb", C.c_double), ("hmat_dense_mb", C.c_double),
        ("pc_mlp_fallbacks", C.c_int), ("pc_coarse_n", C.c_int), ("t_coarse_ms", C.c_double),
        ("probe_fallbacks", C.c_int), ("pipelined", C.c_int), ("probe_max", C.c_double),
        ("hmat_entries", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PbPlanewave(C.Structure):
    _fields_ = [("theta_deg", C.c_double), ("phi_deg", C.c_double), ("pol", C.c_int),
                ("pad_", C.c_int), ("amp", C.c_double), ("phase_deg", C.c_double)]


class PbSource(C.Structure):
    """pb_source_t (include/peec_b200.h)."""
    _fields_ = [("n1", C.c_int), ("n2", C.c_int), ("isvsrc", C.c_int), ("pad_", C.c_int),
                ("amp", C.c_double), ("phase_deg", C.c_double)]


def ptr(a):
    """Address of a contiguous numpy array (None for None / empty)."""
    if a is None or a.size == 0:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def problem_struct(prob):
    """Fill a PbProblem from a openpeec_b200.problem.Problem (arrays kept alive by prob)."""
    s = PbProblem()
    s.nseg, s.seg = len(prob.seg), ptr(prob.seg)
    s.nchg, s.chg, s.chgnode = len(prob.chg), ptr(prob.chg), ptr(prob.chgnode)
    s.npv, s.pv = len(prob.pv) // 3, ptr(prob.pv)
    s.maxid = int(prob.maxid)
    s.nport, s.port = len(prob.port), ptr(prob.port)
    s.nlump, s.lump = len(prob.lump), ptr(prob.lump)
    s.nmut, s.mut = len(prob.mut), ptr(prob.mut)
    s.capacitance, s.retardation = int(prob.capacitance), int(prob.retardation)
    s.skin, s.gp = int(prob.skin), int(prob.gp)
    s.gpz, s.gmin = float(prob.gpz), float(prob.gmin)
    return s


_lib = None


def lib():
    """Load libpeec_b200.so (built in-tree). Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libpeec_b200.so is not built (run `python -m openpeec_b200.build` or "
            "__graft_entry__.build()); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    L.pb_last_error.restype = C.c_char_p
    L.pb_device_count.restype = C.c_int
    L.pb_create.argtypes = [C.POINTER(PbProblem), C.POINTER(_vp)]
    L.pb_destroy.argtypes = [_vp]
    L.pb_sizes.argtypes = [_vp] + [C.POINTER(C.c_int)] * 5
    L.pb_lp_fill.argtypes = [_vp, C.c_double, C.c_int, _vp]
    L.pb_pot_fill.argtypes = [_vp, C.c_double, C.c_int, _vp]
    L.pb_sweep.argtypes = [_vp, C.c_int, _vp, C.POINTER(PbSweepOpts), _vp, _vp,
                           C.POINTER(PbSweepStats)]
    L.pb_sweep_dist.argtypes = [_vp, C.c_int, _vp, C.POINTER(PbSweepOpts), _vp, _vp, _vp,
                                C.POINTER(PbSweepStats)]
    L.pb_planewave.argtypes = [_vp, C.c_int, _vp, C.POINTER(PbSweepOpts), C.POINTER(PbPlanewave),
                               _vp, _vp, C.POINTER(PbSweepStats)]
    L.pb_lu_decomp.argtypes = [C.c_int, _vp, _vp]
    L.pb_lu_solve.argtypes = [C.c_int, _vp, _vp, _vp]
    L.pb_lu_decomp_batched_dev.argtypes = [C.c_int, C.c_int, _vp, _vp, _vp]
    L.pb_fp32_peak.argtypes = [C.POINTER(C.c_double)]
    L.pb_lu_decomp_batched32_dev.argtypes = [C.c_int, C.c_int, _vp, _vp, _vp, C.c_int]
    L.pb_cgemm_sub_batched_dev.argtypes = [C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int,
                                           C.c_longlong, C.c_int, C.c_int]
    L.pb_lp_fill_noalloc.argtypes = [C.c_int, _vp, C.c_int, C.c_double, C.c_double, C.c_int, _vp]
    L.pb_device_sync.restype = C.c_int
    L.pb_sources.argtypes = [_vp, C.c_int, _vp, C.POINTER(PbSweepOpts), C.c_int, _vp, _vp,
                             C.POINTER(PbSweepStats)]
    L.pb_farfield.argtypes = [_vp, C.c_int, _vp, _vp, C.c_longlong, _vp, C.c_int, C.c_int, _vp, _vp, _vp,
                              _vp, _vp, _vp]
    L.pb_transient.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _vp, _vp, _vp, _vp]
    L.pb_sweep_many.argtypes = [C.c_int, _vp, _vp, _vp, C.POINTER(PbSweepOpts), _vp, _vp, C.c_int]
    L.pb_mlp_nparam.restype = C.c_int
    L.pb_pc_samples.argtypes = [_vp, C.c_double, C.POINTER(PbSweepOpts), _vp, _vp]
    L.pb_mlp_train.argtypes = [_vp, C.c_int, _vp, _vp, C.c_int, C.c_float, _vp]
    L.pb_mlp_grad.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp]
    L.pb_mlp_predict.argtypes = [_vp, C.c_int, _vp, _vp]
    _lib = L
    return L


def last_error():
    return lib().pb_last_error().decode(errors="replace")
