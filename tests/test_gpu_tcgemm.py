"""The LU's trailing update C -= A B (complex FP32) on the tensor cores and on the SIMT
pipes, against an FP64 product of the same inputs; and the batched FP32 factorisation
that uses it, against its backward error.

The update is the row update of the reference's lu_decomp (src/lu.c:54-62) done for a
block of rows and columns at once. The tensor-core kernel splits every FP32 operand into
three BF16 terms and sums the six products of significance >= 2^-16 with FP32
accumulation, so its error is that of an FP32 product: the bar below is 1e-6 of the
entrywise bound |A||B| (FP32 accumulation over k terms included). Without accumulation
error the six products are 1000x closer than a two-term split and 1e5x closer than one
BF16 product (checked on the CPU in test_bf16_split_bound).
"""
import ctypes as C

import numpy as np
import pytest

from openpeec_b200 import abi

TOL = 1e-6          # max |C - C_ref| / max (|A| |B|), FP32-class accuracy


def _bf16(x):
    """Round FP32 values to BF16 (8 significant bits, nearest even), returned as FP32."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16).astype(np.uint32)
    return b.view(np.float32)


def _terms(x, n):
    out, r = [], np.asarray(x, np.float32).copy()
    for _ in range(n):
        t = _bf16(r)
        r = (r - t).astype(np.float32)
        out.append(t.astype(np.float64))
    return out


def test_bf16_split_bound():
    """CPU check of the arithmetic the kernel relies on: the six products of the three-term
    BF16 split meet the bar; one BF16 product, or the three products of a two-term split,
    do not."""
    rng = np.random.default_rng(3)
    k = 512
    a = rng.standard_normal((64, k)).astype(np.float32)
    b = rng.standard_normal((k, 64)).astype(np.float32)
    ref = a.astype(np.float64) @ b.astype(np.float64)
    bound = np.max(np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64))
    a3, b3 = _terms(a, 3), _terms(b, 3)
    six = sum(a3[i] @ b3[j] for i, j in ((0, 0), (0, 1), (1, 0), (0, 2), (1, 1), (2, 0)))
    two = a3[0] @ b3[0] + a3[0] @ b3[1] + a3[1] @ b3[0]
    e6 = np.max(np.abs(six - ref)) / bound
    assert e6 < TOL / 100
    assert np.max(np.abs(two - ref)) / bound > 300 * e6
    assert np.max(np.abs(a3[0] @ b3[0] - ref)) / bound > 1e5 * e6


def _crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _run_update(kind, m, nc, k, nb, ld, seed, expect=abi.PB_OK):
    """A, B, C as sub-blocks of nb row-major ld x ld matrices, like the LU's panels:
    A = rows [o, o+m) x cols [0, k), B = rows [0, k) x cols [o, o+nc), C = rows [o, o+m) x
    cols [o, o+nc), with the offset o = k rounded up to a multiple of 8."""
    import torch
    rng = np.random.default_rng(seed)
    big = _crand(rng, (nb, ld, ld))
    o = (k + 7) // 8 * 8
    assert o + m <= ld and o + nc <= ld
    A = big[:, o:o + m, 0:k]
    B = big[:, 0:k, o:o + nc]
    Cm = big[:, o:o + m, o:o + nc]
    ref = Cm.astype(np.complex128) - np.einsum("bik,bkj->bij", A.astype(np.complex128), B.astype(np.complex128))
    bound = np.einsum("bik,bkj->bij", np.abs(A).astype(np.float64), np.abs(B).astype(np.float64))
    dev = torch.from_numpy(big.view(np.float32).copy()).cuda()
    base = dev.data_ptr()
    cs = 8      # bytes per complex
    pa = base + (o * ld + 0) * cs
    pb = base + (0 * ld + o) * cs
    pc = base + (o * ld + o) * cs
    r = abi.lib().pb_cgemm_sub_batched_dev(m, nc, k, pa, ld, pb, ld, pc, ld, ld * ld, nb, kind)
    assert r == expect, abi.last_error()
    if expect != abi.PB_OK:
        return None
    torch.cuda.synchronize()
    out = dev.cpu().numpy().view(np.complex64).reshape(nb, ld, ld)
    got = out[:, o:o + m, o:o + nc]
    err = np.max(np.abs(got.astype(np.complex128) - ref)) / np.max(bound)
    # nothing outside C may change
    mask = np.ones((nb, ld, ld), bool)
    mask[:, o:o + m, o:o + nc] = False
    assert np.array_equal(out[mask], big[mask])
    return err


@pytest.mark.gpu
@pytest.mark.parametrize("m,nc,k,nb,ld", [
    (128, 128, 16, 1, 160),          # exactly one tile and one stage
    (256, 384, 512, 2, 1024),        # whole tiles
    (300, 200, 100, 3, 420),         # ragged rows, columns and k (TMA zero fill, epilogue guards)
    (1000, 520, 777, 2, 1800),       # many tiles, k not a multiple of the stage
])
def test_tc_update_matches_fp64(m, nc, k, nb, ld):
    err = _run_update(abi.LU_TC, m, nc, k, nb, ld, seed=m + nc + k)
    assert err < TOL, err


@pytest.mark.gpu
@pytest.mark.parametrize("m,nc,k,nb,ld", [(64, 32, 32, 2, 128), (300, 200, 100, 3, 420), (129, 65, 17, 1, 211)])
def test_simt_update_matches_fp64(m, nc, k, nb, ld):
    err = _run_update(abi.LU_FP32, m, nc, k, nb, ld, seed=7 * m + k)
    assert err < TOL, err


@pytest.mark.gpu
def test_tc_update_rejects_what_tma_cannot_address():
    """Odd leading dimensions break the 16-byte TMA stride rule and updates under one
    128 x 128 x 16 tile are not the kernel's: the entry point refuses them for the
    tensor-core kind (the factorisation sends them to the SIMT kernel instead)."""
    _run_update(abi.LU_TC, 256, 256, 64, 2, 515, seed=11, expect=abi.PB_ERR_UNSUP)
    _run_update(abi.LU_TC, 100, 256, 64, 1, 512, seed=12, expect=abi.PB_ERR_UNSUP)
    err = _run_update(abi.LU_FP32, 256, 256, 64, 2, 515, seed=11)
    assert err < TOL, err


def _lu_backward_error(a, lu, piv):
    n = a.shape[0]
    L = np.tril(lu, -1) + np.eye(n)
    U = np.triu(lu)
    pa = a.copy()
    for kk in range(n):
        j = piv[kk]
        if j != kk:
            pa[[kk, j]] = pa[[j, kk]]
    return np.max(np.abs(pa - L @ U)) / np.max(np.abs(a))


@pytest.mark.gpu
@pytest.mark.parametrize("n,nb", [(520, 3), (1036, 2), (517, 2)])
def test_fp32_lu_with_tc_updates(n, nb):
    """Batched FP32 LU whose trailing updates run on the tcgen05 kernel: backward error at
    FP32 level, no zero pivot, and the same pivots as the SIMT-update factorisation on
    well-separated pivots (diagonally weighted random matrices)."""
    import torch
    rng = np.random.default_rng(n)
    a = _crand(rng, (nb, n, n))
    a += (np.arange(n)[None, :, None] == np.arange(n)[None, None, :]) * (3.0 * np.sqrt(n))
    out = {}
    for kind in (abi.LU_TC, abi.LU_FP32):
        dev = torch.from_numpy(a.view(np.float32).copy()).cuda()
        piv = torch.zeros((nb, n), dtype=torch.int32, device="cuda")
        info = (C.c_int * nb)()
        r = abi.lib().pb_lu_decomp_batched32_dev(n, nb, dev.data_ptr(), piv.data_ptr(), info, kind)
        assert r == abi.PB_OK, abi.last_error()
        assert all(v == -1 for v in info)
        out[kind] = (dev.cpu().numpy().view(np.complex64).reshape(nb, n, n), piv.cpu().numpy())
    for b in range(nb):
        lu, pv = out[abi.LU_TC]
        be = _lu_backward_error(a[b].astype(np.complex128), lu[b].astype(np.complex128), pv[b])
        assert be < 2e-5, be
        assert np.array_equal(pv[b], out[abi.LU_FP32][1][b])


@pytest.mark.gpu
@pytest.mark.parametrize("n,nb", [(520, 3), (1036, 2), (517, 2), (45, 4)])
def test_fp32_ldlt_of_complex_symmetric(n, nb):
    """L D L^T without pivoting of complex-symmetric matrices (the reduced MNA form): only the
    lower triangle is read (the upper one holds garbage here), the factors come back as an
    unpivoted LU with U = D L^T, piv the identity, and L U reproduces A to FP32 level."""
    import torch
    rng = np.random.default_rng(7 * n)
    a = _crand(rng, (nb, n, n))
    a = a + np.swapaxes(a, 1, 2)                       # complex symmetric
    a += (np.arange(n)[None, :, None] == np.arange(n)[None, None, :]) * (3.0 * np.sqrt(n))
    g = a.copy()
    g[:, np.triu_indices(n, 1)[0], np.triu_indices(n, 1)[1]] = 1e3 + 1e3j   # never read
    dev = torch.from_numpy(g.view(np.float32).copy()).cuda()
    piv = torch.zeros((nb, n), dtype=torch.int32, device="cuda")
    info = (C.c_int * nb)()
    r = abi.lib().pb_lu_decomp_batched32_dev(n, nb, dev.data_ptr(), piv.data_ptr(), info, abi.LU_LDLT)
    assert r == abi.PB_OK, abi.last_error()
    assert all(v == -1 for v in info)
    lu = dev.cpu().numpy().view(np.complex64).reshape(nb, n, n).astype(np.complex128)
    pv = piv.cpu().numpy()
    for b in range(nb):
        assert np.array_equal(pv[b], np.arange(n))
        assert _lu_backward_error(a[b], lu[b], pv[b]) < 2e-5
        L = np.tril(lu[b], -1) + np.eye(n)
        assert np.allclose(np.triu(lu[b]), np.diag(np.diag(lu[b])) @ L.T, rtol=0, atol=2e-5 * np.abs(a[b]).max())


@pytest.mark.gpu
def test_tc_update_has_no_accumulation_drift():
    """A long accumulation (k = 2048) stays as accurate as an FP32 product: the tensor
    core truncates when it adds into its accumulator, so the kernel sums TMEM only over
    chunks of 64 k and adds the chunks in FP32 registers. Without the chunking the result
    shrinks by ~1.2e-5 relative at this k (a systematic drift, measured on B200)."""
    import torch
    rng = np.random.default_rng(5)
    m = nc = 240
    k = 2048
    A = _crand(rng, (m, k))
    B = _crand(rng, (k, nc))
    ref = -(A.astype(np.complex128) @ B.astype(np.complex128))
    res = {}
    for kind in (abi.LU_TC, abi.LU_FP32):
        a = torch.from_numpy(A.view(np.float32).copy()).cuda()
        b = torch.from_numpy(B.view(np.float32).copy()).cuda()
        c = torch.zeros((m, 2 * nc), dtype=torch.float32, device="cuda")
        r = abi.lib().pb_cgemm_sub_batched_dev(m, nc, k, a.data_ptr(), k, b.data_ptr(), nc, c.data_ptr(), nc,
                                               m * nc, 1, kind)
        assert r == abi.PB_OK, abi.last_error()
        torch.cuda.synchronize()
        got = c.cpu().numpy().view(np.complex64).astype(np.complex128)
        res[kind] = (np.linalg.norm(got - ref) / np.linalg.norm(ref), abs(np.mean(np.real(got / ref)) - 1))
    rel_tc, drift_tc = res[abi.LU_TC]
    rel_simt, _ = res[abi.LU_FP32]
    assert drift_tc < 1.5e-6, drift_tc
    assert rel_tc < 3 * rel_simt, (rel_tc, rel_simt)
