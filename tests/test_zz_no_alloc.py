"""The fill entry point that allocates no device memory (pb_lp_fill_noalloc).

It serves host programs that manage all GPU memory themselves and may not call
cudaMalloc: they hand in the cells and the output buffer already in device memory, and
the library uses only its fixed scratch array. This file is collected last on purpose,
so that a run stopping at its first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from openpeec_b200 import abi, api, configs, geometry

pytestmark = pytest.mark.gpu
C0 = 2.99792458e8


def _problem():
    # 16 x 8 plate over ground + feed wire: 284 current cells, within the 512-cell limit
    return geometry.build(geometry.parse_peec(configs.cfg2(16, 8, 4)))


@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-12), (abi.PREC_MIXED, 1e-12)])
def test_noalloc_matches_allocating_entry_point(prec, tol):
    """Two calls in a row through the C ABI give the matrix of pb_lp_fill."""
    import torch
    prob = _problem()
    n = len(prob.seg)
    kw = 2 * np.pi * 1.28e9 / C0
    with api.Context(prob) as ctx:
        ref = ctx.lp_fill(kw, prec)
    cells = torch.from_numpy(prob.seg.view(np.uint8).copy()).cuda()
    out = torch.empty((n, n, 2), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for call in range(2):
        out.fill_(np.nan)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        r = abi.lib().pb_lp_fill_noalloc(n, cells.data_ptr(), int(prob.gp), float(prob.gpz),
                                         float(kw), int(prec), out.data_ptr())
        assert r == abi.PB_OK, abi.last_error()
        if call == 1:
            # after the first call (which may load the library's kernels), a call takes no
            # device memory: the driver's free-memory count is unchanged
            assert torch.cuda.mem_get_info()[0] == free0
        got = out.cpu().numpy()
        got = got[..., 0] + 1j * got[..., 1]
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(got - ref)) <= tol * scale


def test_noalloc_rejects_oversized_and_polygon_input():
    import torch
    prob = _problem()
    cells = torch.from_numpy(prob.seg.view(np.uint8).copy()).cuda()
    out = torch.empty(16, dtype=torch.float64, device="cuda")
    r = abi.lib().pb_lp_fill_noalloc(513, cells.data_ptr(), 0, 0.0, 1.0, 1, out.data_ptr())
    assert r == abi.PB_ERR_ARG and "512" in abi.last_error()
    poly = prob.seg[:4].copy()
    poly["npv"][1] = 4
    pc = torch.from_numpy(poly.view(np.uint8).copy()).cuda()
    out = torch.empty((4, 4, 2), dtype=torch.float64, device="cuda")
    r = abi.lib().pb_lp_fill_noalloc(4, pc.data_ptr(), 0, 0.0, 1.0, 1, out.data_ptr())
    assert r == abi.PB_ERR_UNSUP
