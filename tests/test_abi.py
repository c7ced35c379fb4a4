"""The C ABI library: builds for sm_100a, loads, exports every declared entry point, and
refuses to compute without a GPU (no host fallback)."""
import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from openpeec_b200 import abi, configs, geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        txt = re.sub(r"typedef[^;]*;", "", txt)
        txt = re.sub(r"static inline[^{]*\{[^}]*\}", "", txt)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", txt):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.append(name)
    return sorted(set(names))


def test_library_exports_all_declared_symbols():
    L = abi.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert len(declared_functions()) >= 10


def test_struct_layout_matches_header(tmp_path):
    """sizeof/offsetof of the header's structs (compiled with gcc) == the ctypes mirror."""
    src = tmp_path / "lay.c"
    src.write_text('''
#include <stdio.h>
#include <stddef.h>
#include "peec_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(pb_cell_t), sizeof(pb_port_t), sizeof(pb_lump_t),
         sizeof(pb_mutual_t), sizeof(pb_problem_t), sizeof(pb_sweep_opts), sizeof(pb_sweep_stats));
  printf("%zu %zu %zu %zu %zu\\n", offsetof(pb_cell_t, aL), offsetof(pb_cell_t, n1),
         offsetof(pb_cell_t, pvoff), offsetof(pb_problem_t, gpz), offsetof(pb_sweep_stats, max_iters));
  return 0;
}
''')
    exe = tmp_path / "lay"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [int(v) for v in out]
    want = [abi.CELL_DTYPE.itemsize, abi.PORT_DTYPE.itemsize, abi.LUMP_DTYPE.itemsize,
            abi.MUT_DTYPE.itemsize, C.sizeof(abi.PbProblem), C.sizeof(abi.PbSweepOpts),
            C.sizeof(abi.PbSweepStats),
            abi.CELL_DTYPE.fields["aL"][1], abi.CELL_DTYPE.fields["n1"][1],
            abi.CELL_DTYPE.fields["pvoff"][1], abi.PbProblem.gpz.offset,
            abi.PbSweepStats.max_iters.offset]
    assert got == want


def test_no_host_fallback_without_device():
    if abi.lib().pb_device_count() > 0:
        pytest.skip("a CUDA device is present")
    from openpeec_b200 import api
    p = geometry.build(geometry.parse_peec(configs.CFG1))
    with pytest.raises(api.PbError) as e:
        api.Context(p)
    assert e.value.code == abi.PB_ERR_CUDA
    assert "no CUDA device" in str(e.value)
    r, _, _ = (None, None, None)
    a = np.eye(3, dtype=complex)
    assert abi.lib().pb_lu_decomp(3, a.ctypes.data, np.zeros(3, np.int32).ctypes.data) == -2


def test_bad_arguments_rejected():
    s = abi.PbProblem()
    h = C.c_void_p()
    s.nport = 0
    assert abi.lib().pb_create(C.byref(s), C.byref(h)) == abi.PB_ERR_ARG


def test_loads_after_an_older_cublas():
    """A host that loaded another libcublas.so.12 first keeps it for every later library
    (the loader matches the soname). PyTorch's bundled cuBLAS (12.8) lacks
    cublasSetEmulationStrategy (12.9), so the library resolves it at run time instead of
    linking it, and loads either way (the BF16x9 updates then fall back to the SIMT GEMM)."""
    try:
        import nvidia.cublas
    except ImportError:
        pytest.skip("no second cuBLAS in this environment")
    d = os.path.join(list(nvidia.cublas.__path__)[0], "lib")
    if not os.path.exists(os.path.join(d, "libcublas.so.12")):
        pytest.skip("no second cuBLAS in this environment")
    code = ("import ctypes, os, sys; d = sys.argv[1]; "
            "ctypes.CDLL(os.path.join(d, 'libcublasLt.so.12'), mode=ctypes.RTLD_GLOBAL); "
            "ctypes.CDLL(os.path.join(d, 'libcublas.so.12'), mode=ctypes.RTLD_GLOBAL); "
            "from openpeec_b200 import abi; abi.lib(); print('loaded')")
    r = subprocess.run([sys.executable, "-c", code, d], cwd=ROOT, capture_output=True, text=True, timeout=240)
    assert r.returncode == 0 and "loaded" in r.stdout, r.stderr[-2000:]
