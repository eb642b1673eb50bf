"""casphy_join_indel_noalloc: the join for callers that cannot allocate
device memory (a framework owning the GPU's memory pool, or a loop that must
not take cudaMalloc/cudaFree's device-wide synchronisation).

It is called through the C ABI with device buffers the test owns and must
give exactly the bytes casphy_join_indel gives, on two calls in a row (the
second call reuses the library's fixed scratch array, which still holds the
first call's data).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from casphy_b200 import synth

pytestmark = pytest.mark.gpu


def _case(seed, ncell, nsite, weights):
    raw = synth.lineage_states(ncell, nsite, 12, 0.05, 24, 1.4, 0.1, seed=seed)
    codes, ns = synth.regularize(raw)
    rng = np.random.default_rng(seed)
    if weights == "unit":
        w = np.ones((ns, nsite))
    else:
        w = rng.uniform(0.05, 3.0, size=(ns, nsite)).round(3)
    tip = rng.integers(1, 5, size=ncell).astype(np.uint32)
    return codes, ns, w, tip


def _noalloc(lib, torch, codes, ns, w, tip, min_size, min_ratio):
    ntip, ncol = codes.shape
    d_codes = torch.from_numpy(codes.view(np.int32)).cuda()
    d_edge = torch.full((2 * ntip - 2, 2), -7, dtype=torch.int32, device="cuda")
    d_state = torch.full((ntip - 1, ncol), -7, dtype=torch.int32, device="cuda")
    f = lib.casphy_join_indel_noalloc
    f.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                  C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
    wf = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
    ts = np.ascontiguousarray(tip, dtype=np.uint32)
    torch.cuda.synchronize()
    rc = f(ntip, ncol, d_codes.data_ptr(), ns, wf.ctypes.data, ts.ctypes.data, min_size, min_ratio,
           d_edge.data_ptr(), d_state.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.casphy_last_error()
    torch.cuda.synchronize()
    return (d_edge.cpu().numpy().view(np.uint32), d_state.cpu().numpy().view(np.uint32))


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    import casphy_b200.lib as L
    lib = L.lib()
    lib.casphy_last_error.restype = C.c_char_p
    cases = [(_case(41, 1500, 96, "unit"), 0, 2.0), (_case(42, 700, 64, "real"), 3, 1.5)]
    for (codes, ns, w, tip), ms, mr in cases:
        e0, s0, _ = L.join_indel(codes, ns, w, tip, ms, mr)
        e1, s1 = _noalloc(lib, torch, codes, ns, w, tip, ms, mr)
        assert np.array_equal(e1, e0)
        assert np.array_equal(s1, s0)


def test_noalloc_rejects_oversized_input():
    torch = pytest.importorskip("torch")
    import casphy_b200.lib as L
    lib = L.lib()
    lib.casphy_last_error.restype = C.c_char_p
    f = lib.casphy_join_indel_noalloc
    f.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                  C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
    w = np.ones(4 * 1024)
    tip = np.ones(100000, dtype=np.uint32)
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")  # never touched: the size check comes first
    p = buf.data_ptr()
    rc = f(100000, 1024, p, 4, w.ctypes.data, tip.ctypes.data, 0, 2.0, p, p, None)
    assert rc == 2
    assert b"scratch" in lib.casphy_last_error()


def test_noalloc_integer_weights_near_the_limit():
    """6,000 cells x 512 sites with integer weights 0..2 (about two thirds of
    the fixed scratch), against the allocating entry point."""
    torch = pytest.importorskip("torch")
    import casphy_b200.lib as L
    lib = L.lib()
    lib.casphy_last_error.restype = C.c_char_p
    raw = synth.lineage_states(6000, 512, 16, 0.03, 48, 1.3, 0.15, seed=43)
    codes, ns = synth.regularize(raw)
    w = np.random.default_rng(43).integers(0, 3, size=(ns, 512)).astype(np.float64)
    tip = np.ones(6000, dtype=np.uint32)
    e0, s0, st = L.join_indel(codes, ns, w, tip, 0, 2.0)
    assert st["int_path"] == 1
    e1, s1 = _noalloc(lib, torch, codes, ns, w, tip, 0, 2.0)
    assert np.array_equal(e1, e0) and np.array_equal(s1, s0)


_FRESH = r"""
import ctypes as C, json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import casphy_b200.lib as L
from casphy_b200 import synth
lib = L.lib()
raw = synth.lineage_states(900, 64, 12, 0.05, 24, 1.4, 0.1, seed=44)
codes, ns = synth.regularize(raw)
ntip, ncol = codes.shape
w = np.ones(ns * ncol)
tip = np.ones(ntip, dtype=np.uint32)
d_codes = torch.from_numpy(codes.view(np.int32)).cuda()
d_edge = torch.zeros((2 * ntip - 2, 2), dtype=torch.int32, device="cuda")
d_state = torch.zeros((ntip - 1, ncol), dtype=torch.int32, device="cuda")
f = lib.casphy_join_indel_noalloc
f.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
              C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
torch.cuda.synchronize()
free = []
for call in range(3):
    free.append(torch.cuda.mem_get_info()[0])
    rc = f(ntip, ncol, d_codes.data_ptr(), ns, w.ctypes.data, tip.ctypes.data, 0, 2.0, d_edge.data_ptr(),
           d_state.data_ptr(), None)
    assert rc == 0
torch.cuda.synchronize()
free.append(torch.cuda.mem_get_info()[0])
print(json.dumps(free))
"""


def test_noalloc_first_in_a_fresh_process_then_allocates_nothing():
    """In a fresh process whose first join is the no-alloc call: the first
    call may reserve the library's scratch array (the CUDA runtime loads the
    library's device code on first use), after which further calls leave the
    device's free memory unchanged."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    out = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    free = json.loads(out.stdout.strip().splitlines()[-1])
    # before call 2, before call 3 and after call 3: no change
    assert free[1] == free[2] == free[3], free
    # the first call's reservation, if any, is the scratch array (64 MiB), not more
    assert free[0] - free[1] <= (64 << 20) + (8 << 20), free
