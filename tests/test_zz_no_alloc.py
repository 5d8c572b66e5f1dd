"""The no-allocation column balance of v (atjup_gpu_balance_column_v_noalloc) against the
ordinary entry point (atjup_gpu_balance_column_v), through the C ABI, on two calls in a row.

The no-allocation variant exists for callers that cannot allocate device memory (a host model
with a preallocated memory pool, code running under stream capture); it keeps its scratch in a
fixed file-scope device array. This file sorts last so that a failure here stops a -x run only
after every other test has run."""
import ctypes

import numpy as np
import pytest

from atjup_b200.gpu import load_library
from helpers import gpu_from, synthetic_case

pytestmark = pytest.mark.gpu


def test_noalloc_matches_balance_column_v_twice():
    import torch

    L = load_library()
    fn = L.atjup_gpu_balance_column_v_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                   ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                   ctypes.c_int32, ctypes.c_void_p]
    p, g, f = synthetic_case(41, 61, 97)
    ref = gpu_from(p, g, f)        # the ordinary entry point, on the context's scratch
    dut = gpu_from(p, g, f)        # the same state, balanced through the no-allocation entry
    im, jm, km = p.im, p.jm, p.km
    topo = torch.from_numpy(np.ascontiguousarray(g["topo"], np.int32)).cuda()
    rad = torch.from_numpy(np.ascontiguousarray(g["rad"], np.float64)).cuda()
    v_ptr, pitch = dut.field_ptr("v")
    torch.cuda.synchronize()
    for call in range(2):
        ref.balance_column_v()
        rc = fn(ctypes.c_void_p(v_ptr), ctypes.c_void_p(topo.data_ptr()),
                ctypes.c_void_p(rad.data_ptr()), im, jm, km, pitch, p.dr,
                p.v_massbal_zonal, None)
        assert rc == 0, L.atjup_gpu_last_error().decode()
        dut.synchronize()
        torch.cuda.synchronize()
        a, b = ref.download("v"), dut.download("v")
        rel = np.linalg.norm(a - b) / np.linalg.norm(a)
        assert rel <= 1e-14, f"call {call}: relative L2 difference {rel:.3e}"


def test_noalloc_rejects_sizes_above_its_scratch():
    L = load_library()
    fn = L.atjup_gpu_balance_column_v_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                   ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                   ctypes.c_int32, ctypes.c_void_p]
    dummy = ctypes.c_void_p(16)    # never dereferenced: the size check rejects the call first
    rc = fn(dummy, dummy, dummy, 41, 300, 361, 368, 0.025, 1, None)
    assert rc == 1 and b"above the fixed scratch limits" in L.atjup_gpu_last_error()
    rc = fn(dummy, dummy, dummy, 41, 181, 361, 1024, 0.025, 1, None)
    assert rc == 1
