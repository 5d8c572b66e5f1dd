"""The no-allocation column balance of v (atjup_gpu_balance_column_v_noalloc) against the
ordinary entry point (atjup_gpu_balance_column_v), through the C ABI, on two calls in a row.

The no-allocation variant exists for callers that cannot allocate device memory: a host model
whose GPU memory is one pool sized at start-up, or an embedding that must not fail part-way
through a run on an allocation. It keeps its scratch in a fixed file-scope device array. Both
forms of the balance are covered: the plain column means, and the zonal variant that also
removes the row mean of the column means (it keeps those row means after the column means in
the same array). This file sorts last so that a failure here stops a -x run only after every
other test has run."""
import ctypes

import numpy as np
import pytest

from atjup_b200.gpu import load_library
from helpers import DRY_ENV, gpu_from, synthetic_case

pytestmark = pytest.mark.gpu

_ARGTYPES = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
             ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p]


def _entry(L):
    fn = L.atjup_gpu_balance_column_v_noalloc
    fn.argtypes = _ARGTYPES
    fn.restype = ctypes.c_int
    return fn


@pytest.mark.parametrize("zonal", [0, 1])
def test_noalloc_matches_balance_column_v_twice(zonal):
    import torch

    L = load_library()
    fn = _entry(L)
    env = {**DRY_ENV, "ATJUP_V_MASSBAL_ZONAL": str(zonal)}
    p, g, f = synthetic_case(41, 61, 97, env=env)
    assert p.v_massbal_zonal == zonal
    ref = gpu_from(p, g, f)        # the ordinary entry point, on the context's scratch
    dut = gpu_from(p, g, f)        # the same state, balanced through the no-allocation entry
    im, jm, km = p.im, p.jm, p.km
    topo = torch.from_numpy(np.ascontiguousarray(g["topo"], np.int32)).cuda()
    rad = torch.from_numpy(np.ascontiguousarray(g["rad"], np.float64)).cuda()
    v_ptr, pitch = dut.field_ptr("v")
    v0 = dut.download("v")
    torch.cuda.synchronize()
    for call in range(2):
        ref.balance_column_v()
        rc = fn(ctypes.c_void_p(v_ptr), ctypes.c_void_p(topo.data_ptr()),
                ctypes.c_void_p(rad.data_ptr()), im, jm, km, pitch, p.dr, zonal, None)
        assert rc == 0, L.atjup_gpu_last_error().decode()
        dut.synchronize()
        torch.cuda.synchronize()
        a, b = ref.download("v"), dut.download("v")
        assert not np.array_equal(a, v0), "the balance left v unchanged: nothing was compared"
        rel = np.linalg.norm(a - b) / np.linalg.norm(a)
        assert rel <= 1e-14, f"zonal={zonal} call {call}: relative L2 difference {rel:.3e}"


def test_noalloc_rejects_sizes_above_its_scratch():
    import torch

    L = load_library()
    fn = _entry(L)
    # Real device buffers, large enough for every size asked for below: the size check refuses
    # the call before any launch, and had it not, the kernels would still only touch valid
    # device memory.
    n = max(41 * 300 * 368, 41 * 181 * 1024)
    buf = torch.zeros(n, dtype=torch.float64, device="cuda")
    ptr = ctypes.c_void_p(buf.data_ptr())
    rc = fn(ptr, ptr, ptr, 41, 300, 361, 368, 0.025, 1, None)
    assert rc == 1 and b"above the fixed scratch limits" in L.atjup_gpu_last_error()
    rc = fn(ptr, ptr, ptr, 41, 181, 361, 1024, 0.025, 1, None)
    assert rc == 1 and b"above the fixed scratch limits" in L.atjup_gpu_last_error()
    torch.cuda.synchronize()
    assert torch.count_nonzero(buf).item() == 0
