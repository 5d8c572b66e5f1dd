"""The asynchronous field exchange (atjup_gpu_upload_async, atjup_gpu_apply_uploads,
atjup_gpu_download_async): a caller that keeps the state on the host and exchanges it every step
must get exactly what the synchronous atjup_gpu_upload / atjup_gpu_download give, although its
copies run on the library's copy streams and overlap the compute of neighbouring steps.

* Three full-physics steps, each with its own inputs (so a stale or early copy would show), the
  results of every step downloaded: bit-identical to the synchronous path.
* Two downloads of one field around a step, with no upload in between (the same staging buffer
  reused): the first holds the state before the step, the second after it.
* atjup_gpu_stream returns the stream the context issues on, before and after atjup_gpu_set_stream."""
import numpy as np
import pytest

from moist_cases import PROGNOSTIC, gpu_moist_model, synthetic_moist_case

STEPS = 3


def inputs(f, k):
    """the host state handed in at step k: the synthetic fields, t and the vapour nudged by k"""
    out = {}
    for n in PROGNOSTIC:
        a = np.ascontiguousarray(f[n], dtype=np.float64).copy()
        if n in ("t", "h2o"):
            a *= 1.0 + 1.0e-7 * k
        out[n] = a
    return out


@pytest.mark.gpu
def test_async_exchange_matches_synchronous():
    P, PH, MC, g, f = synthetic_moist_case(13, 37, 49, seed=61)
    sync = gpu_moist_model(P, PH, MC, g, f)
    want = []
    for k in range(1, STEPS + 1):
        for n, a in inputs(f, k).items():
            sync.upload(n, a)
        sync.step(k, first=(k == 1))
        want.append({n: sync.download(n) for n in PROGNOSTIC})
    sync.close()

    m = gpu_moist_model(P, PH, MC, g, f)
    keep_in, got = [], []
    for k in range(1, STEPS + 1):
        ins = inputs(f, k)
        keep_in.append(ins)                       # alive until synchronize
        for n, a in ins.items():
            m.upload_async(n, a)
        m.apply_uploads()
        m.step(k, first=(k == 1))
        outs = {n: np.empty(m.shape) for n in PROGNOSTIC}
        for n, o in outs.items():
            m.download_async(n, o)
        got.append(outs)
    m.synchronize()
    m.close()
    for k in range(STEPS):
        for n in PROGNOSTIC:
            assert np.array_equal(got[k][n], want[k][n], equal_nan=True), f"step {k + 1}: {n} differs"


@pytest.mark.gpu
def test_async_download_reuses_its_buffer_in_order():
    P, PH, MC, g, f = synthetic_moist_case(13, 37, 49, seed=62)
    ref = gpu_moist_model(P, PH, MC, g, f)
    before = ref.download("t")
    ref.step(1, first=True)
    after = ref.download("t")
    ref.close()
    m = gpu_moist_model(P, PH, MC, g, f)
    a, b = np.empty(m.shape), np.empty(m.shape)
    m.download_async("t", a)
    m.step(1, first=True)
    m.download_async("t", b)
    m.synchronize()
    m.close()
    assert np.array_equal(a, before)
    assert np.array_equal(b, after)


@pytest.mark.gpu
def test_stream_handle_follows_set_stream():
    import torch
    P, PH, MC, g, f = synthetic_moist_case(13, 37, 49, seed=63)
    m = gpu_moist_model(P, PH, MC, g, f)
    own = m.stream_handle()
    assert own != 0
    s = torch.cuda.Stream()
    m.set_stream(s.cuda_stream)
    assert m.stream_handle() == s.cuda_stream
    m.step(1, first=True)
    m.synchronize()
    m.set_stream(None)                     # back to a stream of the context's own
    assert m.stream_handle() not in (0, s.cuda_stream)
    assert m.nonfinite_count() == 0
    m.close()


@pytest.mark.gpu
def test_stage_group_timing():
    """ATJUP_TK_RK_GROUP: one entry per RK stage, each spanning the stage's scalar kernels (second
    stream) and its dynamics kernel; so it is at least the longer of the two streams' work and at
    most their sum, plus the launch gaps between them (50 us per stage allowed)."""
    P, PH, MC, g, f = synthetic_moist_case(13, 37, 49, seed=64)
    m = gpu_moist_model(P, PH, MC, g, f)
    m.timing(True)
    for it in (1, 2):
        m.step(it, first=(it == 1))
    m.synchronize()
    cls = {n: m.timing_read(i) for i, n in enumerate(m.TIMING_CLASSES)}
    m.timing(False)
    m.close()
    grp_ms, grp_n = cls["rk_group"]
    assert grp_n == 8 and cls["rk_stage"][1] == 8 and cls["species"][1] == 8 and cls["closure"][1] == 8
    side = cls["species"][0] + cls["closure"][0]
    assert max(side, cls["rk_stage"][0]) * 0.999 <= grp_ms <= side + cls["rk_stage"][0] + 8 * 0.05
