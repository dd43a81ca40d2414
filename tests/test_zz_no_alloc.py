"""snn_score_step_noalloc: one greedy step scored without any device
allocation by the library (its scratch is a fixed static device array), for
callers that cannot allocate -- e.g. code running under another runtime's
allocator or a fixed memory budget, or paths that must not let
cudaMalloc/cudaFree synchronise the device.

The test (its own file, collected last) builds the input buffers itself, calls
the entry point twice in a row through the C ABI, and checks each call's
result against the existing entry point (a handle's first greedy step): same
winning feature, same best k, the same FP32 error bit for bit and the FP64
error within 1e-9 relative -- the tolerances of the other parity tests.
"""
import ctypes

import numpy as np
import pytest

from speedynn_b200 import _lib, datagen
from speedynn_b200._lib import _i32p, ptr
from speedynn_b200.selector import Selector

pytestmark = pytest.mark.gpu

FLT_MAX = np.float32(np.finfo(np.float32).max)


def _winner(err32, err64, cands, k_vals):
    """Best k per candidate (first strict minimum in k_vals order), then the
    first strict minimum over candidates in ascending feature order."""
    best = (FLT_MAX, None, None, None)
    for ci, c in enumerate(cands):
        e, m_best = FLT_MAX, -1
        for m in range(len(k_vals)):
            if err32[ci, m] < e:
                e, m_best = err32[ci, m], m
        if m_best >= 0 and e < best[0]:
            best = (e, int(c), int(k_vals[m_best]), float(err64[ci, m_best]))
    return best


@pytest.mark.parametrize("k_list", [[3, 7], [70, 4]])
def test_noalloc_step_matches_handle_step_twice(k_list):
    """k_max <= 64 runs the TMA-fed scorer, k_max 70 the rows-per-lane one.
    The second call must not change the device's free memory (nothing is
    allocated: the scratch was placed when the library's module loaded)."""
    import torch

    torch.cuda.init()
    s = datagen.generate(3000, 1000, 12, n_mag=5, n_heavy=2, seed=71)
    k_vals = np.array(k_list, np.int32)
    n_tr, n_val, p = s.Xtrain.shape[0], s.Xval.shape[0], s.Xtrain.shape[1]

    # existing entry point: the handle API's first greedy step
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=k_vals, num_features=1, method="forward") as sel:
        ref = sel.run()
    want = (ref["errors"][0], int(ref["ordering"][0]), int(ref["step_best_k"][0]), float(ref["errors64"][0]))

    # caller-owned device buffers in the documented layouts (forward step 0: D = 0)
    dev = torch.device("cuda", 0)
    ld = (n_tr + 63) // 64 * 64
    XT = torch.zeros((p, ld), dtype=torch.float32, device=dev)
    XT[:, :n_tr] = torch.from_numpy(np.ascontiguousarray(s.Xtrain.T)).to(dev)
    XV = torch.from_numpy(np.ascontiguousarray(s.Xval.T)).to(dev)
    D = torch.zeros((n_val, ld), dtype=torch.float32, device=dev)
    D[:, n_tr:] = float("inf")
    yt = torch.from_numpy(s.ytrain).to(dev)
    yv = torch.from_numpy(s.yval).to(dev)
    cands = np.arange(p, dtype=np.int32)
    err32 = torch.full((p, k_vals.size), -1.0, dtype=torch.float32, device=dev)
    err64 = torch.full((p, k_vals.size), -1.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()

    L = _lib.lib()
    results = []
    for call in range(2):
        if call == 1:
            free_before = torch.cuda.mem_get_info(dev)[0]
            torch_before = torch.cuda.memory_allocated(dev)
        rc = L.snn_score_step_noalloc(D.data_ptr(), ld, XT.data_ptr(), XV.data_ptr(), n_val, yt.data_ptr(),
                                      yv.data_ptr(), n_val, n_tr, p, ptr(cands, _i32p), p, ptr(k_vals, _i32p),
                                      k_vals.size, 0, err32.data_ptr(), err64.data_ptr(),
                                      ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, _lib.last_error()
        if call == 1:
            assert torch.cuda.mem_get_info(dev)[0] == free_before
            assert torch.cuda.memory_allocated(dev) == torch_before
        e32, e64 = err32.cpu().numpy().copy(), err64.cpu().numpy().copy()
        got = _winner(e32, e64, cands, k_vals)
        assert got[1] == want[1] and got[2] == want[2]
        assert got[0] == want[0]  # FP32 error bit-exact
        assert abs(got[3] - want[3]) <= 1e-9 * abs(want[3])
        results.append((e32, e64))
    np.testing.assert_array_equal(results[0][0], results[1][0])
    np.testing.assert_array_equal(results[0][1], results[1][1])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = _lib.lib()
    k_vals = np.array([5], np.int32)
    cands = np.arange(8, dtype=np.int32)
    # 8 candidates x 1 k x 600,000 rows > 4,194,304 predictions: refused before touching the GPU buffers
    rc = L.snn_score_step_noalloc(1, 64, 1, 1, 600000, 1, 1, 600000, 64, 8, ptr(cands, _i32p), 8,
                                  ptr(k_vals, _i32p), 1, 0, 1, 1, None)
    assert rc == _lib.SNN_ERR_ARG
    assert b"scratch" in L.snn_last_error()


def test_noalloc_rejects_misaligned_device_pointers():
    """D and XT are read by TMA copies, which need 16-byte aligned bases: a
    misaligned pointer is refused up front with a message that says so (no
    kernel is launched, so the pointers are never dereferenced)."""
    L = _lib.lib()
    k_vals = np.array([5], np.int32)
    cands = np.arange(4, dtype=np.int32)
    rc = L.snn_score_step_noalloc(256 + 4, 64, 256, 256, 64, 256, 256, 64, 64, 4, ptr(cands, _i32p), 4,
                                  ptr(k_vals, _i32p), 1, 0, 256, 256, None)
    assert rc == _lib.SNN_ERR_ARG
    assert b"16-byte aligned" in L.snn_last_error()
