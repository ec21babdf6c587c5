"""The allocation-free brute-force entry point against the regular one.

hnsw_gpu_brute_search_batch_noalloc serves callers that cannot allocate
device memory while they run (latency-critical paths, processes whose memory
policy forbids cudaMalloc after start-up, callers that must not let
cudaMalloc/cudaFree synchronise the device). It takes device buffers and
keeps its scratch in a fixed array inside the library. Its results must equal
those of hnsw_gpu_brute_search_batch exactly (both compute FP32 distances in
the reference kernel order), on two calls in a row, since the second call
reuses the scratch the first one left behind.

This file is named to be collected last.
"""

import ctypes as C

import numpy as np
import pytest

import hnsw_gpu as H

pytestmark = pytest.mark.gpu

_lib = C.CDLL(H.LIBRARY_PATH)
_fn = _lib.hnsw_gpu_brute_search_batch_noalloc
_fn.restype = C.c_int
_fn.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_uint32, C.c_void_p, C.c_void_p,
                C.c_void_p, C.c_void_p, C.c_void_p]


def _noalloc(bf, queries, k):
    import torch

    dev = torch.device("cuda", 0)
    q = torch.from_numpy(np.ascontiguousarray(queries, np.float32)).to(dev)
    nq = q.shape[0]
    keys = torch.zeros((nq, max(k, 1)), dtype=torch.int64, device=dev)
    dist = torch.zeros((nq, max(k, 1)), dtype=torch.float32, device=dev)
    count = torch.zeros(nq, dtype=torch.int32, device=dev)
    status = torch.zeros(nq, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = _fn(bf._h, q.data_ptr(), nq, q.shape[1], k, keys.data_ptr(), dist.data_ptr(), count.data_ptr(),
             status.data_ptr(), stream.cuda_stream or 1)
    torch.cuda.synchronize(dev)
    return st, (keys.cpu().numpy().view(np.uint64), dist.cpu().numpy(), count.cpu().numpy().view(np.uint32),
                status.cpu().numpy())


def _same(a, b):
    ak, ad, ac, ast = a
    bk, bd, bc, bst = b
    np.testing.assert_array_equal(ast, bst)
    np.testing.assert_array_equal(ac, bc)
    for i in range(len(ac)):
        c = int(ac[i])
        np.testing.assert_array_equal(ak[i, :c], bk[i, :c])
        np.testing.assert_array_equal(ad[i, :c].view(np.uint32), bd[i, :c].view(np.uint32))


@pytest.mark.parametrize("metric", [0, 2])
def test_noalloc_matches_regular_entry_point_twice(metric):
    base, queries = H.mixture(60000, 400, 128, 50, 0.3, 21)
    bf = H.BruteForceIndex(128, H.Metric(metric))
    bf.insert_batch(np.arange(60000, dtype=np.uint64) * 3 + 1, base)
    first, second = queries[:200], queries[200:]
    st1, got1 = _noalloc(bf, first, 10)
    st2, got2 = _noalloc(bf, second, 10)
    assert st1 == 0 and st2 == 0
    _same(got1, bf.search_arrays(first, 10))
    _same(got2, bf.search_arrays(second, 10))


def test_noalloc_rejects_batches_beyond_its_scratch():
    base, queries = H.gaussian(2000, 0, 768, 3)
    bf = H.BruteForceIndex(768, H.Metric.L2)
    bf.insert_batch(np.arange(2000, dtype=np.uint64), base)
    big = np.zeros((4096, 768), np.float32)  # 4096 * 3 KB of prepared queries > 8 MiB
    st, _ = _noalloc(bf, big, 10)
    assert st == H.Status.INVALID_ARGUMENT
    # The handle still works after the rejection.
    st, got = _noalloc(bf, base[:50], 5)
    assert st == 0
    _same(got, bf.search_arrays(base[:50], 5))
