"""The allocation-free brute-force entry point against the regular one and
the oracle.

hnsw_gpu_brute_search_batch_noalloc serves callers that cannot allocate
device memory while they run (latency-critical paths, processes whose memory
policy forbids cudaMalloc after start-up, callers that must not let
cudaMalloc/cudaFree synchronise the device). It takes device buffers and
keeps its scratch in a fixed array inside the library. Its results must equal
those of hnsw_gpu_brute_search_batch exactly (both compute FP32 distances in
the reference kernel order), and those of the oracle's restatement of
BruteForceIndex::search_batch (src/brute.rs:122-180), on two calls in a row,
since the second call reuses the scratch the first one left behind.

This file is named to be collected last.
"""

import ctypes as C

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O

pytestmark = pytest.mark.gpu

_lib = C.CDLL(H.LIBRARY_PATH)
_fn = _lib.hnsw_gpu_brute_search_batch_noalloc
_fn.restype = C.c_int
_fn.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_uint32, C.c_void_p, C.c_void_p,
                C.c_void_p, C.c_void_p, C.c_void_p]

SCRATCH = 8 << 20  # bytes of the fixed array


def _noalloc(bf, queries, k, null_stream=False):
    import torch

    dev = torch.device("cuda", 0)
    q = torch.from_numpy(np.ascontiguousarray(queries, np.float32)).to(dev)
    nq = q.shape[0]
    keys = torch.zeros((nq, max(k, 1)), dtype=torch.int64, device=dev)
    dist = torch.zeros((nq, max(k, 1)), dtype=torch.float32, device=dev)
    count = torch.zeros(nq, dtype=torch.int32, device=dev)
    status = torch.zeros(nq, dtype=torch.int32, device=dev)
    if null_stream:
        # NULL = the handle's own stream, not ordered with torch's: the
        # inputs must be written before the call and the device synchronised
        # before the outputs are read.
        torch.cuda.synchronize(dev)
        handle = None
    else:
        handle = torch.cuda.current_stream(dev).cuda_stream or 1
    st = _fn(bf._h, q.data_ptr(), nq, q.shape[1], k, keys.data_ptr(), dist.data_ptr(), count.data_ptr(),
             status.data_ptr(), handle)
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


def _oracle(metric, base, keys, queries, k):
    prepared = base if metric != 2 else O.normalize_rows(base)
    return O.brute(metric, prepared, queries, k, keys=keys)


@pytest.mark.parametrize("metric", [0, 2])
def test_noalloc_matches_regular_entry_point_and_oracle_twice(metric):
    base, queries = H.mixture(60000, 400, 128, 50, 0.3, 21)
    keys = np.arange(60000, dtype=np.uint64) * 3 + 1
    bf = H.BruteForceIndex(128, H.Metric(metric))
    bf.insert_batch(keys, base)
    first, second = queries[:200], queries[200:]
    st1, got1 = _noalloc(bf, first, 10)
    st2, got2 = _noalloc(bf, second, 10)
    assert st1 == 0 and st2 == 0
    _same(got1, bf.search_arrays(first, 10))
    _same(got2, bf.search_arrays(second, 10))
    _same(got1, _oracle(metric, base, keys, first, 10))
    _same(got2, _oracle(metric, base, keys, second, 10))


def test_noalloc_with_fewer_slices_than_the_regular_path():
    # 8000 queries x 128 dims x 4 B = 4,096,000 B of prepared queries and
    # 8000 x 64 x 8 B = 4,096,000 B per row slice: one slice fits the array
    # (the regular path would cut 60000 rows into 8 slices), so the queries'
    # top-k lists sit right after the prepared queries and the merge reads a
    # single slice.
    base, queries = H.mixture(60000, 8000, 128, 40, 0.3, 5)
    keys = np.arange(60000, dtype=np.uint64)[::-1].copy()
    bf = H.BruteForceIndex(128, H.Metric.L2)
    bf.insert_batch(keys, base)
    for _ in range(2):
        st, got = _noalloc(bf, queries, 64)
        assert st == 0
        _same(got, bf.search_arrays(queries, 64))
    sample = slice(0, 400)
    ref = _oracle(0, base, keys, queries[sample], 64)
    _same(tuple(x[sample] for x in got), ref)


def test_noalloc_size_limit_is_the_documented_rule():
    # round_up(nq * 4 * round_up(dim, 32), 256) + nq * 8 * max(1, min(k, n)) <= 8 MiB.
    dim, n, k = 96, 3000, 32
    base, queries = H.gaussian(n, 0, dim, 9)
    bf = H.BruteForceIndex(dim, H.Metric.L2)
    bf.insert_batch(np.arange(n, dtype=np.uint64), base)

    def need(nq):
        return (nq * 4 * 96 + 255) // 256 * 256 + nq * 8 * k

    nq = 1
    while need(nq + 1) <= SCRATCH:
        nq += 1
    assert need(nq) <= SCRATCH < need(nq + 1)
    rng = np.random.default_rng(4)
    q = rng.standard_normal((nq + 1, dim)).astype(np.float32)
    st, got = _noalloc(bf, q[:nq], k)
    assert st == 0
    sample = slice(0, 200)
    _same(tuple(x[sample] for x in got), O.brute(0, base, q[sample], k))
    st, _ = _noalloc(bf, q, k)
    assert st == H.Status.INVALID_ARGUMENT
    # k = 0 still takes 8 bytes per query (one slot per slice).
    st, got = _noalloc(bf, q[:50], 0)
    assert st == 0 and (got[2] == 0).all() and (got[3] == 0).all()


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


def test_noalloc_on_the_handles_own_stream():
    base, queries = H.mixture(20000, 300, 64, 20, 0.4, 8)
    bf = H.BruteForceIndex(64, H.Metric.InnerProduct)
    bf.insert_batch(np.arange(20000, dtype=np.uint64), base)
    for _ in range(2):
        st, got = _noalloc(bf, queries, 16, null_stream=True)
        assert st == 0
        _same(got, bf.search_arrays(queries, 16))
    _same(got, O.brute(1, base, queries, 16))
