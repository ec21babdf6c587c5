"""Failure paths on the GPU, made without faulting it.

The reference reports failures as values and never panics on bad input
(src/error.rs, src/hnsw/io.rs:30-37, tests/hostile_files.rs). The device
library adds two failure kinds of its own, and both are provoked here from
the host:

* HNSW_ERR_TIMEOUT: the tensor-core scoring kernel bounds every barrier wait
  by a clock budget. A test switch makes its MMA issuer wait on a barrier
  nothing arrives at, so that wait runs out; the kernel must record it, let
  its copies finish, free its tensor memory and return, and the same handle
  must then search correctly.
* HNSW_ERR_OUT_OF_DEVICE_MEMORY: a host-side hook makes the next device
  allocations fail as cudaMalloc would when memory runs out. The call must
  fail with that status and the handle must work afterwards.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from conftest import build_index

pytestmark = pytest.mark.gpu


def _same(a, b):
    np.testing.assert_array_equal(a[3], b[3])
    np.testing.assert_array_equal(a[2], b[2])
    for i in range(len(a[2])):
        c = int(a[2][i])
        np.testing.assert_array_equal(a[0][i, :c], b[0][i, :c])
        np.testing.assert_array_equal(a[1][i, :c].view(np.uint32), b[1][i, :c].view(np.uint32))


@pytest.mark.parametrize("precision", [H.Precision.BF16X3, H.Precision.BF16])
def test_tensor_core_wait_runs_out_then_the_handle_still_works(precision):
    base, queries = H.mixture(20000, 300, 128, 30, 0.4, 12)
    bf = H.BruteForceIndex(128, H.Metric.L2)
    bf.insert_batch(np.arange(20000, dtype=np.uint64), base)
    exact = bf.search_arrays(queries, 10, H.Precision.FP32)
    # About 1 ms of SM clock: the stalled wait gives up quickly.
    bf.set_wait_limits(2_000_000, inject_stall=True)
    with pytest.raises(H.Error) as e:
        bf.search_arrays(queries, 10, precision)
    assert e.value.status == H.Status.TIMEOUT
    # Twice: the error word and the pipeline are reset per search.
    with pytest.raises(H.Error) as e:
        bf.search_arrays(queries, 10, precision)
    assert e.value.status == H.Status.TIMEOUT
    bf.set_wait_limits()  # default budget, no stall
    got = bf.search_arrays(queries, 10, precision)
    _same(got, exact)
    _same(got, O.brute(0, base, queries, 10))


def test_allocation_failure_reports_out_of_device_memory_and_recovers():
    base, queries = H.gaussian(3000, 400, 32, 6)
    queries, more = queries[:50], queries
    data = build_index(base, metric=0, m=8, seed=4)
    gi = H.HnswIndex.from_bytes(data)
    ref = O.Index(data).search(queries, 10, 40)
    try:
        H.debug_fail_allocations(1)  # a fresh handle's first search allocates its scratch
        with pytest.raises(H.Error) as e:
            gi.search_arrays(queries, 10, 40)
        assert e.value.status == H.Status.OUT_OF_DEVICE_MEMORY
    finally:
        H.debug_fail_allocations(0)
    _same(gi.search_arrays(queries, 10, 40), ref)
    # The same on the brute-force handle, at its first allocation and in the
    # middle of them; each batch is larger than the last, so its buffers grow.
    bf = H.BruteForceIndex(32, H.Metric.L2)
    bf.insert_batch(np.arange(3000, dtype=np.uint64), base)
    for n, q in ((1, queries), (3, more)):
        try:
            H.debug_fail_allocations(n)
            with pytest.raises(H.Error) as e:
                bf.search_arrays(q, 10)
            assert e.value.status == H.Status.OUT_OF_DEVICE_MEMORY
        finally:
            H.debug_fail_allocations(0)
        _same(bf.search_arrays(q, 10), O.brute(0, base, q, 10))


def test_allocation_failure_at_open_leaves_nothing_behind():
    base, _ = H.gaussian(2000, 0, 16, 2)
    data = build_index(base, metric=0, m=8, seed=1)
    try:
        H.debug_fail_allocations(2)
        with pytest.raises(H.Error) as e:
            H.HnswIndex.from_bytes(data)
        assert e.value.status == H.Status.OUT_OF_DEVICE_MEMORY
    finally:
        H.debug_fail_allocations(0)
    gi = H.HnswIndex.from_bytes(data)
    assert gi.len() == 2000
