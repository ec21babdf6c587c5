"""GPU exact brute force vs the CPU oracle (BruteForceIndex, src/brute.rs).

FP32 precision is bit-exact: same keys and distance bits as the oracle's
restatement of BruteForceIndex::search_batch with the AVX2 kernels.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O

pytestmark = pytest.mark.gpu


def check_exact(metric, base, queries, k, keys=None):
    b = H.BruteForceIndex(base.shape[1], H.Metric(metric))
    kk = np.arange(base.shape[0], dtype=np.uint64) if keys is None else keys
    b.insert_batch(kk, base)
    got = b.search_arrays(queries, k)
    prepared = base if metric != 2 else O.normalize_rows(base)
    ref = O.brute(metric, prepared, queries, k, keys=kk)
    np.testing.assert_array_equal(got[3], ref[3])
    np.testing.assert_array_equal(got[2], ref[2])
    for i in range(len(queries)):
        c = int(got[2][i])
        np.testing.assert_array_equal(got[0][i, :c], ref[0][i, :c])
        np.testing.assert_array_equal(got[1][i, :c].view(np.uint32), ref[1][i, :c].view(np.uint32))


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [1, 5, 8, 32, 40, 128])
def test_brute_exact_small(metric, dim):
    base, queries = H.gaussian(3000, 37, dim, 11 + dim)
    if metric == 2:
        base[:, 0] += 2.0
        queries[:, 0] += 2.0
    check_exact(metric, base, queries, 10)


def test_brute_k_variants_and_keys():
    base, queries = H.mixture(5000, 20, 64, 10, 0.3, 1)
    keys = (np.arange(5000, dtype=np.uint64) * 7 + 3)[::-1].copy()
    for k in [1, 10, 100, 700]:
        check_exact(0, base, queries, k, keys=keys)


def test_brute_ties_break_by_key():
    """src/brute.rs:218-252."""
    b = H.BruteForceIndex(1, H.Metric.L2)
    b.insert_batch(np.array([5, 3, 9, 1], np.uint64), np.array([5, 3, 9, 1], np.float32))
    hits = b.search([4.0], 3)
    assert [h.key for h in hits] == [3, 5, 1]
    assert hits[0].distance == 1.0
    assert b.search([4.0], 0) == []
    assert len(b.search([4.0], 100)) == 4
    t = H.BruteForceIndex(1, H.Metric.L2)
    t.insert_batch(np.array([7, 2, 4], np.uint64), np.array([1, -1, 1], np.float32))
    assert [h.key for h in t.search([0.0], 3)] == [2, 4, 7]


def test_brute_768_cosine_medium():
    base, queries = H.mixture(20000, 64, 768, 64, 0.5, 3)
    check_exact(2, base, queries, 100)
