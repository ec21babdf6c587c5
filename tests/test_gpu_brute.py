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


def _same(got, ref):
    np.testing.assert_array_equal(got[3], ref[3])
    np.testing.assert_array_equal(got[2], ref[2])
    for i in range(len(got[2])):
        c = int(got[2][i])
        np.testing.assert_array_equal(got[0][i, :c], ref[0][i, :c])
        np.testing.assert_array_equal(got[1][i, :c].view(np.uint32), ref[1][i, :c].view(np.uint32))


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_brute_search_filtered_key_bitmaps(metric):
    """BruteForceIndex::search_filtered (src/brute.rs:131-160): shared,
    per-query and banked key bitmaps, some queries unfiltered."""
    base, queries = H.gaussian(4000, 40, 24, 70 + metric)
    if metric == 2:
        base[:, 0] += 2.0
        queries[:, 0] += 2.0
    keys = np.arange(4000, dtype=np.uint64) * 3 + 1
    bf = H.BruteForceIndex(24, H.Metric(metric))
    bf.insert_batch(keys, base)
    prepared = base if metric != 2 else O.normalize_rows(base)
    rng = np.random.default_rng(metric)
    nbits = int(keys.max()) + 1
    words = (nbits + 63) // 64
    shared = H.key_bitmap(keys[rng.random(4000) < 0.1], nbits)
    got = bf.search_arrays(queries, 10, filter_bits=shared, filter_nbits=nbits)
    _same(got, O.brute_filtered(metric, prepared, queries, 10, shared, nbits, keys=keys))
    per = np.zeros((40, words), np.uint64)
    for i in range(40):
        per[i] = H.key_bitmap(keys[rng.random(4000) < rng.uniform(0.001, 0.5)], nbits)
    used = (rng.random(40) < 0.7).astype(np.uint8)
    got = bf.search_arrays(queries, 25, filter_bits=per, filter_nbits=nbits, filter_stride=words, filter_used=used)
    ref_bits = per.copy()
    ref_bits[used == 0] = H.key_bitmap(keys, nbits)  # unfiltered queries admit every key
    _same(got, O.brute_filtered(metric, prepared, queries, 25, ref_bits, nbits, words, keys=keys))
    ids = rng.integers(0, 5, 40).astype(np.uint32)
    got = bf.search_arrays(queries, 7, filter_bits=per[:5], filter_nbits=nbits, filter_stride=words, filter_ids=ids)
    _same(got, O.brute_filtered(metric, prepared, queries, 7, per[ids], nbits, words, keys=keys))


def test_brute_search_filtered_closure_on_sparse_keys():
    base, queries = H.gaussian(3000, 6, 16, 91)
    rng = np.random.default_rng(92)
    keys = np.unique(rng.integers(1 << 40, 1 << 63, 3100, dtype=np.uint64))[:3000]
    rng.shuffle(keys)
    bf = H.BruteForceIndex(16, H.Metric.L2)
    bf.insert_batch(keys, base)
    pred = lambda key: key % 5 == 2  # noqa: E731
    rows = np.array([i for i, k in enumerate(keys.tolist()) if pred(k)], np.uint64)
    bits = H.key_bitmap(rows, 3000)
    for i in range(6):
        got = bf.search_filtered(queries[i], 12, pred)
        ref = O.brute_filtered(0, base, queries[i:i + 1], 12, bits, 3000, by_row=True, keys=keys)
        assert [n.key for n in got] == ref[0][0, :int(ref[2][0])].tolist()
        assert all(pred(n.key) for n in got)
    assert bf.search_filtered(queries[0], 5, lambda key: False) == []
    # k above the admitted count returns every admitted row; k is capped at len.
    only = keys[:3]
    got = bf.search_filtered(queries[0], 100, lambda key: key in set(only.tolist()))
    assert sorted(n.key for n in got) == sorted(only.tolist())
