"""Tensor-core brute force (tcgen05 BF16 and 3-term BF16 scoring, exact FP32
re-rank) against the exact FP32 path and the oracle.

Candidate thresholds carry a proven bound on |approximate - FP32| distance,
and the survivors are re-ranked with FP32 distances in the reference kernel
order, so the results must be bit-identical to BruteForceIndex::search_batch
(src/brute.rs:169-180) whatever the BF16 rounding.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O

pytestmark = pytest.mark.gpu


def run(metric, base, queries, k, precision, keys=None, max_candidates=None):
    bf = H.BruteForceIndex(base.shape[1], H.Metric(metric))
    kk = np.arange(base.shape[0], dtype=np.uint64) if keys is None else keys
    bf.insert_batch(kk, base)
    tcres = bf.search_arrays(queries, k, precision)
    if max_candidates is not None:
        # The scores must really filter: a broken GEMM (e.g. all zeros) would
        # make every row a candidate and still re-rank exactly.
        per_query = bf.last_candidates_per_query()
        assert 0 < per_query <= max_candidates, per_query
    return tcres, bf.search_arrays(queries, k, H.Precision.FP32)


def same(a, b):
    np.testing.assert_array_equal(a[3], b[3])
    np.testing.assert_array_equal(a[2], b[2])
    for i in range(len(a[2])):
        c = int(a[2][i])
        np.testing.assert_array_equal(a[0][i, :c], b[0][i, :c])
        np.testing.assert_array_equal(a[1][i, :c].view(np.uint32), b[1][i, :c].view(np.uint32))


@pytest.mark.parametrize("precision", [H.Precision.BF16X3, H.Precision.BF16])
def test_tensor_cosine_768_matches_fp32(precision):
    base, queries = H.mixture(30000, 150, 768, 128, 0.5, 3)
    tcres, fp = run(2, base, queries, 100, precision, max_candidates=8000)
    same(tcres, fp)


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [16, 100, 128])
def test_tensor_metrics_match_fp32_and_oracle(metric, dim):
    base, queries = H.mixture(9000, 70, dim, 40, 0.4, dim + metric)
    if metric == 2:
        base[:, 0] += 2.0
        queries[:, 0] += 2.0
    tcres, fp = run(metric, base, queries, 10, H.Precision.BF16X3, max_candidates=4500)
    same(tcres, fp)
    prepared = base if metric != 2 else O.normalize_rows(base)
    ref = O.brute(metric, prepared, queries, 10)
    same(tcres, ref)


def test_tensor_small_and_edge_cases():
    base, queries = H.gaussian(300, 5, 32, 4)
    for k in [1, 7, 300, 500]:
        tcres, fp = run(0, base, queries, k, H.Precision.BF16X3)
        same(tcres, fp)
    keys = (np.arange(300, dtype=np.uint64) * 13 + 5)[::-1].copy()
    tcres, fp = run(1, base, queries, 20, H.Precision.BF16, keys=keys)
    same(tcres, fp)
    # k = 1000 of 10000 rows: about 10% of every tile passes the threshold,
    # more than a lane's 16 staging slots, so the epilogue appends mid-tile.
    base2, queries2 = H.gaussian(10000, 40, 64, 8)
    for precision in (H.Precision.BF16, H.Precision.BF16X3):
        tcres, fp = run(0, base2, queries2, 1000, precision)
        same(tcres, fp)


# The paired kernel (two CTAs per 256 x 256 tile, cta_group::2 MMAs): the
# same results, bit for bit, and the scores still filter.

def run_pairs(metric, base, queries, k, precision, max_candidates=None):
    bf = H.BruteForceIndex(base.shape[1], H.Metric(metric))
    bf.insert_batch(np.arange(base.shape[0], dtype=np.uint64), base)
    bf.set_pairs(True)
    tcres = bf.search_arrays(queries, k, precision)
    if max_candidates is not None:
        per_query = bf.last_candidates_per_query()
        assert 0 < per_query <= max_candidates, per_query
    again = bf.search_arrays(queries, k, precision)
    bf.set_pairs(False)
    single = bf.search_arrays(queries, k, precision)
    return tcres, again, single, bf.search_arrays(queries, k, H.Precision.FP32)


@pytest.mark.parametrize("precision", [H.Precision.BF16X3, H.Precision.BF16])
def test_paired_kernel_matches_fp32(precision):
    base, queries = H.mixture(30000, 300, 768, 128, 0.5, 8)
    tcres, again, single, fp = run_pairs(2, base, queries, 100, precision, max_candidates=8000)
    same(tcres, fp)
    same(again, fp)
    same(single, fp)


@pytest.mark.parametrize("metric", [0, 1])
def test_paired_kernel_metrics_and_ragged_batches(metric):
    # 130 queries: the second query tile of the pair is mostly padding.
    base, queries = H.mixture(7000, 130, 100, 30, 0.4, 17 + metric)
    tcres, again, single, fp = run_pairs(metric, base, queries, 10, H.Precision.BF16X3, max_candidates=4000)
    same(tcres, fp)
    same(again, fp)
    same(tcres, O.brute(metric, base, queries, 10))
