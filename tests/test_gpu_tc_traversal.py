"""Tensor-core traversal (hnsw_search_opts.traversal = BF16 / BF16X3) against the oracle.

The graph walk computes each neighbor list's distances on the tensor cores,
so it may step differently from the reference's f32 walk where distances
nearly tie; the ef results are then re-ranked with exact f32 distances, as
the quantized search does (src/hnsw/mod.rs:494-498). The bar:

* every returned distance is the exact f32 distance of its key in the
  reference's kernel order (oracle `distance`), bit for bit, and each list is
  sorted by (distance, key) with no key twice;
* recall@k against exact ground truth (oracle brute force) within 0.002 of
  the f32 search's (the reference's) for BF16X3 and within 0.01 for BF16, on
  these query sets;
* BF16X3 returns the f32 search's list unchanged for at least 99% of queries;
* filters and tombstones are honoured exactly (no key outside the filter, no
  deleted key).
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from conftest import build_index

pytestmark = pytest.mark.gpu

TOL = {H.Traversal.BF16: 0.01, H.Traversal.BF16X3: 0.002}


def stored_rows(metric, base):
    return O.normalize_rows(base) if metric == 2 else np.ascontiguousarray(base, np.float32)


def check_exact(metric, base, keys_of_rows, queries, got, k):
    """Distances bit-equal to the oracle's for the returned keys; sorted by
    (distance, key); no duplicates."""
    gk, gd, gc, gs = got
    rows = stored_rows(metric, base)
    row_of = {int(key): i for i, key in enumerate(keys_of_rows)}
    for i in range(len(gc)):
        assert gs[i] == 0
        c = int(gc[i])
        assert c <= k
        _, q = O.prepare_query(metric, queries[i])
        ks = gk[i, :c]
        assert len(set(ks.tolist())) == c
        for j in range(c):
            ref = O.distance(metric, q, rows[row_of[int(ks[j])]])
            assert np.float32(gd[i, j]).view(np.uint32) == np.float32(ref).view(np.uint32), (i, j)
        order = sorted(range(c), key=lambda j: (float(gd[i, j]), int(ks[j])))
        assert order == list(range(c))


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("traversal", [H.Traversal.BF16, H.Traversal.BF16X3])
@pytest.mark.parametrize("mode", [0, 1])
def test_recall_parity_and_exact_distances(metric, traversal, mode):
    # dim 100: rows padded to 128 values in the tensor-core layout.
    base, queries = H.mixture(8000, 400, 100, 40, 0.4, 13)
    data = build_index(base, metric=metric, m=16, seed=5)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    k, ef = 10, 64
    ref = oi.search(queries, k, ef)
    got = gi.search_arrays(queries, k, ef, mode=mode, traversal=traversal)
    check_exact(metric, base, np.arange(8000, dtype=np.uint64), queries, got, k)
    tk, _, tc, _ = O.brute(metric, stored_rows(metric, base), queries, k)
    r_ref = O.recall_at_k(tk, tc, ref[0], ref[2], k)
    r_tc = O.recall_at_k(tk, tc, got[0], got[2], k)
    assert abs(r_tc - r_ref) <= TOL[traversal], (r_tc, r_ref)
    if traversal == H.Traversal.BF16X3:
        same = sum(int(got[2][i] == ref[2][i] and np.array_equal(got[0][i, :got[2][i]], ref[0][i, :ref[2][i]]))
                   for i in range(len(queries)))
        assert same >= 0.99 * len(queries), same


@pytest.mark.parametrize("traversal", [H.Traversal.BF16, H.Traversal.BF16X3])
@pytest.mark.parametrize("mode", [0, 1])
def test_filters_tombstones_and_retry_passes(traversal, mode):
    """The general kernels (filters, tombstones), the cold-list variant and
    the retry passes in their tensor-core builds: a small schedule sends
    queries to the retry kernels."""
    base, queries = H.mixture(6000, 200, 64, 30, 0.4, 21)
    rng = np.random.default_rng(3)
    dead = np.nonzero(rng.random(6000) < 0.05)[0]
    data = build_index(base, metric=0, m=12, seed=4, deleted_keys=dead)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    keys = np.arange(6000, dtype=np.uint64)
    accepted = keys[keys % 9 == 2]
    bits = H.key_bitmap(accepted, 6000)
    k, ef = 10, 48
    ref = oi.search(queries, k, ef, filter_bits=bits, filter_nbits=6000)
    live = np.setdiff1d(keys, dead.astype(np.uint64))
    truth = O.brute_filtered(0, base[live.astype(np.int64)], queries, k, bits, 6000, keys=live)
    r_ref = O.recall_at_k(truth[0], truth[2], ref[0], ref[2], k)
    for sched in [None, dict(ef_cap=64, cand_cap=64, hash_cap=1024, warps_per_block=4, cold=0),
                  dict(ef_cap=64, cand_cap=64, hash_cap=1024, warps_per_block=4, cold=1)]:
        if sched:
            gi.set_schedule(**sched)
        got = gi.search_arrays(queries, k, ef, filter_bits=bits, filter_nbits=6000, mode=mode, traversal=traversal)
        check_exact(0, base, keys, queries, got, k)
        assert np.isin(got[0][:, :k][np.arange(k)[None, :] < got[2][:, None]], accepted).all()
        assert not np.isin(got[0][:, :k][np.arange(k)[None, :] < got[2][:, None]], dead).any()
        r_tc = O.recall_at_k(truth[0], truth[2], got[0], got[2], k)
        assert abs(r_tc - r_ref) <= TOL[traversal], (sched, r_tc, r_ref)
    gi.set_schedule()


def test_upper_layers_and_entry_on_tensor_cores():
    """k = 1 and ef = 1: the answer is the greedy descent's end plus one
    layer-0 step, all on tensor-core distances; with BF16X3 it matches f32."""
    base, queries = H.gaussian(4000, 300, 32, 9)
    data = build_index(base, metric=0, m=8, seed=2)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    ref = oi.search(queries, 1, 1)
    got = gi.search_arrays(queries, 1, 1, traversal=H.Traversal.BF16X3)
    check_exact(0, base, np.arange(4000, dtype=np.uint64), queries, got, 1)
    same = int((got[0][:, 0] == ref[0][:, 0]).sum())
    assert same >= 0.99 * len(queries)


def test_rejects_quantized_and_unknown_traversal():
    base, queries = H.gaussian(2000, 4, 32, 1)
    data = build_index(base, metric=0, m=8, seed=1, quantize=True)
    gi = H.HnswIndex.from_bytes(data)
    with pytest.raises(H.Error) as e:
        gi.search_arrays(queries, 5, 20, quantized=True, traversal=H.Traversal.BF16)
    assert e.value.status == H.Status.INVALID_ARGUMENT
    with pytest.raises(H.Error) as e:
        gi.search_arrays(queries, 5, 20, traversal=7)
    assert e.value.status == H.Status.INVALID_ARGUMENT
    # The handle still answers exactly afterwards.
    oi = O.Index(data)
    got = gi.search_arrays(queries, 5, 20)
    ref = oi.search(queries, 5, 20)
    np.testing.assert_array_equal(got[0], ref[0])


def test_search_with_options_traversal():
    """SearchOptions.traversal reaches the device path through search_with."""
    base, queries = H.gaussian(3000, 20, 48, 12)
    data = build_index(base, metric=2, m=12, seed=6)
    gi = H.HnswIndex.from_bytes(data)
    arr = gi.search_arrays(queries, 10, 64, traversal=H.Traversal.BF16X3)
    for i in range(len(queries)):
        got = gi.search_with(queries[i], 10, H.SearchOptions(64).traversal(H.Traversal.BF16X3))
        c = int(arr[2][i])
        assert [n.key for n in got] == arr[0][i, :c].tolist()
        assert [np.float32(n.distance).view(np.uint32) for n in got] == arr[1][i, :c].view(np.uint32).tolist()
