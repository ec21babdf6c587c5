"""GPU HNSW search vs the CPU oracle, through the C ABI.

The bar is bit-exact: the same keys, the same f32 distance bits and the same
counts as the oracle's restatement of HnswIndex::search_batch / search_with
(src/hnsw/mod.rs:412-536) on the same index file and queries. The integer
and visited/filter/tombstone logic is exact by construction, and distances
are computed in the reference AVX2 kernel order, so no tolerance is needed.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from conftest import build_index

pytestmark = pytest.mark.gpu


def assert_same(gpu, ref, label=""):
    gk, gd, gc, gs = gpu
    rk, rd, rc, rs = ref
    np.testing.assert_array_equal(gs, rs, err_msg=f"{label}: status")
    np.testing.assert_array_equal(gc, rc, err_msg=f"{label}: counts")
    for i in range(len(gc)):
        c = int(gc[i])
        np.testing.assert_array_equal(gk[i, :c], rk[i, :c], err_msg=f"{label}: keys of query {i}")
        np.testing.assert_array_equal(gd[i, :c].view(np.uint32), rd[i, :c].view(np.uint32),
                                      err_msg=f"{label}: distance bits of query {i}")


@pytest.fixture(scope="module")
def gaussian_10k():
    """10k x 128 N(0,1) base from seed 42, queries from seed 43, L2, M=16, level seed 7."""
    base, _ = H.gaussian(10_000, 0, 128, 42)
    _, queries = H.gaussian(0, 1000, 128, 43)
    data = build_index(base, metric=0, m=16, seed=7)
    return base, queries, data


def test_gaussian_10k_bit_exact(gaussian_10k):
    base, queries, data = gaussian_10k
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    gpu = gi.search_arrays(queries, 10, 64)
    ref = oi.search(queries, 10, 64)
    assert_same(gpu, ref, "gaussian 10k x 128")
    tk, _, tc, _ = O.brute(0, base, queries, 10)
    r_gpu = O.recall_at_k(tk, tc, gpu[0], gpu[2], 10)
    r_ref = O.recall_at_k(tk, tc, ref[0], ref[2], 10)
    assert r_gpu == r_ref


@pytest.mark.parametrize("ef", [1, 10, 16, 32, 100, 128, 256, 512])
def test_ef_sweep_bit_exact(gaussian_10k, ef):
    _, queries, data = gaussian_10k
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    assert_same(gi.search_arrays(queries[:300], 10, ef), oi.search(queries[:300], 10, ef), f"ef={ef}")


def test_persistent_mode_matches_plain(gaussian_10k):
    _, queries, data = gaussian_10k
    gi = H.HnswIndex.from_bytes(data)
    a = gi.search_arrays(queries, 10, 64, mode=0)
    b = gi.search_arrays(queries, 10, 64, mode=1)
    assert_same(a, b, "persistent")


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [1, 7, 8, 31, 33, 40, 96])
def test_metrics_and_dims(metric, dim):
    base, queries = H.gaussian(1500, 40, dim, 100 + dim)
    if metric == 2:
        base[:, 0] += np.where(base[:, 0] >= 0, 1.0, -1.0)
        queries[:, 0] += 1.0
    data = build_index(base, metric=metric, m=8, seed=3)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    assert_same(gi.search_arrays(queries, 7, 20), oi.search(queries, 7, 20), f"metric={metric} dim={dim}")


def test_m0_above_32_and_large_k():
    base, queries = H.mixture(4000, 60, 24, 40, 0.4, 9)
    data = build_index(base, metric=1, m=24, seed=5)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    for k, ef in [(1, 16), (10, 64), (100, 100), (100, 300)]:
        assert_same(gi.search_arrays(queries, k, ef), oi.search(queries, k, ef), f"k={k} ef={ef}")


def test_complete_graph_equals_brute_force():
    """src/hnsw/tests.rs:113-127: n <= M with simple selection is exhaustive."""
    base, queries = H.gaussian(16, 20, 8, 3)
    data = build_index(base, metric=0, m=16, seed=0, parallel=False,
                       selection=H.NeighborSelection.simple())
    gi = H.HnswIndex.from_bytes(data)
    got = gi.search_arrays(queries, 5, 5)
    tk, td, tc, ts = O.brute(0, base, queries, 5)
    np.testing.assert_array_equal(got[0], tk)
    np.testing.assert_array_equal(got[1].view(np.uint32), td.view(np.uint32))


def test_tombstones_including_entry_point():
    """src/hnsw/tests.rs:220-248."""
    base, queries = H.gaussian(300, 5, 8, 9)
    data0 = build_index(base, metric=0, m=16, seed=0, parallel=False)
    info = H.validate_bytes(data0)
    entry_key = info.entry  # keys are ids here
    deleted = set(range(0, 300, 2)) | {entry_key}
    data = build_index(base, metric=0, m=16, seed=0, parallel=False, deleted_keys=sorted(deleted))
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    got = gi.search_arrays(queries, 20, 50)
    assert_same(got, oi.search(queries, 20, 50), "tombstones")
    for i in range(len(queries)):
        assert got[2][i] == 20
        assert all(int(k) % 2 == 1 and int(k) != entry_key for k in got[0][i, :20])


def test_removing_everything_gives_empty_results():
    base, queries = H.gaussian(50, 1, 4, 4)
    data = build_index(base, metric=0, parallel=False, deleted_keys=range(50))
    gi = H.HnswIndex.from_bytes(data)
    assert gi.search(queries[0], 5, 10) == []


def test_filters_during_traversal():
    """src/hnsw/tests.rs:293-313, plus the retry path for selective filters."""
    base, queries = H.gaussian(2000, 10, 8, 8)
    data = build_index(base, metric=0, parallel=False)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    nbits = 2000
    keys = np.arange(2000, dtype=np.uint64)
    for accepted, k, ef in [(keys[keys % 10 == 3], 10, 64), (np.array([1234], np.uint64), 3, 10),
                            (np.zeros(0, np.uint64), 3, 10), (keys[keys % 100 == 7], 10, 32),
                            (keys[keys % 3 == 0], 50, 200)]:
        bits = H.key_bitmap(accepted, nbits)
        got = gi.search_arrays(queries, k, ef, filter_bits=bits, filter_nbits=nbits)
        ref = oi.search(queries, k, ef, filter_bits=bits, filter_nbits=nbits)
        assert_same(got, ref, f"filter {accepted.size} keys")
    only = gi.search_filtered(queries[0], 3, 10, lambda k: k == 1234)
    assert [n.key for n in only] == [1234]
    assert gi.search_filtered(queries[0], 3, 10, lambda k: False) == []


def test_per_query_filters_k_ef():
    base, queries = H.mixture(3000, 64, 16, 20, 0.5, 4)
    data = build_index(base, metric=0, m=12, seed=2)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    rng = np.random.default_rng(0)
    nbits = 3000
    words = (nbits + 63) // 64
    bits = np.zeros((64, words), np.uint64)
    for i in range(64):
        sel = rng.random(3000) < rng.uniform(0.01, 0.9)
        bits[i] = H.key_bitmap(np.nonzero(sel)[0].astype(np.uint64), nbits)
    used = (rng.random(64) < 0.7).astype(np.uint8)
    ks = rng.choice([1, 10, 100], 64).astype(np.uint32)
    efs = rng.choice([16, 32, 64, 128, 256], 64).astype(np.uint32)
    got = gi.search_arrays(queries, 100, 16, filter_bits=bits, filter_nbits=nbits, filter_stride=words,
                           filter_used=used, ks=ks, efs=efs)
    ref = oi.search(queries, 100, 16, filter_bits=bits, filter_nbits=nbits, filter_stride=words,
                    filter_used=used, ks=ks, efs=efs)
    assert_same(got, ref, "per-query")


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_quantized_traversal_and_exact_rerank(metric):
    """src/hnsw/tests.rs:336-368: reported distances are exact."""
    base, queries = H.gaussian(2000, 20, 32, 12)
    data = build_index(base, metric=metric, parallel=False, quantize=True)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    got = gi.search_arrays(queries, 10, 64, quantized=True)
    assert_same(got, oi.search(queries, 10, 64, quantized=True), "quantized")
    # Distances equal the exact metric recomputed by the reference kernel.
    pq = queries if metric != 2 else O.normalize_rows(queries)
    stored = base if metric != 2 else O.normalize_rows(base)
    for i in range(len(queries)):
        for j in range(int(got[2][i])):
            want = O.distance(metric, pq[i], stored[int(got[0][i, j])])
            assert np.float32(got[1][i, j]).view(np.uint32) == want.view(np.uint32)


def test_quantization_disabled_status():
    base, queries = H.gaussian(200, 2, 8, 1)
    data = build_index(base)
    gi = H.HnswIndex.from_bytes(data)
    with pytest.raises(H.Error) as e:
        gi.search_arrays(queries, 5, 10, quantized=True)
    assert e.value.status == H.Status.QUANTIZATION_DISABLED


def test_invalid_queries_have_statuses():
    base, _ = H.gaussian(300, 0, 4, 2)
    data = build_index(base, metric=2)
    gi = H.HnswIndex.from_bytes(data)
    # 6.521909e18 squared lies between f32::MAX / 8 and 2^125: rejected (src/vector.rs:16,36-38).
    q = np.array([[1, 0, 0, 0], [np.nan, 1, 0, 0], [0, 0, 0, 0], [3e19, 0, 0, 0], [np.inf, 0, 0, 0],
                  [6.521909e18, 0, 0, 0]], np.float32)
    keys, dist, count, status = gi.search_arrays(q, 3, 10, raise_on_error=False)
    assert list(status) == [0, 3, 4, 3, 3, 3]
    assert O.prepare_query(2, q[5])[0] == 3
    assert count[0] == 3 and all(count[1:] == 0)
    with pytest.raises(H.Error):
        gi.search(q[1], 3, 10)
    with pytest.raises(H.Error) as e:
        gi.search_batch(np.zeros(6, np.float32), 3, 10)
    assert e.value.status == H.Status.DIMENSION_MISMATCH


def test_k_and_ef_edge_cases():
    """src/hnsw/tests.rs:208-218."""
    base, queries = H.gaussian(100, 1, 4, 2)
    data = build_index(base, parallel=False)
    gi = H.HnswIndex.from_bytes(data)
    assert gi.search(queries[0], 0, 10) == []
    assert len(gi.search(queries[0], 10, 1)) == 10
    assert len(gi.search(queries[0], 500, 500)) == 100


def test_inner_product_and_cosine_known_answers():
    """src/hnsw/tests.rs:370-388."""
    b = H.IndexBuilder(2, H.Metric.InnerProduct)
    b.insert_batch(np.array([1, 2, 3], np.uint64), np.array([[1, 0], [3, 0], [0, 1]], np.float32))
    ip = H.HnswIndex.from_bytes(b.to_bytes())
    hits = ip.search([1.0, 0.0], 3, 10)
    assert [h.key for h in hits] == [2, 1, 3]
    assert hits[0].distance == -3.0
    c = H.IndexBuilder(2, H.Metric.Cosine)
    c.insert_batch(np.array([1, 2], np.uint64), np.array([[10, 0], [1, 1]], np.float32))
    cos = H.HnswIndex.from_bytes(c.to_bytes())
    hits = cos.search([0.1, 0.0], 2, 10)
    assert hits[0].key == 1 and abs(hits[0].distance) < 1e-6
    assert abs(hits[1].distance - (1.0 - np.float32(np.sqrt(0.5)))) < 1e-6


def test_empty_index():
    b = H.IndexBuilder(3, H.Metric.L2)
    gi = H.HnswIndex.from_bytes(b.to_bytes())
    assert gi.search([0.0, 0.0, 0.0], 5, 10) == []


def test_concurrent_searches_match(gaussian_10k):
    """tests/concurrency.rs:22-58: many host threads on one handle."""
    import threading

    _, queries, data = gaussian_10k
    gi = H.HnswIndex.from_bytes(data)
    want = gi.search_arrays(queries[:200], 10, 48)
    errors = []

    def worker(t):
        try:
            for _ in range(3):
                got = gi.search_arrays(queries[:200], 10, 48)
                assert_same(got, want, f"thread {t}")
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors[0]


def test_search_batch_equals_individual_searches():
    """tests/concurrency.rs:61-70."""
    base, queries = H.gaussian(2000, 50, 16, 5)
    data = build_index(base, parallel=False)
    gi = H.HnswIndex.from_bytes(data)
    batch = gi.search_batch(queries, 10, 40)
    for i in range(len(queries)):
        assert batch[i] == gi.search(queries[i], 10, 40)
    with pytest.raises(H.Error):
        gi.search_batch(queries.reshape(-1)[:15], 10, 40)


def test_set_tombstones_on_device():
    base, queries = H.gaussian(1000, 30, 16, 21)
    data = build_index(base, parallel=False)
    gi = H.HnswIndex.from_bytes(data)
    dead = np.zeros(1000, np.uint8)
    dead[::3] = 1
    gi.set_tombstones(dead)
    data2 = build_index(base, parallel=False, deleted_keys=range(0, 1000, 3))
    oi = O.Index(data2)
    assert_same(gi.search_arrays(queries, 10, 40), oi.search(queries, 10, 40), "device tombstones")


@pytest.mark.parametrize("mode", [0, 1])
def test_visited_and_candidate_overflow_paths(mode):
    """A 0.5%-selective filter with ef=32 cannot fill the results, so every
    query visits the whole connected graph: the shared-memory visited hash and
    candidate array overflow. Plain mode re-runs such queries in the retry
    kernel; persistent mode continues them in per-warp global spill areas."""
    base, queries = H.gaussian(5000, 48, 16, 77)
    data = build_index(base, metric=0, m=8, seed=1)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    keys = np.arange(5000, dtype=np.uint64)
    for accepted, k, ef in [(keys[keys % 200 == 11], 10, 32), (keys[keys % 7 == 0], 10, 32),
                            (keys[keys % 50 == 3], 25, 64)]:
        bits = H.key_bitmap(accepted, 5000)
        got = gi.search_arrays(queries, k, ef, filter_bits=bits, filter_nbits=5000, mode=mode)
        ref = oi.search(queries, k, ef, filter_bits=bits, filter_nbits=5000)
        assert_same(got, ref, f"mode={mode} filter={accepted.size}")
    # The same handle keeps giving exact answers after spilled queries.
    assert_same(gi.search_arrays(queries, 10, 40, mode=mode), oi.search(queries, 10, 40), "after spill")


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("quant", [False, True])
def test_distance_ties_bit_exact(mode, quant):
    """Small-integer points with ~40 copies each: most distances tie, so the
    heap order falls back to ids (src/hnsw/search.rs:36-44) and results that
    tie with the worst one are evicted unexpanded. Unfiltered batches take the
    single-array layer-0 variant, whose tie list overflows here and sends
    those queries to the retry pass; every answer must still be the oracle's."""
    rng = np.random.default_rng(11)
    base = rng.integers(0, 3, size=(3000, 4)).astype(np.float32)
    queries = np.vstack([rng.integers(0, 3, size=(150, 4)), rng.integers(-1, 4, size=(50, 4))]).astype(np.float32)
    data = build_index(base, metric=0, m=8, seed=3, quantize=quant)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    for k, ef in [(1, 1), (10, 16), (10, 40), (32, 64), (50, 200)]:
        got = gi.search_arrays(queries, k, ef, mode=mode, quantized=quant)
        assert_same(got, oi.search(queries, k, ef, quantized=quant), f"k={k} ef={ef}")


@pytest.mark.parametrize("mode", [0, 1])
def test_modes_on_quantized_filtered_tombstoned_mixture(mode):
    base, queries = H.mixture(6000, 96, 32, 30, 0.4, 8)
    rng = np.random.default_rng(5)
    dead = np.nonzero(rng.random(6000) < 0.05)[0]
    data = build_index(base, metric=1, m=12, seed=4, deleted_keys=dead, quantize=True)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    words = (6000 + 63) // 64
    bits = np.zeros((96, words), np.uint64)
    for i in range(96):
        sel = rng.random(6000) < np.exp(rng.uniform(np.log(0.01), np.log(0.9)))
        bits[i] = H.key_bitmap(np.nonzero(sel)[0].astype(np.uint64), 6000)
    ks = rng.choice([1, 10, 100], 96).astype(np.uint32)
    efs = rng.choice([16, 32, 64, 128, 256, 512], 96).astype(np.uint32)
    got = gi.search_arrays(queries, 100, 16, quantized=True, filter_bits=bits, filter_nbits=6000,
                           filter_stride=words, ks=ks, efs=efs, mode=mode)
    ref = oi.search(queries, 100, 16, quantized=True, filter_bits=bits, filter_nbits=6000,
                    filter_stride=words, ks=ks, efs=efs)
    assert_same(got, ref, f"IP mixture, int8, filters, tombstones, mode={mode}")


def test_shared_filter_bitmaps_by_id():
    base, queries = H.gaussian(3000, 64, 16, 12)
    data = build_index(base, metric=0, m=12, seed=2)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    rng = np.random.default_rng(9)
    words = (3000 + 63) // 64
    bank = np.zeros((5, words), np.uint64)
    for j in range(5):
        bank[j] = H.key_bitmap(np.nonzero(rng.random(3000) < 0.1 * (j + 1))[0].astype(np.uint64), 3000)
    ids = rng.integers(0, 5, 64).astype(np.uint32)
    got = gi.search_arrays(queries, 10, 48, filter_bits=bank, filter_nbits=3000, filter_stride=words, filter_ids=ids)
    ref = oi.search(queries, 10, 48, filter_bits=bank[ids], filter_nbits=3000, filter_stride=words)
    assert_same(got, ref, "filter ids")


def test_node_bitmaps_for_sparse_u64_keys():
    """Closure filters on keys far above the node count (src/hnsw/mod.rs:432-440):
    the bitmap is indexed by node id, so its size is the node count."""
    base, queries = H.gaussian(2500, 40, 24, 14)
    rng = np.random.default_rng(15)
    keys = np.unique(rng.integers(1 << 40, 1 << 63, 2600, dtype=np.uint64))[:2500]
    rng.shuffle(keys)
    data = build_index(base, metric=0, m=12, seed=3, keys=keys, deleted_keys=keys[:40:3])
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    for pred, k, ef in [(lambda key: key % 7 == 1, 10, 64), (lambda key: key >= (1 << 62), 5, 32),
                        (lambda key: False, 3, 10)]:
        for i in range(0, 40, 13):
            got = gi.search_filtered(queries[i], k, ef, pred)
            ref = oi.search(queries[i:i + 1], k, ef, filter_bits=gi._filter_bits(pred)[0], filter_nbits=2500,
                            filter_by_node=True)
            c = int(ref[2][0])
            assert [n.key for n in got] == ref[0][0, :c].tolist()
            assert all(pred(n.key) for n in got)
    # Per-query node bitmaps through the batched entry point.
    words = (2500 + 63) // 64
    bank = np.zeros((40, words), np.uint64)
    for j in range(40):
        bank[j] = H.key_bitmap(np.nonzero(rng.random(2500) < 0.2)[0].astype(np.uint64), 2500)
    got = gi.search_arrays(queries, 10, 48, filter_bits=bank, filter_nbits=2500, filter_stride=words,
                           filter_by_node=True, mode=1)
    ref = oi.search(queries, 10, 48, filter_bits=bank, filter_nbits=2500, filter_stride=words, filter_by_node=True)
    assert_same(got, ref, "node bitmaps")


@pytest.mark.parametrize("mode", [0, 1])
def test_cold_candidate_list_under_selective_filters(mode):
    """Filters so selective that ef results never fill: the beam explores
    most of the graph and the candidate queue grows towards the node count
    (the reference's heap is unbounded). The queue's cold list, its refills
    and the evictions of the array's upper half must not change a result."""
    base, queries = H.mixture(20000, 48, 16, 40, 0.4, 31)
    data = build_index(base, metric=0, m=8, seed=5, deleted_keys=range(0, 20000, 97))
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    rng = np.random.default_rng(32)
    nbits, words = 20000, (20000 + 63) // 64
    sels = [0.0003, 0.002, 0.01, 0.05, 0.3]
    bank = np.zeros((len(sels), words), np.uint64)
    for j, p in enumerate(sels):
        bank[j] = H.key_bitmap(np.nonzero(rng.random(nbits) < p)[0].astype(np.uint64), nbits)
    ids = rng.integers(0, len(sels), 48).astype(np.uint32)
    ks = rng.choice([1, 10, 100], 48).astype(np.uint32)
    efs = rng.choice([16, 64, 256, 512], 48).astype(np.uint32)
    ref = oi.search(queries, 100, 16, filter_bits=bank[ids], filter_nbits=nbits, filter_stride=words, ks=ks, efs=efs)
    # cold_chunks=1: the shared pools run dry at once, so the queries end in
    # the last-resort pass (private regions).
    for sched in [None, dict(ef_cap=512, cand_cap=512, hash_cap=4096, warps_per_block=2),
                  dict(ef_cap=512, cand_cap=512, hash_cap=4096, warps_per_block=2, cold=1),
                  dict(ef_cap=512, cand_cap=1056, hash_cap=8192, warps_per_block=1, cold_chunks=1),
                  dict(ef_cap=512, cand_cap=1056, hash_cap=8192, warps_per_block=1, cold_chunks=1, cold=1)]:
        if sched:
            gi.set_schedule(**sched)
        got = gi.search_arrays(queries, 100, 16, filter_bits=bank, filter_nbits=nbits, filter_stride=words,
                               filter_ids=ids, ks=ks, efs=efs, mode=mode)
        assert_same(got, ref, f"schedule {sched}")
    # The smallest arrays: every few insertions move half the queue to the cold list.
    small = np.minimum(efs, 64).astype(np.uint32)
    ks_small = np.minimum(ks, 10).astype(np.uint32)
    ref = oi.search(queries, 10, 16, filter_bits=bank[ids], filter_nbits=nbits, filter_stride=words, ks=ks_small,
                    efs=small)
    for cold in (0, 1):
        gi.set_schedule(ef_cap=64, cand_cap=64, hash_cap=1024, warps_per_block=4, cold=cold)
        got = gi.search_arrays(queries, 10, 16, filter_bits=bank, filter_nbits=nbits, filter_stride=words,
                               filter_ids=ids, ks=ks_small, efs=small, mode=mode)
        assert_same(got, ref, f"cand_cap 64, cold {cold}")
    gi.set_schedule()


def test_fixed_schedule_gives_identical_results(gaussian_10k):
    _, queries, data = gaussian_10k
    gi = H.HnswIndex.from_bytes(data)
    want = gi.search_arrays(queries[:200], 10, 64, mode=1)
    for ef_cap, hash_cap, wpb, stage in [(512, 32768, 1, 0), (64, 1024, 4, 0), (128, 4096, 2, 0), (64, 2048, 4, 16),
                                         (128, 4096, 2, 32), (64, 2048, 1, 5)]:
        gi.set_schedule(ef_cap=ef_cap, hash_cap=hash_cap, warps_per_block=wpb, stage_rows=stage)
        for mode in (0, 1):
            assert_same(gi.search_arrays(queries[:200], 10, 64, mode=mode), want, f"schedule {ef_cap}/{hash_cap}")
    gi.set_schedule()


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [7, 33, 96])
def test_staged_gathers_match_oracle(metric, dim):
    """Rows gathered into shared memory by cp.async: f32 and int8 traversal,
    upper layers and layer 0, every metric, dims with scalar tails."""
    base, queries = H.mixture(3000, 40, dim, 30, 0.5, 200 + dim)
    if metric == 2:
        base[:, 0] += np.where(base[:, 0] >= 0, 1.0, -1.0)
        queries[:, 0] += 1.0
    data = build_index(base, metric=metric, m=12, seed=3, quantize=True)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    for stage, wpb in [(32, 2), (8, 4), (3, 1)]:
        gi.set_schedule(ef_cap=128, hash_cap=4096, warps_per_block=wpb, stage_rows=stage)
        for quant in (False, True):
            for mode in (0, 1):
                got = gi.search_arrays(queries, 10, 100, quantized=quant, mode=mode)
                assert_same(got, oi.search(queries, 10, 100, quantized=quant), f"stage {stage} quant {quant}")
    gi.set_schedule()


def test_autotune_installs_schedules_without_changing_results(gaussian_10k):
    _, queries, data = gaussian_10k
    gi = H.HnswIndex.from_bytes(data)
    sample = queries[:300]
    want = gi.search_arrays(sample, 10, 64, mode=1)
    best, trials = gi.autotune(sample, 10, 64, reps=2)
    assert len(trials) > 8
    assert {t["mode"] for t in trials} == {0, 1}
    assert sum(t["heuristic"] for t in trials) == 2
    assert all(t["ms"] > 0 for t in trials)
    assert best["ms"] == min(t["ms"] for t in trials)
    for mode in (H.MODE_PLAIN, H.MODE_PERSISTENT, H.MODE_AUTO):
        assert_same(gi.search_arrays(sample, 10, 64, mode=mode), want, f"tuned, mode {mode}")
    # A filtered batch with per-query k and ef, tuned in its own bucket.
    rng = np.random.default_rng(4)
    bits = H.key_bitmap(np.nonzero(rng.random(10_000) < 0.2)[0].astype(np.uint64), 10_000)
    efs = rng.choice([32, 100, 200], 300).astype(np.uint32)
    kw = dict(filter_bits=bits, filter_nbits=10_000, efs=efs)
    want_f = gi.search_arrays(sample, 10, 16, mode=0, **kw)
    gi.autotune(sample, 10, 16, reps=1, **kw)
    assert_same(gi.search_arrays(sample, 10, 16, mode=H.MODE_AUTO, **kw), want_f, "tuned filtered")
    gi.clear_tuning()
    assert_same(gi.search_arrays(sample, 10, 64, mode=H.MODE_AUTO), want, "after clear")


def test_cuda_graph_replays_the_search(gaussian_10k):
    import torch

    _, queries, data = gaussian_10k
    gi = H.HnswIndex.from_bytes(data)
    want = gi.search_arrays(queries[:256], 10, 64)
    dev = torch.device("cuda", 0)
    q = torch.zeros((256, 128), dtype=torch.float32, device=dev)
    keys = torch.zeros((256, 10), dtype=torch.int64, device=dev)
    dist = torch.zeros((256, 10), dtype=torch.float32, device=dev)
    cnt = torch.zeros(256, dtype=torch.int32, device=dev)
    st = torch.zeros(256, dtype=torch.int32, device=dev)
    g = gi.graph(q.data_ptr(), 256, 10, 64, keys.data_ptr(), dist.data_ptr(), cnt.data_ptr(), st.data_ptr())
    for _ in range(2):
        q.copy_(torch.from_numpy(queries[:256]))
        torch.cuda.synchronize()
        g.launch()
        torch.cuda.synchronize()
        got = (keys.cpu().numpy().view(np.uint64), dist.cpu().numpy(), cnt.cpu().numpy().view(np.uint32),
               st.cpu().numpy())
        assert_same(got, want, "graph")
    g.close()


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("quant", [False, True])
def test_planner_exact_scan_for_selective_filters(metric, quant):
    """Queries whose filter admits few nodes get the exact top-k among the
    admitted live nodes (BruteForceIndex::search_filtered on the index's own
    rows); the others keep the graph walk's results."""
    base, queries = H.mixture(6000, 48, 20, 30, 0.5, 300 + metric)
    if metric == 2:
        base[:, 0] += np.where(base[:, 0] >= 0, 1.0, -1.0)
        queries[:, 0] += 1.0
    dead = list(range(0, 6000, 37))
    data = build_index(base, metric=metric, m=10, seed=4, deleted_keys=dead, quantize=True)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    rng = np.random.default_rng(metric)
    words = (6000 + 63) // 64
    sels = [0.002, 0.01, 0.03, 0.5]
    bank = np.zeros((len(sels), words), np.uint64)
    for j, p in enumerate(sels):
        bank[j] = H.key_bitmap(np.nonzero(rng.random(6000) < p)[0].astype(np.uint64), 6000)
    ids = rng.integers(0, len(sels), 48).astype(np.uint32)
    kw = dict(filter_bits=bank, filter_nbits=6000, filter_stride=words, filter_ids=ids, quantized=quant)
    got = gi.search_arrays(queries, 10, 40, exact_below=0.05, mode=1, **kw)
    graph = oi.search(queries, 10, 40, filter_bits=bank[ids], filter_nbits=6000, filter_stride=words, quantized=quant)
    alive = np.ones(6000, bool)
    alive[dead] = False
    rows = base if metric != 2 else O.normalize_rows(base)
    live_bank = bank.copy()
    for j in range(len(sels)):
        live_bank[j] = H.key_bitmap(np.nonzero(np.unpackbits(bank[j].view(np.uint8), bitorder="little")[:6000]
                                               .astype(bool) & alive)[0].astype(np.uint64), 6000)
    exact = O.brute_filtered(metric, rows, queries, 10, live_bank[ids], 6000, words)
    planned = 0
    for i in range(48):
        admitted = int(np.unpackbits(bank[ids[i]].view(np.uint8), bitorder="little")[:6000].sum())
        ref = exact if admitted <= int(0.05 * len(alive[alive])) else graph
        planned += ref is exact
        c = int(ref[2][i])
        assert int(got[2][i]) == c
        np.testing.assert_array_equal(got[0][i, :c], ref[0][i, :c])
        np.testing.assert_array_equal(got[1][i, :c].view(np.uint32), ref[1][i, :c].view(np.uint32))
    assert 0 < planned < 48
