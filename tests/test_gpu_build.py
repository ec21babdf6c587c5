"""Device graph construction (hnsw_builder_insert_batch_gpu / compact_gpu).

Parity: a build whose waves are single nodes (max_wave=1) must produce the
same file, byte for byte, as the sequential host insert() sequence
(HnswIndex::insert, src/hnsw/mod.rs:290-302; link, src/hnsw/build.rs:41-150),
for every metric and selection strategy, when extending an existing graph,
when the visited hash spills and when the scratch lives in HBM. Wave builds
are checked as the reference checks its parallel build: structural
invariants and connectivity (src/hnsw/tests.rs:137-166), the recall pins of
tests/recall.rs:43-82, compaction (src/hnsw/tests.rs:266-291), and
determinism (the device plan depends only on the inputs).
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from test_builder_and_abi import assert_invariants, parse, reachable

pytestmark = pytest.mark.gpu

SELECTIONS = [H.NeighborSelection.simple(), H.NeighborSelection(), H.NeighborSelection(True, False, True)]


def cpu_sequential(base, metric, params, keys=None):
    b = H.IndexBuilder(base.shape[1], metric, params)
    keys = np.arange(len(base), dtype=np.uint64) if keys is None else keys
    for i in range(len(base)):
        b.insert(int(keys[i]), base[i])
    return b


def gpu_build(base, metric, params, keys=None, **opts):
    b = H.IndexBuilder(base.shape[1], metric, params)
    keys = np.arange(len(base), dtype=np.uint64) if keys is None else keys
    b.insert_batch_gpu(keys, base, device=0, **opts)
    return b


@pytest.mark.parametrize("metric", [H.Metric.L2, H.Metric.InnerProduct, H.Metric.Cosine])
@pytest.mark.parametrize("sel", range(3))
def test_single_node_waves_equal_sequential_insert(metric, sel):
    base, _ = H.gaussian(1200, 0, 24, 11 + sel)
    params = H.HnswParams(m=8, ef_construction=48, seed=3, selection=SELECTIONS[sel])
    want = cpu_sequential(base, metric, params).to_bytes()
    b = gpu_build(base, metric, params, max_wave=1)
    assert b.to_bytes() == want
    st = b.gpu_stats()
    assert st["inexact"] == 0 and st["waves"] == 1199 and st["nodes"] == 1200
    assert st["shrinks"] > 0


def test_gpu_link_extends_an_existing_graph():
    base, _ = H.mixture(1500, 0, 40, 12, 0.4, 8)
    params = H.HnswParams(m=6, ef_construction=40, seed=9)
    want = cpu_sequential(base, H.Metric.L2, params).to_bytes()
    b = H.IndexBuilder(40, H.Metric.L2, params)
    for i in range(600):
        b.insert(i, base[i])
    b.insert_batch_gpu(np.arange(600, 1500, dtype=np.uint64), base[600:], max_wave=1)
    assert b.to_bytes() == want


def test_visited_spill_and_global_scratch_keep_parity():
    base, _ = H.gaussian(700, 0, 16, 21)
    # A 64-entry hash spills on almost every layer search.
    params = H.HnswParams(m=8, ef_construction=40, seed=1)
    want = cpu_sequential(base, H.Metric.L2, params).to_bytes()
    b = gpu_build(base, H.Metric.L2, params, max_wave=1, hash_cap=64)
    assert b.to_bytes() == want
    assert b.gpu_stats()["spills"] > 0
    # ef_construction beyond what fits on chip: the search scratch lives in HBM.
    base, _ = H.gaussian(400, 0, 8, 22)
    params = H.HnswParams(m=4, ef_construction=12000, seed=2)
    want = cpu_sequential(base, H.Metric.L2, params).to_bytes()
    assert gpu_build(base, H.Metric.L2, params, max_wave=1).to_bytes() == want


def test_wide_rows_and_large_m0():
    base, _ = H.mixture(500, 0, 768, 10, 0.5, 4)
    params = H.HnswParams(m=24, m0=48, ef_construction=64, seed=5)
    want = cpu_sequential(base, H.Metric.Cosine, params).to_bytes()
    assert gpu_build(base, H.Metric.Cosine, params, max_wave=1).to_bytes() == want


def test_upper_layers_with_small_level_multiplier_base():
    # mL = 1 / ln 2: about half the nodes above layer 0, many promotions.
    base, _ = H.gaussian(800, 0, 12, 31)
    params = H.HnswParams(m=4, ef_construction=24, seed=17, level_multiplier=1.0 / np.log(2.0))
    want = cpu_sequential(base, H.Metric.L2, params).to_bytes()
    assert gpu_build(base, H.Metric.L2, params, max_wave=1).to_bytes() == want
    p = parse(gpu_build(base, H.Metric.L2, params).to_bytes())
    assert_invariants(p)


@pytest.mark.parametrize("sel", [0, 1, 2])
def test_wave_builds_satisfy_invariants_and_stay_connected(sel):
    # src/hnsw/tests.rs:137-166 with the device's parallel waves.
    selection = [H.NeighborSelection.simple(), H.NeighborSelection(), H.NeighborSelection(True, True, True)][sel]
    base, _ = H.mixture(3000, 1, 16, 20, 0.35, 5)
    params = H.HnswParams(m=8, selection=selection)
    for frac in (0.02, 0.25):
        data = gpu_build(base, H.Metric.L2, params, wave_fraction=frac).to_bytes()
        p = parse(data)
        assert_invariants(p)
        if selection.heuristic:
            assert reachable(p) >= 2970
        mean_degree = sum(len(p["lists"][i][0]) for i in range(3000)) / 3000
        assert 4.0 < mean_degree <= 16.0
        # The plan depends only on the inputs: the same file every time.
        assert gpu_build(base, H.Metric.L2, params, wave_fraction=frac).to_bytes() == data


def recall_of(data, base, queries, metric=0, k=10, ef=100):
    tk, _, tc, _ = O.brute(metric, base, queries, k)
    gi = H.HnswIndex.from_bytes(data, device=0)
    fk, _, fc, fs = gi.search_arrays(queries, k, ef)
    assert (fs == 0).all()
    return O.recall_at_k(tk, tc, fk, fc, k)


@pytest.fixture(scope="module")
def gaussian_10k():
    return H.gaussian(10_000, 200, 128, 42)


def test_recall_pins_gaussian_10k(gaussian_10k):
    # tests/recall.rs:43-72: M = 32 reaches 0.95 at ef = 100; M = 16 stays
    # within 0.02 of hnswlib's 0.889.
    base, queries = gaussian_10k
    keys = np.arange(10_000, dtype=np.uint64)
    r32 = recall_of(gpu_build(base, H.Metric.L2, H.HnswParams(m=32), keys).to_bytes(), base, queries)
    r16 = recall_of(gpu_build(base, H.Metric.L2, H.HnswParams(m=16), keys).to_bytes(), base, queries)
    assert r32 >= 0.95, r32
    assert abs(r16 - 0.889) <= 0.02, r16


def test_recall_pin_clustered_10k():
    # tests/recall.rs:74-82.
    base, queries = H.mixture(10_000, 200, 128, 50, 0.35, 42)
    r = recall_of(gpu_build(base, H.Metric.L2, H.HnswParams(m=16)).to_bytes(), base, queries)
    assert r >= 0.95, r


def test_sequential_device_build_at_10k_equals_host(gaussian_10k):
    base, _ = gaussian_10k
    params = H.HnswParams(m=16, ef_construction=100)
    want = cpu_sequential(base[:4000], H.Metric.L2, params).to_bytes()
    assert gpu_build(base[:4000], H.Metric.L2, params, max_wave=1).to_bytes() == want


def test_compact_gpu_drops_tombstones_and_keeps_live_keys():
    # src/hnsw/tests.rs:266-291 with the device link step.
    base, queries = H.gaussian(1000, 20, 16, 6)
    params = H.HnswParams()

    def tombstoned():
        b = cpu_sequential(base, H.Metric.L2, params)
        b.enable_quantization()
        for key in range(0, 1000, 3):
            assert b.remove(key)
        return b

    b = tombstoned()
    b.compact_gpu(device=0)
    data = b.to_bytes()
    info = H.validate_bytes(data)
    live = 1000 - len(range(0, 1000, 3))
    assert (info.nodes, info.live, info.quantized) == (live, live, 1)
    p = parse(data)
    assert_invariants(p)
    assert reachable(p) * 100 >= live * 99
    keep = np.array([k for k in range(1000) if k % 3 != 0], np.uint64)
    tk, _, tc, _ = O.brute(0, base[keep.astype(np.int64)], queries, 10, keys=keep)
    gi = H.HnswIndex.from_bytes(data, device=0)
    fk, _, fc, _ = gi.search_arrays(queries, 10, 100)
    assert O.recall_at_k(tk, tc, fk, fc, 10) > 0.95
    # With single-node waves the device compaction equals the host's.
    a = tombstoned()
    a.compact(threads=1)
    c = tombstoned()
    c.compact_gpu(device=0, max_wave=1)
    assert a.to_bytes() == c.to_bytes()
    # Without tombstones compaction changes nothing.
    before = c.to_bytes()
    c.compact_gpu(device=0)
    assert c.to_bytes() == before


def test_errors_leave_the_builder_unchanged():
    base, _ = H.gaussian(300, 0, 8, 2)
    b = H.IndexBuilder(8, H.Metric.Cosine, H.HnswParams(m=4))
    b.insert_batch_gpu(np.arange(200, dtype=np.uint64), base[:200])
    before = b.to_bytes()
    bad = base[200:].copy()
    bad[5, 3] = np.nan
    with pytest.raises(H.Error) as e:
        b.insert_batch_gpu(np.arange(200, 300, dtype=np.uint64), bad)
    assert e.value.status == H.Status.NON_FINITE_VECTOR
    zero = base[200:].copy()
    zero[7] = 0.0
    with pytest.raises(H.Error) as e:
        b.insert_batch_gpu(np.arange(200, 300, dtype=np.uint64), zero)
    assert e.value.status == H.Status.ZERO_VECTOR
    with pytest.raises(H.Error) as e:
        b.insert_batch_gpu(np.arange(150, 250, dtype=np.uint64), base[200:])
    assert e.value.status == H.Status.DUPLICATE_KEY
    with pytest.raises(H.Error) as e:
        b.insert_batch_gpu(np.arange(200, 300, dtype=np.uint64), base[200:], wave_fraction=0.0)
    assert e.value.status == H.Status.INVALID_ARGUMENT
    assert b.to_bytes() == before
    b.insert_batch_gpu(np.arange(200, 300, dtype=np.uint64), base[200:])
    assert_invariants(parse(b.to_bytes()))
