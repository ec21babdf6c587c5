"""The oracle's restatement of construction (HnswIndex::insert /
insert_batch, src/hnsw/build.rs:19-222, src/hnsw/mod.rs:318-349) and of the
split mixture generator, against the product's host builder and generator.

Linking one node at a time in id order is deterministic, so the oracle's
sequential build and the product's sequential `insert` sequence must write
the same format-v1 file byte for byte, for every metric and selection
strategy. A parallel build (nondeterministic, as the reference's is,
mod.rs:306-312) must give a file the product's validating loader accepts,
with the same recall as the sequential one within a small margin. The recall
pins of tests/recall.rs (0.9620 / 0.8900) are checked on the oracle's own
builder in test_oracle_golden.py.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O


def _product_sequential(base, metric, m, efc, seed, selection=None, keys=None):
    n, dim = base.shape
    keys = np.arange(n, dtype=np.uint64) if keys is None else keys
    b = H.IndexBuilder(dim, H.Metric(metric), H.HnswParams(m=m, ef_construction=efc, seed=seed, selection=selection))
    for i in range(n):
        b.insert(int(keys[i]), base[i])
    return b.to_bytes()


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_sequential_build_is_byte_identical_to_the_product_builder(metric):
    base, _ = H.mixture(2500, 0, 20, 12, 0.4, 30 + metric)
    keys = (np.arange(2500, dtype=np.uint64) * np.uint64(104729)) ^ np.uint64(1 << 62)
    prod = _product_sequential(base, metric, 8, 60, 11, keys=keys)
    orc = O.build(base, keys=keys, metric=metric, m=8, ef_construction=60, seed=11, threads=1)
    assert prod == orc


@pytest.mark.parametrize("extend,keep", [(False, False), (True, False), (False, True), (True, True)])
def test_sequential_build_selection_variants(extend, keep):
    base, _ = H.gaussian(1200, 0, 12, 9)
    sel = H.NeighborSelection(heuristic=True, extend_candidates=extend, keep_pruned=keep)
    prod = _product_sequential(base, 0, 6, 40, 3, selection=sel)
    orc = O.build(base, metric=0, m=6, ef_construction=40, seed=3, selection=1, extend_candidates=extend,
                  keep_pruned=keep, threads=1)
    assert prod == orc


def test_sequential_build_simple_selection():
    base, _ = H.gaussian(1000, 0, 10, 4)
    prod = _product_sequential(base, 1, 5, 30, 8, selection=H.NeighborSelection.simple())
    orc = O.build(base, metric=1, m=5, ef_construction=30, seed=8, selection=0, threads=1)
    assert prod == orc


def test_parallel_build_validates_and_keeps_recall():
    base, queries = O.mixture_split(6000, 200, 32, 30, 0.4, 5, 6)
    par = O.build(base, metric=0, m=12, ef_construction=100, seed=2, threads=4)
    seq = O.build(base, metric=0, m=12, ef_construction=100, seed=2, threads=1)
    H.validate_bytes(par)
    H.validate_bytes(seq)
    tk, _, tc, _ = O.brute(0, base, queries, 10)
    r = []
    for data in (par, seq):
        k, d, c, s = O.Index(data).search(queries, 10, 64)
        r.append(O.recall_at_k(tk, tc, k, c, 10))
    assert abs(r[0] - r[1]) <= 0.02 and r[0] >= 0.9


def test_tombstones_in_the_written_file():
    base, queries = H.gaussian(800, 20, 8, 2)
    dead = [3, 100, 799]
    orc = O.build(base, metric=0, m=6, ef_construction=40, seed=1, threads=1, deleted_keys=dead)
    b = H.IndexBuilder(8, H.Metric.L2, H.HnswParams(m=6, ef_construction=40, seed=1))
    for i in range(800):
        b.insert(i, base[i])
    for k in dead:
        b.remove(k)
    assert b.to_bytes() == orc
    k, _, c, _ = O.Index(orc).search(queries, 5, 40)
    assert not np.isin(k[:, :5], np.array(dead, np.uint64)).any()


def test_split_mixture_equals_the_product_generator():
    for args in ((3000, 100, 16, 25, 0.3, 1, 2), (777, 13, 7, 3, 0.5, 9, 10), (0, 5, 4, 2, 1.0, 3, 4)):
        a = O.mixture_split(*args)
        b = H.mixture_split(*args)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
