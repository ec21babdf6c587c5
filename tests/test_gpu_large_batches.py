"""Large host-buffer batches (4096-9000 queries) with every per-query input
(k, ef, filter flags, bitmap ids, per-query bitmaps, one shared bitmap) and
invalid queries late in the batch: the arrays must equal the oracle's
restatement of HnswIndex::search_batch / search_with
(src/hnsw/mod.rs:448-536) bit for bit, statuses included, and the call's
error is the first failing query's status."""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from conftest import build_index
from test_gpu_search import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mix():
    base, queries = H.mixture(4000, 9000, 24, 30, 0.5, 21)
    data = build_index(base, metric=0, m=8, seed=5)
    return base, queries, data


@pytest.mark.parametrize("nq", [4096, 5000, 9000])
@pytest.mark.parametrize("mode", [0, 1])
def test_large_uniform(mix, nq, mode):
    _, queries, data = mix
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    got = gi.search_arrays(queries[:nq], 10, 40, mode=mode)
    assert_same(got, oi.search(queries[:nq], 10, 40), f"nq={nq} mode={mode}")


def test_large_per_query_inputs(mix):
    _, queries, data = mix
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    rng = np.random.default_rng(8)
    nq, nbits = 9000, 4000
    words = (nbits + 63) // 64
    ks = rng.choice([1, 10, 50], nq).astype(np.uint32)
    efs = rng.choice([16, 64, 128], nq).astype(np.uint32)
    used = (rng.random(nq) < 0.5).astype(np.uint8)
    # A bank of 16 bitmaps, chosen per query by id ...
    bank = np.zeros((16, words), np.uint64)
    for i in range(16):
        sel = rng.random(nbits) < rng.uniform(0.05, 0.9)
        bank[i] = H.key_bitmap(np.nonzero(sel)[0].astype(np.uint64), nbits)
    fids = rng.integers(0, 16, nq).astype(np.uint32)
    per_query = np.ascontiguousarray(bank[fids])
    ref = oi.search(queries, 50, 16, filter_bits=per_query, filter_nbits=nbits, filter_stride=words,
                    filter_used=used, ks=ks, efs=efs)
    got = gi.search_arrays(queries, 50, 16, filter_bits=bank, filter_nbits=nbits, filter_stride=words,
                           filter_used=used, filter_ids=fids, ks=ks, efs=efs, mode=1)
    assert_same(got, ref, "bitmap ids")
    # ... and the same filters as one bitmap per query.
    got = gi.search_arrays(queries, 50, 16, filter_bits=per_query, filter_nbits=nbits, filter_stride=words,
                           filter_used=used, ks=ks, efs=efs, mode=0)
    assert_same(got, ref, "per-query bitmaps")
    # One bitmap shared by every query.
    shared = bank[3]
    got = gi.search_arrays(queries, 10, 32, filter_bits=shared, filter_nbits=nbits)
    assert_same(got, oi.search(queries, 10, 32, filter_bits=shared, filter_nbits=nbits), "shared bitmap")


def test_large_statuses(mix):
    """Invalid queries at rows 6000 and 8500: their statuses, the call's
    error (the first failing query's) and every other row."""
    _, queries, data = mix
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    q = queries.copy()
    q[6000, 3] = np.nan
    q[8500, :] = np.inf
    got = gi.search_arrays(q, 10, 40, raise_on_error=False)
    assert_same(got, oi.search(q, 10, 40), "statuses")
    assert got[3][6000] == H.Status.NON_FINITE_VECTOR and got[3][8500] == H.Status.NON_FINITE_VECTOR
    with pytest.raises(H.Error) as e:
        gi.search_arrays(q, 10, 40)
    assert e.value.status == H.Status.NON_FINITE_VECTOR
