"""The traversal's visited hash in both storage forms, against the oracle.

By default a power-of-two visited hash stores 16-bit tags (the id's low bits
after a bijection, beside the probe distance from its home slot) instead of
32-bit ids. The visited set decides which neighbors get distances and enter
the heaps (src/hnsw/search.rs:120-136), so any error in it changes results:
every case here must equal the oracle bit for bit. Widening the id space
(hnsw_gpu_debug_visit_tags with k bits) leaves fewer bits for the probe
distance; at 1-4 distance bits most collisions exceed what a tag records,
which sends plain-mode queries to the retry pass and moves persistent warps'
sets into their spill bitmaps mid-query.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from conftest import build_index
from test_gpu_search import assert_same

pytestmark = pytest.mark.gpu

# 0: automatic (tags), -1: 32-bit ids, 24 / 27: 4 / 1 distance bits at a
# 4096-entry hash.
TAG_MODES = [0, -1, 24, 27]


@pytest.fixture(scope="module")
def gauss():
    base, _ = H.gaussian(10_000, 0, 64, 142)
    _, queries = H.gaussian(0, 400, 64, 143)
    data = build_index(base, metric=0, m=16, seed=7)
    return base, queries, data


@pytest.fixture(autouse=True)
def _restore_tags():
    yield
    H.debug_visit_tags(0)


@pytest.mark.parametrize("tags", TAG_MODES)
@pytest.mark.parametrize("mode", [0, 1])
def test_visit_tags_unfiltered(gauss, tags, mode):
    _, queries, data = gauss
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    H.debug_visit_tags(tags)
    for ef in (16, 64, 200):
        gi.set_schedule(ef_cap=256, hash_cap=4096, warps_per_block=2)
        got = gi.search_arrays(queries, 10, ef, mode=mode)
        assert_same(got, oi.search(queries, 10, ef), f"tags={tags} mode={mode} ef={ef}")
    # Small hashes: the load limit spills too (persistent) or retries (plain).
    gi.set_schedule(ef_cap=64, hash_cap=256, warps_per_block=4)
    got = gi.search_arrays(queries, 10, 64, mode=mode)
    assert_same(got, oi.search(queries, 10, 64), f"tags={tags} mode={mode} hash=256")
    gi.set_schedule()


@pytest.mark.parametrize("tags", TAG_MODES)
@pytest.mark.parametrize("mode", [0, 1])
def test_visit_tags_filtered_tombstoned(tags, mode):
    """Filters and tombstones take the general layer-0 kernels (both the
    spill-array and cold-list variants in persistent mode)."""
    base, queries = H.mixture(5000, 64, 24, 20, 0.4, 9)
    rng = np.random.default_rng(3)
    dead = np.nonzero(rng.random(5000) < 0.05)[0]
    data = build_index(base, metric=0, m=12, seed=4, deleted_keys=dead)
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    words = (5000 + 63) // 64
    bits = np.zeros((64, words), np.uint64)
    for i in range(64):
        sel = rng.random(5000) < np.exp(rng.uniform(np.log(0.02), np.log(0.9)))
        bits[i] = H.key_bitmap(np.nonzero(sel)[0].astype(np.uint64), 5000)
    H.debug_visit_tags(tags)
    ref = oi.search(queries, 10, 48, filter_bits=bits, filter_nbits=5000, filter_stride=words)
    for cold in (0, 1):
        gi.set_schedule(ef_cap=64, hash_cap=1024, warps_per_block=4, cold=cold)
        got = gi.search_arrays(queries, 10, 48, filter_bits=bits, filter_nbits=5000, filter_stride=words,
                               mode=mode)
        assert_same(got, ref, f"tags={tags} mode={mode} cold={cold}")
    gi.set_schedule()
