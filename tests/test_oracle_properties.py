"""Properties of the oracle's search on random small indexes, after the
reference's own property tests (tests/properties.rs:108-159): results sorted
by (total_cmp distance, key), at most k, unique, live and admitted by the
filter, and every distance bit-identical to a recomputation with the metric
(src/hnsw/mod.rs:483-510 re-ranks quantized results with exact distances).
The GPU path is compared with this oracle bit for bit, so these pin what the
device results satisfy too."""

import numpy as np
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import hnsw_gpu as H
import oracle as O
from conftest import build_index


def total_cmp_key(d: np.float32) -> int:
    b = int(np.float32(d).view(np.int32))
    return b ^ (0x7FFFFFFF if b < 0 else 0)


@settings(max_examples=40, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(seed=st.integers(0, 2**31 - 1), n=st.integers(1, 160), dim=st.integers(1, 12), metric=st.sampled_from([0, 1, 2]),
       m=st.integers(2, 12), k=st.integers(0, 20), ef=st.integers(1, 64), dead_every=st.sampled_from([0, 2, 3, 7]),
       filt=st.sampled_from([0, 2, 5]), quant=st.booleans())
def test_search_results_satisfy_the_reference_properties(seed, n, dim, metric, m, k, ef, dead_every, filt, quant):
    rng = np.random.default_rng(seed)
    base = rng.standard_normal((n, dim)).astype(np.float32)
    queries = rng.standard_normal((6, dim)).astype(np.float32)
    keys = (np.arange(n, dtype=np.uint64) * np.uint64(2654435761)) % np.uint64(1 << 40)
    deleted = [int(keys[i]) for i in range(n) if dead_every and i % dead_every == 0]
    # n <= M with simple selection: every node lists every other one.
    complete = n <= m
    data = build_index(base, metric=metric, m=m, seed=seed % 1000, parallel=False, keys=keys,
                       deleted_keys=deleted, quantize=quant,
                       selection=H.NeighborSelection.simple() if complete else None)
    fbits, fnbits = None, 0
    admitted = set(int(x) for x in keys) - set(deleted)
    if filt:
        allowed = keys[(np.arange(n) % filt) == 1]
        fnbits = int(keys.max()) + 1
        fbits = H.key_bitmap(allowed, fnbits)
        admitted &= set(int(x) for x in allowed)
    got_k, got_d, got_c, got_s = O.Index(data).search(queries, k, ef, quantized=quant, filter_bits=fbits,
                                                      filter_nbits=fnbits)
    stored = O.normalize_rows(base) if metric == 2 else base
    pq = O.normalize_rows(queries) if metric == 2 else queries
    row_of = {int(key): i for i, key in enumerate(keys)}
    for qi in range(len(queries)):
        assert got_s[qi] == 0
        c = int(got_c[qi])
        assert c <= k
        ks = [int(x) for x in got_k[qi, :c]]
        assert len(set(ks)) == c, "duplicate keys"
        assert set(ks) <= admitted, "a deleted or filtered key was returned"
        order = [(total_cmp_key(got_d[qi, j]), ks[j]) for j in range(c)]
        assert order == sorted(order), "not sorted by (distance, key)"
        for j, key in enumerate(ks):
            want = O.distance(metric, pq[qi], stored[row_of[key]])
            assert np.float32(got_d[qi, j]).view(np.uint32) == np.float32(want).view(np.uint32)
        if complete:
            # Every node is evaluated from the first layer-0 expansion, so
            # the search returns min(k, admitted) results, as the complete
            # graph case of src/hnsw/tests.rs:113-127.
            assert c == min(k, len(admitted))
