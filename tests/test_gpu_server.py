"""Request loop: continuous batching over a resident index.

Each request submitted to the server must return exactly what the same
search returns alone (search_with, src/hnsw/mod.rs:448-455): the batches mix
k, ef and filters, run concurrently on several streams, and the kernel keeps
every query's traversal independent.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from conftest import build_index

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served():
    base, queries = H.mixture(20000, 600, 32, 40, 0.4, 31)
    data = build_index(base, metric=0, m=16, seed=3)
    return base, queries, data


def make_requests(queries, nbits, seed, bank_size=8):
    """Per request k in {10, 100}, ef log-uniform in [32, 512], 30% filtered by
    one of `bank_size` key bitmaps of selectivity 5%-50%."""
    rng = np.random.default_rng(seed)
    n = len(queries)
    ks = rng.choice([10, 100], n).astype(np.uint32)
    efs = np.exp(rng.uniform(np.log(32), np.log(512), n)).astype(np.uint32)
    words = (nbits + 63) // 64
    bank = np.zeros((bank_size, words), np.uint64)
    for j in range(bank_size):
        sel = rng.random(nbits) < rng.uniform(0.05, 0.5)
        bank[j] = H.key_bitmap(np.nonzero(sel)[0].astype(np.uint64), nbits)
    fids = np.where(rng.random(n) < 0.3, rng.integers(0, bank_size, n), -1).astype(np.int32)
    return ks, efs, fids, bank


def oracle_results(oi, queries, ks, efs, fids, bank, nbits):
    words = bank.shape[1]
    bits = np.zeros((len(queries), words), np.uint64)
    bits[fids >= 0] = bank[fids[fids >= 0]]
    used = (fids >= 0).astype(np.uint8)
    return oi.search(queries, 100, 16, ks=ks.astype(np.uint64), efs=efs.astype(np.uint64), filter_bits=bits,
                     filter_nbits=nbits, filter_stride=words, filter_used=used)


def alone(gi, queries, ks, efs, fids, bank, nbits):
    """Each request searched alone (one query per call) on the GPU."""
    out = []
    for i in range(len(queries)):
        fb = bank[fids[i]] if fids[i] >= 0 else None
        g = gi.search_arrays(queries[i:i + 1], int(ks[i]), int(efs[i]), filter_bits=fb,
                             filter_nbits=nbits if fb is not None else 0)
        out.append(g)
    return out


def test_submitted_requests_equal_alone_results(served):
    base, queries, data = served
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    nbits = 20000
    q = queries[:200]
    ks, efs, fids, bank = make_requests(q, nbits, 1)
    srv = H.Server(gi, max_batch=64, max_inflight=3, filter_nbits=nbits, filter_bank=bank)
    tickets = [srv.submit(q[i], int(ks[i]), int(efs[i]), int(fids[i])) for i in range(len(q))]
    results = [srv.wait(t) for t in tickets]
    batches, launched = srv.stats()
    srv.stop()
    assert launched == len(q) and batches >= 2
    one = alone(gi, q, ks, efs, fids, bank, nbits)
    ref = oracle_results(oi, q, ks, efs, fids, bank, nbits)
    for i, (keys, dist, status, lat) in enumerate(results):
        assert status == 0
        c = int(ref[2][i])
        np.testing.assert_array_equal(keys, ref[0][i, :c])
        np.testing.assert_array_equal(dist.view(np.uint32), ref[1][i, :c].view(np.uint32))
        np.testing.assert_array_equal(keys, one[i][0][0, :int(one[i][2][0])])
        assert lat >= 0


def test_open_loop_replay_mixes_requests_and_matches(served):
    base, queries, data = served
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    nbits = 20000
    ks, efs, fids, bank = make_requests(queries, nbits, 2)
    rng = np.random.default_rng(3)
    arrivals = np.cumsum(rng.exponential(1e6 / 200000.0, len(queries)))  # 200k requests/s
    srv = H.Server(gi, max_batch=128, max_inflight=4, filter_nbits=nbits, filter_bank=bank, linger_us=50)
    keys, dist, cnt, st, lat = srv.replay(queries, arrivals, ks, efs, fids)
    batches, launched = srv.stats()
    srv.stop()
    assert (st == 0).all()
    assert batches > 1
    ref = oracle_results(oi, queries, ks, efs, fids, bank, nbits)
    for i in range(len(queries)):
        c = int(ref[2][i])
        assert cnt[i] == c
        np.testing.assert_array_equal(keys[i, :c], ref[0][i, :c])
        np.testing.assert_array_equal(dist[i, :c].view(np.uint32), ref[1][i, :c].view(np.uint32))
    assert (lat > 0).all()


def test_admission_rejects_when_queue_is_full(served):
    base, queries, data = served
    gi = H.HnswIndex.from_bytes(data)
    srv = H.Server(gi, max_batch=8, max_inflight=1, max_pending=16)
    accepted, rejected = [], 0
    for i in range(400):
        try:
            accepted.append(srv.submit(queries[i % len(queries)], 10, 512))
        except H.Error as e:
            assert e.status == H.Status.ADMISSION_REJECTED
            rejected += 1
    for t in accepted:
        _, _, status, _ = srv.wait(t)
        assert status == 0
    srv.stop()
    assert rejected > 0 and len(accepted) >= 16


def test_cancelled_requests_report_cancelled_and_others_stand(served):
    """hnsw_gpu_cancel on queued requests (one batch slot of 8 queries, so
    most wait on the host) and on requests already launched: a cancelled
    request reports CANCELLED with no results; every other request returns
    the oracle's answer, and the server keeps serving afterwards."""
    base, queries, data = served
    gi = H.HnswIndex.from_bytes(data)
    oi = O.Index(data)
    q = queries[:200]
    srv = H.Server(gi, max_batch=8, max_inflight=1, linger_us=0)
    try:
        tickets = [srv.submit(q[i], 10, 256) for i in range(len(q))]
        # Every third request, from the first (likely launched) to the last (queued).
        cancelled = {i: srv.cancel(tickets[i]) for i in range(0, len(q), 3)}
        results = [srv.wait(t, timeout_ms=20000) for t in tickets]
        after = [srv.wait(srv.submit(q[i], 10, 256), timeout_ms=20000) for i in range(8)]
    finally:
        srv.stop()
    assert sum(cancelled.values()) >= len(cancelled) // 2
    ref = oi.search(q, 10, 256)
    for i, (keys, dist, status, _) in enumerate(results):
        if cancelled.get(i):
            assert status == H.Status.CANCELLED and len(keys) == 0
        else:
            assert status == 0
            c = int(ref[2][i])
            np.testing.assert_array_equal(keys, ref[0][i, :c])
            np.testing.assert_array_equal(dist.view(np.uint32), ref[1][i, :c].view(np.uint32))
    for i, (keys, _, status, _) in enumerate(after):
        assert status == 0
        np.testing.assert_array_equal(keys, ref[0][i, :int(ref[2][i])])
