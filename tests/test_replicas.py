"""Multi-GPU replica path, host logic on CPU: two gloo ranks each search a
shard of the batch (with the oracle standing in for the device search) and
all-gather the results; the gathered arrays must equal one search of the
whole batch. Uneven batches, per-query k/ef/filters and an empty shard are
covered."""

import os
import socket

import numpy as np
import pytest

import replicas as R


def test_query_shard_covers_every_query_once():
    for nq in (0, 1, 5, 16, 17, 1000):
        for world in (1, 2, 3, 8):
            seen = np.zeros(nq, int)
            for r in range(world):
                s = R.query_shard(nq, r, world)
                seen[s] += 1
                assert (s.stop - s.start) in (nq // world, nq // world + 1)
            assert (seen == 1).all()
    with pytest.raises(ValueError):
        R.query_shard(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, data, queries, kw, nq, out_path):
    import torch.distributed as dist

    import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        oi = O.Index(data)
        got = R.search_replicated(oi.search, queries[:nq], 10, 48, **kw)
        if rank == 0:
            np.savez(out_path, keys=got[0], dist=got[1], count=got[2], status=got[3])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nq", [33, 1])
def test_two_gloo_ranks_gather_the_batch(tmp_path, nq):
    import multiprocessing as mp

    import hnsw_gpu as H
    import oracle as O
    from conftest import build_index

    base, queries = H.mixture(3000, 40, 16, 20, 0.5, 61)
    data = build_index(base, metric=0, m=12, seed=4)
    rng = np.random.default_rng(5)
    ks = rng.choice([1, 10, 30], 40).astype(np.uint64)
    efs = rng.choice([16, 48, 100], 40).astype(np.uint64)
    words = (3000 + 63) // 64
    bits = np.zeros((40, words), np.uint64)
    for i in range(40):
        bits[i] = H.key_bitmap(np.nonzero(rng.random(3000) < 0.3)[0].astype(np.uint64), 3000)
    used = (rng.random(40) < 0.5).astype(np.uint8)
    kw = dict(ks=ks[:nq], efs=efs[:nq], filter_used=used[:nq], filter_bits=bits[:nq], filter_nbits=3000,
              filter_stride=words)
    out = str(tmp_path / "gathered.npz")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, data, queries, kw, nq, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = np.load(out)
    ref = O.Index(data).search(queries[:nq], 10, 48, **kw)
    stride = got["keys"].shape[1]
    np.testing.assert_array_equal(got["status"], ref[3])
    np.testing.assert_array_equal(got["count"], ref[2])
    for i in range(nq):
        c = int(ref[2][i])
        np.testing.assert_array_equal(got["keys"][i, :c], ref[0][i, :c])
        np.testing.assert_array_equal(got["dist"][i, :c].view(np.uint32), ref[1][i, :c].view(np.uint32))
    assert stride >= int(ks[:nq].max())
