"""Base-sharded search, host logic on CPU: the top-k merge against a
sequential merge, and two gloo ranks that each search their own slice of the
base (the oracle standing in for the device search) and exchange results.
Sharded exact search must equal unsharded exact search bit for bit; sharded
HNSW must equal the merge of each shard's own search."""

import os
import socket

import numpy as np
import pytest
import torch

import shards as SH


def _sequential_merge(keys, dist, count, status, k):
    """The reference's final order, (f32::total_cmp distance, key)
    (src/neighbor.rs:17-21), over the union of the shards' valid prefixes."""
    S, nq, _ = keys.shape
    ok = np.zeros((nq, k), np.uint64)
    od = np.zeros((nq, k), np.float32)
    oc = np.zeros(nq, np.int64)
    ost = np.zeros(nq, np.int32)
    for q in range(nq):
        bad = [int(status[r, q]) for r in range(S) if status[r, q] != 0]
        if bad:
            ost[q] = bad[0]
            continue
        cand = []
        for r in range(S):
            for j in range(int(count[r, q])):
                b = int(dist[r, q, j].view(np.int32))
                cand.append((b ^ (0x7FFFFFFF if b < 0 else 0), int(keys[r, q, j]), dist[r, q, j]))
        cand.sort(key=lambda x: (x[0], x[1]))
        cand = cand[:k]
        oc[q] = len(cand)
        for j, (_, key, d) in enumerate(cand):
            ok[q, j], od[q, j] = key, d
    return ok, od, oc, ost


def _assert_same(got, ref, label=""):
    gk, gd, gc, gs = got
    rk, rd, rc, rs = ref
    np.testing.assert_array_equal(np.asarray(gs), np.asarray(rs), err_msg=f"{label}: status")
    np.testing.assert_array_equal(np.asarray(gc).astype(np.int64), np.asarray(rc).astype(np.int64),
                                  err_msg=f"{label}: count")
    for q in range(len(gc)):
        c = int(gc[q])
        np.testing.assert_array_equal(gk[q, :c], rk[q, :c], err_msg=f"{label}: keys of query {q}")
        np.testing.assert_array_equal(gd[q, :c].view(np.uint32), rd[q, :c].view(np.uint32),
                                      err_msg=f"{label}: distance bits of query {q}")


def test_merge_topk_matches_a_sequential_merge():
    rng = np.random.default_rng(0)
    specials = np.array([0.0, -0.0, 1.5, -2.0, 1e-30, -1e-30, 3.0, np.inf, -np.inf], np.float32)
    for trial in range(300):
        S, nq, s, k = int(rng.integers(1, 4)), int(rng.integers(0, 6)), int(rng.integers(1, 6)), int(rng.integers(0, 8))
        keys = np.zeros((S, nq, s), np.uint64)
        for q in range(nq):
            flat = rng.choice(10**6 if trial % 2 else 2**62, size=S * s, replace=False).astype(np.uint64)
            if rng.random() < 0.3:
                flat |= np.uint64(1 << 63)  # keys above i64::MAX keep the u64 order
            keys[:, q, :] = flat.reshape(S, s)
        if trial % 3 == 0:
            dist = rng.choice(specials, size=(S, nq, s)).astype(np.float32)  # many ties, signed zeros
        else:
            dist = rng.standard_normal((S, nq, s)).astype(np.float32)
        count = rng.integers(0, s + 1, size=(S, nq))
        status = np.where(rng.random((S, nq)) < 0.1, rng.integers(1, 5, size=(S, nq)), 0).astype(np.int32)
        got = SH.merge_topk(torch.from_numpy(keys.view(np.int64)), torch.from_numpy(dist.view(np.int32)),
                            torch.from_numpy(count.astype(np.int64)), torch.from_numpy(status), k)
        gk, gd, gc, gs = (t.numpy() for t in got)
        _assert_same((gk.view(np.uint64), gd.view(np.float32), gc, gs),
                     _sequential_merge(keys, dist, count, status, k), f"trial {trial}")
        for q in range(nq):
            assert (gk[q, int(gc[q]):] == 0).all() and (gd[q, int(gc[q]):] == 0).all()


def test_base_shards_cover_every_row_once():
    for n in (0, 1, 7, 1000):
        for world in (1, 2, 3, 8):
            seen = np.zeros(n, int)
            for r in range(world):
                seen[SH.base_shard(n, r, world)] += 1
            assert (seen == 1).all()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, kind, base, keys, queries, k, ef, metric, out_path):
    import torch.distributed as dist

    import oracle as O
    import shards

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = shards.base_shard(len(base), rank, world)
        if kind == "brute":
            def search(q, k_, ef_):
                return O.brute(metric, base[sh], q, k_, keys=keys[sh])
        else:
            from conftest import build_index
            data = build_index(base[sh], metric=metric, m=8, seed=2, keys=keys[sh], parallel=False)
            oi = O.Index(data)

            def search(q, k_, ef_):
                return oi.search(q, k_, ef_)
        got = shards.search_sharded(search, queries, k, ef)
        np.savez(out_path + f".{rank}.npz", keys=got[0], dist=got[1], count=got[2], status=got[3])
    finally:
        dist.destroy_process_group()


def _run_ranks(tmp_path, world, *args):
    import multiprocessing as mp

    out = str(tmp_path / "merged")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port) + args + (out,)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = [np.load(out + f".{r}.npz") for r in range(world)]
    for r in range(1, world):  # every rank ends with the same merged answer
        for name in ("keys", "dist", "count", "status"):
            np.testing.assert_array_equal(res[r][name], res[0][name])
    return res[0]["keys"], res[0]["dist"], res[0]["count"], res[0]["status"]


@pytest.mark.parametrize("metric,k", [(0, 10), (1, 25), (0, 700), (0, 0)])
def test_two_gloo_ranks_sharded_brute_force_equals_unsharded(tmp_path, metric, k):
    import hnsw_gpu as H
    import oracle as O

    base, queries = H.mixture(1200, 30, 12, 10, 0.5, 21)
    # Ties between shards: duplicate rows on both sides of the split.
    base[700:710] = base[100:110]
    keys = (np.arange(1200, dtype=np.uint64) * np.uint64(7919)) ^ np.uint64(1 << 63)
    queries = np.vstack([queries, base[100:102], np.full((1, 12), np.nan, np.float32)]).astype(np.float32)
    got = _run_ranks(tmp_path, 2, "brute", base, keys, queries, k, 0, metric)
    ref = O.brute(metric, base, queries, k, keys=keys)
    _assert_same(got, (ref[0][:, :k], ref[1][:, :k], ref[2], ref[3]), "sharded brute force")
    assert int(got[3][-1]) != 0  # the NaN query reports its status from every shard


def test_two_gloo_ranks_sharded_hnsw_equals_merge_of_shard_searches(tmp_path):
    import hnsw_gpu as H
    import oracle as O
    from conftest import build_index

    base, queries = H.mixture(2000, 40, 16, 20, 0.5, 33)
    keys = np.arange(2000, dtype=np.uint64) + np.uint64(10**9)
    k, ef = 10, 40
    got = _run_ranks(tmp_path, 2, "hnsw", base, keys, queries, k, ef, 0)
    parts = []
    for r in range(2):
        sh = SH.base_shard(2000, r, 2)
        data = build_index(base[sh], metric=0, m=8, seed=2, keys=keys[sh], parallel=False)
        parts.append(O.Index(data).search(queries, k, ef))
    stack = [np.stack([p[i][:, :k] if i < 2 else p[i] for p in parts]) for i in range(4)]
    _assert_same(got, _sequential_merge(*stack, k), "sharded hnsw")
    truth = O.brute(0, base, queries, k, keys=keys)
    assert O.recall_at_k(truth[0], truth[2], got[0], got[2], k) >= 0.9


@pytest.mark.gpu
def test_merge_topk_on_the_device_equals_the_host_merge():
    # The exchange merges on the device that holds the gathered rows (a GPU
    # under NCCL): same result as on the host, bit for bit.
    rng = np.random.default_rng(1)
    S, nq, s, k = 4, 257, 16, 10
    keys = rng.choice(2**62, size=(S, nq, s), replace=False).astype(np.uint64)
    keys[1] |= np.uint64(1 << 63)
    dist = rng.choice(np.array([0.0, -0.0, 0.25, 0.5, 1.0, 2.0], np.float32), size=(S, nq, s)).astype(np.float32)
    count = rng.integers(0, s + 1, size=(S, nq))
    status = np.where(rng.random((S, nq)) < 0.02, 3, 0).astype(np.int32)
    args = (torch.from_numpy(keys.view(np.int64)), torch.from_numpy(dist.view(np.int32)),
            torch.from_numpy(count.astype(np.int64)), torch.from_numpy(status))
    host = SH.merge_topk(*args, k)
    dev = SH.merge_topk(*(a.cuda() for a in args), k)
    for h, d in zip(host, dev):
        assert d.is_cuda
        assert torch.equal(h, d.cpu())
