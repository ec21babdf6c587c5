"""Base-sharded search over several GPUs: one process per GPU, each holding
the index of its own slice of the base vectors, every rank searching every
query, and one exchange step that merges the per-shard top-k.

Replicas (``replicas.py``) are the default multi-GPU form because the index
fits one GPU many times over. Base sharding is the form for a base that does
not: each rank opens an index built from its rows only (with the global
keys), so device memory per rank falls with the rank count, and the query
batch is searched on every rank.

The exchange: each rank's fixed-width result rows [nq, k] (keys, distance
bits, count, status) are all-gathered (NCCL over NVLink when `device` is a
CUDA device, gloo on CPU), then merged on the same device by the order of the
reference's final sort, (distance by ``f32::total_cmp``, key)
(src/neighbor.rs:17-21, src/hnsw/mod.rs:501-510), keeping k. A query's status
is the first non-OK status over the shards in rank order; its count is then 0.

What the merge returns:
- for exact search (BruteForceIndex::search_batch, src/brute.rs:122-180) it is
  the unsharded answer, bit for bit: the global top-k by (distance, key) is
  the top-k of the union of the per-shard top-k;
- for HNSW it is the merge of each shard's own HnswIndex::search_batch
  (src/hnsw/mod.rs:520-536) — each shard's graph is the graph of its rows, so
  this differs from searching one graph of all rows, as any sharded HNSW
  deployment does.
"""

from __future__ import annotations

from typing import Callable, Tuple

import numpy as np

from replicas import query_shard

Result = Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]


def base_shard(n: int, rank: int, world: int) -> slice:
    """Contiguous, balanced slice of `n` base rows held by `rank` of `world`."""
    return query_shard(n, rank, world)


def _total_cmp_key(dist_bits):
    """int32 bits of f32 values -> int64 keys ordered as f32::total_cmp
    (the sign-magnitude bits made two's complement, src/neighbor.rs:17-21)."""
    import torch

    b = dist_bits.to(torch.int32)
    return (b ^ ((b >> 31) & 0x7FFFFFFF)).to(torch.int64)


def merge_topk(keys, dist_bits, count, status, k: int):
    """Merges S shards' results into the top `k` per query.

    keys: int64 tensor [S, nq, s] (u64 keys as their bit patterns);
    dist_bits: int32 tensor [S, nq, s] (f32 distances as bits);
    count: int64 tensor [S, nq] (valid prefix of each row, <= s);
    status: int32 tensor [S, nq].
    Returns (keys int64 [nq, k], dist_bits int32 [nq, k], count int64 [nq],
    status int32 [nq]), on the input device. Entries past a query's count
    are zero.
    """
    import torch

    S, nq, s = keys.shape
    dev = keys.device
    out_k = torch.zeros((nq, k), dtype=torch.int64, device=dev)
    out_d = torch.zeros((nq, k), dtype=torch.int32, device=dev)
    # First non-OK status per query, in rank order (queries are validated
    # before k is looked at, so k = 0 still reports them).
    bad = status != 0
    st = torch.zeros(nq, dtype=torch.int32, device=dev)
    if nq:
        first_bad = bad.to(torch.int32).argmax(0)
        st = torch.where(bad.any(0), status.gather(0, first_bad.unsqueeze(0)).squeeze(0), st)
    if nq == 0 or k == 0 or s == 0:
        return out_k, out_d, torch.zeros(nq, dtype=torch.int64, device=dev), st
    # [nq, S*s] candidate rows; entries past a shard's count sort last.
    ck = keys.permute(1, 0, 2).reshape(nq, S * s)
    cd = dist_bits.permute(1, 0, 2).reshape(nq, S * s)
    pos = torch.arange(s, device=dev).view(1, 1, s)
    valid = (pos < count.unsqueeze(-1)) & (status == 0).unsqueeze(-1)
    valid = valid.permute(1, 0, 2).reshape(nq, S * s)
    primary = torch.where(valid, _total_cmp_key(cd), torch.full_like(ck, 1 << 40))
    # Lexicographic (distance, key): stable sort by key (u64 order through
    # the sign-flipped int64), then stable sort by distance.
    order = torch.sort(ck ^ (-(1 << 63)), dim=1, stable=True).indices
    order = order.gather(1, torch.sort(primary.gather(1, order), dim=1, stable=True).indices)
    kk = min(k, S * s)
    top = order[:, :kk]
    n_valid = valid.sum(1)
    cnt = torch.clamp(n_valid, max=k)
    cnt = torch.where(st == 0, cnt, torch.zeros_like(cnt))
    keep = torch.arange(kk, device=dev).view(1, kk) < cnt.unsqueeze(1)
    out_k[:, :kk] = torch.where(keep, ck.gather(1, top), torch.zeros_like(top))
    out_d[:, :kk] = torch.where(keep, cd.gather(1, top).to(torch.int32), torch.zeros((nq, kk), dtype=torch.int32,
                                                                                       device=dev))
    return out_k, out_d, cnt, st


def search_sharded(search: Callable[..., Result], queries: np.ndarray, k: int, ef: int, *, group=None,
                   device=None, **search_kw) -> Result:
    """Searches every query on this rank's shard and merges all shards.

    `search(queries, k, ef, **search_kw)` is this rank's local search (for
    example ``HnswIndex.search_arrays`` of the index opened from this rank's
    shard file, or a brute-force search over its rows returning global keys)
    and returns (keys [nq, s], dist [nq, s], count [nq], status [nq]) with
    s >= k. Every rank passes the same queries and arguments and receives
    the merged (keys [nq, k], dist [nq, k], count [nq], status [nq]).
    `device` is where the exchange and the merge run (a CUDA device for
    NCCL, None for CPU/gloo).
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    nq = len(queries)
    keys = np.zeros((nq, k), np.uint64)
    dist_ = np.zeros((nq, k), np.float32)
    count = np.zeros(nq, np.uint32)
    status = np.zeros(nq, np.int32)
    if nq:
        # Called for k = 0 too: the local search validates every query
        # before it looks at k (src/hnsw/mod.rs:460-477), so a NaN or zero
        # query still reports its status; a zero-width result is empty.
        kk, dd, cc, ss = search(queries, k, ef, **search_kw)
        w = min(k, kk.shape[1] if kk.ndim == 2 else 0)
        keys[:, :w], dist_[:, :w] = kk[:, :w], dd[:, :w]
        count[:], status[:] = np.minimum(cc, k), ss
    # One int64 tensor per rank: keys | distance bits | count | status.
    packed = np.zeros((nq, 2 * k + 2), np.int64)
    packed[:, :k] = keys.view(np.int64)
    packed[:, k:2 * k] = dist_.view(np.int32).astype(np.int64)
    packed[:, 2 * k] = count.astype(np.int64)
    packed[:, 2 * k + 1] = status.astype(np.int64)
    t = torch.from_numpy(packed)
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    g = torch.stack(parts)  # [S, nq, 2k+2]
    mk, md, mc, ms = merge_topk(g[:, :, :k], g[:, :, k:2 * k].to(torch.int32), g[:, :, 2 * k],
                                g[:, :, 2 * k + 1].to(torch.int32), k)
    out_k = mk.cpu().numpy().view(np.uint64)
    out_d = md.cpu().numpy().view(np.float32)
    return out_k, out_d, mc.cpu().numpy().astype(np.uint32), ms.cpu().numpy().astype(np.int32)
