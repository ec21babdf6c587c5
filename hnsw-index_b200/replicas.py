"""Replicated search over several GPUs: one process per GPU, each holding the
whole index, each searching its share of a batch; no collective on the data
path except the final gather of the results.

Queries are independent (HnswIndex::search_batch maps `search` over rows,
src/hnsw/mod.rs:520-536), so a batch splits into contiguous shards, one per
rank, and the concatenation of the shard results is the batch result. The
index (about 0.7 GB at 1M x 128, 8 GB at 10M x 128) fits every GPU, so no
base sharding is needed.

``search_replicated`` runs the rank's shard with the given search function
(normally ``HnswIndex.search_arrays`` on this rank's device) and all-gathers
the fixed-width result arrays, so every rank ends with the whole batch's
(keys, dist, count, status).
"""

from __future__ import annotations

from typing import Callable, Tuple

import numpy as np


def query_shard(nq: int, rank: int, world: int) -> slice:
    """Contiguous, balanced share of `nq` queries for `rank` of `world`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(nq, world)
    lo = rank * base + min(rank, extra)
    return slice(lo, lo + base + (1 if rank < extra else 0))


def search_replicated(search: Callable[..., Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]],
                      queries: np.ndarray, k: int, ef: int, *, group=None, device=None, **search_kw):
    """Searches this rank's shard of `queries` and gathers every shard.

    `search(queries, k, ef, **search_kw)` returns (keys [n, s], dist [n, s],
    count [n], status [n]) for its rows, with a row stride `s` >= max k.
    Per-query arguments (ks, efs, filter_used, filter_ids) in `search_kw`
    that have one entry per query are sliced to the shard, and so are
    per-query filter bitmaps (filter_stride set, no filter_ids: one bitmap
    row per query). `device` is where the gather runs (a CUDA device for
    NCCL, None for CPU/gloo).
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nq = len(queries)
    sh = query_shard(nq, rank, world)
    per_query_bitmaps = bool(search_kw.get("filter_stride")) and search_kw.get("filter_ids") is None
    kw = {}
    for name, v in search_kw.items():
        if name in ("ks", "efs", "filter_used", "filter_ids") and v is not None and len(v) == nq:
            v = v[sh]
        elif name == "filter_bits" and per_query_bitmaps and v is not None and np.ndim(v) == 2 and len(v) == nq:
            v = v[sh]
        kw[name] = v
    n = sh.stop - sh.start
    stride = max(int(np.max(search_kw["ks"])) if search_kw.get("ks") is not None and nq else k, 1)
    keys = np.zeros((n, stride), np.uint64)
    dist_ = np.zeros((n, stride), np.float32)
    count = np.zeros(n, np.uint32)
    status = np.zeros(n, np.int32)
    if n:
        kk, dd, cc, ss = search(queries[sh], k, ef, **kw)
        w = min(stride, kk.shape[1])
        keys[:, :w], dist_[:, :w], count[:], status[:] = kk[:, :w], dd[:, :w], cc, ss
    # Fixed-width rows: pad every shard to the largest shard.
    rows = -(-nq // world)
    packed = np.zeros((rows, 2 * stride + 2), np.int64)
    packed[:n, :stride] = keys.view(np.int64)
    packed[:n, stride:2 * stride] = dist_.view(np.int32).astype(np.int64)
    packed[:n, 2 * stride] = count.astype(np.int64)
    packed[:n, 2 * stride + 1] = status.astype(np.int64)
    t = torch.from_numpy(packed)
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out_k = np.zeros((nq, stride), np.uint64)
    out_d = np.zeros((nq, stride), np.float32)
    out_c = np.zeros(nq, np.uint32)
    out_s = np.zeros(nq, np.int32)
    for r, p in enumerate(parts):
        s = query_shard(nq, r, world)
        m = s.stop - s.start
        a = p.cpu().numpy()[:m]
        out_k[s] = a[:, :stride].view(np.uint64)
        out_d[s] = a[:, stride:2 * stride].astype(np.int32).view(np.float32)
        out_c[s] = a[:, 2 * stride].astype(np.uint32)
        out_s[s] = a[:, 2 * stride + 1].astype(np.int32)
    return out_k, out_d, out_c, out_s
