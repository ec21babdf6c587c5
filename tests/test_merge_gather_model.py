"""CPU model of the traversal's gather merges (merge_gather and
batch_merge_gather in hnsw-index_b200/csrc/warp_sort.cuh), lane by lane.

New entries (distinct, none in the array) know their lower bound in the
ascending array and their rank among themselves; every output position of
a 32-position chunk, top chunk first, takes either the new entry of its rank
or the old entry below it, positions at or above the limit dropped. The
model checks the result equals a sorted merge for random arrays, offsets,
limits and lane sets, which is what the layer-0 heaps
(src/hnsw/search.rs:120-136) need.
"""

import bisect
import random


def gather_merge(A, lo, hi, lanes, x, limit):
    """The kernel's steps; lanes: the set S, x: per-lane entries."""
    rk = {l: sum(1 for j in lanes if x[j] < x[l]) for l in lanes}
    pa = {l: bisect.bisect_left(A, x[l], lo, hi) for l in lanes}
    scratch = [None] * 32
    for l in lanes:
        scratch[rk[l]] = x[l]
    q = {l: pa[l] + rk[l] for l in lanes}
    pmin = min(pa.values())
    end = min(hi + len(lanes), limit)
    if pmin >= end:
        return
    for c in range((end - 1) >> 5, (pmin >> 5) - 1, -1):
        b = c << 5
        M = 0  # OR reduction of the new entries' positions in this chunk
        nb = 0  # add reduction: new entries below the chunk
        for l in lanes:
            if b <= q[l] < b + 32:
                M |= 1 << (q[l] - b)
            if q[l] < b:
                nb += 1
        vals = {}
        for lane in range(32):
            o = b + lane
            nle = nb + bin(M & (((2 << lane) - 1) & 0xFFFFFFFF)).count("1")
            if pmin <= o < end:
                vals[o] = scratch[nle - 1] if (M >> lane) & 1 else A[o - nle]
        for o, v in vals.items():  # all lanes read, then write
            A[o] = v


def test_gather_merge_equals_sorted_merge():
    rng = random.Random(2)
    for _ in range(4000):
        lo = rng.randint(0, 40)
        n = rng.randint(0, 120)
        hi = lo + n
        pool = rng.sample(range(10 ** 6), n + 32)
        old = sorted(pool[:n])
        k = rng.randint(1, 32)
        lanes = rng.sample(range(32), k)
        new = pool[n:n + k]
        limit = rng.randint(hi, hi + 40) if rng.random() < 0.7 else rng.randint(lo, hi + k)
        prefix = [-1 - i for i in range(lo)][::-1]
        A = prefix + old + [None] * 80
        x = [0] * 32
        for l, v in zip(lanes, new):
            x[l] = v
        gather_merge(A, lo, hi, set(lanes), x, limit)
        end = min(hi + k, limit)
        assert A[:end] == (prefix + sorted(old + new))[:end]
