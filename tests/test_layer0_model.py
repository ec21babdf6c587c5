"""CPU model of the single-array layer-0 search used by the device kernels
for batches that admit every node (search.cu: layer0_single; build.cu: the
construction search), checked against a direct restatement of the
reference's search_layer (src/hnsw/search.rs:81-142) with its two heaps.

The model keeps results and live candidates in one sorted list whose entries
carry an "expanded" flag, plus a tie list (capacity 32) of results evicted
before expansion whose distance equals the new worst result's. On random
graphs with heavily tied distances it must expand the same nodes in the same
order and return the same results as the two-heap search, unless its tie
list overflows (the kernel then hands the query to the general queue, which
the GPU parity tests cover)."""

import heapq

import numpy as np

TIE_CAP = 32


def reference_search_layer(adj, dist, entry, ef):
    """search_layer with every node admitted: candidates a min-heap by
    (distance, id), results a max-heap of at most ef entries."""
    visited = {entry}
    cand = [(dist[entry], entry)]
    res = [(-dist[entry], -entry)]  # max-heap by (distance, id)
    order = []
    while cand:
        d, c = heapq.heappop(cand)
        worst = (-res[0][0], -res[0][1])
        if len(res) >= ef and d > worst[0]:
            break
        order.append(c)
        for n in adj[c]:
            if n in visited:
                continue
            visited.add(n)
            dn = dist[n]
            if len(res) < ef or dn < -res[0][0]:
                heapq.heappush(cand, (dn, n))
                heapq.heappush(res, (-dn, -n))
                if len(res) > ef:
                    heapq.heappop(res)
    return sorted((-a, -b) for a, b in res), order


def single_array_search_layer(adj, dist, entry, ef, stats=None):
    """The kernels' single sorted array U of [distance, id, expanded] plus
    the tie list T. Returns (results, expansion order) or None when T
    overflows. `stats["tie_expansions"]` counts expansions taken from T."""
    visited = {entry}
    U = [[dist[entry], entry, False]]
    T = []
    order = []

    def tie_add(x, wd):
        if T and T[0][0] > wd:
            T.clear()
        if len(T) >= TIE_CAP:
            return False
        T.append(x)
        T.sort(key=lambda e: (e[0], e[1]))
        return True

    while True:
        nxt = next((e for e in U if not e[2]), None)
        if nxt is not None:
            nxt[2] = True
            cur = nxt
        else:
            if not T:
                break
            cur = T.pop(0)
            if len(U) >= ef and cur[0] > U[-1][0]:
                break
            if stats is not None:
                stats["tie_expansions"] = stats.get("tie_expansions", 0) + 1
        order.append(cur[1])
        for n in adj[cur[1]]:
            if n in visited:
                continue
            visited.add(n)
            dn = dist[n]
            if not (len(U) < ef or dn < U[-1][0]):
                continue
            U.append([dn, n, False])
            U.sort(key=lambda e: (e[0], e[1]))
            if len(U) > ef:
                ev = U.pop()
                if not ev[2] and ev[0] == U[-1][0] and not tie_add(ev, U[-1][0]):
                    return None
    return [(e[0], e[1]) for e in U], order


def random_case(rng):
    n = int(rng.integers(2, 300))
    m0 = int(rng.integers(1, 33))
    levels = int(rng.integers(1, 6))
    # Few distinct distances: most comparisons tie, and ids decide the order.
    values = rng.integers(0, levels, size=n).astype(np.float32) * np.float32(0.5)
    adj = []
    for v in range(n):
        deg = int(rng.integers(0, min(m0, n - 1) + 1))
        others = rng.choice(np.delete(np.arange(n), v), size=deg, replace=False)
        adj.append([int(x) for x in others])
    entry = int(rng.integers(0, n))
    ef = int(rng.integers(1, 48))
    return adj, [float(x) for x in values], entry, ef


def test_single_array_search_equals_two_heap_search():
    rng = np.random.default_rng(2024)
    compared = 0
    stats = {}
    for _ in range(3000):
        adj, dist, entry, ef = random_case(rng)
        want = reference_search_layer(adj, dist, entry, ef)
        got = single_array_search_layer(adj, dist, entry, ef, stats)
        if got is None:
            continue
        assert got[1] == want[1], "expansion order differs"
        assert got[0] == want[0], "results differ"
        compared += 1
    assert compared > 2500
    assert stats.get("tie_expansions", 0) > 0  # evicted ties were expanded from T


def test_tie_list_overflow_is_reported():
    # The entry (distance 2) lists 40 nodes at distance 1, then 40 at 0.5,
    # with ef = 40: each 0.5 node evicts an unexpanded 1.0 node while the
    # worst result is still 1.0, so 39 ties queue up, more than T holds.
    dist = [2.0] + [1.0] * 40 + [0.5] * 40
    adj = [list(range(1, 81))] + [[] for _ in range(80)]
    assert single_array_search_layer(adj, dist, 0, 40) is None
    res, _ = reference_search_layer(adj, dist, 0, 40)
    assert res == [(0.5, i) for i in range(41, 81)]


def test_distinct_distances_never_use_the_tie_list():
    rng = np.random.default_rng(7)
    for _ in range(500):
        adj, _, entry, ef = random_case(rng)
        dist = [float(x) for x in rng.permutation(len(adj)).astype(np.float32)]
        got = single_array_search_layer(adj, dist, entry, ef)
        assert got is not None
        assert got == reference_search_layer(adj, dist, entry, ef)
