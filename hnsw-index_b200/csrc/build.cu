// Graph construction on sm_100a: one warp per inserted node, then one warp
// per list that receives reverse edges.
//
// Restates HnswIndex::link and its helpers (src/hnsw/build.rs:41-222) for a
// wave of nodes that all see the graph as it stood before the wave:
//   * greedy descent on the layers above the node's level and the ef-bounded
//     beam on each layer below (src/hnsw/search.rs:49-142), with the previous
//     layer's results as entry points; distances in the reference's AVX2
//     order (common.cuh), so every comparison sees the reference's bits;
//   * select_neighbors (simple, or the heuristic with extend_candidates and
//     keep_pruned) on the sorted results, m neighbors on every layer;
//   * the node's own lists are written directly (nobody else links to a node
//     of the running wave); every chosen neighbor yields a reverse-edge
//     record, and the records are grouped by target list;
//   * connect (build.rs:121-150): per list, records in ascending order of the
//     new node's id, each pushed when there is room, otherwise the list plus
//     the new node is re-selected with the list's capacity. Distances between
//     a list's owner and its members are symmetric bit for bit (the AVX2
//     terms are (a-b)^2 or a*b), so the one computed by the new node's search
//     is reused.
// With extend_candidates the connect step reads other lists, so its results
// go to a side buffer and are copied after every list is done: each list then
// sees the lists as they stood after the search step.
#include <algorithm>

#include "build.hpp"
#include "common.cuh"
#include "device.hpp"
#include "warp_sort.cuh"

namespace hnswgpu {
namespace dev {
namespace {

__host__ __device__ __forceinline__ size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

struct BWarp {
    uint32_t* H;     // visited hash (hash_cap words); the selection stage aliases its region
    float* q;        // dp: the inserted node's row
    float* selrows;  // sel_rows * dp, or null
    uint64_t* R;     // ef + 33: results; after a layer, the next layer's entry points
    uint64_t* T;     // kTieCap + 1: evicted ties (candidates outside R)
    uint64_t* disc;  // mm
    uint32_t* fr;    // 32
    float* fd;       // 32
    uint32_t* sel;   // mm
    float* seld;     // mm
    uint32_t* sslot; // mm
    uint32_t hash_cap;
    bool bitmap;
    uint32_t* spill;
    uint32_t spill_words;
    // Work counters (warp-uniform).
    uint32_t nd, nl0, nlU;
};

__device__ __forceinline__ uint32_t list_cap(const BuildGraph& g, uint32_t layer) { return layer == 0 ? g.m0 : g.m; }
__device__ __forceinline__ uint32_t* list_ptr(const BuildGraph& g, uint32_t layer, uint32_t id) {
    return layer == 0 ? g.adj0 + size_t(id) * g.m0p : g.adjU + (size_t(__ldg(g.up_off + id)) + layer - 1) * g.mp;
}
__device__ __forceinline__ uint32_t list_key(const BuildGraph& g, uint32_t layer, uint32_t id) {
    return layer == 0 ? id : g.n + __ldg(g.up_off + id) + layer - 1;
}

// Metric distance of `row` against `q` (any memory, 16-byte aligned, padded
// rows) for the lane's group of eight; valid in every lane of the group.
// The terms are (q - row)^2 or q * row: the reference's distance(q, row).
__device__ __forceinline__ float pair_distance(int metric, const float* row, const float* q, int dim, int g8) {
    float s = metric == 0 ? group_sum<true, true>(row, q, dim, g8) : group_sum<false, true>(row, q, dim, g8);
    s = __shfl_sync(kFull, s, lane_id() & ~7);
    return metric_from_sum(metric, s);
}

// Distances from the query row (shared) to the lanes in F (ids in lane
// order `my_id`): fd[lane] for each lane of F.
__device__ __forceinline__ void fresh_distances(const BuildGraph& g, BWarp& w, uint32_t my_id, uint32_t F) {
    const int lane = lane_id();
    const int gi = lane >> 3, g8 = lane & 7;
    if ((F >> lane) & 1u) w.fr[__popc(F & ((1u << lane) - 1u))] = uint32_t(lane);
    __syncwarp();
    const uint32_t nf = __popc(F);
    uint32_t r = 0;
    for (; r + 4 < nf; r += 8) {
        const uint32_t sa = r + uint32_t(gi), sb = r + 4 + uint32_t(gi);
        const bool aa = sa < nf, ab = sb < nf;
        const uint32_t pa = aa ? w.fr[sa] : w.fr[0], pb = ab ? w.fr[sb] : w.fr[0];
        const uint32_t ida = __shfl_sync(kFull, my_id, int(pa)), idb = __shfl_sync(kFull, my_id, int(pb));
        float s0, s1;
        if (g.metric == 0)
            group_sum2<true>(g.vec + size_t(ida) * g.dp, g.vec + size_t(idb) * g.dp, w.q, int(g.dim), g8, s0, s1);
        else
            group_sum2<false>(g.vec + size_t(ida) * g.dp, g.vec + size_t(idb) * g.dp, w.q, int(g.dim), g8, s0, s1);
        s0 = __shfl_sync(kFull, s0, lane & ~7);
        s1 = __shfl_sync(kFull, s1, lane & ~7);
        if (aa && g8 == 0) w.fd[pa] = metric_from_sum(g.metric, s0);
        if (ab && g8 == 0) w.fd[pb] = metric_from_sum(g.metric, s1);
    }
    if (r < nf) {
        const uint32_t slot = r + uint32_t(gi);
        const bool act = slot < nf;
        const uint32_t pos = act ? w.fr[slot] : w.fr[0];
        const uint32_t id = __shfl_sync(kFull, my_id, int(pos));
        float s = g.metric == 0 ? group_sum<true>(g.vec + size_t(id) * g.dp, w.q, int(g.dim), g8)
                                : group_sum<false>(g.vec + size_t(id) * g.dp, w.q, int(g.dim), g8);
        s = __shfl_sync(kFull, s, lane & ~7);
        if (act && g8 == 0) w.fd[pos] = metric_from_sum(g.metric, s);
    }
    __syncwarp();
}

// Distance from the query row to one node, in every lane.
__device__ __forceinline__ float query_distance(const BuildGraph& g, const BWarp& w, uint32_t id) {
    const int g8 = lane_id() & 7;
    float s = g.metric == 0 ? group_sum<true>(g.vec + size_t(id) * g.dp, w.q, int(g.dim), g8)
                            : group_sum<false>(g.vec + size_t(id) * g.dp, w.q, int(g.dim), g8);
    s = __shfl_sync(kFull, s, 0);
    return metric_from_sum(g.metric, s);
}

__device__ __forceinline__ bool bvisit(BWarp& w, uint32_t id) {
    if (w.bitmap) {
        const uint32_t bit = 1u << (id & 31);
        return (atomicOr(&w.spill[id >> 5], bit) & bit) == 0;
    }
    uint32_t h = uint32_t((uint64_t(id * 0x9E3779B1u) * w.hash_cap) >> 32);
    for (uint32_t probe = 0; probe < w.hash_cap; ++probe) {
        const uint32_t old = atomicCAS(&w.H[h], kEmpty, id);
        if (old == kEmpty) return true;
        if (old == id) return false;
        h = h + 1 == w.hash_cap ? 0u : h + 1;
    }
    return true;  // unreachable below the load limit
}

// Moves the visited hash into the warp's bitmap.
__device__ __forceinline__ void bspill(BWarp& w) {
    const int lane = lane_id();
    for (uint32_t i = lane; i < w.hash_cap; i += 32) {
        const uint32_t v = w.H[i];
        if (v != kEmpty) atomicOr(&w.spill[v >> 5], 1u << (v & 31));
    }
    __syncwarp();
    w.bitmap = true;
}

// greedy_closest (src/hnsw/search.rs:49-68) on an upper layer.
__device__ uint64_t bgreedy(const BuildGraph& g, BWarp& w, uint64_t best, uint32_t layer) {
    const int lane = lane_id();
    const uint32_t cap = list_cap(g, layer);
    for (;;) {
        const uint32_t from = pid(best);
        const uint32_t* blk = list_ptr(g, layer, from);
        float bd = pdist(best);
        uint32_t bid = from;
        ++w.nlU;
        for (uint32_t b = 0; b < cap; b += 32) {
            const uint32_t id = (b + lane < cap) ? __ldg(blk + b + lane) : kEmpty;
            const uint32_t V = __ballot_sync(kFull, id != kEmpty);
            if (V == 0) break;
            fresh_distances(g, w, id, V);
            w.nd += __popc(V);
            float d = ((V >> lane) & 1u) ? w.fd[lane] : __int_as_float(0x7f800000);
            int idx = lane;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float od = __shfl_down_sync(kFull, d, off);
                const int oi = __shfl_down_sync(kFull, idx, off);
                if (od < d || (od == d && oi < idx)) {
                    d = od;
                    idx = oi;
                }
            }
            d = __shfl_sync(kFull, d, 0);
            idx = __shfl_sync(kFull, idx, 0);
            if (((V >> idx) & 1u) && d < bd) {
                bd = d;
                bid = __shfl_sync(kFull, id, idx);
            }
            if (V != kFull) break;
        }
        if (bid == from) return best;
        best = pack(bd, bid);
    }
}

// search_layer (src/hnsw/search.rs:81-142) from the entry points R[0, ne)
// (ascending, distinct: the previous layer's results) with admission
// `n != self` (build.rs:71-72). Results ascending in R; returns their count.
//
// One array serves as the results heap and as the live part of the
// candidate heap: every candidate the reference can still expand is a
// result not yet expanded (flag bit clear) or an evicted tie in T. The next
// expansion is the first unexpanded result, else the first tie; the
// reference's stop rule can only fire on a tie.
__device__ uint32_t bsearch_layer(const BuildGraph& g, BWarp& w, uint32_t self, uint32_t layer, uint32_t ne,
                                  uint32_t ef, uint32_t& inexact, uint32_t& spilled) {
    const int lane = lane_id();
    const uint32_t cap = list_cap(g, layer);
    uint64_t* U = w.R;
    uint64_t* T = w.T;
    for (uint32_t i = lane; i < w.hash_cap; i += 32) w.H[i] = kEmpty;
    __syncwarp();
    w.bitmap = false;
    const uint32_t hash_limit = (w.hash_cap >> 2) * 3;
    uint32_t visited = ne;
    if (ne > hash_limit) {
        w.bitmap = true;
        spilled = 1;
    }
    for (uint32_t i = lane; i < ne; i += 32) {
        bvisit(w, pid(U[i]));
        U[i] = to_upack(U[i]);
    }
    __syncwarp();
    uint32_t rs = ne, nt = 0, nx = 0;
    for (;;) {
        // Next candidate: the first unexpanded result, else the first tie.
        uint32_t p = rs;
        for (uint32_t b = nx; b < rs; b += 32) {
            const uint32_t i = b + lane;
            const uint32_t M = __ballot_sync(kFull, i < rs && !(U[i] & 1ull));
            if (M) {
                p = b + uint32_t(__ffs(int(M)) - 1);
                break;
            }
        }
        uint64_t cur;
        if (p < rs) {
            cur = U[p];
            __syncwarp();
            if (lane == 0) U[p] = cur | 1ull;
            nx = p + 1;
        } else {
            if (nt == 0) break;
            cur = T[0];
            for (uint32_t b = 0; b + 1 < nt; b += 32) {
                const uint32_t i = b + lane;
                const uint64_t v = i + 1 < nt ? T[i + 1] : 0;
                __syncwarp();
                if (i + 1 < nt) T[i] = v;
            }
            --nt;
            nx = rs;
            if (rs >= ef && pdist(cur) > pdist(U[rs - 1])) break;
        }
        __syncwarp();
        const uint32_t* row = list_ptr(g, layer, uint32_t(cur) >> 1);
        if (layer) ++w.nlU;
        else ++w.nl0;
        for (uint32_t b = 0; b < cap; b += 32) {
            const uint32_t id = (b + lane < cap) ? __ldg(row + b + lane) : kEmpty;
            const bool valid = id != kEmpty;
            const uint32_t V = __ballot_sync(kFull, valid);
            if (V == 0) break;
            if (!w.bitmap && visited + __popc(V) > hash_limit) {
                bspill(w);
                spilled = 1;
            }
            const bool fresh = valid && bvisit(w, id);
            const uint32_t F = __ballot_sync(kFull, fresh);
            visited += __popc(F);
            if (F != 0) {
                fresh_distances(g, w, id, F);
                w.nd += __popc(F);
                const bool adm = fresh && id != self;
                const uint32_t A = __ballot_sync(kFull, adm);
                const float my_d = fresh ? w.fd[lane] : 0.0f;
                uint32_t P = F;
                if (rs >= ef) P &= __ballot_sync(kFull, fresh && my_d < pdist(U[rs - 1]));
                // The node itself is never in the graph while it is linked;
                // it would be a candidate that is not a result.
                if (P & ~A) inexact = 1;
                P &= A;
                if (P == 0) {
                    if (V != kFull) break;
                    continue;
                }
                const bool inP = (P >> lane) & 1u;
                const uint64_t my_x = upack(my_d, id);
                // Equal distances among the improving neighbors or with a
                // result make the evaluation order matter: sequential path.
                const float dz = __fadd_rn(my_d, 0.0f);
                const unsigned same =
                    __match_any_sync(kFull, inP ? __float_as_uint(dz) : (0x7FC00000u | uint32_t(lane)));
                uint32_t pr = 0;
                bool tie = inP && __popc(same) > 1;
                if (inP) {
                    pr = lower_bound(U, 0, rs, my_x);
                    if (pr < rs && pdist(U[pr]) == my_d) tie = true;
                    if (pr > 0 && pdist(U[pr - 1]) == my_d) tie = true;
                }
                if (!__any_sync(kFull, tie)) {
                    // Rank among the results and the improving neighbors
                    // before it in list order: it improves iff below ef.
                    uint32_t before = 0;
                    for (uint32_t bits = P; bits; bits &= bits - 1) {
                        const int j = __ffs(bits) - 1;
                        const uint64_t xj = __shfl_sync(kFull, my_x, j);
                        before += (j < lane && xj < my_x) ? 1u : 0u;
                    }
                    const uint32_t I = __ballot_sync(kFull, inP && pr + before < ef);
                    if (I) {
                        nx = min(nx, merge_all(U, rs, I, my_x));
                        const uint32_t total = rs + uint32_t(__popc(I));
                        if (total > ef) {
                            // Evicted entries that tie with the new worst.
                            const float wd = pdist(U[ef - 1]);
                            const uint32_t i = ef + uint32_t(lane);
                            const uint64_t v = i < total ? U[i] : 0;
                            uint32_t E = __ballot_sync(kFull, i < total && !(v & 1ull) && pdist(v) == wd);
                            while (E) {
                                const int j = __ffs(int(E)) - 1;
                                E &= E - 1;
                                tie_add(T, nt, __shfl_sync(kFull, v, j), wd, inexact);
                            }
                            rs = ef;
                        } else {
                            rs = total;
                        }
                    }
                } else {
                    while (P) {
                        const int i = __ffs(P) - 1;
                        P &= P - 1;
                        const float d = __shfl_sync(kFull, my_d, i);
                        const uint32_t nid = __shfl_sync(kFull, id, i);
                        const bool improves = rs < ef || d < pdist(U[rs - 1]);
                        if (!improves) continue;
                        const uint32_t pos = sorted_insert(U, 0, rs, upack(d, nid));
                        nx = min(nx, pos);
                        if (++rs > ef) {
                            rs = ef;
                            const uint64_t v = U[ef];
                            if (!(v & 1ull) && pdist(v) == pdist(U[ef - 1])) tie_add(T, nt, v, pdist(v), inexact);
                        }
                    }
                }
            }
            if (V != kFull) break;
        }
    }
    for (uint32_t i = lane; i < rs; i += 32) U[i] = from_upack(U[i]);
    __syncwarp();
    if (w.bitmap) {
        for (uint32_t i = lane; i < w.spill_words; i += 32) w.spill[i] = 0;
        __syncwarp();
        w.bitmap = false;
    }
    return rs;
}

// The heuristic of select_neighbors (build.rs:165-197) over the ascending
// candidates X[0, n), at most mm kept. Candidate rows are staged on chip in
// chunks of stage_rows (cp.async); the kept rows stay in the stage (one
// chunk), in `selrows` (several chunks), or are read from HBM. Writes
// sel/seld; returns the count.
__device__ uint32_t bheuristic(const BuildGraph& g, const uint64_t* X, uint32_t n, uint32_t mm, bool keep_pruned,
                               float* stage, uint32_t stage_rows, float* selrows, uint32_t* sel, float* seld,
                               uint32_t* sslot, uint64_t* disc, uint32_t& npair) {
    const int lane = lane_id();
    const int gi = lane >> 3, g8 = lane & 7;
    const uint32_t dp = g.dp;
    const bool single = stage && n <= stage_rows;
    uint32_t nsel = 0, ndisc = 0;
    const uint32_t chunk = stage ? stage_rows : 32u;
    for (uint32_t i0 = 0; i0 < n && nsel < mm; i0 += chunk) {
        const uint32_t nr = min(chunk, n - i0);
        if (stage) {
            const uint32_t cpr = dp >> 2;
            for (uint32_t t = lane; t < nr * cpr; t += 32) {
                const uint32_t slot = t / cpr, part = t - slot * cpr;
                cp_async16(stage + size_t(slot) * dp + part * 4, g.vec + size_t(pid(X[i0 + slot])) * dp + part * 4);
            }
            cp_async_wait_all();
            __syncwarp();
        }
        for (uint32_t r = 0; r < nr && nsel < mm; ++r) {
            const uint64_t x = X[i0 + r];
            const float dc = pdist(x);
            const float* crow = stage ? stage + size_t(r) * dp : g.vec + size_t(pid(x)) * dp;
            bool diverse = true;
            for (uint32_t s0 = 0; s0 < nsel; s0 += 4) {
                const uint32_t s = s0 + uint32_t(gi);
                const bool act = s < nsel;
                const uint32_t sc = act ? s : 0u;
                const float* srow = single ? stage + size_t(sslot[sc]) * dp
                                           : (selrows ? selrows + size_t(sc) * dp : g.vec + size_t(sel[sc]) * dp);
                const float d = pair_distance(g.metric, srow, crow, int(g.dim), g8);
                npair += min(4u, nsel - s0);
                if (__any_sync(kFull, act && !(d >= dc))) {
                    diverse = false;
                    break;
                }
            }
            if (diverse) {
                if (lane == 0) {
                    sel[nsel] = pid(x);
                    seld[nsel] = dc;
                    sslot[nsel] = r;
                }
                if (!single && selrows)
                    for (uint32_t k = lane * 4; k < dp; k += 128)
                        *reinterpret_cast<float4*>(selrows + size_t(nsel) * dp + k) =
                            *reinterpret_cast<const float4*>(crow + k);
                ++nsel;
            } else if (keep_pruned && ndisc < mm) {
                if (lane == 0) disc[ndisc] = x;
                ++ndisc;
            }
            __syncwarp();
        }
        __syncwarp();
    }
    const uint32_t take = min(ndisc, mm - nsel);
    for (uint32_t j = lane; j < take; j += 32) {
        sel[nsel + j] = pid(disc[j]);
        seld[nsel + j] = pdist(disc[j]);
    }
    __syncwarp();
    return nsel + take;
}

// The heuristic over an unsorted pool P[0, n) (extend_candidates): the next
// candidate is the pool's minimum, taken out by overwriting it with ~0. Rows
// come from HBM.
__device__ uint32_t bheuristic_pool(const BuildGraph& g, uint64_t* P, uint32_t n, uint32_t mm, bool keep_pruned,
                                    uint32_t* sel, float* seld, uint64_t* disc, uint32_t& npair) {
    const int lane = lane_id();
    const int gi = lane >> 3, g8 = lane & 7;
    uint32_t nsel = 0, ndisc = 0;
    for (uint32_t step = 0; step < n && nsel < mm; ++step) {
        uint64_t best = ~0ull;
        for (uint32_t i = lane; i < n; i += 32) best = min(best, P[i]);
        best = warp_min_u64(best);
        if (best == ~0ull) break;
        for (uint32_t i = lane; i < n; i += 32)
            if (P[i] == best) P[i] = ~0ull;
        __syncwarp();
        const float dc = pdist(best);
        const float* crow = g.vec + size_t(pid(best)) * g.dp;
        bool diverse = true;
        for (uint32_t s0 = 0; s0 < nsel; s0 += 4) {
            const uint32_t s = s0 + uint32_t(gi);
            const bool act = s < nsel;
            const float* srow = g.vec + size_t(sel[act ? s : 0u]) * g.dp;
            const float d = pair_distance(g.metric, srow, crow, int(g.dim), g8);
            npair += min(4u, nsel - s0);
            if (__any_sync(kFull, act && !(d >= dc))) {
                diverse = false;
                break;
            }
        }
        if (diverse) {
            if (lane == 0) {
                sel[nsel] = pid(best);
                seld[nsel] = dc;
            }
            ++nsel;
        } else if (keep_pruned && ndisc < mm) {
            if (lane == 0) disc[ndisc] = best;
            ++ndisc;
        }
        __syncwarp();
    }
    const uint32_t take = min(ndisc, mm - nsel);
    for (uint32_t j = lane; j < take; j += 32) {
        sel[nsel + j] = pid(disc[j]);
        seld[nsel + j] = pdist(disc[j]);
    }
    __syncwarp();
    return nsel + take;
}

// Open-addressing set insert in a global-memory table (lane-parallel).
__device__ __forceinline__ bool gset_insert(uint32_t* T, uint32_t cap, uint32_t id) {
    const uint32_t mask = cap - 1;
    uint32_t h = uint32_t((uint64_t(id * 0x9E3779B1u) * cap) >> 32);
    for (uint32_t probe = 0; probe < cap; ++probe) {
        const uint32_t old = atomicCAS(&T[h], kEmpty, id);
        if (old == kEmpty) return true;
        if (old == id) return false;
        h = (h + 1) & mask;
    }
    return false;
}

// extend_candidates (build.rs:202-222): the pool is X[0, n) plus every
// neighbor (on `layer`) of those candidates not already in it and not the
// base, with its distance to the base row `qrow`. Written to P (unsorted);
// returns the pool size.
__device__ uint32_t extend_pool(const BuildGraph& g, const uint64_t* X, uint32_t n, uint32_t base_id,
                                const float* qrow, uint32_t layer, uint64_t* P, uint32_t pcap, uint32_t* T,
                                uint32_t tcap, uint32_t* fr, uint32_t& npair) {
    const int lane = lane_id();
    const int gi = lane >> 3, g8 = lane & 7;
    for (uint32_t i = lane; i < tcap; i += 32) T[i] = kEmpty;
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) {
        gset_insert(T, tcap, pid(X[i]));
        P[i] = X[i];
    }
    if (lane == 0) gset_insert(T, tcap, base_id);
    __syncwarp();
    uint32_t np = n;
    const uint32_t cap = list_cap(g, layer);
    for (uint32_t c = 0; c < n; ++c) {
        const uint32_t* blk = list_ptr(g, layer, pid(X[c]));
        for (uint32_t b = 0; b < cap; b += 32) {
            const uint32_t id = (b + lane < cap) ? blk[b + lane] : kEmpty;
            const uint32_t V = __ballot_sync(kFull, id != kEmpty);
            if (V == 0) break;
            const bool fresh = id != kEmpty && gset_insert(T, tcap, id);
            const uint32_t F = __ballot_sync(kFull, fresh);
            if ((F >> lane) & 1u) fr[__popc(F & ((1u << lane) - 1u))] = id;
            __syncwarp();
            const uint32_t nf = __popc(F);
            npair += nf;
            for (uint32_t r = 0; r < nf; r += 4) {
                const uint32_t slot = r + uint32_t(gi);
                const bool act = slot < nf;
                const uint32_t nid = fr[act ? slot : 0u];
                const float d = pair_distance(g.metric, g.vec + size_t(nid) * g.dp, qrow, int(g.dim), g8);
                if (act && g8 == 0 && np + slot < pcap) P[np + slot] = pack(d, nid);
            }
            np = min(np + nf, pcap);
            __syncwarp();
            if (V != kFull) break;
        }
    }
    return np;
}

__device__ void carve_search(BWarp& w, char* p, const BuildArgs& a, uint32_t mm) {
    const uint32_t dp = a.g.dp;
    w.H = reinterpret_cast<uint32_t*>(p);
    p += a16(size_t(a.region_bytes));
    w.q = reinterpret_cast<float*>(p);
    p += a16(size_t(dp) * 4);
    w.selrows = a.sel_rows ? reinterpret_cast<float*>(p) : nullptr;
    if (a.sel_in_stage) w.selrows = reinterpret_cast<float*>(w.H) + size_t(a.stage_rows) * dp;
    p += a16(size_t(a.sel_rows) * dp * 4);
    w.R = reinterpret_cast<uint64_t*>(p);
    p += a16(size_t(a.ef + 33) * 8);
    w.T = reinterpret_cast<uint64_t*>(p);
    p += a16(size_t(kTieCap + 1) * 8);
    w.disc = reinterpret_cast<uint64_t*>(p);
    p += a16(size_t(mm) * 8);
    w.fr = reinterpret_cast<uint32_t*>(p);
    p += 128;
    w.fd = reinterpret_cast<float*>(p);
    p += 128;
    w.sel = reinterpret_cast<uint32_t*>(p);
    p += a16(size_t(mm) * 4);
    w.seld = reinterpret_cast<float*>(p);
    p += a16(size_t(mm) * 4);
    w.sslot = reinterpret_cast<uint32_t*>(p);
    w.hash_cap = a.hash_cap;
    w.bitmap = false;
    w.nd = w.nl0 = w.nlU = 0;
}

// Appends the reverse edges sel[j] <- self on `layer` (one record each).
__device__ __forceinline__ void emit_records(const BuildArgs& a, const BWarp& w, uint32_t self, uint32_t layer,
                                             uint32_t nsel) {
    const int lane = lane_id();
    uint32_t rb = 0;
    if (lane == 0 && nsel) rb = atomicAdd(&a.wc->nrec, nsel);
    rb = __shfl_sync(kFull, rb, 0);
    for (uint32_t j = lane; j < nsel; j += 32) {
        const uint32_t u = w.sel[j];
        const uint32_t key = list_key(a.g, layer, u);
        const uint32_t rank = atomicAdd(&a.cnt[key], 1u);
        if (rank == 0) {
            const uint32_t t = atomicAdd(&a.wc->ntouched, 1u);
            a.touched[t] = (uint64_t(layer) << 32) | u;
        }
        if (rb + j < a.max_records) a.rec[rb + j] = EdgeRecord{key, rank, self, __float_as_uint(w.seld[j])};
    }
}

__global__ void build_search_kernel(BuildArgs a) {
    extern __shared__ __align__(16) char smem[];
    const int lane = lane_id();
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * a.warps_per_block + warp;
    const uint32_t mm = a.g.m;
    char* base = a.gscratch ? a.gscratch + size_t(slot) * a.bytes_per_warp : smem + size_t(warp) * a.bytes_per_warp;
    BWarp w;
    carve_search(w, base, a, mm);
    w.spill = a.spill + size_t(slot) * a.spill_words;
    w.spill_words = a.spill_words;
    const BuildGraph& g = a.g;
    uint32_t inexact_total = 0, spills_total = 0, npair = 0;
    for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(&a.wc->next, 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= a.count) break;
        const uint32_t self = a.first + i;
        const float* src = g.vec + size_t(self) * g.dp;
        for (uint32_t k = lane * 4; k < g.dp; k += 128)
            *reinterpret_cast<float4*>(w.q + k) = *reinterpret_cast<const float4*>(src + k);
        __syncwarp();
        const uint32_t level = __ldg(g.levels + self);
        uint64_t ep = pack(query_distance(g, w, a.entry), a.entry);
        ++w.nd;
        for (uint32_t layer = a.top; layer > level; --layer) ep = bgreedy(g, w, ep, layer);
        if (lane == 0) w.R[0] = ep;
        __syncwarp();
        uint32_t ne = 1;
        for (int layer = int(min(level, a.top)); layer >= 0; --layer) {
            uint32_t inexact = 0, spilled = 0;
            const uint32_t rs = bsearch_layer(g, w, self, uint32_t(layer), ne, a.ef, inexact, spilled);
            inexact_total += inexact;
            spills_total += spilled;
            // select_neighbors(self, query, found, m, layer)
            uint32_t nsel;
            if (a.selection == 0) {
                nsel = min(rs, mm);
                for (uint32_t j = lane; j < nsel; j += 32) {
                    w.sel[j] = pid(w.R[j]);
                    w.seld[j] = pdist(w.R[j]);
                }
                __syncwarp();
            } else if (a.extend) {
                uint64_t* P = a.ext + size_t(slot) * a.ext_cap;
                uint32_t* T = a.ext_hash + size_t(slot) * a.ext_hash_cap;
                const uint32_t np =
                    extend_pool(g, w.R, rs, self, w.q, uint32_t(layer), P, a.ext_cap, T, a.ext_hash_cap, w.fr, npair);
                nsel = bheuristic_pool(g, P, np, mm, a.keep_pruned != 0, w.sel, w.seld, w.disc, npair);
            } else {
                nsel = bheuristic(g, w.R, rs, mm, a.keep_pruned != 0, a.stage_rows ? reinterpret_cast<float*>(w.H) : nullptr,
                                  a.stage_rows, w.selrows, w.sel, w.seld, w.sslot, w.disc, npair);
            }
            // install_own_neighbors: the node's list is still empty.
            uint32_t* own = list_ptr(g, uint32_t(layer), self);
            for (uint32_t j = lane; j < nsel; j += 32) own[j] = w.sel[j];
            emit_records(a, w, self, uint32_t(layer), nsel);
            __syncwarp();
            // The results are the next layer's entry points (the search
            // always returns its admitted entries, so rs > 0).
            ne = rs;
            __syncwarp();
        }
    }
    if (lane == 0) {
        if (inexact_total | spills_total) {
            atomicAdd(&a.totals->inexact, (unsigned long long)inexact_total);
            atomicAdd(&a.totals->spills, (unsigned long long)spills_total);
        }
        atomicAdd(&a.totals->dist_search, (unsigned long long)w.nd);
        atomicAdd(&a.totals->dist_select, (unsigned long long)npair);
        atomicAdd(&a.totals->lists0, (unsigned long long)w.nl0);
        atomicAdd(&a.totals->listsU, (unsigned long long)w.nlU);
    }
}

__device__ __forceinline__ uint32_t ukey(const BuildGraph& g, uint64_t t) {
    const uint32_t layer = uint32_t(t >> 32), u = uint32_t(t);
    return layer == 0 ? u : g.n + g.up_off[u] + layer - 1;
}

__global__ void bucket_base_kernel(BuildArgs a) {
    const uint32_t nt = a.wc->ntouched;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        const uint32_t key = ukey(a.g, a.touched[t]);
        a.base[key] = atomicAdd(&a.wc->cursor, a.cnt[key]);
    }
}

__global__ void bucket_fill_kernel(BuildArgs a) {
    const uint32_t nr = min(a.wc->nrec, a.max_records);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += gridDim.x * blockDim.x) {
        const EdgeRecord e = a.rec[r];
        a.bkt[a.base[e.key] + e.rank] = (uint64_t(e.v) << 32) | e.dbits;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.totals->records, (unsigned long long)nr);
}

struct CWarp {
    float* q;        // dp: the list owner's row
    float* stage;    // stage_rows * dp
    float* selrows;  // sel_rows * dp or null
    uint32_t* lid;   // cap + 1
    float* du;       // cap + 1 (NaN: not computed yet)
    uint64_t* X;     // cap + 1
    uint64_t* X2;    // cap + 1
    uint64_t* disc;  // cap
    uint32_t* sel;   // cap
    float* seld;     // cap
    uint32_t* sslot; // cap
    uint32_t* fr;    // 32
    float* fd;       // 32
};

__device__ void carve_connect(CWarp& w, char* p, const BuildArgs& a, uint32_t cap) {
    const uint32_t dp = a.g.dp;
    w.q = reinterpret_cast<float*>(p);
    p += a16(size_t(dp) * 4);
    w.stage = reinterpret_cast<float*>(p);
    p += a16(size_t(a.c_stage_rows) * dp * 4);
    w.selrows = a.c_sel_rows ? reinterpret_cast<float*>(p) : nullptr;
    p += a16(size_t(a.c_sel_rows) * dp * 4);
    w.X = reinterpret_cast<uint64_t*>(p);
    p += a16(size_t(cap + 1) * 8);
    w.X2 = reinterpret_cast<uint64_t*>(p);
    p += a16(size_t(cap + 1) * 8);
    w.disc = reinterpret_cast<uint64_t*>(p);
    p += a16(size_t(cap) * 8);
    w.lid = reinterpret_cast<uint32_t*>(p);
    p += a16(size_t(cap + 1) * 4);
    w.du = reinterpret_cast<float*>(p);
    p += a16(size_t(cap + 1) * 4);
    w.sel = reinterpret_cast<uint32_t*>(p);
    p += a16(size_t(cap) * 4);
    w.seld = reinterpret_cast<float*>(p);
    p += a16(size_t(cap) * 4);
    w.sslot = reinterpret_cast<uint32_t*>(p);
    p += a16(size_t(cap) * 4);
    w.fr = reinterpret_cast<uint32_t*>(p);
    p += 128;
    w.fd = reinterpret_cast<float*>(p);
}

// connect(u, v, layer) for every record of a list, in ascending v.
__global__ void build_connect_kernel(BuildArgs a) {
    extern __shared__ __align__(16) char smem[];
    const int lane = lane_id();
    const int gi = lane >> 3, g8 = lane & 7;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * a.c_warps_per_block + warp;
    const uint32_t nwarps = gridDim.x * a.c_warps_per_block;
    const BuildGraph& g = a.g;
    const uint32_t capmax = max(g.m0, g.m);
    char* base = a.c_gscratch ? a.c_gscratch + size_t(slot) * a.c_bytes_per_warp
                              : smem + size_t(warp) * a.c_bytes_per_warp;
    CWarp w;
    carve_connect(w, base, a, capmax);
    const uint32_t nt = a.wc->ntouched;
    uint32_t shrinks = 0, ndist = 0;
    for (uint32_t t = slot; t < nt; t += nwarps) {
        const uint64_t te = a.touched[t];
        const uint32_t layer = uint32_t(te >> 32), u = uint32_t(te);
        const uint32_t key = ukey(g, te);
        const uint32_t cap = list_cap(g, layer);
        uint32_t* row = list_ptr(g, layer, u);
        const uint32_t nb = a.cnt[key];
        uint64_t* bk = a.bkt + a.base[key];
        // Current list.
        uint32_t c = 0;
        for (uint32_t b = 0; b < cap; b += 32) {
            const uint32_t id = (b + lane < cap) ? row[b + lane] : kEmpty;
            if (id != kEmpty) {
                w.lid[b + lane] = id;
                w.du[b + lane] = __int_as_float(0x7fc00000);
            }
            const uint32_t V = __ballot_sync(kFull, id != kEmpty);
            c += __popc(V);
            if (V != kFull) break;
        }
        const float* src = g.vec + size_t(u) * g.dp;
        for (uint32_t k = lane * 4; k < g.dp; k += 128)
            *reinterpret_cast<float4*>(w.q + k) = *reinterpret_cast<const float4*>(src + k);
        __syncwarp();
        for (uint32_t step = 0; step < nb; ++step) {
            uint64_t best = ~0ull;
            for (uint32_t i = lane; i < nb; i += 32) best = min(best, bk[i]);
            best = warp_min_u64(best);
            for (uint32_t i = lane; i < nb; i += 32)
                if (bk[i] == best) bk[i] = ~0ull;
            const uint32_t v = uint32_t(best >> 32);
            const float dv = __uint_as_float(uint32_t(best));
            if (v >= g.n) continue;  // never: every bucket slot holds a record
            bool present = false;
            for (uint32_t b = 0; b < c; b += 32) present |= __any_sync(kFull, b + lane < c && w.lid[b + lane] == v);
            __syncwarp();
            if (present) continue;
            if (c < cap) {
                if (lane == 0) {
                    w.lid[c] = v;
                    w.du[c] = dv;
                }
                ++c;
                __syncwarp();
                continue;
            }
            // write_shrunk: distances of the members to u, then selection
            // over the sorted candidates with the list's capacity.
            ++shrinks;
            if (lane == 0) {
                w.lid[c] = v;
                w.du[c] = dv;
            }
            __syncwarp();
            const uint32_t n = c + 1;
            for (uint32_t b = 0; b < n; b += 32) {
                const uint32_t i = b + lane;
                const bool need = i < n && isnan(w.du[i]);
                const uint32_t F = __ballot_sync(kFull, need);
                if ((F >> lane) & 1u) w.fr[__popc(F & ((1u << lane) - 1u))] = i;
                __syncwarp();
                const uint32_t nf = __popc(F);
                ndist += nf;
                for (uint32_t r = 0; r < nf; r += 4) {
                    const uint32_t s = r + uint32_t(gi);
                    const bool act = s < nf;
                    const uint32_t idx = w.fr[act ? s : 0u];
                    const float d = pair_distance(g.metric, g.vec + size_t(w.lid[idx]) * g.dp, w.q, int(g.dim), g8);
                    if (act && g8 == 0) w.du[idx] = d;
                }
                __syncwarp();
            }
            for (uint32_t i = lane; i < n; i += 32) w.X[i] = pack(w.du[i], w.lid[i]);
            __syncwarp();
            // Rank sort (entries are distinct).
            for (uint32_t i = lane; i < n; i += 32) {
                const uint64_t x = w.X[i];
                uint32_t r = 0;
                for (uint32_t j = 0; j < n; ++j) r += w.X[j] < x ? 1u : 0u;
                w.X2[r] = x;
            }
            __syncwarp();
            uint32_t ns;
            if (a.selection == 0) {
                ns = min(n, cap);
                for (uint32_t j = lane; j < ns; j += 32) {
                    w.sel[j] = pid(w.X2[j]);
                    w.seld[j] = pdist(w.X2[j]);
                }
                __syncwarp();
            } else if (a.extend) {
                uint64_t* P = a.ext + size_t(slot) * a.ext_cap;
                uint32_t* T = a.ext_hash + size_t(slot) * a.ext_hash_cap;
                const uint32_t np =
                    extend_pool(g, w.X2, n, u, w.q, layer, P, a.ext_cap, T, a.ext_hash_cap, w.fr, ndist);
                ns = bheuristic_pool(g, P, np, cap, a.keep_pruned != 0, w.sel, w.seld, w.disc, ndist);
            } else {
                ns = bheuristic(g, w.X2, n, cap, a.keep_pruned != 0, a.c_stage_rows ? w.stage : nullptr,
                                a.c_stage_rows, w.selrows, w.sel, w.seld, w.sslot, w.disc, ndist);
            }
            for (uint32_t j = lane; j < ns; j += 32) {
                w.lid[j] = w.sel[j];
                w.du[j] = w.seld[j];
            }
            c = ns;
            __syncwarp();
        }
        // The new list, padded with the sentinel.
        uint32_t* out = a.extend ? a.side + size_t(t) * a.side_stride : row;
        for (uint32_t j = lane; j < cap; j += 32) out[j] = j < c ? w.lid[j] : kEmpty;
        if (!a.extend && lane == 0) a.cnt[key] = 0;
        __syncwarp();
    }
    if (lane == 0 && (shrinks | ndist)) {
        atomicAdd(&a.totals->shrinks, (unsigned long long)shrinks);
        atomicAdd(&a.totals->dist_connect, (unsigned long long)ndist);
    }
}

// Extension mode: copies the new lists into the graph and clears the counts.
__global__ void build_apply_kernel(BuildArgs a) {
    const uint32_t nt = a.wc->ntouched;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = lane_id();
    for (uint32_t t = warp; t < nt; t += nwarps) {
        const uint64_t te = a.touched[t];
        const uint32_t layer = uint32_t(te >> 32), u = uint32_t(te);
        const uint32_t cap = list_cap(a.g, layer);
        uint32_t* row = list_ptr(a.g, layer, u);
        const uint32_t* in = a.side + size_t(t) * a.side_stride;
        for (uint32_t j = lane; j < cap; j += 32) row[j] = in[j];
        if (lane == 0) a.cnt[ukey(a.g, te)] = 0;
    }
}

}  // namespace
}  // namespace dev

size_t build_search_bytes(uint32_t dp, uint32_t ef, uint32_t region_bytes, uint32_t mm, uint32_t sel_rows) {
    using dev::a16;
    return a16(size_t(region_bytes)) + a16(size_t(dp) * 4) + a16(size_t(sel_rows) * dp * 4) +
           a16(size_t(ef + 33) * 8) + a16(size_t(dev::kTieCap + 1) * 8) + a16(size_t(mm) * 8) + 256 +
           3 * a16(size_t(mm) * 4);
}

size_t build_connect_bytes(uint32_t dp, uint32_t cap, uint32_t stage_rows, uint32_t sel_rows) {
    using dev::a16;
    return a16(size_t(dp) * 4) + a16(size_t(stage_rows) * dp * 4) + a16(size_t(sel_rows) * dp * 4) +
           2 * a16(size_t(cap + 1) * 8) + a16(size_t(cap) * 8) + 2 * a16(size_t(cap + 1) * 4) +
           3 * a16(size_t(cap) * 4) + 256;
}

cudaError_t gpu_build_occupancy(bool search, int threads, size_t smem, int* blocks) {
    const void* f = search ? reinterpret_cast<const void*>(dev::build_search_kernel)
                           : reinterpret_cast<const void*>(dev::build_connect_kernel);
    cudaError_t e = raise_smem_limit(f);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, f, threads, smem);
}

cudaError_t launch_build_search(const BuildArgs& a, uint32_t search_blocks, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(a.wc, 0, sizeof(WaveCounters), stream);
    if (e != cudaSuccess) return e;
    const size_t s_smem = a.gscratch ? 0 : size_t(a.bytes_per_warp) * a.warps_per_block;
    if (s_smem > 48 * 1024 && (e = raise_smem_limit(reinterpret_cast<const void*>(dev::build_search_kernel))) !=
                                  cudaSuccess)
        return e;
    dev::build_search_kernel<<<search_blocks, a.warps_per_block * 32, s_smem, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_build_connect(const BuildArgs& a, uint32_t connect_blocks, uint32_t small_blocks,
                                 cudaStream_t stream) {
    cudaError_t e;
    dev::bucket_base_kernel<<<small_blocks, 256, 0, stream>>>(a);
    dev::bucket_fill_kernel<<<small_blocks, 256, 0, stream>>>(a);
    const size_t c_smem = a.c_gscratch ? 0 : size_t(a.c_bytes_per_warp) * a.c_warps_per_block;
    if (c_smem > 48 * 1024 && (e = raise_smem_limit(reinterpret_cast<const void*>(dev::build_connect_kernel))) !=
                                  cudaSuccess)
        return e;
    dev::build_connect_kernel<<<connect_blocks, a.c_warps_per_block * 32, c_smem, stream>>>(a);
    if (a.extend) dev::build_apply_kernel<<<small_blocks, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace hnswgpu
