// Device-side graph construction: the launch interface of the kernels that
// link a wave of new nodes into a graph resident in HBM.
//
// A wave is a run of consecutive node ids. Every node of the wave searches
// the graph as it stood before the wave (greedy descent, then an ef-bounded
// beam per layer with the previous layer's results as entry points), selects
// its neighbors and writes its own lists; the reverse edges are then grouped
// by target list and applied in ascending order of the new node's id, each as
// HnswIndex::connect does (push, or shrink with the selection strategy when
// the list is full). A wave of one node reproduces the sequential insertion
// exactly (src/hnsw/build.rs:41-150).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hnswgpu {

// Graph under construction, in the layout of the search index: vector rows
// padded to dp floats, neighbor rows of m0p (layer 0) / mp (upper layers)
// ids with kSentinel after the live prefix; a node's upper-layer lists are
// consecutive blocks from up_off[node].
struct BuildGraph {
    uint32_t n = 0, dim = 0, dp = 0;
    uint32_t m = 0, m0 = 0, mp = 0, m0p = 0;
    int metric = 0;
    const float* vec = nullptr;
    uint32_t* adj0 = nullptr;
    const uint32_t* up_off = nullptr;
    uint32_t* adjU = nullptr;
    const uint8_t* levels = nullptr;
};

// Reverse edge u <- v on one layer, emitted by the search kernel. `key`
// names the target list: u for layer 0, n + up_off[u] + layer - 1 above.
struct EdgeRecord {
    uint32_t key, rank, v, dbits;
};

// Per-wave counters (zeroed before each wave).
struct WaveCounters {
    uint32_t next;      // search work counter
    uint32_t nrec;      // records written
    uint32_t ntouched;  // target lists with at least one record
    uint32_t cursor;    // bucket slots handed out
};

// Totals over a build (device, accumulated).
struct BuildTotals {
    unsigned long long spills;   // layer searches whose visited set moved to the bitmap
    unsigned long long inexact;  // candidate queues that had to drop a live entry
    unsigned long long shrinks;  // full lists re-selected on a reverse edge
    unsigned long long records;  // reverse edges
    // Work counters (the roofline's algorithmic traffic): distances of the
    // layer searches (greedy and beam), of the selections (pairs of rows),
    // of the connect step (owner to member and pairs), and lists read.
    unsigned long long dist_search, dist_select, dist_connect;
    unsigned long long lists0, listsU;
};

struct BuildArgs {
    BuildGraph g;
    uint32_t selection = 1;  // 0 simple, 1 heuristic
    uint32_t extend = 0, keep_pruned = 0;
    uint32_t first = 0, count = 0;  // wave nodes [first, first + count)
    uint32_t entry = 0, top = 0;    // entry point of the graph before the wave
    uint32_t ef = 0;                // max(ef_construction, m)
    // Search scratch per warp (dynamic shared memory, or global memory at
    // `gscratch` when one warp's share does not fit on chip).
    uint32_t hash_cap = 0, warps_per_block = 1, bytes_per_warp = 0;
    uint32_t stage_rows = 0, sel_rows = 0;  // rows staged for the selection; selected rows kept on chip
    uint32_t sel_in_stage = 0;  // selected rows live in the hash region after the staged rows
    uint32_t region_bytes = 0;  // the hash region (>= hash_cap * 4)
    char* gscratch = nullptr;
    uint32_t* spill = nullptr;  // per warp slot, spill_words words (zero between uses)
    uint32_t spill_words = 0;
    uint64_t* ext = nullptr;    // per warp slot, ext_cap entries (candidate extension)
    uint32_t ext_cap = 0;
    uint32_t* ext_hash = nullptr;  // per warp slot, ext_hash_cap words
    uint32_t ext_hash_cap = 0;
    // Reverse edges.
    WaveCounters* wc = nullptr;
    BuildTotals* totals = nullptr;
    EdgeRecord* rec = nullptr;
    uint32_t* cnt = nullptr;   // per target list
    uint32_t* base = nullptr;  // per target list
    uint64_t* touched = nullptr;  // (layer << 32) | u
    uint64_t* bkt = nullptr;      // (v << 32) | distance bits, grouped by list
    // Connect scratch.
    uint32_t c_warps_per_block = 1, c_bytes_per_warp = 0, c_stage_rows = 0, c_sel_rows = 0;
    char* c_gscratch = nullptr;
    uint32_t* side = nullptr;  // extension: new lists, (cap_max + 1) words per touched list
    uint32_t side_stride = 0;
    uint32_t max_records = 0;
};

// Per-warp search scratch bytes for ef, hash region bytes, selection size
// mm and row floats dp.
size_t build_search_bytes(uint32_t dp, uint32_t ef, uint32_t region_bytes, uint32_t mm, uint32_t sel_rows);
size_t build_connect_bytes(uint32_t dp, uint32_t cap, uint32_t stage_rows, uint32_t sel_rows);

// Resident blocks per SM of the search (search = true) or connect kernel.
cudaError_t gpu_build_occupancy(bool search, int threads, size_t smem, int* blocks);

// One wave in two launches on `stream`: the search step (clears the wave
// counters, then searches, selects and writes the own lists) and the connect
// step (buckets the reverse edges and applies them). `search_blocks` /
// `connect_blocks` bound the persistent grids.
cudaError_t launch_build_search(const BuildArgs& a, uint32_t search_blocks, cudaStream_t stream);
cudaError_t launch_build_connect(const BuildArgs& a, uint32_t connect_blocks, uint32_t small_blocks,
                                 cudaStream_t stream);

}  // namespace hnswgpu
