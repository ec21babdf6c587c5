// Device graph construction driven from the host builder.
#pragma once

#include <cstdint>

#include "host_index.hpp"

namespace hnswgpu {

struct GpuBuildOptions {
    double wave_fraction = 0.05;  // nodes per wave = max(1, floor(linked * fraction))
    uint32_t max_wave = 65536;
    uint32_t hash_cap = 0;        // visited-hash entries per warp (0: 16 per unit of ef)
    uint32_t timing = 0;          // record per-phase device times
};

struct GpuBuildReport {
    uint32_t waves = 0, nodes = 0;
    uint64_t spills = 0, inexact = 0, shrinks = 0, records = 0;
    double device_ms = 0.0, search_ms = 0.0, connect_ms = 0.0;
    uint64_t dist_search = 0, dist_select = 0, dist_connect = 0, lists0 = 0, listsU = 0;
    uint32_t search_warps_per_block = 0, search_blocks_per_sm = 0;
    uint32_t connect_warps_per_block = 0, connect_blocks_per_sm = 0;
    uint32_t hash_cap = 0;
};

void gpu_build_defaults(GpuBuildOptions* o);

// Links nodes [first, node_count) of `ix` on `device`: their vectors, keys
// and levels are stored and their lists empty; existing lists gain reverse
// edges. On success the lists and the entry point of `ix` are replaced; on
// failure `ix` is unchanged. Returns an HNSW_* status (message recorded).
int gpu_link(HostIndex& ix, uint32_t first, int device, const GpuBuildOptions& opt, GpuBuildReport* rep);

}  // namespace hnswgpu
