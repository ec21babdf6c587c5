// Host-side index: the in-memory form of a format-v1 file, its validating
// loader and writer, and the construction path that produces such files.
//
// Construction is not accelerated here: it is the input side of the device
// query path (the device index is flattened from a loaded HostIndex).
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

namespace hnswgpu {

constexpr uint32_t kMaxDim = 1u << 16;          // MAX_DIM (src/lib.rs:70)
constexpr uint64_t kMaxNodes = 0xFFFFFFFFull - 1; // MAX_NODES (src/lib.rs:74)
constexpr uint8_t kMaxLevel = 31;               // MAX_LEVEL (src/hnsw/mod.rs:26)
constexpr uint32_t kNoEntry = 0xFFFFFFFFu;

struct Params {
    uint32_t m = 16, m0 = 32, ef_construction = 200;
    double level_multiplier = 0.0;
    uint32_t selection = 1;  // 0 simple, 1 heuristic
    bool extend_candidates = false, keep_pruned = false;
    uint64_t seed = 0;
};

// HnswParams::new (src/params.rs:78-87).
Params default_params(uint32_t m);
// HnswParams::validate (src/params.rs:163-182). Returns "" or the name of the
// offending parameter.
const char* validate_params(const Params& p);

// Error carrier for the host side: a status plus the reference's message.
struct Err {
    int status = 0;
    std::string what;
    uint64_t a = 0, b = 0;  // extra fields (checksum stored/computed, memory required/limit)
    explicit operator bool() const { return status != 0; }
};

struct HostIndex {
    uint32_t dim = 0;
    int metric = 0;
    Params params;
    std::vector<float> vectors;
    std::vector<uint64_t> keys;
    std::vector<uint8_t> levels;
    std::vector<uint8_t> deleted;
    // Layer 0: (m0 + 1) words per node: count, then ids (src/hnsw/graph.rs:26-33).
    std::vector<uint32_t> l0;
    // Upper layers: per node, level * (m + 1) words.
    std::vector<std::vector<uint32_t>> upper;
    uint64_t entry_word = ~0ull;  // (level << 32) | id, or all ones
    std::unordered_map<uint64_t, uint32_t> key_to_id;  // live keys
    bool quantized = false;
    std::vector<float> q_offset;
    float q_scale = 1.0f;

    size_t node_count() const { return keys.size(); }
    const float* vector(uint32_t id) const { return vectors.data() + size_t(id) * dim; }
    bool has_entry() const { return entry_word != ~0ull; }
    uint32_t entry_id() const { return uint32_t(entry_word); }
    uint32_t top_level() const { return uint32_t(entry_word >> 32); }
    uint32_t capacity(unsigned layer) const { return layer == 0 ? params.m0 : params.m; }
    uint32_t* block(uint32_t id, unsigned layer) {
        return layer == 0 ? l0.data() + size_t(id) * (params.m0 + 1)
                          : upper[id].data() + size_t(layer - 1) * (params.m + 1);
    }
    const uint32_t* block(uint32_t id, unsigned layer) const {
        return const_cast<HostIndex*>(this)->block(id, layer);
    }
};

// CRC-32 IEEE (src/crc32.rs), slicing-by-8.
uint32_t crc32(const uint8_t* p, size_t n);

// io::read (src/hnsw/io.rs:236-267): every check, in the reference's order.
// max_memory == 0 selects default_memory_limit (io.rs:271-275).
Err load_index(const uint8_t* bytes, size_t len, uint64_t max_memory, HostIndex* out,
               uint64_t* required_memory);

// The stages of load_index, for a loader that verifies the checksum, the
// vectors and the neighbor lists elsewhere (the device ingest) while keeping
// the reference's order of checks and its messages.
struct FileLayout {
    uint8_t metric = 0;
    bool quantized = false;
    Params params;
    uint32_t dim = 0, n = 0, entry_id = 0;
    size_t body_len = 0;
    const uint8_t *keys = nullptr, *levels = nullptr, *dead = nullptr, *vectors = nullptr;
    size_t links_begin = 0, links_end = 0;  // byte range of the neighbor lists
    std::vector<uint64_t> node_off;         // byte offset of each node's first list
    uint64_t level_sum = 0, required = 0;
};
// Magic, version and minimum length; *body_len bytes are covered by *stored.
Err check_envelope(const uint8_t* bytes, size_t len, size_t* body_len, uint32_t* stored);
Err checksum_error(uint32_t stored, uint32_t computed);
// Header, columns, list counts and the memory limit, on a verified body.
Err scan_layout(const uint8_t* bytes, size_t body_len, uint64_t max_memory, FileLayout* out);
// Quantizer section and trailing bytes (after the lists).
Err scan_tail(const uint8_t* bytes, const FileLayout& layout, std::vector<float>* q_offset, float* q_scale);
// Entry point (last check of io.rs:517-540).
Err check_entry(const FileLayout& layout, uint64_t* entry_word);
// The messages of the checks the device ingest runs (invalid field names).
Err invalid_field(const char* what);
// io::write (src/hnsw/io.rs:103-169).
std::vector<uint8_t> write_index(const HostIndex& ix);

// f32 kernels in the reference AVX2 backend's order (src/kernels/x86.rs).
float dot_ref(const float* a, const float* b, size_t n);
float l2_ref(const float* a, const float* b, size_t n);
float metric_distance(int metric, const float* a, const float* b, size_t n);

// build::sample_level (src/hnsw/build.rs:19-28).
uint8_t sample_level(uint64_t seed, uint32_t id, double ml);

// vector::check (src/vector.rs:22-40). Returns 0 or a status, norm in *norm_sq.
int check_vector(const float* v, size_t dim, double* norm_sq);

// Construction (src/hnsw/mod.rs:181-400, src/hnsw/build.rs).
class Builder {
public:
    Builder(uint32_t dim, int metric, const Params& p);
    ~Builder();
    Err insert(uint64_t key, const float* v);
    Err insert_batch(const uint64_t* keys, const float* v, size_t n, int threads);
    bool remove(uint64_t key);
    void enable_quantization();
    const HostIndex& index() const { return ix_; }

    // The validation and append half of insert_batch: the batch is checked
    // whole, then its nodes are stored (levels sampled) without links.
    // *first is the first new id. Used by linkers outside this class.
    Err append_batch(const uint64_t* keys, const float* v, size_t n, uint32_t* first);
    // Drops the nodes from `first` on (undoes append_batch).
    void truncate(uint32_t first);
    // link_parallel (src/hnsw/mod.rs:340-349) on `threads` host threads.
    void link_range(uint32_t first, int threads);
    // The graph a linker writes (lists and entry point).
    HostIndex& graph() { return ix_; }
    // compact (src/hnsw/mod.rs:381-400) up to the linking step: a new
    // builder holding the live nodes (keys, vectors, levels re-sampled by
    // their new ids), unlinked; null when there are no tombstones.
    std::unique_ptr<Builder> compacted_unlinked() const;
    // compact with link_parallel on `threads` host threads; the index is
    // unchanged when there are no tombstones.
    void compact(int threads);

private:
    struct Impl;
    HostIndex ix_;
    std::unique_ptr<Impl> impl_;
    Err prepare(const float* v, std::vector<float>* out) const;
    uint32_t push_nodes(const uint64_t* keys, size_t n);
    void link(uint32_t id, int thread);
};

// Dataset generators (src/synthetic.rs:23-124).
void synthetic_gaussian(size_t nb, size_t nq, size_t dim, uint64_t seed, float* base, float* queries);
void synthetic_mixture(size_t nb, size_t nq, size_t dim, size_t clusters, double sigma, uint64_t seed,
                       float* base, float* queries);
void synthetic_mixture_split(size_t nb, size_t nq, size_t dim, size_t clusters, double sigma, uint64_t base_seed,
                             uint64_t query_seed, float* base, float* queries);

}  // namespace hnswgpu
