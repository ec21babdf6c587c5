// Device-side ingest of a format-v1 index file (src/hnsw/io.rs:236-540):
// the file is copied to the device once, and the checks that touch every
// byte or every node run there in parallel, writing the device layout
// directly: the CRC-32 of the body, the vector checks (finite, bounded norm,
// unit length under cosine), the neighbor-list checks (ids in range, not the
// node itself, on a node of that level, no duplicates) together with the
// CSR write, the tombstone bitmap and the duplicate-live-key check. The host
// keeps the sequential checks (header, columns, list counts) and reports the
// first failing check in the reference's order: each kernel records the
// earliest failing position, which is what a sequential reader would hit.
#include <algorithm>

#include "common.cuh"
#include "device.hpp"

namespace hnswgpu {
namespace dev {

// Reflected CRC-32 (IEEE 802.3) generator, x^32 implicit.
constexpr uint32_t kCrcPoly = 0xEDB88320u;

// Product of two polynomials mod the generator, in the reflected
// representation (bit 31 is the coefficient of x^0, bit 0 that of x^31).
// Accumulates b * x^j for every coefficient a_j of a; multiplying by x is a
// right shift with a reduction when the x^31 coefficient moves to x^32.
__host__ __device__ __forceinline__ uint32_t crc_mulmod(uint32_t a, uint32_t b) {
    uint32_t p = 0;
    for (int j = 0; j < 32; ++j) {
        if ((a >> (31 - j)) & 1u) p ^= b;
        b = (b >> 1) ^ ((b & 1u) ? kCrcPoly : 0u);
    }
    return p;
}

// Raw CRC (zero initial register, no final xor) of each chunk of the body,
// one thread per chunk, byte at a time through a 256-entry table.
__global__ void crc_chunks_kernel(const uint8_t* __restrict__ data, size_t len, size_t chunk,
                                  uint32_t* __restrict__ part, size_t nchunks) {
    __shared__ uint32_t table[256];
    for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
        uint32_t r = i;
        for (int k = 0; k < 8; ++k) r = (r >> 1) ^ ((r & 1u) ? kCrcPoly : 0u);
        table[i] = r;
    }
    __syncthreads();
    const size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const size_t begin = c * chunk, end = min(len, begin + chunk);
    uint32_t r = 0;
    size_t i = begin;
    // chunk is a multiple of 16 and the buffer 256-byte aligned: 16-byte loads.
    for (; i + 16 <= end; i += 16) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(data + i));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int b = 0; b < 4; ++b) r = table[(r ^ (w[q] >> (8 * b))) & 0xFFu] ^ (r >> 8);
    }
    for (; i < end; ++i) r = table[(r ^ data[i]) & 0xFFu] ^ (r >> 8);
    part[c] = r;
}

// x^(8 * bytes) mod the generator, from pow8[j] = x^(8 * 2^j).
__device__ __forceinline__ uint32_t crc_shift_factor(uint64_t bytes, const uint32_t* pow8) {
    uint32_t f = 0x80000000u;  // x^0
    for (int j = 0; bytes; ++j, bytes >>= 1)
        if (bytes & 1u) f = crc_mulmod(f, pow8[j]);
    return f;
}

// Combines the chunk CRCs: raw(A || B) = raw(A) * x^(8|B|) + raw(B), so the
// body's raw CRC is the xor over chunks of raw(chunk) * x^(8 * bytes after it).
__global__ void crc_combine_kernel(const uint32_t* __restrict__ part, size_t nchunks, size_t chunk, size_t len,
                                   const uint32_t* __restrict__ pow8, uint32_t* out) {
    const size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    uint32_t v = 0;
    if (c < nchunks) {
        const size_t end = min(len, (c + 1) * chunk);
        v = crc_mulmod(part[c], crc_shift_factor(len - end, pow8));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v ^= __shfl_xor_sync(kFull, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicXor(out, v);
}

// vector::check (src/vector.rs:90-104) of every row, and the unit-length
// check under cosine (io.rs:460-470): the f64 sum in the row's order, one
// thread per node. Records min(node * 2 + kind), kind 0 = "vector out of
// range", 1 = "cosine vector is not unit length".
__global__ void check_vectors_kernel(const float* __restrict__ vec, uint32_t n, uint32_t dim, uint32_t dp,
                                     int cosine, unsigned long long* first) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* v = vec + size_t(i) * dp;
    double s = 0.0;
    bool bad = false;
    for (uint32_t j = 0; j < dim; ++j) {
        const float x = v[j];
        if (!isfinite(x)) {
            bad = true;
            break;
        }
        s = __dadd_rn(s, __dmul_rn(double(x), double(x)));
    }
    if (!bad && s > double(3.40282346638528859812e+38F) / 8.0) bad = true;
    if (bad) atomicMin(first, (unsigned long long)i * 2ull);
    else if (cosine && fabs(s - 1.0) > 1e-3) atomicMin(first, (unsigned long long)i * 2ull + 1ull);
}

// read_links (io.rs:487-514) for every node, one warp per node: each list
// (count word, then ids) must hold ids below n, not the node itself, on
// nodes whose level reaches the list's layer, without duplicates. Valid
// lists are written into the device CSR (layer 0 rows, upper-layer blocks).
// Records min(list byte offset * 2 + kind), kind 0 = "neighbor id", 1 =
// "duplicate neighbor id" (a list with a bad id reports that first, as the
// sequential reader does).
__global__ void links_kernel(const uint32_t* __restrict__ words, const uint64_t* __restrict__ node_off,
                             uint64_t links_begin, const uint8_t* __restrict__ levels, uint32_t n, uint32_t m0p,
                             uint32_t mp, const uint32_t* __restrict__ up_off, uint32_t* __restrict__ adj0,
                             uint32_t* __restrict__ adjU, unsigned long long* first) {
    const uint32_t node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (node >= n) return;
    uint64_t pos = (node_off[node] - links_begin) >> 2;  // word index of the node's first list
    const unsigned top = levels[node];
    for (unsigned layer = 0; layer <= top; ++layer) {
        const uint64_t list_byte = links_begin + (pos << 2);
        const uint32_t count = words[pos];
        const uint32_t* ids = words + pos + 1;
        bool bad = false;
        for (uint32_t j = lane; j < count; j += 32) {
            const uint32_t nb = ids[j];
            bad |= !(nb < n && nb != node && levels[nb] >= layer);
        }
        bad = __any_sync(kFull, bad);
        bool dup = false;
        if (!bad) {
            for (uint32_t a = 0; a < count; a += 32) {
                const uint32_t ia = a + lane;
                const uint32_t va = ia < count ? ids[ia] : kEmpty;
                // duplicates within this 32-id chunk
                const unsigned same = __match_any_sync(kFull, va);  // ids are below kEmpty
                dup |= ia < count && __popc(same) > 1;
                // against every later chunk
                for (uint32_t b = a + 32; b < count; b += 32) {
                    const uint32_t ib = b + lane;
                    const uint32_t vb = ib < count ? ids[ib] : kEmpty;
                    for (int s = 0; s < 32; ++s) {
                        const uint32_t x = __shfl_sync(kFull, va, s);
                        dup |= ib < count && a + uint32_t(s) < count && x == vb;
                    }
                }
            }
            dup = __any_sync(kFull, dup);
        }
        if (bad || dup) {
            if (lane == 0) atomicMin(first, (unsigned long long)list_byte * 2ull + (bad ? 0ull : 1ull));
            return;
        }
        uint32_t* row = layer == 0 ? adj0 + size_t(node) * m0p : adjU + size_t(up_off[node] + layer - 1) * mp;
        for (uint32_t j = lane; j < count; j += 32) row[j] = ids[j];
        pos += 1 + count;
    }
}

// Tombstone bitmap from the byte column.
__global__ void dead_bitmap_kernel(const uint8_t* __restrict__ flags, uint32_t n, uint32_t* __restrict__ dead,
                                   unsigned long long* dead_count) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (size_t(w) * 32 >= n) return;
    uint32_t bits = 0;
    for (uint32_t b = 0; b < 32; ++b) {
        const uint32_t i = w * 32 + b;
        if (i < n && flags[i]) bits |= 1u << b;
    }
    dead[w] = bits;
    if (bits) atomicAdd(dead_count, (unsigned long long)__popc(bits));
}

// finish (io.rs:517-540): live keys must be distinct. Open-addressing set of
// `cap` (a power of two) slots, ~0 marking an empty slot; the key ~0 itself
// is counted apart. Sets *dup when a live key repeats; *not_ids when some
// key differs from its node id.
__global__ void live_keys_kernel(const uint64_t* __restrict__ keys, const uint8_t* __restrict__ flags, uint32_t n,
                                 unsigned long long* __restrict__ table, uint64_t cap, unsigned int* special,
                                 unsigned int* dup, unsigned int* not_ids) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = keys[i];
    if (key != uint64_t(i)) *not_ids = 1u;
    if (flags[i]) return;
    if (key == ~0ull) {
        if (atomicAdd(special, 1u) >= 1u) *dup = 1u;
        return;
    }
    uint64_t h = (key * 0x9E3779B97F4A7C15ull) & (cap - 1);
    for (uint64_t probe = 0; probe < cap; ++probe) {
        const unsigned long long old = atomicCAS(table + h, ~0ull, (unsigned long long)key);
        if (old == ~0ull) return;
        if (old == key) {
            *dup = 1u;
            return;
        }
        h = (h + 1) & (cap - 1);
    }
}

}  // namespace dev

cudaError_t ingest_crc(const uint8_t* data, size_t len, uint32_t* part, uint32_t* pow8, uint32_t* out,
                       uint32_t* crc, cudaStream_t stream) {
    // pow8[j] = x^(8 * 2^j) mod the generator, j = 0..63.
    uint32_t h[64];
    h[0] = 0x80000000u >> 8;  // x^8
    for (int j = 1; j < 64; ++j) h[j] = dev::crc_mulmod(h[j - 1], h[j - 1]);
    cudaError_t e = cudaMemcpyAsync(pow8, h, sizeof h, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(out, 0, 4, stream);
    if (e != cudaSuccess) return e;
    const size_t nchunks = (len + kIngestCrcChunk - 1) / kIngestCrcChunk;
    if (nchunks) {
        const uint32_t threads = 256;
        dev::crc_chunks_kernel<<<uint32_t((nchunks + threads - 1) / threads), threads, 0, stream>>>(
            data, len, kIngestCrcChunk, part, nchunks);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        dev::crc_combine_kernel<<<uint32_t((nchunks + threads - 1) / threads), threads, 0, stream>>>(
            part, nchunks, kIngestCrcChunk, len, pow8, out);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    uint32_t raw = 0;
    e = cudaMemcpyAsync(&raw, out, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    // The initial register 0xFFFFFFFF shifted through the body, then the final xor.
    uint32_t f = 0x80000000u;
    for (int j = 0; j < 64; ++j)
        if ((uint64_t(len) >> j) & 1u) f = dev::crc_mulmod(f, h[j]);
    *crc = raw ^ dev::crc_mulmod(0xFFFFFFFFu, f) ^ 0xFFFFFFFFu;
    return cudaSuccess;
}

cudaError_t ingest_check_vectors(const float* vec, uint32_t n, uint32_t dim, uint32_t dp, bool cosine,
                                 unsigned long long* first, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    dev::check_vectors_kernel<<<(n + 127) / 128, 128, 0, stream>>>(vec, n, dim, dp, cosine ? 1 : 0, first);
    return cudaGetLastError();
}

cudaError_t ingest_links(const uint32_t* words, const uint64_t* node_off, uint64_t links_begin, const uint8_t* levels,
                         uint32_t n, uint32_t m0p, uint32_t mp, const uint32_t* up_off, uint32_t* adj0,
                         uint32_t* adjU, unsigned long long* first, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint64_t blocks = (uint64_t(n) * 32 + 255) / 256;
    dev::links_kernel<<<uint32_t(blocks), 256, 0, stream>>>(words, node_off, links_begin, levels, n, m0p, mp, up_off,
                                                          adj0, adjU, first);
    return cudaGetLastError();
}

cudaError_t ingest_dead(const uint8_t* flags, uint32_t n, uint32_t* dead, unsigned long long* dead_count,
                        cudaStream_t stream) {
    const uint32_t words = (n + 31) / 32;
    if (words == 0) return cudaSuccess;
    dev::dead_bitmap_kernel<<<(words + 255) / 256, 256, 0, stream>>>(flags, n, dead, dead_count);
    return cudaGetLastError();
}

cudaError_t ingest_live_keys(const uint64_t* keys, const uint8_t* flags, uint32_t n, unsigned long long* table,
                             uint64_t cap, unsigned int* flags_out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    dev::live_keys_kernel<<<(n + 255) / 256, 256, 0, stream>>>(keys, flags, n, table, cap, flags_out, flags_out + 1,
                                                            flags_out + 2);
    return cudaGetLastError();
}

}  // namespace hnswgpu
