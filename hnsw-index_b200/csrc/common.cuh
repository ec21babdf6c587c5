// Device helpers shared by the search and brute-force kernels.
//
// Every floating-point operation that feeds a distance is an explicit
// round-to-nearest intrinsic (__fmaf_rn, __fadd_rn, __fsub_rn, __fmul_rn), so
// nvcc cannot contract or reassociate it: the kernels reproduce the reference
// AVX2 backend's summation order bit for bit (src/kernels/x86.rs:19-131).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <set>
#include <utility>

namespace hnswgpu {

// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum, once per (kernel, device). The limit is process-wide state, so
// setting it to each launch's size would race with host threads launching the
// same kernel with other sizes (a launch above the current limit fails).
inline cudaError_t raise_smem_limit(const void* func) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    std::lock_guard<std::mutex> lock(mu);
    if (done.count({func, dev})) return cudaSuccess;
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, func);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - int(fa.sharedSizeBytes));
    if (e == cudaSuccess) done.insert({func, dev});
    return e;
}
namespace dev {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

// Monotone u32 image of Rust's f32::total_cmp order: the signed-integer
// transform b ^ ((u32)(b >> 31) >> 1), with the sign bit flipped so that
// unsigned comparison matches.
__device__ __forceinline__ uint32_t fkey(float d) {
    int32_t s = __float_as_int(d);
    s ^= int32_t(uint32_t(s >> 31) >> 1);
    return uint32_t(s) ^ 0x80000000u;
}
__device__ __forceinline__ float kdec(uint32_t k) {
    int32_t s = int32_t(k ^ 0x80000000u);
    s ^= int32_t(uint32_t(s >> 31) >> 1);
    return __int_as_float(s);
}
// Candidate (distance, id) packed so that u64 order == (total_cmp, id) order
// (src/hnsw/search.rs:36-44).
__device__ __forceinline__ uint64_t pack(float d, uint32_t id) { return (uint64_t(fkey(d)) << 32) | id; }
__device__ __forceinline__ float pdist(uint64_t p) { return kdec(uint32_t(p >> 32)); }
__device__ __forceinline__ uint32_t pid(uint64_t p) { return uint32_t(p); }

__device__ __forceinline__ float4 ldg_f4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// Row loads: read-only global path, or shared memory (rows staged by cp.async).
template <bool SMEM>
__device__ __forceinline__ float4 row_f4(const float* p) {
    if (SMEM) return *reinterpret_cast<const float4*>(p);
    return ldg_f4(p);
}
template <bool SMEM>
__device__ __forceinline__ float row_f1(const float* p) {
    if (SMEM) return *p;
    return __ldg(p);
}
template <bool SMEM>
__device__ __forceinline__ int4 row_i4(const int8_t* p) {
    if (SMEM) return *reinterpret_cast<const int4*>(p);
    return __ldg(reinterpret_cast<const int4*>(p));
}

// Asynchronous 16-byte (and 4-byte) copies global -> shared, completed by
// cp_async_wait_all (a hardware wait, no spin).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Asks the memory system to bring `bytes` (multiple of 16, 16-byte aligned
// source) into L2 without occupying registers or shared memory.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// One 32-float step of four AVX2 lanes held by this GPU lane.
template <bool L2>
__device__ __forceinline__ void acc4(const float4 x, const float4 y, float (&a)[4]) {
    if (L2) {
        float d0 = __fsub_rn(y.x, x.x), d1 = __fsub_rn(y.y, x.y), d2 = __fsub_rn(y.z, x.z), d3 = __fsub_rn(y.w, x.w);
        a[0] = __fmaf_rn(d0, d0, a[0]);
        a[1] = __fmaf_rn(d1, d1, a[1]);
        a[2] = __fmaf_rn(d2, d2, a[2]);
        a[3] = __fmaf_rn(d3, d3, a[3]);
    } else {
        a[0] = __fmaf_rn(y.x, x.x, a[0]);
        a[1] = __fmaf_rn(y.y, x.y, a[1]);
        a[2] = __fmaf_rn(y.z, x.z, a[2]);
        a[3] = __fmaf_rn(y.w, x.w, a[3]);
    }
}

// Reduces the 32 AVX2 partial sums held by an aligned group of eight lanes
// (lane g8 holds chain g8/2, AVX lanes 4*(g8&1)+e) in the reference order:
// lane-wise (c0+c1)+(c2+c3), then ((v0+v4)+(v1+v5))+((v2+v6)+(v3+v7)).
// The result is valid in the group's lane g8 == 0. All 32 lanes must call.
__device__ __forceinline__ float reduce_avx2_order(const float (&a)[4]) {
    float t[4], v[4], p[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) t[e] = __fadd_rn(a[e], __shfl_down_sync(kFull, a[e], 2, 8));
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = __fadd_rn(t[e], __shfl_down_sync(kFull, t[e], 4, 8));
#pragma unroll
    for (int e = 0; e < 4; ++e) p[e] = __fadd_rn(v[e], __shfl_down_sync(kFull, v[e], 1, 8));
    return __fadd_rn(__fadd_rn(p[0], p[1]), __fadd_rn(p[2], p[3]));
}

// Raw sum (dot product, or squared L2) of `row` against `q` (both 16-byte
// aligned, padded to a multiple of 32 floats) for this lane's group of
// eight. Valid in lane g8 == 0 of the group. All 32 lanes must call with the
// same `dim`.
template <bool L2, bool SMEM = false>
__device__ __forceinline__ float group_sum(const float* __restrict__ row, const float* __restrict__ q, int dim,
                                           int g8) {
    float a[4] = {0.f, 0.f, 0.f, 0.f};
    const int nfull = dim >> 5;
    const float* r = row + 4 * g8;
    const float* qq = q + 4 * g8;
#pragma unroll 4
    for (int k = 0; k < nfull; ++k)
        acc4<L2>(row_f4<SMEM>(r + 32 * k), *reinterpret_cast<const float4*>(qq + 32 * k), a);
    // 8-wide remainder blocks go into chain 0 (lanes g8 = 0, 1).
    const int rem8 = (dim & 31) >> 3;
    if (g8 < 2)
        for (int s = 0; s < rem8; ++s)
            acc4<L2>(row_f4<SMEM>(r + 32 * nfull + 8 * s), *reinterpret_cast<const float4*>(qq + 32 * nfull + 8 * s),
                     a);
    float sum = reduce_avx2_order(a);
    if (g8 == 0)
        for (int i = (nfull << 5) + (rem8 << 3); i < dim; ++i) {
            if (L2) {
                float d = __fsub_rn(q[i], row_f1<SMEM>(row + i));
                sum = __fadd_rn(sum, __fmul_rn(d, d));
            } else {
                sum = __fadd_rn(sum, __fmul_rn(q[i], row_f1<SMEM>(row + i)));
            }
        }
    return sum;
}

// group_sum of two rows at once (the loads of both rows issued together, so
// one memory round trip serves eight rows per warp). Results valid in lane
// g8 == 0 of the group, each bit-identical to group_sum on its row.
template <bool L2>
__device__ __forceinline__ void group_sum2(const float* __restrict__ row0, const float* __restrict__ row1,
                                           const float* __restrict__ q, int dim, int g8, float& s0, float& s1) {
    float a[4] = {0.f, 0.f, 0.f, 0.f}, b[4] = {0.f, 0.f, 0.f, 0.f};
    const int nfull = dim >> 5;
    const float* r0 = row0 + 4 * g8;
    const float* r1 = row1 + 4 * g8;
    const float* qq = q + 4 * g8;
#pragma unroll 4
    for (int k = 0; k < nfull; ++k) {
        const float4 x0 = ldg_f4(r0 + 32 * k), x1 = ldg_f4(r1 + 32 * k);
        const float4 y = *reinterpret_cast<const float4*>(qq + 32 * k);
        acc4<L2>(x0, y, a);
        acc4<L2>(x1, y, b);
    }
    const int rem8 = (dim & 31) >> 3;
    if (g8 < 2)
        for (int s = 0; s < rem8; ++s) {
            const float4 y = *reinterpret_cast<const float4*>(qq + 32 * nfull + 8 * s);
            acc4<L2>(ldg_f4(r0 + 32 * nfull + 8 * s), y, a);
            acc4<L2>(ldg_f4(r1 + 32 * nfull + 8 * s), y, b);
        }
    s0 = reduce_avx2_order(a);
    s1 = reduce_avx2_order(b);
    if (g8 == 0)
        for (int i = (nfull << 5) + (rem8 << 3); i < dim; ++i) {
            if (L2) {
                const float d0 = __fsub_rn(q[i], __ldg(row0 + i)), d1 = __fsub_rn(q[i], __ldg(row1 + i));
                s0 = __fadd_rn(s0, __fmul_rn(d0, d0));
                s1 = __fadd_rn(s1, __fmul_rn(d1, d1));
            } else {
                s0 = __fadd_rn(s0, __fmul_rn(q[i], __ldg(row0 + i)));
                s1 = __fadd_rn(s1, __fmul_rn(q[i], __ldg(row1 + i)));
            }
        }
}

// Metric::distance (src/metric.rs:35-41) from a raw sum.
__device__ __forceinline__ float metric_from_sum(int metric, float s) {
    return metric == 0 ? s : (metric == 1 ? -s : __fsub_rn(1.0f, s));
}

// Integer dot product of an int8 code row with the query code for the
// group of eight lanes (dc bytes, multiple of 16). Exact; valid in all lanes
// of the group.
template <bool SMEM = false>
__device__ __forceinline__ int group_i8dot(const int8_t* __restrict__ row, const int8_t* __restrict__ qc, int dc,
                                           int g8) {
    int acc = 0;
    const int n16 = dc >> 4;
    for (int p = g8; p < n16; p += 8) {
        int4 x = row_i4<SMEM>(row + 16 * p);
        int4 y = *(reinterpret_cast<const int4*>(qc) + p);
        acc = __dp4a(x.x, y.x, acc);
        acc = __dp4a(x.y, y.y, acc);
        acc = __dp4a(x.z, y.z, acc);
        acc = __dp4a(x.w, y.w, acc);
    }
    acc += __shfl_xor_sync(kFull, acc, 1, 8);
    acc += __shfl_xor_sync(kFull, acc, 2, 8);
    acc += __shfl_xor_sync(kFull, acc, 4, 8);
    return acc;
}

// ScalarQuantizer::distance (src/quantization.rs:85-92): exact integer sum
// converted to f32 (round to nearest), times scale^2, without contraction.
__device__ __forceinline__ float sq_distance(int metric, long long dot, long long l2, float s2) {
    if (metric == 0) return __fmul_rn(__ll2float_rn(l2), s2);
    if (metric == 1) return __fmul_rn(-__ll2float_rn(dot), s2);
    return __fsub_rn(1.0f, __fmul_rn(__ll2float_rn(dot), s2));
}

// ScalarQuantizer::encode_into (src/quantization.rs:73-81) of one component.
__device__ __forceinline__ int8_t sq_encode1(float x, float o, float inv) {
    float v = roundf(__fmul_rn(__fsub_rn(x, o), inv));
    v = fminf(127.0f, fmaxf(-127.0f, v));
    return int8_t(v);
}

}  // namespace dev
}  // namespace hnswgpu
