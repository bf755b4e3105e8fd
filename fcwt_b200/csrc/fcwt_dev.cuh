// Device helpers shared by the CUDA-core row engine (fcwt_kernels.cu) and the
// tensor-core row engine (fcwt_tc.cu): daughter weights of the reference's
// product (src/fcwt/fcwt.cpp:197-311), output stores, bulk-async (TMA) store
// helpers and the swizzled staging layout of the output tensor map.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fcwt_fft.cuh"
#include "fcwt_internal.h"

namespace fcwt {
namespace dev {

// Output staging for tensor-map stores: 4 boxes of [256 a][8 columns] complex64.
constexpr int kBoxRows = 256;
constexpr int kBoxBytes = kBoxRows * kGroupCols * 8;

// Bounded waits give up after this much wall time and record kErrWaitTimeout.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Daughter weight of bin q (reference: mother[(int)min(N-1, step*q)] for the
// row that last wrote bin q into O1; 0 if no row did).
__device__ __forceinline__ float bin_weight(const RowDesc& R, const float* __restrict__ mother,
                                           const float* __restrict__ pool, float nm1, int q) {
    if (R.mode == 1) {
        const float u = R.ca * (float)q - R.cb;
        return R.cnorm * expf(-0.5f * u * u);
    }
    float s;
    if (q < R.proc)
        s = R.step;
    else if (R.stale >= 0)
        s = __ldg(pool + R.stale + q);
    else
        return 0.0f;
    if (!(s > 0.0f)) return 0.0f;
    int w = (int)fminf(nm1, __fmul_rn(s, (float)q));
    return __ldg(mother + w);
}

// Z[q] = Ihat[q] * W[q] * out_scale. out_scale is 1 or 1/N, a power of two,
// so scaling the weight is exact and equals scaling the output.
__device__ __forceinline__ float2 bin_value(const RowDesc& R, const SigDesc& S, const float* __restrict__ pool,
                                           float nm1, int q) {
    if (q < R.lo || q >= R.hi) return make_float2(0.0f, 0.0f);
    const float m = bin_weight(R, S.mother, pool, nm1, q) * R.out_scale;
    const float2 xv = __ldg(S.X + q);
    // imag_frequency: i * m * Ihat (the reference's AVX product, src/fcwt/fcwt.cpp:255-262)
    return R.imag ? make_float2(-xv.y * m, xv.x * m) : make_float2(xv.x * m, xv.y * m);
}

template <int OT>
__device__ __forceinline__ void store_out(void* base, long long idx, float2 v) {
    if constexpr (OT == OUT_C64) {
        __stcs(reinterpret_cast<float2*>(base) + idx, v);
    } else if constexpr (OT == OUT_BF16) {
        __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        __stcs(reinterpret_cast<unsigned*>(base) + idx, *reinterpret_cast<unsigned*>(&h));
    } else if constexpr (OT == OUT_F16) {
        __half2 h = __floats2half2_rn(v.x, v.y);
        __stcs(reinterpret_cast<unsigned*>(base) + idx, *reinterpret_cast<unsigned*>(&h));
    } else {
        const float p = v.x * v.x + v.y * v.y;
        __stcs(reinterpret_cast<float*>(base) + idx, OT == OUT_POWER ? p : 10.0f * log10f(p));
    }
}

// ---- bulk-async (TMA) store helpers
// Orders a tensor map that a host copy wrote into global memory before this
// thread's TMA operations that use it (tensor-map proxy acquire, system scope).
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;"
                 ::"l"(reinterpret_cast<unsigned long long>(map)) : "memory");
}
// EVICT_FIRST marks the written lines evict-first in L2 (the output is a
// stream that is not read again by the kernel).
template <bool EVICT_FIRST = false>
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* smem, int c0, int c1, int c2) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (EVICT_FIRST) {
        unsigned long long pol;
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
        asm volatile(
            "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%2, %3, %4}], [%1], %5;"
            ::"l"(reinterpret_cast<unsigned long long>(map)), "r"(s), "r"(c0), "r"(c1), "r"(c2), "l"(pol)
            : "memory");
    } else {
        asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
                     ::"l"(reinterpret_cast<unsigned long long>(map)), "r"(s), "r"(c0), "r"(c1), "r"(c2)
                     : "memory");
    }
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Byte offset of staging element (a, w) in the 64B-swizzled box layout the
// tensor map expects: 16-byte chunk bits [4:5] XOR address bits [7:8].
__device__ __forceinline__ unsigned stage_off(int a, int w) {
    const unsigned lin = (unsigned)((a & (kBoxRows - 1)) * (kGroupCols * 8) + w * 8);
    return (unsigned)(a >> 8) * kBoxBytes + (lin ^ (((lin >> 7) & 3u) << 4));
}
// The same for 4-byte outputs (BF16 / FP16 complex pairs): boxes of
// [256 a][8 columns] x 4 bytes in the 32B-swizzled layout (16-byte chunk bit 4
// XOR address bit 7).
__device__ __forceinline__ unsigned stage16_off(int a, int w) {
    const unsigned lin = (unsigned)((a & (kBoxRows - 1)) * (kGroupCols * 4) + w * 4);
    return (unsigned)(a >> 8) * (kBoxBytes / 2) + (lin ^ (((lin >> 7) & 1u) << 4));
}

// Complex value as the 4-byte element of a 4-byte output type (16-bit pair,
// power or dB).
template <int OT>
__device__ __forceinline__ unsigned pack16(float2 v) {
    if constexpr (OT == OUT_BF16) {
        __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        return *reinterpret_cast<unsigned*>(&h);
    } else if constexpr (OT == OUT_F16) {
        __half2 h = __floats2half2_rn(v.x, v.y);
        return *reinterpret_cast<unsigned*>(&h);
    } else {
        const float p = v.x * v.x + v.y * v.y;
        return __float_as_uint(OT == OUT_POWER ? p : 10.0f * log10f(p));
    }
}

// w_N^e with e < N from the low table (SMEM) and the high table (SMEM when
// M <= 1024, else global).
__device__ __forceinline__ float2 tw_n(const float2* __restrict__ twlo, const float2* __restrict__ twhi,
                                      unsigned e) {
    return cmul(twlo[e & 1023u], twhi[e >> 10]);
}

}  // namespace dev
}  // namespace fcwt
