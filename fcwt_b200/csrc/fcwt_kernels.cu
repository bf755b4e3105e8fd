// sm_100a kernels of the fCWT transform path.
//
//   k_mother      Morlet frequency-domain mother table (Morlet::generate(int),
//                 src/fcwt/fcwt.cpp:51-67): float operations in the
//                 reference's order, exp evaluated in float64 then rounded.
//   k_twiddle     two-level twiddle table w_N^j (float64 sincospi, rounded).
//   (the forward FFT of the signal is in fcwt_fwd.cu)
//   k_row_engine  persistent row engine: daughter multiply (fcwt.cpp:197-311),
//                 inverse FFT (fcwt.cpp:418-429), normalisation
//                 (fcwt.cpp:431-445) and crop to n (fcwt.cpp:396-416), fused,
//                 driven by a work queue of per-row items.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "fcwt_dev.cuh"
#include "fcwt_fft.cuh"
#include "fcwt_internal.h"

namespace fcwt {
namespace dev {

// ------------------------------------------------------------------ tables

__global__ void k_mother(float fb, int N, float norm, float* __restrict__ out) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= N) return;
    const float two_pi = 2.0f * 3.14159265358979323846f;  // 2*PI in float, as the reference
    float toradians = __fdiv_rn(two_pi, (float)N);
    float t = __fmul_rn(__fmul_rn(2.0f, __fmul_rn((float)w, toradians)), fb);
    t = __fsub_rn(t, __fmul_rn(two_pi, fb));
    t = __fdiv_rn(-__fmul_rn(t, t), 2.0f);
    float e = (float)exp((double)t);
    out[w] = __fmul_rn(norm, e);
}

// tw[j] = w_N^j for j < 1024; tw[1024 + j] = w_N^{1024 j} for j < max(M, 1).
// w_N = exp(+2 pi i / N).
__global__ void k_twiddle(int log2N, float2* __restrict__ tw) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = 1 << log2N;
    const int M = N >= 1024 ? N / 1024 : 1;
    if (j >= 1024 + M) return;
    long long e = j < 1024 ? j : (long long)(j - 1024) * 1024;
    e &= (long long)N - 1;
    double s, c;
    sincospi(2.0 * (double)e / (double)N, &s, &c);
    tw[j] = make_float2((float)c, (float)s);
}

// --------------------------------------------------------------- row engine

// Shared-memory layout of the row engine, per CTA (units of float2):
//   region0: G of a fused row (<= 8192) / per-warp transposes (8 x 32x33) /
//            output staging [1024][9] of 8 columns
//   zs:      phase-1 input tile [K][kChunk]
//   twlo:    w_N^j, j < 1024, of the current N
//   t2:      w_1024^{a l} at [a*32 + l]
//   twhi:    w_N^{1024 j} = w_M^j, j < M, of the current N (M <= 512), or
//            w_M^j for j < 32 followed by w_M^{32 j} for j < M / 32 (M > 512)
constexpr int kStagePitch = kGroupCols + 1;
constexpr int kRegion0 = kP2 * kStagePitch;
constexpr int kZs = kChunk * kMaxK;
constexpr int kTwhiSmem = 512;
static_assert(32 + (1 << (kMaxLog2N - kLog2P2)) / 32 <= kTwhiSmem, "split w_M tables of the largest N fit");
constexpr int kSmemFloat2 = kRegion0 + kZs + kP2 + kP2 + kTwhiSmem;
constexpr size_t kSmemAlign = 1024;  // the 64B-swizzled staging tile wants 1 KB alignment
constexpr size_t kEngineSmemBytes = (size_t)kSmemFloat2 * sizeof(float2) + kSmemAlign;
static_assert(4 * kBoxBytes <= kRegion0 * 8, "staging boxes fit in region0");
constexpr int kFetchBatch = 2;  // work items claimed per queue access
static_assert(kRegion0 >= kMaxFusedN, "fused rows keep G in region0");
static_assert(kRegion0 >= (kThreads / 32) * 32 * 33, "per-warp transposes live in region0");

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait until *p >= target: gives up after kWaitLimitNs of wall time
// (or when another CTA already reported an error) and returns false; the
// timeout is recorded in *err.

__device__ bool wait_counter(const unsigned* p, unsigned target, int* err) {
    if (ld_acquire(p) >= target) return true;
    const unsigned long long t0 = global_ns();
    unsigned it = 0;
    while (ld_acquire(p) < target) {
        if (*((volatile int*)err) != 0) return false;
        if ((++it & 63u) == 0 && global_ns() - t0 > kWaitLimitNs) {
            atomicOr(err, kErrWaitTimeout);
            return false;
        }
        __nanosleep(256);
    }
    return true;
}

// w_M^x (x < M) of the current N from shared memory: the table itself when
// M <= kTwhiSmem, otherwise the product of a[x mod 32] = w_M^{x mod 32} and
// b[x / 32] = w_M^{32 (x / 32)} (32 + M / 32 <= 288 entries for M <= 8192).
struct TwM {
    const float2* a;
    const float2* b;  // null: a is the whole table
    __device__ __forceinline__ float2 operator[](unsigned x) const {
        return b ? cmul(a[x & 31u], b[x >> 5]) : a[x];
    }
};
// w_N^e with e < N from the low table w_N^j (j < 1024) and w_M.
__device__ __forceinline__ float2 tw_n(const float2* __restrict__ twlo, const TwM& twhi, unsigned e) {
    return cmul(twlo[e & 1023u], twhi[e >> 10]);
}

// Phase 1 of one chunk of kChunk k2 values of a row (see fcwt_internal.h):
// loads Z into the tile zs[k1][k2], then every (k2, v) task runs a K-point
// DFT and writes G[c][k2] (c = v + R u) times w_N^{(k2+L) c}.
template <int K, bool TO_GLOBAL>
__device__ __forceinline__ void phase1_chunk(const SigDesc& S, const RowDesc& R, const float* __restrict__ pool, int k2_0,
                             float2* __restrict__ zs, const float2* __restrict__ twlo,
                             const TwM twhi, float2* __restrict__ gdst) {
    const int tid = threadIdx.x;
    const int log2N = S.log2N;
    const int N = 1 << log2N;
    const unsigned Nm = (unsigned)N - 1u;
    const int M = N >> kLog2P2;
    const int Rr = M / K;
    const float nm1 = (float)N - 1.0f;
    // (a) input tile
    for (int idx = tid; idx < K * kChunk; idx += kThreads) {
        const int k1 = idx / kChunk;
        const int kl = idx - k1 * kChunk;
        zs[idx] = bin_value(R, S, pool, nm1, R.L + k2_0 + kl + kP2 * k1);
    }
    __syncthreads();
    // (b) tasks
    for (int t = tid; t < kChunk * Rr; t += kThreads) {
        const int kl = t % kChunk;
        const int v = t / kChunk;
        float2 z[K];
#pragma unroll
        for (int k1 = 0; k1 < K; k1++) z[k1] = zs[k1 * kChunk + kl];
        if (v != 0) {
            // pre-twiddle w_M^{v k1}: exact table value every 8 steps, a
            // running product (at most 7 multiplies) in between
            const float2 step = twhi[v];
            float2 w = make_float2(1.0f, 0.0f);
#pragma unroll
            for (int k1 = 1; k1 < K; k1++) {
                w = (k1 & 7) ? cmul(w, step) : twhi[v * k1];
                z[k1] = cmul(z[k1], w);
            }
        }
        fft_reg<K, +1>(z);
        const int k2 = k2_0 + kl;
        const unsigned k2L = (unsigned)(k2 + R.L);
        const unsigned base = (k2L * (unsigned)v) & Nm;   // exponent of u = 0
        const unsigned d = (k2L * (unsigned)Rr) & Nm;     // exponent step per u
        float2* __restrict__ dst = gdst + k2;
        // post-twiddle w_N^{base + d u}: exact every 8 outputs, running
        // product in between
        // (output address and exponent advance by a step, which keeps the
        // 32-output case from holding all addresses in registers)
        const float2 wd = tw_n(twlo, twhi, d);
        float2 w = make_float2(1.0f, 0.0f);
        float2* p = dst + (size_t)v * kP2;
        const size_t pstep = (size_t)Rr * kP2;
        unsigned eu = base;
#pragma unroll
        for (int u = 0; u < K; u++) {
            w = (u & 7) ? cmul(w, wd) : tw_n(twlo, twhi, eu & Nm);
            eu += d;
            const float2 g = cmul(z[u], w);
            if constexpr (TO_GLOBAL)
                __stcg(p, g);
            else
                *p = g;
            p += pstep;
        }
    }
    __syncthreads();
}

template <bool TO_GLOBAL>
__device__ void phase1_chunk_dispatch(int K, const SigDesc& S, const RowDesc& R, const float* pool,
                                      int k2_0, float2* zs, const float2* twlo, const TwM twhi,
                                      float2* gdst) {
    switch (K) {
        case 1: phase1_chunk<1, TO_GLOBAL>(S, R, pool, k2_0, zs, twlo, twhi, gdst); break;
        case 2: phase1_chunk<2, TO_GLOBAL>(S, R, pool, k2_0, zs, twlo, twhi, gdst); break;
        case 4: phase1_chunk<4, TO_GLOBAL>(S, R, pool, k2_0, zs, twlo, twhi, gdst); break;
        case 8: phase1_chunk<8, TO_GLOBAL>(S, R, pool, k2_0, zs, twlo, twhi, gdst); break;
        case 16: phase1_chunk<16, TO_GLOBAL>(S, R, pool, k2_0, zs, twlo, twhi, gdst); break;
        default: phase1_chunk<32, TO_GLOBAL>(S, R, pool, k2_0, zs, twlo, twhi, gdst); break;
    }
}

// Phase 1 of a wide row (K = 32*K2 > 32): warp w handles k2 = k2_0 + w; for
// every v the warp runs the K-point DFT cooperatively (in-lane K2-point DFT
// over j, twiddle w_K^{l p}, SMEM transpose, FFT32 over l on lanes p < K2,
// output u = p + K2 q), the CTA stages the 8 k2 columns of outputs and writes
// G[v + R u][k2_0 .. k2_0+7] in 64-byte runs with the w_N^{(k2+L) c} twiddle.
template <int K2>
__device__ void phase1_wide(const SigDesc& S, const RowDesc& R, const float* __restrict__ pool, int k2_0,
                            const float2* __restrict__ twlo, const TwM twhi,
                            float2* __restrict__ region0, float2* __restrict__ G) {
    constexpr int K = 32 * K2;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int log2N = S.log2N;
    const int N = 1 << log2N;
    const unsigned Nm = (unsigned)N - 1u;
    const int M = N >> kLog2P2;
    const int Rr = M / K;
    const float nm1 = (float)N - 1.0f;
    const int k2 = k2_0 + warp;
    float2* tb = region0 + warp * (32 * 33);
    for (int v = 0; v < Rr; v++) {
        float2 z[K2];
#pragma unroll
        for (int j = 0; j < K2; j++) {
            const int k1 = lane + 32 * j;
            float2 a = bin_value(R, S, pool, nm1, R.L + k2 + kP2 * k1);
            if (v != 0) a = cmul(a, twhi[v * k1]);
            z[j] = a;
        }
        fft_reg<K2, +1>(z);
#pragma unroll
        for (int p = 1; p < K2; p++) z[p] = cmul(z[p], twhi[(lane * p * Rr) & (M - 1)]);
#pragma unroll
        for (int p = 0; p < K2; p++) tb[p * 33 + lane] = z[p];
        __syncwarp();
        float2 y[32];
        if (lane < K2) {
#pragma unroll
            for (int l = 0; l < 32; l++) y[l] = tb[lane * 33 + l];
            fft_reg<32, +1>(y);
        }
        __syncthreads();  // all transposes done before staging overwrites region0
        if (lane < K2) {
#pragma unroll
            for (int q = 0; q < 32; q++) region0[(lane + K2 * q) * kWideChunk + warp] = y[q];
        }
        __syncthreads();
        for (int idx = tid; idx < K * kWideChunk; idx += kThreads) {
            const int u = idx / kWideChunk;
            const int w = idx - u * kWideChunk;
            const int c = v + Rr * u;
            const unsigned e = ((unsigned)(k2_0 + w + R.L) * (unsigned)c) & Nm;
            __stcg(G + (size_t)c * kP2 + k2_0 + w, cmul(region0[idx], tw_n(twlo, twhi, e)));
        }
        __syncthreads();
    }
}

// Phase 1 of a wide row with 64 <= K = 32 K2 <= 512, for k2 in [k2_0, k2_0 + 8).
// The K-point DFT over k1 = j + K2 i is split as
//     DFT_K[u1 + 32 u2] = sum_j w_K2^{j u2} w_K^{j u1} sum_i x[j + K2 i] w_32^{i u1}:
// step B runs one register FFT32 over i per (v, j, k2) task, step C one
// K2-point DFT over j per (v, u1, k2) task; every thread works in both steps.
// The spectrum x weights of the 8 k2 columns are loaded into SMEM once per
// item (zt[k1][8]); the FFT32 outputs of a batch of v values go through SMEM
// (Y[u1][task], padded rows). When the step-B tasks of all v are exactly one
// per thread (M = 1024, any K), all v run as one batch and Y overwrites zt
// once every thread holds its inputs in registers. Outputs:
// G[c = v + R u][k2] w_N^{(k2+L) c}.
template <int K2>
__device__ void phase1_big(const SigDesc& S, const RowDesc& R, const float* __restrict__ pool, int k2_0,
                           const float2* __restrict__ twlo, const TwM twhi,
                           float2* __restrict__ region0, float2* __restrict__ G) {
    constexpr int K = 32 * K2;
    constexpr int W = kWideChunk;
    static_assert(W == 8, "task indexing assumes 8 k2 per item");
    constexpr int kYPad = 4;
    constexpr int VBmax = (kRegion0 - 32 * kYPad - K * W) / (K * W);
    static_assert(VBmax >= 1, "zt and one batch of Y fit in region0");
    const int tid = threadIdx.x;
    const int log2N = S.log2N;
    const int N = 1 << log2N;
    const unsigned Nm = (unsigned)N - 1u;
    const int M = N >> kLog2P2;
    const unsigned Mm = (unsigned)M - 1u;
    const int Rr = M / K;
    const float nm1 = (float)N - 1.0f;
    float2* zt = region0;
    const bool whole = Rr * K2 * W == kThreads;
    static_assert(32 * (kThreads + kYPad) <= kRegion0, "one batch of Y over zt fits in region0");
    float2* Y = whole ? region0 : region0 + K * W;
    const int VBn = whole ? Rr : VBmax;
    for (int idx = tid; idx < K * W; idx += kThreads) {
        const int k1 = idx >> 3;
        const int kk = idx & 7;
        zt[idx] = bin_value(R, S, pool, nm1, R.L + k2_0 + kk + kP2 * k1);
    }
    __syncthreads();
    // (B) task t = (vb K2 + j) 8 + kk: FFT32 over i of the pre-twiddled column,
    // then the twiddle w_K^{j u1} = w_M^{j u1 R}
    auto fft32_task = [&](int t, int v0, float2 (&x)[32]) {
        const int kk = t & 7;
        const int j = (t >> 3) % K2;
        const int v = v0 + (t >> 3) / K2;
        // pre-twiddle w_M^{v k1}: exact table value every 8 steps, running product in between
        const float2 stp = twhi[((unsigned)v * (unsigned)K2) & Mm];
        float2 w = make_float2(1.0f, 0.0f);
#pragma unroll
        for (int i = 0; i < 32; i++) {
            if ((i & 7) == 0) w = twhi[((unsigned)v * (unsigned)(j + K2 * i)) & Mm];
            x[i] = cmul(zt[(j + K2 * i) * W + kk], w);
            w = cmul(w, stp);
        }
        fft_reg<32, +1>(x);
    };
    // twiddle w_K^{j u1} = w_M^{j u1 R} of task t, applied as the FFT32 outputs are stored
    auto post_tw = [&](int t, int u1) -> float2 {
        const int j = (t >> 3) % K2;
        return twhi[((unsigned)(j * u1 * Rr)) & Mm];
    };
    for (int v0 = 0; v0 < Rr; v0 += VBn) {
        const int VB = min(VBn, Rr - v0);
        const int T = VB * K2 * W;
        const int TP = T + kYPad;
        if (whole) {
            // one task per thread; Y overwrites zt after every thread has read its inputs
            float2 x[32];
            fft32_task(tid, v0, x);
            __syncthreads();
            Y[tid] = x[0];
#pragma unroll
            for (int u1 = 1; u1 < 32; u1++) Y[u1 * TP + tid] = cmul(x[u1], post_tw(tid, u1));
        } else {
            for (int t = tid; t < T; t += kThreads) {
                float2 x[32];
                fft32_task(t, v0, x);
                Y[t] = x[0];
#pragma unroll
                for (int u1 = 1; u1 < 32; u1++) Y[u1 * TP + t] = cmul(x[u1], post_tw(t, u1));
            }
        }
        __syncthreads();
        // (C) K2-point DFT over j, task t = (vb 32 + u1) 8 + kk
        for (int t = tid; t < VB * 32 * W; t += kThreads) {
            const int kk = t & 7;
            const int u1 = (t >> 3) & 31;
            const int vb = t >> 8;
            float2 z[K2];
#pragma unroll
            for (int j = 0; j < K2; j++) z[j] = Y[u1 * TP + (vb * K2 + j) * W + kk];
            fft_reg<K2, +1>(z);
            const int k2 = k2_0 + kk;
            const unsigned k2L = (unsigned)(k2 + R.L);
            const unsigned c0 = (unsigned)(v0 + vb + Rr * u1);
            const unsigned dc = (unsigned)(32 * Rr);
            const float2 st = tw_n(twlo, twhi, (k2L * dc) & Nm);
            float2 w = make_float2(1.0f, 0.0f);
#pragma unroll
            for (int u2 = 0; u2 < K2; u2++) {
                const unsigned c = c0 + dc * (unsigned)u2;
                if ((u2 & 7) == 0) w = tw_n(twlo, twhi, (k2L * c) & Nm);
                __stcg(G + (size_t)c * kP2 + k2, cmul(z[u2], w));
                w = cmul(w, st);
            }
        }
        __syncthreads();
    }
}

__device__ void phase1_wide_dispatch(int K, const SigDesc& S, const RowDesc& R, const float* pool, int k2_0,
                                     const float2* twlo, const TwM twhi, float2* region0, float2* G) {
    switch (K) {
        case 64: phase1_big<2>(S, R, pool, k2_0, twlo, twhi, region0, G); break;
        case 128: phase1_big<4>(S, R, pool, k2_0, twlo, twhi, region0, G); break;
        case 256: phase1_big<8>(S, R, pool, k2_0, twlo, twhi, region0, G); break;
        case 512: phase1_big<16>(S, R, pool, k2_0, twlo, twhi, region0, G); break;
        default: phase1_wide<32>(S, R, pool, k2_0, twlo, twhi, region0, G); break;
    }
}

// Warp-level 1024-point DFT (sign +): on entry lane l holds x[m] = G[l + 32 m];
// on exit lane l holds x[h] = Y[l + 32 h]. tbuf: 32*33 float2 of this warp.
__device__ __forceinline__ void dft1024_warp(float2 (&x)[32], int lane, float2* __restrict__ tbuf,
                                             const float2* __restrict__ t2) {
    fft_reg<32, +1>(x);
#pragma unroll
    for (int a = 1; a < 32; a++) x[a] = cmul(x[a], t2[a * 32 + lane]);
#pragma unroll
    for (int a = 0; a < 32; a++) tbuf[a * 33 + lane] = x[a];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 32; k++) x[k] = tbuf[lane * 33 + k];
    __syncwarp();
    fft_reg<32, +1>(x);
}

// Phase 2 of columns [c0, c0 + 8) of a row: one warp per column runs the
// 1024-point DFT; the outputs y[c0 + w + M a] go out either through the tensor
// map (4 bulk stores of [256 a][8 w] boxes from a swizzled SMEM tile, issued by
// thread 0 and completed asynchronously; the partial last stripe a = n / M is
// stored by threads) or, without a tensor map, as runs of 8 samples stored by
// all threads from a padded SMEM tile.
//
// Time decimation D: output sample t' = c' + M a (M = the decimated column
// count N / 1024 / D, n = the decimated length) is y[D t'], i.e. column
// c = D c' of G; only those columns are transformed.
template <int OT>
__device__ __forceinline__ void phase2_item(const float2* __restrict__ G, int c0, int M, int n, int D, void* outb,
                                         long long out_off, int out_row, float2* __restrict__ region0,
                                         const float2* __restrict__ t2, const CUtensorMap* omap, bool tma) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const float2* __restrict__ col = G + (size_t)(c0 + warp) * (size_t)D * kP2 + lane;
    float2 x[32];
#pragma unroll
    for (int m = 0; m < 32; m++) x[m] = __ldcg(col + 32 * m);
    dft1024_warp(x, lane, region0 + warp * (32 * 33), t2);
    __syncthreads();
    const long long row0 = out_off + c0;
    if (tma) {
        unsigned char* stage = reinterpret_cast<unsigned char*>(region0);
        if constexpr (OT == OUT_C64) {
#pragma unroll
            for (int h = 0; h < 32; h++)
                *reinterpret_cast<float2*>(stage + stage_off(lane + 32 * h, warp)) = x[h];
        } else {
#pragma unroll
            for (int h = 0; h < 32; h++)
                *reinterpret_cast<unsigned*>(stage + stage16_off(lane + 32 * h, warp)) = pack16<OT>(x[h]);
        }
        fence_proxy_async_smem();
        __syncthreads();
        const int n_full = n / M;  // stripes a < n_full are complete
        constexpr int box_bytes = OT == OUT_C64 ? kBoxBytes : kBoxBytes / 2;
        if (tid == 0) {
            // complex64 output lines evict-first in L2: they are not read again,
            // and the spectrum and scratch the engine re-reads stay resident
            for (int j = 0; j < 4 && j * kBoxRows < n_full; j++)
                tma_store_3d<OT == OUT_C64>(omap, stage + j * box_bytes, c0, j * kBoxRows, out_row);
            bulk_commit();
        }
        const int tail = n - n_full * M;  // samples of the partial stripe a = n_full
        if (tid < kGroupCols && c0 + tid < tail && n_full < kP2) {
            const long long o = row0 + tid + (long long)M * n_full;
            if constexpr (OT == OUT_C64)
                store_out<OT>(outb, o, *reinterpret_cast<const float2*>(stage + stage_off(n_full, tid)));
            else
                __stcs(reinterpret_cast<unsigned*>(outb) + o,
                       *reinterpret_cast<const unsigned*>(stage + stage16_off(n_full, tid)));
        }
        // region0 is reused only after thread 0 waited for the bulk reads
    } else {
#pragma unroll
        for (int h = 0; h < 32; h++) region0[(lane + 32 * h) * kStagePitch + warp] = x[h];
        __syncthreads();
        for (int idx = tid; idx < kGroupCols * kP2; idx += kThreads) {
            const int w = idx & (kGroupCols - 1);
            const int a = idx >> 3;
            if (c0 + w + M * a < n) store_out<OT>(outb, row0 + w + (long long)M * a, region0[a * kStagePitch + w]);
        }
        __syncthreads();
    }
}

template <int OT>
__global__ void __launch_bounds__(kThreads, 2)
    k_row_engine(const __grid_constant__ EngineParams P, const __grid_constant__ CUtensorMap omap) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float2* smem = reinterpret_cast<float2*>(
        smem_raw + ((kSmemAlign - ((size_t)__cvta_generic_to_shared(smem_raw) & (kSmemAlign - 1))) & (kSmemAlign - 1)));
    float2* region0 = smem;
    float2* zs = smem + kRegion0;
    float2* twlo = zs + kZs;
    float2* t2 = twlo + kP2;
    float2* twhi_s = t2 + kP2;
    __shared__ int s_item;
    __shared__ int s_log2N;
    __shared__ int s_ok;
    __shared__ RowDesc s_rows[kFetchBatch];
    __shared__ SigDesc s_sigs[kFetchBatch];
    __shared__ Item s_its[kFetchBatch];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;

    // t2[a*32 + l] = w_1024^{a l}
    for (int j = tid; j < kP2; j += kThreads) {
        const int a = j >> 5, l = j & 31;
        double s, c;
        sincospi(2.0 * (double)((a * l) & 1023) / 1024.0, &s, &c);
        t2[j] = make_float2((float)c, (float)s);
    }
    if (tid == 0) s_log2N = -1;
    __syncthreads();

    unsigned* a_done = P.counters + 1;
    unsigned* b_done = P.counters + 1 + P.n_rows;

    // Items are claimed kFetchBatch at a time (one atomic and one round of
    // descriptor loads per batch) and processed in claim order.
    for (;;) {
        if (tid == 0) {
            const int i = (int)atomicAdd(P.counters, (unsigned)kFetchBatch);
            s_item = i;
#pragma unroll
            for (int b = 0; b < kFetchBatch; b++)
                if (i + b < P.n_items) s_its[b] = P.items[i + b];
#pragma unroll
            for (int b = 0; b < kFetchBatch; b++)
                if (i + b < P.n_items) s_rows[b] = P.rows[s_its[b].row];
#pragma unroll
            for (int b = 0; b < kFetchBatch; b++)
                if (i + b < P.n_items) s_sigs[b] = P.sigs[s_rows[b].sig];
        }
        __syncthreads();
        if (s_item >= P.n_items) break;
      for (int bi = 0; bi < kFetchBatch && s_item + bi < P.n_items; bi++) {
        const Item& item = s_its[bi];
        const RowDesc& R = s_rows[bi];
        const SigDesc& S = s_sigs[bi];
        const int log2N = S.log2N;
        const int N = 1 << log2N;
        const int n = S.n;
        void* outb = P.outs[R.out_buf];
        const int Mcols = N >> kLog2P2;
        const TwM twhi = Mcols <= kTwhiSmem ? TwM{twhi_s, nullptr} : TwM{twhi_s, twhi_s + 32};

        // region0 may still be read by the bulk stores of the previous phase-2 item
        if (P.tma_store && (item.type == ITEM_PHASE2 || item.type == ITEM_FUSED || item.type == ITEM_PHASE1W)) {
            if (tid == 0) bulk_wait_read_all();
            __syncthreads();
        }
        // twiddle tables of this N into SMEM
        if (s_log2N != log2N) {
            for (int j = tid; j < kP2; j += kThreads) twlo[j] = S.tw[j];
            if (Mcols <= kTwhiSmem) {
                for (int j = tid; j < Mcols; j += kThreads) twhi_s[j] = S.tw[kP2 + j];
            } else {
                for (int j = tid; j < 32; j += kThreads) twhi_s[j] = S.tw[kP2 + j];
                for (int j = tid; j < Mcols / 32; j += kThreads) twhi_s[32 + j] = S.tw[kP2 + 32 * j];
            }
            __syncthreads();
            if (tid == 0) s_log2N = log2N;
        }

        if (item.type == ITEM_SMALL) {
            // N < 1024: direct DFT over the row's nonzero bins.
            const int lo = R.lo, hi = R.hi;
            const float nm1 = (float)N - 1.0f;
            for (int q = lo + tid; q < hi; q += kThreads) zs[q - lo] = bin_value(R, S, P.stale_pool, nm1, q);
            __syncthreads();
            for (int to = tid; to < R.n_out; to += kThreads) {
                const int t = to * R.dec;
                float2 acc = make_float2(0.0f, 0.0f);
                for (int q = lo; q < hi; q++) {
                    const float2 w = twlo[(q * t) & (N - 1)];
                    const float2 z = zs[q - lo];
                    acc.x += z.x * w.x - z.y * w.y;
                    acc.y += z.x * w.y + z.y * w.x;
                }
                store_out<OT>(outb, R.out_off + to, acc);
            }
        } else if (item.type == ITEM_FUSED) {
            // whole row in this CTA (N <= 8192, M <= 8 columns): phase 1 into
            // SMEM, then one warp per column
            const int M = N >> kLog2P2;
            for (int k2_0 = 0; k2_0 < kP2; k2_0 += kChunk)
                phase1_chunk_dispatch<false>(R.K, S, R, P.stale_pool, k2_0, zs, twlo, twhi, region0);
            float2 x[32];
            if (warp < M) {
#pragma unroll
                for (int m = 0; m < 32; m++) x[m] = region0[warp * kP2 + lane + 32 * m];
            }
            __syncthreads();
            if (warp < M) dft1024_warp(x, lane, region0 + warp * (32 * 33), t2);
            __syncthreads();
            if (warp < M) {
#pragma unroll
                for (int h = 0; h < 32; h++) region0[(lane + 32 * h) * kStagePitch + warp] = x[h];
            }
            __syncthreads();
            const int log2M = log2N - kLog2P2;
            for (int to = tid; to < R.n_out; to += kThreads) {
                const int t = to * R.dec;
                const int c = t & (M - 1);
                const int a = t >> log2M;
                store_out<OT>(outb, R.out_off + to, region0[a * kStagePitch + c]);
            }
        } else if (item.type == ITEM_PHASE1) {
            if (tid == 0) {
                s_ok = 1;
                if (R.wait_row >= 0)
                    s_ok = wait_counter(b_done + R.wait_row, (unsigned)P.rows[R.wait_row].n_b, P.err) ? 1 : 0;
            }
            __syncthreads();
            if (s_ok) {
                float2* G = P.scratch + (size_t)R.slot * (size_t)P.slot_elems;
                phase1_chunk_dispatch<true>(R.K, S, R, P.stale_pool, item.part * kChunk, zs, twlo, twhi, G);
                if (tid == 0) {
                    __threadfence();
                    red_release_add(a_done + item.row, 1u);
                }
            }
        } else if (item.type == ITEM_PHASE1W) {
            if (tid == 0) {
                s_ok = 1;
                if (R.wait_row >= 0)
                    s_ok = wait_counter(b_done + R.wait_row, (unsigned)P.rows[R.wait_row].n_b, P.err) ? 1 : 0;
            }
            __syncthreads();
            if (s_ok) {
                float2* G = P.scratch + (size_t)R.slot * (size_t)P.slot_elems;
                phase1_wide_dispatch(R.K, S, R, P.stale_pool, item.part * kWideChunk, twlo, twhi, region0, G);
                if (tid == 0) {
                    __threadfence();
                    red_release_add(a_done + item.row, 1u);
                }
            }
        } else if (item.type == ITEM_PHASE2) {
            if (tid == 0) s_ok = wait_counter(a_done + item.row, (unsigned)R.n_a, P.err) ? 1 : 0;
            __syncthreads();
            if (s_ok) {
                const float2* G = P.scratch + (size_t)R.slot * (size_t)P.slot_elems;
                phase2_item<OT>(G, item.part * kGroupCols, (N >> kLog2P2) / R.dec, R.n_out, R.dec, outb, R.out_off,
                                R.out_row, region0, t2, &omap, P.tma_store != 0 && R.out_buf == 0);
                if (tid == 0) {
                    __threadfence();
                    red_release_add(b_done + item.row, 1u);
                }
            }
        } else {
            if (tid == 0) atomicOr(P.err, kErrBadItem);
        }
        __syncthreads();
      }
    }
    if (tid == 0 && P.tma_store) bulk_wait_all();
}

}  // namespace dev

// ------------------------------------------------------------ launch glue

size_t engine_smem_bytes() { return dev::kEngineSmemBytes; }

cudaError_t launch_mother(float fb, int N, float norm, float* out, cudaStream_t st) {
    const int tb = 256;
    dev::k_mother<<<(N + tb - 1) / tb, tb, 0, st>>>(fb, N, norm, out);
    return cudaGetLastError();
}

cudaError_t launch_twiddle(int log2N, float2* tw, cudaStream_t st) {
    const int N = 1 << log2N;
    const int M = N >= 1024 ? N / 1024 : 1;
    const int total = 1024 + M;
    dev::k_twiddle<<<(total + 255) / 256, 256, 0, st>>>(log2N, tw);
    return cudaGetLastError();
}

// Forward FFT of the zero-padded input into `out` (N complex values), using
// `tmp` (N complex) as the ping-pong buffer.
// ---- doublesided wavelets (src/fcwt/fcwt.cpp:241-273): the product also
// writes bins b in [N - proc, N) with weight mother[idx(N - 1 - b)] on the
// mirrored spectrum Ihat[b] = conj(Ihat[N - b]) (fcwt.cpp:507-510). With
// q = N - 1 - b that half of a row is exp(-2 pi i t / N) conj(V[t]), V the
// ordinary single-sided row of the same weights on the shifted spectrum
//     J[q] = Ihat[q + 1] (q < N/2 - 1),  J[N/2 - 1] = conj(Ihat[N/2]).
namespace dev {
__global__ void k_shift_spectrum(const float2* __restrict__ X, int N, float2* __restrict__ J) {
    const int half = N >> 1;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N; q += gridDim.x * blockDim.x) {
        float2 v = make_float2(0.0f, 0.0f);
        if (q + 1 < half)
            v = X[q + 1];
        else if (q + 1 == half)
            v = make_float2(X[half].x, -X[half].y);
        J[q] = v;
    }
}

// out[r][t'] += sgn * exp(-2 pi i t / N) * conj(V[r][t']) for rows r < rows,
// output samples t' < n (t = dec t', the row's sample).
__global__ void k_doublesided_combine(float2* __restrict__ out, const float2* __restrict__ V, long long rows, int n,
                                      int dec, int log2N, const float2* __restrict__ tw, float sgn) {
    const long long total = rows * (long long)n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(i % n) * dec;
        const float2 w = tw_lookup(tw, log2N, (unsigned)t);  // exp(+2 pi i t / N)
        const float2 v = V[i];
        // exp(-2 pi i t/N) conj(v) = conj(w v)
        const float2 p = cmul(w, v);
        float2 o = out[i];
        o.x += sgn * p.x;
        o.y -= sgn * p.y;
        out[i] = o;
    }
}
}  // namespace dev

// ---- the reference's odd-n row shift (compat mode, src/fcwt/fcwt.cpp:418-445)
// A shifted row r keeps at element 0 what row r - 1's inverse FFT wrote past
// its n samples, sample n of that row, normalised by both rows' fft_normalize:
//   out[r][0] = extra * sum_q Z_{r-1}[q] exp(2 pi i q n / N)
// (Z includes the first 1/N when normalising; extra is the second).
namespace dev {
__global__ void k_align_spill(const SigDesc* __restrict__ sigs, const RowDesc* __restrict__ rows,
                              const int* __restrict__ list, const float* __restrict__ pool, float2* __restrict__ out,
                              int n, float extra) {
    const int r = list[blockIdx.x];
    const RowDesc R = rows[r - 1];
    const SigDesc S = sigs[R.sig];
    const int N = 1 << S.log2N;
    const float nm1 = (float)N - 1.0f;
    float2 acc = make_float2(0.0f, 0.0f);
    for (int q = R.lo + threadIdx.x; q < R.hi; q += blockDim.x) {
        const float2 z = bin_value(R, S, pool, nm1, q);
        const float2 w = tw_lookup(S.tw, S.log2N, (unsigned)(((long long)q * n) & (N - 1)));
        acc = cadd(acc, cmul(z, w));
    }
    __shared__ float2 red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float2 s = make_float2(0.0f, 0.0f);
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = cadd(s, red[w]);
        out[(long long)r * n] = make_float2(s.x * extra, s.y * extra);
    }
}
}  // namespace dev

cudaError_t launch_align_spill(const SigDesc* sigs, const RowDesc* rows, const int* list, int nlist,
                               const float* pool, float2* out, int n, float extra, cudaStream_t st) {
    if (nlist <= 0) return cudaSuccess;
    dev::k_align_spill<<<nlist, 256, 0, st>>>(sigs, rows, list, pool, out, n, extra);
    return cudaGetLastError();
}

cudaError_t launch_shift_spectrum(const float2* X, int log2N, float2* J, cudaStream_t st) {
    const int N = 1 << log2N;
    dev::k_shift_spectrum<<<std::max(1, std::min(1184, (N + 255) / 256)), 256, 0, st>>>(X, N, J);
    return cudaGetLastError();
}

cudaError_t launch_doublesided_combine(float2* out, const float2* V, long long rows, int n, int dec, int log2N,
                                       const float2* tw, float sgn, cudaStream_t st) {
    const long long total = rows * (long long)n;
    if (total <= 0) return cudaSuccess;
    const int grid = (int)std::max(1LL, std::min(148LL * 16, (total + 255) / 256));
    dev::k_doublesided_combine<<<grid, 256, 0, st>>>(out, V, rows, n, dec, log2N, tw, sgn);
    return cudaGetLastError();
}

cudaError_t fft_configure();

cudaError_t engine_configure() {
    cudaError_t e = fft_configure();
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(dev::k_row_engine<OUT_C64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dev::kEngineSmemBytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(dev::k_row_engine<OUT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dev::kEngineSmemBytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(dev::k_row_engine<OUT_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dev::kEngineSmemBytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(dev::k_row_engine<OUT_POWER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dev::kEngineSmemBytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(dev::k_row_engine<OUT_DB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dev::kEngineSmemBytes);
}

// Resident CTAs of the row engine per SM (the persistent grid is SMs x this).
cudaError_t engine_blocks_per_sm(int* out) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, dev::k_row_engine<OUT_C64>, kThreads,
                                                         dev::kEngineSmemBytes);
}

cudaError_t launch_engine(const EngineParams& p, const CUtensorMap& omap, int grid, cudaStream_t st) {
    switch (p.out_type) {
        case OUT_BF16: dev::k_row_engine<OUT_BF16><<<grid, kThreads, dev::kEngineSmemBytes, st>>>(p, omap); break;
        case OUT_F16: dev::k_row_engine<OUT_F16><<<grid, kThreads, dev::kEngineSmemBytes, st>>>(p, omap); break;
        case OUT_POWER: dev::k_row_engine<OUT_POWER><<<grid, kThreads, dev::kEngineSmemBytes, st>>>(p, omap); break;
        case OUT_DB: dev::k_row_engine<OUT_DB><<<grid, kThreads, dev::kEngineSmemBytes, st>>>(p, omap); break;
        default: dev::k_row_engine<OUT_C64><<<grid, kThreads, dev::kEngineSmemBytes, st>>>(p, omap); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_engine(const EngineParams& p, int grid, cudaStream_t st) {
    CUtensorMap none;
    memset(&none, 0, sizeof(none));
    EngineParams q = p;
    q.tma_store = 0;
    return launch_engine(q, none, grid, st);
}

}  // namespace fcwt
