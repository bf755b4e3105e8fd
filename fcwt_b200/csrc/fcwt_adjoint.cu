// Adjoint (backward) kernels of the differentiable Morlet CWT.
//
// Forward (continuous mode of the row engine), per signal b and row i:
//   y[b,i,t] = c * IFFTraw( X_b * g_i )[t],  t < n,   c = 1/N (normalised) or 1,
//   g_i(q) = A exp(-u^2/2),  u = 2 pi sigma (s_i q / N - 1),  s_i = fs / f_i,
// with X_b = FFT_N(zero-padded x_b) on bins q < N/2 (the single-sided Morlet).
// For an incoming gradient G (torch's convention, dL = Re<G, dy>) and
// Ghat[b,i] = FFT_N(zero-padded G[b,i]):
//   dL/dx_b   = Re( c * IFFTraw( sum_i g_i * Ghat[b,i] ) )[0:n]
//   dL/dsigma = Re( c * sum_{b,i,q} X_b(q) dg_i/dsigma(q) conj(Ghat[b,i](q)) )
//   dL/df_i   = Re( c * sum_{b,q}   X_b(q) dg_i/df_i(q)   conj(Ghat[b,i](q)) )
// dg/dsigma = -g u^2 / sigma;  dg/df = g u * 2 pi sigma (q/N) * fs / f^2.
// The spectra X_b are recomputed in the backward instead of being stored.
#include <cuda_runtime.h>

#include "fcwt_fft.cuh"
#include "fcwt_internal.h"

namespace fcwt {
namespace dev {

// Per-row constants of the continuous Morlet.
struct AdjRow {
    float ca;     // 2 pi sigma s / N
    float dfdq;   // 2 pi sigma (1/N) fs / f^2  (du/df = -dfdq * q)
};

constexpr int kAdjThreads = 256;
constexpr int kAdjMaxRows = 8;  // rows per accumulation pass

// One pass over a chunk of `nr` rows: H[b][q] += sum_i g_i(q) Ghat[b,i](q) and
// the parameter-gradient partial sums, reduced per block, accumulated in double.
__global__ void __launch_bounds__(kAdjThreads) k_adjoint_accum(const float2* __restrict__ Xs, const float2* __restrict__ Gh,
                                                              float2* __restrict__ H, const AdjRow* __restrict__ rows,
                                                              int nr, int half, long long Nstride, float cb, float amp,
                                                              float inv_sigma, double* __restrict__ acc_sigma,
                                                              double* __restrict__ acc_f) {
    const int b = blockIdx.y;
    const int q = blockIdx.x * kAdjThreads + threadIdx.x;
    float dsig = 0.0f;
    float df[kAdjMaxRows];
#pragma unroll
    for (int i = 0; i < kAdjMaxRows; i++) df[i] = 0.0f;
    if (q < half) {
        const float2 xq = Xs[(size_t)b * Nstride + q];
        float2 h = H[(size_t)b * Nstride + q];
        const float qf = (float)q;
#pragma unroll
        for (int i = 0; i < kAdjMaxRows; i++) {
            if (i < nr) {
                const AdjRow r = rows[i];
                const float u = r.ca * qf - cb;
                const float g = amp * expf(-0.5f * u * u);
                const float2 gh = Gh[((size_t)b * nr + i) * Nstride + q];
                h.x += g * gh.x;
                h.y += g * gh.y;
                // Re(X * conj(Gh))
                const float re = xq.x * gh.x + xq.y * gh.y;
                dsig += -g * u * u * inv_sigma * re;
                df[i] += g * u * r.dfdq * qf * re;
            }
        }
        H[(size_t)b * Nstride + q] = h;
    }
    // block reductions
    __shared__ float red[kAdjThreads / 32][kAdjMaxRows + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dsig += __shfl_xor_sync(0xffffffffu, dsig, o);
#pragma unroll
    for (int i = 0; i < kAdjMaxRows; i++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) df[i] += __shfl_xor_sync(0xffffffffu, df[i], o);
    }
    if (lane == 0) {
        red[warp][kAdjMaxRows] = dsig;
#pragma unroll
        for (int i = 0; i < kAdjMaxRows; i++) red[warp][i] = df[i];
    }
    __syncthreads();
    if (threadIdx.x <= kAdjMaxRows) {
        const int i = threadIdx.x;
        if (i == kAdjMaxRows || i < nr) {
            double s = 0.0;
            for (int w = 0; w < kAdjThreads / 32; w++) s += (double)red[w][i];
            if (i == kAdjMaxRows)
                atomicAdd(acc_sigma, s);
            else
                atomicAdd(acc_f + i, s);
        }
    }
}

// ---- fused row adjoint for N = 1024 M, M <= 16
// One CTA per (signal b, chunk of kAdjFusedRows rows): each incoming gradient
// row G[b,i] is transformed in shared memory (never written back), and its
// spectrum is consumed on the spot. Forward DFT (sign -) of the zero-padded
// row with t = c + M a, q = k2 + 1024 k1:
//   Ghat[k2 + 1024 k1] = sum_c w_M^{-k1 c} w_N^{-k2 c} DFT1024_-(G[c + M a])[k2]
// warp c runs the column DFT (as conj(DFT_+(conj))), the twiddled columns go
// to shared memory, and each thread then runs the M-point DFTs of its two k2
// values and accumulates, for its bins q < N/2, H[b][q] (in registers across
// the chunk's rows) and the sigma / frequency partial sums.
constexpr int kAdjFusedThreads = 512;
constexpr int kAdjFusedRows = 8;
constexpr int kAdjColPitch = kP2 + 1;  // column pitch (float2) of the shared buffer: conflict-free rows and columns

template <int M>
__global__ void __launch_bounds__(kAdjFusedThreads, 1)
    k_adjoint_rows(const float2* __restrict__ G, const float2* __restrict__ Xs, const AdjRow* __restrict__ rows,
                   int n, int fn, const float2* __restrict__ tw, float cb, float amp, float inv_sigma,
                   float2* __restrict__ H, double* __restrict__ acc_sigma, double* __restrict__ acc_f) {
    constexpr int N = kP2 * M;
    constexpr int HALF = N / 2;
    constexpr int LOGM = ilog2c(M);
    constexpr int KH = M >= 2 ? M / 2 : 1;  // bins per k2 below N/2
    extern __shared__ __align__(16) float2 adj_sm[];
    float2* S = adj_sm;                              // [M][kAdjColPitch]
    float2* t2 = adj_sm + M * kAdjColPitch;          // 32 x 32 DFT twiddles
    float2* twlo = t2 + kP2;                         // w_N^j, j < 1024
    float2* twhi = twlo + kP2;                       // w_N^{1024 j}, j < M
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int b = blockIdx.y;
    const int i0 = blockIdx.x * kAdjFusedRows;
    const int nr = min(kAdjFusedRows, fn - i0);
    for (int j = tid; j < kP2; j += kAdjFusedThreads) {
        const int a = j >> 5, l = j & 31;
        double sn, cs;
        sincospi(2.0 * (double)((a * l) & 1023) / 1024.0, &sn, &cs);
        t2[j] = make_float2((float)cs, (float)sn);
        twlo[j] = tw[j];
    }
    if (tid < M) twhi[tid] = M > 1 ? tw[kP2 + tid] : make_float2(1.0f, 0.0f);
    const unsigned Nm = (unsigned)N - 1u;
    float2 h[2][KH];
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
        for (int k = 0; k < KH; k++) h[u][k] = make_float2(0.0f, 0.0f);
    float dsig = 0.0f;
    __shared__ float s_df[kAdjFusedRows];  // per-row dL/df partial sums of the CTA
    if (tid < kAdjFusedRows) s_df[tid] = 0.0f;
    const float2* __restrict__ Xb = Xs + (size_t)b * N;
    __syncthreads();
    for (int r = 0; r < nr; r++) {
        const int i = i0 + r;
        const float2* __restrict__ g = G + ((size_t)b * fn + i) * (size_t)n;
        // (a) the row, conjugated, column-major: S[c][a] = conj(G[c + M a]), zero past n
        for (int t = tid; t < N; t += kAdjFusedThreads) {
            const float2 v = t < n ? __ldcs(g + t) : make_float2(0.0f, 0.0f);
            S[(t & (M - 1)) * kAdjColPitch + (t >> LOGM)] = make_float2(v.x, -v.y);
        }
        __syncthreads();
        // (b) column DFTs, twiddle w_N^{-k2 c}, back into the column
        if (warp < M) {
            float2* col = S + warp * kAdjColPitch;
            float2 x[32];
#pragma unroll
            for (int m = 0; m < 32; m++) x[m] = col[lane + 32 * m];
            __syncwarp();
            dft1024_warp_xor(x, lane, col, t2);
#pragma unroll
            for (int hh = 0; hh < 32; hh++) {
                const int k2 = lane + 32 * hh;
                const unsigned e = ((unsigned)k2 * (unsigned)warp) & Nm;
                const float2 w = cmul(twlo[e & 1023u], twhi[e >> 10]);
                // conj(x) * conj(w)
                const float2 y = make_float2(x[hh].x * w.x - x[hh].y * w.y, -(x[hh].x * w.y + x[hh].y * w.x));
                col[k2] = y;
            }
        }
        __syncthreads();
        // (c) M-point DFTs (sign -) across the columns; accumulate bins q < N/2
        const AdjRow rc = rows[i];
        float dfl = 0.0f;
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int k2 = tid + kAdjFusedThreads * u;
            float2 z[M];
#pragma unroll
            for (int c = 0; c < M; c++) z[c] = S[c * kAdjColPitch + k2];
            fft_reg<M, -1>(z);
#pragma unroll
            for (int k1 = 0; k1 < KH; k1++) {
                const int q = k2 + kP2 * k1;
                if (q < HALF) {
                    const float qf = (float)q;
                    const float uu = rc.ca * qf - cb;
                    const float gw = amp * expf(-0.5f * uu * uu);
                    const float2 gh = z[k1];
                    h[u][k1].x += gw * gh.x;
                    h[u][k1].y += gw * gh.y;
                    const float2 xq = __ldg(Xb + q);
                    const float re = xq.x * gh.x + xq.y * gh.y;
                    dsig += -gw * uu * uu * inv_sigma * re;
                    dfl += gw * uu * rc.dfdq * qf * re;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dfl += __shfl_xor_sync(0xffffffffu, dfl, o);
        if (lane == 0) atomicAdd(&s_df[r], dfl);
        __syncthreads();
    }
    // H[b][q] += h (only bins this chunk touched), then the parameter sums
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int k2 = tid + kAdjFusedThreads * u;
#pragma unroll
        for (int k1 = 0; k1 < KH; k1++) {
            const int q = k2 + kP2 * k1;
            if (q < HALF && (h[u][k1].x != 0.0f || h[u][k1].y != 0.0f)) {
                float* hp = reinterpret_cast<float*>(H + (size_t)b * N + q);
                atomicAdd(hp, h[u][k1].x);
                atomicAdd(hp + 1, h[u][k1].y);
            }
        }
    }
    __shared__ float red[kAdjFusedThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dsig += __shfl_xor_sync(0xffffffffu, dsig, o);
    if (lane == 0) red[warp] = dsig;
    __syncthreads();
    if (tid == 0) {
        double sacc = 0.0;
        for (int w = 0; w < kAdjFusedThreads / 32; w++) sacc += (double)red[w];
        atomicAdd(acc_sigma, sacc);
    }
    if (tid < nr) atomicAdd(acc_f + i0 + tid, (double)s_df[tid]);
}

// grad_x[b][t] = scale * Re(Y[b][t]) for t < n.
__global__ void k_take_real(const float2* __restrict__ Y, long long Nstride, int n, float scale,
                            float* __restrict__ gx) {
    const int b = blockIdx.y;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) gx[(size_t)b * n + t] = scale * Y[(size_t)b * Nstride + t].x;
}

}  // namespace dev

cudaError_t launch_adjoint_accum(const float2* Xs, const float2* Gh, float2* H, const void* rows, int nr, int half,
                                 long long Nstride, int batch, float cb, float amp, float inv_sigma, double* acc_sigma,
                                 double* acc_f, cudaStream_t st) {
    if (nr > dev::kAdjMaxRows) return cudaErrorInvalidValue;
    dim3 grid((half + dev::kAdjThreads - 1) / dev::kAdjThreads, batch);
    dev::k_adjoint_accum<<<grid, dev::kAdjThreads, 0, st>>>(Xs, Gh, H, static_cast<const dev::AdjRow*>(rows), nr, half,
                                                           Nstride, cb, amp, inv_sigma, acc_sigma, acc_f);
    return cudaGetLastError();
}

cudaError_t launch_take_real(const float2* Y, long long Nstride, int n, int batch, float scale, float* gx,
                             cudaStream_t st) {
    dim3 grid((n + 255) / 256, batch);
    dev::k_take_real<<<grid, 256, 0, st>>>(Y, Nstride, n, scale, gx);
    return cudaGetLastError();
}

int adjoint_rows_per_pass() { return dev::kAdjMaxRows; }

size_t adjoint_fused_smem(int M) { return sizeof(float2) * ((size_t)M * dev::kAdjColPitch + 2 * kP2 + 16); }

// The fused row adjoint for N = 1024 M, M in {1, 2, 4, 8, 16}; returns
// cudaErrorInvalidValue for other N (the caller then uses the FFT passes).
cudaError_t launch_adjoint_rows(const float2* G, const float2* Xs, const void* rows, int n, int log2N, int fn,
                                int batch, const float2* tw, float cb, float amp, float inv_sigma, float2* H,
                                double* acc_sigma, double* acc_f, cudaStream_t st) {
    const int M = log2N >= kLog2P2 ? 1 << (log2N - kLog2P2) : 0;
    if (M < 1 || M > 16) return cudaErrorInvalidValue;
    const dim3 grid((fn + dev::kAdjFusedRows - 1) / dev::kAdjFusedRows, batch);
    const size_t sm = adjoint_fused_smem(M);
    const auto* r = static_cast<const dev::AdjRow*>(rows);
    cudaError_t e = cudaSuccess;
#define FCWT_ADJ_CASE(MM)                                                                                   \
    case MM:                                                                                                \
        e = cudaFuncSetAttribute(dev::k_adjoint_rows<MM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
        if (e != cudaSuccess) return e;                                                                     \
        dev::k_adjoint_rows<MM><<<grid, dev::kAdjFusedThreads, sm, st>>>(G, Xs, r, n, fn, tw, cb, amp, inv_sigma, \
                                                                          H, acc_sigma, acc_f);             \
        break;
    switch (M) {
        FCWT_ADJ_CASE(1)
        FCWT_ADJ_CASE(2)
        FCWT_ADJ_CASE(4)
        FCWT_ADJ_CASE(8)
        FCWT_ADJ_CASE(16)
        default: return cudaErrorInvalidValue;
    }
#undef FCWT_ADJ_CASE
    return cudaGetLastError();
}

}  // namespace fcwt
