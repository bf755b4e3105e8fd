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

}  // namespace fcwt
