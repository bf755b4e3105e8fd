// Forward (and unnormalised inverse) FFTs of whole signals: the spectrum
// Ihat = FFT_N(zero-padded signal) that every row of the transform reads
// (replaces fftwf r2c / c2c FORWARD, src/fcwt/fcwt.cpp:486-500, and the
// conjugate mirror of fcwt.cpp:507-510).
//
// A length-C complex FFT (C = 2^p) runs as one or two passes through global
// memory (L2-resident at these sizes); inside a pass each CTA transforms a
// tile of B columns x L points in shared memory with radix-16/8/4/2 Stockham
// stages:
//   p <= 12: one pass, the whole signal in one CTA;
//   p >= 13: C = C1 C2, j = j1 + C1 j2, k = k2 + C2 k1 (four-step):
//     pass A  for each j1, the C2-point DFT over j2, times w_C^{j1 k2}
//             -> T[j1 + C1 k2];
//     pass B  for each k2, the C1-point DFT over j1 -> Z[k2 + C2 k1].
// Columns are interleaved in shared memory (element i of column cc at
// i B + cc) so that the B columns of a tile are read and written as B
// consecutive elements of global memory.
//
// A real signal of N = 2C samples is transformed as the C-point FFT of its
// sample pairs z[j] = x[2j] + i x[2j+1], then split into all N bins
// (k_r2c_split). Complex inputs and the inverse transforms run the C = N
// complex FFT.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fcwt_dev.cuh"
#include "fcwt_fft.cuh"
#include "fcwt_internal.h"

namespace fcwt {
namespace dev {

constexpr int kFftThreads = 128;
constexpr int kFftMaxLog2Tile = 12;  // B L <= 4096 complex values per CTA (2 x 32 KB)
constexpr int kFftSmemBytes = 2 * (1 << kFftMaxLog2Tile) * 8;
constexpr int kFftTargetCtas = 2 * 148;  // about two CTAs per SM of a B200

// Element idx of a signal with implicit zero padding: a complex sample, or
// (r2c) the real pair (x[2 idx], x[2 idx + 1]).
__device__ __forceinline__ float2 fwd_input(const float* __restrict__ in_r, const float2* __restrict__ in_c,
                                            int n_in, int idx, int r2c) {
    if (in_r && r2c) {
        const int i0 = 2 * idx;
        return make_float2(i0 < n_in ? __ldg(in_r + i0) : 0.0f, i0 + 1 < n_in ? __ldg(in_r + i0 + 1) : 0.0f);
    }
    if (idx >= n_in) return make_float2(0.0f, 0.0f);
    return in_r ? make_float2(__ldg(in_r + idx), 0.0f) : __ldg(in_c + idx);
}

// w_T^{SIGN e} from the two-level table of T = 2^log2T (which holds w_T^{+e}).
template <int SIGN>
__device__ __forceinline__ float2 fft_tw(const float2* __restrict__ tw, int log2T, unsigned e) {
    float2 w = tw_lookup(tw, log2T, e);
    if (SIGN < 0) w.y = -w.y;
    return w;
}

// w_L^{SIGN e}, e < L, from the CTA's two-level table of w_L^{SIGN j}:
// tl[j] for j < 64 and th[j] = w_L^{SIGN 64 j} for j < L / 64.
__device__ __forceinline__ float2 stage_tw(const float2* __restrict__ tl, const float2* __restrict__ th, unsigned e) {
    return e < 64u ? tl[e] : cmul(tl[e & 63u], th[e >> 6]);
}

// One radix-R Stockham stage over L = 2^log2L points of B = 2^log2B
// interleaved columns: k = j mod Ns, v_r = in[j + r L/R] w_{Ns R}^{SIGN r k},
// V = DFT_R(v), out[(j - k) R + k + m Ns] = V_m.
template <int R, int SIGN>
__device__ __forceinline__ void smem_stage(const float2* __restrict__ in, float2* __restrict__ out, int log2L,
                                           int log2B, int log2Ns, const float2* __restrict__ tl,
                                           const float2* __restrict__ th) {
    constexpr int LR = ilog2c(R);
    const int B = 1 << log2B;
    const int Lr = 1 << (log2L - LR);
    const int tasks = Lr << log2B;
    const int shift = log2L - log2Ns - LR;  // w_{Ns R} = w_L^{2^shift}
    for (int t = threadIdx.x; t < tasks; t += kFftThreads) {
        const int cc = t & (B - 1);
        const int j = t >> log2B;
        const int k = j & ((1 << log2Ns) - 1);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            float2 x = in[((j + r * Lr) << log2B) + cc];
            if (r > 0 && k > 0) x = cmul(x, stage_tw(tl, th, (unsigned)(r * k) << shift));
            v[r] = x;
        }
        fft_reg<R, SIGN>(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int m = 0; m < R; m++) out[((base + (m << log2Ns)) << log2B) + cc] = v[m];
    }
}

// All stages of an L-point FFT on the tile in `a` (natural order in and
// out); returns the buffer that holds the result.
template <int SIGN>
__device__ __forceinline__ float2* smem_fft(float2* a, float2* b, int log2L, int log2B, const float2* __restrict__ tl,
                                            const float2* __restrict__ th) {
    int log2Ns = 0;
    while (log2Ns < log2L) {
        const int lr = min(4, log2L - log2Ns);
        switch (lr) {
            case 4: smem_stage<16, SIGN>(a, b, log2L, log2B, log2Ns, tl, th); break;
            case 3: smem_stage<8, SIGN>(a, b, log2L, log2B, log2Ns, tl, th); break;
            case 2: smem_stage<4, SIGN>(a, b, log2L, log2B, log2Ns, tl, th); break;
            default: smem_stage<2, SIGN>(a, b, log2L, log2B, log2Ns, tl, th); break;
        }
        __syncthreads();
        float2* s = a;
        a = b;
        b = s;
        log2Ns += lr;
    }
    return a;
}

// One pass over a length-2^log2C array of the job blockIdx.y (or `one` when
// jobs is null). The CTA takes columns [B blockIdx.x, B blockIdx.x + B) of
// the S = C / L columns:
//   mode 0 (pass A): column col holds elements col + S i; its results are
//                    multiplied by w_C^{SIGN col k};
//   mode 1 (pass B): column col holds elements col L + i.
// Result k of column col goes to col + S k in both modes. src/dst: 0 = the
// job's input (zero padded; r2c: sample pairs), 1 = its spectrum X, 2 = its
// tmp buffer.
template <int SIGN>
__global__ void __launch_bounds__(kFftThreads) k_fft_cols(const FwdJob* __restrict__ jobs, FwdJob one, int src_sel,
                                                          int dst_sel, int log2C, int log2L, int log2B, int mode,
                                                          int r2c, const float2* __restrict__ tw, int log2T) {
    extern __shared__ float2 fft_sm[];
    __shared__ float2 tl[64], th[64];
    const FwdJob J = jobs ? jobs[blockIdx.y] : one;
    const int L = 1 << log2L;
    const int B = 1 << log2B;
    const int log2S = log2C - log2L;
    const int tot = L << log2B;
    const int c0 = blockIdx.x << log2B;
    float2* a = fft_sm;
    float2* b = fft_sm + tot;
    const float2* src = src_sel == 1 ? J.X : J.tmp;
    // stage twiddles w_L^{SIGN j}: tl for j < 64, th for multiples of 64
    for (int t = threadIdx.x; t < 128; t += kFftThreads) {
        const unsigned e = t < 64 ? (unsigned)t : (unsigned)(t - 64) << 6;
        if (e < (unsigned)L) (t < 64 ? tl[t] : th[t - 64]) = fft_tw<SIGN>(tw, log2T, e << (log2T - log2L));
    }
    for (int t = threadIdx.x; t < tot; t += kFftThreads) {
        int i, cc;
        if (mode == 0) {
            cc = t & (B - 1);
            i = t >> log2B;
        } else {
            i = t & (L - 1);
            cc = t >> log2L;
        }
        const int col = c0 + cc;
        const int j = mode == 0 ? col + (i << log2S) : (col << log2L) + i;
        a[(i << log2B) + cc] = src_sel == 0 ? fwd_input(J.in_r, J.in_c, J.n, j, r2c) : src[j];
    }
    __syncthreads();
    const float2* res = smem_fft<SIGN>(a, b, log2L, log2B, tl, th);
    float2* dst = dst_sel == 1 ? J.X : J.tmp;
    for (int t = threadIdx.x; t < tot; t += kFftThreads) {
        const int cc = t & (B - 1);
        const int k = t >> log2B;
        const int col = c0 + cc;
        float2 v = res[t];
        if (mode == 0 && col > 0 && k > 0)
            v = cmul(v, fft_tw<SIGN>(tw, log2T, (unsigned)(col * k) << (log2T - log2C)));
        dst[col + (k << log2S)] = v;
    }
}

// Real-input split: with Z = FFT_{N/2}(z), E = (Z[k] + conj Z[N/2-k]) / 2 and
// O = -i (Z[k] - conj Z[N/2-k]) / 2,
//   X[k] = E + w_N^{-k} O,   X[N/2 - k] = conj(E - w_N^{-k} O),
// and X[N - k] = conj X[k] (real input). Thread k in [0, N/4] writes bins
// k, N/2 - k, N/2 + k and N - k, so all N bins are written once.
__global__ void k_r2c_split(const FwdJob* __restrict__ jobs, FwdJob one, int log2N, const float2* __restrict__ tw) {
    const FwdJob J = jobs ? jobs[blockIdx.y] : one;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = 1 << log2N;
    const int H = N >> 1;
    if (k > N / 4) return;
    const float2* __restrict__ Z = J.tmp;
    float2* __restrict__ X = J.X;
    const float2 A = Z[k];
    const float2 Bz = Z[(H - k) & (H - 1)];
    const float2 E = make_float2(0.5f * (A.x + Bz.x), 0.5f * (A.y - Bz.y));
    const float2 O = make_float2(0.5f * (A.y + Bz.y), -0.5f * (A.x - Bz.x));
    const float2 wo = cmul(fft_tw<-1>(tw, log2N, (unsigned)k), O);
    const float2 xk = make_float2(E.x + wo.x, E.y + wo.y);
    const float2 yk = make_float2(E.x - wo.x, wo.y - E.y);
    X[k] = xk;
    if (k == 0) {
        X[H] = yk;
        return;
    }
    X[N - k] = make_float2(xk.x, -xk.y);
    if (2 * k < H) {
        X[H - k] = yk;
        X[H + k] = make_float2(yk.x, -yk.y);
    }
}

}  // namespace dev

cudaError_t fft_configure() {
    cudaError_t e = cudaFuncSetAttribute(dev::k_fft_cols<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         dev::kFftSmemBytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(dev::k_fft_cols<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev::kFftSmemBytes);
}

// FFTs of njobs signals of length N = 2^log2N (jobs in device memory, or
// `one` for a single signal). SIGN -1: forward, real inputs (real) as r2c
// when N >= 4, result in each job's X (all N bins); SIGN +1: unnormalised
// inverse of complex inputs. tw: the two-level table of N.
template <int SIGN>
static cudaError_t fft_signals(const FwdJob* jobs, const FwdJob& one, int njobs, int log2N, const float2* tw,
                               bool real, cudaStream_t st, int* n_kernels) {
    *n_kernels = 0;
    if (njobs <= 0) return cudaSuccess;
    if (log2N < 1) return cudaErrorInvalidValue;
    const int r2c = (SIGN < 0 && real && log2N >= 2) ? 1 : 0;
    const int log2C = log2N - r2c;
    auto pass = [&](int src, int dst, int log2L, int mode) -> cudaError_t {
        const int log2cols = log2C - log2L;
        // B = 2^log2B columns per CTA: at most 4096 / L, at most 8, and no more
        // than leaves about two CTAs per SM when there are enough columns
        int log2B = std::min(3, std::min(dev::kFftMaxLog2Tile - log2L, log2cols));
        while (log2B > 2 && ((long long)njobs << (log2cols - log2B)) < dev::kFftTargetCtas) log2B--;
        const int tile = 1 << (log2L + log2B);
        dim3 grid(1u << (log2cols - log2B), (unsigned)njobs);
        dev::k_fft_cols<SIGN><<<grid, dev::kFftThreads, (size_t)tile * 16, st>>>(jobs, one, src, dst, log2C, log2L,
                                                                                   log2B, mode, r2c, tw, log2N);
        (*n_kernels)++;
        return cudaGetLastError();
    };
    cudaError_t e;
    // the last pass writes X, or tmp when the split follows; pass A of r2c
    // writes into X (free until the split)
    const int last = r2c ? 2 : 1;
    if (log2C <= dev::kFftMaxLog2Tile) {
        e = pass(0, last, log2C, 1);
    } else {
        const int log2C2 = log2C / 2;  // pass A length (C2 <= C1)
        e = pass(0, r2c ? 1 : 2, log2C2, 0);
        if (e == cudaSuccess) e = pass(r2c ? 1 : 2, last, log2C - log2C2, 1);
    }
    if (e != cudaSuccess) return e;
    if (r2c) {
        const int threads = (1 << log2N) / 4 + 1;
        dev::k_r2c_split<<<dim3((threads + 255) / 256, (unsigned)njobs), 256, 0, st>>>(jobs, one, log2N, tw);
        (*n_kernels)++;
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_forward(const float* in_r, const float2* in_c, int n, int log2N, const float2* tw,
                           float2* out, float2* tmp, cudaStream_t st, int* n_kernels) {
    *n_kernels = 0;
    if (log2N == 0) {
        // N == 1: the DFT is the identity (one sample or none).
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float2), st);
        if (e != cudaSuccess) return e;
        if (n >= 1) {
            if (in_r)
                e = cudaMemcpy2DAsync(out, sizeof(float2), in_r, sizeof(float), sizeof(float), 1,
                                      cudaMemcpyDeviceToDevice, st);
            else
                e = cudaMemcpyAsync(out, in_c, sizeof(float2), cudaMemcpyDeviceToDevice, st);
        }
        return e;
    }
    FwdJob one;
    one.in_r = in_r;
    one.in_c = in_r ? nullptr : in_c;
    one.n = n;
    one.pad = 0;
    one.X = out;
    one.tmp = tmp;
    return fft_signals<-1>(nullptr, one, 1, log2N, tw, in_r != nullptr, st, n_kernels);
}

cudaError_t launch_forward_batched(const FwdJob* jobs, int njobs, int log2N, const float2* tw, cudaStream_t st,
                                   int* n_kernels, bool real) {
    FwdJob none{};
    return fft_signals<-1>(jobs, none, njobs, log2N, tw, real, st, n_kernels);
}

cudaError_t launch_inverse_batched(const FwdJob* jobs, int njobs, int log2N, const float2* tw, cudaStream_t st,
                                   int* n_kernels) {
    FwdJob none{};
    return fft_signals<+1>(jobs, none, njobs, log2N, tw, false, st, n_kernels);
}

}  // namespace fcwt
