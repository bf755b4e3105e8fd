// Register-resident power-of-two DFTs with compile-time twiddles, plus small
// complex helpers. Radix-2 decimation in time; the bit-reversal permutation is
// resolved at compile time (pure register renaming). Trivial rotations (1, ±i,
// (1±i)/sqrt2 and their negatives) are special-cased so no multiply is spent
// on them.
#pragma once

#include <cuda_runtime.h>

namespace fcwt {
namespace dev {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// cos(2*pi*j/64), j = 0..16
constexpr float kCos64[17] = {
    1.000000000e+00f, 9.951847267e-01f, 9.807852804e-01f, 9.569403357e-01f, 9.238795325e-01f,
    8.819212643e-01f, 8.314696123e-01f, 7.730104534e-01f, 7.071067812e-01f, 6.343932842e-01f,
    5.555702330e-01f, 4.713967368e-01f, 3.826834324e-01f, 2.902846773e-01f, 1.950903220e-01f,
    9.801714033e-02f, 0.0f};

// a * exp(SIGN * 2*pi*i * J/64) for 0 <= J < 32.
template <int J, int SIGN>
__device__ __forceinline__ float2 rot64(float2 a) {
    constexpr float r = 7.071067812e-01f;
    if constexpr (J == 0) {
        return a;
    } else if constexpr (J == 16) {
        return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
    } else if constexpr (J == 8) {
        return SIGN > 0 ? make_float2((a.x - a.y) * r, (a.x + a.y) * r)
                        : make_float2((a.x + a.y) * r, (a.y - a.x) * r);
    } else if constexpr (J == 24) {
        return SIGN > 0 ? make_float2(-(a.x + a.y) * r, (a.x - a.y) * r)
                        : make_float2((a.y - a.x) * r, -(a.x + a.y) * r);
    } else {
        constexpr float c = J <= 16 ? kCos64[J] : -kCos64[32 - J];
        constexpr float s0 = J <= 16 ? kCos64[16 - J] : kCos64[J - 16];
        constexpr float s = SIGN > 0 ? s0 : -s0;
        return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
    }
}

__host__ __device__ constexpr int ilog2c(int k) { return k <= 1 ? 0 : 1 + ilog2c(k / 2); }
__host__ __device__ constexpr int brev(int x, int bits) {
    int r = 0;
    for (int i = 0; i < bits; i++) r = (r << 1) | ((x >> i) & 1);
    return r;
}

// Butterfly (a + w b, a - w b) with w = exp(SIGN 2 pi i JJ / 64), JJ not a
// multiple of 16, in six FMA-pipe instructions instead of eight: with
// w = c + i s and |c| >= |s|, w b = c * (b (1 + i s/c)), so
// b' = (b.x - r b.y, b.y + r b.x) (r = s/c, two FMAs) and the outputs are
// a +- c b' (four FMAs); with |s| > |c| the same with w b = s * (b (c/s + i)).
template <int JJ, int SIGN>
__device__ __forceinline__ void bfly64(float2& ya, float2& yb) {
    constexpr float c = JJ <= 16 ? kCos64[JJ] : -kCos64[32 - JJ];
    constexpr float s0 = JJ <= 16 ? kCos64[16 - JJ] : kCos64[JJ - 16];
    constexpr float s = SIGN > 0 ? s0 : -s0;
    const float2 a = ya, b = yb;
    if constexpr ((c >= 0 ? c : -c) >= (s >= 0 ? s : -s)) {
        constexpr float r = s / c;
        const float2 bp = make_float2(fmaf(-r, b.y, b.x), fmaf(r, b.x, b.y));
        ya = make_float2(fmaf(c, bp.x, a.x), fmaf(c, bp.y, a.y));
        yb = make_float2(fmaf(-c, bp.x, a.x), fmaf(-c, bp.y, a.y));
    } else {
        constexpr float r = c / s;
        const float2 bp = make_float2(fmaf(r, b.x, -b.y), fmaf(r, b.y, b.x));
        ya = make_float2(fmaf(s, bp.x, a.x), fmaf(s, bp.y, a.y));
        yb = make_float2(fmaf(-s, bp.x, a.x), fmaf(-s, bp.y, a.y));
    }
}

template <int K, int SIGN, int LEN, int J>
__device__ __forceinline__ void dit_stage(float2 (&y)[K]) {
    if constexpr (J < LEN / 2) {
        constexpr int JJ = J * (64 / LEN);
#pragma unroll
        for (int b = 0; b < K; b += LEN) {
            if constexpr (JJ % 16 != 0) {
                bfly64<JJ, SIGN>(y[b + J], y[b + J + LEN / 2]);
            } else {
                float2 a = y[b + J];
                float2 t = rot64<JJ, SIGN>(y[b + J + LEN / 2]);
                y[b + J] = cadd(a, t);
                y[b + J + LEN / 2] = csub(a, t);
            }
        }
        dit_stage<K, SIGN, LEN, J + 1>(y);
    }
}

template <int K, int SIGN, int LEN>
__device__ __forceinline__ void dit_stages(float2 (&y)[K]) {
    if constexpr (LEN <= K) {
        dit_stage<K, SIGN, LEN, 0>(y);
        dit_stages<K, SIGN, LEN * 2>(y);
    }
}

// In-place K-point DFT, natural order in and out:
//   x[u] <- sum_j x[j] * exp(SIGN * 2*pi*i * j*u / K),  K in {1,2,...,32}.
template <int K, int SIGN>
__device__ __forceinline__ void fft_reg(float2 (&x)[K]) {
    static_assert(K >= 1 && K <= 32 && (K & (K - 1)) == 0, "K must be a power of two <= 32");
    if constexpr (K > 1) {
        constexpr int LG = ilog2c(K);
        float2 y[K];
#pragma unroll
        for (int i = 0; i < K; i++) y[i] = x[brev(i, LG)];
        dit_stages<K, SIGN, 2>(y);
#pragma unroll
        for (int i = 0; i < K; i++) x[i] = y[i];
    }
}

// Warp-level 1024-point DFT (sign +) with an XOR-swizzled 32 x 32 transpose
// buffer (8 KB): on entry lane l holds x[m] = G[l + 32 m]; on exit lane l
// holds x[h] = Y[l + 32 h]. t2[a * 32 + l] = exp(+2 pi i a l / 1024).
__device__ __forceinline__ void dft1024_warp_xor(float2 (&x)[32], int lane, float2* __restrict__ tb,
                                                 const float2* __restrict__ t2) {
    fft_reg<32, +1>(x);
#pragma unroll
    for (int a = 1; a < 32; a++) x[a] = cmul(x[a], t2[a * 32 + lane]);
#pragma unroll
    for (int a = 0; a < 32; a++) tb[a * 32 + (lane ^ a)] = x[a];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 32; k++) x[k] = tb[lane * 32 + (k ^ lane)];
    __syncwarp();
    fft_reg<32, +1>(x);
}

// w_N^e from the two-level table of a transform length N = 2^log2N:
// tw[0..1023] = w_N^j, tw[1024 + j] = w_N^{1024 j}. SIGN < 0 conjugates.
__device__ __forceinline__ float2 tw_lookup(const float2* __restrict__ tw, int log2N, unsigned e) {
    if (log2N <= 10) return __ldg(tw + (e & ((1u << log2N) - 1)));
    e &= (1u << log2N) - 1;
    return cmul(__ldg(tw + (e & 1023u)), __ldg(tw + 1024 + (e >> 10)));
}

}  // namespace dev
}  // namespace fcwt
