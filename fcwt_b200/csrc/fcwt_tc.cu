// Tensor-core row engine (sm_100a: tcgen05 MMA with tensor-memory operands).
//
// Same transform as the CUDA-core engine (fcwt_kernels.cu): the daughter
// product of the reference (src/fcwt/fcwt.cpp:197-311), the inverse FFT
// (fcwt.cpp:418-429), the normalisation (fcwt.cpp:431-445) and the crop to n
// (fcwt.cpp:396-416). With t = c + M a and q = L + k2 + 1024 k1 (L a multiple
// of 1024, k2 < 1024, k1 < Kp), the four-step inverse transform of a row is
//     G[c][k2]   = w_N^{k2 c} * sum_{k1 < Kp} Z[L + k2 + 1024 k1] * B[k1][c],
//     B[k1][c]   = w_M^{k1 c} * w_N^{L c},
//     y[c + M a] = DFT_1024(G[c][.])[a],
// (w_X = exp(+2 pi i / X), Z = spectrum x daughter weights x 1/N). For rows
// whose window spans at most 16 blocks of 1024 bins, the first line is a
// complex GEMM [1024 k2 x Kp] x [Kp x M] with a short inner dimension; this
// engine runs it on the tensor cores in split FP16 (hi + lo, three products,
// FP32 accumulation: about 2^-21 relative error per element), so phase 1
// costs no FFT work and no scratch round trip through L2.
//
// One persistent CTA of 16 warps per SM takes rows from a queue. Per row:
//   pre-pass  all warps evaluate Z on the window, scale it by 2^e
//             (max |Z| 2^e in [2^14, 2^15)), split it into FP16 hi + lo and
//             store it in tensor memory as the A operand: tile t is lanes
//             0..127 (lane 32 q + l holds k2 = l + 32 (8 q + t)), columns
//             [(2t + p) Kp, +Kp) for p = hi, lo; column k1 holds (re, im) as a
//             half2, i.e. GEMM K index 2 k1 + {0, 1}.
//   groups    the two halves of the CTA (8 warps each) take alternating groups
//             of 8 columns c. Per group: B (16 x 2Kp, K-major, FP16 hi + lo)
//             in SMEM, rows 0..7 giving Re G and rows 8..15 Im G of the 8
//             columns; 24 or 48 MMAs (M=128, N=16, K=16; hi*hi + lo*hi +
//             hi*lo) into the half's accumulator columns, completion signalled
//             on an mbarrier; drain (tcgen05.ld), twiddle w_N^{k2 c} 2^-e, SMEM
//             column tiles; one warp per column runs the 1024-point DFT;
//             swizzled staging and TMA tensor stores of [256 a][8 c] boxes.
//             The MMAs of the half's next group are issued before its DFT.
//             For BF16 / FP16 outputs the column DFTs run on the tensor cores
//             as well (two radix-32 GEMM stages, row_tc_dft).
// Tensor memory: 512 columns per CTA (A: 0..255, accumulators of half h:
// 256 + 128 h + 16 t for tile t).
#include <initializer_list>

#include "fcwt_dev.cuh"

namespace fcwt {
namespace dev {

constexpr int kTcThreads = 512;
constexpr int kTcCols = 8;          // columns per group (one per warp of a half)
static_assert(kTcCols == kGroupCols, "the planner counts tensor-core groups in kGroupCols");
constexpr int kTcTmemCols = 512;
constexpr int kTcDcol = 256;        // first accumulator column
constexpr int kTcTwhiSmem = 512;    // w_M table kept in SMEM when M <= this
constexpr int kTcGbufBytes = kTcCols * kP2 * 8;   // 64 KB: G tiles / output staging of one half
constexpr int kTcOffTwlo = 2 * kTcGbufBytes;
constexpr int kTcOffT2 = kTcOffTwlo + kP2 * 8;
constexpr int kTcOffTwhi = kTcOffT2 + kP2 * 8;
constexpr int kTcOffB = kTcOffTwhi + kTcTwhiSmem * 8;
constexpr int kTcBBytes = 16 * 2 * kTcMaxKp * 2;  // one B operand (16 rows x 2Kp halves), 1 KB
constexpr int kTcOffTg = kTcOffB + 2 * 2 * kTcBBytes;
constexpr int kTcOffW32 = (kTcOffTg + 2 * 32 * 8 + 1023) & ~1023;  // DFT-32 matrix, 128B-swizzled
constexpr int kTcW32Bytes = 64 * 128;
constexpr int kTcOffEnd = kTcOffW32 + kTcW32Bytes;
constexpr size_t kTcSmemBytes = (size_t)kTcOffEnd + 1024;
constexpr int kTcStageBlock = 128 * 128;  // one 128-row block of a DFT-stage operand (16 KB)
static_assert(4 * kBoxBytes == kTcGbufBytes, "staging boxes fill one G buffer");

// Instruction descriptor: D f32, A/B f16, both K-major, N = 16, M = 128.
constexpr uint32_t kTcIdesc = (1u << 4) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle: core matrices of
// 8 rows x 16 bytes; lbo = byte distance between core matrices along K, sbo =
// between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
// DFT stages: D f32, A/B f16, both K-major, N = 64, M = 128.
constexpr uint32_t kTcIdescDft = (1u << 4) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// Byte offset of byte `kb` of row r in a K-major operand with 128-byte rows in
// the 128B-swizzled layout (8-row atoms of 1 KB; 16-byte chunk index XOR row % 8).
__device__ __forceinline__ uint32_t sw128_off(int r, int kb) {
    return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((((kb >> 4) ^ r) & 7) << 4) + (kb & 15));
}
// Shared-memory matrix descriptor of a 128B-swizzled K-major operand (atoms
// 1 KB apart along M/N); K steps of 16 elements advance the address by 32 B.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}
__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// tcgen05.wait::ld with the destination registers of the loads it completes
// as operands, so that no read of them can be placed before the wait.
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
    asm volatile(""
                 : "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* r) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}

// Bounded wait for phase `parity` of an mbarrier (gives up after
// kWaitLimitNs, recording kErrWaitTimeout). Each try_wait may suspend the
// thread until the phase completes, for at most kTrySuspendNs, so that waiting
// warps do not take issue slots from the working ones.
constexpr uint32_t kTrySuspendNs = 20000;
__device__ bool mbar_wait(uint32_t mbar, uint32_t parity, int* err) {
    unsigned long long t0 = 0;
    for (unsigned it = 0;; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity), "r"(kTrySuspendNs)
            : "memory");
        if (done) return true;
        if (it == 0) {
            t0 = global_ns();
        } else if ((it & 7u) == 0 && global_ns() - t0 > kWaitLimitNs) {
            atomicOr(err, kErrWaitTimeout);
            return false;
        }
    }
}

__device__ __forceinline__ void half_bar(int h) { asm volatile("bar.sync %0, 256;" ::"r"(1 + h) : "memory"); }

__device__ __forceinline__ uint32_t h2bits(__half2 v) { return *reinterpret_cast<uint32_t*>(&v); }

// B operand of group g: rows j (Re G) and 8 + j (Im G) of column c = 8 g + j,
// K index 2 k1 + {re, im}; byte offset of element (n, k) in the canonical
// K-major layout: (k / 16) * 512 + (n / 8) * 256 + ((k / 8) % 2) * 128 +
// (n % 8) * 16 + (k % 8) * 2.
// With time decimation D the group's columns are c = D (8 g + j).
template <int KP, bool LO = true>
__device__ __forceinline__ void build_b(float2* __restrict__ tg, int g, int ht, int M, unsigned Nm, int L, const float2* __restrict__ twlo,
                                        const float2* __restrict__ twhi, unsigned char* bhi, unsigned char* blo,
                                        int D = 1) {
    if (ht >= 224) tg[ht - 224] = tw_n(twlo, twhi, ((unsigned)(ht - 224) * (unsigned)(D * g * kTcCols)) & Nm);
    if (ht < kTcCols * KP) {
        const int j = ht / KP;
        const int k1 = ht - j * KP;
        const int c = D * (g * kTcCols + j);
        const float2 w = cmul(twhi[(unsigned)(k1 * c) & (unsigned)(M - 1)],
                              tw_n(twlo, twhi, ((unsigned)L * (unsigned)c) & Nm));
        const int k = 2 * k1;
        const int off0 = (k >> 4) * 512 + ((k >> 3) & 1) * 128 + j * 16 + (k & 7) * 2;  // row j
        const int off1 = off0 + 256;                                                     // row 8 + j
        const __half2 h0 = __floats2half2_rn(w.x, -w.y);
        const __half2 h1 = __floats2half2_rn(w.y, w.x);
        [[maybe_unused]] const float2 f0 = __half22float2(h0);
        [[maybe_unused]] const float2 f1 = __half22float2(h1);
        *reinterpret_cast<__half2*>(bhi + off0) = h0;
        *reinterpret_cast<__half2*>(bhi + off1) = h1;
        if constexpr (LO) {
            *reinterpret_cast<__half2*>(blo + off0) = __floats2half2_rn(w.x - f0.x, -w.y - f0.y);
            *reinterpret_cast<__half2*>(blo + off1) = __floats2half2_rn(w.y - f1.x, w.x - f1.y);
        }
    }
}

// The MMAs of one group: for each k2 tile, D = A_hi B_hi + A_lo B_hi + A_hi B_lo
// (LO) or D = A_hi B_hi.
template <int KP, bool LO = true>
__device__ __forceinline__ void issue_group(int t, uint32_t tmem, uint32_t dcol, uint32_t bhi, uint32_t blo) {
    {
        const uint32_t d = dcol + 16u * t;
#pragma unroll
        for (int p = 0; p < (LO ? 3 : 1); p++) {
            const uint32_t a = tmem + (uint32_t)((2 * t + (p == 1 ? 1 : 0)) * KP);
            const uint32_t b = p == 2 ? blo : bhi;
#pragma unroll
            for (int kb = 0; kb < KP / 8; kb++)
                mma_ts(d, a + 8u * kb, umma_desc(b + 512u * kb, 128, 256), (p | kb) != 0 ? 1u : 0u);
        }
    }
}

// Runtime switch between the two window widths (8 or 16 blocks): only the
// B operand, the MMA issue and the pre-pass depend on it, so the group loop
// of a row is compiled once (half the instruction footprint of the hot loop).
template <bool LO>
__device__ __forceinline__ void build_b_kp(bool kp16, float2* __restrict__ tg, int g, int ht, int M, unsigned Nm,
                                           int L, const float2* __restrict__ twlo, const float2* __restrict__ twhi,
                                           unsigned char* bhi, unsigned char* blo, int D) {
    if (kp16)
        build_b<16, LO>(tg, g, ht, M, Nm, L, twlo, twhi, bhi, blo, D);
    else
        build_b<8, LO>(tg, g, ht, M, Nm, L, twlo, twhi, bhi, blo, D);
}
template <bool LO>
__device__ __forceinline__ void issue_group_kp(bool kp16, int t, uint32_t tmem, uint32_t dcol, uint32_t bhi,
                                               uint32_t blo) {
    if (kp16)
        issue_group<16, LO>(t, tmem, dcol, bhi, blo);
    else
        issue_group<8, LO>(t, tmem, dcol, bhi, blo);
}

// Pre-pass of a row: Z on the window, scaled by 2^e (max |Z| 2^e in
// [2^14, 2^15)) and split into FP16 hi + lo, into tensor memory as the A
// operand (tile t, lane 32 q + l holds k2 = l + 32 (8 q + t)). Returns 2^-e.
// Without LO only the hi part is stored.
template <int KP, bool LO = true>
__device__ __forceinline__ float tc_prepass(const TcParams& P, const RowDesc& R, const SigDesc& S, uint32_t tmem,
                                            float* s_red) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int qd = warp & 3;
    const uint32_t lane_base = (uint32_t)(32 * qd) << 16;
    const float* __restrict__ wrow = P.wts + R.woff;
    const int tsel = warp >> 2;  // this warp's tiles: tsel, tsel + 4
    float2 z[2][KP];
    float mx = 0.0f;
#pragma unroll
    for (int ti = 0; ti < 2; ti++) {
        const int k2 = lane + 32 * (8 * qd + tsel + 4 * ti);
#pragma unroll
        for (int k1 = 0; k1 < KP; k1++) {
            const int q = R.L + k2 + kP2 * k1;
            const float m = __ldg(wrow + k2 + kP2 * k1);
            const float2 xv = (q >= R.lo && q < R.hi) ? __ldg(S.X + q) : make_float2(0.0f, 0.0f);
            const float2 v = R.imag ? make_float2(-xv.y * m, xv.x * m) : make_float2(xv.x * m, xv.y * m);
            z[ti][k1] = v;
            mx = fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y)));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) s_red[warp] = mx;
    __syncthreads();
    mx = 0.0f;
#pragma unroll
    for (int w = 0; w < kTcThreads / 32; w++) mx = fmaxf(mx, s_red[w]);
    int ex = 0;
    if (mx > 0.0f) frexpf(mx, &ex);
    const int e2 = max(-126, min(126, 15 - ex));
    const float scale = ldexpf(1.0f, e2);
#pragma unroll
    for (int ti = 0; ti < 2; ti++) {
        const int t = tsel + 4 * ti;
        uint32_t hv[KP], lv[KP];
#pragma unroll
        for (int k1 = 0; k1 < KP; k1++) {
            const float a = z[ti][k1].x * scale;
            const float b = z[ti][k1].y * scale;
            const __half2 hh = __floats2half2_rn(a, b);
            hv[k1] = h2bits(hh);
            if constexpr (LO) {
                const float2 hf = __half22float2(hh);
                lv[k1] = h2bits(__floats2half2_rn(a - hf.x, b - hf.y));
            }
        }
        const uint32_t ta = tmem + lane_base + (uint32_t)(2 * t * KP);
#pragma unroll
        for (int q = 0; q < KP / 8; q++) {
            tmem_st8(ta + 8u * q, hv + 8 * q);
            if constexpr (LO) tmem_st8(ta + KP + 8u * q, lv + 8 * q);
        }
    }
    tmem_wait_st();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return ldexpf(1.0f, -e2);
}

// Claims the CTA's next row from the queue into the other row slot and pulls
// its weights and spectrum window into L2.
__device__ __forceinline__ void tc_claim_next(const TcParams& P, int* next_idx, RowDesc* next_R, SigDesc* next_S,
                                              int* next_unit) {
    const int i = (int)atomicAdd(P.counter, 1u);
    *next_idx = i;
    if (i < P.n_list) {
        const int e = P.row_list[i];
        *next_unit = e;
        *next_R = P.rows[e & kUnitRowMask];
        *next_S = P.sigs[next_R->sig];
        const unsigned wb = (unsigned)(kP2 * next_R->kp) * 4u;
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(P.wts + next_R->woff), "r"(wb) : "memory");
        const int Nn = 1 << next_S->log2N;
        const int xe = min(kP2 * next_R->kp, Nn - next_R->L);
        if (xe > 0)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(next_S->X + next_R->L),
                         "r"((unsigned)xe * 8u) : "memory");
    }
}

template <int OT, bool DEC>
__device__ __forceinline__ void row_tc(const TcParams& P, const CUtensorMap* omap, const RowDesc& R,
                                       const SigDesc& S, unsigned char* sm, const float2* __restrict__ twlo,
                                       const float2* __restrict__ twhi, const float2* __restrict__ t2, uint32_t tmem,
                                       uint32_t mbar_h, uint32_t& phase, float* s_red, int* next_idx,
                                       RowDesc* next_R, SigDesc* next_S, int* next_unit, int unit, bool kp16) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int h = warp >> 3;
    const int ht = tid & 255;
    const int wl = warp & 7;
    const int qd = warp & 3;
    const int log2N = S.log2N;
    const int N = 1 << log2N;
    const int M = N >> kLog2P2;
    const unsigned Nm = (unsigned)N - 1u;
    const int D = DEC ? R.dec : 1;  // time decimation: column c = D c', output sample t' = c' + Mo a
    const int Mo = M / D;
    const int n = R.n_out;     // output samples of the row
    const uint32_t lane_base = (uint32_t)(32 * qd) << 16;

    const float inv = (kp16 ? tc_prepass<16>(P, R, S, tmem, s_red) : tc_prepass<8>(P, R, S, tmem, s_red));

    // ---- column groups
    const int ng = Mo / kTcCols;
    int gb, ge;  // this unit's column groups [gb, ge)
    tc_unit_groups(unit, ng, &gb, &ge);
    float2* gbuf = reinterpret_cast<float2*>(sm + h * kTcGbufBytes);
    unsigned char* bhi = sm + kTcOffB + h * 2 * kTcBBytes;
    unsigned char* blo = bhi + kTcBBytes;
    float2* tg = reinterpret_cast<float2*>(sm + kTcOffTg) + 32 * h;
    const uint32_t bhi_a = smem_u32(bhi), blo_a = smem_u32(blo);
    const uint32_t dcol = tmem + (uint32_t)(kTcDcol + 128 * h);
    // the tensor map of this row's output buffer: the launch's map (buffer 0) or, for
    // many outputs, the buffer's own map in global memory
    const CUtensorMap* map = P.tmaps ? P.tmaps + R.out_buf : omap;
    const bool tma = P.tma_store != 0 &&
                     (P.tmaps ? ((P.tmap_mask[R.out_buf >> 6] >> (R.out_buf & 63)) & 1ull) != 0 : R.out_buf == 0);
    if (P.tmaps && tma) tensormap_acquire(map);
    void* outb = P.outs[R.out_buf];
    int g = gb + h;
    if (g < ge) {
        build_b_kp<true>(kp16, tg, g, ht, M, Nm, R.L, twlo, twhi, bhi, blo, D);
        fence_proxy_async_smem();
        half_bar(h);
        if (lane == 0) {
            tc_fence_after();
            issue_group_kp<true>(kp16, wl, tmem, dcol, bhi_a, blo_a);
            mma_commit(mbar_h);
        }
    }
    const int tb = (wl >> 2) * 4;  // this warp drains tiles tb .. tb + 3
    const int amax = (n + Mo - 1) / Mo;  // stripes a that hold output samples
    // the halves run the same per-group sequence; starting half 1 a little later
    // keeps their DFT (issue-bound) and staging/store (SMEM-bound) phases apart
    if (h == 1 && wl == 7 && lane == 0) tc_claim_next(P, next_idx, next_R, next_S, next_unit);
    while (g < ge) {
        mbar_wait(mbar_h, phase, P.err);
        phase ^= 1u;
        tc_fence_after();
        const int c0 = g * kTcCols;  // first output column c' of the group (column D c0 of the row)
        float2 gv[4][kTcCols];
#pragma unroll
        for (int tt = 0; tt < 4; tt++) {
            uint32_t r[16];
            tmem_ld16(dcol + lane_base + 16u * (tb + tt), r);
            tmem_wait_ld(r);
            const int k2 = lane + 32 * (8 * qd + tb + tt);
            float2 w = cmul(tw_n(twlo, twhi, ((unsigned)(k2 - lane) * (unsigned)(D * c0)) & Nm), cscale(tg[lane], inv));
            const float2 stp = DEC ? tw_n(twlo, twhi, ((unsigned)k2 * (unsigned)D) & Nm) : twlo[k2];
#pragma unroll
            for (int j = 0; j < kTcCols; j++) {
                gv[tt][j] = cmul(make_float2(__uint_as_float(r[j]), __uint_as_float(r[8 + j])), w);
                if (j + 1 < kTcCols) w = cmul(w, stp);
            }
        }
        tc_fence_before();
        if (tma && lane == 0 && wl >= 4) bulk_wait_read_all();
        half_bar(h);  // accumulators drained; the G buffer is free
        const int gn = g + 2;
        if (gn < ge) build_b_kp<true>(kp16, tg, gn, ht, M, Nm, R.L, twlo, twhi, bhi, blo, D);
#pragma unroll
        for (int tt = 0; tt < 4; tt++) {
            const int k2 = lane + 32 * (8 * qd + tb + tt);
#pragma unroll
            for (int j = 0; j < kTcCols; j++) gbuf[j * kP2 + k2] = gv[tt][j];
        }
        fence_proxy_async_smem();
        half_bar(h);  // G tiles and the next B in SMEM
        if (lane == 0 && gn < ge) {
            tc_fence_after();
            issue_group_kp<true>(kp16, wl, tmem, dcol, bhi_a, blo_a);
            mma_commit(mbar_h);
        }
        // phase 2: one column per warp
        float2* col = gbuf + wl * kP2;
        float2 x[32];
#pragma unroll
        for (int m = 0; m < 32; m++) x[m] = col[lane + 32 * m];
        __syncwarp();
        dft1024_warp_xor(x, lane, col, t2);
        half_bar(h);  // every column is in registers
        unsigned char* stage = reinterpret_cast<unsigned char*>(gbuf);
        if constexpr (OT == OUT_C64) {
#pragma unroll
            for (int hh = 0; hh < 32; hh++)
                if (lane + 32 * hh < amax) *reinterpret_cast<float2*>(stage + stage_off(lane + 32 * hh, wl)) = x[hh];
        } else {
#pragma unroll
            for (int hh = 0; hh < 32; hh++)
                if (lane + 32 * hh < amax)
                    *reinterpret_cast<unsigned*>(stage + stage16_off(lane + 32 * hh, wl)) = pack16<OT>(x[hh]);
        }
        const long long row0 = R.out_off + c0;
        constexpr int box_bytes = OT == OUT_C64 ? kBoxBytes : kBoxBytes / 2;
        if (tma) {
            fence_proxy_async_smem();
            half_bar(h);
            const int n_full = n / Mo;
            if (lane == 0 && wl >= 4) {
                const int j = wl - 4;
                // complex64 output lines evict-first in L2 (measured ~1% faster; slower for 4-byte types)
                if (j * kBoxRows < n_full)
                    tma_store_3d<OT == OUT_C64>(map, stage + j * box_bytes, c0, j * kBoxRows, R.out_row);
                bulk_commit();
            }
            const int tail = n - n_full * Mo;
            if (ht < kTcCols && c0 + ht < tail && n_full < kP2) {
                const long long idx = row0 + ht + (long long)Mo * n_full;
                if constexpr (OT == OUT_C64)
                    store_out<OT>(outb, idx, *reinterpret_cast<const float2*>(stage + stage_off(n_full, ht)));
                else
                    __stcs(reinterpret_cast<unsigned*>(outb) + idx,
                           *reinterpret_cast<const unsigned*>(stage + stage16_off(n_full, ht)));
            }
        } else {
            half_bar(h);
            for (int idx = ht; idx < kTcCols * kP2; idx += 256) {
                const int w = idx & (kTcCols - 1);
                const int a = idx >> 3;
                if (c0 + w + (long long)Mo * a < n) {
                    const long long o = row0 + w + (long long)Mo * a;
                    if constexpr (OT == OUT_C64)
                        store_out<OT>(outb, o, *reinterpret_cast<const float2*>(stage + stage_off(a, w)));
                    else
                        __stcs(reinterpret_cast<unsigned*>(outb) + o,
                               *reinterpret_cast<const unsigned*>(stage + stage16_off(a, w)));
                }
            }
        }
        g = gn;
    }
}

// The 16-bit outputs (BF16 / FP16 pairs) also run the column DFTs on the
// tensor cores. With k2 = kl + 32 kb and a = a1 + 32 a2,
//     H[c][kl][a1]     = sum_kb G[c][kl + 32 kb] w_32^{a1 kb}                 (stage 1)
//     y[c + M (a1 + 32 a2)] = sum_kl H[c][kl][a1] w_1024^{a1 kl} w_32^{a2 kl}  (stage 2)
// Each stage is a real GEMM [256 x 64] x [64 x 64] (complex values as
// (re, im) pairs, FP16 operands, FP32 accumulation) against the DFT-32
// matrix W / 32 in SMEM, both operands K-major and 128B-swizzled. The scale
// factors are fixed powers of two: |G| / Kp <= 2^15.5 and a stage cannot grow
// the largest value (the 1/32 in W), so no FP16 operand overflows; the output
// scale 2^-e Kp 1024 is applied once at the end. Row orders: stage 1, block
// c / 4, row 32 (c % 4) + kl (each thread writes 16-byte pieces of four kb);
// stage 2, block a1 / 16, row 8 (a1 % 16) + c, so that a warp's stage-2
// accumulators are [4 a][8 c] tiles of the output staging. Both stages reuse
// the half's 128 accumulator columns; the phase-1 MMAs of the half's next group
// are issued once the stage-2 results are in registers. Phase 1 runs in plain
// FP16 here (Z and B rounded once, about 2^-12 relative per element), a third
// of the split-FP16 MMAs: the 16-bit output rounding dominates the error.
__device__ __forceinline__ void issue_dft_stage(uint32_t d, uint32_t a, uint32_t w) {
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int kb = 0; kb < 4; kb++)
            mma_ss(d + 64u * m, umma_desc_sw128(a + (uint32_t)(kTcStageBlock * m) + 32u * kb),
                   umma_desc_sw128(w + 32u * kb), kTcIdescDft, kb != 0 ? 1u : 0u);
}

template <int OT, bool DEC>
__device__ __forceinline__ void row_tc_dft(const TcParams& P, const CUtensorMap* omap, const RowDesc& R,
                                           const SigDesc& S, unsigned char* sm, const float2* __restrict__ twlo,
                                           const float2* __restrict__ twhi, const float2* __restrict__ t2,
                                           uint32_t tmem, uint32_t mbar_h, uint32_t& phase, uint32_t mbar2_h,
                                           uint32_t& phase2, float* s_red, int* next_idx, RowDesc* next_R,
                                           SigDesc* next_S, int* next_unit, int unit, bool kp16) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int h = warp >> 3;
    const int ht = tid & 255;
    const int wl = warp & 7;
    const int qd = warp & 3;
    const int log2N = S.log2N;
    const int N = 1 << log2N;
    const int M = N >> kLog2P2;
    const unsigned Nm = (unsigned)N - 1u;
    const int D = DEC ? R.dec : 1;  // time decimation: column c = D c', output sample t' = c' + Mo a
    const int Mo = M / D;
    const int n = R.n_out;     // output samples of the row
    const uint32_t lane_base = (uint32_t)(32 * qd) << 16;

    const float inv = (kp16 ? tc_prepass<16, false>(P, R, S, tmem, s_red) : tc_prepass<8, false>(P, R, S, tmem, s_red));
    const float s1 = kp16 ? 1.0f / 16.0f : 1.0f / 8.0f;
    const float fin = inv * (float)((kp16 ? 16 : 8) * 1024);

    const int ng = Mo / kTcCols;
    int gb, ge;  // this unit's column groups [gb, ge)
    tc_unit_groups(unit, ng, &gb, &ge);
    unsigned char* abuf = sm + h * kTcGbufBytes;        // DFT-stage A operand, 32 KB
    unsigned char* stage = abuf + kTcGbufBytes / 2;     // output staging, 32 KB
    unsigned char* bhi = sm + kTcOffB + h * 2 * kTcBBytes;
    unsigned char* blo = bhi + kTcBBytes;
    float2* tg = reinterpret_cast<float2*>(sm + kTcOffTg) + 32 * h;
    const uint32_t bhi_a = smem_u32(bhi), blo_a = smem_u32(blo);
    const uint32_t abuf_a = smem_u32(abuf), w32_a = smem_u32(sm + kTcOffW32);
    const uint32_t dcol = tmem + (uint32_t)(kTcDcol + 128 * h);
    const CUtensorMap* map = P.tmaps ? P.tmaps + R.out_buf : omap;
    const bool tma = P.tma_store != 0 &&
                     (P.tmaps ? ((P.tmap_mask[R.out_buf >> 6] >> (R.out_buf & 63)) & 1ull) != 0 : R.out_buf == 0);
    if (P.tmaps && tma) tensormap_acquire(map);
    void* outb = P.outs[R.out_buf];
    int g = gb + h;
    if (g < ge) {
        build_b_kp<false>(kp16, tg, g, ht, M, Nm, R.L, twlo, twhi, bhi, blo, D);
        fence_proxy_async_smem();
        half_bar(h);
        if (lane == 0) {
            tc_fence_after();
            issue_group_kp<false>(kp16, wl, tmem, dcol, bhi_a, blo_a);
            mma_commit(mbar_h);
        }
    }
    const int tb = (wl >> 2) * 4;      // this warp drains phase-1 tiles tb .. tb + 3
    const int amax = (n + Mo - 1) / Mo;  // stripes a that hold output samples
    // stage-1 operand: this thread's rows 32 (j % 4) + lane of block j / 4, bytes 4 kb for kb = 8 qd + tb + 0..3
    const uint32_t a1_off = (uint32_t)((lane >> 3) * 1024 + (lane & 7) * 128 + ((((2 * qd + (tb >> 2)) ^ lane) & 7) << 4));
    // stage-2 operand: row 8 (a1 % 16) + wl of block a1 / 16, bytes 4 lane
    const uint32_t a2_off = (uint32_t)(wl * 128 + ((((lane >> 2) ^ wl) & 7) << 4) + (lane & 3) * 4);
    // stage-2 accumulators of this thread: a1 = 16 (wl / 4) + 4 qd + lane / 8, column c = lane % 8
    const int my_a1 = 16 * (wl >> 2) + 4 * qd + (lane >> 3);
    const int my_c = lane & 7;
    unsigned char* my_stage = stage + stage16_off(my_a1, my_c);
    const uint32_t dsrc = dcol + lane_base + 64u * (uint32_t)(wl >> 2);
    if (h == 1 && wl == 7 && lane == 0) tc_claim_next(P, next_idx, next_R, next_S, next_unit);
    while (g < ge) {
        mbar_wait(mbar_h, phase, P.err);
        phase ^= 1u;
        tc_fence_after();
        const int c0 = g * kTcCols;  // first output column c' of the group (column D c0 of the row)
        {
            uint32_t pk[kTcCols][4];
#pragma unroll
            for (int tt = 0; tt < 4; tt++) {
                uint32_t r[16];
                tmem_ld16(dcol + lane_base + 16u * (tb + tt), r);
                tmem_wait_ld(r);
                const int k2 = lane + 32 * (8 * qd + tb + tt);
                float2 w = cmul(tw_n(twlo, twhi, ((unsigned)(k2 - lane) * (unsigned)(D * c0)) & Nm), cscale(tg[lane], s1));
                const float2 stp = DEC ? tw_n(twlo, twhi, ((unsigned)k2 * (unsigned)D) & Nm) : twlo[k2];
#pragma unroll
                for (int j = 0; j < kTcCols; j++) {
                    const float2 v = cmul(make_float2(__uint_as_float(r[j]), __uint_as_float(r[8 + j])), w);
                    pk[j][tt] = h2bits(__floats2half2_rn(v.x, v.y));
                    if (j + 1 < kTcCols) w = cmul(w, stp);
                }
            }
#pragma unroll
            for (int j = 0; j < kTcCols; j++)
                *reinterpret_cast<uint4*>(abuf + (j >> 2) * kTcStageBlock + (j & 3) * 4096 + a1_off) =
                    make_uint4(pk[j][0], pk[j][1], pk[j][2], pk[j][3]);
        }
        tc_fence_before();
        fence_proxy_async_smem();
        half_bar(h);  // phase-1 accumulators drained; stage-1 operand in SMEM
        if (wl == 0 && lane == 0) {
            tc_fence_after();
            issue_dft_stage(dcol, abuf_a, w32_a);
            mma_commit(mbar2_h);
        }
        const int gn = g + 2;
        if (gn < ge) {
            build_b_kp<false>(kp16, tg, gn, ht, M, Nm, R.L, twlo, twhi, bhi, blo, D);
            fence_proxy_async_smem();
        }
        mbar_wait(mbar2_h, phase2, P.err);
        phase2 ^= 1u;
        tc_fence_after();
        // stage-1 results of column c = wl, kl = lane: twiddle, stage-2 operand
#pragma unroll
        for (int q2 = 0; q2 < 2; q2++) {
            uint32_t r[32];
            tmem_ld16(dsrc + 32u * q2, *reinterpret_cast<uint32_t(*)[16]>(r));
            tmem_ld16(dsrc + 32u * q2 + 16u, *reinterpret_cast<uint32_t(*)[16]>(r + 16));
            tmem_wait_ld(r);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int a1 = 16 * q2 + i;
                const float2 v = cmul(make_float2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1])),
                                      t2[a1 * 32 + lane]);
                *reinterpret_cast<uint32_t*>(abuf + (a1 >> 4) * kTcStageBlock + (a1 & 15) * 1024 + a2_off) =
                    h2bits(__floats2half2_rn(v.x, v.y));
            }
        }
        tc_fence_before();
        fence_proxy_async_smem();
        half_bar(h);  // stage-1 accumulators drained; stage-2 operand in SMEM
        if (wl == 0 && lane == 0) {
            tc_fence_after();
            issue_dft_stage(dcol, abuf_a, w32_a);
            mma_commit(mbar2_h);
        }
        mbar_wait(mbar2_h, phase2, P.err);
        phase2 ^= 1u;
        tc_fence_after();
        uint32_t yv[32];
#pragma unroll
        for (int q2 = 0; q2 < 2; q2++) {
            uint32_t r[32];
            tmem_ld16(dsrc + 32u * q2, *reinterpret_cast<uint32_t(*)[16]>(r));
            tmem_ld16(dsrc + 32u * q2 + 16u, *reinterpret_cast<uint32_t(*)[16]>(r + 16));
            tmem_wait_ld(r);
#pragma unroll
            for (int i = 0; i < 16; i++)
                yv[16 * q2 + i] = pack16<OT>(
                    make_float2(__uint_as_float(r[2 * i]) * fin, __uint_as_float(r[2 * i + 1]) * fin));
        }
        tc_fence_before();
        if (tma && lane == 0 && wl >= 4) bulk_wait_read_all();
        half_bar(h);  // accumulators free for the next group; staging free
        if (lane == 0 && gn < ge) {
            tc_fence_after();
            issue_group_kp<false>(kp16, wl, tmem, dcol, bhi_a, blo_a);
            mma_commit(mbar_h);
        }
        // a = my_a1 + 32 a2 with my_a1 < 32: box a2 / 8, box row my_a1 + 32 (a2 % 8), same swizzle bit
#pragma unroll
        for (int a2 = 0; a2 < 32; a2++)
            if (my_a1 + 32 * a2 < amax)
                *reinterpret_cast<unsigned*>(my_stage + (a2 >> 3) * (kBoxBytes / 2) + (a2 & 7) * 1024) = yv[a2];
        const long long row0 = R.out_off + c0;
        constexpr int box_bytes = kBoxBytes / 2;
        if (tma) {
            fence_proxy_async_smem();
            half_bar(h);
            const int n_full = n / Mo;
            if (lane == 0 && wl >= 4) {
                const int j = wl - 4;
                if (j * kBoxRows < n_full) tma_store_3d(map, stage + j * box_bytes, c0, j * kBoxRows, R.out_row);
                bulk_commit();
            }
            const int tail = n - n_full * Mo;
            if (ht < kTcCols && c0 + ht < tail && n_full < kP2) {
                const long long idx = row0 + ht + (long long)Mo * n_full;
                __stcs(reinterpret_cast<unsigned*>(outb) + idx,
                       *reinterpret_cast<const unsigned*>(stage + stage16_off(n_full, ht)));
            }
        } else {
            half_bar(h);
            for (int idx = ht; idx < kTcCols * kP2; idx += 256) {
                const int w = idx & (kTcCols - 1);
                const int a = idx >> 3;
                if (c0 + w + (long long)Mo * a < n) {
                    const long long o = row0 + w + (long long)Mo * a;
                    __stcs(reinterpret_cast<unsigned*>(outb) + o,
                           *reinterpret_cast<const unsigned*>(stage + stage16_off(a, w)));
                }
            }
        }
        g = gn;
    }
}

// DEC: the launch holds time-decimated rows (RowDesc::dec > 1); without it the
// decimation arithmetic is compiled out.
template <int OT, bool DEC = false>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_row_tc(const __grid_constant__ TcParams P, const __grid_constant__ CUtensorMap omap) {
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    unsigned char* sm = tc_smem_raw + ((1024u - (smem_u32(tc_smem_raw) & 1023u)) & 1023u);
    float2* twlo = reinterpret_cast<float2*>(sm + kTcOffTwlo);
    float2* t2 = reinterpret_cast<float2*>(sm + kTcOffT2);
    float2* twhi_s = reinterpret_cast<float2*>(sm + kTcOffTwhi);
    // Completion of the phase-1 MMAs of half h. The 16-bit outputs use one
    // barrier per tile half p (tiles 4 p .. 4 p + 3, issued and drained by warps
    // 4 p .. 4 p + 3 of the half), so that a warp waits only for the tiles it
    // drains: 4% faster for BF16; complex64 measured 0.2% slower with it and
    // keeps one barrier per half.
    constexpr bool kSplitP1 = OT == OUT_BF16 || OT == OUT_F16;
    __shared__ __align__(8) unsigned long long s_mbar[4];
    __shared__ __align__(8) unsigned long long s_mbar2[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_idx[2];
    __shared__ int s_unit[2];
    __shared__ int s_log2N;
    __shared__ RowDesc s_R[2];
    __shared__ SigDesc s_S[2];
    __shared__ float s_red[kTcThreads / 32];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int h = warp >> 3;

    for (int j = tid; j < kP2; j += kTcThreads) {
        const int a = j >> 5, l = j & 31;
        double s, c;
        sincospi(2.0 * (double)((a * l) & 1023) / 1024.0, &s, &c);
        t2[j] = make_float2((float)c, (float)s);
    }
    if constexpr (OT == OUT_BF16 || OT == OUT_F16) {
        // W / 32 for the DFT stages: row n = 2 a + {re, im}, K index 2 k + {re, im}
        unsigned char* w32 = sm + kTcOffW32;
        for (int j = tid; j < 64 * 64; j += kTcThreads) {
            const int nr = j >> 6, k = j & 63;
            double s, c;
            sincospi((double)(((nr >> 1) * (k >> 1)) & 31) / 16.0, &s, &c);
            const float cv = (float)c * (1.0f / 32.0f), sv = (float)s * (1.0f / 32.0f);
            const float v = (nr & 1) == 0 ? ((k & 1) == 0 ? cv : -sv) : ((k & 1) == 0 ? sv : cv);
            *reinterpret_cast<__half*>(w32 + sw128_off(nr, 2 * k)) = __float2half_rn(v);
        }
        fence_proxy_async_smem();
    }
    if (tid == 0) {
        for (int k = 0; k < 4; k++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_mbar[k])), "r"(kSplitP1 ? 4 : 8));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar2[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar2[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_log2N = -1;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t mbar_h = smem_u32(&s_mbar[kSplitP1 ? 2 * h + ((warp & 7) >> 2) : h]);
    const uint32_t mbar2_h = smem_u32(&s_mbar2[h]);
    uint32_t phase = 0, phase2 = 0;

    if (tid == 0) {
        const int i = (int)atomicAdd(P.counter, 1u);
        s_idx[0] = i;
        if (i < P.n_list) {
            s_unit[0] = P.row_list[i];
            s_R[0] = P.rows[s_unit[0] & kUnitRowMask];
            s_S[0] = P.sigs[s_R[0].sig];
        }
    }
    __syncthreads();
    int sl = 0;
    for (;;) {
        if (s_idx[sl] >= P.n_list) break;
        const RowDesc& R = s_R[sl];
        const SigDesc& S = s_S[sl];
        const int log2N = S.log2N;
        const int M = 1 << (log2N - kLog2P2);
        if (log2N != s_log2N) {
            for (int j = tid; j < kP2; j += kTcThreads) twlo[j] = S.tw[j];
            if (M <= kTcTwhiSmem)
                for (int j = tid; j < M; j += kTcThreads) twhi_s[j] = S.tw[kP2 + j];
        }
        __syncthreads();
        if (tid == 0) s_log2N = log2N;
        const float2* twhi = M <= kTcTwhiSmem ? twhi_s : S.tw + kP2;
        if constexpr (OT == OUT_BF16 || OT == OUT_F16) {
            row_tc_dft<OT, DEC>(P, &omap, R, S, sm, twlo, twhi, t2, tmem, mbar_h, phase, mbar2_h, phase2, s_red,
                                &s_idx[sl ^ 1], &s_R[sl ^ 1], &s_S[sl ^ 1], &s_unit[sl ^ 1], s_unit[sl], R.kp > 8);
        } else {
            row_tc<OT, DEC>(P, &omap, R, S, sm, twlo, twhi, t2, tmem, mbar_h, phase, s_red, &s_idx[sl ^ 1],
                            &s_R[sl ^ 1], &s_S[sl ^ 1], &s_unit[sl ^ 1], s_unit[sl], R.kp > 8);
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        sl ^= 1;
    }
    if ((tid & 31) == 0 && ((tid >> 5) & 7) >= 4 && P.tma_store) bulk_wait_all();
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
}

// Plan-time weight table of the tensor-core rows: wts[woff + i] = daughter
// weight of bin q = L + i times out_scale (0 outside [lo, hi)), the same
// float product the engines apply per bin, so that the per-row pre-pass reads
// it with coalesced loads instead of gathering the mother table.
__global__ void k_tc_weights(const SigDesc* __restrict__ sigs, const RowDesc* __restrict__ rows,
                             const int* __restrict__ row_list, const float* __restrict__ pool,
                             float* __restrict__ wts) {
    const RowDesc R = rows[row_list[blockIdx.x]];
    const SigDesc S = sigs[R.sig];
    const float nm1 = (float)(1 << S.log2N) - 1.0f;
    const int len = kP2 * R.kp;
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
        const int q = R.L + i;
        wts[R.woff + i] = (q >= R.lo && q < R.hi) ? bin_weight(R, S.mother, pool, nm1, q) * R.out_scale : 0.0f;
    }
}

}  // namespace dev

cudaError_t launch_tc_weights(const SigDesc* sigs, const RowDesc* rows, const int* row_list, int n_list,
                              const float* pool, float* wts, cudaStream_t st) {
    if (n_list <= 0) return cudaSuccess;
    dev::k_tc_weights<<<n_list, 256, 0, st>>>(sigs, rows, row_list, pool, wts);
    return cudaGetLastError();
}

size_t tc_smem_bytes() { return dev::kTcSmemBytes; }

template <int OT, bool DEC>
cudaError_t tc_configure_one() {
    return cudaFuncSetAttribute(dev::k_row_tc<OT, DEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dev::kTcSmemBytes);
}

cudaError_t tc_configure() {
    cudaError_t e = cudaSuccess;
    for (cudaError_t r : {tc_configure_one<OUT_C64, false>(), tc_configure_one<OUT_C64, true>(),
                          tc_configure_one<OUT_BF16, false>(), tc_configure_one<OUT_BF16, true>(),
                          tc_configure_one<OUT_F16, false>(), tc_configure_one<OUT_F16, true>(),
                          tc_configure_one<OUT_POWER, false>(), tc_configure_one<OUT_POWER, true>(),
                          tc_configure_one<OUT_DB, false>(), tc_configure_one<OUT_DB, true>()})
        if (r != cudaSuccess && e == cudaSuccess) e = r;
    return e;
}

template <bool DEC>
void launch_tc_dec(const TcParams& p, const CUtensorMap& omap, int out_type, int grid, cudaStream_t st) {
    switch (out_type) {
        case OUT_BF16: dev::k_row_tc<OUT_BF16, DEC><<<grid, dev::kTcThreads, dev::kTcSmemBytes, st>>>(p, omap); break;
        case OUT_F16: dev::k_row_tc<OUT_F16, DEC><<<grid, dev::kTcThreads, dev::kTcSmemBytes, st>>>(p, omap); break;
        case OUT_POWER: dev::k_row_tc<OUT_POWER, DEC><<<grid, dev::kTcThreads, dev::kTcSmemBytes, st>>>(p, omap); break;
        case OUT_DB: dev::k_row_tc<OUT_DB, DEC><<<grid, dev::kTcThreads, dev::kTcSmemBytes, st>>>(p, omap); break;
        default: dev::k_row_tc<OUT_C64, DEC><<<grid, dev::kTcThreads, dev::kTcSmemBytes, st>>>(p, omap); break;
    }
}

cudaError_t launch_tc(const TcParams& p, const CUtensorMap& omap, int out_type, int grid, cudaStream_t st) {
    if (p.decimated)
        launch_tc_dec<true>(p, omap, out_type, grid, st);
    else
        launch_tc_dec<false>(p, omap, out_type, grid, st);
    return cudaGetLastError();
}

}  // namespace fcwt
