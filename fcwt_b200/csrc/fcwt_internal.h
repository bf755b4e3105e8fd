// Internal declarations shared by the host planner (fcwt_host.cpp), the CUDA
// kernels (fcwt_kernels.cu) and the C-ABI layer (fcwt_capi.cu).
//
// Transform recap (reference: src/fcwt/fcwt.cpp:447-529). For one signal of n
// samples, N = 2^find2power(n). Ihat = FFT_N(zero-padded signal). Row i of the
// output is
//     y_i[t] = s * sum_{q < N/2} Ihat[q] * W_i[q] * exp(+2 pi i q t / N),  t < n,
// with s = 1/N when normalising. W_i[q] = mother[idx_i(q)] for q < proc_i, and
// for proc_i <= q the weight the most recent earlier row wrote into the reused
// O1 buffer (0 if none). idx_i(q) = (int)min(N-1, (float)(scale_i/2) * q).
//
// Device decomposition of the inverse transform, per row, with P2 = 1024:
//   t = c + M*a      (c < M = N/1024 columns, a < 1024)
//   q = L + k2 + 1024*k1   (L a multiple of 1024, k2 < 1024, k1 < K)
//   phase 1 (per k2, per v < R = M/K):
//       G[c = v + R*u][k2] = w_N^{(k2+L)c} * DFT_K( Z[L+k2+1024 k1] * w_M^{v k1} )[u]
//   phase 2 (per column c): y[c + M a] = DFT_1024( G[c][.] )[a]
// where w_X = exp(+2 pi i / X) and Z = Ihat * W.
#pragma once

#include <stdint.h>

#include <cuda.h>
#include <vector_types.h>

namespace fcwt {

constexpr int kP2 = 1024;          // phase-2 transform length
constexpr int kLog2P2 = 10;
constexpr int kMaxLog2N = 23;      // N <= 8M samples
constexpr int kMaxFusedN = 8192;   // rows of N <= this run whole inside one CTA
constexpr int kThreads = 256;      // threads per CTA of the row engine (2 CTAs per SM)
constexpr int kChunk = 64;         // phase-1 k2 values per work item
constexpr int kMaxK = 32;          // phase-1 transform length held in registers
constexpr int kGroupCols = 8;      // phase-2 columns per work item (one per warp)
constexpr int kMaxOuts = 1024;     // output buffers per launch

// One input signal of a launch (a batch may hold several).
struct SigDesc {
    const float2* X;       // forward spectrum, >= N/2 bins
    const float* mother;   // mother table, N entries
    const float2* tw;      // [0,1024): w_N^j ; [1024, 1024+M): w_N^{1024 j}
    int log2N;
    int n;
};

// One output row.
struct RowDesc {
    int sig;          // index into SigDesc[]
    int proc;         // own truncation length (bins [0, proc) use this row's scale)
    float step;       // (float)(scale / 2.0)
    int K;            // phase-1 length (power of two, 1..M)
    int L;            // window start bin (multiple of 1024 when N >= 1024)
    int lo, hi;       // bins outside [lo, hi) are treated as zero weight
    int stale;        // offset of the stale-step table in the pool, -1 when none
    int slot;         // scratch slot (two-phase rows), -1 otherwise
    int wait_row;     // row whose phase-2 items must finish before this row's
                      // phase 1 reuses its scratch slot (-1: none)
    int n_a;          // number of phase-1 items of this row
    int n_b;          // number of phase-2 items of this row
    int out_buf;      // index of the output buffer
    long long out_off;  // element offset of the row inside that buffer
    float out_scale;  // 1/N or 1
    int out_row;      // row index inside that buffer (for tensor-map stores)
    int mode;         // 0: reference mother-table weights; 1: continuous Morlet
    float ca, cb;     // continuous Morlet: u = ca*q - cb
    float cnorm;      // continuous Morlet amplitude (the mother table's norm)
    int kp;           // tensor-core rows: 1024-bin blocks of the window, padded to 8 or 16
    long long woff;   // tensor-core rows: offset of the row's 1024*kp weights in the plan's table
    int imag;         // 1: wavelet with imag_frequency, every product multiplied by i
    int dec;          // time decimation D (power of two): output sample t' is y[D t']
    int n_out;        // output samples of the row: ceil(n / D)
    int pad_;
};

enum ItemType : int { ITEM_FUSED = 0, ITEM_PHASE1 = 1, ITEM_PHASE2 = 2, ITEM_SMALL = 3, ITEM_PHASE1W = 4 };

// Rows whose window needs K > kMaxK use warp-cooperative phase-1 items: each
// covers kWideChunk consecutive k2 (one per warp) for all v.
constexpr int kWideChunk = kThreads / 32;

struct Item {
    int type;
    int row;
    int part;   // chunk / column-group index
    int pad;
};

enum OutType : int { OUT_C64 = 0, OUT_BF16 = 1, OUT_F16 = 2, OUT_POWER = 3, OUT_DB = 4 };

// One signal of a batched forward FFT: input (real or complex), its length,
// the spectrum it produces and a ping-pong buffer of N complex values.
struct FwdJob {
    const float* in_r;
    const float2* in_c;
    int n;
    int pad;
    float2* X;
    float2* tmp;
};

// Everything the row engine needs for one launch.
struct EngineParams {
    const SigDesc* sigs;
    const RowDesc* rows;
    const Item* items;
    int n_items;
    const float* stale_pool;
    float2* scratch;           // S slots of (N_max) complex values
    long long slot_elems;      // complex values per slot
    unsigned* counters;        // [0]: queue head; then a_done[rows], b_done[rows]
    int n_rows;
    void* outs[kMaxOuts];      // output buffers (passed by value with the launch)
    int out_type;
    int* err;                  // device error word (0 = ok)
    int tma_store;             // phase-2 outputs via the tensor map (buffer 0, complex64, even n)
};

// Tensor-core row engine (fcwt_tc.cu): rows whose window [L, L + 1024 kp)
// (L a multiple of 1024) spans at most kTcMaxKp blocks, for N >= kTcMinN.
constexpr int kTcMaxKp = 16;
constexpr int kTcMinN = 16384;

// Entries of the tensor-core engine's work list: a row index, or one of 2, 4
// or 8 parts of a row's column groups (the last entries of a launch, so that
// its final wave is finer than whole rows): row | log2(parts) << 24 | part << 26.
constexpr int kUnitRowBits = 24;
constexpr int kUnitRowMask = (1 << kUnitRowBits) - 1;
__host__ __device__ constexpr int tc_unit(int row, int log2parts, int part) {
    return row | (log2parts << kUnitRowBits) | (part << (kUnitRowBits + 2));
}
// Column groups [gb, ge) of a unit of a row with ng groups; part ranges hold an
// even number of groups so that the two halves of a CTA share them evenly.
__host__ __device__ inline void tc_unit_groups(int entry, int ng, int* gb, int* ge) {
    const int lp = (entry >> kUnitRowBits) & 3;
    const int part = (entry >> (kUnitRowBits + 2)) & 7;
    if (lp == 0) {
        *gb = 0;
        *ge = ng;
        return;
    }
    const int parts = 1 << lp;
    const int chunk = (((ng + parts - 1) / parts) + 1) & ~1;
    *gb = part * chunk < ng ? part * chunk : ng;
    *ge = *gb + chunk < ng ? *gb + chunk : ng;
}

struct TcParams {
    const SigDesc* sigs;
    const RowDesc* rows;
    const int* row_list;       // work units of this launch (tc_unit entries), in queue order
    int n_list;
    const float* stale_pool;
    const float* wts;          // per-row daughter weights x out_scale on [L, L + 1024 kp)
    unsigned* counter;         // row queue head
    void* outs[kMaxOuts];
    int* err;
    int tma_store;             // outputs via the tensor map (buffer 0, complex64, even n)
    int decimated;             // some row has RowDesc::dec > 1 (selects the decimating kernel)
    // many outputs (batched plans): one tensor map per output buffer in global
    // memory, used where bit `out_buf` of tmap_mask is set
    const CUtensorMap* tmaps;
    unsigned long long tmap_mask[kMaxOuts / 64];
};

// Error bits written by device code into EngineParams::err.
constexpr int kErrWaitTimeout = 1;
constexpr int kErrBadItem = 2;

// ---------------------------------------------------------------- host side
// Implemented in fcwt_host.cpp (no CUDA dependency).
namespace host {

int find2power(int n);
void scales(int scaletype, int fs, float f0, float f1, int fn, float* out);
void frequencies(const float* scales, int fn, int fs, float* out);
float mother_norm();
void mother_table(float fb, int N, float* out);
int morlet_support(float fb, float scale);
void morlet_time(float fb, float scale, int size, float* real, float* imag);
void morlet_wavelet(float fb, float scale, int pn, float* out_interleaved);
int row_proc(int N, float scale, int threads, bool avx);
float row_step(float scale);
int row_index(int N, float step, int q);

}  // namespace host
}  // namespace fcwt
