// Host planner: turns (signal length, scales, threads, flags) into the per-row
// description the device engine executes. No CUDA dependency.
#pragma once

#include <string>
#include <vector>

namespace fcwt {

// Flags of the C ABI (mirrored in include/fcwt_b200.h).
constexpr unsigned kFlagNorm = 1u << 0;
constexpr unsigned kFlagScalarTrunc = 1u << 1;
constexpr unsigned kFlagExactSupport = 1u << 2;
constexpr unsigned kFlagContinuous = 1u << 3;
constexpr unsigned kFlagStrict = 1u << 4;

// Relative weight below which a bin's daughter value is skipped (unless
// kFlagExactSupport): mother[w] < kTrimRel * max(mother). The skipped terms
// change each output by at most kTrimRel * max|W| * sum|Ihat| / N, i.e.
// 1.5e-11 of the largest weight: far below float32 resolution.
constexpr double kTrimRel = 1.4551915228366852e-11;  // 2^-36

struct RowPlan {
    int proc = 0;     // own truncation length
    float step = 0;   // (float)(scale/2.0)
    int E = 0;        // largest truncation length of the earlier rows
    int table = -1;   // stale table index (into SignalPlan::tables), -1: none
    int lo = 0, hi = 0;  // bins with non-negligible weight: [lo, hi)
    int K = 1;        // phase-1 length
    int L = 0;        // window start
    float ca = 0, cb = 0;  // continuous Morlet: u = ca*q - cb, weight = norm*exp(-u*u/2)
};

struct SignalPlan {
    int n = 0, N = 1, log2N = 0, M = 0;
    bool is_complex = false;
    float fb = 0;
    int threads = 1;
    unsigned flags = 0;
    std::vector<RowPlan> rows;
    int half = 0;                           // N/2 (>= 1), length of each stale table
    std::vector<std::vector<float>> tables; // stale step tables, `half` floats each
    int w_lo = 0, w_hi = -1;                // mother indices with non-negligible weight
};

// Returns 0 on success, otherwise fills `err`. `mother` (N floats) replaces the
// Morlet(fb) table for trimming when the caller supplies its own wavelet.
int plan_signal(int n, bool is_complex, float fb, const float* scales, int fn, int threads,
                unsigned flags, SignalPlan& out, std::string& err, const float* mother = nullptr);

}  // namespace fcwt
