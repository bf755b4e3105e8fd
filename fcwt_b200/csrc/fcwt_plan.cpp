// Host planner for the device row engine.
//
// For every output row it computes, bit-exactly with the reference's float
// operations (src/fcwt/fcwt.cpp:197-311):
//   - proc: the number of leading bins the reference multiplies for the row;
//   - step: the scale/2 factor of the mother-table index;
//   - the "stale" bins: the reference reuses one O1 buffer for all rows
//     (fcwt.cpp:459-467, 514-518), so bins [proc_i, max_{j<i} proc_j) of row i
//     still hold the product written by the most recent earlier row j that
//     covered them. Those sources are captured in per-run step tables (a run is
//     a maximal stretch of rows with non-increasing proc; all rows of a run see
//     the same source for any bin above their own proc).
// and then the row's bin window for the device engine.
#include "fcwt_plan.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>

#include "fcwt_internal.h"

namespace fcwt {

namespace {

struct StackEntry {
    int proc;
    float step;
};

int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// First q in [a, b) with pred(q) true, for a predicate that is false then true.
template <class F>
int first_true(int a, int b, F pred) {
    while (a < b) {
        int m = a + (b - a) / 2;
        if (pred(m))
            b = m;
        else
            a = m + 1;
    }
    return a;
}

}  // namespace

int plan_signal(int n, bool is_complex, float fb, const float* scales, int fn, int threads,
                unsigned flags, SignalPlan& out, std::string& err, const float* mother_in) {
    if (n < 0) {
        err = "signal length must be >= 0";
        return 1;
    }
    if (fn < 0) {
        err = "number of scales must be >= 0";
        return 1;
    }
    if (threads < 1) {
        err = "threads must be >= 1 (it sets the reference's truncation rule)";
        return 1;
    }
    if (!(fb > 0.0f) || !std::isfinite(fb)) {
        err = "Morlet bandwidth must be a positive finite number";
        return 1;
    }
    const int log2N = host::find2power(n);
    if (log2N > kMaxLog2N) {
        err = "signal too long: padded length exceeds 2^23";
        return 1;
    }
    for (int i = 0; i < fn; i++) {
        if (!(scales[i] > 0.0f) || !std::isfinite(scales[i])) {
            err = "scales must be positive finite numbers";
            return 1;
        }
        // strict mode: centre frequency fs/scale above fs/2 (the reference's
        // Nyquist asserts, src/fcwt/fcwt.cpp:148,167,184, in terms of the scale)
        if ((flags & kFlagStrict) && scales[i] < 2.0f) {
            err = "scale " + std::to_string(scales[i]) + " of row " + std::to_string(i) +
                  " puts its centre frequency above the Nyquist rate fs/2 (strict mode)";
            return 1;
        }
    }
    const int N = 1 << log2N;
    out = SignalPlan();
    out.n = n;
    out.N = N;
    out.log2N = log2N;
    out.M = N >= kP2 ? N / kP2 : 0;
    out.is_complex = is_complex;
    out.fb = fb;
    out.threads = threads;
    out.flags = flags;
    out.half = std::max(N / 2, 1);
    out.rows.resize((size_t)fn);
    const bool avx = (flags & kFlagScalarTrunc) == 0;
    const bool exact = (flags & kFlagExactSupport) != 0;

    if (flags & kFlagContinuous) {
        // Differentiable Morlet: weight(q) = norm * exp(-u^2/2), u = 2 pi fb (s q / N - 1),
        // no index rounding, no truncation, no reused bins. Window: |u| <= sqrt(2 ln(1/tau)).
        const double two_pi = 6.283185307179586;
        const double umax = exact ? 1e30 : std::sqrt(2.0 * std::log(1.0 / kTrimRel));
        for (int i = 0; i < fn; i++) {
            RowPlan& R = out.rows[(size_t)i];
            const double sc = scales[i];
            R.ca = (float)(two_pi * fb * sc / N);
            R.cb = (float)(two_pi * fb);
            const double qlo = (1.0 - umax / (two_pi * fb)) * N / sc;
            const double qhi = (1.0 + umax / (two_pi * fb)) * N / sc;
            int lo = (int)std::max(0.0, std::floor(qlo));
            int hi = (int)std::min((double)out.half, std::ceil(qhi) + 1.0);
            if (N < 2) hi = 0;
            if (hi <= lo) lo = hi = 0;
            R.proc = hi;
            R.step = 0.0f;
            R.lo = lo;
            R.hi = hi;
            if (N >= kP2) {
                const int M = out.M;
                if (hi <= lo) {
                    R.K = 1;
                    R.L = 0;
                } else {
                    int L = (lo / kP2) * kP2;
                    int K = next_pow2((hi - L + kP2 - 1) / kP2);
                    if (K >= M || (long long)L + (long long)K * kP2 > N) {
                        K = M;
                        L = 0;
                    }
                    R.K = K;
                    R.L = L;
                }
            }
        }
        return 0;
    }
    for (int i = 0; i < fn; i++) {
        out.rows[(size_t)i].proc = std::min(host::row_proc(N, scales[i], threads, avx), N / 2);
        out.rows[(size_t)i].step = host::row_step(scales[i]);
    }

    // ---- stale sources: monotone stack over earlier rows (strictly decreasing
    // proc from bottom to top, most recent on top).
    std::vector<StackEntry> stack;
    stack.reserve(64);
    int run_start = 0;
    bool run_needs_table = false;
    auto close_run = [&](int run_end) {
        if (run_needs_table) {
            std::vector<float> T((size_t)out.half, 0.0f);
            // entry k covers [proc_{k+1}, proc_k) as the most recent coverer.
            for (size_t k = 0; k < stack.size(); k++) {
                int top = stack[k].proc;
                int bot = (k + 1 < stack.size()) ? stack[k + 1].proc : 0;
                for (int q = bot; q < top && q < out.half; q++) T[(size_t)q] = stack[k].step;
            }
            int id = (int)out.tables.size();
            out.tables.push_back(std::move(T));
            for (int r = run_start; r < run_end; r++)
                if (out.rows[(size_t)r].E > out.rows[(size_t)r].proc) out.rows[(size_t)r].table = id;
        }
        run_needs_table = false;
    };
    for (int i = 0; i < fn; i++) {
        RowPlan& R = out.rows[(size_t)i];
        if (i > 0 && R.proc > out.rows[(size_t)i - 1].proc) {
            close_run(i);
            run_start = i;
        }
        R.E = stack.empty() ? 0 : stack.front().proc;
        while (!stack.empty() && stack.back().proc <= R.proc) stack.pop_back();
        if (R.E > R.proc) run_needs_table = true;
        stack.push_back({R.proc, R.step});
        if ((long long)out.tables.size() * out.half > (1ll << 28)) {
            err = "scale sequence needs too many distinct stale-bin tables";
            return 2;
        }
    }
    close_run(fn);

    // ---- significant mother indices (for trimming negligible weights).
    if (!exact) {
        std::vector<float> mother((size_t)N);
        if (mother_in)
            std::copy(mother_in, mother_in + N, mother.begin());
        else
            host::mother_table(fb, N, mother.data());
        float mx = 0.0f;
        for (float v : mother) mx = std::max(mx, std::fabs(v));
        const double thr = kTrimRel * (double)mx;
        int wl = 0, wh = N - 1;
        while (wl < N && std::fabs((double)mother[(size_t)wl]) < thr) wl++;
        while (wh >= 0 && std::fabs((double)mother[(size_t)wh]) < thr) wh--;
        out.w_lo = wl;
        out.w_hi = wh;
    } else {
        out.w_lo = 0;
        out.w_hi = N - 1;
    }

    // per-table significance prefix/suffix structures (trimmed mode only)
    std::vector<std::vector<int>> next_sig, prev_sig;
    if (!exact) {
        next_sig.resize(out.tables.size());
        prev_sig.resize(out.tables.size());
        for (size_t t = 0; t < out.tables.size(); t++) {
            const std::vector<float>& T = out.tables[t];
            std::vector<int>& nx = next_sig[t];
            std::vector<int>& pv = prev_sig[t];
            nx.assign((size_t)out.half + 1, INT_MAX);
            pv.assign((size_t)out.half + 1, -1);
            auto sig = [&](int q) {
                float s = T[(size_t)q];
                if (!(s > 0.0f)) return false;
                int w = host::row_index(N, s, q);
                return w >= out.w_lo && w <= out.w_hi;
            };
            for (int q = out.half - 1; q >= 0; q--) nx[(size_t)q] = sig(q) ? q : nx[(size_t)q + 1];
            for (int q = 0; q < out.half; q++) pv[(size_t)q + 1] = sig(q) ? q : pv[(size_t)q];
        }
    }

    // ---- per-row bin window
    for (int i = 0; i < fn; i++) {
        RowPlan& R = out.rows[(size_t)i];
        int lo, hi;
        if (exact) {
            lo = 0;
            hi = std::max(R.proc, R.table >= 0 ? R.E : 0);
            if (hi == 0) lo = 0;
        } else {
            // own bins: idx(q) is non-decreasing in q
            int qa = first_true(0, R.proc, [&](int q) { return host::row_index(N, R.step, q) >= out.w_lo; });
            int qb = first_true(qa, R.proc, [&](int q) { return host::row_index(N, R.step, q) > out.w_hi; });
            lo = INT_MAX;
            hi = INT_MIN;
            if (qa < qb) {
                lo = qa;
                hi = qb;
            }
            if (R.table >= 0 && R.E > R.proc) {
                int e = std::min(R.E, out.half);
                int f = next_sig[(size_t)R.table][(size_t)R.proc];
                int l = prev_sig[(size_t)R.table][(size_t)e];
                if (f < e && l >= R.proc) {
                    lo = std::min(lo, f);
                    hi = std::max(hi, l + 1);
                }
            }
            if (lo >= hi) {
                lo = 0;
                hi = 0;
            }
        }
        R.lo = lo;
        R.hi = hi;
        if (N >= kP2) {
            const int M = out.M;
            if (hi <= lo) {
                R.K = 1;
                R.L = 0;
            } else {
                int L = (lo / kP2) * kP2;
                int span = hi - L;
                int K = next_pow2((span + kP2 - 1) / kP2);
                if (K >= M || (long long)L + (long long)K * kP2 > N) {
                    K = M;
                    L = 0;
                }
                R.K = K;
                R.L = L;
            }
        } else {
            R.K = 1;
            R.L = 0;
        }
    }
    return 0;
}

}  // namespace fcwt
