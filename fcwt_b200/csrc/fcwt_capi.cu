// C ABI of the B200 fCWT path: contexts, plans, transforms and tuning files.
// See include/fcwt_b200.h for the contract of each entry point.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <array>
#include <map>
#include <initializer_list>
#include <queue>
#include <vector>

#include "../../include/fcwt_b200.h"
#include "fcwt_internal.h"
#include "fcwt_plan.h"

namespace fcwt {
size_t engine_smem_bytes();
cudaError_t launch_mother(float fb, int N, float norm, float* out, cudaStream_t st);
cudaError_t launch_twiddle(int log2N, float2* tw, cudaStream_t st);
cudaError_t launch_forward(const float* in_r, const float2* in_c, int n, int log2N, const float2* tw,
                           float2* out, float2* tmp, cudaStream_t st, int* n_kernels);
cudaError_t launch_forward_batched(const FwdJob* jobs, int njobs, int log2N, const float2* tw, cudaStream_t st,
                                   int* n_kernels, bool real);
cudaError_t launch_inverse_batched(const FwdJob* jobs, int njobs, int log2N, const float2* tw, cudaStream_t st,
                                   int* n_kernels);
cudaError_t launch_adjoint_accum(const float2* Xs, const float2* Gh, float2* H, const void* rows, int nr, int half,
                                 long long Nstride, int batch, float cb, float amp, float inv_sigma, double* acc_sigma,
                                 double* acc_f, cudaStream_t st);
cudaError_t launch_take_real(const float2* Y, long long Nstride, int n, int batch, float scale, float* gx,
                             cudaStream_t st);
int adjoint_rows_per_pass();
cudaError_t launch_adjoint_rows(const float2* G, const float2* Xs, const void* rows, int n, int log2N, int fn,
                                int batch, const float2* tw, float cb, float amp, float inv_sigma, float2* H,
                                double* acc_sigma, double* acc_f, cudaStream_t st);
cudaError_t engine_configure();
cudaError_t engine_blocks_per_sm(int* out);
cudaError_t launch_engine(const EngineParams& p, int grid, cudaStream_t st);
cudaError_t launch_engine(const EngineParams& p, const CUtensorMap& omap, int grid, cudaStream_t st);
cudaError_t tc_configure();
cudaError_t launch_tc_weights(const SigDesc* sigs, const RowDesc* rows, const int* row_list, int n_list,
                              const float* pool, float* wts, cudaStream_t st);
cudaError_t launch_tc(const TcParams& p, const CUtensorMap& omap, int out_type, int grid, cudaStream_t st);
cudaError_t launch_shift_spectrum(const float2* X, int log2N, float2* J, cudaStream_t st);
cudaError_t launch_align_spill(const SigDesc* sigs, const RowDesc* rows, const int* list, int nlist,
                               const float* pool, float2* out, int n, float extra, cudaStream_t st);
cudaError_t launch_doublesided_combine(float2* out, const float2* V, long long rows, int n, int dec, int log2N,
                                       const float2* tw, float sgn, cudaStream_t st);
}  // namespace fcwt

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define FCWT_CUDA_TRY(expr)                                                                  \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            return fail(e_ == cudaErrorMemoryAllocation ? FCWT_ERR_NOMEM : FCWT_ERR_CUDA,    \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                \
        }                                                                                    \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t b) {
        if (b <= bytes && p) return cudaSuccess;
        release();
        if (b == 0) b = 16;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            bytes = 0;
            return e;
        }
        bytes = b;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

// Scheduling choices of the two-phase row engine for one padded length.
struct TuneChoice {
    int scratch_mb = 64;  // budget of the scratch ring
    int lag = 12;         // rows between a row's phase 1 and phase 2 items
    int engine = 0;       // 0: tensor-core engine for the rows it takes; 1: CUDA-core engine only
};

// Where a caller's pointer lives: 0 host memory (pageable or pinned), 1 memory
// the kernels of device `dev` may use directly (that device's memory, or
// managed memory), -1 another device's memory, which the kernels of `dev`
// must not touch (without peer access that is an illegal-address fault).
int pointer_kind(const void* p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (a.type == cudaMemoryTypeManaged) return 1;
    if (a.type == cudaMemoryTypeDevice) return a.device == dev ? 1 : -1;
    return 0;
}

bool is_device_pointer(const void* p) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return pointer_kind(p, dev) == 1;
}

// FCWT_OK when no pointer of `ptrs` lives on a device other than `dev`.
int check_pointer_devices(std::initializer_list<const void*> ptrs, int dev) {
    for (const void* p : ptrs) {
        if (p && pointer_kind(p, dev) < 0)
            return fail(FCWT_ERR_INVALID, "a buffer lives on another GPU than the context's device " +
                                              std::to_string(dev));
    }
    return FCWT_OK;
}

size_t out_elem_bytes(int out_type) { return out_type == FCWT_OUT_C64 ? 8 : 4; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// Tensor map of a complex64 [rows][n] output seen as [rows][n / M][M]
// (8-byte elements), boxes of [1][256][8], 64B swizzle. Only complete
// stripes a < n / M are covered. Requires n even and a 16-byte aligned base.
bool encode_output_map(void* base, int n, int M, int rows, CUtensorMap* map) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || (n & 1) || ((uintptr_t)base & 15) || n / M < 1 || rows < 1) return false;
    cuuint64_t dims[3] = {(cuuint64_t)M, (cuuint64_t)(n / M), (cuuint64_t)rows};
    cuuint64_t strides[2] = {(cuuint64_t)M * 8, (cuuint64_t)n * 8};
    cuuint32_t box[3] = {8, 256, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Tensor map of a 16-bit complex output (one 4-byte element per sample),
// boxes of [256 a][8 columns], 32-byte swizzle. n must be a multiple of 4 so
// that the row stride is a multiple of 16 bytes.
bool encode_output_map16(void* base, int n, int M, int rows, CUtensorMap* map) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || (n & 3) || ((uintptr_t)base & 15) || n / M < 1 || rows < 1) return false;
    cuuint64_t dims[3] = {(cuuint64_t)M, (cuuint64_t)(n / M), (cuuint64_t)rows};
    cuuint64_t strides[2] = {(cuuint64_t)M * 4, (cuuint64_t)n * 4};
    cuuint32_t box[3] = {8, 256, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

struct fcwt_plan;

struct fcwt_context {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    int engine_ctas = 0;  // persistent grid of the row engine
    int engine_mode = FCWT_ENGINE_AUTO;  // which rows the tensor-core engine takes
    DevBuf in_stage, out_stage, tmp, scratch, counters, err;
    int* err_host = nullptr;  // pinned mirror of the device error word
    TuneChoice tune[fcwt::kMaxLog2N + 1];
    struct CacheEntry {
        int n, is_complex, fn, threads;
        unsigned flags;
        float fb;
        std::vector<float> scales;
        fcwt_plan* plan;
        unsigned long long last_use;
    };
    std::vector<CacheEntry> cache;
    unsigned long long use_clock = 0;
    // every live plan created on this context (cached or caller-owned): destroying
    // the context releases their device resources and detaches them
    std::vector<fcwt_plan*> plans;
    // host-output pipeline: copy stream, per-slot "rows done" / "block copied" events
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pipe_done[2] = {nullptr, nullptr}, pipe_copied[2] = {nullptr, nullptr};
    // profiling
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_used, ev_free;
    long long kernel_launches = 0;
    // workspace of the differentiable transform's backward
    DevBuf adj_tw, adj_x, adj_g, adj_tmp, adj_h, adj_jobs, adj_rows, adj_acc;
    int adj_tw_log2N = -1;
    void* adj_jobs_host = nullptr;
    size_t adj_jobs_host_bytes = 0;
};

// One signal of a plan.
struct PlanSignal {
    fcwt::SignalPlan sp;
    int rb = 0, re = 0;  // rows of this signal produced by the plan: rb, rb + rstride, ... < re
    int rstride = 1;     // row decimation
    int dec = 1;         // time decimation (power of two): output sample t' is y[dec t']
    int rows_out() const { return re > rb ? (re - rb + rstride - 1) / rstride : 0; }
    int n_out() const { return (sp.n + dec - 1) / dec; }
    int row0 = 0;        // global index of its first produced row
    int table = 0;       // index into fcwt_plan::tables
    DevBuf X;            // forward spectrum, N complex
};

// Tables shared by all signals of one padded length.
struct PlanTables {
    int log2N = 0;
    DevBuf mother, tw;
};

struct fcwt_plan {
    fcwt_context* ctx = nullptr;
    float fb = 0;
    bool is_complex = false;
    std::vector<PlanSignal> sig;
    std::vector<PlanTables> tables;
    DevBuf pool, sigs, rows, items, fwd_jobs, fwd_tmp, graph_jobs, tc_rows, tc_wts;
    DevBuf tc_units;  // work list of the tensor-core engine (rows, the last ones possibly split)
    int n_units = 0;
    // Per-execution uploads of batched plans (forward jobs, per-output tensor
    // maps) go through a ring of pinned host slots; a slot is rewritten only
    // after the copy that read it has run (its event), so back-to-back
    // executions with different buffers never see each other's data.
    struct UploadSlot {
        void* host = nullptr;
        size_t bytes = 0;
        cudaEvent_t done = nullptr;
        bool pending = false;
    };
    std::array<UploadSlot, 4> uploads;
    int upload_next = 0;
    DevBuf tmaps, graph_tmaps;               // per-output tensor maps (batched plans), device copies
    std::array<unsigned long long, fcwt::kMaxOuts / 64> graph_tmap_mask{};
    int n_items = 0;
    int n_rows = 0;
    int n_tc = 0;  // rows run by the tensor-core engine
    std::vector<float> custom_mother;  // caller's wavelet table (N floats), empty for Morlet(fb)
    bool imag = false;         // wavelet with imag_frequency: every product times i
    bool doublesided = false;  // wavelet with doublesided: second pass on the shifted spectrum
    bool compat_align = false; // reference's odd-n row shift (FCWT_COMPAT_ALIGN)
    DevBuf shifted;            // compat_align: the rows written one sample to the right
    int n_shifted = 0;
    DevBuf Xs, sigs2, ds_tmp;  // doublesided: shifted spectrum, its signal descriptor, second-pass rows
    int slots = 0;
    long long slot_elems = 0;
    bool two_phase = false;
    // CUDA graph of the last device-resident batched execution
    cudaGraphExec_t graph = nullptr;
    std::vector<const void*> graph_key;
    int graph_out_type = -1;
};

namespace {

int ctx_prepare(fcwt_context* ctx) {
    if (!ctx) return fail(FCWT_ERR_INVALID, "null context");
    FCWT_CUDA_TRY(cudaSetDevice(ctx->device));
    return FCWT_OK;
}

// Releases the device and pinned resources of a plan; the plan stays valid as
// an empty shell (idempotent).
void plan_release(fcwt_plan* p) {
    if (p->graph) cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
    for (auto& s : p->sig) s.X.release();
    for (auto& t : p->tables) {
        t.mother.release();
        t.tw.release();
    }
    p->pool.release();
    p->sigs.release();
    p->rows.release();
    p->items.release();
    p->fwd_jobs.release();
    p->fwd_tmp.release();
    p->graph_jobs.release();
    p->tc_rows.release();
    p->tc_units.release();
    p->tc_wts.release();
    p->Xs.release();
    p->sigs2.release();
    p->ds_tmp.release();
    p->shifted.release();
    for (auto& u : p->uploads) {
        if (u.pending && u.done) cudaEventSynchronize(u.done);
        if (u.host) cudaFreeHost(u.host);
        if (u.done) cudaEventDestroy(u.done);
        u = fcwt_plan::UploadSlot{};
    }
    p->tmaps.release();
    p->graph_tmaps.release();
}

fcwt_plan* plan_new(fcwt_context* ctx) {
    fcwt_plan* P = new fcwt_plan();
    P->ctx = ctx;
    ctx->plans.push_back(P);
    return P;
}

void plan_free(fcwt_plan* p) {
    if (!p) return;
    if (p->ctx) {
        auto& v = p->ctx->plans;
        v.erase(std::remove(v.begin(), v.end(), p), v.end());
    }
    plan_release(p);
    delete p;
}

// Finish time of a queue of work units on `ctas` persistent CTAs that claim
// them in order (the earliest free CTA takes the next unit).
double queue_makespan(const std::vector<double>& cost, int ctas) {
    std::priority_queue<double, std::vector<double>, std::greater<double>> q;
    for (int i = 0; i < ctas; i++) q.push(0.0);
    double end = 0.0;
    for (double c : cost) {
        const double t = q.top() + c;
        q.pop();
        q.push(t);
        end = std::max(end, t);
    }
    return end;
}

// Work list of the tensor-core engine: the rows in order, with the last K
// rows split into 2, 4 or 8 parts of their column groups when a simulation of
// the queue says that finishes sooner. Cost model in column-group times: a
// unit costs its groups plus about 1.2 for the per-row pre-pass and prologue.
std::vector<int> plan_tc_units(const std::vector<int>& tc_rows, const std::vector<int>& groups, int ctas) {
    constexpr double kUnitOverhead = 1.2;
    const int n = (int)tc_rows.size();
    std::vector<int> best;
    for (int g : tc_rows) best.push_back(g);
    if (n == 0 || ctas <= 1) return best;
    std::vector<double> cost;
    for (int i = 0; i < n; i++) cost.push_back(kUnitOverhead + groups[(size_t)i]);
    double best_t = queue_makespan(cost, ctas);
    for (int lp = 1; lp <= 3; lp++) {
        const int parts = 1 << lp;
        for (int K : {ctas / 8, ctas / 4, ctas / 2, ctas, 2 * ctas}) {
            K = std::min(K, n);
            if (K <= 0) continue;
            std::vector<int> units;
            cost.clear();
            for (int i = 0; i < n; i++) {
                const int ng = groups[(size_t)i];
                if (i < n - K || ng < 2 * parts) {
                    units.push_back(tc_rows[(size_t)i]);
                    cost.push_back(kUnitOverhead + ng);
                    continue;
                }
                for (int part = 0; part < parts; part++) {
                    const int e = fcwt::tc_unit(tc_rows[(size_t)i], lp, part);
                    int gb, ge;
                    fcwt::tc_unit_groups(e, ng, &gb, &ge);
                    if (ge <= gb) continue;
                    units.push_back(e);
                    cost.push_back(kUnitOverhead + (ge - gb));
                }
            }
            const double t = queue_makespan(cost, ctas);
            if (t < best_t * 0.995) {
                best_t = t;
                best = units;
            }
        }
    }
    return best;
}

// Builds descriptors and the work list of all signals. Rows of N < 1024 get a
// direct-DFT item, rows of N <= 8192 one fused item; two-phase rows (all
// signals, in order) get phase-1 items and phase-2 items, phase 2 of row r
// issued after phase 1 of row r + lag, scratch slots reused round-robin.
int plan_build(fcwt_plan* P) {
    using namespace fcwt;
    fcwt_context* ctx = P->ctx;
    cudaStream_t st = ctx->stream;
    const int nsig = (int)P->sig.size();
    if (nsig > kMaxOuts) return fail(FCWT_ERR_INVALID, "at most 1024 signals per plan");
    // tables per padded length
    for (auto& S : P->sig) {
        int t = -1;
        for (size_t i = 0; i < P->tables.size(); i++)
            if (P->tables[i].log2N == S.sp.log2N) t = (int)i;
        if (t < 0) {
            P->tables.emplace_back();
            P->tables.back().log2N = S.sp.log2N;
            t = (int)P->tables.size() - 1;
        }
        S.table = t;
    }
    std::vector<float> pool;
    std::vector<RowDesc> rows;
    std::vector<int> two_phase_rows;  // global indices, in order
    std::vector<int> tc_rows;         // rows of the tensor-core engine, in order
    long long tc_wts_elems = 0;       // size of their weight table
    std::vector<int> wts_rows;        // rows that own a weight-table entry
    std::map<std::array<uint32_t, 12>, long long> wts_owner;
    std::vector<Item> items;
    std::vector<int> compat_rows;     // compat_align: shifted rows (descriptor indices)
    int max_two_phase_log2N = 0;
    for (int s = 0; s < nsig; s++) {
        PlanSignal& S = P->sig[(size_t)s];
        const SignalPlan& sp = S.sp;
        const long long pool_off = (long long)pool.size();
        for (const auto& T : sp.tables) pool.insert(pool.end(), T.begin(), T.end());
        if ((long long)pool.size() > (1ll << 30)) return fail(FCWT_ERR_INVALID, "stale-bin tables too large");
        const float out_scale = (sp.flags & kFlagNorm) ? 1.0f / (float)sp.N : 1.0f;
        S.row0 = (int)rows.size();
        const int Mfull = sp.N >= kP2 ? sp.N / kP2 : 1;
        if (S.dec > 1 && sp.N > kMaxFusedN && Mfull / S.dec < kGroupCols)
            return fail(FCWT_ERR_UNSUPPORTED, "time decimation " + std::to_string(S.dec) + " needs N >= 8192 x " +
                                                  std::to_string(S.dec) + " for a padded length above 8192 (N = " +
                                                  std::to_string(sp.N) + ")");
        for (int r = S.rb; r < S.re; r += S.rstride) {
            const RowPlan& rp = sp.rows[(size_t)r];
            const int ro = (r - S.rb) / S.rstride;  // output row
            RowDesc d;
            std::memset(&d, 0, sizeof(d));
            d.sig = s;
            d.proc = rp.proc;
            d.step = rp.step;
            d.K = rp.K;
            d.L = rp.L;
            d.lo = rp.lo;
            d.hi = rp.hi;
            d.stale = rp.table >= 0 ? (int)(pool_off + (long long)rp.table * sp.half) : -1;
            d.slot = -1;
            d.wait_row = -1;
            d.out_buf = s;
            d.dec = S.dec;
            d.n_out = S.n_out();
            d.out_off = (long long)ro * d.n_out;
            if (P->compat_align && (sp.n & 1) && (r & 1) && r < sp.rows.size() - 1) {
                // written through std::align: one sample to the right, n - 1 samples
                d.out_off += 1;
                d.n_out -= 1;
                compat_rows.push_back((int)rows.size());
            }
            d.out_scale = out_scale;
            d.out_row = ro;
            d.mode = (sp.flags & kFlagContinuous) ? 1 : 0;
            d.ca = rp.ca;
            d.cb = rp.cb;
            d.cnorm = host::mother_norm();
            d.kp = 0;
            d.imag = P->imag ? 1 : 0;
            const int g = (int)rows.size();
            // tensor-core rows: window [L, L + 1024 kp), L a multiple of 1024, kp <= 16
            int tc_kp = 0;
            const bool tc_on = ctx->engine_mode == FCWT_ENGINE_TENSOR_CORES ||
                               (ctx->engine_mode == FCWT_ENGINE_AUTO && ctx->tune[sp.log2N].engine == 0);
            if (tc_on && sp.N >= kTcMinN && Mfull / S.dec >= kGroupCols) {
                const int L = rp.hi > rp.lo ? (rp.lo / kP2) * kP2 : 0;
                const int kw = rp.hi > rp.lo ? (rp.hi - L + kP2 - 1) / kP2 : 0;
                if (kw <= kTcMaxKp) tc_kp = kw <= 8 ? 8 : 16;
                if (tc_kp) d.L = L;
            }
            d.kp = tc_kp;
            d.woff = 0;
            if (tc_kp) {
                // rows whose weights are the same function of q share one table entry
                // (e.g. many channels on one grid); rows with stale bins never do
                bool shared = false;
                std::array<uint32_t, 12> key{};
                if (d.stale < 0) {
                    const float fk[6] = {d.step, d.ca, d.cb, d.cnorm, d.out_scale, 0.0f};
                    key = {(uint32_t)sp.log2N, (uint32_t)d.mode, (uint32_t)d.L, (uint32_t)d.lo, (uint32_t)d.hi,
                           (uint32_t)d.proc, (uint32_t)d.kp, 0, 0, 0, 0, 0};
                    for (int k = 0; k < 5; k++) std::memcpy(&key[7 + k], &fk[k], 4);
                    auto it = wts_owner.find(key);
                    if (it != wts_owner.end()) {
                        d.woff = it->second;
                        shared = true;
                    }
                }
                if (!shared) {
                    d.woff = tc_wts_elems;
                    tc_wts_elems += (long long)kP2 * tc_kp;
                    if (d.stale < 0) wts_owner.emplace(key, d.woff);
                    wts_rows.push_back((int)rows.size());
                }
            }
            rows.push_back(d);
            if (tc_kp) {
                tc_rows.push_back(g);
            } else if (sp.N > kMaxFusedN) {
                two_phase_rows.push_back(g);
                max_two_phase_log2N = std::max(max_two_phase_log2N, sp.log2N);
            } else {
                items.push_back({sp.N < kP2 ? ITEM_SMALL : ITEM_FUSED, g, 0, 0});
            }
        }
    }
    P->n_rows = (int)rows.size();
    P->two_phase = !two_phase_rows.empty();
    P->slots = 0;
    P->slot_elems = 0;
    if (P->two_phase) {
        const TuneChoice& tc = ctx->tune[max_two_phase_log2N];
        const long long slot_elems = 1ll << max_two_phase_log2N;
        const int nt = (int)two_phase_rows.size();
        int S = (int)std::max(4LL, std::min(40LL, ((long long)tc.scratch_mb << 20) / (slot_elems * 8)));
        S = std::min(S, std::max(1, nt));
        int D = std::max(1, std::min(tc.lag, S / 2));
        if (S == 1) D = 1;
        if (D >= S && S > 1) return fail(FCWT_ERR_INVALID, "internal: lag >= slots");
        for (int i = 0; i < nt; i++) {
            RowDesc& d = rows[(size_t)two_phase_rows[(size_t)i]];
            const int M = (int)(1ll << (P->sig[(size_t)d.sig].sp.log2N - kLog2P2));
            d.slot = i % S;
            d.wait_row = i >= S ? two_phase_rows[(size_t)(i - S)] : -1;
            d.n_a = d.K > kMaxK ? kP2 / kWideChunk : kP2 / kChunk;
            d.n_b = M / d.dec / kGroupCols;
        }
        for (int step = 0; step < nt + D; step++) {
            if (step < nt) {
                const int g = two_phase_rows[(size_t)step];
                const int type = rows[(size_t)g].K > kMaxK ? ITEM_PHASE1W : ITEM_PHASE1;
                for (int a = 0; a < rows[(size_t)g].n_a; a++) items.push_back({type, g, a, 0});
            }
            const int rb = step - D;
            if (rb >= 0 && rb < nt) {
                const int g = two_phase_rows[(size_t)rb];
                for (int b = 0; b < rows[(size_t)g].n_b; b++) items.push_back({ITEM_PHASE2, g, b, 0});
            }
        }
        P->slots = S;
        P->slot_elems = slot_elems;
    }
    P->n_items = (int)items.size();
    P->n_tc = (int)tc_rows.size();

    // device buffers and tables
    for (auto& T : P->tables) {
        const int N = 1 << T.log2N;
        const int M = N >= kP2 ? N / kP2 : 1;
        FCWT_CUDA_TRY(T.mother.ensure((size_t)N * sizeof(float)));
        FCWT_CUDA_TRY(T.tw.ensure((size_t)(1024 + M) * sizeof(float2)));
        if (!P->custom_mother.empty() && (int)P->custom_mother.size() == N)
            FCWT_CUDA_TRY(cudaMemcpyAsync(T.mother.p, P->custom_mother.data(), (size_t)N * sizeof(float),
                                          cudaMemcpyHostToDevice, st));
        else
            FCWT_CUDA_TRY(launch_mother(P->fb, N, host::mother_norm(), T.mother.as<float>(), st));
        FCWT_CUDA_TRY(launch_twiddle(T.log2N, T.tw.as<float2>(), st));
    }
    std::vector<SigDesc> sds((size_t)nsig);
    size_t tmp_elems = 0;
    for (int s = 0; s < nsig; s++) {
        PlanSignal& S = P->sig[(size_t)s];
        FCWT_CUDA_TRY(S.X.ensure((size_t)S.sp.N * sizeof(float2)));
        sds[(size_t)s].X = S.X.as<float2>();
        sds[(size_t)s].mother = P->tables[(size_t)S.table].mother.as<float>();
        sds[(size_t)s].tw = P->tables[(size_t)S.table].tw.as<float2>();
        sds[(size_t)s].log2N = S.sp.log2N;
        sds[(size_t)s].n = S.sp.n;
        tmp_elems += (size_t)S.sp.N;
    }
    if (nsig > 1) {
        FCWT_CUDA_TRY(P->fwd_tmp.ensure(tmp_elems * sizeof(float2)));
        FCWT_CUDA_TRY(P->fwd_jobs.ensure((size_t)nsig * sizeof(FwdJob)));
        FCWT_CUDA_TRY(P->tmaps.ensure((size_t)nsig * sizeof(CUtensorMap)));
    }
    FCWT_CUDA_TRY(P->pool.ensure(std::max<size_t>(pool.size(), 1) * sizeof(float)));
    FCWT_CUDA_TRY(P->sigs.ensure(sds.size() * sizeof(SigDesc)));
    FCWT_CUDA_TRY(P->rows.ensure(std::max<size_t>(rows.size(), 1) * sizeof(RowDesc)));
    FCWT_CUDA_TRY(P->items.ensure(std::max<size_t>(items.size(), 1) * sizeof(Item)));
    if (!pool.empty())
        FCWT_CUDA_TRY(cudaMemcpyAsync(P->pool.p, pool.data(), pool.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    FCWT_CUDA_TRY(cudaMemcpyAsync(P->sigs.p, sds.data(), sds.size() * sizeof(SigDesc), cudaMemcpyHostToDevice, st));
    if (!rows.empty())
        FCWT_CUDA_TRY(cudaMemcpyAsync(P->rows.p, rows.data(), rows.size() * sizeof(RowDesc), cudaMemcpyHostToDevice, st));
    if (!items.empty())
        FCWT_CUDA_TRY(cudaMemcpyAsync(P->items.p, items.data(), items.size() * sizeof(Item), cudaMemcpyHostToDevice, st));
    if (!tc_rows.empty()) {
        FCWT_CUDA_TRY(P->tc_rows.ensure(tc_rows.size() * sizeof(int)));
        FCWT_CUDA_TRY(cudaMemcpyAsync(P->tc_rows.p, tc_rows.data(), tc_rows.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, st));
        std::vector<int> groups;
        for (int g : tc_rows) {
            const RowDesc& d = rows[(size_t)g];
            groups.push_back((1 << (P->sig[(size_t)d.sig].sp.log2N - kLog2P2)) / d.dec / kGroupCols);
        }
        const std::vector<int> units = plan_tc_units(tc_rows, groups, ctx->num_sms);
        P->n_units = (int)units.size();
        FCWT_CUDA_TRY(P->tc_units.ensure(units.size() * sizeof(int)));
        FCWT_CUDA_TRY(cudaMemcpyAsync(P->tc_units.p, units.data(), units.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, st));
        FCWT_CUDA_TRY(P->tc_wts.ensure((size_t)tc_wts_elems * sizeof(float)));
        DevBuf owners;
        FCWT_CUDA_TRY(owners.ensure(wts_rows.size() * sizeof(int)));
        FCWT_CUDA_TRY(cudaMemcpyAsync(owners.p, wts_rows.data(), wts_rows.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, st));
        FCWT_CUDA_TRY(launch_tc_weights(P->sigs.as<SigDesc>(), P->rows.as<RowDesc>(), owners.as<int>(),
                                        (int)wts_rows.size(), P->pool.as<float>(), P->tc_wts.as<float>(), st));
        FCWT_CUDA_TRY(cudaStreamSynchronize(st));
        owners.release();
    }
    if (!compat_rows.empty()) {
        FCWT_CUDA_TRY(P->shifted.ensure(compat_rows.size() * sizeof(int)));
        FCWT_CUDA_TRY(cudaMemcpyAsync(P->shifted.p, compat_rows.data(), compat_rows.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, st));
    }
    P->n_shifted = (int)compat_rows.size();
    if (P->doublesided) {
        const PlanSignal& S = P->sig[0];
        FCWT_CUDA_TRY(P->Xs.ensure((size_t)S.sp.N * sizeof(float2)));
        SigDesc s2 = sds[0];
        s2.X = P->Xs.as<float2>();
        FCWT_CUDA_TRY(P->sigs2.ensure(sizeof(SigDesc)));
        FCWT_CUDA_TRY(cudaMemcpyAsync(P->sigs2.p, &s2, sizeof(SigDesc), cudaMemcpyHostToDevice, st));
        FCWT_CUDA_TRY(P->ds_tmp.ensure(std::max<size_t>((size_t)S.rows_out() * (size_t)S.n_out(), 1) * sizeof(float2)));
    }
    FCWT_CUDA_TRY(cudaStreamSynchronize(st));
    return FCWT_OK;
}

// Queue counters of one execution: [0] item queue; a_done[rows]; b_done[rows];
// tensor-core row queue.
size_t plan_counters(const fcwt_plan* P) { return 2 + 2 * (size_t)P->n_rows; }

// (table, count) groups of the batched forward jobs, in table order.
void job_groups(const fcwt_plan* P, std::vector<std::pair<int, int>>& groups) {
    groups.clear();
    for (size_t t = 0; t < P->tables.size(); t++) {
        int c = 0;
        for (const auto& S : P->sig) c += S.table == (int)t;
        groups.push_back({(int)t, c});
    }
}

// A pinned host buffer of at least `bytes` that no enqueued copy still reads.
int upload_slot(fcwt_plan* P, size_t bytes, fcwt_plan::UploadSlot** out) {
    fcwt_plan::UploadSlot& u = P->uploads[(size_t)P->upload_next];
    P->upload_next = (P->upload_next + 1) % (int)P->uploads.size();
    if (u.pending) FCWT_CUDA_TRY(cudaEventSynchronize(u.done));
    u.pending = false;
    if (!u.done) FCWT_CUDA_TRY(cudaEventCreateWithFlags(&u.done, cudaEventDisableTiming));
    if (u.bytes < bytes) {
        if (u.host) cudaFreeHost(u.host);
        u.host = nullptr;
        u.bytes = 0;
        FCWT_CUDA_TRY(cudaMallocHost(&u.host, bytes));
        u.bytes = bytes;
    }
    *out = &u;
    return FCWT_OK;
}

// The tensor maps of every output of a batched plan (entry s for output s)
// and the mask of the outputs whose map could be encoded.
void build_output_maps(const fcwt_plan* P, void* const* dout, int out_type, CUtensorMap* maps,
                       unsigned long long* mask) {
    for (int i = 0; i < fcwt::kMaxOuts / 64; i++) mask[i] = 0;
    for (size_t s = 0; s < P->sig.size(); s++) {
        const PlanSignal& S = P->sig[s];
        std::memset(&maps[s], 0, sizeof(CUtensorMap));
        if (S.rows_out() == 0 || S.sp.N < fcwt::kTcMinN) continue;
        const bool ok = out_type == FCWT_OUT_C64
                            ? encode_output_map(dout[s], S.n_out(), S.sp.M / S.dec, S.rows_out(), &maps[s])
                            : encode_output_map16(dout[s], S.n_out(), S.sp.M / S.dec, S.rows_out(), &maps[s]);
        if (ok) mask[s >> 6] |= 1ull << (s & 63);
    }
}

// Fills `jobs` with the forward jobs of all signals ordered by table.
void build_jobs(fcwt_plan* P, const void* const* din, std::vector<std::pair<int, int>>& groups, fcwt::FwdJob* jobs) {
    using namespace fcwt;
    const int nsig = (int)P->sig.size();
    std::vector<size_t> tmp_off((size_t)nsig);
    size_t acc = 0;
    for (int s = 0; s < nsig; s++) {
        tmp_off[(size_t)s] = acc;
        acc += (size_t)P->sig[(size_t)s].sp.N;
    }
    int k = 0;
    for (size_t t = 0; t < P->tables.size(); t++) {
        for (int s = 0; s < nsig; s++) {
            PlanSignal& S = P->sig[(size_t)s];
            if (S.table != (int)t) continue;
            FwdJob& j = jobs[k++];
            j.in_r = S.sp.is_complex ? nullptr : (const float*)din[s];
            j.in_c = S.sp.is_complex ? (const float2*)din[s] : nullptr;
            j.n = S.sp.n;
            j.pad = 0;
            j.X = S.X.as<float2>();
            j.tmp = P->fwd_tmp.as<float2>() + tmp_off[(size_t)s];
        }
    }
    job_groups(P, groups);
}

int enqueue_rows(fcwt_plan* P, const fcwt::SigDesc* dsigs, void* const* dout, int out_type,
                 bool graph_maps = false);
int enqueue_forward(fcwt_plan* P, const void* const* din, const fcwt::FwdJob* graph_jobs);

// Enqueues the forward FFTs and the row engine for device-resident inputs and
// outputs (no host synchronisation, so it can be captured into a graph).
// graph_jobs: device copy of the forward jobs prepared before a capture; the
// per-output tensor maps of a batched plan are then plan->graph_tmaps.
int plan_enqueue(fcwt_plan* P, const void* const* din, void* const* dout, int out_type, bool allow_profiling,
                 const fcwt::FwdJob* graph_jobs = nullptr) {
    using namespace fcwt;
    fcwt_context* ctx = P->ctx;
    cudaStream_t st = ctx->stream;
    if (P->doublesided && out_type != FCWT_OUT_C64)
        return fail(FCWT_ERR_UNSUPPORTED, "doublesided wavelets write complex64 outputs only");
    if (P->compat_align && out_type != FCWT_OUT_C64)
        return fail(FCWT_ERR_UNSUPPORTED, "FCWT_COMPAT_ALIGN writes complex64 outputs only");
    int rc = enqueue_forward(P, din, graph_jobs);
    if (rc) return rc;
    FCWT_CUDA_TRY(ctx->err.ensure(sizeof(int)));
    FCWT_CUDA_TRY(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), st));
    std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
    const bool prof = ctx->profiling && allow_profiling;
    if (prof) {
        if (!ctx->ev_free.empty()) {
            ev = ctx->ev_free.back();
            ctx->ev_free.pop_back();
        } else {
            FCWT_CUDA_TRY(cudaEventCreate(&ev.first));
            FCWT_CUDA_TRY(cudaEventCreate(&ev.second));
        }
        FCWT_CUDA_TRY(cudaEventRecord(ev.first, st));
    }
    rc = enqueue_rows(P, P->sigs.as<SigDesc>(), dout, out_type, graph_jobs != nullptr);
    if (rc) return rc;
    if (P->doublesided) {
        // the mirrored half: exp(-2 pi i t / N) conj(V), V the rows on the shifted spectrum
        const PlanSignal& S = P->sig[0];
        const float2* tw = P->tables[(size_t)S.table].tw.as<float2>();
        FCWT_CUDA_TRY(launch_shift_spectrum(S.X.as<float2>(), S.sp.log2N, P->Xs.as<float2>(), st));
        void* tmp_out[1] = {P->ds_tmp.p};
        rc = enqueue_rows(P, P->sigs2.as<SigDesc>(), tmp_out, out_type);
        if (rc) return rc;
        FCWT_CUDA_TRY(launch_doublesided_combine(static_cast<float2*>(dout[0]), P->ds_tmp.as<float2>(),
                                                 S.rows_out(), S.n_out(), S.dec, S.sp.log2N, tw,
                                                 P->imag ? -1.0f : 1.0f, st));
        ctx->kernel_launches += 2;
    }
    if (P->n_shifted > 0) {
        const PlanSignal& S = P->sig[0];
        if (((uintptr_t)dout[0] & 15) != 0)
            return fail(FCWT_ERR_INVALID, "FCWT_COMPAT_ALIGN needs a 16-byte aligned output");
        const float extra = (S.sp.flags & kFlagNorm) ? 1.0f / (float)S.sp.N : 1.0f;
        FCWT_CUDA_TRY(launch_align_spill(P->sigs.as<SigDesc>(), P->rows.as<RowDesc>(), P->shifted.as<int>(),
                                         P->n_shifted, P->pool.as<float>(), static_cast<float2*>(dout[0]), S.sp.n,
                                         extra, st));
        ctx->kernel_launches += 1;
    }
    if (prof) {
        FCWT_CUDA_TRY(cudaEventRecord(ev.second, st));
        ctx->ev_used.push_back(ev);
    }
    FCWT_CUDA_TRY(cudaMemcpyAsync(ctx->err_host, ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    return FCWT_OK;
}

// The forward FFTs of all signals of a plan into their spectra.
int enqueue_forward(fcwt_plan* P, const void* const* din, const fcwt::FwdJob* graph_jobs) {
    using namespace fcwt;
    fcwt_context* ctx = P->ctx;
    cudaStream_t st = ctx->stream;
    const int nsig = (int)P->sig.size();
    if (nsig == 1) {
        PlanSignal& S = P->sig[0];
        FCWT_CUDA_TRY(ctx->tmp.ensure((size_t)S.sp.N * sizeof(float2)));
        int n_fwd = 0;
        FCWT_CUDA_TRY(launch_forward(S.sp.is_complex ? nullptr : (const float*)din[0],
                                     S.sp.is_complex ? (const float2*)din[0] : nullptr, S.sp.n, S.sp.log2N,
                                     P->tables[(size_t)S.table].tw.as<float2>(), S.X.as<float2>(),
                                     ctx->tmp.as<float2>(), st, &n_fwd));
        ctx->kernel_launches += n_fwd;
    } else {
        // batched forward FFTs, one launch sequence per padded length
        std::vector<std::pair<int, int>> groups;
        const FwdJob* djobs = graph_jobs;
        if (!djobs) {
            fcwt_plan::UploadSlot* u = nullptr;
            int rc = upload_slot(P, (size_t)nsig * sizeof(FwdJob), &u);
            if (rc) return rc;
            build_jobs(P, din, groups, static_cast<FwdJob*>(u->host));
            FCWT_CUDA_TRY(cudaMemcpyAsync(P->fwd_jobs.p, u->host, (size_t)nsig * sizeof(FwdJob),
                                          cudaMemcpyHostToDevice, st));
            FCWT_CUDA_TRY(cudaEventRecord(u->done, st));
            u->pending = true;
            djobs = P->fwd_jobs.as<FwdJob>();
        } else {
            job_groups(P, groups);
        }
        int off = 0;
        for (auto& g : groups) {
            int n_fwd = 0;
            FCWT_CUDA_TRY(launch_forward_batched(djobs + off, g.second, P->tables[(size_t)g.first].log2N,
                                                 P->tables[(size_t)g.first].tw.as<float2>(), st, &n_fwd,
                                                 !P->is_complex));
            ctx->kernel_launches += n_fwd;
            off += g.second;
        }
    }
    return FCWT_OK;
}

// The row-engine launches of one pass over the plan's rows, reading the
// spectra of `dsigs` and writing `dout`.
int enqueue_rows(fcwt_plan* P, const fcwt::SigDesc* dsigs, void* const* dout, int out_type, bool graph_maps) {
    using namespace fcwt;
    fcwt_context* ctx = P->ctx;
    cudaStream_t st = ctx->stream;
    const int nsig = (int)P->sig.size();
    const size_t n_counters = plan_counters(P);
    FCWT_CUDA_TRY(ctx->counters.ensure(n_counters * sizeof(unsigned)));
    FCWT_CUDA_TRY(cudaMemsetAsync(ctx->counters.p, 0, n_counters * sizeof(unsigned), st));
    if (P->two_phase)
        FCWT_CUDA_TRY(ctx->scratch.ensure((size_t)P->slots * (size_t)P->slot_elems * sizeof(float2)));
    EngineParams ep;
    std::memset(&ep, 0, sizeof(ep));
    ep.sigs = dsigs;
    ep.rows = P->rows.as<RowDesc>();
    ep.items = P->items.as<Item>();
    ep.n_items = P->n_items;
    ep.stale_pool = P->pool.as<float>();
    ep.scratch = P->two_phase ? ctx->scratch.as<float2>() : nullptr;
    ep.slot_elems = P->slot_elems;
    ep.counters = ctx->counters.as<unsigned>();
    ep.n_rows = P->n_rows;
    for (int s = 0; s < nsig; s++) ep.outs[s] = dout[s];
    ep.out_type = out_type;
    ep.err = ctx->err.as<int>();
    CUtensorMap omap;
    std::memset(&omap, 0, sizeof(omap));
    int map_ok = 0;
    if (nsig == 1 && (P->two_phase || P->n_tc > 0)) {
        const PlanSignal& S = P->sig[0];
        if (out_type == FCWT_OUT_C64)
            map_ok = encode_output_map(dout[0], S.n_out(), S.sp.M / S.dec, S.rows_out(), &omap) ? 1 : 0;
        else
            map_ok = encode_output_map16(dout[0], S.n_out(), S.sp.M / S.dec, S.rows_out(), &omap) ? 1 : 0;
    }
    // the CUDA-core engine's two-phase rows store through the same map
    ep.tma_store = P->two_phase ? map_ok : 0;
    const int grid = std::max(1, std::min(P->n_items, ctx->engine_ctas));
    if (P->n_tc > 0) {
        TcParams tp;
        std::memset(&tp, 0, sizeof(tp));
        tp.sigs = ep.sigs;
        tp.rows = ep.rows;
        tp.row_list = P->tc_units.as<int>();
        tp.n_list = P->n_units;
        tp.stale_pool = ep.stale_pool;
        tp.wts = P->tc_wts.as<float>();
        tp.counter = ctx->counters.as<unsigned>() + n_counters - 1;
        for (int s = 0; s < nsig; s++) tp.outs[s] = dout[s];
        tp.err = ep.err;
        tp.tma_store = map_ok;
        tp.decimated = P->sig.size() == 1 && P->sig[0].dec > 1;
        if (nsig > 1) {
            // one tensor map per output, in device memory
            if (graph_maps) {
                tp.tmaps = P->graph_tmaps.as<CUtensorMap>();
                for (int k = 0; k < kMaxOuts / 64; k++) tp.tmap_mask[k] = P->graph_tmap_mask[(size_t)k];
            } else {
                fcwt_plan::UploadSlot* u = nullptr;
                int rc = upload_slot(P, (size_t)nsig * sizeof(CUtensorMap), &u);
                if (rc) return rc;
                build_output_maps(P, dout, out_type, static_cast<CUtensorMap*>(u->host), tp.tmap_mask);
                FCWT_CUDA_TRY(cudaMemcpyAsync(P->tmaps.p, u->host, (size_t)nsig * sizeof(CUtensorMap),
                                              cudaMemcpyHostToDevice, st));
                FCWT_CUDA_TRY(cudaEventRecord(u->done, st));
                u->pending = true;
                tp.tmaps = P->tmaps.as<CUtensorMap>();
            }
            tp.tma_store = 1;
        }
        FCWT_CUDA_TRY(launch_tc(tp, omap, out_type, std::max(1, std::min(P->n_units, ctx->num_sms)), st));
        ctx->kernel_launches += 1;
    }
    if (P->n_items > 0) {
        FCWT_CUDA_TRY(launch_engine(ep, omap, grid, st));
        ctx->kernel_launches += 1;
    }
    return FCWT_OK;
}

// Host-output pipeline of a single-signal plan whose rows all run on the
// tensor-core engine (rows independent of each other): rows are transformed
// in blocks of about kPipeBlockBytes of output into two device staging slots,
// and block b is copied to the host on a second stream while block b + 1 is
// computed. Device staging is two blocks instead of the whole output, and
// the transform overlaps the (PCIe-bound) copy.
constexpr size_t kPipeBlockBytes = 256ull << 20;

bool pipeline_applies(const fcwt_plan* P, size_t out_bytes) {
    return P->sig.size() == 1 && P->n_items == 0 && P->n_tc == P->n_rows && !P->doublesided &&
           P->n_shifted == 0 && out_bytes > kPipeBlockBytes;
}

int run_pipelined(fcwt_plan* P, const void* din, void* hout, int out_type) {
    using namespace fcwt;
    fcwt_context* ctx = P->ctx;
    cudaStream_t st = ctx->stream;
    const PlanSignal& S = P->sig[0];
    const size_t esz = out_elem_bytes(out_type);
    const size_t row_bytes = (size_t)S.n_out() * esz;
    const int rows = P->n_rows;
    const int blk = (int)std::max<size_t>(1, kPipeBlockBytes / row_bytes);
    const int nblk = (rows + blk - 1) / blk;
    FCWT_CUDA_TRY(ctx->out_stage.ensure(2 * (size_t)blk * row_bytes + 256));
    if (!ctx->copy_stream) FCWT_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; i++) {
        if (!ctx->pipe_done[i]) FCWT_CUDA_TRY(cudaEventCreateWithFlags(&ctx->pipe_done[i], cudaEventDisableTiming));
        if (!ctx->pipe_copied[i])
            FCWT_CUDA_TRY(cudaEventCreateWithFlags(&ctx->pipe_copied[i], cudaEventDisableTiming));
    }
    const void* din_arr[1] = {din};
    int rc = enqueue_forward(P, din_arr, nullptr);
    if (rc) return rc;
    FCWT_CUDA_TRY(ctx->err.ensure(sizeof(int)));
    FCWT_CUDA_TRY(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), st));
    FCWT_CUDA_TRY(ctx->counters.ensure((size_t)nblk * sizeof(unsigned)));
    FCWT_CUDA_TRY(cudaMemsetAsync(ctx->counters.p, 0, (size_t)nblk * sizeof(unsigned), st));
    std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
    const bool prof = ctx->profiling;
    if (prof) {
        if (!ctx->ev_free.empty()) {
            ev = ctx->ev_free.back();
            ctx->ev_free.pop_back();
        } else {
            FCWT_CUDA_TRY(cudaEventCreate(&ev.first));
            FCWT_CUDA_TRY(cudaEventCreate(&ev.second));
        }
        FCWT_CUDA_TRY(cudaEventRecord(ev.first, st));
    }
    const size_t slot_bytes = (size_t)blk * row_bytes;
    for (int b = 0; b < nblk; b++) {
        const int slot = b & 1;
        const int r0 = b * blk, r1 = std::min(rows, r0 + blk);
        char* stage = static_cast<char*>(ctx->out_stage.p) + (size_t)slot * slot_bytes;
        // the slot is free once the copy of block b - 2 is done
        if (b >= 2) FCWT_CUDA_TRY(cudaStreamWaitEvent(st, ctx->pipe_copied[slot], 0));
        // rows r0.. of the plan write at out_off = r * row elements: shift the base so they land in the
        // slot (an address below the slot that no access uses; only base + out_off is dereferenced)
        char* base = reinterpret_cast<char*>(reinterpret_cast<uintptr_t>(stage) - (uintptr_t)r0 * row_bytes);
        CUtensorMap omap;
        std::memset(&omap, 0, sizeof(omap));
        const int map_ok = out_type == FCWT_OUT_C64
                               ? (encode_output_map(base, S.n_out(), S.sp.M / S.dec, r1, &omap) ? 1 : 0)
                               : (encode_output_map16(base, S.n_out(), S.sp.M / S.dec, r1, &omap) ? 1 : 0);
        TcParams tp;
        std::memset(&tp, 0, sizeof(tp));
        tp.sigs = P->sigs.as<SigDesc>();
        tp.rows = P->rows.as<RowDesc>();
        tp.row_list = P->tc_rows.as<int>() + r0;  // tc_rows lists the rows in order
        tp.n_list = r1 - r0;
        tp.stale_pool = P->pool.as<float>();
        tp.wts = P->tc_wts.as<float>();
        tp.counter = ctx->counters.as<unsigned>() + b;
        tp.outs[0] = base;
        tp.err = ctx->err.as<int>();
        tp.tma_store = map_ok;
        tp.decimated = P->sig.size() == 1 && P->sig[0].dec > 1;
        FCWT_CUDA_TRY(launch_tc(tp, omap, out_type, std::max(1, std::min(r1 - r0, ctx->num_sms)), st));
        ctx->kernel_launches += 1;
        FCWT_CUDA_TRY(cudaEventRecord(ctx->pipe_done[slot], st));
        FCWT_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ctx->pipe_done[slot], 0));
        FCWT_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(hout) + (size_t)r0 * row_bytes, stage,
                                      (size_t)(r1 - r0) * row_bytes, cudaMemcpyDeviceToHost, ctx->copy_stream));
        FCWT_CUDA_TRY(cudaEventRecord(ctx->pipe_copied[slot], ctx->copy_stream));
    }
    if (prof) {
        FCWT_CUDA_TRY(cudaEventRecord(ev.second, st));
        ctx->ev_used.push_back(ev);
    }
    FCWT_CUDA_TRY(cudaMemcpyAsync(ctx->err_host, ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    FCWT_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
    FCWT_CUDA_TRY(cudaStreamSynchronize(st));
    if (*ctx->err_host != 0)
        return fail(FCWT_ERR_DEVICE, "row engine reported error bits " + std::to_string(*ctx->err_host));
    return FCWT_OK;
}

// Runs a plan on host or device buffers: host inputs are staged in, host
// outputs are copied back (and the call waits for them).
int plan_run_multi(fcwt_plan* P, const void* const* inputs, void* const* outputs, int out_type) {
    using namespace fcwt;
    fcwt_context* ctx = P->ctx;
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (out_type < FCWT_OUT_C64 || out_type > FCWT_OUT_DB)
        return fail(FCWT_ERR_INVALID, "unknown output type");
    if (P->n_rows == 0) return FCWT_OK;
    const int nsig = (int)P->sig.size();
    if (!inputs || !outputs) return fail(FCWT_ERR_INVALID, "null input or output array");
    cudaStream_t st = ctx->stream;
    std::vector<const void*> din((size_t)nsig);
    std::vector<void*> dout((size_t)nsig);
    std::vector<size_t> out_bytes((size_t)nsig), out_off((size_t)nsig);
    size_t in_total = 0, out_total = 0;
    std::vector<size_t> in_off((size_t)nsig);
    for (int s = 0; s < nsig; s++) {
        const PlanSignal& S = P->sig[(size_t)s];
        if (S.re == S.rb || S.sp.n == 0) continue;
        if (!inputs[s] || !outputs[s]) return fail(FCWT_ERR_INVALID, "null input or output pointer");
        rc = check_pointer_devices({inputs[s], outputs[s]}, ctx->device);
        if (rc) return rc;
        in_off[(size_t)s] = in_total;
        if (!is_device_pointer(inputs[s])) in_total += ((size_t)S.sp.n * (S.sp.is_complex ? 8 : 4) + 255) & ~(size_t)255;
        out_off[(size_t)s] = out_total;
        out_bytes[(size_t)s] = (size_t)S.rows_out() * (size_t)S.n_out() * out_elem_bytes(out_type);
        if (!is_device_pointer(outputs[s])) out_total += (out_bytes[(size_t)s] + 255) & ~(size_t)255;
    }
    if (nsig == 1 && !is_device_pointer(outputs[0]) && pipeline_applies(P, out_bytes[0])) {
        const PlanSignal& S = P->sig[0];
        const void* din0 = inputs[0];
        if (!is_device_pointer(inputs[0])) {
            FCWT_CUDA_TRY(ctx->in_stage.ensure(in_total));
            FCWT_CUDA_TRY(cudaMemcpyAsync(ctx->in_stage.p, inputs[0], (size_t)S.sp.n * (S.sp.is_complex ? 8 : 4),
                                          cudaMemcpyHostToDevice, st));
            din0 = ctx->in_stage.p;
        }
        return run_pipelined(P, din0, outputs[0], out_type);
    }
    if (in_total) FCWT_CUDA_TRY(ctx->in_stage.ensure(in_total));
    if (out_total) FCWT_CUDA_TRY(ctx->out_stage.ensure(out_total));
    bool any_host_out = false;
    for (int s = 0; s < nsig; s++) {
        const PlanSignal& S = P->sig[(size_t)s];
        din[(size_t)s] = inputs[s];
        dout[(size_t)s] = outputs[s];
        if (S.re == S.rb || S.sp.n == 0) continue;
        if (!is_device_pointer(inputs[s])) {
            void* d = (char*)ctx->in_stage.p + in_off[(size_t)s];
            FCWT_CUDA_TRY(cudaMemcpyAsync(d, inputs[s], (size_t)S.sp.n * (S.sp.is_complex ? 8 : 4),
                                          cudaMemcpyHostToDevice, st));
            din[(size_t)s] = d;
        }
        if (!is_device_pointer(outputs[s])) {
            dout[(size_t)s] = (char*)ctx->out_stage.p + out_off[(size_t)s];
            any_host_out = true;
        }
    }
    rc = plan_enqueue(P, din.data(), dout.data(), out_type, true);
    if (rc) return rc;
    if (any_host_out) {
        for (int s = 0; s < nsig; s++)
            if (dout[(size_t)s] != outputs[s] && out_bytes[(size_t)s])
                FCWT_CUDA_TRY(cudaMemcpyAsync(outputs[s], dout[(size_t)s], out_bytes[(size_t)s], cudaMemcpyDeviceToHost, st));
        FCWT_CUDA_TRY(cudaStreamSynchronize(st));
        if (*ctx->err_host != 0)
            return fail(FCWT_ERR_DEVICE, "row engine reported error bits " + std::to_string(*ctx->err_host));
    }
    return FCWT_OK;
}

int plan_run(fcwt_plan* P, const void* input, void* output, int out_type) {
    return plan_run_multi(P, &input, &output, out_type);
}

bool key_match(const fcwt_context::CacheEntry& e, int n, int cplx, float fb, const float* scales, int fn,
               int threads, unsigned flags) {
    return e.n == n && e.is_complex == cplx && e.fb == fb && e.fn == fn && e.threads == threads &&
           e.flags == flags && std::memcmp(e.scales.data(), scales, sizeof(float) * (size_t)fn) == 0;
}

int cached_plan(fcwt_context* ctx, int n, int cplx, float fb, const float* scales, int fn, int threads,
                unsigned flags, fcwt_plan** out) {
    for (auto& e : ctx->cache) {
        if (key_match(e, n, cplx, fb, scales, fn, threads, flags)) {
            e.last_use = ++ctx->use_clock;
            *out = e.plan;
            return FCWT_OK;
        }
    }
    fcwt_plan* p = nullptr;
    int rc = fcwt_plan_create(ctx, n, cplx, fb, scales, fn, threads, flags, 0, fn, &p);
    if (rc) return rc;
    if (ctx->cache.size() >= 4) {
        auto victim = std::min_element(ctx->cache.begin(), ctx->cache.end(),
                                       [](const auto& a, const auto& b) { return a.last_use < b.last_use; });
        fcwt_plan_destroy(victim->plan);
        ctx->cache.erase(victim);
    }
    fcwt_context::CacheEntry e;
    e.n = n;
    e.is_complex = cplx;
    e.fn = fn;
    e.threads = threads;
    e.flags = flags;
    e.fb = fb;
    e.scales.assign(scales, scales + fn);
    e.plan = p;
    e.last_use = ++ctx->use_clock;
    ctx->cache.push_back(std::move(e));
    *out = p;
    return FCWT_OK;
}

int transform(fcwt_context* ctx, const float* input, int n, int cplx, float fb, const float* scales, int fn,
              int threads, unsigned flags, void* output, int out_type) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (n < 0 || fn < 0) return fail(FCWT_ERR_INVALID, "negative size");
    if (n == 0 || fn == 0) return FCWT_OK;
    if (!scales) return fail(FCWT_ERR_INVALID, "null scales");
    fcwt_plan* p = nullptr;
    rc = cached_plan(ctx, n, cplx, fb, scales, fn, threads, flags, &p);
    if (rc) return rc;
    return plan_run(p, input, output, out_type);
}

std::string tune_path(const char* dir, int N, int threads) {
    std::string d = dir && *dir ? std::string(dir) : std::string(".");
    if (d.back() != '/') d += '/';
    return d + "n" + std::to_string(N) + "_t" + std::to_string(threads) + ".wis";
}

}  // namespace

namespace fcwt {
// Lets other translation units of the library set the message that
// fcwt_last_error() returns for the calling thread.
void record_error(const std::string& msg) { g_err = msg; }
}  // namespace fcwt

// =================================================================== C ABI

extern "C" {

int fcwt_version(void) { return 100; }

const char* fcwt_last_error(void) { return g_err.c_str(); }

int fcwt_context_create(int device, fcwt_context** out) {
    if (!out) return fail(FCWT_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int count = 0;
    FCWT_CUDA_TRY(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(FCWT_ERR_INVALID, "no such CUDA device");
    FCWT_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    FCWT_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(FCWT_ERR_UNSUPPORTED, "this library is built for sm_100a (B200) only");
    fcwt_context* c = new fcwt_context();
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&c->err_host, sizeof(int));
    if (e == cudaSuccess) e = fcwt::engine_configure();
    if (e == cudaSuccess) e = fcwt::tc_configure();
    int per_sm = 0;
    if (e == cudaSuccess) e = fcwt::engine_blocks_per_sm(&per_sm);
    c->engine_ctas = std::max(1, per_sm) * c->num_sms;
    if (e != cudaSuccess) {
        if (c->own) cudaStreamDestroy(c->own);
        if (c->err_host) cudaFreeHost(c->err_host);
        delete c;
        return fail(FCWT_ERR_CUDA, std::string("context setup: ") + cudaGetErrorString(e));
    }
    *c->err_host = 0;
    c->stream = c->own;
    *out = c;
    return FCWT_OK;
}

int fcwt_context_destroy(fcwt_context* ctx) {
    if (!ctx) return FCWT_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& e : ctx->cache) plan_free(e.plan);
    ctx->cache.clear();
    // plans the caller still holds: free their resources now, keep the handles
    // valid (fcwt_plan_destroy on them only frees the handle)
    for (fcwt_plan* p : ctx->plans) {
        plan_release(p);
        p->ctx = nullptr;
    }
    ctx->plans.clear();
    ctx->in_stage.release();
    ctx->out_stage.release();
    ctx->tmp.release();
    ctx->scratch.release();
    ctx->counters.release();
    ctx->err.release();
    if (ctx->err_host) cudaFreeHost(ctx->err_host);
    for (DevBuf* b : {&ctx->adj_tw, &ctx->adj_x, &ctx->adj_g, &ctx->adj_tmp, &ctx->adj_h, &ctx->adj_jobs,
                      &ctx->adj_rows, &ctx->adj_acc})
        b->release();
    if (ctx->adj_jobs_host) cudaFreeHost(ctx->adj_jobs_host);
    for (auto& ev : ctx->ev_used) {
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    for (auto& ev : ctx->ev_free) {
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    for (int i = 0; i < 2; i++) {
        if (ctx->pipe_done[i]) cudaEventDestroy(ctx->pipe_done[i]);
        if (ctx->pipe_copied[i]) cudaEventDestroy(ctx->pipe_copied[i]);
    }
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return FCWT_OK;
}

int fcwt_context_set_stream(fcwt_context* ctx, void* stream) {
    if (!ctx) return fail(FCWT_ERR_INVALID, "null context");
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
    return FCWT_OK;
}

int fcwt_context_set_engine(fcwt_context* ctx, int mode) {
    if (!ctx) return fail(FCWT_ERR_INVALID, "null context");
    if (mode != FCWT_ENGINE_AUTO && mode != FCWT_ENGINE_CUDA_CORES && mode != FCWT_ENGINE_TENSOR_CORES)
        return fail(FCWT_ERR_INVALID, "unknown engine mode");
    if (mode != ctx->engine_mode) {
        // cached plans were built for the previous mode
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto& e : ctx->cache) plan_free(e.plan);
        ctx->cache.clear();
        ctx->engine_mode = mode;
    }
    return FCWT_OK;
}

int fcwt_synchronize(fcwt_context* ctx) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    FCWT_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (*ctx->err_host != 0) {
        int bits = *ctx->err_host;
        *ctx->err_host = 0;
        return fail(FCWT_ERR_DEVICE, "row engine reported error bits " + std::to_string(bits));
    }
    return FCWT_OK;
}

int fcwt_profile_enable(fcwt_context* ctx, int enable) {
    if (!ctx) return fail(FCWT_ERR_INVALID, "null context");
    ctx->profiling = enable != 0;
    return FCWT_OK;
}

int fcwt_profile_read(fcwt_context* ctx, double* engine_ms, int* engine_launches, int* kernel_launches) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    double total = 0.0;
    int count = 0;
    for (auto& ev : ctx->ev_used) {
        FCWT_CUDA_TRY(cudaEventSynchronize(ev.second));
        float ms = 0.0f;
        FCWT_CUDA_TRY(cudaEventElapsedTime(&ms, ev.first, ev.second));
        total += ms;
        count++;
        ctx->ev_free.push_back(ev);
    }
    ctx->ev_used.clear();
    if (engine_ms) *engine_ms = total;
    if (engine_launches) *engine_launches = count;
    if (kernel_launches) *kernel_launches = (int)ctx->kernel_launches;
    ctx->kernel_launches = 0;
    return FCWT_OK;
}

int fcwt_find2power(int n) { return fcwt::host::find2power(n); }

int fcwt_scales(int scaletype, int fs, float f0, float f1, int fn, float* out) {
    if (fn < 0 || (fn > 0 && !out)) return fail(FCWT_ERR_INVALID, "bad scales output");
    if (scaletype < 0 || scaletype > 2) return fail(FCWT_ERR_INVALID, "unknown scale type");
    fcwt::host::scales(scaletype, fs, f0, f1, fn, out);
    return FCWT_OK;
}

int fcwt_scales_checked(int scaletype, int fs, float f0, float f1, int fn, unsigned flags, float* out) {
    if (flags & FCWT_STRICT) {
        if (f1 > (float)fs / 2.0f)
            return fail(FCWT_ERR_INVALID, "f1 = " + std::to_string(f1) + " Hz is above the Nyquist rate fs/2 = " +
                                              std::to_string((float)fs / 2.0f) + " Hz");
        if (scaletype == FCWT_LOGSCALES && !(f0 < f1)) return fail(FCWT_ERR_INVALID, "LOGSCALES needs f0 < f1");
    }
    return fcwt_scales(scaletype, fs, f0, f1, fn, out);
}

int fcwt_frequencies(const float* scales, int fn, int fs, float* out) {
    if (fn < 0 || (fn > 0 && (!out || !scales))) return fail(FCWT_ERR_INVALID, "bad arguments");
    fcwt::host::frequencies(scales, fn, fs, out);
    return FCWT_OK;
}

int fcwt_morlet_support(float fb, float scale) { return fcwt::host::morlet_support(fb, scale); }

int fcwt_morlet_time(float fb, float scale, int size, float* real, float* imag) {
    if (!real || !imag) return fail(FCWT_ERR_INVALID, "null output");
    fcwt::host::morlet_time(fb, scale, size, real, imag);
    return FCWT_OK;
}

int fcwt_morlet_wavelet(float fb, float scale, float* out, int pn) {
    if (pn < 0 || (pn > 0 && !out)) return fail(FCWT_ERR_INVALID, "bad output");
    fcwt::host::morlet_wavelet(fb, scale, pn, out);
    return FCWT_OK;
}

int fcwt_morlet_mother_host(float fb, int N, float* out) {
    if (N < 0 || (N > 0 && !out)) return fail(FCWT_ERR_INVALID, "bad output");
    fcwt::host::mother_table(fb, N, out);
    return FCWT_OK;
}

int fcwt_row_truncation(int n, float fb, const float* scales, int fn, int threads, unsigned flags,
                        int* proc_out, int* lo_out, int* hi_out) {
    if (fn < 0 || (fn > 0 && (!scales || !proc_out))) return fail(FCWT_ERR_INVALID, "bad arguments");
    fcwt::SignalPlan sp;
    std::string err;
    if (fcwt::plan_signal(n, false, fb, scales, fn, threads, flags, sp, err))
        return fail(FCWT_ERR_INVALID, err);
    for (int i = 0; i < fn; i++) {
        proc_out[i] = sp.rows[(size_t)i].proc;
        if (lo_out) lo_out[i] = sp.rows[(size_t)i].lo;
        if (hi_out) hi_out[i] = sp.rows[(size_t)i].hi;
    }
    return FCWT_OK;
}

int fcwt_morlet_mother(fcwt_context* ctx, float fb, int N, float* out) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (N <= 0 || !out) return fail(FCWT_ERR_INVALID, "bad arguments");
    if (!(fb > 0.0f)) return fail(FCWT_ERR_INVALID, "bandwidth must be positive");
    rc = check_pointer_devices({out}, ctx->device);
    if (rc) return rc;
    if (is_device_pointer(out)) {
        FCWT_CUDA_TRY(fcwt::launch_mother(fb, N, fcwt::host::mother_norm(), out, ctx->stream));
        return FCWT_OK;
    }
    DevBuf tmp;
    FCWT_CUDA_TRY(tmp.ensure((size_t)N * sizeof(float)));
    cudaError_t e = fcwt::launch_mother(fb, N, fcwt::host::mother_norm(), tmp.as<float>(), ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, tmp.p, (size_t)N * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    tmp.release();
    if (e != cudaSuccess) return fail(FCWT_ERR_CUDA, cudaGetErrorString(e));
    return FCWT_OK;
}

int fcwt_plan_create(fcwt_context* ctx, int n, int is_complex, float fb, const float* scales, int fn,
                     int threads, unsigned flags, int row_begin, int row_end, fcwt_plan** out) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (!out) return fail(FCWT_ERR_INVALID, "null plan output");
    *out = nullptr;
    if (fn < 0 || n < 0) return fail(FCWT_ERR_INVALID, "negative size");
    if (fn > 0 && !scales) return fail(FCWT_ERR_INVALID, "null scales");
    if (row_begin < 0 || row_end > fn || row_begin > row_end)
        return fail(FCWT_ERR_INVALID, "row range outside [0, fn]");
    fcwt_plan* P = plan_new(ctx);
    P->fb = fb;
    P->is_complex = is_complex != 0;
    P->sig.resize(1);
    P->sig[0].rb = row_begin;
    P->sig[0].re = row_end;
    P->compat_align = (flags & FCWT_COMPAT_ALIGN) != 0;
    if (P->compat_align && (row_begin != 0 || row_end != fn)) {
        plan_free(P);
        return fail(FCWT_ERR_UNSUPPORTED, "FCWT_COMPAT_ALIGN applies to whole plans (all rows)");
    }
    std::string err;
    if (fcwt::plan_signal(n, is_complex != 0, fb, scales, fn, threads, flags, P->sig[0].sp, err)) {
        plan_free(P);
        return fail(FCWT_ERR_INVALID, err);
    }
    rc = plan_build(P);
    if (rc) {
        std::string keep = g_err;
        plan_free(P);
        g_err = keep;
        return rc;
    }
    *out = P;
    return FCWT_OK;
}

int fcwt_plan_create_strided(fcwt_context* ctx, int n, int is_complex, float fb, const float* scales, int fn,
                             int threads, unsigned flags, int row_begin, int row_end, int row_stride,
                             int time_stride, fcwt_plan** out) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (!out) return fail(FCWT_ERR_INVALID, "null plan output");
    *out = nullptr;
    if (row_stride < 1) return fail(FCWT_ERR_INVALID, "row_stride must be >= 1");
    if (time_stride < 1 || (time_stride & (time_stride - 1)))
        return fail(FCWT_ERR_INVALID, "time_stride must be a power of two >= 1");
    if (flags & FCWT_COMPAT_ALIGN) return fail(FCWT_ERR_UNSUPPORTED, "FCWT_COMPAT_ALIGN with decimation");
    if (fn < 0 || n < 0) return fail(FCWT_ERR_INVALID, "negative size");
    if (fn > 0 && !scales) return fail(FCWT_ERR_INVALID, "null scales");
    if (row_begin < 0 || row_end > fn || row_begin > row_end)
        return fail(FCWT_ERR_INVALID, "row range outside [0, fn]");
    fcwt_plan* P = plan_new(ctx);
    P->fb = fb;
    P->is_complex = is_complex != 0;
    P->sig.resize(1);
    P->sig[0].rb = row_begin;
    P->sig[0].re = row_end;
    P->sig[0].rstride = row_stride;
    P->sig[0].dec = time_stride;
    std::string err;
    if (fcwt::plan_signal(n, is_complex != 0, fb, scales, fn, threads, flags, P->sig[0].sp, err)) {
        plan_free(P);
        return fail(FCWT_ERR_INVALID, err);
    }
    if (time_stride > std::max(1, n)) {
        plan_free(P);
        return fail(FCWT_ERR_INVALID, "time_stride larger than the signal");
    }
    rc = plan_build(P);
    if (rc) {
        std::string keep = g_err;
        plan_free(P);
        g_err = keep;
        return rc;
    }
    *out = P;
    return FCWT_OK;
}

int fcwt_plan_output_shape(const fcwt_plan* plan, int* rows, int* cols) {
    if (!plan) return fail(FCWT_ERR_INVALID, "null plan");
    if (plan->sig.size() != 1) return fail(FCWT_ERR_INVALID, "batched plans have one shape per signal");
    if (rows) *rows = plan->sig[0].rows_out();
    if (cols) *cols = plan->sig[0].n_out();
    return FCWT_OK;
}

int fcwt_plan_create_mother(fcwt_context* ctx, int n, int is_complex, const float* mother, int mother_size,
                            const float* scales, int fn, int threads, unsigned flags, int row_begin, int row_end,
                            fcwt_plan** out) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (!out) return fail(FCWT_ERR_INVALID, "null plan output");
    *out = nullptr;
    if (fn < 0 || n < 0) return fail(FCWT_ERR_INVALID, "negative size");
    if (fn > 0 && !scales) return fail(FCWT_ERR_INVALID, "null scales");
    if (row_begin < 0 || row_end > fn || row_begin > row_end)
        return fail(FCWT_ERR_INVALID, "row range outside [0, fn]");
    if (flags & FCWT_CONTINUOUS) return fail(FCWT_ERR_INVALID, "FCWT_CONTINUOUS is the Morlet's own mode");
    const int log2N = fcwt::host::find2power(n);
    if (log2N > fcwt::kMaxLog2N) return fail(FCWT_ERR_INVALID, "signal too long: padded length exceeds 2^23");
    const int N = 1 << log2N;
    if (!mother || mother_size != N)
        return fail(FCWT_ERR_INVALID, "the mother table must hold N = 2^find2power(n) = " + std::to_string(N) +
                                          " values");
    for (int i = 0; i < N; i++)
        if (!std::isfinite(mother[i])) return fail(FCWT_ERR_INVALID, "the mother table holds a non-finite value");
    if ((flags & FCWT_DOUBLESIDED) && N < 2) return fail(FCWT_ERR_INVALID, "doublesided wavelets need n >= 2");
    fcwt_plan* P = plan_new(ctx);
    P->fb = 1.0f;
    P->is_complex = is_complex != 0;
    P->custom_mother.assign(mother, mother + N);
    P->imag = (flags & FCWT_IMAG_FREQUENCY) != 0;
    P->doublesided = (flags & FCWT_DOUBLESIDED) != 0;
    P->compat_align = (flags & FCWT_COMPAT_ALIGN) != 0;
    if (P->compat_align && (P->doublesided || row_begin != 0 || row_end != fn)) {
        plan_free(P);
        return fail(FCWT_ERR_UNSUPPORTED, "FCWT_COMPAT_ALIGN applies to whole plans of single-sided wavelets");
    }
    P->sig.resize(1);
    P->sig[0].rb = row_begin;
    P->sig[0].re = row_end;
    std::string err;
    if (fcwt::plan_signal(n, is_complex != 0, 1.0f, scales, fn, threads, flags, P->sig[0].sp, err, mother)) {
        plan_free(P);
        return fail(FCWT_ERR_INVALID, err);
    }
    rc = plan_build(P);
    if (rc) {
        std::string keep = g_err;
        plan_free(P);
        g_err = keep;
        return rc;
    }
    *out = P;
    return FCWT_OK;
}

int fcwt_cwt_mother(fcwt_context* ctx, const void* input, int n, int is_complex, const float* mother,
                    int mother_size, const float* scales, int fn, int threads, unsigned flags, void* output,
                    int out_type) {
    fcwt_plan* P = nullptr;
    int rc = fcwt_plan_create_mother(ctx, n, is_complex, mother, mother_size, scales, fn, threads, flags, 0, fn, &P);
    if (rc) return rc;
    rc = plan_run(P, input, output, out_type);
    std::string keep = g_err;
    fcwt_plan_destroy(P);
    g_err = keep;
    return rc;
}

int fcwt_plan_create_batched(fcwt_context* ctx, int nsig, const int* ns, int is_complex, float fb,
                             const float* const* scales, const int* fns, int threads, unsigned flags,
                             fcwt_plan** out) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (!out) return fail(FCWT_ERR_INVALID, "null plan output");
    *out = nullptr;
    if (nsig < 1 || nsig > fcwt::kMaxOuts) return fail(FCWT_ERR_INVALID, "nsig must be in [1, 1024]");
    if (!ns || !scales || !fns) return fail(FCWT_ERR_INVALID, "null array argument");
    fcwt_plan* P = plan_new(ctx);
    P->fb = fb;
    P->is_complex = is_complex != 0;
    P->sig.resize((size_t)nsig);
    for (int s = 0; s < nsig; s++) {
        if (ns[s] < 0 || fns[s] < 0 || (fns[s] > 0 && !scales[s])) {
            plan_free(P);
            return fail(FCWT_ERR_INVALID, "bad size or scales of signal " + std::to_string(s));
        }
        std::string err;
        if (fcwt::plan_signal(ns[s], is_complex != 0, fb, scales[s], fns[s], threads, flags, P->sig[(size_t)s].sp,
                              err)) {
            plan_free(P);
            return fail(FCWT_ERR_INVALID, "signal " + std::to_string(s) + ": " + err);
        }
        P->sig[(size_t)s].rb = 0;
        P->sig[(size_t)s].re = fns[s];
    }
    rc = plan_build(P);
    if (rc) {
        std::string keep = g_err;
        plan_free(P);
        g_err = keep;
        return rc;
    }
    *out = P;
    return FCWT_OK;
}

int fcwt_plan_execute(fcwt_plan* plan, const void* input, void* output, int out_type) {
    if (!plan) return fail(FCWT_ERR_INVALID, "null plan");
    if (!plan->ctx) return fail(FCWT_ERR_INVALID, "the plan's context was destroyed");
    if (plan->sig.size() != 1) return fail(FCWT_ERR_INVALID, "batched plan: use fcwt_plan_execute_batched");
    return plan_run(plan, input, output, out_type);
}

int fcwt_plan_execute_batched(fcwt_plan* plan, const void* const* inputs, void* const* outputs, int out_type) {
    if (!plan) return fail(FCWT_ERR_INVALID, "null plan");
    if (!plan->ctx) return fail(FCWT_ERR_INVALID, "the plan's context was destroyed");
    return plan_run_multi(plan, inputs, outputs, out_type);
}

int fcwt_plan_execute_graph(fcwt_plan* plan, const void* const* inputs, void* const* outputs, int out_type) {
    if (!plan) return fail(FCWT_ERR_INVALID, "null plan");
    if (!plan->ctx) return fail(FCWT_ERR_INVALID, "the plan's context was destroyed");
    fcwt_context* ctx = plan->ctx;
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (out_type < FCWT_OUT_C64 || out_type > FCWT_OUT_DB)
        return fail(FCWT_ERR_INVALID, "unknown output type");
    if (!inputs || !outputs) return fail(FCWT_ERR_INVALID, "null input or output array");
    const int nsig = (int)plan->sig.size();
    std::vector<const void*> key;
    for (int s = 0; s < nsig; s++) {
        rc = check_pointer_devices({inputs[s], outputs[s]}, ctx->device);
        if (rc) return rc;
        if (!is_device_pointer(inputs[s]) || !is_device_pointer(outputs[s]))
            return fail(FCWT_ERR_INVALID, "graph execution needs device inputs and outputs");
        key.push_back(inputs[s]);
        key.push_back(outputs[s]);
    }
    cudaStream_t st = ctx->stream;
    if (!plan->graph || key != plan->graph_key || out_type != plan->graph_out_type) {
        if (plan->graph) {
            cudaGraphExecDestroy(plan->graph);
            plan->graph = nullptr;
        }
        // make sure every buffer the enqueue touches exists before capturing
        size_t maxN = 1;
        for (auto& S : plan->sig) maxN = std::max(maxN, (size_t)S.sp.N);
        FCWT_CUDA_TRY(ctx->tmp.ensure(maxN * sizeof(float2)));
        FCWT_CUDA_TRY(ctx->counters.ensure(plan_counters(plan) * sizeof(unsigned)));
        FCWT_CUDA_TRY(ctx->err.ensure(sizeof(int)));
        if (plan->two_phase)
            FCWT_CUDA_TRY(ctx->scratch.ensure((size_t)plan->slots * (size_t)plan->slot_elems * sizeof(float2)));
        const fcwt::FwdJob* gj = nullptr;
        if (nsig > 1) {
            // the graph reads its jobs and tensor maps from buffers of its own,
            // filled once here (synchronously, before the capture)
            std::vector<std::pair<int, int>> groups;
            std::vector<fcwt::FwdJob> jobs((size_t)nsig);
            build_jobs(plan, inputs, groups, jobs.data());
            FCWT_CUDA_TRY(plan->graph_jobs.ensure((size_t)nsig * sizeof(fcwt::FwdJob)));
            FCWT_CUDA_TRY(cudaMemcpy(plan->graph_jobs.p, jobs.data(), (size_t)nsig * sizeof(fcwt::FwdJob),
                                     cudaMemcpyHostToDevice));
            std::vector<CUtensorMap> maps((size_t)nsig);
            build_output_maps(plan, outputs, out_type, maps.data(), plan->graph_tmap_mask.data());
            FCWT_CUDA_TRY(plan->graph_tmaps.ensure((size_t)nsig * sizeof(CUtensorMap)));
            FCWT_CUDA_TRY(cudaMemcpy(plan->graph_tmaps.p, maps.data(), (size_t)nsig * sizeof(CUtensorMap),
                                     cudaMemcpyHostToDevice));
            gj = plan->graph_jobs.as<fcwt::FwdJob>();
        }
        // capture on the context's own stream (the legacy default stream
        // cannot be captured); the graph is then launched on the caller's
        FCWT_CUDA_TRY(cudaStreamSynchronize(st));
        cudaGraph_t g = nullptr;
        cudaStream_t user = ctx->stream;
        ctx->stream = ctx->own;
        cudaError_t e = cudaStreamBeginCapture(ctx->own, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            ctx->stream = user;
            return fail(FCWT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        }
        rc = plan_enqueue(plan, inputs, outputs, out_type, false, gj);
        e = cudaStreamEndCapture(ctx->own, &g);
        ctx->stream = user;
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail(FCWT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&plan->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            plan->graph = nullptr;
            return fail(FCWT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        plan->graph_key = key;
        plan->graph_out_type = out_type;
    }
    FCWT_CUDA_TRY(cudaGraphLaunch(plan->graph, st));
    return FCWT_OK;
}

int fcwt_plan_stats(const fcwt_plan* plan, int* rows, int* tensor_core_rows) {
    if (!plan) return fail(FCWT_ERR_INVALID, "null plan");
    if (rows) *rows = plan->n_rows;
    if (tensor_core_rows) *tensor_core_rows = plan->n_tc;
    return FCWT_OK;
}

int fcwt_plan_destroy(fcwt_plan* plan) {
    if (!plan) return FCWT_OK;
    fcwt_context* ctx = plan->ctx;
    if (ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
    }
    plan_free(plan);
    return FCWT_OK;
}

int fcwt_cwt(fcwt_context* ctx, const float* input, int n, float fb, const float* scales, int fn, int threads,
             unsigned flags, void* output, int out_type) {
    return transform(ctx, input, n, 0, fb, scales, fn, threads, flags, output, out_type);
}

int fcwt_ccwt(fcwt_context* ctx, const float* input, int n, float fb, const float* scales, int fn,
              int threads, unsigned flags, void* output, int out_type) {
    return transform(ctx, input, n, 1, fb, scales, fn, threads, flags, output, out_type);
}

int fcwt_morlet_cwt_backward(fcwt_context* ctx, const float* x, int n, int batch, float fb, const float* freqs,
                             int fn, float fs, unsigned flags, const void* grad_out, float* grad_x, double* grad_fb,
                             double* grad_freqs) {
    using namespace fcwt;
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (n < 0 || batch < 0 || fn < 0) return fail(FCWT_ERR_INVALID, "negative size");
    if (!(fb > 0.0f) || !(fs > 0.0f)) return fail(FCWT_ERR_INVALID, "fb and fs must be positive");
    if (grad_fb) *grad_fb = 0.0;
    if (grad_freqs)
        for (int i = 0; i < fn; i++) grad_freqs[i] = 0.0;
    if (n == 0 || batch == 0) return FCWT_OK;
    if (!x || !grad_out || !grad_x || (fn > 0 && !freqs))
        return fail(FCWT_ERR_INVALID, "null pointer argument");
    rc = check_pointer_devices({x, grad_out, grad_x}, ctx->device);
    if (rc) return rc;
    if (!is_device_pointer(x) || !is_device_pointer(grad_out) || !is_device_pointer(grad_x))
        return fail(FCWT_ERR_INVALID, "x, grad_out and grad_x must be device pointers");
    const int log2N = host::find2power(n);
    if (log2N > kMaxLog2N) return fail(FCWT_ERR_INVALID, "signal too long");
    const int N = 1 << log2N;
    cudaStream_t st = ctx->stream;
    const float scale = (flags & FCWT_NORM) ? 1.0f / (float)N : 1.0f;
    if (N < 2 || fn == 0) {
        FCWT_CUDA_TRY(cudaMemsetAsync(grad_x, 0, sizeof(float) * (size_t)n * batch, st));
        return FCWT_OK;
    }
    const int half = N / 2;
    const int RP = adjoint_rows_per_pass();
    const int nchunks = (fn + RP - 1) / RP;
    // tables
    if (ctx->adj_tw_log2N != log2N) {
        FCWT_CUDA_TRY(ctx->adj_tw.ensure((size_t)(1024 + std::max(N / 1024, 1)) * sizeof(float2)));
        FCWT_CUDA_TRY(launch_twiddle(log2N, ctx->adj_tw.as<float2>(), st));
        ctx->adj_tw_log2N = log2N;
    }
    const size_t BN = (size_t)batch * N;
    FCWT_CUDA_TRY(ctx->adj_x.ensure(BN * sizeof(float2)));
    FCWT_CUDA_TRY(ctx->adj_h.ensure(BN * sizeof(float2)));
    FCWT_CUDA_TRY(ctx->adj_g.ensure(BN * RP * sizeof(float2)));
    FCWT_CUDA_TRY(ctx->adj_tmp.ensure(BN * RP * sizeof(float2)));
    const size_t njobs_total = (size_t)batch * (2 + (size_t)fn);
    FCWT_CUDA_TRY(ctx->adj_jobs.ensure(njobs_total * sizeof(FwdJob)));
    if (ctx->adj_jobs_host_bytes < njobs_total * sizeof(FwdJob)) {
        // the previous backward's uploads must have been consumed before the
        // pinned staging is replaced
        FCWT_CUDA_TRY(cudaStreamSynchronize(st));
        if (ctx->adj_jobs_host) cudaFreeHost(ctx->adj_jobs_host);
        ctx->adj_jobs_host = nullptr;
        FCWT_CUDA_TRY(cudaMallocHost(&ctx->adj_jobs_host, njobs_total * sizeof(FwdJob)));
        ctx->adj_jobs_host_bytes = njobs_total * sizeof(FwdJob);
    } else {
        FCWT_CUDA_TRY(cudaStreamSynchronize(st));  // staging reused: earlier uploads must be done
    }
    FwdJob* jh = static_cast<FwdJob*>(ctx->adj_jobs_host);
    FwdJob* jd = ctx->adj_jobs.as<FwdJob>();
    // per-row constants
    struct AdjRowH {
        float ca, dfdq;
    };
    std::vector<AdjRowH> rowc((size_t)fn);
    const double two_pi = 6.283185307179586;
    for (int i = 0; i < fn; i++) {
        const double f = freqs[i];
        if (!(f > 0.0)) return fail(FCWT_ERR_INVALID, "frequencies must be positive");
        rowc[(size_t)i].ca = (float)(two_pi * fb * (fs / f) / N);
        rowc[(size_t)i].dfdq = (float)(two_pi * fb / N * fs / (f * f));
    }
    FCWT_CUDA_TRY(ctx->adj_rows.ensure(rowc.size() * sizeof(AdjRowH)));
    FCWT_CUDA_TRY(ctx->adj_acc.ensure((1 + (size_t)fn) * sizeof(double)));
    FCWT_CUDA_TRY(cudaMemcpyAsync(ctx->adj_rows.p, rowc.data(), rowc.size() * sizeof(AdjRowH), cudaMemcpyHostToDevice, st));
    FCWT_CUDA_TRY(cudaMemsetAsync(ctx->adj_acc.p, 0, (1 + (size_t)fn) * sizeof(double), st));
    FCWT_CUDA_TRY(cudaMemsetAsync(ctx->adj_h.p, 0, BN * sizeof(float2), st));
    const float2* tw = ctx->adj_tw.as<float2>();
    int nk = 0;
    // X_b = FFT(x_b)
    size_t jo = 0;
    for (int b = 0; b < batch; b++) {
        FwdJob& j = jh[jo + b];
        j.in_r = x + (size_t)b * n;
        j.in_c = nullptr;
        j.n = n;
        j.pad = 0;
        j.X = ctx->adj_x.as<float2>() + (size_t)b * N;
        j.tmp = ctx->adj_tmp.as<float2>() + (size_t)b * N;
    }
    FCWT_CUDA_TRY(cudaMemcpyAsync(jd + jo, jh + jo, (size_t)batch * sizeof(FwdJob), cudaMemcpyHostToDevice, st));
    FCWT_CUDA_TRY(launch_forward_batched(jd + jo, batch, log2N, tw, st, &nk, true));
    ctx->kernel_launches += nk;
    jo += batch;
    // rows in chunks: Ghat = FFT(G), accumulate H and the parameter sums
    const float2* G = static_cast<const float2*>(grad_out);
    const bool fused = log2N >= kLog2P2 && log2N <= kLog2P2 + 4;  // N = 1024 .. 16384: one kernel, in SMEM
    if (fused) {
        FCWT_CUDA_TRY(launch_adjoint_rows(G, ctx->adj_x.as<float2>(), ctx->adj_rows.p, n, log2N, fn, batch, tw,
                                          (float)(two_pi * fb), host::mother_norm(), 1.0f / fb,
                                          ctx->adj_h.as<float2>(), ctx->adj_acc.as<double>(),
                                          ctx->adj_acc.as<double>() + 1, st));
        ctx->kernel_launches += 1;
    }
    for (int c = 0; c < (fused ? 0 : nchunks); c++) {
        const int i0 = c * RP;
        const int nr = std::min(RP, fn - i0);
        for (int b = 0; b < batch; b++) {
            for (int i = 0; i < nr; i++) {
                FwdJob& j = jh[jo + (size_t)b * nr + i];
                j.in_r = nullptr;
                j.in_c = G + ((size_t)b * fn + i0 + i) * n;
                j.n = n;
                j.pad = 0;
                j.X = ctx->adj_g.as<float2>() + ((size_t)b * nr + i) * N;
                j.tmp = ctx->adj_tmp.as<float2>() + ((size_t)b * nr + i) * N;
            }
        }
        FCWT_CUDA_TRY(cudaMemcpyAsync(jd + jo, jh + jo, (size_t)batch * nr * sizeof(FwdJob), cudaMemcpyHostToDevice, st));
        FCWT_CUDA_TRY(launch_forward_batched(jd + jo, batch * nr, log2N, tw, st, &nk, false));
        ctx->kernel_launches += nk;
        jo += (size_t)batch * nr;
        FCWT_CUDA_TRY(launch_adjoint_accum(ctx->adj_x.as<float2>(), ctx->adj_g.as<float2>(), ctx->adj_h.as<float2>(),
                                           static_cast<const AdjRowH*>(ctx->adj_rows.p) + i0, nr, half, N, batch,
                                           (float)(two_pi * fb), host::mother_norm(), 1.0f / fb,
                                           ctx->adj_acc.as<double>(), ctx->adj_acc.as<double>() + 1 + i0, st));
        ctx->kernel_launches += 1;
    }
    // dL/dx = Re(scale * IFFTraw(H))[0:n]
    for (int b = 0; b < batch; b++) {
        FwdJob& j = jh[jo + b];
        j.in_r = nullptr;
        j.in_c = ctx->adj_h.as<float2>() + (size_t)b * N;
        j.n = N;
        j.pad = 0;
        j.X = ctx->adj_g.as<float2>() + (size_t)b * N;
        j.tmp = ctx->adj_tmp.as<float2>() + (size_t)b * N;
    }
    FCWT_CUDA_TRY(cudaMemcpyAsync(jd + jo, jh + jo, (size_t)batch * sizeof(FwdJob), cudaMemcpyHostToDevice, st));
    FCWT_CUDA_TRY(launch_inverse_batched(jd + jo, batch, log2N, tw, st, &nk));
    ctx->kernel_launches += nk;
    FCWT_CUDA_TRY(launch_take_real(ctx->adj_g.as<float2>(), N, n, batch, scale, grad_x, st));
    ctx->kernel_launches += 1;
    std::vector<double> acc(1 + (size_t)fn);
    FCWT_CUDA_TRY(cudaMemcpyAsync(acc.data(), ctx->adj_acc.p, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    FCWT_CUDA_TRY(cudaStreamSynchronize(st));
    if (grad_fb) *grad_fb = scale * acc[0];
    if (grad_freqs)
        for (int i = 0; i < fn; i++) grad_freqs[i] = scale * acc[1 + (size_t)i];
    return FCWT_OK;
}

int fcwt_load_optimization_plan(fcwt_context* ctx, int n, int threads, const char* directory) {
    if (!ctx) return fail(FCWT_ERR_INVALID, "null context");
    const int log2N = fcwt::host::find2power(n);
    if (log2N > fcwt::kMaxLog2N) return fail(FCWT_ERR_INVALID, "signal too long");
    const std::string path = tune_path(directory, 1 << log2N, threads);
    std::ifstream f(path);
    if (!f) return fail(FCWT_ERR_IO, "optimization plan '" + path + "' was not found");
    std::string magic;
    std::getline(f, magic);
    if (magic != "fcwt-b200-tune 1") return fail(FCWT_ERR_IO, "optimization plan '" + path + "' is malformed");
    TuneChoice tc;
    std::string line;
    int got = 0;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::string key;
        long long v;
        if (!(ls >> key >> v)) continue;
        if (key == "scratch_mb" && v >= 1 && v <= 4096) {
            tc.scratch_mb = (int)v;
            got |= 1;
        } else if (key == "lag" && v >= 1 && v <= 64) {
            tc.lag = (int)v;
            got |= 2;
        } else if (key == "engine" && (v == 0 || v == 1)) {
            tc.engine = (int)v;
        }
    }
    if (got != 3) return fail(FCWT_ERR_IO, "optimization plan '" + path + "' is malformed");
    ctx->tune[log2N] = tc;
    // cached plans of that size were built with the old choices
    for (auto it = ctx->cache.begin(); it != ctx->cache.end();) {
        if (it->plan->sig[0].sp.log2N == log2N) {
            fcwt_plan_destroy(it->plan);
            it = ctx->cache.erase(it);
        } else {
            ++it;
        }
    }
    return FCWT_OK;
}

int fcwt_create_optimization_plan(fcwt_context* ctx, int maxsize, int threads, int level, const char* directory) {
    int rc = ctx_prepare(ctx);
    if (rc) return rc;
    if (threads < 1) return fail(FCWT_ERR_INVALID, "threads must be >= 1");
    if (level < 0 || level > 3) return fail(FCWT_ERR_INVALID, "level must be 0..3");
    const int nt = fcwt::host::find2power(maxsize);
    if (nt > fcwt::kMaxLog2N) return fail(FCWT_ERR_INVALID, "maxsize too large");
    for (int i = 11; i <= nt; i++) {
        const int N = 1 << i;
        TuneChoice best;
        if (level > 0 && N > fcwt::kMaxFusedN) {
            // candidate grid grows with the level
            std::vector<TuneChoice> cands;
            const int mbs[] = {16, 32, 64, 96};
            const int lags[] = {4, 8, 12, 16};
            const int nm = level == 1 ? 2 : (level == 2 ? 3 : 4);
            // CUDA-core engine: scratch budget x lag grid; tensor-core engine: one candidate
            for (int a = 0; a < nm; a++)
                for (int b = 0; b < nm; b++) cands.push_back({mbs[a + (4 - nm)], lags[b], 1});
            if (N >= fcwt::kTcMinN) cands.push_back(TuneChoice{});
            // synthetic workload: N samples, 256 log-spaced scales over the band
            const int fn = 256;
            std::vector<float> sc((size_t)fn), x((size_t)N);
            fcwt::host::scales(FCWT_LOGSCALES, 1000, 1.0f, 400.0f, fn, sc.data());
            for (int t = 0; t < N; t++) x[(size_t)t] = (float)std::sin(0.01 * t) + 0.1f * (float)((t * 7919) % 13);
            DevBuf din, dout;
            FCWT_CUDA_TRY(din.ensure((size_t)N * 4));
            FCWT_CUDA_TRY(dout.ensure((size_t)N * fn * 8));
            FCWT_CUDA_TRY(cudaMemcpy(din.p, x.data(), (size_t)N * 4, cudaMemcpyHostToDevice));
            double best_t = 1e30;
            for (const TuneChoice& tc : cands) {
                ctx->tune[i] = tc;
                fcwt_plan* p = nullptr;
                rc = fcwt_plan_create(ctx, N, 0, 2.0f, sc.data(), fn, threads, FCWT_NORM, 0, fn, &p);
                if (rc) return rc;
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                rc = plan_run(p, din.p, dout.p, FCWT_OUT_C64);  // warm-up
                cudaEventRecord(e0, ctx->stream);
                for (int r = 0; r < 3 && rc == 0; r++) rc = plan_run(p, din.p, dout.p, FCWT_OUT_C64);
                cudaEventRecord(e1, ctx->stream);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                fcwt_plan_destroy(p);
                if (rc) return rc;
                rc = fcwt_synchronize(ctx);
                if (rc) return rc;
                if (ms < best_t) {
                    best_t = ms;
                    best = tc;
                }
            }
            din.release();
            dout.release();
        }
        ctx->tune[i] = best;
        const std::string path = tune_path(directory, N, threads);
        std::ofstream f(path);
        if (!f) return fail(FCWT_ERR_IO, "cannot write '" + path + "'");
        f << "fcwt-b200-tune 1\n";
        f << "N " << N << "\n";
        f << "threads " << threads << "\n";
        f << "scratch_mb " << best.scratch_mb << "\n";
        f << "lag " << best.lag << "\n";
        f << "engine " << best.engine << "\n";
        if (!f) return fail(FCWT_ERR_IO, "cannot write '" + path + "'");
    }
    // cached plans were built with the previous choices
    cudaStreamSynchronize(ctx->stream);
    for (auto& e : ctx->cache) plan_free(e.plan);
    ctx->cache.clear();
    return FCWT_OK;
}

}  // extern "C"
