// fcwt_cwt_noalloc: the real-input transform for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs on a real-time thread (an audio or sensor
// callback that must not block), where cudaMalloc/cudaFree can stall and
// implicitly synchronize the device; plug-ins hosted by a framework that owns
// all device memory; and callers that fix their memory footprint at start-up.
//
// Everything the call needs on the device besides the caller's input and
// output lives in one file-scope __device__ array of kNoAllocScratchBytes
// (about 2.3 MB, held by every GPU that loads the library until the process
// exits): the spectrum, the FFT ping-pong buffer, the mother and twiddle
// tables, the stale-bin tables, the row and work-item descriptors, the work
// queue counters and the scratch ring of the two-phase rows. Its limits:
// n <= 16384 samples, fn <= 1024 scales, at most 8 distinct stale-bin tables.
//
// The call copies nothing from host memory with cudaMemcpy: the row
// descriptors and stale-bin tables it plans on the host travel to the array
// as kernel parameters of small copy kernels (each launch carries its own
// copy of them), and the work list is generated on the device. So no pageable
// host-to-device copy makes the host wait for earlier work in the stream, and
// no copy refers to host memory after the call returns. The host-side planning
// does use the C++ heap; device memory is never allocated.
//
// Every call shares that array and leaves its contents behind; each call
// clears the counters and error word it needs before its kernels run. Calls
// whose GPU work overlaps (different streams, or different host threads on
// one device) race on the array: serialize them on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fcwt_b200.h"
#include "fcwt_internal.h"
#include "fcwt_plan.h"

namespace fcwt {
cudaError_t launch_mother(float fb, int N, float norm, float* out, cudaStream_t st);
cudaError_t launch_twiddle(int log2N, float2* tw, cudaStream_t st);
cudaError_t launch_forward(const float* in_r, const float2* in_c, int n, int log2N, const float2* tw,
                           float2* out, float2* tmp, cudaStream_t st, int* n_kernels);
cudaError_t engine_configure();
cudaError_t engine_blocks_per_sm(int* out);
cudaError_t launch_engine(const EngineParams& p, int grid, cudaStream_t st);
void record_error(const std::string& msg);  // message returned by fcwt_last_error()
}  // namespace fcwt

namespace {

using namespace fcwt;

constexpr int kNaMaxN = 16384;
constexpr int kNaMaxRows = 1024;
constexpr int kNaMaxTables = 8;
constexpr int kNaSlots = 8;
constexpr int kNaMaxItems = kNaMaxRows * (kP2 / kChunk + kNaMaxN / kP2 / kGroupCols);

// byte offsets of the sub-buffers inside the array (256-byte aligned)
constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }
constexpr size_t kOffX = 0;
constexpr size_t kOffTmp = align256(kOffX + sizeof(float2) * kNaMaxN);
constexpr size_t kOffMother = align256(kOffTmp + sizeof(float2) * kNaMaxN);
constexpr size_t kOffTw = align256(kOffMother + sizeof(float) * kNaMaxN);
constexpr size_t kOffPool = align256(kOffTw + sizeof(float2) * (kP2 + kNaMaxN / kP2));
constexpr size_t kOffRows = align256(kOffPool + sizeof(float) * kNaMaxTables * (kNaMaxN / 2));
constexpr size_t kOffItems = align256(kOffRows + sizeof(RowDesc) * kNaMaxRows);
constexpr size_t kOffSig = align256(kOffItems + sizeof(Item) * kNaMaxItems);
constexpr size_t kOffCounters = align256(kOffSig + sizeof(SigDesc));
constexpr size_t kOffErr = align256(kOffCounters + sizeof(unsigned) * (1 + 2 * kNaMaxRows));
constexpr size_t kOffScratch = align256(kOffErr + sizeof(int));
constexpr size_t kNoAllocScratchBytes = align256(kOffScratch + sizeof(float2) * kNaSlots * kNaMaxN);

// The array itself. Host code must not use its name as an address: on the
// host it is only a stand-in symbol; the device address comes from
// cudaGetSymbolAddress during the per-device set-up below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// ---- descriptor delivery by kernel parameters (at most 32764 bytes each)
constexpr int kRowsPerCopy = 232;    // RowDesc per launch (232 x 120 B)
constexpr int kFloatsPerCopy = 7680; // 30 KB of stale-bin table entries

struct RowCopy {
    SigDesc sig;
    int first;
    int count;
    int write_sig;
    int pad;
    RowDesc rows[kRowsPerCopy];
};
struct PoolCopy {
    int first;
    int count;
    float v[kFloatsPerCopy];
};
static_assert(sizeof(RowCopy) <= 32000 && sizeof(PoolCopy) <= 32000, "kernel parameter limit");

__global__ void k_na_rows(const __grid_constant__ RowCopy c, RowDesc* __restrict__ dst, SigDesc* __restrict__ dsig) {
    for (int i = threadIdx.x; i < c.count; i += blockDim.x) dst[c.first + i] = c.rows[i];
    if (c.write_sig && threadIdx.x == 0) *dsig = c.sig;
}

__global__ void k_na_pool(const __grid_constant__ PoolCopy c, float* __restrict__ dst) {
    for (int i = threadIdx.x; i < c.count; i += blockDim.x) dst[c.first + i] = c.v[i];
}

// The work list of the row engine, the same sequence the host builds for a
// plan: one item per row when rows run whole (type), otherwise per step s,
// the n_a phase-1 items of row s (s < fn) followed by the n_b phase-2 items of
// row s - lag (0 <= s - lag < fn). One thread per step.
__global__ void k_na_items(int fn, int two_phase, int type, int n_a, int n_b, int lag, Item* __restrict__ items) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (!two_phase) {
        if (s < fn) items[s] = Item{type, s, 0, 0};
        return;
    }
    if (s >= fn + lag) return;
    int base = n_a * min(s, fn) + n_b * max(0, min(s - lag, fn));
    if (s < fn)
        for (int a = 0; a < n_a; a++) items[base++] = Item{ITEM_PHASE1, s, a, 0};
    const int rb = s - lag;
    if (rb >= 0 && rb < fn)
        for (int b = 0; b < n_b; b++) items[base++] = Item{ITEM_PHASE2, rb, b, 0};
}

int na_fail(int code, const std::string& msg) {
    record_error(msg);
    return code;
}

struct DeviceSetup {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_noalloc_scratch on that device
    int grid = 0;                   // persistent grid of the row engine
};

std::mutex g_setup_mu;
DeviceSetup g_setup[64];

// Once per device, with that device current: resolve the array's device
// address and configure the row engine.
int setup_device(int dev, DeviceSetup** out) {
    if (dev < 0 || dev >= 64) return na_fail(FCWT_ERR_UNSUPPORTED, "device index >= 64");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return na_fail(FCWT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        e = engine_configure();
        if (e != cudaSuccess) return na_fail(FCWT_ERR_CUDA, std::string("engine set-up: ") + cudaGetErrorString(e));
        int per_sm = 0, sms = 0;
        e = engine_blocks_per_sm(&per_sm);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return na_fail(FCWT_ERR_CUDA, std::string("engine set-up: ") + cudaGetErrorString(e));
        s.base = static_cast<unsigned char*>(p);
        s.grid = std::max(1, per_sm) * sms;
        s.ready = true;
    }
    *out = &s;
    return FCWT_OK;
}

// 0 host memory, 1 memory the kernels of device `dev` may use (that device's
// memory, or managed memory), -1 memory of another device.
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

}  // namespace

#define NA_TRY(expr)                                                                          \
    do {                                                                                      \
        cudaError_t e_ = (expr);                                                              \
        if (e_ != cudaSuccess) return na_fail(FCWT_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

extern "C" int fcwt_cwt_noalloc(const float* input, int n, float fb, const float* scales, int fn, int threads,
                                unsigned flags, void* output, void* stream, int* status) {
    if (n < 0 || fn < 0) return na_fail(FCWT_ERR_INVALID, "fcwt_cwt_noalloc: negative size");
    if (n > kNaMaxN)
        return na_fail(FCWT_ERR_INVALID, "fcwt_cwt_noalloc: n = " + std::to_string(n) +
                                             " exceeds the static scratch limit of 16384 samples");
    if (fn > kNaMaxRows)
        return na_fail(FCWT_ERR_INVALID, "fcwt_cwt_noalloc: fn = " + std::to_string(fn) +
                                             " exceeds the static scratch limit of 1024 scales");
    if (status) *status = 0;
    if (n == 0 || fn == 0) return FCWT_OK;
    if (!input || !output || !scales) return na_fail(FCWT_ERR_INVALID, "fcwt_cwt_noalloc: null pointer");
    int dev = 0;
    NA_TRY(cudaGetDevice(&dev));
    if (pointer_kind(input, dev) != 1 || pointer_kind(output, dev) != 1)
        return na_fail(FCWT_ERR_INVALID,
                       "fcwt_cwt_noalloc: input and output must be device pointers of the current device " +
                           std::to_string(dev));
    if (pointer_kind(scales, dev) != 0)
        return na_fail(FCWT_ERR_INVALID, "fcwt_cwt_noalloc: scales must be a host array");
    DeviceSetup* S = nullptr;
    int rc = setup_device(dev, &S);
    if (rc) return rc;

    SignalPlan sp;
    std::string err;
    if (plan_signal(n, false, fb, scales, fn, threads, flags, sp, err)) return na_fail(FCWT_ERR_INVALID, err);
    if ((int)sp.tables.size() > kNaMaxTables)
        return na_fail(FCWT_ERR_INVALID, "fcwt_cwt_noalloc: the scale sequence needs more than 8 stale-bin tables");
    const int N = sp.N;
    const int M = sp.M;
    for (const RowPlan& rp : sp.rows)
        if (N >= kP2 && rp.K > kMaxK) return na_fail(FCWT_ERR_UNSUPPORTED, "fcwt_cwt_noalloc: row support too wide");

    // row descriptors (same rows as a plan of the row engine)
    std::vector<RowDesc> rows((size_t)fn);
    const float out_scale = (flags & kFlagNorm) ? 1.0f / (float)N : 1.0f;
    const bool two_phase = N > kMaxFusedN;
    const int S_slots = two_phase ? std::min(kNaSlots, fn) : 0;
    const int lag = two_phase ? std::max(1, std::min(12, S_slots / 2)) : 0;
    const int n_a = two_phase ? kP2 / kChunk : 0;
    const int n_b = two_phase ? M / kGroupCols : 0;
    for (int r = 0; r < fn; r++) {
        const RowPlan& rp = sp.rows[(size_t)r];
        RowDesc& d = rows[(size_t)r];
        std::memset(&d, 0, sizeof(d));
        d.sig = 0;
        d.proc = rp.proc;
        d.step = rp.step;
        d.K = rp.K;
        d.L = rp.L;
        d.lo = rp.lo;
        d.hi = rp.hi;
        d.stale = rp.table >= 0 ? rp.table * sp.half : -1;
        d.slot = two_phase ? r % S_slots : -1;
        d.wait_row = two_phase && r >= S_slots ? r - S_slots : -1;
        d.n_a = n_a;
        d.n_b = n_b;
        d.out_buf = 0;
        d.dec = 1;
        d.n_out = n;
        d.out_off = (long long)r * n;
        d.out_scale = out_scale;
        d.out_row = r;
        d.mode = (flags & kFlagContinuous) ? 1 : 0;
        d.ca = rp.ca;
        d.cb = rp.cb;
        d.cnorm = host::mother_norm();
    }
    const int n_items = two_phase ? fn * (n_a + n_b) : fn;

    unsigned char* base = S->base;
    float2* X = reinterpret_cast<float2*>(base + kOffX);
    float2* tmp = reinterpret_cast<float2*>(base + kOffTmp);
    float* mother = reinterpret_cast<float*>(base + kOffMother);
    float2* tw = reinterpret_cast<float2*>(base + kOffTw);
    float* dpool = reinterpret_cast<float*>(base + kOffPool);
    RowDesc* drows = reinterpret_cast<RowDesc*>(base + kOffRows);
    Item* ditems = reinterpret_cast<Item*>(base + kOffItems);
    SigDesc* dsig = reinterpret_cast<SigDesc*>(base + kOffSig);
    unsigned* counters = reinterpret_cast<unsigned*>(base + kOffCounters);
    int* derr = reinterpret_cast<int*>(base + kOffErr);
    float2* scratch = reinterpret_cast<float2*>(base + kOffScratch);

    cudaStream_t st = (cudaStream_t)stream;
    {
        // descriptors and stale tables, in kernel-parameter chunks
        static thread_local RowCopy rc_buf;
        RowCopy& c = rc_buf;
        c.sig.X = X;
        c.sig.mother = mother;
        c.sig.tw = tw;
        c.sig.log2N = sp.log2N;
        c.sig.n = n;
        for (int r0 = 0; r0 < fn; r0 += kRowsPerCopy) {
            c.first = r0;
            c.count = std::min(kRowsPerCopy, fn - r0);
            c.write_sig = r0 == 0;
            std::memcpy(c.rows, rows.data() + r0, sizeof(RowDesc) * (size_t)c.count);
            k_na_rows<<<1, 256, 0, st>>>(c, drows, dsig);
            NA_TRY(cudaGetLastError());
        }
        static thread_local PoolCopy pc_buf;
        PoolCopy& pc = pc_buf;
        for (size_t t = 0; t < sp.tables.size(); t++) {
            const std::vector<float>& T = sp.tables[t];
            const size_t len = std::min(T.size(), (size_t)sp.half);
            for (size_t i0 = 0; i0 < len; i0 += kFloatsPerCopy) {
                pc.first = (int)(t * (size_t)sp.half + i0);  // table t starts at t * half (RowDesc::stale)
                pc.count = (int)std::min((size_t)kFloatsPerCopy, len - i0);
                std::memcpy(pc.v, T.data() + i0, sizeof(float) * (size_t)pc.count);
                k_na_pool<<<1, 256, 0, st>>>(pc, dpool);
                NA_TRY(cudaGetLastError());
            }
        }
        k_na_items<<<(fn + lag + 127) / 128, 128, 0, st>>>(fn, two_phase ? 1 : 0, N < kP2 ? ITEM_SMALL : ITEM_FUSED,
                                                             n_a, n_b, lag, ditems);
        NA_TRY(cudaGetLastError());
    }
    NA_TRY(cudaMemsetAsync(counters, 0, sizeof(unsigned) * (1 + 2 * (size_t)fn), st));
    NA_TRY(cudaMemsetAsync(derr, 0, sizeof(int), st));
    NA_TRY(launch_mother(fb, N, host::mother_norm(), mother, st));
    NA_TRY(launch_twiddle(sp.log2N, tw, st));
    int n_fwd = 0;
    NA_TRY(launch_forward(input, nullptr, n, sp.log2N, tw, X, tmp, st, &n_fwd));
    EngineParams ep;
    std::memset(&ep, 0, sizeof(ep));
    ep.sigs = dsig;
    ep.rows = drows;
    ep.items = ditems;
    ep.n_items = n_items;
    ep.stale_pool = dpool;
    ep.scratch = two_phase ? scratch : nullptr;
    ep.slot_elems = two_phase ? N : 0;
    ep.counters = counters;
    ep.n_rows = fn;
    ep.outs[0] = output;
    ep.out_type = OUT_C64;
    ep.err = derr;
    NA_TRY(launch_engine(ep, std::max(1, std::min(ep.n_items, S->grid)), st));
    if (status) {
        int h = 0;
        NA_TRY(cudaMemcpyAsync(&h, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
        NA_TRY(cudaStreamSynchronize(st));
        *status = h;
        if (h != 0) return na_fail(FCWT_ERR_DEVICE, "fcwt_cwt_noalloc: row engine reported error bits " + std::to_string(h));
    }
    return FCWT_OK;
}
