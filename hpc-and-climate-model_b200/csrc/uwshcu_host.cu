// uwshcu_host.cu -- host side of libuwshcu_b200.so: constants, saturation table, device arena,
// pinned staging and the C ABI declared in include/uwshcu.h.
//
// The reference drop-in (src/physics/bxcompute_uwshcu_inv.cpp:6195-6496, 6887-7043) allocates and
// frees ~50 device arrays and ~35 pinned arrays on every call and runs findsp on the CPU.  Here the
// device arena and the pinned staging area are allocated once per device and grown on demand,
// every column-physics step (findsp included) runs on the GPU, and a call costs one H2D copy of the
// packed inputs, one kernel launch and one D2H copy of the packed outputs.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "uwshcu.h"
#include "uwshcu_common.cuh"
#include "uw_state.cuh"
#include "uw_math.h"

#define UW_DECL(KP, NC)                                                                              \
    extern "C" cudaError_t uw_fp64_set_constants_k##KP##n##NC(const UwConst* h, const double* tbl); \
    extern "C" cudaError_t uw_fp64_launch_k##KP##n##NC(const UwArgs* a, int mode, int* wl, int* wl_count, \
                                                       int nthreads, int block, cudaStream_t stream);
UW_DECL(32, 5)
UW_DECL(64, 5)
UW_DECL(32, 32)
UW_DECL(64, 32)
#undef UW_DECL
#define UW_DECL_FAST(KP, NC)                                                                              \
    extern "C" cudaError_t uw_fast_set_constants_k##KP##n##NC(const UwConst* h, const double* tbl);       \
    extern "C" cudaError_t uw_fast_launch_k##KP##n##NC(const UwArgs* a, int mode, int* wl, int* wl_count, \
                                                       int nthreads, int block, cudaStream_t stream);
UW_DECL_FAST(32, 5)
UW_DECL_FAST(64, 5)
UW_DECL_FAST(32, 32)
UW_DECL_FAST(64, 32)
#undef UW_DECL_FAST
extern "C" cudaError_t uw_budget_launch(int mix, int mkx, int iend, int inv, double dt, double latvap,
                                        double latice, double g, const double* s0, const double* qv0,
                                        const double* ql0, const double* qi0, const double* u0,
                                        const double* v0, const double* dp0, const double* sten,
                                        const double* qvten, const double* qlten, const double* qiten,
                                        const double* uten, const double* vten, const double* precip,
                                        const double* snow, const double* rliq, double* te_rer,
                                        double* tw_rer, cudaStream_t stream);
extern "C" cudaError_t uw_adj_set_constants_k32n5(const UwConst* h, const double* tbl);
extern "C" cudaError_t uw_adj_launch_k32n5(const UwArgs* a, const void* slots, const uwshcu_adjoint* c, int phase,
                                           cudaStream_t stream);
extern "C" size_t uw_adj_row_bytes_k32n5();   // the same for both units: 32 records per row
extern "C" cudaError_t uw_adj_forward_occupancy_k32n5(int* warps_per_sm);
extern "C" cudaError_t uw_adj_forward_occupancy_k64n5(int* warps_per_sm);
extern "C" cudaError_t uw_adj_set_constants_k64n5(const UwConst* h, const double* tbl);
extern "C" cudaError_t uw_adj_launch_k64n5(const UwArgs* a, const void* slots, const uwshcu_adjoint* c, int phase,
                                           cudaStream_t stream);
extern "C" cudaError_t uw_tl_set_constants_k32n5(const UwConst* h, const double* tbl);
extern "C" cudaError_t uw_tl_set_constants_k64n5(const UwConst* h, const double* tbl);
extern "C" cudaError_t uw_tl_launch_k32n5(const UwArgs* a, const uwshcu_tangent* t, int mode, int* wl,
                                           int* wl_count, int nthreads, int block, cudaStream_t stream);
extern "C" cudaError_t uw_tl_launch_k64n5(const UwArgs* a, const uwshcu_tangent* t, int mode, int* wl,
                                           int* wl_count, int nthreads, int block, cudaStream_t stream);
#define UW_DECL_MIXED(KP, NC)                                                                              \
    extern "C" cudaError_t uw_mixed_set_constants_k##KP##n##NC(const UwConst* h, const double* tbl);       \
    extern "C" cudaError_t uw_mixed_launch_k##KP##n##NC(const UwArgs* a, int mode, int* wl, int* wl_count, \
                                                        int nthreads, int block, cudaStream_t stream);
UW_DECL_MIXED(32, 5)
UW_DECL_MIXED(64, 5)
#undef UW_DECL_MIXED

namespace {

constexpr int kMaxDev = 16;
constexpr int kModeAll = 0, kModeTrigger = 1, kModeList = 2, kModeList1 = 3, kModeResume = 4;
// Largest hand-off region of the split worklist pass (bytes of column state per region); a call
// with more implicit-CIN columns than fit finishes the rest in the first launch.
constexpr size_t kHandBytes = (size_t)4 << 30;

cudaError_t set_constants_all(const UwConst* k, const double* tbl)
{
    cudaError_t e;
    if ((e = uw_fp64_set_constants_k32n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_fp64_set_constants_k64n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_fp64_set_constants_k32n32(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_fp64_set_constants_k64n32(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_fast_set_constants_k32n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_fast_set_constants_k64n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_fast_set_constants_k32n32(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_fast_set_constants_k64n32(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_tl_set_constants_k32n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_adj_set_constants_k32n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_adj_set_constants_k64n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_tl_set_constants_k64n5(k, tbl)) != cudaSuccess) return e;
    if ((e = uw_mixed_set_constants_k32n5(k, tbl)) != cudaSuccess) return e;
    return uw_mixed_set_constants_k64n5(k, tbl);
}

cudaError_t launch_mode(const UwArgs* a, int prec, int mode, int* wl, int* wl_count, int nthreads, int block,
                        cudaStream_t st)
{
    if (prec == UWSHCU_PREC_MIXED) {
        if (a->mkx + 1 <= 32 && a->ncnst <= 5) return uw_mixed_launch_k32n5(a, mode, wl, wl_count, nthreads, block, st);
        if (a->mkx + 1 <= 64 && a->ncnst <= 5) return uw_mixed_launch_k64n5(a, mode, wl, wl_count, nthreads, block, st);
        return cudaErrorInvalidValue;
    }
    if (prec == UWSHCU_PREC_FAST) {
        if (a->mkx + 1 <= 32 && a->ncnst <= 5) return uw_fast_launch_k32n5(a, mode, wl, wl_count, nthreads, block, st);
        if (a->mkx + 1 <= 64 && a->ncnst <= 5) return uw_fast_launch_k64n5(a, mode, wl, wl_count, nthreads, block, st);
        if (a->mkx + 1 <= 32 && a->ncnst <= UW_NCMAX) return uw_fast_launch_k32n32(a, mode, wl, wl_count, nthreads, block, st);
        if (a->mkx + 1 <= 64 && a->ncnst <= UW_NCMAX) return uw_fast_launch_k64n32(a, mode, wl, wl_count, nthreads, block, st);
        return cudaErrorInvalidValue;
    }
    if (a->mkx + 1 <= 32 && a->ncnst <= 5) return uw_fp64_launch_k32n5(a, mode, wl, wl_count, nthreads, block, st);
    if (a->mkx + 1 <= 64 && a->ncnst <= 5) return uw_fp64_launch_k64n5(a, mode, wl, wl_count, nthreads, block, st);
    if (a->mkx + 1 <= 32 && a->ncnst <= UW_NCMAX) return uw_fp64_launch_k32n32(a, mode, wl, wl_count, nthreads, block, st);
    if (a->mkx + 1 <= 64 && a->ncnst <= UW_NCMAX) return uw_fp64_launch_k64n32(a, mode, wl, wl_count, nthreads, block, st);
    return cudaErrorInvalidValue;
}

// One hand-off region of the split worklist pass: [UwHand][count, hist][col][key][order][state].
struct HandRegion {
    char* base = nullptr;
    size_t cap = 0, words = 0;
    char* dsort = nullptr;       // uwshcu_set_depth_order: the keys and the sort of a worklist
    size_t dsort_bytes = 0;
};

// What a device-array call (uwshcu_compute_device, uwshcu_compute_member, the tangent-linear and
// adjoint entries) needs besides its arguments, one set per caller stream, so that calls on different
// streams whose GPU work overlaps do not share a worklist, a hand-off region or an endrun word.
struct StreamCtx {
    cudaStream_t stream = nullptr;
    bool used = false;
    unsigned long long last = 0;   // LRU tick of the last call
    unsigned int* err = nullptr;   // endrun bits of the calls since the last uwshcu_device_status
    int* wl = nullptr;             // worklist of convecting columns: [0] = count, [1..] = column ids
    size_t wl_cap = 0;
    int* dkey = nullptr;           // uwshcu_set_depth_order: each column's key from the last call
    size_t dkey_cap = 0;
    HandRegion hand;               // hand-off region of the sorted schedule
};

struct DeviceState {
    unsigned uploaded_gen = 0;   // generation of the constants in this device's __constant__ bank
    // per caller stream; a call on a new stream when all are taken reuses the least recently used
    // one after a cudaDeviceSynchronize (that stream's uncollected endrun bits are dropped)
    static constexpr int kStreamCtx = 32;
    StreamCtx sctx[kStreamCtx];
    unsigned long long tick = 0;
    int* last_count = nullptr;   // worklist count of the last device-array call (profiling)
    cudaStream_t stream = nullptr;
    double* d_buf = nullptr;     // device arena (doubles)
    size_t d_cap = 0;
    double* h_buf = nullptr;     // pinned staging (doubles)
    size_t h_cap = 0;
    int* d_wl = nullptr;         // host-array calls: per chunk [count, endrun bits, column ids]
    size_t wl_cap = 0;
    // opt-in per-launch timing: events around the trigger and worklist launches of each call
    static constexpr int kSlots = 256;
    cudaEvent_t ev[kSlots][3] = {};
    int nrec = 0;                // calls recorded since the last read (capped at kSlots)
    // host-array calls: column chunks pipelined over kPipe streams (copy in, compute, copy out);
    // stream j has the j-th highest priority, so earlier chunks finish first and their copies out
    // overlap the later chunks' computation
    static constexpr int kPipe = 8;
    cudaStream_t pipe[kPipe] = {};
    cudaStream_t pin = nullptr, pout = nullptr;   // copy-in and copy-out streams
    std::vector<cudaEvent_t> done, ev_in, ev_comp;   // per chunk: copied out, copied in, computed
    // hand-off regions of the split worklist pass of host-array calls: [1 + j] pipe stream j ([0]
    // unused: device-array calls use their stream's StreamCtx)
    HandRegion hand[1 + kPipe];
    // adjoint tapes, adjoints and tables, kept between adjoint calls (uwshcu_adjoint_release)
    void* adj_buf = nullptr;
    size_t adj_bytes = 0;
    void* adj_aux = nullptr;     // the adjoint's ordering pass: level indices, a copy of cush, sort keys
    size_t adj_aux_bytes = 0;
    int* hkey = nullptr;         // uwshcu_set_depth_order, host-array calls: the key of every column
    size_t hkey_cap = 0;
};

struct State {
    std::mutex mu;
    bool init = false;
    unsigned gen = 0;            // bumped by every uwshcu_init / uwshcu_set_rpen
    UwConst k{};
    double tbl[UW_TBL];
    int precision = UWSHCU_PREC_FP64;
    int schedule = UWSHCU_SCHED_SORTED;
    int hand_slots = 0;          // cap of the hand-off slots per region (0: by kHandBytes only)
    int adj_records = 0;         // largest tape of the last adjoint call (rows per warp)
    int adj_rows = 0;            // tape rows per warp for the next adjoint call (0: the unit's full capacity)
    int block = 128;
    bool profiling = false;
    int chunk_columns = 32768;   // host-array calls: columns per pipeline chunk (0: one chunk)
    int pipe_streams = 4;        // host-array calls: streams the chunks alternate over
    bool pipe_auto = true;       // until uwshcu_set_pipeline: the shape follows the call's size
    bool depth_order = false;    // uwshcu_set_depth_order
    bool pipe_ramp = true;       // smaller first and last chunks (the auto shape, chunk_columns < -1)
    DeviceState dev[kMaxDev];
    char lasterr[256] = "";
};

State& S()
{
    static State s;
    return s;
}

// ---- saturation table: gffgch (gffgch.F90:1-127) tabulated by gestbl (wv_saturation.F90:82-204)
double gffgch(double t, int itype, double tmelt)
{
    double tr, es, eswtr = 0.0;
    int itp = itype;
    if (itp < 0) {
        tr = std::fabs((double)itp);
        itp = 1;
    } else {
        tr = 0.0;
    }
    if (!(t < (tmelt - tr) && itp == 1)) {
        const double ps = 1013.246, ts = 373.16;
        double e1 = 11.344 * (1.0 - t / ts);
        double e2 = -3.49149 * (ts / t - 1.0);
        double f1 = -7.90298 * (ts / t - 1.0);
        double f2 = 5.02808 * std::log10(ts / t);
        double f3 = -1.3816 * (std::pow(10.0, e1) - 1.0) / 10000000.0;
        double f4 = 8.1328 * (std::pow(10.0, e2) - 1.0) / 1000.0;
        double f5 = std::log10(ps);
        double f = f1 + f2 + f3 + f4 + f5;
        es = (std::pow(10.0, f)) * 100.0;
        eswtr = es;
        if (t >= tmelt || itp == 0) return es;
    }
    double t0 = tmelt;
    double term1 = 2.01889049 / (t0 / t);
    double term2 = 3.56654 * std::log(t0 / t);
    double term3 = 20.947031 * (t0 / t);
    es = 575.185606e10 * std::exp(-(term1 + term2 + term3));
    if (t < (tmelt - tr)) return es;
    double weight = std::min((tmelt - t) / tr, 1.0);
    return weight * es + (1.0 - weight) * eswtr;
}

void build_table(double* tbl, double tmin, double tmax, double ttrice, int icephs, double tmelt)
{
    int lentbl = (int)(tmax - tmin + 2.000001);
    if (lentbl > UW_TBL) lentbl = UW_TBL;
    int itype = icephs ? (ttrice != 0.0 ? (int)(-ttrice) : 1) : 0;
    double t = tmin - 1.0;
    for (int n = 0; n < lentbl; n++) {
        t = t + 1.0;
        tbl[n] = gffgch(t, itype, tmelt);
    }
    for (int n = lentbl; n < UW_TBL; n++) tbl[n] = -99999.0;
}

int cuda_fail(cudaError_t e)
{
    std::snprintf(S().lasterr, sizeof(S().lasterr), "%s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? UWSHCU_ERR_ALLOC : UWSHCU_ERR_CUDA;
}

int status_from_bits(unsigned bits)
{
    if (bits & UW_ERRBIT_ENTHALPY) return UWSHCU_ERR_FINDSP_ENTHALPY;
    if (bits & UW_ERRBIT_FINDSP) return UWSHCU_ERR_FINDSP_NONCONVERGED;
    if (bits & UW_ERRBIT_MU) return UWSHCU_ERR_MU_INCONSISTENT;
    if (bits & UW_ERRBIT_NONFINITE) return UWSHCU_WARN_NONFINITE_INPUT;
    return UWSHCU_OK;
}

// Make the current device ready: constants uploaded, error word and stream created.
int ensure_device(DeviceState** out)
{
    State& s = S();
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) {
        std::snprintf(s.lasterr, sizeof(s.lasterr), "%s", e != cudaSuccess ? cudaGetErrorString(e) : "no device");
        return UWSHCU_ERR_NO_DEVICE;
    }
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e);
    if (dev < 0 || dev >= kMaxDev) return UWSHCU_ERR_NO_DEVICE;
    DeviceState& d = s.dev[dev];
    if (!d.stream) {
        if ((e = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e);
    }
    if (d.uploaded_gen != s.gen) {
        if ((e = set_constants_all(&s.k, s.tbl)) != cudaSuccess) return cuda_fail(e);
        d.uploaded_gen = s.gen;
    }
    *out = &d;
    return UWSHCU_OK;
}

int grow(DeviceState& d, size_t ndev_doubles, size_t nhost_doubles)
{
    cudaError_t e;
    if (ndev_doubles > d.d_cap) {
        if (d.d_buf) cudaFree(d.d_buf);
        d.d_buf = nullptr;
        d.d_cap = 0;
        if ((e = cudaMalloc(&d.d_buf, ndev_doubles * sizeof(double))) != cudaSuccess) return cuda_fail(e);
        d.d_cap = ndev_doubles;
    }
    if (nhost_doubles > d.h_cap) {
        if (d.h_buf) cudaFreeHost(d.h_buf);
        d.h_buf = nullptr;
        d.h_cap = 0;
        if ((e = cudaMallocHost(&d.h_buf, nhost_doubles * sizeof(double))) != cudaSuccess) return cuda_fail(e);
        d.h_cap = nhost_doubles;
    }
    return UWSHCU_OK;
}

// A strided copy between a caller array (rows of `ld` doubles) and the compact staging area (rows
// of n doubles), split over a few host threads for the large calls.
struct Plane {
    const double* src;
    double* dst;
    size_t rows;
    size_t src_ld, dst_ld, n;
    double* dev;   // device address of the compact (staging-side) end
};

// Whether [p, p + bytes) is page-locked host memory (cudaMallocHost, cudaHostAlloc,
// cudaHostRegister): its first and last bytes are.
bool pinned_range(const void* p, size_t bytes)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || a.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        return false;
    }
    if (cudaPointerGetAttributes(&a, static_cast<const char*>(p) + bytes - 1) != cudaSuccess ||
        a.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        return false;
    }
    return true;
}

void copy_planes(const std::vector<Plane>& planes)
{
    size_t total = 0;
    for (const Plane& p : planes) total += p.rows * p.n;
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    unsigned nth = (unsigned)std::min<size_t>(std::min(hw, 16u), std::max<size_t>(1, total / (1u << 20)));
    // flatten to (plane, row) work items
    std::vector<std::pair<size_t, size_t>> items;
    for (size_t p = 0; p < planes.size(); p++)
        for (size_t r = 0; r < planes[p].rows; r++) items.emplace_back(p, r);
    auto work = [&](unsigned t) {
        for (size_t w = t; w < items.size(); w += nth) {
            const Plane& p = planes[items[w].first];
            size_t r = items[w].second;
            std::memcpy(p.dst + r * p.dst_ld, p.src + r * p.src_ld, p.n * sizeof(double));
        }
    };
    if (nth <= 1) {
        work(0);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nth; t++) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
}

// A worklist of at least n ints (cudaFree waits for the device, so no call still uses the old one).
int grow_ints(int*& buf, size_t& cap, size_t n)
{
    if (n <= cap) return UWSHCU_OK;
    if (buf) cudaFree(buf);
    buf = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&buf, n * sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e);
    cap = n;
    return UWSHCU_OK;
}

int grow_worklist(DeviceState& d, size_t ncol) { return grow_ints(d.d_wl, d.wl_cap, ncol + 1); }

// The context of caller stream st on device d (created on first use).
int stream_ctx(DeviceState& d, cudaStream_t st, StreamCtx** out)
{
    StreamCtx* c = nullptr;
    for (StreamCtx& x : d.sctx)
        if (x.used && x.stream == st) c = &x;
    if (!c) {
        for (StreamCtx& x : d.sctx)
            if (!x.used && (!c || x.err)) c = &x;   // a free slot, one with buffers first
        if (!c) {
            c = &d.sctx[0];
            for (StreamCtx& x : d.sctx)
                if (x.last < c->last) c = &x;
            cudaError_t e = cudaDeviceSynchronize();   // its stream's work may still use its buffers
            if (e != cudaSuccess) return cuda_fail(e);
        }
        cudaError_t e;
        if (!c->err && (e = cudaMalloc(&c->err, sizeof(unsigned int))) != cudaSuccess) return cuda_fail(e);
        if ((e = cudaMemset(c->err, 0, sizeof(unsigned int))) != cudaSuccess) return cuda_fail(e);
        c->stream = st;
        c->used = true;
    }
    c->last = ++d.tick;
    *out = c;
    return UWSHCU_OK;
}

// ---- split worklist pass -----------------------------------------------------------------------
// Counting sort of the hand-off slots by key: histogram, exclusive scan, scatter.  The order inside
// a key is that of the atomics; a column's result does not depend on which columns share its warp.
__global__ void hand_hist_kernel(const UwHand* __restrict__ H)
{
    const int n = min(*H->count, H->cap);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        atomicAdd(&H->hist[H->key[t]], 1);
}

__global__ void hand_scan_kernel(const UwHand* __restrict__ H)
{
    if (threadIdx.x != 0) return;
    int acc = 0;
    for (int b = 0; b < UW_HAND_KEYS; b++) {
        const int c = H->hist[b];
        H->hist[b] = acc;
        acc += c;
    }
}

__global__ void hand_scatter_kernel(const UwHand* __restrict__ H)
{
    const int n = min(*H->count, H->cap);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        H->order[atomicAdd(&H->hist[H->key[t]], 1)] = t;
}

// Hand-off region r sized for calls of iend columns with mkx levels and ncnst tracers; nullptr when
// the device has no room for it (the caller then runs the unsplit worklist pass).
// Offset of the [count, hist] block in a hand-off region.
constexpr size_t kHandCountOffset = (sizeof(UwHand) + 255) & ~(size_t)255;

// One hand-off region of cap slots of words doubles: its device UwHand at the start; nullptr when
// the device has no room for it.
char* hand_alloc(size_t cap, size_t words)
{
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t o_cnt = kHandCountOffset, o_col = o_cnt + up((1 + UW_HAND_KEYS) * sizeof(int)),
                 o_key = o_col + up(cap * sizeof(int)), o_ord = o_key + up(cap * sizeof(int)),
                 o_st = o_ord + up(cap * sizeof(int)), bytes = o_st + words * cap * sizeof(double);
    char* base = nullptr;
    if (cudaMalloc(&base, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    UwHand u{};
    u.state = reinterpret_cast<double*>(base + o_st);
    u.cap = (int)cap;
    u.count = reinterpret_cast<int*>(base + o_cnt);
    u.hist = u.count + 1;
    u.col = reinterpret_cast<int*>(base + o_col);
    u.key = reinterpret_cast<int*>(base + o_key);
    u.order = reinterpret_cast<int*>(base + o_ord);
    if (cudaMemcpy(base, &u, sizeof(u), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(base);
        return nullptr;
    }
    return base;
}

// Slots of a region for calls of iend columns with state of words doubles per slot.
size_t hand_slots_for(int iend, size_t words)
{
    size_t cap = std::min((size_t)iend, kHandBytes / (words * sizeof(double)));
    if (S().hand_slots > 0) cap = std::min(cap, (size_t)S().hand_slots);
    return std::max(cap, (size_t)32);
}

const UwHand* hand_region(HandRegion& h, int iend, int mkx, int ncnst)
{
    const size_t words = uw_state_words(mkx, ncnst);
    size_t cap = hand_slots_for(iend, words);
    if (S().hand_slots > 0 && h.base && h.cap > cap) {   // a smaller limit applies to this region now
        cudaFree(h.base);
        h = HandRegion{};
    }
    if (h.base && h.cap >= cap && h.words >= words) return reinterpret_cast<const UwHand*>(h.base);
    cap = std::max(cap, h.cap);
    const size_t nw = std::max(words, h.words);
    if (h.base) cudaFree(h.base);
    h = HandRegion{};
    char* base = hand_alloc(cap, nw);
    if (!base) return nullptr;
    h.base = base;
    h.cap = cap;
    h.words = nw;
    return reinterpret_cast<const UwHand*>(base);
}

// The worklist pass over list[0 .. *count): one UW_MODE_LIST launch, or with the sorted schedule
// the split pass through hand-off region r: UW_MODE_LIST1, the sort of the handed-off
// columns by iteration-1 updraft depth, UW_MODE_RESUME.
// The key of worklist entry j for the ordering by the last call's depth (list entries beyond the
// count sort last).
__global__ void depth_list_key_kernel(const int* __restrict__ list, const int* __restrict__ count, int n,
                                      const int* __restrict__ dkey, int* __restrict__ key)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    key[j] = j < *count ? dkey[list[j]] : 255;
}

// A key array of at least n entries, zero where new (the keys of columns no call has computed yet).
int grow_keys(int*& buf, size_t& cap, size_t n)
{
    if (n <= cap) return UWSHCU_OK;
    cudaError_t e;
    if (buf && (e = cudaFree(buf)) != cudaSuccess) return cuda_fail(e);
    buf = nullptr;
    cap = 0;
    if ((e = cudaMalloc(&buf, n * sizeof(int))) != cudaSuccess) return cuda_fail(e);
    if ((e = cudaMemset(buf, 0, n * sizeof(int))) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess)
        return cuda_fail(e);
    cap = n;
    return UWSHCU_OK;
}

// list[0 .. *count) in ascending order of dkey[column] (stable), through the region's sort buffers.
cudaError_t order_by_depth(HandRegion& h, int* list, const int* count, int n, const int* dkey, cudaStream_t st)
{
    cudaError_t e;
    size_t pb = 0;
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, pb, (const int*)nullptr, (int*)nullptr, (const int*)nullptr,
                                             (int*)nullptr, n, 0, 8, st)) != cudaSuccess)
        return e;
    const size_t seg = ((size_t)n * sizeof(int) + 255) / 256 * 256, need = 3 * seg + pb;
    if (need > h.dsort_bytes) {
        if (h.dsort && (e = cudaFree(h.dsort)) != cudaSuccess) return e;
        h.dsort = nullptr;
        h.dsort_bytes = 0;
        if ((e = cudaMalloc(&h.dsort, need + need / 8)) != cudaSuccess) return e;
        h.dsort_bytes = need + need / 8;
    }
    int* key = reinterpret_cast<int*>(h.dsort);
    int* key_o = reinterpret_cast<int*>(h.dsort + seg);
    int* list_o = reinterpret_cast<int*>(h.dsort + 2 * seg);
    depth_list_key_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(list, count, n, dkey, key);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cub::DeviceRadixSort::SortPairs(h.dsort + 3 * seg, pb, key, key_o, list, list_o, n, 0, 8, st)) != cudaSuccess)
        return e;
    return cudaMemcpyAsync(list, list_o, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, st);
}

// dkey (optional): each column's ordering key, read to order list[] before the first worklist
// launch and rewritten by it for the next call (uwshcu_set_depth_order).
cudaError_t worklist_pass(HandRegion& h, UwArgs A, int* list, int* count, cudaStream_t st, int* dkey)
{
    State& s = S();
    if (dkey) {
        A.depth_key = dkey;
        const cudaError_t e = order_by_depth(h, list, count, A.iend, dkey, st);
        if (e != cudaSuccess) return e;
    }
    const UwHand* H = nullptr;
    if (s.schedule == UWSHCU_SCHED_SORTED) H = hand_region(h, A.iend, A.mkx, A.ncnst);
    if (!H) return launch_mode(&A, s.precision, kModeList, list, count, A.iend, s.block, st);
    cudaError_t e;
    A.hand = H;
    int* cnt = reinterpret_cast<int*>(h.base + kHandCountOffset);
    if ((e = cudaMemsetAsync(cnt, 0, (1 + UW_HAND_KEYS) * sizeof(int), st)) != cudaSuccess) return e;
    if ((e = launch_mode(&A, s.precision, kModeList1, list, count, A.iend, s.block, st)) != cudaSuccess) return e;
    const int nb = (int)std::min((h.cap + 255) / 256, (size_t)1184);
    hand_hist_kernel<<<nb, 256, 0, st>>>(H);
    hand_scan_kernel<<<1, 32, 0, st>>>(H);
    hand_scatter_kernel<<<nb, 256, 0, st>>>(H);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_mode(&A, s.precision, kModeResume, nullptr, nullptr, (int)h.cap, s.block, st);
}

// Enqueue the column computation for A on st with the selected schedule.
// A device-array call on stream st with the stream's context c (A.err is set here).
int enqueue(DeviceState& d, StreamCtx& c, UwArgs A, cudaStream_t st)
{
    State& s = S();
    cudaError_t e;
    A.err = c.err;
    if (s.schedule == UWSHCU_SCHED_SINGLE_PASS) {
        if ((e = launch_mode(&A, s.precision, kModeAll, nullptr, nullptr, A.iend, s.block, st)) != cudaSuccess) return cuda_fail(e);
        return UWSHCU_OK;
    }
    int rc = grow_ints(c.wl, c.wl_cap, (size_t)A.iend + 1);
    if (rc != UWSHCU_OK) return rc;
    int* count = c.wl;
    int* list = c.wl + 1;
    d.last_count = count;
    cudaEvent_t* ev = nullptr;
    if (s.profiling && d.nrec < DeviceState::kSlots) {
        ev = d.ev[d.nrec];
        for (int j = 0; j < 3; j++)
            if (!ev[j] && (e = cudaEventCreate(&ev[j])) != cudaSuccess) return cuda_fail(e);
        d.nrec++;
    }
    if ((e = cudaMemsetAsync(count, 0, sizeof(int), st)) != cudaSuccess) return cuda_fail(e);
    if (ev && (e = cudaEventRecord(ev[0], st)) != cudaSuccess) return cuda_fail(e);
    if ((e = launch_mode(&A, s.precision, kModeTrigger, list, count, A.iend, s.block, st)) != cudaSuccess) return cuda_fail(e);
    if (ev && (e = cudaEventRecord(ev[1], st)) != cudaSuccess) return cuda_fail(e);
    int* dkey = nullptr;
    if (s.depth_order) {
        if ((rc = grow_keys(c.dkey, c.dkey_cap, (size_t)A.iend)) != UWSHCU_OK) return rc;
        dkey = c.dkey;
    }
    if ((e = worklist_pass(c.hand, A, list, count, st, dkey)) != cudaSuccess) return cuda_fail(e);
    if (ev && (e = cudaEventRecord(ev[2], st)) != cudaSuccess) return cuda_fail(e);
    return UWSHCU_OK;
}

bool bad_dims(int mix, int mkx, int iend, int ncnst)
{
    if (S().precision == UWSHCU_PREC_MIXED && ncnst > 5) return true;
    return mix < 1 || mkx < 3 || mkx > UWSHCU_MAX_LEVELS || iend < 0 || iend > mix || ncnst < 3 ||
           ncnst > UWSHCU_MAX_TRACERS || ncnst != S().k.ncnst;
}

// Host-pointer call shared by compute_uwshcu_ (inv = 0) and compute_uwshcu_inv_ (inv = 1), and by
// the compute_zwshcu entries (omega: the pressure velocity (mix, mkx) in the call's level order).
// Column arrays use leading dimension mix on the host and n = iend on the device.
int host_call(int inv, int mix, int mkx, int iend, int ncnst, double dt, const double* ps0,
              const double* zs0, const double* p0, const double* z0, const double* dp0,
              const double* u0, const double* v0, const double* qv0, const double* ql0,
              const double* qi0, const double* t0, const double* s0, const double* tr0,
              const double* tke, const double* pblh, double* cush, double* umf, double* slflx,
              double* qtflx, double* flxprc1, double* flxsnow1, double* qvten, double* qlten,
              double* qiten, double* sten, double* uten, double* vten, double* trten,
              double* qrten, double* qsten, double* precip, double* snow, double* evapc,
              double* cufrc, double* qcu, double* qlu, double* qiu, double* cbmf, double* qc,
              double* rliq, double* cnt, double* cnb, const double* dpdry0, double* wu,
              const double* omega)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (bad_dims(mix, mkx, iend, ncnst)) return UWSHCU_ERR_BAD_ARGS;
    if (omega && s.precision != UWSHCU_PREC_FP64) return UWSHCU_ERR_BAD_ARGS;   // compute_zwshcu: FP64
    const void* need[] = {ps0, zs0, p0, z0, dp0, u0, v0, qv0, ql0, qi0, t0, s0, tr0, tke, pblh, cush,
                          umf, slflx, qtflx, flxprc1, flxsnow1, qvten, qlten, qiten, sten, uten, vten,
                          trten, qrten, qsten, precip, snow, evapc, cufrc, qcu, qlu, qiu, cbmf, qc, rliq,
                          cnt, cnb, dpdry0, wu};
    for (const void* p : need)
        if (!p) return UWSHCU_ERR_BAD_ARGS;
    if (iend == 0) return UWSHCU_OK;
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;

    const size_t n = (size_t)iend, ld = (size_t)mix, KI = (size_t)mkx + 1, KL = (size_t)mkx;
    const size_t KT = KL * (size_t)ncnst;
    // Column chunks, each a compact (nc-column) copy of its inputs and outputs in the arena (and, for
    // pageable caller arrays, in the pinned staging area).  Three-stage pipeline: the copy-in stream
    // takes every chunk's inputs back to back, chunk c computes (trigger + worklist pass) on
    // pipe[c % pipe_streams] once its inputs are in, and the copy-out stream takes its outputs once
    // it is computed.  The host packs chunk c+1 while the GPU works on chunk c and unpacks the
    // chunks in order as they arrive.  Each chunk has its own worklist and endrun word.
    const size_t per_in = 3 * KI + 11 * KL + KT + 2 + (omega ? KL : 0);   // doubles per column, input block
    const size_t per_out = 6 * KI + 14 * KL + KT + 7;    // doubles per column, output block
    // Default shape: chunks of n/8 columns (32,768 .. 262,144, a multiple of 1,024), 4 streams up to
    // 65,536-column chunks and 2 above: enough convecting columns in flight to fill the GPU (a
    // chunk's worklist pass lasts as long as its deepest columns, whatever its size), few enough
    // chunks for the copies to overlap.  Measured at 1,048,576 columns (page-locked arrays): 217 ms
    // with 131,072 x 2 against 272 ms with 32,768 x 4, 210 ms with the ramped ends below; at
    // 259,200 columns 32,768 x 4 is best.
    size_t csz = s.chunk_columns > 0 ? (size_t)s.chunk_columns : n;
    size_t nstreams = (size_t)s.pipe_streams;
    if (s.pipe_auto) {
        csz = std::min<size_t>(std::max<size_t>((n / 8 + 1023) / 1024 * 1024, 32768), 262144);
        nstreams = csz > 65536 ? 2 : 4;
    }
    // The chunks: [c0, c0 + nc).  The auto shape (and an explicit chunk_columns below -1) ramps at
    // both ends (a quarter, then a half of the chunk size first and last, 32,768 columns at least):
    // the first chunk's inputs are in, and the last chunk's outputs are out, sooner.
    std::vector<std::pair<size_t, size_t>> chunks;
    {
        std::vector<size_t> head, tail;
        size_t rest = n;
        if (s.pipe_ramp && csz < n)
            for (size_t f = 4; f >= 2; f /= 2) {
                const size_t r = std::max<size_t>(csz / f, 32768);
                if (r >= csz || rest < 2 * r + 2 * csz) break;
                head.push_back(r);
                tail.push_back(r);
                rest -= 2 * r;
            }
        size_t c0 = 0;
        auto put = [&](size_t nc) {
            chunks.emplace_back(c0, nc);
            c0 += nc;
        };
        for (size_t nc : head) put(nc);
        for (size_t body = rest; body > 0;) {
            const size_t nc = std::min(csz, body);
            put(nc);
            body -= nc;
        }
        for (size_t j = tail.size(); j-- > 0;) put(tail[j]);
    }
    const size_t nch = chunks.size();
    const size_t nin = per_in * n, nout = per_out * n;
    // Page-locked caller arrays: every plane goes straight between them and the device with a
    // strided copy (no host packing, no staging); otherwise through the pinned staging area.
    bool direct = true;
    {
        const double* arrays[] = {ps0, zs0, tke, p0, z0, dp0, u0, v0, qv0, ql0, qi0, t0, s0, dpdry0, tr0, pblh,
                                  cush, umf, slflx, qtflx, flxprc1, flxsnow1, wu, qvten, qlten, qiten, sten,
                                  uten, vten, qrten, qsten, evapc, cufrc, qcu, qlu, qiu, qc, trten, precip,
                                  snow, cbmf, rliq, cnt, cnb};
        const size_t rows[] = {KI, KI, KI, KL, KL, KL, KL, KL, KL, KL, KL, KL, KL, KL, KT, 1,
                               1, KI, KI, KI, KI, KI, KI, KL, KL, KL, KL,
                               KL, KL, KL, KL, KL, KL, KL, KL, KL, KL, KT, 1,
                               1, 1, 1, 1, 1};
        static_assert(sizeof(arrays) / sizeof(arrays[0]) == sizeof(rows) / sizeof(rows[0]), "one row count per array");
        for (size_t a = 0; a < sizeof(rows) / sizeof(rows[0]) && direct; a++)
            direct = pinned_range(arrays[a], ((rows[a] - 1) * ld + n) * sizeof(double));
        if (direct && omega) direct = pinned_range(omega, ((KL - 1) * ld + n) * sizeof(double));
    }
    if ((rc = grow(*d, nin + nout, direct ? 2 * nch : nin + nout + 2 * nch)) != UWSHCU_OK) return rc;
    if ((rc = grow_worklist(*d, n + 2 * nch)) != UWSHCU_OK) return rc;
    if (s.depth_order && (rc = grow_keys(d->hkey, d->hkey_cap, n)) != UWSHCU_OK) return rc;
    cudaError_t e;
    if (!d->pipe[0]) {
        int least = 0, greatest = 0;
        if ((e = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess) return cuda_fail(e);
        for (int j = 0; j < DeviceState::kPipe; j++) {
            const int prio = greatest + (least - greatest) * j / (DeviceState::kPipe - 1);
            if ((e = cudaStreamCreateWithPriority(&d->pipe[j], cudaStreamNonBlocking, prio)) != cudaSuccess)
                return cuda_fail(e);
        }
    }
    if (!d->pin) {
        if ((e = cudaStreamCreateWithFlags(&d->pin, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e);
        if ((e = cudaStreamCreateWithFlags(&d->pout, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e);
    }
    for (std::vector<cudaEvent_t>* v : {&d->done, &d->ev_in, &d->ev_comp})
        while (v->size() < nch) {
            cudaEvent_t ev;
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_fail(e);
            v->push_back(ev);
        }
    unsigned int* hbits = reinterpret_cast<unsigned int*>(d->h_buf + (direct ? 0 : nin + nout));   // nch words

    std::vector<std::vector<Plane>> outs(nch);
    size_t base_in = 0, base_out = 0;
    for (size_t c = 0; c < nch; c++) {
        const size_t c0 = chunks[c].first, nc = chunks[c].second;
        double* hin = direct ? nullptr : d->h_buf + base_in;
        double* hout = direct ? nullptr : d->h_buf + nin + base_out;
        double* din = d->d_buf + base_in;
        double* dout = d->d_buf + nin + base_out;
        base_in += per_in * nc;
        base_out += per_out * nc;
        std::vector<Plane> in;
        size_t off = 0;
        auto add_in = [&](const double* a, size_t rows) -> const double* {
            in.push_back(Plane{a + c0, direct ? nullptr : hin + off, rows, ld, nc, nc, din + off});
            const double* dp = din + off;
            off += rows * nc;
            return dp;
        };
        UwArgs A{};
        A.mix = (int)nc;
        A.mkx = mkx;
        A.iend = (int)nc;
        A.ncnst = ncnst;
        A.inv = inv;
        A.dt = dt;
        A.ps0 = add_in(ps0, KI);
        A.zs0 = add_in(zs0, KI);
        A.tke = add_in(tke, KI);
        A.p0 = add_in(p0, KL);
        A.z0 = add_in(z0, KL);
        A.dp0 = add_in(dp0, KL);
        A.u0 = add_in(u0, KL);
        A.v0 = add_in(v0, KL);
        A.qv0 = add_in(qv0, KL);
        A.ql0 = add_in(ql0, KL);
        A.qi0 = add_in(qi0, KL);
        A.t0 = add_in(t0, KL);
        A.s0 = add_in(s0, KL);
        A.dpdry0 = add_in(dpdry0, KL);
        A.tr0 = add_in(tr0, KT);   // (mix, mkx, ncnst): mkx*ncnst rows of mix
        A.pblh = add_in(pblh, 1);
        A.cush = const_cast<double*>(add_in(cush, 1));
        A.omega = omega ? add_in(omega, KL) : nullptr;
        if (!direct) copy_planes(in);

        std::vector<Plane>& out = outs[c];
        size_t oo = 0;
        auto add_out = [&](double* a, size_t rows) -> double* {
            out.push_back(Plane{direct ? nullptr : hout + oo, a + c0, rows, nc, ld, nc, dout + oo});
            double* dp = dout + oo;
            oo += rows * nc;
            return dp;
        };
        A.umf = add_out(umf, KI);
        A.slflx = add_out(slflx, KI);
        A.qtflx = add_out(qtflx, KI);
        A.flxprc1 = add_out(flxprc1, KI);
        A.flxsnow1 = add_out(flxsnow1, KI);
        A.wu = add_out(wu, KI);
        A.qvten = add_out(qvten, KL);
        A.qlten = add_out(qlten, KL);
        A.qiten = add_out(qiten, KL);
        A.sten = add_out(sten, KL);
        A.uten = add_out(uten, KL);
        A.vten = add_out(vten, KL);
        A.qrten = add_out(qrten, KL);
        A.qsten = add_out(qsten, KL);
        A.evapc = add_out(evapc, KL);
        A.cufrc = add_out(cufrc, KL);
        A.qcu = add_out(qcu, KL);
        A.qlu = add_out(qlu, KL);
        A.qiu = add_out(qiu, KL);
        A.qc = add_out(qc, KL);
        A.trten = add_out(trten, KT);
        A.precip = add_out(precip, 1);
        A.snow = add_out(snow, 1);
        A.cbmf = add_out(cbmf, 1);
        A.rliq = add_out(rliq, 1);
        A.cnt = add_out(cnt, 1);
        A.cnb = add_out(cnb, 1);
        // cush is in/out: the kernel rewrites it in place in the input block
        out.push_back(Plane{direct ? nullptr : hin + (A.cush - din), cush + c0, 1, nc, ld, nc, A.cush});
        // this chunk's worklist region: [0] count, [1] endrun bits, [2 ..] column ids
        int* wreg = d->d_wl + (c0 + 2 * c);
        A.err = reinterpret_cast<unsigned int*>(wreg + 1);
        A.diag_int = nullptr;
        A.diag_real = nullptr;

        cudaStream_t st = d->pipe[c % nstreams];
        if ((e = cudaMemsetAsync(wreg, 0, 2 * sizeof(int), d->pin)) != cudaSuccess) return cuda_fail(e);
        if (direct) {
            for (const Plane& p : in)
                if ((e = cudaMemcpy2DAsync(p.dev, p.dst_ld * sizeof(double), p.src, p.src_ld * sizeof(double),
                                           p.n * sizeof(double), p.rows, cudaMemcpyHostToDevice, d->pin)) != cudaSuccess)
                    return cuda_fail(e);
        } else if ((e = cudaMemcpyAsync(din, hin, per_in * nc * sizeof(double), cudaMemcpyHostToDevice, d->pin)) != cudaSuccess) {
            return cuda_fail(e);
        }
        if ((e = cudaEventRecord(d->ev_in[c], d->pin)) != cudaSuccess) return cuda_fail(e);
        if ((e = cudaStreamWaitEvent(st, d->ev_in[c], 0)) != cudaSuccess) return cuda_fail(e);
        if (s.schedule == UWSHCU_SCHED_SINGLE_PASS) {
            if ((e = launch_mode(&A, s.precision, kModeAll, nullptr, nullptr, A.iend, s.block, st)) != cudaSuccess)
                return cuda_fail(e);
        } else {
            if ((e = launch_mode(&A, s.precision, kModeTrigger, wreg + 2, wreg, A.iend, s.block, st)) != cudaSuccess)
                return cuda_fail(e);
            if ((e = worklist_pass(d->hand[1 + c % nstreams], A, wreg + 2, wreg, st,
                                   s.depth_order ? d->hkey + c0 : nullptr)) != cudaSuccess)
                return cuda_fail(e);
        }
        if ((e = cudaEventRecord(d->ev_comp[c], st)) != cudaSuccess) return cuda_fail(e);
        if ((e = cudaStreamWaitEvent(d->pout, d->ev_comp[c], 0)) != cudaSuccess) return cuda_fail(e);
        if (direct) {
            for (const Plane& p : out)
                if ((e = cudaMemcpy2DAsync(p.dst, p.dst_ld * sizeof(double), p.dev, p.src_ld * sizeof(double),
                                           p.n * sizeof(double), p.rows, cudaMemcpyDeviceToHost, d->pout)) != cudaSuccess)
                    return cuda_fail(e);
        } else {
            if ((e = cudaMemcpyAsync(hout, dout, per_out * nc * sizeof(double), cudaMemcpyDeviceToHost, d->pout)) != cudaSuccess)
                return cuda_fail(e);
            if ((e = cudaMemcpyAsync(hin + (A.cush - din), A.cush, nc * sizeof(double), cudaMemcpyDeviceToHost, d->pout)) != cudaSuccess)
                return cuda_fail(e);
        }
        if ((e = cudaMemcpyAsync(hbits + c, wreg + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, d->pout)) != cudaSuccess)
            return cuda_fail(e);
        if ((e = cudaEventRecord(d->done[c], d->pout)) != cudaSuccess) return cuda_fail(e);
    }
    unsigned int bits = 0;
    for (size_t c = 0; c < nch; c++) {
        if ((e = cudaEventSynchronize(d->done[c])) != cudaSuccess) return cuda_fail(e);
        if (!direct) copy_planes(outs[c]);
        bits |= hbits[c];
    }
    return status_from_bits(bits);
}

// Zeroes the adjoints of the index space warp w used: (nin + rows of the warp) x 32 doubles at
// adj + w * astride, one block per warp.
__global__ void adj_zero_kernel(double* __restrict__ adj, size_t astride, const int* __restrict__ nrow, int nin,
                                int rcap)
{
    const int w = blockIdx.x;
    const size_t n = (size_t)(nin + min(nrow[w], rcap)) * 32 / 2;
    double2* p = reinterpret_cast<double2*>(adj + (size_t)w * astride);
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) p[j] = make_double2(0.0, 0.0);
}

// The ordering key of candidate j (column wl[j]) from the FP64 path's level indices: the
// implicit-CIN columns (a second full iteration) after the explicit ones, then the updraft depth
// kpen - krel, the trip count of the column's updraft level loops.
__global__ void adj_key_kernel(const int* __restrict__ wl, int n, const int* __restrict__ diag, int mix,
                               int* __restrict__ key)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int i = wl[j];
    const int depth = diag[UW_DI_KPEN * (size_t)mix + i] - diag[UW_DI_KREL * (size_t)mix + i];
    const int implicit_cin = (diag[UW_DI_LIMIT * (size_t)mix + i] & UW_L_DELCIN) ? 0 : 1;
    key[j] = implicit_cin * 64 + min(max(depth, 0), 63);
}

__global__ void eval_math_kernel(int fn, const double* __restrict__ x, const double* __restrict__ y,
                                 double* __restrict__ out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v;
    switch (fn) {
    case 0: v = uw_exp(x[i]); break;
    case 1: v = uw_log(x[i]); break;
    case 2: v = uw_pow(x[i], y[i]); break;
    default: v = uw_erfc(x[i]); break;
    }
    out[i] = v;
}

}  // namespace

// ================================================================================== C ABI ======

extern "C" {

int uwshcu_init(double xlv, double cp, double xlf, double zvir, double r, double g, double ep2,
                double tmin, double tmax, double ttrice, int icephs, double epsqs, double rgasv,
                double tmelt, int ncnst, const double* qmin, const int* cnst_wet, int ixnumliq,
                int ixnumice)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (ncnst < 3 || ncnst > UWSHCU_MAX_TRACERS || !qmin || !cnst_wet || ixnumliq < 1 ||
        ixnumliq > ncnst || ixnumice < 1 || ixnumice > ncnst || !(cp > 0.0) || !(tmax > tmin) ||
        (int)(tmax - tmin + 2.000001) > UW_TBL)
        return UWSHCU_ERR_BAD_ARGS;
    double rpen = s.init ? s.k.rpen : 10.0;
    UwConst k{};
    // init_uwshcu (uwshcu.F90:230-239)
    k.xlv = xlv;
    k.xlf = xlf;
    k.xls = k.xlv + k.xlf;
    k.cp = cp;
    k.zvir = zvir;
    k.r = r;
    k.g = g;
    k.ep2 = ep2;
    k.p00 = 1.e5;
    k.rovcp = k.r / k.cp;
    k.rinv = 1.0 / k.r;
    k.rpen = rpen;
    k.rle = s.init ? s.k.rle : 0.1;       // uwshcu.F90:1036
    k.rkm = s.init ? s.k.rkm : 14.0;      // uwshcu.F90:1038
    k.criqc = s.init ? s.k.criqc : 0.7e-3; // uwshcu.F90:1065
    // compute_zwshcu options (zwshcu.F90:30-57; cloud_fraction.F90:52): the reference's defaults
    k.zw_lf = s.init ? s.k.zw_lf : 1;
    k.zw_fwcrit = s.init ? s.k.zw_fwcrit : 1.0;
    k.zw_ent = s.init ? s.k.zw_ent : 0;
    k.zw_ent0 = s.init ? s.k.zw_ent0 : 0.015;
    k.zw_cloud_sh = s.init ? s.k.zw_cloud_sh : 0;
    k.zw_ufrcd = s.init ? s.k.zw_ufrcd : 2.0;
    k.zw_ufrc0 = s.init ? s.k.zw_ufrc0 : 2.0;
    k.zw_ufrcz = s.init ? s.k.zw_ufrcz : 2.0;
    // gestbl (wv_saturation.F90:129-138, 181-185); esinti passes latvap, latice, rh2o, cpair
    k.tmin = tmin;
    k.tmax = tmax;
    k.ttrice = ttrice;
    k.icephs = icephs ? 1 : 0;
    k.epsqs = epsqs;
    k.hlatv = xlv;
    k.hlatf = xlf;
    k.rgasv = rgasv;
    k.cpws = cp;
    k.tmelt = tmelt;
    k.pcf[0] = 5.04469588506e-01;
    k.pcf[1] = -5.47288442819e+00;
    k.pcf[2] = -3.67471858735e-01;
    k.pcf[3] = -8.95963532403e-03;
    k.pcf[4] = -7.78053686625e-05;
    k.pcf[5] = 0.0;
    k.omeps = 1.0 - k.epsqs;
    k.trinv = (ttrice != 0.0) ? 1.0 / ttrice : 0.0;
    k.ncnst = ncnst;
    k.ixnumliq = ixnumliq;
    k.ixnumice = ixnumice;
    for (int m = 0; m < ncnst; m++) {
        k.qmin[m] = qmin[m];
        k.wet[m] = cnst_wet[m] != 0;
    }
    build_table(s.tbl, tmin, tmax, ttrice, k.icephs, tmelt);
    s.k = k;
    s.init = true;
    s.gen++;
    return UWSHCU_OK;
}

int uwshcu_set_params(double rpen, double rle, double rkm, double criqc)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (!(rpen > 0.0) || !(rle > 0.0) || !(rkm > 0.0) || !(criqc >= 0.0)) return UWSHCU_ERR_BAD_ARGS;
    s.k.rpen = rpen;
    s.k.rle = rle;
    s.k.rkm = rkm;
    s.k.criqc = criqc;
    s.gen++;
    return UWSHCU_OK;
}

int uwshcu_set_rpen(double rpen)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    s.k.rpen = rpen;
    s.gen++;
    return UWSHCU_OK;
}

int uwshcu_init_default(void)
{
    // CESM shr_const values (rair = R/mwdair, rh2o = R/mwwv, zvir = rh2o/rair - 1, epsilo = mwwv/mwdair)
    const double boltz = 1.38065e-23, avogad = 6.02214e26, rgas = avogad * boltz;
    const double mwdair = 28.966, mwwv = 18.016;
    const double rdair = rgas / mwdair, rwv = rgas / mwwv, zv = (rwv / rdair) - 1.0;
    const double qmin[5] = {1.e-12, 0.0, 0.0, 0.0, 0.0};
    const int wet[5] = {1, 1, 1, 1, 1};
    int rc = uwshcu_init(2.501e6, 1.00464e3, 3.337e5, zv, rdair, 9.80616, mwwv / mwdair, 173.16, 375.16,
                         20.0, 1, mwwv / mwdair, rwv, 273.15, 5, qmin, wet, 4, 5);
    if (rc != UWSHCU_OK) return rc;
    return uwshcu_set_params(10.0, 0.1, 14.0, 0.7e-3);
}

int uwshcu_set_precision(int mode)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (mode != UWSHCU_PREC_FP64 && mode != UWSHCU_PREC_MIXED && mode != UWSHCU_PREC_FAST) return UWSHCU_ERR_BAD_ARGS;
    s.precision = mode;
    return UWSHCU_OK;
}

int uwshcu_set_schedule(int schedule)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (schedule != UWSHCU_SCHED_SINGLE_PASS && schedule != UWSHCU_SCHED_TWO_PHASE &&
        schedule != UWSHCU_SCHED_SORTED)
        return UWSHCU_ERR_BAD_ARGS;
    s.schedule = schedule;
    return UWSHCU_OK;
}

int uwshcu_set_hand_slots(int slots)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (slots < 0) return UWSHCU_ERR_BAD_ARGS;
    s.hand_slots = slots == 0 ? 0 : std::max(slots, 32);
    return UWSHCU_OK;
}

int uwshcu_set_profiling(int on)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    s.profiling = on != 0;
    for (int dv = 0; dv < kMaxDev; dv++) s.dev[dv].nrec = 0;
    return UWSHCU_OK;
}

int uwshcu_profile_read(int* calls, double* trigger_ms, double* list_ms, int* list_columns)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!calls || !trigger_ms || !list_ms) return UWSHCU_ERR_BAD_ARGS;
    *calls = 0;
    *trigger_ms = 0.0;
    *list_ms = 0.0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return UWSHCU_ERR_NO_DEVICE;
    DeviceState& d = s.dev[dev];
    cudaError_t e;
    for (int n = 0; n < d.nrec; n++) {
        float a = 0.f, b = 0.f;
        if ((e = cudaEventSynchronize(d.ev[n][2])) != cudaSuccess) return cuda_fail(e);
        if ((e = cudaEventElapsedTime(&a, d.ev[n][0], d.ev[n][1])) != cudaSuccess) return cuda_fail(e);
        if ((e = cudaEventElapsedTime(&b, d.ev[n][1], d.ev[n][2])) != cudaSuccess) return cuda_fail(e);
        *trigger_ms += a;
        *list_ms += b;
    }
    *calls = d.nrec;
    if (list_columns) {
        int cnt = 0;
        if (d.last_count && (e = cudaMemcpy(&cnt, d.last_count, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_fail(e);
        *list_columns = cnt;
    }
    d.nrec = 0;
    return UWSHCU_OK;
}

int uwshcu_set_pipeline(int chunk_columns, int streams)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (chunk_columns == -1) {   // back to the shape that follows each call's size
        s.pipe_auto = true;
        s.pipe_ramp = true;
        return UWSHCU_OK;
    }
    if (streams < 1 || streams > DeviceState::kPipe) return UWSHCU_ERR_BAD_ARGS;
    // below -1: chunks of -chunk_columns columns with the automatic shape's ramped ends
    s.pipe_ramp = chunk_columns < -1;
    s.chunk_columns = chunk_columns < -1 ? -chunk_columns : chunk_columns;
    s.pipe_streams = streams;
    s.pipe_auto = false;
    return UWSHCU_OK;
}

int uwshcu_set_depth_order(int on)
{
    if (on != 0 && on != 1) return UWSHCU_ERR_BAD_ARGS;
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    s.depth_order = on != 0;
    return UWSHCU_OK;
}

int uwshcu_set_block(int threads)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (threads == 0) threads = 128;
    if (threads < 32 || threads > 128 || threads % 32) return UWSHCU_ERR_BAD_ARGS;
    s.block = threads;
    return UWSHCU_OK;
}

int uwshcu_get_estbl(double* out250)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (!out250) return UWSHCU_ERR_BAD_ARGS;
    std::memcpy(out250, s.tbl, sizeof(s.tbl));
    return UWSHCU_OK;
}

int uwshcu_finalize(void)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    int cur = 0;
    bool have = cudaGetDevice(&cur) == cudaSuccess;
    for (int dv = 0; dv < kMaxDev; dv++) {
        DeviceState& d = s.dev[dv];
        if (!d.d_buf && !d.h_buf && !d.stream && !d.pipe[0] && !d.adj_buf && !d.adj_aux && !d.sctx[0].err) continue;
        cudaSetDevice(dv);
        if (d.d_buf) cudaFree(d.d_buf);
        if (d.h_buf) cudaFreeHost(d.h_buf);
        if (d.d_wl) cudaFree(d.d_wl);
        for (StreamCtx& c : d.sctx) {
            if (c.err) cudaFree(c.err);
            if (c.wl) cudaFree(c.wl);
            if (c.hand.base) cudaFree(c.hand.base);
            if (c.hand.dsort) cudaFree(c.hand.dsort);
            if (c.dkey) cudaFree(c.dkey);
        }
        for (HandRegion& h : d.hand) {
            if (h.base) cudaFree(h.base);
            if (h.dsort) cudaFree(h.dsort);
        }
        if (d.hkey) cudaFree(d.hkey);
        if (d.adj_buf) cudaFree(d.adj_buf);
        if (d.adj_aux) cudaFree(d.adj_aux);
        for (int n = 0; n < DeviceState::kSlots; n++)
            for (int j = 0; j < 3; j++)
                if (d.ev[n][j]) cudaEventDestroy(d.ev[n][j]);
        if (d.stream) cudaStreamDestroy(d.stream);
        for (int j = 0; j < DeviceState::kPipe; j++)
            if (d.pipe[j]) cudaStreamDestroy(d.pipe[j]);
        for (cudaEvent_t ev : d.done) cudaEventDestroy(ev);
        for (cudaEvent_t ev : d.ev_in) cudaEventDestroy(ev);
        for (cudaEvent_t ev : d.ev_comp) cudaEventDestroy(ev);
        if (d.pin) cudaStreamDestroy(d.pin);
        if (d.pout) cudaStreamDestroy(d.pout);
        d = DeviceState{};
    }
    if (have) cudaSetDevice(cur);
    return UWSHCU_OK;
}

const char* uwshcu_last_cuda_error(void) { return S().lasterr; }

int compute_uwshcu_(const int* mix, const int* mkx, const int* iend, const int* ncnst, const double* dt,
                    const double* ps0_in, const double* zs0_in, const double* p0_in, const double* z0_in,
                    const double* dp0_in, const double* u0_in, const double* v0_in, const double* qv0_in,
                    const double* ql0_in, const double* qi0_in, const double* t0_in, const double* s0_in,
                    const double* tr0_in, const double* tke_in, const double* cldfrct_in,
                    const double* concldfrct_in, const double* pblh_in, double* cush_inout,
                    double* umf_out, double* slflx_out, double* qtflx_out, double* flxprc1_out,
                    double* flxsnow1_out, double* qvten_out, double* qlten_out, double* qiten_out,
                    double* sten_out, double* uten_out, double* vten_out, double* trten_out,
                    double* qrten_out, double* qsten_out, double* precip_out, double* snow_out,
                    double* evapc_out, double* cufrc_out, double* qcu_out, double* qlu_out,
                    double* qiu_out, double* cbmf_out, double* qc_out, double* rliq_out,
                    const double* massflx_sh, double* cnt_out, double* cnb_out, void* qsat,
                    const int* lchnk, const double* dpdry0_in, double* wu_out)
{
    (void)cldfrct_in;
    (void)concldfrct_in;
    (void)massflx_sh;
    (void)qsat;
    (void)lchnk;
    if (!mix || !mkx || !iend || !ncnst || !dt) return UWSHCU_ERR_BAD_ARGS;
    return host_call(0, *mix, *mkx, *iend, *ncnst, *dt, ps0_in, zs0_in, p0_in, z0_in, dp0_in, u0_in, v0_in,
                     qv0_in, ql0_in, qi0_in, t0_in, s0_in, tr0_in, tke_in, pblh_in, cush_inout, umf_out,
                     slflx_out, qtflx_out, flxprc1_out, flxsnow1_out, qvten_out, qlten_out, qiten_out,
                     sten_out, uten_out, vten_out, trten_out, qrten_out, qsten_out, precip_out, snow_out,
                     evapc_out, cufrc_out, qcu_out, qlu_out, qiu_out, cbmf_out, qc_out, rliq_out,
                     cnt_out, cnb_out, dpdry0_in, wu_out, nullptr);
}

int compute_uwshcu_inv_(const int* mix, const int* mkx, const int* iend, const int* ncnst, const double* dt,
                        const double* ps0_inv, const double* zs0_inv, const double* p0_inv,
                        const double* z0_inv, const double* dp0_inv, const double* u0_inv,
                        const double* v0_inv, const double* qv0_inv, const double* ql0_inv,
                        const double* qi0_inv, const double* t0_inv, const double* s0_inv,
                        const double* tr0_inv, const double* tke_inv, const double* cldfrct_inv,
                        const double* concldfrct_inv, const double* pblh, double* cush,
                        const double* tpert2, const double* qpert2, const double* massflx_sh,
                        double* umf_inv, double* slflx_inv, double* qtflx_inv, double* flxprc1_inv,
                        double* flxsnow1_inv, double* qvten_inv, double* qlten_inv, double* qiten_inv,
                        double* sten_inv, double* uten_inv, double* vten_inv, double* trten_inv,
                        double* qrten_inv, double* qsten_inv, double* precip, double* snow,
                        double* evapc_inv, double* cufrc_inv, double* qcu_inv, double* qlu_inv,
                        double* qiu_inv, double* cbmf, double* qc_inv, double* rliq, double* cnt_inv,
                        double* cnb_inv, void* qsat, const int* lchnk, const double* dpdry0_inv,
                        double* wu_inv)
{
    (void)cldfrct_inv;
    (void)concldfrct_inv;
    (void)tpert2;
    (void)qpert2;
    (void)massflx_sh;
    (void)qsat;
    (void)lchnk;
    if (!mix || !mkx || !iend || !ncnst || !dt) return UWSHCU_ERR_BAD_ARGS;
    return host_call(1, *mix, *mkx, *iend, *ncnst, *dt, ps0_inv, zs0_inv, p0_inv, z0_inv, dp0_inv, u0_inv,
                     v0_inv, qv0_inv, ql0_inv, qi0_inv, t0_inv, s0_inv, tr0_inv, tke_inv, pblh, cush,
                     umf_inv, slflx_inv, qtflx_inv, flxprc1_inv, flxsnow1_inv, qvten_inv, qlten_inv,
                     qiten_inv, sten_inv, uten_inv, vten_inv, trten_inv, qrten_inv, qsten_inv, precip,
                     snow, evapc_inv, cufrc_inv, qcu_inv, qlu_inv, qiu_inv, cbmf, qc_inv, rliq, cnt_inv,
                     cnb_inv, dpdry0_inv, wu_inv, nullptr);
}

// ---- compute_zwshcu (zwshcu.F90), the CAS-ESM variant: the same column code with the pressure
// velocity omega and the options of uwshcu_set_zw_options.

int compute_zwshcu_(const int* mix, const int* mkx, const int* iend, const int* ncnst, const double* dt,
                    const double* ps0_in, const double* zs0_in, const double* p0_in, const double* z0_in,
                    const double* dp0_in, const double* u0_in, const double* v0_in, const double* qv0_in,
                    const double* ql0_in, const double* qi0_in, const double* t0_in, const double* s0_in,
                    const double* tr0_in, const double* tke_in, const double* cldfrct_in,
                    const double* concldfrct_in, const double* pblh_in, double* cush_inout,
                    double* umf_out, double* slflx_out, double* qtflx_out, double* flxprc1_out,
                    double* flxsnow1_out, double* qvten_out, double* qlten_out, double* qiten_out,
                    double* sten_out, double* uten_out, double* vten_out, double* trten_out,
                    double* qrten_out, double* qsten_out, double* precip_out, double* snow_out,
                    double* evapc_out, double* cufrc_out, double* qcu_out, double* qlu_out,
                    double* qiu_out, double* cbmf_out, double* qc_out, double* rliq_out,
                    const double* omega, const double* massflx_sh, const double* tpert2,
                    double* cnt_out, double* cnb_out, void* qsat, const int* lchnk,
                    const double* dpdry0_in, double* wu_out)
{
    (void)cldfrct_in;
    (void)concldfrct_in;
    (void)massflx_sh;
    (void)tpert2;
    (void)qsat;
    (void)lchnk;
    if (!mix || !mkx || !iend || !ncnst || !dt || !omega) return UWSHCU_ERR_BAD_ARGS;
    return host_call(0, *mix, *mkx, *iend, *ncnst, *dt, ps0_in, zs0_in, p0_in, z0_in, dp0_in, u0_in, v0_in,
                     qv0_in, ql0_in, qi0_in, t0_in, s0_in, tr0_in, tke_in, pblh_in, cush_inout, umf_out,
                     slflx_out, qtflx_out, flxprc1_out, flxsnow1_out, qvten_out, qlten_out, qiten_out,
                     sten_out, uten_out, vten_out, trten_out, qrten_out, qsten_out, precip_out, snow_out,
                     evapc_out, cufrc_out, qcu_out, qlu_out, qiu_out, cbmf_out, qc_out, rliq_out,
                     cnt_out, cnb_out, dpdry0_in, wu_out, omega);
}

int compute_zwshcu_inv_(const int* mix, const int* mkx, const int* iend, const int* ncnst, const double* dt,
                        const double* ps0_inv, const double* zs0_inv, const double* p0_inv,
                        const double* z0_inv, const double* dp0_inv, const double* u0_inv,
                        const double* v0_inv, const double* qv0_inv, const double* ql0_inv,
                        const double* qi0_inv, const double* t0_inv, const double* s0_inv,
                        const double* tr0_inv, const double* tke_inv, const double* cldfrct_inv,
                        const double* concldfrct_inv, const double* pblh, double* cush,
                        const double* omega_inv, const double* tpert2, const double* qpert2,
                        const double* gradt, const double* gradq, const double* landfrac,
                        const double* lat, const double* lon, const double* massflx_sh,
                        double* umf_inv, double* slflx_inv, double* qtflx_inv, double* flxprc1_inv,
                        double* flxsnow1_inv, double* qvten_inv, double* qlten_inv, double* qiten_inv,
                        double* sten_inv, double* uten_inv, double* vten_inv, double* trten_inv,
                        double* qrten_inv, double* qsten_inv, double* precip, double* snow,
                        double* evapc_inv, double* cufrc_inv, double* qcu_inv, double* qlu_inv,
                        double* qiu_inv, double* cbmf, double* qc_inv, double* rliq, double* cnt_inv,
                        double* cnb_inv, void* qsat, const int* lchnk, const double* dpdry0_inv,
                        double* wu_inv)
{
    (void)cldfrct_inv;
    (void)concldfrct_inv;
    (void)tpert2;
    (void)qpert2;
    (void)gradt;
    (void)gradq;
    (void)landfrac;
    (void)lat;
    (void)lon;
    (void)massflx_sh;
    (void)qsat;
    (void)lchnk;
    if (!mix || !mkx || !iend || !ncnst || !dt || !omega_inv) return UWSHCU_ERR_BAD_ARGS;
    return host_call(1, *mix, *mkx, *iend, *ncnst, *dt, ps0_inv, zs0_inv, p0_inv, z0_inv, dp0_inv, u0_inv,
                     v0_inv, qv0_inv, ql0_inv, qi0_inv, t0_inv, s0_inv, tr0_inv, tke_inv, pblh, cush,
                     umf_inv, slflx_inv, qtflx_inv, flxprc1_inv, flxsnow1_inv, qvten_inv, qlten_inv,
                     qiten_inv, sten_inv, uten_inv, vten_inv, trten_inv, qrten_inv, qsten_inv, precip,
                     snow, evapc_inv, cufrc_inv, qcu_inv, qlu_inv, qiu_inv, cbmf, qc_inv, rliq, cnt_inv,
                     cnb_inv, dpdry0_inv, wu_inv, omega_inv);
}

int uwshcu_set_zw_options(int lf, double fwcrit, int ent, double ent0, int cloud_sh, double ufrcd,
                          double ufrc0, double ufrcz)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (!(fwcrit >= 0.0) || !(ent0 >= 0.0) || !(ufrc0 >= 0.0) || !(ufrcd >= 0.0) || !(ufrcz > -1.0))
        return UWSHCU_ERR_BAD_ARGS;
    s.k.zw_lf = lf != 0;
    s.k.zw_fwcrit = fwcrit;
    s.k.zw_ent = ent != 0;
    s.k.zw_ent0 = ent0;
    s.k.zw_cloud_sh = cloud_sh != 0;
    s.k.zw_ufrcd = ufrcd;
    s.k.zw_ufrc0 = ufrc0;
    s.k.zw_ufrcz = ufrcz;
    s.gen++;
    return UWSHCU_OK;
}

int bxcompute_uwshcu_inv_(const int* pcols, const int* pver, const int* ncol, const int* pcnst,
                          const double* ztodt, const double* ps0_inv, const double* zs0_inv,
                          const double* p0_inv, const double* z0_inv, const double* dp0_inv,
                          const double* u0_inv, const double* v0_inv, const double* qv0_inv,
                          const double* ql0_inv, const double* qi0_inv, const double* t0_inv,
                          const double* s0_inv, const double* tr0_inv, const double* tke_inv,
                          const double* cldfrct_inv, const double* concldfrct_inv, const double* pblh,
                          double* cush, double* umf_inv, double* slflx_inv, double* qtflx_inv,
                          double* flxprc1_inv, double* flxsnow1_inv, double* qvten_inv,
                          double* qlten_inv, double* qiten_inv, double* sten_inv, double* uten_inv,
                          double* vten_inv, double* trten_inv, double* qrten_inv, double* qsten_inv,
                          double* precip, double* snow, double* evapc_inv, double* cufrc_inv,
                          double* qcu_inv, double* qlu_inv, double* qiu_inv, double* cbmf,
                          double* qc_inv, double* rliq, double* cnt_inv, double* cnb_inv,
                          const int* lchnk, const double* dpdry0_inv, double* wu_inv)
{
    return compute_uwshcu_inv_(pcols, pver, ncol, pcnst, ztodt, ps0_inv, zs0_inv, p0_inv, z0_inv, dp0_inv,
                               u0_inv, v0_inv, qv0_inv, ql0_inv, qi0_inv, t0_inv, s0_inv, tr0_inv, tke_inv,
                               cldfrct_inv, concldfrct_inv, pblh, cush, nullptr, nullptr, nullptr, umf_inv,
                               slflx_inv, qtflx_inv, flxprc1_inv, flxsnow1_inv, qvten_inv, qlten_inv,
                               qiten_inv, sten_inv, uten_inv, vten_inv, trten_inv, qrten_inv, qsten_inv,
                               precip, snow, evapc_inv, cufrc_inv, qcu_inv, qlu_inv, qiu_inv, cbmf, qc_inv,
                               rliq, cnt_inv, cnb_inv, nullptr, lchnk, dpdry0_inv, wu_inv);
}

// A member's arrays are all given (the diagnostics are optional) and its sizes are valid.
static bool member_ok(const uwshcu_member& m, int ncnst)
{
    if (bad_dims(m.mix, m.mkx, m.iend, ncnst) || (m.inv != 0 && m.inv != 1)) return false;
    const void* need[] = {m.ps0, m.zs0, m.p0, m.z0, m.dp0, m.u0, m.v0, m.qv0, m.ql0, m.qi0, m.t0, m.s0, m.tr0,
                          m.tke, m.pblh, m.cush, m.umf, m.slflx, m.qtflx, m.flxprc1, m.flxsnow1, m.qvten,
                          m.qlten, m.qiten, m.sten, m.uten, m.vten, m.trten, m.qrten, m.qsten, m.precip,
                          m.snow, m.evapc, m.cufrc, m.qcu, m.qlu, m.qiu, m.cbmf, m.qc, m.rliq, m.cnt,
                          m.cnb, m.dpdry0, m.wu};
    for (const void* p : need)
        if (!p) return false;
    return true;
}

// The kernel arguments of one member.
static UwArgs member_args(const uwshcu_member& m, int ncnst, unsigned int* err)
{
    UwArgs A{};
    A.mix = m.mix; A.mkx = m.mkx; A.iend = m.iend; A.ncnst = ncnst; A.inv = m.inv; A.dt = m.dt;
    A.ps0 = m.ps0; A.zs0 = m.zs0; A.p0 = m.p0; A.z0 = m.z0; A.dp0 = m.dp0; A.u0 = m.u0; A.v0 = m.v0;
    A.qv0 = m.qv0; A.ql0 = m.ql0; A.qi0 = m.qi0; A.t0 = m.t0; A.s0 = m.s0; A.tr0 = m.tr0; A.tke = m.tke;
    A.pblh = m.pblh; A.cush = m.cush; A.umf = m.umf; A.slflx = m.slflx; A.qtflx = m.qtflx;
    A.flxprc1 = m.flxprc1; A.flxsnow1 = m.flxsnow1; A.qvten = m.qvten; A.qlten = m.qlten; A.qiten = m.qiten;
    A.sten = m.sten; A.uten = m.uten; A.vten = m.vten; A.trten = m.trten; A.qrten = m.qrten;
    A.qsten = m.qsten; A.precip = m.precip; A.snow = m.snow; A.evapc = m.evapc; A.cufrc = m.cufrc;
    A.qcu = m.qcu; A.qlu = m.qlu; A.qiu = m.qiu; A.cbmf = m.cbmf; A.qc = m.qc; A.rliq = m.rliq;
    A.cnt = m.cnt; A.cnb = m.cnb; A.dpdry0 = m.dpdry0; A.wu = m.wu; A.diag_int = m.diag_int;
    A.diag_real = m.diag_real; A.diag_level = m.diag_level; A.err = err;
    return A;
}

int uwshcu_compute_member(const uwshcu_member* m, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (!m || !member_ok(*m, s.k.ncnst)) return UWSHCU_ERR_BAD_ARGS;
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    StreamCtx* c = nullptr;
    if ((rc = stream_ctx(*d, (cudaStream_t)stream, &c)) != UWSHCU_OK) return rc;
    return enqueue(*d, *c, member_args(*m, s.k.ncnst, c->err), (cudaStream_t)stream);
}

int uwshcu_compute_device(int mix, int mkx, int iend, int ncnst, double dt, int inv, const double* ps0,
                          const double* zs0, const double* p0, const double* z0, const double* dp0,
                          const double* u0, const double* v0, const double* qv0, const double* ql0,
                          const double* qi0, const double* t0, const double* s0, const double* tr0,
                          const double* tke, const double* pblh, double* cush, double* umf,
                          double* slflx, double* qtflx, double* flxprc1, double* flxsnow1,
                          double* qvten, double* qlten, double* qiten, double* sten, double* uten,
                          double* vten, double* trten, double* qrten, double* qsten, double* precip,
                          double* snow, double* evapc, double* cufrc, double* qcu, double* qlu,
                          double* qiu, double* cbmf, double* qc, double* rliq, double* cnt,
                          double* cnb, const double* dpdry0, double* wu, int* diag_int,
                          double* diag_real, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (bad_dims(mix, mkx, iend, ncnst) || (inv != 0 && inv != 1)) return UWSHCU_ERR_BAD_ARGS;
    const void* need[] = {ps0, zs0, p0, z0, dp0, u0, v0, qv0, ql0, qi0, t0, s0, tr0, tke, pblh, cush,
                          umf, slflx, qtflx, flxprc1, flxsnow1, qvten, qlten, qiten, sten, uten, vten,
                          trten, qrten, qsten, precip, snow, evapc, cufrc, qcu, qlu, qiu, cbmf, qc, rliq,
                          cnt, cnb, dpdry0, wu};
    for (const void* p : need)
        if (!p) return UWSHCU_ERR_BAD_ARGS;
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    UwArgs A{};
    A.mix = mix; A.mkx = mkx; A.iend = iend; A.ncnst = ncnst; A.inv = inv; A.dt = dt;
    A.ps0 = ps0; A.zs0 = zs0; A.p0 = p0; A.z0 = z0; A.dp0 = dp0; A.u0 = u0; A.v0 = v0; A.qv0 = qv0;
    A.ql0 = ql0; A.qi0 = qi0; A.t0 = t0; A.s0 = s0; A.tr0 = tr0; A.tke = tke; A.pblh = pblh; A.cush = cush;
    A.umf = umf; A.slflx = slflx; A.qtflx = qtflx; A.flxprc1 = flxprc1; A.flxsnow1 = flxsnow1;
    A.qvten = qvten; A.qlten = qlten; A.qiten = qiten; A.sten = sten; A.uten = uten; A.vten = vten;
    A.trten = trten; A.qrten = qrten; A.qsten = qsten; A.precip = precip; A.snow = snow; A.evapc = evapc;
    A.cufrc = cufrc; A.qcu = qcu; A.qlu = qlu; A.qiu = qiu; A.cbmf = cbmf; A.qc = qc; A.rliq = rliq;
    A.cnt = cnt; A.cnb = cnb; A.dpdry0 = dpdry0; A.wu = wu; A.diag_int = diag_int; A.diag_real = diag_real;
    StreamCtx* c = nullptr;
    if ((rc = stream_ctx(*d, (cudaStream_t)stream, &c)) != UWSHCU_OK) return rc;
    return enqueue(*d, *c, A, (cudaStream_t)stream);
}

// compute_zwshcu on device-resident arrays: uwshcu_compute_device plus omega (mix, mkx).
int compute_zwshcu_device(int mix, int mkx, int iend, int ncnst, double dt, int inv, const double* ps0,
                          const double* zs0, const double* p0, const double* z0, const double* dp0,
                          const double* u0, const double* v0, const double* qv0, const double* ql0,
                          const double* qi0, const double* t0, const double* s0, const double* tr0,
                          const double* tke, const double* pblh, const double* omega, double* cush, double* umf,
                          double* slflx, double* qtflx, double* flxprc1, double* flxsnow1,
                          double* qvten, double* qlten, double* qiten, double* sten, double* uten,
                          double* vten, double* trten, double* qrten, double* qsten, double* precip,
                          double* snow, double* evapc, double* cufrc, double* qcu, double* qlu,
                          double* qiu, double* cbmf, double* qc, double* rliq, double* cnt,
                          double* cnb, const double* dpdry0, double* wu, int* diag_int,
                          double* diag_real, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (bad_dims(mix, mkx, iend, ncnst) || (inv != 0 && inv != 1)) return UWSHCU_ERR_BAD_ARGS;
    if (s.precision != UWSHCU_PREC_FP64) return UWSHCU_ERR_BAD_ARGS;   // compute_zwshcu: FP64 only
    const void* need[] = {ps0, zs0, p0, z0, dp0, u0, v0, qv0, ql0, qi0, t0, s0, tr0, tke, pblh, omega, cush,
                          umf, slflx, qtflx, flxprc1, flxsnow1, qvten, qlten, qiten, sten, uten, vten,
                          trten, qrten, qsten, precip, snow, evapc, cufrc, qcu, qlu, qiu, cbmf, qc, rliq,
                          cnt, cnb, dpdry0, wu};
    for (const void* p : need)
        if (!p) return UWSHCU_ERR_BAD_ARGS;
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    UwArgs A{};
    A.mix = mix; A.mkx = mkx; A.iend = iend; A.ncnst = ncnst; A.inv = inv; A.dt = dt;
    A.ps0 = ps0; A.zs0 = zs0; A.p0 = p0; A.z0 = z0; A.dp0 = dp0; A.u0 = u0; A.v0 = v0; A.qv0 = qv0;
    A.ql0 = ql0; A.qi0 = qi0; A.t0 = t0; A.s0 = s0; A.tr0 = tr0; A.tke = tke; A.pblh = pblh; A.cush = cush;
    A.umf = umf; A.slflx = slflx; A.qtflx = qtflx; A.flxprc1 = flxprc1; A.flxsnow1 = flxsnow1;
    A.qvten = qvten; A.qlten = qlten; A.qiten = qiten; A.sten = sten; A.uten = uten; A.vten = vten;
    A.trten = trten; A.qrten = qrten; A.qsten = qsten; A.precip = precip; A.snow = snow; A.evapc = evapc;
    A.cufrc = cufrc; A.qcu = qcu; A.qlu = qlu; A.qiu = qiu; A.cbmf = cbmf; A.qc = qc; A.rliq = rliq;
    A.cnt = cnt; A.cnb = cnb; A.dpdry0 = dpdry0; A.wu = wu; A.diag_int = diag_int; A.diag_real = diag_real;
    A.omega = omega;
    StreamCtx* c = nullptr;
    if ((rc = stream_ctx(*d, (cudaStream_t)stream, &c)) != UWSHCU_OK) return rc;
    return enqueue(*d, *c, A, (cudaStream_t)stream);
}

int uwshcu_budget_device(int mix, int mkx, int iend, int inv, double dt, const double* s0,
                         const double* qv0, const double* ql0, const double* qi0, const double* u0,
                         const double* v0, const double* dp0, const double* sten, const double* qvten,
                         const double* qlten, const double* qiten, const double* uten,
                         const double* vten, const double* precip, const double* snow,
                         const double* rliq, double* te_rer, double* tw_rer, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (mix < 1 || mkx < 1 || iend < 0 || iend > mix || (inv != 0 && inv != 1)) return UWSHCU_ERR_BAD_ARGS;
    const void* need[] = {s0, qv0, ql0, qi0, u0, v0, dp0, sten, qvten, qlten, qiten, uten, vten, precip,
                          snow, rliq, te_rer, tw_rer};
    for (const void* p : need)
        if (!p) return UWSHCU_ERR_BAD_ARGS;
    cudaError_t e = uw_budget_launch(mix, mkx, iend, inv, dt, s.k.xlv, s.k.xlf, s.k.g, s0, qv0, ql0, qi0, u0, v0,
                                     dp0, sten, qvten, qlten, qiten, uten, vten, precip, snow, rliq, te_rer,
                                     tw_rer, (cudaStream_t)stream);
    return e == cudaSuccess ? UWSHCU_OK : cuda_fail(e);
}

int uwshcu_tangent_device(const uwshcu_member* m, const uwshcu_tangent* t, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (!m || !t) return UWSHCU_ERR_BAD_ARGS;
    const int ncnst = s.k.ncnst;
    if (s.precision != UWSHCU_PREC_FP64 || ncnst > 5 || m->mkx + 1 > 64) return UWSHCU_ERR_BAD_ARGS;
    if (!member_ok(*m, ncnst)) return UWSHCU_ERR_BAD_ARGS;
    const void* need[] = {t->cush, t->umf, t->slflx, t->qtflx, t->flxprc1, t->flxsnow1, t->qvten, t->qlten,
                          t->qiten, t->sten, t->uten, t->vten, t->trten, t->qrten, t->qsten, t->precip,
                          t->snow, t->evapc, t->cufrc, t->qcu, t->qlu, t->qiu, t->cbmf, t->qc, t->rliq, t->wu};
    for (const void* p : need)
        if (!p) return UWSHCU_ERR_BAD_ARGS;
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    StreamCtx* c = nullptr;
    if ((rc = stream_ctx(*d, st, &c)) != UWSHCU_OK) return rc;
    UwArgs A = member_args(*m, ncnst, c->err);
    // the forward path's two-phase schedule: trigger pass, then the convecting columns
    auto launch = (m->mkx + 1 <= 32) ? uw_tl_launch_k32n5 : uw_tl_launch_k64n5;
    cudaError_t e;
    if ((rc = grow_ints(c->wl, c->wl_cap, (size_t)m->iend + 1)) != UWSHCU_OK) return rc;
    int* wl = c->wl;
    if ((e = cudaMemsetAsync(wl, 0, sizeof(int), st)) != cudaSuccess) return cuda_fail(e);
    if ((e = launch(&A, t, kModeTrigger, wl + 1, wl, m->iend, 128, st)) != cudaSuccess) return cuda_fail(e);
    if ((e = launch(&A, t, kModeList, wl + 1, wl, m->iend, 128, st)) != cudaSuccess) return cuda_fail(e);
    return UWSHCU_OK;
}

// Tape rows per warp of the adjoint model (32 records of 24 B each) at full capacity: a warp of
// convecting 30-level columns takes ~1.3e5 rows, of 51-level columns about twice that.
constexpr int kAdjRows32 = 1 << 18, kAdjRows64 = 1 << 19;

// The adjoint call; with `defect` (device, mix) each batch runs the reverse sweep three times on its
// tape: the two parts of a split of the cotangents (their gradients kept in the buffer), then the
// cotangents themselves, whose sweep writes the gradients and the defect of linearity per column.
static int adjoint_run(const uwshcu_member* m, const uwshcu_adjoint* a, double* defect, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (!m || !a) return UWSHCU_ERR_BAD_ARGS;
    const int ncnst = s.k.ncnst;
    if (s.precision != UWSHCU_PREC_FP64 || ncnst > 5 || m->mkx + 1 > 64) return UWSHCU_ERR_BAD_ARGS;
    if (!member_ok(*m, ncnst)) return UWSHCU_ERR_BAD_ARGS;
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    StreamCtx* sc = nullptr;
    if ((rc = stream_ctx(*d, (cudaStream_t)stream, &sc)) != UWSHCU_OK) return rc;
    const UwArgs A = member_args(*m, ncnst, sc->err);
    const size_t mix = (size_t)m->mix, mkx = (size_t)m->mkx;
    // the unit for the level count: KP = 32 or 64 levels
    const bool k32 = m->mkx + 1 <= 32;
    auto adj_launch = k32 ? uw_adj_launch_k32n5 : uw_adj_launch_k64n5;
    const int full_rows = k32 ? kAdjRows32 : kAdjRows64, kp = k32 ? 32 : 64;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    // gradients start at zero: the columns that leave the scheme in the trigger pass keep it
    const std::pair<double*, size_t> grads[] = {{a->t0, mix * mkx}, {a->qv0, mix * mkx}, {a->tke, mix * (mkx + 1)},
                                                {a->pblh, mix}, {a->rpen, mix}, {a->rle, mix}, {a->rkm, mix},
                                                {a->criqc, mix}};
    for (const auto& g : grads)
        if (g.first && (e = cudaMemsetAsync(g.first, 0, g.second * sizeof(double), st)) != cudaSuccess) return cuda_fail(e);
    if (defect && (e = cudaMemsetAsync(defect, 0, mix * sizeof(double), st)) != cudaSuccess) return cuda_fail(e);
    if (m->iend == 0) return UWSHCU_OK;
    // trigger pass of the FP64 path: the exit columns' outputs and the worklist of the others
    if ((rc = grow_ints(sc->wl, sc->wl_cap, (size_t)m->iend + 1)) != UWSHCU_OK) return rc;
    if ((e = cudaMemsetAsync(sc->wl, 0, sizeof(int), st)) != cudaSuccess) return cuda_fail(e);
    if ((e = launch_mode(&A, UWSHCU_PREC_FP64, kModeTrigger, sc->wl + 1, sc->wl, m->iend, 128, st)) != cudaSuccess)
        return cuda_fail(e);
    int ncand = 0;
    if ((e = cudaMemcpyAsync(&ncand, sc->wl, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e);
    s.adj_records = 0;
    if (ncand == 0) return UWSHCU_OK;
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    // The candidates' order in the warps: by the FP64 path's implicit-CIN branch and updraft depth
    // (adj_key_kernel), so that the lanes of a warp climb about as far and the warp's tape holds
    // fewer rows; ties in ascending column order.  The FP64 worklist pass gives the level indices,
    // on a copy of cush (which the taped forward sweep reads as the trigger pass left it).
    size_t pair_bytes = 0;
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, pair_bytes, (const int*)nullptr, (int*)nullptr,
                                             (const int*)nullptr, (int*)nullptr, ncand, 0, 7, st)) != cudaSuccess)
        return cuda_fail(e);
    const size_t x_diag = 0, x_cush = x_diag + up(8 * mix * sizeof(int)), x_key = x_cush + up((size_t)m->iend * sizeof(double));
    const size_t x_keyo = x_key + up((size_t)ncand * sizeof(int)), x_wlo = x_keyo + up((size_t)ncand * sizeof(int));
    const size_t x_tmp = x_wlo + up((size_t)ncand * sizeof(int)), x_bytes = x_tmp + up(pair_bytes);
    if (x_bytes > d->adj_aux_bytes) {
        if (d->adj_aux) cudaFree(d->adj_aux);
        d->adj_aux = nullptr;
        d->adj_aux_bytes = 0;
        if ((e = cudaMalloc(&d->adj_aux, x_bytes + x_bytes / 8)) != cudaSuccess) return cuda_fail(e);
        d->adj_aux_bytes = x_bytes + x_bytes / 8;
    }
    char* const xb = static_cast<char*>(d->adj_aux);
    int* const x_diag_p = reinterpret_cast<int*>(xb + x_diag);
    double* const x_cush_p = reinterpret_cast<double*>(xb + x_cush);
    {
        UwArgs A2 = A;
        A2.diag_int = x_diag_p;
        A2.diag_real = nullptr;
        A2.diag_level = nullptr;
        if ((e = cudaMemcpyAsync(x_cush_p, m->cush, (size_t)m->iend * sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess ||
            (e = launch_mode(&A2, UWSHCU_PREC_FP64, kModeList, sc->wl + 1, sc->wl, m->iend, 128, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(m->cush, x_cush_p, (size_t)m->iend * sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
            return cuda_fail(e);
    }
    // Batches of warps (32 slots each) whose tapes fit 85 % of the device memory that is free or
    // already held by the adjoint buffer.  The tape capacity is sized from the previous call's largest
    // tape (+1/16); a batch that overflows it makes the call start again at the full capacity.  A
    // batch costs about one warp's forward sweep whatever its size (the sweep is a latency chain per
    // warp), so the sizing aims at one batch for all candidates, or at batches of as many warps as
    // the GPU holds at once.
    const size_t nin = 3 * mkx + 6, rowb = uw_adj_row_bytes_k32n5();
    const size_t nids = (size_t)(25 + 5) * kp;   // output-index table entries per slot (NC = 5)
    const size_t nw_need = ((size_t)ncand + 31) / 32;
    // the candidates in ascending column order, then stably by the ordering key: the warps' columns,
    // and with them the tapes and the order of every reduction, do not depend on the order the
    // trigger pass appended them in
    int end_bit = 1;
    while (end_bit < 31 && ((size_t)1 << end_bit) < (size_t)m->iend) end_bit++;
    size_t sort_bytes = 0;
    if ((e = cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, sc->wl + 1, sc->wl + 1, ncand, 0, end_bit, st)) !=
        cudaSuccess)
        return cuda_fail(e);
    bool restart = false;
    double* cush_saved = nullptr;
    for (size_t rcap = s.adj_rows > 0 ? std::min((size_t)s.adj_rows, (size_t)full_rows) : (size_t)full_rows;;
         restart = true) {
        const size_t astride = (nin + rcap) * 32;
        const size_t nsave = defect ? 2 * nin : 0;   // the split sweeps' gradients, per slot
        const size_t per_warp = rcap * rowb + astride * sizeof(double) + 32 * nids * sizeof(int) + 2 * sizeof(int) +
                                32 * nsave * sizeof(double) + 1024;
        size_t freeb = 0, totalb = 0;
        if ((e = cudaMemGetInfo(&freeb, &totalb)) != cudaSuccess) return cuda_fail(e);
        const size_t avail = (freeb + d->adj_bytes) / 20 * 17;
        // at most the warps the GPU holds at once: a warp of a batch that waits for a place would
        // start its chain when the first ones end, and the batch would last two chains
        int per_sm = 0, nsm = 0, dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
            (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
            (e = (k32 ? uw_adj_forward_occupancy_k32n5 : uw_adj_forward_occupancy_k64n5)(&per_sm)) != cudaSuccess)
            return cuda_fail(e);
        const size_t resident = std::max<size_t>(1, (size_t)nsm * (size_t)per_sm);
        const size_t nw = std::min(std::min(nw_need, resident), std::max((size_t)1, avail / per_warp)), nb = 32 * nw;
        // carve the buffer: tapes (operand indices, partials), adjoints, tables, counters, status
        const size_t o_ab = 0, o_d = o_ab + up(nw * rcap * 32 * 8), o_adj = o_d + up(nw * rcap * 32 * 16);
        const size_t o_ids = o_adj + up(nw * astride * sizeof(double)), o_nrow = o_ids + up(nb * nids * sizeof(int));
        const size_t o_st = o_nrow + up(2 * nw * sizeof(int)), o_wl = o_st + 256, o_tmp = o_wl + up(ncand * sizeof(int));
        const size_t o_cush = o_tmp + up(sort_bytes), o_gs = o_cush + up((size_t)m->iend * sizeof(double));
        const size_t bytes = o_gs + up(nb * nsave * sizeof(double));
        // cush is read and written by the forward sweep: a call that starts again puts back the values
        // the trigger pass left (saved in the buffer before it may be replaced), then saves them anew
        if (restart && (e = cudaMemcpyAsync(m->cush, cush_saved, (size_t)m->iend * sizeof(double),
                                            cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
            return cuda_fail(e);
        if (bytes > d->adj_bytes) {   // grown with 1/32 to spare, so that calls of similar size reuse it
            const size_t held = freeb + d->adj_bytes;
            if (d->adj_buf) cudaFree(d->adj_buf);
            d->adj_buf = nullptr;
            d->adj_bytes = 0;
            const size_t want = std::min(bytes + bytes / 32, std::max(bytes, held / 20 * 18));
            if ((e = cudaMalloc(&d->adj_buf, want)) != cudaSuccess) return cuda_fail(e);
            d->adj_bytes = want;
        }
        char* base = static_cast<char*>(d->adj_buf);
        cush_saved = reinterpret_cast<double*>(base + o_cush);
        if ((e = cudaMemcpyAsync(cush_saved, m->cush, (size_t)m->iend * sizeof(double), cudaMemcpyDeviceToDevice, st)) !=
            cudaSuccess)
            return cuda_fail(e);
        int* nrow = reinterpret_cast<int*>(base + o_nrow);
        unsigned int* status = reinterpret_cast<unsigned int*>(base + o_st);
        int* wl = reinterpret_cast<int*>(base + o_wl);
        size_t tmp_bytes = sort_bytes;
        if ((e = cudaMemsetAsync(status, 0, sizeof(unsigned int), st)) != cudaSuccess ||
            (e = cub::DeviceRadixSort::SortKeys(base + o_tmp, tmp_bytes, sc->wl + 1, wl, ncand, 0, end_bit, st)) !=
                cudaSuccess)
            return cuda_fail(e);
        {
            int* const key = reinterpret_cast<int*>(xb + x_key);
            int* const wl_o = reinterpret_cast<int*>(xb + x_wlo);
            size_t pb = pair_bytes;
            adj_key_kernel<<<(unsigned)((ncand + 255) / 256), 256, 0, st>>>(wl, ncand, x_diag_p, m->mix, key);
            if ((e = cudaGetLastError()) != cudaSuccess ||
                (e = cub::DeviceRadixSort::SortPairs(xb + x_tmp, pb, key, reinterpret_cast<int*>(xb + x_keyo), wl, wl_o,
                                                     ncand, 0, 7, st)) != cudaSuccess ||
                (e = cudaMemcpyAsync(wl, wl_o, (size_t)ncand * sizeof(int), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
                return cuda_fail(e);
        }
        std::vector<int> counts(nw);
        int most = 0;
        unsigned int bits = 0;
        for (size_t b0 = 0; b0 < (size_t)ncand && !bits; b0 += nb) {
            UwAdjHost h{};
            h.wl = wl;
            h.b0 = (int)b0;
            h.nb = (int)std::min(nb, (size_t)ncand - b0);
            h.ab = base + o_ab;
            h.d = base + o_d;
            h.rcap = (int)rcap;
            h.ids = reinterpret_cast<int*>(base + o_ids);
            h.cap = (int)nb;
            h.nrow = nrow;
            h.ovf = nrow + nw;
            h.adj = reinterpret_cast<double*>(base + o_adj);
            h.astride = astride;
            h.status = status;
            h.gsave = reinterpret_cast<double*>(base + o_gs);
            h.defect = defect;
            const size_t used = ((size_t)h.nb + 31) / 32;   // warps holding a slot
            if ((e = cudaMemsetAsync(h.ids, 0xff, nb * nids * sizeof(int), st)) != cudaSuccess ||
                (e = adj_launch(&A, &h, a, 0, st)) != cudaSuccess)
                return cuda_fail(e);
            for (int split = defect ? 1 : 0;; split = (split + 1) % 3) {   // 1, 2, 0 or 0
                h.split = split;
                adj_zero_kernel<<<(unsigned)used, 512, 0, st>>>(h.adj, astride, nrow, (int)nin, (int)rcap);
                if ((e = cudaGetLastError()) != cudaSuccess || (e = adj_launch(&A, &h, a, 1, st)) != cudaSuccess)
                    return cuda_fail(e);
                if (split == 0) break;
            }
            if ((e = cudaMemcpyAsync(counts.data(), nrow, used * sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaMemcpyAsync(&bits, status, sizeof(unsigned int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaStreamSynchronize(st)) != cudaSuccess)
                return cuda_fail(e);
            for (size_t j = 0; j < used; j++) most = std::max(most, counts[j]);
        }
        s.adj_records = most;
        if (bits && rcap < (size_t)full_rows) {   // the sized capacity was too small: again at the full one
            rcap = full_rows;
            continue;
        }
        s.adj_rows = (int)std::min((size_t)full_rows, ((size_t)most + most / 16 + 4095) / 4096 * 4096);
        if (bits) {
            s.adj_rows = 0;
            std::snprintf(s.lasterr, sizeof(s.lasterr),
                          "uwshcu_adjoint_device: a warp's tape exceeds %d rows (largest %d)", full_rows, most);
            return UWSHCU_ERR_TOO_LARGE;
        }
        return UWSHCU_OK;
    }
}

int uwshcu_adjoint_device(const uwshcu_member* m, const uwshcu_adjoint* a, void* stream)
{
    return adjoint_run(m, a, nullptr, stream);
}

int uwshcu_adjoint_device_checked(const uwshcu_member* m, const uwshcu_adjoint* a, double* defect, void* stream)
{
    if (!defect) return UWSHCU_ERR_BAD_ARGS;
    return adjoint_run(m, a, defect, stream);
}

int uwshcu_set_adjoint_rows(int rows)
{
    if (rows < 0 || rows > kAdjRows64) return UWSHCU_ERR_BAD_ARGS;
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    s.adj_rows = rows;
    return UWSHCU_OK;
}

int uwshcu_adjoint_release(void)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int dv = 0; dv < kMaxDev; dv++) {
        DeviceState& d = s.dev[dv];
        if (!d.adj_buf && !d.adj_aux) continue;
        cudaSetDevice(dv);
        for (void** p : {&d.adj_buf, &d.adj_aux}) {
            if (!*p) continue;
            const cudaError_t f = cudaFree(*p);
            if (f != cudaSuccess) e = f;
            *p = nullptr;
        }
        d.adj_bytes = 0;
        d.adj_aux_bytes = 0;
    }
    if (have) cudaSetDevice(cur);
    return e == cudaSuccess ? UWSHCU_OK : cuda_fail(e);
}

int uwshcu_adjoint_last_records(void) { return S().adj_records; }

int uwshcu_eval_math(int fn, const double* x, const double* y, double* out, int n, void* stream)
{
    if (fn < 0 || fn > 3 || n < 0 || (n > 0 && (!x || !out || (fn == 2 && !y)))) return UWSHCU_ERR_BAD_ARGS;
    if (n == 0) return UWSHCU_OK;
    eval_math_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(fn, x, fn == 2 ? y : x, out, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> lock(S().mu);
        return cuda_fail(e);
    }
    return UWSHCU_OK;
}

int uwshcu_device_status(void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    cudaError_t e;
    unsigned int bits = 0;
    if ((e = cudaStreamSynchronize((cudaStream_t)stream)) != cudaSuccess) return cuda_fail(e);
    StreamCtx* c = nullptr;
    for (StreamCtx& x : d->sctx)
        if (x.used && x.stream == (cudaStream_t)stream) c = &x;
    if (!c) return UWSHCU_OK;   // no device-array call on this stream since the last status
    if ((e = cudaMemcpy(&bits, c->err, sizeof(bits), cudaMemcpyDeviceToHost)) != cudaSuccess) return cuda_fail(e);
    if ((e = cudaMemset(c->err, 0, sizeof(unsigned int))) != cudaSuccess) return cuda_fail(e);
    return status_from_bits(bits);
}

}  // extern "C"

// ---- uwshcu_compute_device_noalloc: the two-phase schedule with a fixed, library-owned worklist
//
// For callers that cannot allocate device memory at the point where they call the scheme: a host
// model whose memory manager claims the device's memory at start-up and hands out only its own
// pool (a cudaMalloc of ours would fail or fragment that pool), and codes that must not call
// cudaMalloc/cudaFree inside a time step because those calls can synchronize the device.  The
// worklist of convecting columns (count, endrun bits, column ids), which uwshcu_compute_device
// grows with cudaMalloc, lives here in one file-scope device array sized for
// UWSHCU_NOALLOC_MAX_COLUMNS columns (4 MiB + 256 B).  Every GPU that loads the library holds the
// array until the process exits.  In host code g_noalloc_scratch is only a host-side stand-in for
// the symbol; its device address comes from cudaGetSymbolAddress, once per device, with that
// device current.
constexpr int kNoallocHeader = 64;   // ints before the column ids: [0] count, [1] endrun bits
static __device__ __align__(256) int g_noalloc_scratch[kNoallocHeader + UWSHCU_NOALLOC_MAX_COLUMNS];

namespace {

struct NoallocDevice {
    int* scratch = nullptr;          // device address of g_noalloc_scratch on this device
};
NoallocDevice g_noalloc_dev[kMaxDev];

// Set-up of the current device without allocating: the scratch's device address, and the
// constants (cudaMemcpyToSymbol into the kernels' __constant__ banks) when they are missing or
// older than the last uwshcu_init / uwshcu_set_rpen.
int noalloc_device(int** scratch)
{
    State& s = S();
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) {
        std::snprintf(s.lasterr, sizeof(s.lasterr), "%s", e != cudaSuccess ? cudaGetErrorString(e) : "no device");
        return UWSHCU_ERR_NO_DEVICE;
    }
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e);
    if (dev < 0 || dev >= kMaxDev) return UWSHCU_ERR_NO_DEVICE;
    NoallocDevice& nd = g_noalloc_dev[dev];
    if (!nd.scratch) {
        void* ptr = nullptr;
        if ((e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch)) != cudaSuccess) return cuda_fail(e);
        nd.scratch = static_cast<int*>(ptr);
    }
    DeviceState& d = s.dev[dev];
    if (d.uploaded_gen != s.gen) {
        if ((e = set_constants_all(&s.k, s.tbl)) != cudaSuccess) return cuda_fail(e);
        d.uploaded_gen = s.gen;
    }
    *scratch = nd.scratch;
    return UWSHCU_OK;
}

}  // namespace

extern "C" int uwshcu_compute_device_noalloc(
    int mix, int mkx, int iend, int ncnst, double dt, int inv, const double* ps0, const double* zs0,
    const double* p0, const double* z0, const double* dp0, const double* u0, const double* v0,
    const double* qv0, const double* ql0, const double* qi0, const double* t0, const double* s0,
    const double* tr0, const double* tke, const double* pblh, double* cush, double* umf, double* slflx,
    double* qtflx, double* flxprc1, double* flxsnow1, double* qvten, double* qlten, double* qiten,
    double* sten, double* uten, double* vten, double* trten, double* qrten, double* qsten,
    double* precip, double* snow, double* evapc, double* cufrc, double* qcu, double* qlu, double* qiu,
    double* cbmf, double* qc, double* rliq, double* cnt, double* cnb, const double* dpdry0, double* wu,
    int* diag_int, double* diag_real, unsigned int* status_bits, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (bad_dims(mix, mkx, iend, ncnst) || (inv != 0 && inv != 1)) return UWSHCU_ERR_BAD_ARGS;
    if (iend > UWSHCU_NOALLOC_MAX_COLUMNS) {
        std::snprintf(s.lasterr, sizeof(s.lasterr),
                      "uwshcu_compute_device_noalloc: iend = %d exceeds its fixed worklist of %d columns "
                      "(UWSHCU_NOALLOC_MAX_COLUMNS); split the call or use uwshcu_compute_device",
                      iend, UWSHCU_NOALLOC_MAX_COLUMNS);
        return UWSHCU_ERR_TOO_LARGE;
    }
    const void* need[] = {ps0, zs0, p0, z0, dp0, u0, v0, qv0, ql0, qi0, t0, s0, tr0, tke, pblh, cush,
                          umf, slflx, qtflx, flxprc1, flxsnow1, qvten, qlten, qiten, sten, uten, vten,
                          trten, qrten, qsten, precip, snow, evapc, cufrc, qcu, qlu, qiu, cbmf, qc, rliq,
                          cnt, cnb, dpdry0, wu};
    for (const void* p : need)
        if (!p) return UWSHCU_ERR_BAD_ARGS;
    int* scratch = nullptr;
    int rc = noalloc_device(&scratch);
    if (rc != UWSHCU_OK) return rc;
    UwArgs A{};
    A.mix = mix; A.mkx = mkx; A.iend = iend; A.ncnst = ncnst; A.inv = inv; A.dt = dt;
    A.ps0 = ps0; A.zs0 = zs0; A.p0 = p0; A.z0 = z0; A.dp0 = dp0; A.u0 = u0; A.v0 = v0; A.qv0 = qv0;
    A.ql0 = ql0; A.qi0 = qi0; A.t0 = t0; A.s0 = s0; A.tr0 = tr0; A.tke = tke; A.pblh = pblh; A.cush = cush;
    A.umf = umf; A.slflx = slflx; A.qtflx = qtflx; A.flxprc1 = flxprc1; A.flxsnow1 = flxsnow1;
    A.qvten = qvten; A.qlten = qlten; A.qiten = qiten; A.sten = sten; A.uten = uten; A.vten = vten;
    A.trten = trten; A.qrten = qrten; A.qsten = qsten; A.precip = precip; A.snow = snow; A.evapc = evapc;
    A.cufrc = cufrc; A.qcu = qcu; A.qlu = qlu; A.qiu = qiu; A.cbmf = cbmf; A.qc = qc; A.rliq = rliq;
    A.cnt = cnt; A.cnb = cnb; A.dpdry0 = dpdry0; A.wu = wu; A.diag_int = diag_int; A.diag_real = diag_real;
    int* count = scratch;
    int* list = scratch + kNoallocHeader;
    A.err = status_bits ? status_bits : reinterpret_cast<unsigned int*>(scratch + 1);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    // the array keeps the previous call's contents: the count and the endrun bits start at zero
    if ((e = cudaMemsetAsync(scratch, 0, 2 * sizeof(int), st)) != cudaSuccess) return cuda_fail(e);
    if (status_bits && (e = cudaMemsetAsync(status_bits, 0, sizeof(unsigned int), st)) != cudaSuccess)
        return cuda_fail(e);
    if ((e = launch_mode(&A, s.precision, kModeTrigger, list, count, iend, s.block, st)) != cudaSuccess)
        return cuda_fail(e);
    if ((e = launch_mode(&A, s.precision, kModeList, list, count, iend, s.block, st)) != cudaSuccess)
        return cuda_fail(e);
    return UWSHCU_OK;
}

// ---- batched uneven launches: plans ----------------------------------------------------------------
#define UW_DECL_BATCH(KP, NC)                                                                         \
    extern "C" cudaError_t uw_fp64_batch_k##KP##n##NC(const UwBatch* b, int phase, int grid, int block, \
                                                      int minb, cudaStream_t stream);                 \
    extern "C" cudaError_t uw_fp64_batch_occupancy_k##KP##n##NC(int minb, int block, int* blocks_per_sm);
UW_DECL_BATCH(32, 5)
UW_DECL_BATCH(64, 5)
UW_DECL_BATCH(32, 32)
UW_DECL_BATCH(64, 32)
#undef UW_DECL_BATCH
#define UW_DECL_BATCH_P(P, KP, NC)                                                                     \
    extern "C" cudaError_t uw_##P##_batch_k##KP##n##NC(const UwBatch* b, int phase, int grid, int block, \
                                                       int minb, cudaStream_t stream);                 \
    extern "C" cudaError_t uw_##P##_batch_occupancy_k##KP##n##NC(int minb, int block, int* blocks_per_sm);
UW_DECL_BATCH_P(fast, 32, 5)
UW_DECL_BATCH_P(fast, 64, 5)
UW_DECL_BATCH_P(fast, 32, 32)
UW_DECL_BATCH_P(fast, 64, 32)
UW_DECL_BATCH_P(mixed, 32, 5)
UW_DECL_BATCH_P(mixed, 64, 5)
#undef UW_DECL_BATCH_P

namespace {

// Level/tracer classes of the compiled instantiations: bit 0 = 64-level bound, bit 1 = 32 tracers.
constexpr int kClasses = 4;
typedef cudaError_t (*BatchFn)(const UwBatch*, int, int, int, int, cudaStream_t);
typedef cudaError_t (*BatchOccFn)(int, int, int*);
// the batch launch hooks of a precision mode and class (null: not compiled)
BatchFn batch_fn(int prec, int cls)
{
    static const BatchFn fp64[kClasses] = {uw_fp64_batch_k32n5, uw_fp64_batch_k64n5, uw_fp64_batch_k32n32,
                                           uw_fp64_batch_k64n32};
    static const BatchFn fast[kClasses] = {uw_fast_batch_k32n5, uw_fast_batch_k64n5, uw_fast_batch_k32n32,
                                           uw_fast_batch_k64n32};
    static const BatchFn mixed[kClasses] = {uw_mixed_batch_k32n5, uw_mixed_batch_k64n5, nullptr, nullptr};
    return prec == UWSHCU_PREC_FAST ? fast[cls] : prec == UWSHCU_PREC_MIXED ? mixed[cls] : fp64[cls];
}
BatchOccFn batch_occ_fn(int prec, int cls)
{
    static const BatchOccFn fp64[kClasses] = {uw_fp64_batch_occupancy_k32n5, uw_fp64_batch_occupancy_k64n5,
                                              uw_fp64_batch_occupancy_k32n32, uw_fp64_batch_occupancy_k64n32};
    static const BatchOccFn fast[kClasses] = {uw_fast_batch_occupancy_k32n5, uw_fast_batch_occupancy_k64n5,
                                              uw_fast_batch_occupancy_k32n32, uw_fast_batch_occupancy_k64n32};
    static const BatchOccFn mixed[kClasses] = {uw_mixed_batch_occupancy_k32n5, uw_mixed_batch_occupancy_k64n5,
                                               nullptr, nullptr};
    return prec == UWSHCU_PREC_FAST ? fast[cls] : prec == UWSHCU_PREC_MIXED ? mixed[cls] : fp64[cls];
}
cudaError_t batch_launch(int prec, int cls, const UwBatch* b, int phase, int grid, int block, int minb, cudaStream_t st)
{
    BatchFn f = batch_fn(prec, cls);
    return f ? f(b, phase, grid, block, minb, st) : cudaErrorInvalidValue;
}
cudaError_t batch_occupancy(int prec, int cls, int minb, int block, int* per_sm)
{
    BatchOccFn f = batch_occ_fn(prec, cls);
    if (!f) {
        *per_sm = 0;
        return cudaErrorInvalidValue;
    }
    return f(minb, block, per_sm);
}
// register caps compiled per precision and class: FP64 with 5 tracers carries 168/128/80 registers,
// the others only the 128-register one
bool batch_has_minb(int prec, int cls, int minb)
{
    if (prec == UWSHCU_PREC_FP64 && cls < 2) return minb == 3 || minb == 4 || minb == 6;
    return minb == 4;
}

struct BatchPlan {
    int dev = 0;
    int prec = UWSHCU_PREC_FP64;  // precision mode at creation
    int nm = 0;
    uwshcu_member mem[UWSHCU_MAX_MEMBERS];
    int ncls = 0;
    int cls_id[kClasses];          // class of each used slot
    UwBatch b[kClasses];           // per used class
    int trig_grid[kClasses];
    int* d_scratch = nullptr;      // [0, 64): counts of all members, [64, 64 + kClasses): task heads,
                                   // [64 + kClasses, 64 + 2 kClasses): resume task heads, worklists
    bool sorted = false;           // created under the sorted schedule, with a region per member
    char* hand[UWSHCU_MAX_MEMBERS] = {};
    unsigned int* d_err = nullptr;
    double* d_cush_save = nullptr; // autotune only
    int block = 128, minb = 4, chunk = 1;
    int nsm = 1;
    cudaGraphExec_t exec = nullptr;
};

int plan_enqueue(BatchPlan& P, cudaStream_t st)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(P.d_scratch, 0, (64 + 2 * kClasses) * sizeof(int), st)) != cudaSuccess) return cuda_fail(e);
    for (int j = 0; j < P.nm && P.sorted; j++)
        if ((e = cudaMemsetAsync(P.hand[j] + kHandCountOffset, 0, (1 + UW_HAND_KEYS) * sizeof(int), st)) != cudaSuccess)
            return cuda_fail(e);
    for (int c = 0; c < P.ncls; c++) {
        P.b[c].chunk = P.chunk;
        if ((e = batch_launch(P.prec, P.cls_id[c], &P.b[c], 0, P.trig_grid[c], P.block, 0, st)) != cudaSuccess)
            return cuda_fail(e);
    }
    if (P.sorted) {
        // first worklist launch per class, the sort of each member's hand-off slots, resume launch
        for (int c = 0; c < P.ncls; c++) {
            int per_sm = 0;
            if ((e = batch_occupancy(P.prec, P.cls_id[c], 4, P.block, &per_sm)) != cudaSuccess) return cuda_fail(e);
            if (per_sm <= 0) return UWSHCU_ERR_BAD_ARGS;
            if ((e = batch_launch(P.prec, P.cls_id[c], &P.b[c], 2, P.nsm * per_sm, P.block, 4, st)) != cudaSuccess)
                return cuda_fail(e);
        }
        for (int j = 0; j < P.nm; j++) {
            const UwHand* H = reinterpret_cast<const UwHand*>(P.hand[j]);
            const int nb = (int)std::min(((size_t)P.mem[j].iend + 255) / 256, (size_t)1184);
            hand_hist_kernel<<<nb, 256, 0, st>>>(H);
            hand_scan_kernel<<<1, 32, 0, st>>>(H);
            hand_scatter_kernel<<<nb, 256, 0, st>>>(H);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e);
        for (int c = 0; c < P.ncls; c++)   // 5 resident blocks of 128 threads per SM (launch bounds)
            if ((e = batch_launch(P.prec, P.cls_id[c], &P.b[c], 3, P.nsm * 5 * (128 / P.block), P.block, 0, st)) != cudaSuccess)
                return cuda_fail(e);
        return UWSHCU_OK;
    }
    for (int c = 0; c < P.ncls; c++) {
        int per_sm = 0;
        if ((e = batch_occupancy(P.prec, P.cls_id[c], P.minb, P.block, &per_sm)) != cudaSuccess) return cuda_fail(e);
        if (per_sm <= 0) return UWSHCU_ERR_BAD_ARGS;
        if ((e = batch_launch(P.prec, P.cls_id[c], &P.b[c], 1, P.nsm * per_sm, P.block, P.minb, st)) != cudaSuccess)
            return cuda_fail(e);
    }
    return UWSHCU_OK;
}

void plan_free(BatchPlan* P)
{
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->d_scratch) cudaFree(P->d_scratch);
    if (P->d_err) cudaFree(P->d_err);
    if (P->d_cush_save) cudaFree(P->d_cush_save);
    for (char* h : P->hand)
        if (h) cudaFree(h);
    delete P;
}

}  // namespace

extern "C" int uwshcu_batch_create(int nmembers, const uwshcu_member* members, void** plan)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!plan) return UWSHCU_ERR_BAD_ARGS;
    *plan = nullptr;
    if (!s.init) return UWSHCU_ERR_NOT_INITIALIZED;
    if (nmembers < 1 || nmembers > UWSHCU_MAX_MEMBERS || !members) return UWSHCU_ERR_BAD_ARGS;
    // the plan keeps the precision mode in force now (FP64, FAST, or MIXED with ncnst <= 5)
    const int ncnst = s.k.ncnst;
    size_t total = 0;
    for (int j = 0; j < nmembers; j++) {
        const uwshcu_member& m = members[j];
        if (!member_ok(m, ncnst)) return UWSHCU_ERR_BAD_ARGS;
        total += (size_t)m.iend;
    }
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    BatchPlan* P = new BatchPlan();
    P->nm = nmembers;
    P->prec = s.precision;
    cudaError_t e;
    if ((e = cudaGetDevice(&P->dev)) != cudaSuccess || (e = cudaDeviceGetAttribute(&P->nsm, cudaDevAttrMultiProcessorCount, P->dev)) != cudaSuccess) {
        plan_free(P);
        return cuda_fail(e);
    }
    if ((e = cudaMalloc(&P->d_scratch, (64 + 2 * kClasses + total) * sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&P->d_err, sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaMemset(P->d_err, 0, sizeof(unsigned int))) != cudaSuccess) {
        plan_free(P);
        return cuda_fail(e);
    }
    int cls_slot[kClasses] = {-1, -1, -1, -1};
    size_t wl_off = 64 + 2 * kClasses;
    // sorted schedule: a hand-off region per member (a plan without room for them runs two-phase)
    P->sorted = s.schedule == UWSHCU_SCHED_SORTED;
    for (int j = 0; j < nmembers && P->sorted; j++) {
        const size_t words = uw_state_words(members[j].mkx, ncnst);
        P->hand[j] = hand_alloc(hand_slots_for(members[j].iend, words), words);
        if (!P->hand[j]) {
            for (char*& h : P->hand)
                if (h) {
                    cudaFree(h);
                    h = nullptr;
                }
            P->sorted = false;
        }
    }
    for (int j = 0; j < nmembers; j++) {
        const uwshcu_member& m = members[j];
        P->mem[j] = m;
        const int cls = (m.mkx + 1 <= 32 ? 0 : 1) + (ncnst <= 5 ? 0 : 2);
        if (cls_slot[cls] < 0) {
            cls_slot[cls] = P->ncls;
            P->cls_id[P->ncls] = cls;
            UwBatch& b = P->b[P->ncls];
            b = UwBatch{};
            b.task_head = P->d_scratch + 64 + P->ncls;
            b.task_head2 = P->d_scratch + 64 + kClasses + P->ncls;
            P->trig_grid[P->ncls] = 0;
            P->ncls++;
        }
        const int c = cls_slot[cls];
        UwBatch& b = P->b[c];
        const int slot = b.nm++;
        b.m[slot] = member_args(m, ncnst, P->d_err);
        b.m[slot].hand = reinterpret_cast<const UwHand*>(P->hand[j]);
        b.wl[slot] = P->d_scratch + wl_off;
        wl_off += (size_t)m.iend;
    }
    // per-class member counts sit in consecutive ints of the header; block ranges of the trigger
    int next_count = 0;
    for (int c = 0; c < P->ncls; c++) {
        UwBatch& b = P->b[c];
        b.count = P->d_scratch + next_count;
        next_count += b.nm;
        b.block_start[0] = 0;
        for (int j = 0; j < b.nm; j++)
            b.block_start[j + 1] = b.block_start[j] + (b.m[j].iend + P->block - 1) / P->block;
        P->trig_grid[c] = b.block_start[b.nm];
    }
    *plan = P;
    return UWSHCU_OK;
}

namespace {
// block ranges depend on the block size
void plan_set_block(BatchPlan& P, int block)
{
    P.block = block;
    for (int c = 0; c < P.ncls; c++) {
        UwBatch& b = P.b[c];
        b.block_start[0] = 0;
        for (int j = 0; j < b.nm; j++) b.block_start[j + 1] = b.block_start[j] + (b.m[j].iend + block - 1) / block;
        P.trig_grid[c] = b.block_start[b.nm];
    }
}
}  // namespace

extern "C" int uwshcu_batch_run(void* plan, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!plan) return UWSHCU_ERR_BAD_ARGS;
    BatchPlan& P = *static_cast<BatchPlan*>(plan);
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);   // constants current on this device
    if (rc != UWSHCU_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (P.exec) {
        cudaError_t e = cudaGraphLaunch(P.exec, st);
        return e == cudaSuccess ? UWSHCU_OK : cuda_fail(e);
    }
    return plan_enqueue(P, st);
}

extern "C" int uwshcu_batch_capture(void* plan, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!plan || !stream) return UWSHCU_ERR_BAD_ARGS;   // capture needs a non-default stream
    BatchPlan& P = *static_cast<BatchPlan*>(plan);
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (P.exec) {
        cudaGraphExecDestroy(P.exec);
        P.exec = nullptr;
    }
    cudaError_t e;
    if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return cuda_fail(e);
    rc = plan_enqueue(P, st);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(st, &g);
    if (rc != UWSHCU_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e);
    e = cudaGraphInstantiate(&P.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        P.exec = nullptr;
        return cuda_fail(e);
    }
    return UWSHCU_OK;
}

extern "C" int uwshcu_batch_autotune(void* plan, void* stream, int* block_out, int* minb_out, int* chunk_out)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!plan) return UWSHCU_ERR_BAD_ARGS;
    BatchPlan& P = *static_cast<BatchPlan*>(plan);
    DeviceState* d = nullptr;
    int rc = ensure_device(&d);
    if (rc != UWSHCU_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (P.exec) {
        cudaGraphExecDestroy(P.exec);
        P.exec = nullptr;
    }
    // keep cush (in/out) so that every trial sees the same inputs
    size_t ncush = 0;
    for (int j = 0; j < P.nm; j++) ncush += (size_t)P.mem[j].iend;
    if (!P.d_cush_save && (e = cudaMalloc(&P.d_cush_save, ncush * sizeof(double))) != cudaSuccess) return cuda_fail(e);
    auto save_restore = [&](bool save) -> cudaError_t {
        size_t off = 0;
        for (int j = 0; j < P.nm; j++) {
            const size_t nb = (size_t)P.mem[j].iend * sizeof(double);
            cudaError_t ee = save ? cudaMemcpyAsync(P.d_cush_save + off, P.mem[j].cush, nb, cudaMemcpyDeviceToDevice, st)
                                  : cudaMemcpyAsync(P.mem[j].cush, P.d_cush_save + off, nb, cudaMemcpyDeviceToDevice, st);
            if (ee != cudaSuccess) return ee;
            off += (size_t)P.mem[j].iend;
        }
        return cudaSuccess;
    };
    if ((e = save_restore(true)) != cudaSuccess) return cuda_fail(e);
    cudaEvent_t e0, e1;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) return cuda_fail(e);
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(e);
    }
    const int blocks[] = {128, 64};
    const int minbs[] = {3, 4, 6};
    const int chunks[] = {1, 2};
    float best = 1e30f;
    int bb = P.block, bm = P.minb, bc = P.chunk;
    rc = UWSHCU_OK;
    bool warm = false;
    for (int block : blocks) {
        for (int minb : minbs) {
            bool ok = true;
            for (int c = 0; c < P.ncls; c++) ok = ok && batch_has_minb(P.prec, P.cls_id[c], minb);
            if (!ok) continue;
            for (int chunk : chunks) {
                plan_set_block(P, block);
                P.minb = minb;
                P.chunk = chunk;
                float tmin = 1e30f;
                for (int rep = 0; rep < (warm ? 2 : 3); rep++) {
                    if ((e = save_restore(false)) != cudaSuccess) { rc = cuda_fail(e); break; }
                    if ((e = cudaEventRecord(e0, st)) != cudaSuccess) { rc = cuda_fail(e); break; }
                    if ((rc = plan_enqueue(P, st)) != UWSHCU_OK) break;
                    if ((e = cudaEventRecord(e1, st)) != cudaSuccess || (e = cudaEventSynchronize(e1)) != cudaSuccess) {
                        rc = cuda_fail(e);
                        break;
                    }
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (warm || rep > 0) tmin = std::min(tmin, ms);
                }
                warm = true;
                if (rc != UWSHCU_OK) break;
                if (tmin < best) {
                    best = tmin;
                    bb = block;
                    bm = minb;
                    bc = chunk;
                }
            }
            if (rc != UWSHCU_OK) break;
        }
        if (rc != UWSHCU_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    plan_set_block(P, bb);
    P.minb = bm;
    P.chunk = bc;
    cudaError_t er = save_restore(false);
    if (rc == UWSHCU_OK && er != cudaSuccess) rc = cuda_fail(er);
    if (rc == UWSHCU_OK && (er = cudaStreamSynchronize(st)) != cudaSuccess) rc = cuda_fail(er);
    // runs of the tuner report no endrun status
    cudaMemset(P.d_err, 0, sizeof(unsigned int));
    if (block_out) *block_out = bb;
    if (minb_out) *minb_out = bm;
    if (chunk_out) *chunk_out = bc;
    return rc;
}

extern "C" int uwshcu_batch_status(void* plan, void* stream)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!plan) return UWSHCU_ERR_BAD_ARGS;
    BatchPlan& P = *static_cast<BatchPlan*>(plan);
    cudaError_t e;
    unsigned int bits = 0;
    if ((e = cudaStreamSynchronize((cudaStream_t)stream)) != cudaSuccess) return cuda_fail(e);
    if ((e = cudaMemcpy(&bits, P.d_err, sizeof(bits), cudaMemcpyDeviceToHost)) != cudaSuccess) return cuda_fail(e);
    if ((e = cudaMemset(P.d_err, 0, sizeof(unsigned int))) != cudaSuccess) return cuda_fail(e);
    return status_from_bits(bits);
}

extern "C" int uwshcu_batch_destroy(void* plan)
{
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!plan) return UWSHCU_ERR_BAD_ARGS;
    plan_free(static_cast<BatchPlan*>(plan));
    return UWSHCU_OK;
}
