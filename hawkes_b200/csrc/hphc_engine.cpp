// Host side of the B200 Hawkes likelihood engine and its C ABI (include/hphc.h).
//
// hphc_engine mirrors the state of the reference engines
// (src/NewHawkes.hpp:186-897, src/backend/opencl/OpenCLHawkes.hpp:42-997):
// six parameters plus a stored copy, double-buffered locations for
// store/restore, times, and the last log-likelihood.  Locations and times are
// kept in pinned host mirrors; a change marks the device copy dirty and the
// next evaluation uploads it (and, in FP64 mode, rebuilds the packed records),
// so per-row updateLocations calls (src/benchmark.cpp:167-171) cost a host
// write each rather than a transfer each.
//
// After an evaluation of its own parameters the engine keeps every event's six
// unit pair sums on the device: a later evaluation at the same parameters
// after a few single-event moves updates them in O(N) per moved event
// (incremental path), and one with nothing changed re-runs only the O(N)
// finish.  storeState / restoreState save and bring back those sums.
//
// hphc_multiset holds several independent event sets (uneven sizes) for
// evaluating each at its own parameter vector in one run.
//
// Every sweep goes through hphc::Executor: one launch per stage for any
// number of (event set, parameter vector) problems, replayed from a CUDA graph.
#include <cuda_runtime.h>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "hphc.h"
#include "hphc_executor.h"
#include "hphc_internal.h"
#include "hphc_kernels.cuh"

using namespace hphc;

namespace {

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t count) {
        if (count <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) n = count;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

template <typename T>
struct HostBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t count) {
        if (count <= n && p) return cudaSuccess;
        T* q = nullptr;
        cudaError_t e = cudaMallocHost(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        if (p) {
            std::memcpy(q, p, n * sizeof(T));
            cudaFreeHost(p);
        }
        p = q;
        n = count;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
    void swap(HostBuf& o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
};

// Mean relative error of ex2.approx.ftz.f32 (the instruction rounds low on
// average), measured once per device over 2^20 arguments spread over [-16, 0)
// and cached.  FP32 modes divide it out of the terms that come from it.
constexpr int kMaxDevices = 64;
constexpr int kEx2Samples = 1 << 20;
std::mutex gEx2Mutex;
bool gEx2Done[kMaxDevices] = {};
double gEx2Bias[kMaxDevices] = {};

cudaError_t ex2_bias_for_device(int device, cudaStream_t stream, double* bias) {
    std::lock_guard<std::mutex> lock(gEx2Mutex);
    if (device >= 0 && device < kMaxDevices && gEx2Done[device]) {
        *bias = gEx2Bias[device];
        return cudaSuccess;
    }
    const int blocks = (kEx2Samples + kFinishThreads - 1) / kFinishThreads;
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, blocks * sizeof(double));
    if (e != cudaSuccess) return e;
    std::vector<double> h(blocks);
    e = launch_ex2_bias(kEx2Samples, d, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), d, blocks * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    if (e != cudaSuccess) return e;
    double s = 0.0;
    for (double v : h) s += v;
    *bias = s / kEx2Samples;
    if (device >= 0 && device < kMaxDevices) {
        gEx2Bias[device] = *bias;
        gEx2Done[device] = true;
    }
    return cudaSuccess;
}

// Engine-wide settings derived from the flags.
struct Mode {
    int precision = HPHC_PRECISION_FP64;
    int variant = 2;  // FP32 variant bits: 1 = coordinate lo parts, 2 = software exponential
    bool underflowSkip = true;
    bool symmetric = true;  // each background pair evaluated once for both events
    bool fastTail = true;   // far-tail background tile pairs on the hardware exponential
    bool truncateTail = true;  // background tile pairs below 2^-91 (FP32: 2^-60) of B_ii skipped
};

Mode mode_from_flags(long fl) {
    Mode m;
    // COMPENSATED (with or without FLOAT): FP32 pair terms with compensated
    // sums and FP64 reductions; FLOAT alone: FP32 throughout, the reference's
    // single precision (src/factory.cpp:34, :45).
    m.precision = (fl & HPHC_FLAG_COMPENSATED) ? HPHC_PRECISION_FP32_COMP
                  : (fl & HPHC_FLAG_FLOAT)     ? HPHC_PRECISION_FP32
                                               : HPHC_PRECISION_FP64;
    m.underflowSkip = !(fl & HPHC_FLAG_NO_UNDERFLOW_SKIP);
    m.variant = m.precision == HPHC_PRECISION_FP32
                    ? 8  // plain: hardware exponential, hi parts, plain sums
                    : ((fl & HPHC_FLAG_FP32_SPACE_HILO) ? 1 : 0) |
                          ((fl & HPHC_FLAG_FP32_FAST_EXP) ? 0 : 2);
    m.symmetric = !(fl & HPHC_FLAG_ORDERED);
    m.fastTail = !(fl & HPHC_FLAG_NO_FAST_TAIL);
    m.truncateTail = !(fl & HPHC_FLAG_NO_TAIL_TRUNCATION);
    return m;
}

// One event set on the device with its host mirrors: raw FP64 coordinates and
// times, dense time ranks (FP32 mode), packed FP64 records (FP64 mode) and
// per-tile time bounds on both sides.
struct EventSet {
    int D = 0, N = 0;
    HostBuf<double> hTimes;
    HostBuf<int32_t> hRanks;
    std::vector<double> hTileMin, hTileMax;
    bool sorted = false;
    bool floatTimes = false;  // plain FP32 mode: causality from the times rounded to FP32
    DevBuf<double> dLoc, dTimes, dRecF64, dTileMin, dTileMax;
    DevBuf<int32_t> dRanks;
    DevBuf<int> dTileChanges;  // FP32 mode, sorted times: ranks computed on the device
    DevBuf<int32_t> dOrder2, dOrder4;  // FP32 mode: spatial row order of R = 2 and 4 strips

    cudaError_t alloc(int dim, int n, int precision) {
        D = dim;
        N = n;
        floatTimes = precision == HPHC_PRECISION_FP32;
        const int nTiles = (N + kTile - 1) / kTile;
        cudaError_t e;
        if ((e = hTimes.reserve(N)) || (e = hRanks.reserve(N)) ||
            (e = dLoc.reserve((size_t)N * D)) || (e = dTimes.reserve(N)) ||
            (e = dTileMin.reserve(nTiles)) || (e = dTileMax.reserve(nTiles)))
            return e;
        if (precision == HPHC_PRECISION_FP64) {
            if ((e = dRecF64.reserve((size_t)N * 10))) return e;
        } else if ((e = dRanks.reserve(N)) || (e = dTileChanges.reserve(nTiles)) ||
                   (e = dOrder2.reserve(N)) || (e = dOrder4.reserve(N))) {
            return e;
        }
        std::memset(hTimes.p, 0, (size_t)N * sizeof(double));
        std::memset(hRanks.p, 0, (size_t)N * sizeof(int32_t));
        hTileMin.assign(nTiles, 0.0);
        hTileMax.assign(nTiles, 0.0);
        sorted = true;
        return cudaSuccess;
    }

    void release() {
        hTimes.release();
        hRanks.release();
        dLoc.release();
        dTimes.release();
        dRecF64.release();
        dTileMin.release();
        dTileMax.release();
        dRanks.release();
        dTileChanges.release();
        dOrder2.release();
        dOrder4.release();
    }

    // Host-side derived data of the times: sortedness, dense ranks (equal
    // times share a rank: the exact strict-causality mask of the FP32
    // records), per-tile bounds.  Sorted times (the usual case) take one pass
    // for sortedness and ranks, and the tile bounds are each tile's first and
    // last time.
    // Sortedness and per-tile time bounds on the host.  The dense time ranks
    // of sorted times are computed on the device at upload; unsorted times
    // get them here (hRanks).
    void derive_times(int knownSorted = -1) {
        const double* t = hTimes.p;
        bool asc = knownSorted > 0;
        if (knownSorted < 0)
            for (int i = 1; i < N; ++i) asc &= t[i - 1] <= t[i];
        sorted = asc;
        const int nTiles = (N + kTile - 1) / kTile;
        if (sorted) {
            for (int k = 0; k < nTiles; ++k) {
                hTileMin[k] = t[k * kTile];
                hTileMax[k] = t[std::min(N, (k + 1) * kTile) - 1];
            }
            return;
        }
        std::vector<int> idx(N);
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return t[x] < t[y]; });
        int r = 0;
        for (int k = 0; k < N; ++k) {
            const bool differs = floatTimes ? (float)t[idx[k]] != (float)t[idx[k - (k > 0)]]
                                            : t[idx[k]] != t[idx[k - (k > 0)]];
            if (k > 0 && differs) ++r;
            hRanks.p[idx[k]] = r;
        }
        for (int k = 0; k < nTiles; ++k) {
            double lo = INFINITY, hi = -INFINITY;
            for (int j = k * kTile; j < std::min(N, (k + 1) * kTile); ++j) {
                lo = std::min(lo, t[j]);
                hi = std::max(hi, t[j]);
            }
            hTileMin[k] = lo;
            hTileMax[k] = hi;
        }
    }

    // Upload a location block (host, row-major) and the times; rebuild the
    // device-side derived data.
    cudaError_t upload(const double* hLoc, int precision, cudaStream_t s, int* launches) {
        cudaError_t e;
        if ((e = cudaMemcpyAsync(dLoc.p, hLoc, (size_t)N * D * sizeof(double),
                                 cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(dTimes.p, hTimes.p, (size_t)N * sizeof(double),
                                 cudaMemcpyHostToDevice, s)))
            return e;
        if (precision == HPHC_PRECISION_FP64) {
            e = launch_pack_f64(D, N, dLoc.p, dTimes.p, dRecF64.p, dTileMin.p, dTileMax.p, s);
            *launches += 2;
            return e;
        }
        if ((e = launch_strip_order(D, N, 2, dLoc.p, dOrder2.p, s)) ||
            (e = launch_strip_order(D, N, 4, dLoc.p, dOrder4.p, s)))
            return e;
        for (int S = 2 * kSweepThreads; S <= 4 * kSweepThreads; S *= 2)
            *launches += (N >= S) + (N % S != 0);
        if (sorted) {
            if ((e = launch_tile_bounds(N, dTimes.p, dTileMin.p, dTileMax.p, dTileChanges.p, s,
                                        floatTimes)))
                return e;
            e = launch_sorted_ranks(N, dTimes.p, dTileChanges.p, dRanks.p, s, floatTimes);
            *launches += 3;
        } else {
            if ((e = cudaMemcpyAsync(dRanks.p, hRanks.p, (size_t)N * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, s)))
                return e;
            e = launch_tile_bounds(N, dTimes.p, dTileMin.p, dTileMax.p, nullptr, s);
            *launches += 1;
        }
        return e;
    }

    SetView view() const {
        SetView v;
        v.N = N;
        v.dLoc = dLoc.p;
        v.dTimes = dTimes.p;
        v.dRanks = dRanks.p;
        v.dOrder2 = dOrder2.p;
        v.dOrder4 = dOrder4.p;
        v.dRecF64 = dRecF64.p;
        v.dTileMin = dTileMin.p;
        v.dTileMax = dTileMax.p;
        v.hTimes = hTimes.p;
        v.hTileMin = hTileMin.data();
        v.hTileMax = hTileMax.data();
        v.sorted = sorted;
        return v;
    }
};

int fmt(std::string& dst, int status, const char* f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    dst = buf;
    return status;
}

int cuda_status(std::string& dst, cudaError_t e, const char* what) {
    return fmt(dst, e == cudaErrorMemoryAllocation ? HPHC_ERR_OUT_OF_MEMORY : HPHC_ERR_CUDA,
               "%s: %s", what, cudaGetErrorString(e));
}

// Shared set-up of the engine and multiset handles: device, stream,
// exponential calibration (hardware-exponential mode only), executor.
struct Runtime {
    int device = 0;
    Mode mode;
    cudaStream_t stream = nullptr;
    double ex2Bias = 0.0;
    Executor ex;

    int init(int D, long fl, int dev, std::string& err) {
        mode = mode_from_flags(fl);
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1)
            return fmt(err, HPHC_ERR_NO_DEVICE, "no CUDA device visible");
        device = (dev < 0 || dev >= count) ? 0 : dev;
        DeviceGuard g(device);
        if (!g.ok) return fmt(err, HPHC_ERR_CUDA, "cannot select device %d", device);
        cudaError_t e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_status(err, e, "create stream");
        // FP32-compensated mode: the hardware exponential's mean relative
        // error, divided out of every term that comes from it (all of them in
        // the hardware-exponential variant, the far tail in the default one;
        // the plain FP32 mode keeps it, as the reference's float engine does)
        if (mode.precision == HPHC_PRECISION_FP32_COMP &&
            (e = ex2_bias_for_device(device, stream, &ex2Bias)) != cudaSuccess)
            return cuda_status(err, e, "exponential calibration");
        const int st = ex.init(D, mode.precision, mode.variant, mode.underflowSkip, device, stream,
                               ex2Bias);
        ex.symmetric = mode.symmetric;
        ex.fastTail = mode.fastTail;
        ex.truncateTail = mode.truncateTail;
        if (st) err = ex.error;
        return st;
    }

    void release() {
        DeviceGuard g(device);
        if (stream) cudaStreamSynchronize(stream);
        ex.release();
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }
};

// True if every entry is finite; otherwise *bad = the first that is not.  The
// first pass tests the exponent bits (all ones for NaN and infinity) with a
// branch-free reduction the compiler vectorises.
bool all_finite(const double* v, size_t n, size_t* bad) {
    constexpr uint64_t kExp = 0x7ff0000000000000ULL;
    uint64_t any = 0;
    for (size_t i = 0; i < n; ++i) {
        uint64_t u;
        std::memcpy(&u, v + i, sizeof u);
        any |= (uint64_t)((u & kExp) == kExp);
    }
    if (!any) return true;
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) {
            *bad = i;
            return false;
        }
    return true;
}

// Copies n doubles from src to dst and tests them in the same pass (one read
// of the caller's array instead of one for the test and one for the copy):
// false if any is not finite, with *bad the first such index (dst is then
// partly written and must be discarded).  ASC: *ascending = src is
// non-decreasing.
//
// The destination is a pinned mirror the next upload reads by DMA; with SSE2
// and a 16-byte aligned destination the copy uses streaming stores, which
// write it without first reading it into the cache (a third of the memory
// traffic of the pass).
template <bool ASC>
bool copy_checked(const double* __restrict__ src, double* __restrict__ dst, size_t n,
                  size_t* bad, bool* ascending) {
    constexpr uint64_t kExp = 0x7ff0000000000000ULL;
    uint64_t any = 0, desc = 0;
    size_t i0 = 0;
#if defined(__SSE2__)
    if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0 && n >= 4) {
        const __m128d zero = _mm_setzero_pd();
        __m128d bad2 = zero, desc2 = zero;
        const size_t n2 = n & ~size_t(1);
        for (size_t i = 0; i < n2; i += 2) {
            const __m128d v = _mm_loadu_pd(src + i);
            const __m128d z = _mm_mul_pd(v, zero);  // 0 for finite values, NaN otherwise
            bad2 = _mm_or_pd(bad2, _mm_cmpunord_pd(z, z));
            if (ASC && i > 0) desc2 = _mm_or_pd(desc2, _mm_cmpgt_pd(_mm_loadu_pd(src + i - 1), v));
            _mm_stream_pd(dst + i, v);
        }
        _mm_sfence();
        if (ASC && n2 > 1 && src[0] > src[1]) desc = 1;
        if (_mm_movemask_pd(bad2)) any = 1;
        if (_mm_movemask_pd(desc2)) desc = 1;
        i0 = n2;  // an odd last value goes through the loop below
    }
#endif
    for (size_t i = i0; i < n; ++i) {
        const double v = src[i];
        uint64_t u;
        std::memcpy(&u, &v, sizeof u);
        any |= (uint64_t)((u & kExp) == kExp);
        if (ASC && i > 0) desc |= (uint64_t)(src[i - 1] > v);
        dst[i] = v;
    }
    if (ASC) *ascending = desc == 0;
    if (!any) return true;
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(src[i])) {
            *bad = i;
            return false;
        }
    return true;
}

}  // namespace

struct hphc_engine {
    int D = 0, N = 0;
    long flags = 0;
    std::string lastError;
    Runtime rt;

    // state (src/NewHawkes.hpp:851-866)
    double params[6] = {0, 0, 0, 0, 0, 0};
    double storedParams[6] = {0, 0, 0, 0, 0, 0};
    double sumOfLikContribs = 0.0, storedSumOfLikContribs = 0.0;
    HostBuf<double> hLoc[2];  // double-buffered location mirrors (src/NewHawkes.hpp:869-873)
    int curLoc = 0;
    // A full new location block or time vector is copied and checked in one
    // pass into a spare mirror, which replaces the current one only if every
    // value is finite: a rejected input leaves the events unchanged.
    HostBuf<double> hLocSpare, hTimesSpare;
    EventSet set;
    DevBuf<double> dProbs;
    std::vector<double> hOut;
    bool dirty = true;
    int lastLaunches = 0;

    // Incremental evaluation.  After an evaluation of the engine's own
    // parameters, dSums keeps every event's six unit pair sums (natural
    // units, [6][N]) for sumsParams.  Moving a few events (updateLocations
    // with an index) records their previous locations; the next evaluation at
    // the same parameters updates the sums in O(N) per moved event and
    // re-runs only the O(N) finish, instead of the O(N^2) sweep.  storeState
    // keeps a device copy of the sums, which restoreState brings back.
    bool incremental = true;
    DevBuf<double> dSums, dStoredSums, dRowPartials, dIncBlockSums, dIncOut;
    HostBuf<double> hIncOut;
    bool sumsValid = false, storedSumsValid = false, recStale = false;
    double sumsParams[6] = {0, 0, 0, 0, 0, 0}, storedSumsParams[6] = {0, 0, 0, 0, 0, 0};
    double pendingSumsParams[6] = {0, 0, 0, 0, 0, 0};
    bool pendingSums = false;
    std::vector<int> moved;            // moved events, in order of their first move
    std::vector<double> movedOld;      // their locations when the sums were formed (D each)
    std::vector<int> movedSlot;        // event -> index into moved, or -1
    int maxMoved = 1;
    int lastPath = HPHC_PATH_SWEEP;
    double lastIncTerms = 0.0;  // pair terms of the last incremental evaluation

    // Sharded evaluation: the last sweep_shard ran at shardParams on the
    // current events (cleared when the events change).
    bool shardValid = false;
    double shardParams[6] = {0, 0, 0, 0, 0, 0};

    void clear_moved() {
        for (int k : moved) movedSlot[k] = -1;
        moved.clear();
        movedOld.clear();
    }

    void invalidate_sums() {
        sumsValid = false;
        shardValid = false;
        clear_moved();
    }

    int fail(int status, const char* f, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, f);
        vsnprintf(buf, sizeof buf, f, ap);
        va_end(ap);
        lastError = buf;
        return status;
    }

    int init(int dim, int n, long fl, int dev) {
        D = dim;
        N = n;
        flags = fl;
        int st = rt.init(D, fl, dev, lastError);
        if (st) return st;
        DeviceGuard g(rt.device);
        const size_t nl = (size_t)N * D;
        cudaError_t e;
        if ((e = hLoc[0].reserve(nl)) || (e = hLoc[1].reserve(nl)) ||
            (e = hLocSpare.reserve(nl)) || (e = hTimesSpare.reserve(N)))
            return cuda_status(lastError, e, "pinned host allocation");
        std::memset(hLoc[0].p, 0, nl * sizeof(double));
        std::memset(hLoc[1].p, 0, nl * sizeof(double));
        if ((e = set.alloc(D, N, rt.mode.precision)) || (e = dProbs.reserve(N)))
            return cuda_status(lastError, e, "device allocation");
        incremental = !(fl & HPHC_FLAG_NO_INCREMENTAL);
        if (incremental) {
            if ((e = dSums.reserve((size_t)kNumAcc * N)) ||
                (e = dStoredSums.reserve((size_t)kNumAcc * N)) ||
                (e = dRowPartials.reserve((size_t)kNumAcc * move_event_blocks(N))) ||
                (e = dIncBlockSums.reserve((size_t)8 * finish_blocks(N))) ||
                (e = dIncOut.reserve(8)) || (e = hIncOut.reserve(8)))
                return cuda_status(lastError, e, "device allocation");
            movedSlot.assign(N, -1);
            const int nTiles = (N + kTile - 1) / kTile;
            maxMoved = std::max(1, std::min(64, nTiles / 4));
        }
        set.derive_times();
        dirty = true;
        return HPHC_OK;
    }

    void destroy() {
        rt.release();
        DeviceGuard g(rt.device);
        hLoc[0].release();
        hLoc[1].release();
        hLocSpare.release();
        hTimesSpare.release();
        set.release();
        dProbs.release();
        dSums.release();
        dStoredSums.release();
        dRowPartials.release();
        dIncBlockSums.release();
        dIncOut.release();
        hIncOut.release();
    }

    int faultUploads = 0;  // injected upload failures still to deliver

    int upload_if_dirty() {
        if (!dirty) return HPHC_OK;
        NvtxRange range("hphc upload");
        if (faultUploads > 0) {
            --faultUploads;
            return cuda_status(lastError, cudaErrorMemoryAllocation, "upload (injected)");
        }
        const cudaError_t e = set.upload(hLoc[curLoc].p, rt.mode.precision, rt.stream,
                                         &lastLaunches);
        if (e != cudaSuccess) return cuda_status(lastError, e, "upload");
        dirty = false;
        recStale = false;  // the upload re-packs the records
        return HPHC_OK;
    }

    // The kept background sums serve parameter vectors p (K x 6) when every
    // one has the kept tauX and tauT: the background unit sums depend on the
    // events and those two parameters only.  With no moved event the sums
    // describe the host copy of the events, which enqueue uploads if needed.
    bool kept_background_serves(const double* p, int K) const {
        if (!incremental || !sumsValid || pendingSums || !moved.empty()) return false;
        for (int k = 0; k < K; ++k)
            if (p[6 * k + 1] != sumsParams[1] || p[6 * k + 2] != sumsParams[2]) return false;
        return true;
    }

    // Enqueue K parameter vectors on this engine's events: the full sweep, or
    // (reuse) only the self-excitation terms when the kept background sums
    // serve.
    int enqueue(const double* p, int K, bool wantProbs, bool reuse = true) {
        NvtxRange range("hphc sweep enqueue");
        lastLaunches = 0;
        const bool selfOnly = reuse && kept_background_serves(p, K);
        lastPath = selfOnly ? HPHC_PATH_SELF_EXCITATION : HPHC_PATH_SWEEP;
        // moved events are only on the host, and after incremental row uploads
        // the packed FP64 records are stale: upload and pack everything (the
        // kept sums and the moved list stay a consistent pair)
        if (!moved.empty() || recStale) dirty = true;
        int st = upload_if_dirty();
        if (st) return st;
        std::vector<SetView> sets{set.view()};
        std::vector<int> setOf(K, 0);
        // the evaluation keeps problem 0's sums (a self-excitation-only sweep
        // rewrites rows 3-5 and keeps rows 0-2)
        pendingSums = incremental;
        rt.ex.sumsOut = pendingSums ? dSums.p : nullptr;
        rt.ex.keptB = selfOnly ? dSums.p : nullptr;
        if (pendingSums) {
            invalidate_sums();
            std::memcpy(pendingSumsParams, p, sizeof pendingSumsParams);
        }
        st = rt.ex.enqueue(sets, setOf.data(), p, K, wantProbs ? dProbs.p : nullptr);
        rt.ex.sumsOut = nullptr;
        rt.ex.keptB = nullptr;
        if (st) {
            pendingSums = false;
            return fmt(lastError, st, "%s", rt.ex.error.c_str());
        }
        lastLaunches += rt.ex.lastLaunches;
        return HPHC_OK;
    }

    int wait(int K) {
        hOut.resize((size_t)K * 8);
        const int st = rt.ex.wait(hOut.data());
        if (st) {
            pendingSums = false;
            return fmt(lastError, st, "%s", rt.ex.error.c_str());
        }
        if (pendingSums) {
            sumsValid = true;
            std::memcpy(sumsParams, pendingSumsParams, sizeof sumsParams);
            pendingSums = false;
        }
        return HPHC_OK;
    }

    // The kept sums serve p in full when sigma, tauX, tauT and omega are the
    // kept ones (theta and mu0 enter only the finish).
    bool can_update(const double* p) const {
        return incremental && sumsValid && !pendingSums &&
               std::memcmp(p, sumsParams, 4 * sizeof(double)) == 0;
    }

    // O(N) evaluation from the kept sums: upload and apply each moved event,
    // then the per-event finish.
    int evaluate_incremental(const double* p, double* loglik, double* grad, double* probs) {
        NvtxRange range("hphc kept-sums finish");
        lastLaunches = 0;
        const bool hadMoves = !moved.empty();
        const bool wasDirty = dirty;
        int st = upload_if_dirty();
        if (st) return st;
        cudaStream_t s = rt.stream;
        const PairConsts c = rt.ex.pair_consts(p);
        cudaError_t e = cudaSuccess;
        for (size_t m = 0; m < moved.size(); ++m) {
            MovedEvent mv{};
            mv.k = moved[m];
            for (int a = 0; a < D; ++a) mv.oldLoc[a] = movedOld[m * D + a];
            const size_t off = (size_t)mv.k * D;
            if (!wasDirty &&
                (e = cudaMemcpyAsync(set.dLoc.p + off, hLoc[curLoc].p + off, D * sizeof(double),
                                     cudaMemcpyHostToDevice, s)))
                return cuda_status(lastError, e, "upload moved event");
            if ((e = launch_move_event(D, N, mv, set.dLoc.p, set.dTimes.p, c, dSums.p,
                                       dRowPartials.p, s)) ||
                (e = launch_move_event_row(N, mv.k, dRowPartials.p, dSums.p, s)))
                return cuda_status(lastError, e, "move event");
            lastLaunches += 2;
        }
        if (hadMoves && !wasDirty && rt.mode.precision == HPHC_PRECISION_FP64) recStale = true;
        lastIncTerms = (double)moved.size() * (3.0 * N - 2.0);
        clear_moved();
        const FinishConsts f = rt.ex.finish_consts(p, set.view());
        if ((e = launch_finish_sums(N, dSums.p, set.dTimes.p, f, dIncBlockSums.p,
                                    probs ? dProbs.p : nullptr, dIncOut.p, s)) ||
            (e = cudaMemcpyAsync(hIncOut.p, dIncOut.p, 8 * sizeof(double),
                                 cudaMemcpyDeviceToHost, s)))
            return cuda_status(lastError, e, "finish from kept sums");
        lastLaunches += 2;
        if ((e = cudaStreamSynchronize(s))) return cuda_status(lastError, e, "evaluation");
        if (probs &&
            (e = cudaMemcpy(probs, dProbs.p, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost)))
            return cuda_status(lastError, e, "read probabilities");
        if (loglik) *loglik = hIncOut.p[0];
        if (grad)
            for (int k = 0; k < 6; ++k) grad[k] = hIncOut.p[1 + k];
        lastPath = hadMoves ? HPHC_PATH_INCREMENTAL : HPHC_PATH_KEPT_SUMS;
        return HPHC_OK;
    }

    // Rank `rank` of `world`: this rank's share of the unit pair sums at the
    // current parameters into dPart ([6][N], natural units).
    int sweep_shard(int rank, int world, double* dPart) {
        NvtxRange range("hphc sweep shard");
        lastLaunches = 0;
        lastPath = HPHC_PATH_SWEEP;
        shardValid = false;
        if (!moved.empty() || recStale) dirty = true;
        int st = upload_if_dirty();
        if (st) return st;
        std::vector<SetView> sets{set.view()};
        const int setOf = 0;
        rt.ex.sumsOut = dPart;
        rt.ex.shardRank = rank;
        rt.ex.shardWorld = world;
        st = rt.ex.enqueue(sets, &setOf, params, 1, nullptr);
        if (st == HPHC_OK) {
            lastLaunches += rt.ex.lastLaunches;
            hOut.resize(8);
            st = rt.ex.wait(hOut.data());  // its log-likelihood is of a share: not used
        }
        rt.ex.sumsOut = nullptr;
        rt.ex.shardRank = 0;
        rt.ex.shardWorld = 1;
        if (st) return fmt(lastError, st, "%s", rt.ex.error.c_str());
        shardValid = true;
        std::memcpy(shardParams, params, sizeof shardParams);
        return HPHC_OK;
    }

    // The sums of nParts shares (rank order) become the kept sums at the
    // current parameters.
    int set_unit_sums(const double* dParts, int nParts) {
        if (!incremental)
            return fail(HPHC_ERR_UNSUPPORTED,
                        "unit sums: the engine keeps no sums (HPHC_FLAG_NO_INCREMENTAL)");
        if (!shardValid || dirty || !moved.empty() ||
            std::memcmp(params, shardParams, sizeof shardParams) != 0)
            return fail(HPHC_ERR_BAD_ARGUMENT,
                        "unit sums: events or parameters changed since this engine's "
                        "hphc_sweep_shard");
        const size_t n = (size_t)kNumAcc * N;
        cudaError_t e = launch_sum_parts(dParts, nParts, n, dSums.p, rt.ex.num_sms(), rt.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(rt.stream);
        if (e != cudaSuccess) {
            invalidate_sums();
            return cuda_status(lastError, e, "sum of the shares");
        }
        pendingSums = false;
        sumsValid = true;
        std::memcpy(sumsParams, params, sizeof sumsParams);
        return HPHC_OK;
    }

    int evaluate(const double* p, double* loglik, double* grad, double* probs) {
        NvtxRange range("hphc evaluate");
        DeviceGuard g(rt.device);
        if (!g.ok) return fail(HPHC_ERR_CUDA, "cannot select device %d", rt.device);
        if (can_update(p)) return evaluate_incremental(p, loglik, grad, probs);
        int st = enqueue(p, 1, probs != nullptr);
        if (st) return st;
        if ((st = wait(1))) return st;
        if (probs) {
            cudaError_t e = cudaMemcpy(probs, dProbs.p, (size_t)N * sizeof(double),
                                       cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) return cuda_status(lastError, e, "read probabilities");
        }
        if (loglik) *loglik = hOut[0];
        if (grad)
            for (int k = 0; k < 6; ++k) grad[k] = hOut[1 + k];
        return HPHC_OK;
    }
};

struct hphc_multiset {
    int D = 0, S = 0;
    std::string lastError;
    Runtime rt;
    std::vector<EventSet> sets;
    std::vector<HostBuf<double>> hLoc;
    std::vector<char> ready, dirty;
    // Each set is uploaded as soon as its data arrives (the copy from its
    // pinned mirror overlaps the host work on the next sets); its event marks
    // the end of that copy, which a later setData of the set waits for
    // before it overwrites the mirror.
    std::vector<cudaEvent_t> uploaded;
    std::vector<double> hOut;
    int lastLaunches = 0;

    int init(int dim, int numSets, const int* sizes, long fl, int dev) {
        D = dim;
        S = numSets;
        int st = rt.init(D, fl, dev, lastError);
        if (st) return st;
        DeviceGuard g(rt.device);
        sets.resize(S);
        hLoc.resize(S);
        ready.assign(S, 0);
        dirty.assign(S, 1);
        uploaded.assign(S, nullptr);
        for (int s = 0; s < S; ++s) {
            cudaError_t e;
            if ((e = sets[s].alloc(D, sizes[s], rt.mode.precision)) ||
                (e = hLoc[s].reserve((size_t)sizes[s] * D)) ||
                (e = cudaEventCreateWithFlags(&uploaded[s], cudaEventDisableTiming)))
                return cuda_status(lastError, e, "allocation");
            sets[s].derive_times();
        }
        return HPHC_OK;
    }

    void destroy() {
        rt.release();  // waits for the stream: no copy still reads the mirrors
        DeviceGuard g(rt.device);
        for (auto& ev : uploaded)
            if (ev) cudaEventDestroy(ev);
        for (auto& s : sets) s.release();
        for (auto& h : hLoc) h.release();
    }
};

int hphc::engine_loop_setup(hphc_engine* e, const double* params, int K, EngineLoop* out,
                            std::string* err) {
    DeviceGuard g(e->rt.device);
    if (!g.ok) return fmt(*err, HPHC_ERR_CUDA, "cannot select device %d", e->rt.device);
    // moved events are only on the host, and after incremental row uploads
    // the packed FP64 records are stale: upload and pack everything
    if (!e->moved.empty() || e->recStale) e->dirty = true;
    int st = e->upload_if_dirty();
    if (st) return fmt(*err, st, "%s", e->lastError.c_str());
    std::vector<SetView> sets{e->set.view()};
    std::vector<int> setOf(K, 0);
    // Chains that all have the kept sums' tauX and tauT (the loop keeps them
    // fixed) reuse the kept background sums in every iteration and sweep only
    // the self-excitation terms.  The loop does not write the kept sums.
    e->rt.ex.keptB = e->kept_background_serves(params, K) ? e->dSums.p : nullptr;
    st = e->rt.ex.setup_device_loop(sets, setOf.data(), params, K);
    out->spec = e->rt.ex.consts_spec();
    e->rt.ex.keptB = nullptr;
    if (st) return fmt(*err, st, "%s", e->rt.ex.error.c_str());
    out->device = e->rt.device;
    out->stream = e->rt.stream;
    out->ex = &e->rt.ex;
    return HPHC_OK;
}

// ------------------------------------------------------------------ C ABI --

extern "C" {

const char* hphc_status_string(int status) {
    switch (status) {
        case HPHC_OK: return "ok";
        case HPHC_ERR_INVALID_HANDLE: return "invalid handle";
        case HPHC_ERR_BAD_LENGTH: return "bad length";
        case HPHC_ERR_BAD_ARGUMENT: return "bad argument";
        case HPHC_ERR_NONFINITE: return "non-finite input";
        case HPHC_ERR_UNSUPPORTED: return "unsupported";
        case HPHC_ERR_CUDA: return "CUDA error";
        case HPHC_ERR_NOT_READY: return "not ready";
        case HPHC_ERR_DEVICE_TIMEOUT: return "device wait timed out";
        case HPHC_ERR_NO_DEVICE: return "no CUDA device";
        case HPHC_ERR_OUT_OF_MEMORY: return "out of memory";
        case HPHC_ERR_SCRATCH_TOO_SMALL: return "scratch too small";
        default: return "unknown status";
    }
}

int hphc_create(int embeddingDimension, int locationCount, long flags, int device,
                hphc_engine** out) {
    if (!out) return HPHC_ERR_BAD_ARGUMENT;
    *out = nullptr;
    if (embeddingDimension < 1 || embeddingDimension > kMaxDim) return HPHC_ERR_UNSUPPORTED;
    if (locationCount < 1) return HPHC_ERR_BAD_ARGUMENT;
    if ((long long)locationCount * embeddingDimension > (1LL << 31) - 1) return HPHC_ERR_UNSUPPORTED;
    hphc_engine* e = new (std::nothrow) hphc_engine();
    if (!e) return HPHC_ERR_OUT_OF_MEMORY;
    const int st = e->init(embeddingDimension, locationCount, flags, device);
    if (st != HPHC_OK) {
        e->destroy();
        delete e;
        return st;
    }
    *out = e;
    return HPHC_OK;
}

void hphc_destroy(hphc_engine* engine) {
    if (!engine) return;
    engine->destroy();
    delete engine;
}

const char* hphc_last_error(const hphc_engine* engine) {
    return engine ? engine->lastError.c_str() : "invalid handle";
}

int hphc_set_times_data(hphc_engine* e, const double* data, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!data) return e->fail(HPHC_ERR_BAD_ARGUMENT, "times: null pointer");
    if (length != (size_t)e->N)
        return e->fail(HPHC_ERR_BAD_LENGTH, "times: length %zu != locationCount %d", length, e->N);
    size_t bad = 0;
    bool ascending = false;
    if (!copy_checked<true>(data, e->hTimesSpare.p, length, &bad, &ascending))
        return e->fail(HPHC_ERR_NONFINITE, "times: entry %zu is not finite", bad);
    e->set.hTimes.swap(e->hTimesSpare);
    e->set.derive_times(ascending ? 1 : 0);
    e->dirty = true;
    e->invalidate_sums();
    return HPHC_OK;
}

int hphc_update_locations(hphc_engine* e, int locationIndex, const double* location,
                          size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!location) return e->fail(HPHC_ERR_BAD_ARGUMENT, "locations: null pointer");
    size_t offset = 0;
    if (locationIndex == -1) {
        if (length != (size_t)e->N * e->D)
            return e->fail(HPHC_ERR_BAD_LENGTH, "locations: length %zu != D*N = %zu", length,
                           (size_t)e->N * e->D);
    } else {
        if (locationIndex < 0 || locationIndex >= e->N)
            return e->fail(HPHC_ERR_BAD_ARGUMENT, "locations: index %d out of range",
                           locationIndex);
        if (length != (size_t)e->D)
            return e->fail(HPHC_ERR_BAD_LENGTH, "locations: length %zu != D = %d", length, e->D);
        offset = (size_t)locationIndex * e->D;
    }
    size_t bad = 0;
    if (locationIndex == -1) {
        if (!copy_checked<false>(location, e->hLocSpare.p, length, &bad, nullptr))
            return e->fail(HPHC_ERR_NONFINITE, "locations: entry %zu is not finite", bad);
        e->hLoc[e->curLoc].swap(e->hLocSpare);
        e->invalidate_sums();
        e->dirty = true;
        return HPHC_OK;
    }
    if (!all_finite(location, length, &bad))
        return e->fail(HPHC_ERR_NONFINITE, "locations: entry %zu is not finite", bad);
    double* row = e->hLoc[e->curLoc].p + offset;
    if (locationIndex >= 0 && e->sumsValid) {
        // one event moves: keep the location its sums were formed with
        if (e->movedSlot[locationIndex] < 0) {
            if ((int)e->moved.size() >= e->maxMoved) {
                e->invalidate_sums();  // cheaper to sweep again
                e->dirty = true;
            } else {
                e->movedSlot[locationIndex] = (int)e->moved.size();
                e->moved.push_back(locationIndex);
                e->movedOld.insert(e->movedOld.end(), row, row + e->D);
            }
        }
    } else {
        e->invalidate_sums();
        e->dirty = true;
    }
    std::memcpy(row, location, length * sizeof(double));
    return HPHC_OK;
}

int hphc_set_parameters(hphc_engine* e, const double* data, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!data) return e->fail(HPHC_ERR_BAD_ARGUMENT, "parameters: null pointer");
    if (length != 6) return e->fail(HPHC_ERR_BAD_LENGTH, "parameters: length %zu != 6", length);
    std::memcpy(e->params, data, 6 * sizeof(double));
    return HPHC_OK;
}

int hphc_get_sum_of_lik_contribs(hphc_engine* e, double* out) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!out) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    const int st = e->evaluate(e->params, out, nullptr, nullptr);
    if (st == HPHC_OK) e->sumOfLikContribs = *out;
    return st;
}

int hphc_get_log_likelihood_gradient(hphc_engine* e, double* out, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!out) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    if (length != 6) return e->fail(HPHC_ERR_BAD_LENGTH, "gradient: length %zu != 6", length);
    double ll = 0.0;
    const int st = e->evaluate(e->params, &ll, out, nullptr);
    if (st == HPHC_OK) e->sumOfLikContribs = ll;
    return st;
}

int hphc_get_log_likelihood_and_gradient(hphc_engine* e, double* loglik, double* gradient,
                                         size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!loglik) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    if (gradient && length != 6)
        return e->fail(HPHC_ERR_BAD_LENGTH, "gradient: length %zu != 6", length);
    const int st = e->evaluate(e->params, loglik, gradient, nullptr);
    if (st == HPHC_OK) e->sumOfLikContribs = *loglik;
    return st;
}

int hphc_get_probs_self_excite(hphc_engine* e, double* out, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!out) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    if (length != (size_t)e->N)
        return e->fail(HPHC_ERR_BAD_LENGTH, "probs: length %zu != locationCount %d", length, e->N);
    return e->evaluate(e->params, nullptr, nullptr, out);
}

int hphc_store_state(hphc_engine* e) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    e->storedSumOfLikContribs = e->sumOfLikContribs;
    std::memcpy(e->storedParams, e->params, sizeof e->params);
    std::memcpy(e->hLoc[1 - e->curLoc].p, e->hLoc[e->curLoc].p,
                (size_t)e->N * e->D * sizeof(double));
    // the kept sums describe the stored locations when no event has moved since
    e->storedSumsValid = false;
    if (e->sumsValid && e->moved.empty()) {
        DeviceGuard g(e->rt.device);
        const cudaError_t err = cudaMemcpyAsync(e->dStoredSums.p, e->dSums.p,
                                                (size_t)kNumAcc * e->N * sizeof(double),
                                                cudaMemcpyDeviceToDevice, e->rt.stream);
        if (err != cudaSuccess) return cuda_status(e->lastError, err, "store sums");
        e->storedSumsValid = true;
        std::memcpy(e->storedSumsParams, e->sumsParams, sizeof e->sumsParams);
    }
    return HPHC_OK;
}

int hphc_restore_state(hphc_engine* e) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    e->sumOfLikContribs = e->storedSumOfLikContribs;
    std::memcpy(e->params, e->storedParams, sizeof e->params);
    e->curLoc = 1 - e->curLoc;
    e->dirty = true;
    e->clear_moved();
    if (e->storedSumsValid) {
        std::swap(e->dSums, e->dStoredSums);
        std::memcpy(e->sumsParams, e->storedSumsParams, sizeof e->sumsParams);
        e->sumsValid = true;
        e->storedSumsValid = false;
    } else {
        e->sumsValid = false;
    }
    return HPHC_OK;
}

int hphc_accept_state(hphc_engine* e) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    return HPHC_OK;
}

int hphc_get_internal_dimension(hphc_engine* e, int* out) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!out) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    *out = e->D;
    return HPHC_OK;
}

int hphc_batch_log_likelihood_and_gradient(hphc_engine* e, const double* params, int K,
                                           double* loglik, double* gradient) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!params || !loglik) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null pointer");
    if (K < 1) return e->fail(HPHC_ERR_BAD_ARGUMENT, "K = %d < 1", K);
    DeviceGuard g(e->rt.device);
    if (!g.ok) return e->fail(HPHC_ERR_CUDA, "cannot select device %d", e->rt.device);
    int st = e->enqueue(params, K, false);
    if (st) return st;
    if ((st = e->wait(K))) return st;
    for (int k = 0; k < K; ++k) {
        loglik[k] = e->hOut[(size_t)8 * k];
        if (gradient)
            for (int q = 0; q < 6; ++q)
                gradient[(size_t)6 * k + q] = e->hOut[(size_t)8 * k + 1 + q];
    }
    return HPHC_OK;
}

int hphc_get_precision(hphc_engine* e, int* out) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!out) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    *out = e->rt.mode.precision;
    return HPHC_OK;
}

int hphc_get_stream(hphc_engine* e, void** stream) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!stream) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    *stream = (void*)e->rt.stream;
    return HPHC_OK;
}

int hphc_enqueue_log_likelihood_and_gradient(hphc_engine* e) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    DeviceGuard g(e->rt.device);
    if (!g.ok) return e->fail(HPHC_ERR_CUDA, "cannot select device %d", e->rt.device);
    return e->enqueue(e->params, 1, false, /*reuse=*/false);  // always the full sweep
}

int hphc_read_results(hphc_engine* e, double* loglik, double* gradient, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (gradient && length != 6)
        return e->fail(HPHC_ERR_BAD_LENGTH, "gradient: length %zu != 6", length);
    DeviceGuard g(e->rt.device);
    const int st = e->wait(1);
    if (st) return st;
    if (loglik) *loglik = e->hOut[0];
    if (gradient)
        for (int k = 0; k < 6; ++k) gradient[k] = e->hOut[1 + k];
    return HPHC_OK;
}

// A device pointer on the engine's device (or managed memory).
static bool device_pointer_on(const void* p, int device) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice && a.device == device) ||
           a.type == cudaMemoryTypeManaged;
}

int hphc_sweep_shard(hphc_engine* e, int rank, int world, double* devicePart, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (world < 1 || rank < 0 || rank >= world)
        return e->fail(HPHC_ERR_BAD_ARGUMENT, "shard: rank %d of world %d", rank, world);
    if (length != (size_t)kNumAcc * e->N)
        return e->fail(HPHC_ERR_BAD_LENGTH, "shard: length %zu != 6 * locationCount = %zu",
                       length, (size_t)kNumAcc * e->N);
    DeviceGuard g(e->rt.device);
    if (!g.ok) return e->fail(HPHC_ERR_CUDA, "cannot select device %d", e->rt.device);
    if (!devicePart || !device_pointer_on(devicePart, e->rt.device))
        return e->fail(HPHC_ERR_BAD_ARGUMENT, "shard: output is not device memory of device %d",
                       e->rt.device);
    return e->sweep_shard(rank, world, devicePart);
}

int hphc_set_unit_sums(hphc_engine* e, const double* deviceParts, int numParts, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (numParts < 1) return e->fail(HPHC_ERR_BAD_ARGUMENT, "unit sums: %d parts", numParts);
    if (length != (size_t)numParts * kNumAcc * e->N)
        return e->fail(HPHC_ERR_BAD_LENGTH,
                       "unit sums: length %zu != parts * 6 * locationCount = %zu", length,
                       (size_t)numParts * kNumAcc * e->N);
    DeviceGuard g(e->rt.device);
    if (!g.ok) return e->fail(HPHC_ERR_CUDA, "cannot select device %d", e->rt.device);
    if (!deviceParts || !device_pointer_on(deviceParts, e->rt.device))
        return e->fail(HPHC_ERR_BAD_ARGUMENT,
                       "unit sums: input is not device memory of device %d", e->rt.device);
    return e->set_unit_sums(deviceParts, numParts);
}

int hphc_eval_exponentials(int device, const float* args, size_t n, float* poly,
                           float* hardware) {
    if (!args || !poly || !hardware || n == 0 || n > (size_t(1) << 28))
        return HPHC_ERR_BAD_ARGUMENT;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) return HPHC_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return HPHC_ERR_BAD_ARGUMENT;
    DeviceGuard g(device);
    if (!g.ok) return HPHC_ERR_CUDA;
    float* d = nullptr;
    if (cudaMalloc(&d, 3 * n * sizeof(float)) != cudaSuccess) return HPHC_ERR_OUT_OF_MEMORY;
    cudaError_t e = cudaMemcpy(d, args, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_eval_exponentials((int)n, d, d + n, d + 2 * n, nullptr);
    if (e == cudaSuccess)
        e = cudaMemcpy(poly, d + n, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(hardware, d + 2 * n, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? HPHC_OK : HPHC_ERR_CUDA;
}

int hphc_inject_fault(hphc_engine* e, int stage, int count) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (count < 0 || (count > 0 && (stage < HPHC_FAULT_UPLOAD || stage > HPHC_FAULT_WAIT)))
        return e->fail(HPHC_ERR_BAD_ARGUMENT, "fault injection: stage %d, count %d", stage, count);
    e->faultUploads = 0;
    e->rt.ex.faultStage = 0;
    e->rt.ex.faultCount = 0;
    if (count == 0) return HPHC_OK;
    if (stage == HPHC_FAULT_UPLOAD) {
        e->faultUploads = count;
    } else {
        e->rt.ex.faultStage = stage;
        e->rt.ex.faultCount = count;
    }
    return HPHC_OK;
}

int hphc_get_last_evaluation_path(hphc_engine* e, int* path) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!path) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    *path = e->lastPath;
    return HPHC_OK;
}

int hphc_get_last_launch_stats(hphc_engine* e, int* kernelLaunches, double* backgroundTerms,
                               double* selfExciteTerms) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (kernelLaunches) *kernelLaunches = e->lastLaunches;
    if (e->lastPath == HPHC_PATH_INCREMENTAL || e->lastPath == HPHC_PATH_KEPT_SUMS) {
        // per moved event: its pair with every other event at the old and the
        // new location, and its new row
        if (backgroundTerms) *backgroundTerms = e->lastIncTerms;
        if (selfExciteTerms) *selfExciteTerms = e->lastIncTerms;
        return HPHC_OK;
    }
    if (backgroundTerms || selfExciteTerms) {
        double nb = 0.0, ns = 0.0;
        std::vector<SetView> sets{e->set.view()};
        e->rt.ex.count_terms(sets, &nb, &ns);
        if (backgroundTerms) *backgroundTerms = nb;
        if (selfExciteTerms) *selfExciteTerms = ns;
    }
    return HPHC_OK;
}

int hphc_get_last_launch_evals(hphc_engine* e, double* backgroundEvals) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!backgroundEvals) return HPHC_ERR_BAD_ARGUMENT;
    if (e->lastPath == HPHC_PATH_INCREMENTAL || e->lastPath == HPHC_PATH_KEPT_SUMS) {
        *backgroundEvals = e->lastIncTerms;
        return HPHC_OK;
    }
    double nb = 0.0, ns = 0.0;
    std::vector<SetView> sets{e->set.view()};
    e->rt.ex.count_terms(sets, &nb, &ns, backgroundEvals);
    return HPHC_OK;
}

int hphc_set_sweep_shape(hphc_engine* e, int eventsPerThread, int itemsPerSM) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    const bool fp64 = e->rt.mode.precision == HPHC_PRECISION_FP64;
    const bool okR = eventsPerThread == 0 ||
                     (fp64 ? (eventsPerThread == 1 || eventsPerThread == 2)
                           : (eventsPerThread == 2 || eventsPerThread == 4));
    if (!okR)
        return e->fail(HPHC_ERR_BAD_ARGUMENT, "events per thread %d not supported",
                       eventsPerThread);
    if (itemsPerSM < 0 || itemsPerSM > 1024)
        return e->fail(HPHC_ERR_BAD_ARGUMENT, "items per SM %d out of range", itemsPerSM);
    e->rt.ex.fixedR = eventsPerThread;
    e->rt.ex.fixedItems = itemsPerSM;
    return HPHC_OK;
}

int hphc_get_sweep_shape(hphc_engine* e, int* eventsPerThread, int* itemsPerSM) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (eventsPerThread) *eventsPerThread = e->rt.ex.R;
    if (itemsPerSM) *itemsPerSM = e->rt.ex.itemsPerSM;
    return HPHC_OK;
}

int hphc_set_kernel_timing(hphc_engine* e, int enable) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    e->rt.ex.kernelTiming = enable != 0;
    return HPHC_OK;
}

int hphc_get_kernel_times(hphc_engine* e, float* sweepMs, float* finishMs, float* stepMs) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!e->rt.ex.timedValid)
        return e->fail(HPHC_ERR_NOT_READY, "no evaluation with kernel timing enabled yet");
    if (sweepMs) *sweepMs = e->rt.ex.lastSweepMs;
    if (finishMs) *finishMs = e->rt.ex.lastFinishMs;
    if (stepMs) *stepMs = e->rt.ex.lastStepMs;
    return HPHC_OK;
}

// ---- multiset --------------------------------------------------------------

int hphc_multiset_create(int embeddingDimension, int numSets, const int* setSizes, long flags,
                         int device, hphc_multiset** out) {
    if (!out) return HPHC_ERR_BAD_ARGUMENT;
    *out = nullptr;
    if (embeddingDimension < 1 || embeddingDimension > kMaxDim) return HPHC_ERR_UNSUPPORTED;
    if (numSets < 1 || !setSizes) return HPHC_ERR_BAD_ARGUMENT;
    for (int s = 0; s < numSets; ++s) {
        if (setSizes[s] < 1) return HPHC_ERR_BAD_ARGUMENT;
        if ((long long)setSizes[s] * embeddingDimension > (1LL << 31) - 1)
            return HPHC_ERR_UNSUPPORTED;
    }
    hphc_multiset* m = new (std::nothrow) hphc_multiset();
    if (!m) return HPHC_ERR_OUT_OF_MEMORY;
    const int st = m->init(embeddingDimension, numSets, setSizes, flags, device);
    if (st != HPHC_OK) {
        m->destroy();
        delete m;
        return st;
    }
    *out = m;
    return HPHC_OK;
}

void hphc_multiset_destroy(hphc_multiset* m) {
    if (!m) return;
    m->destroy();
    delete m;
}

const char* hphc_multiset_last_error(const hphc_multiset* m) {
    return m ? m->lastError.c_str() : "invalid handle";
}

int hphc_multiset_set_data(hphc_multiset* m, int set, const double* locations, size_t locLength,
                           const double* times, size_t timesLength) {
    if (!m) return HPHC_ERR_INVALID_HANDLE;
    if (set < 0 || set >= m->S)
        return fmt(m->lastError, HPHC_ERR_BAD_ARGUMENT, "set %d out of range", set);
    if (!locations || !times) return fmt(m->lastError, HPHC_ERR_BAD_ARGUMENT, "null pointer");
    EventSet& es = m->sets[set];
    if (locLength != (size_t)es.N * m->D || timesLength != (size_t)es.N)
        return fmt(m->lastError, HPHC_ERR_BAD_LENGTH,
                   "set %d: lengths %zu, %zu != D*N = %zu, N = %d", set, locLength, timesLength,
                   (size_t)es.N * m->D, es.N);
    size_t bad = 0;
    DeviceGuard g(m->rt.device);
    if (!g.ok) return fmt(m->lastError, HPHC_ERR_CUDA, "cannot select device %d", m->rt.device);
    cudaError_t e;
    int ascending = -1;
    if (m->ready[set] && !m->dirty[set]) {
        // The device holds the set's current data, so the new values are
        // checked while they are copied into the mirrors (one pass each);
        // a rejected input has the mirrors restored from the device copy.
        if ((e = cudaEventSynchronize(m->uploaded[set])) != cudaSuccess)
            return cuda_status(m->lastError, e, "wait for the set's upload");
        bool asc = false;
        if (!copy_checked<false>(locations, m->hLoc[set].p, locLength, &bad, nullptr) ||
            !copy_checked<true>(times, es.hTimes.p, timesLength, &bad, &asc)) {
            if ((e = cudaMemcpy(m->hLoc[set].p, es.dLoc.p, locLength * sizeof(double),
                                cudaMemcpyDeviceToHost)) ||
                (e = cudaMemcpy(es.hTimes.p, es.dTimes.p, timesLength * sizeof(double),
                                cudaMemcpyDeviceToHost)))
                return cuda_status(m->lastError, e, "restore the set after a rejected input");
            return fmt(m->lastError, HPHC_ERR_NONFINITE, "set %d: non-finite input", set);
        }
        ascending = asc ? 1 : 0;
    } else {
        if (!all_finite(locations, locLength, &bad) || !all_finite(times, timesLength, &bad))
            return fmt(m->lastError, HPHC_ERR_NONFINITE, "set %d: non-finite input", set);
        if ((e = cudaEventSynchronize(m->uploaded[set])) != cudaSuccess)
            return cuda_status(m->lastError, e, "wait for the set's upload");
        std::memcpy(m->hLoc[set].p, locations, locLength * sizeof(double));
        std::memcpy(es.hTimes.p, times, timesLength * sizeof(double));
    }
    es.derive_times(ascending);
    m->ready[set] = 1;
    m->dirty[set] = 1;
    // upload now, overlapping the host work on the next sets
    int launches = 0;
    if ((e = es.upload(m->hLoc[set].p, m->rt.mode.precision, m->rt.stream, &launches)) ||
        (e = cudaEventRecord(m->uploaded[set], m->rt.stream)))
        return cuda_status(m->lastError, e, "upload");
    m->dirty[set] = 0;
    return HPHC_OK;
}

int hphc_multiset_log_likelihood_and_gradient(hphc_multiset* m, const double* params,
                                              double* loglik, double* gradient) {
    if (!m) return HPHC_ERR_INVALID_HANDLE;
    if (!params || !loglik) return fmt(m->lastError, HPHC_ERR_BAD_ARGUMENT, "null pointer");
    for (int s = 0; s < m->S; ++s)
        if (!m->ready[s]) return fmt(m->lastError, HPHC_ERR_NOT_READY, "set %d has no data", s);
    DeviceGuard g(m->rt.device);
    if (!g.ok) return fmt(m->lastError, HPHC_ERR_CUDA, "cannot select device %d", m->rt.device);
    NvtxRange range("hphc multiset evaluate");
    m->lastLaunches = 0;
    std::vector<SetView> views(m->S);
    for (int s = 0; s < m->S; ++s) {
        if (m->dirty[s]) {
            const cudaError_t e = m->sets[s].upload(m->hLoc[s].p, m->rt.mode.precision,
                                                    m->rt.stream, &m->lastLaunches);
            if (e != cudaSuccess) return cuda_status(m->lastError, e, "upload");
            m->dirty[s] = 0;
        }
        views[s] = m->sets[s].view();
    }
    std::vector<int> setOf(m->S);
    std::iota(setOf.begin(), setOf.end(), 0);
    int st = m->rt.ex.enqueue(views, setOf.data(), params, m->S, nullptr);
    if (st) return fmt(m->lastError, st, "%s", m->rt.ex.error.c_str());
    m->lastLaunches += m->rt.ex.lastLaunches;
    m->hOut.resize((size_t)m->S * 8);
    if ((st = m->rt.ex.wait(m->hOut.data())))
        return fmt(m->lastError, st, "%s", m->rt.ex.error.c_str());
    for (int s = 0; s < m->S; ++s) {
        loglik[s] = m->hOut[(size_t)8 * s];
        if (gradient)
            for (int q = 0; q < 6; ++q)
                gradient[(size_t)6 * s + q] = m->hOut[(size_t)8 * s + 1 + q];
    }
    return HPHC_OK;
}

int hphc_multiset_set_kernel_timing(hphc_multiset* m, int enable) {
    if (!m) return HPHC_ERR_INVALID_HANDLE;
    m->rt.ex.kernelTiming = enable != 0;
    return HPHC_OK;
}

int hphc_multiset_get_kernel_times(hphc_multiset* m, float* sweepMs, float* finishMs,
                                   float* stepMs) {
    if (!m) return HPHC_ERR_INVALID_HANDLE;
    if (!m->rt.ex.timedValid)
        return fmt(m->lastError, HPHC_ERR_NOT_READY, "no evaluation with kernel timing enabled");
    if (sweepMs) *sweepMs = m->rt.ex.lastSweepMs;
    if (finishMs) *finishMs = m->rt.ex.lastFinishMs;
    if (stepMs) *stepMs = m->rt.ex.lastStepMs;
    return HPHC_OK;
}

int hphc_multiset_get_last_launch_stats(hphc_multiset* m, int* kernelLaunches,
                                        double* backgroundTerms, double* selfExciteTerms) {
    if (!m) return HPHC_ERR_INVALID_HANDLE;
    if (kernelLaunches) *kernelLaunches = m->lastLaunches;
    if (backgroundTerms || selfExciteTerms) {
        std::vector<SetView> views(m->S);
        for (int s = 0; s < m->S; ++s) views[s] = m->sets[s].view();
        double nb = 0.0, ns = 0.0;
        m->rt.ex.count_terms(views, &nb, &ns);
        if (backgroundTerms) *backgroundTerms = nb;
        if (selfExciteTerms) *selfExciteTerms = ns;
    }
    return HPHC_OK;
}

int hphc_multiset_get_last_launch_evals(hphc_multiset* m, double* backgroundEvals) {
    if (!m) return HPHC_ERR_INVALID_HANDLE;
    if (!backgroundEvals) return HPHC_ERR_BAD_ARGUMENT;
    std::vector<SetView> views(m->S);
    for (int s = 0; s < m->S; ++s) views[s] = m->sets[s].view();
    double nb = 0.0, ns = 0.0;
    m->rt.ex.count_terms(views, &nb, &ns, backgroundEvals);
    return HPHC_OK;
}

}  // extern "C"
