// Host side of the B200 Hawkes likelihood engine and its C ABI (include/hphc.h).
//
// One Engine per handle mirrors the state of the reference engines
// (src/NewHawkes.hpp:186-897, src/backend/opencl/OpenCLHawkes.hpp:42-997):
// six parameters plus a stored copy, double-buffered locations for
// store/restore, times, and the last log-likelihood.  Locations and times
// are kept in pinned host mirrors; a change marks the device copy dirty and
// the next evaluation uploads it and rebuilds the packed kernel records (one
// small kernel), so per-row updateLocations calls (src/benchmark.cpp:167-171)
// cost a host write each rather than a transfer each.
//
// Evaluation = sweep kernel (unit pair sums per event and j-chunk) -> finish
// kernel (per-event log-likelihood / gradient / probability, per-CTA sums) ->
// final kernel (fixed-order total), then one device-to-host copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <string>
#include <mutex>
#include <vector>

#include "hphc.h"
#include "hphc_kernels.cuh"

using namespace hphc;

namespace {

constexpr double kInvSqrt2Pi = 0.398942280401432677939946059934;
constexpr double kLog2e = 1.44269504088896340735992468100189214;
constexpr double kTwoPi = 6.28318530717958647692528676655900577;

// Underflow thresholds (natural-log units) for the tile-pair skip.  FP32:
// ex2.approx.ftz returns +0 for any argument below -126; a true exponent
// <= -88 is <= -126.96 in log2 units, which FP32 rounding of the computed
// exponent (relative ~1e-6) cannot lift above -126.  FP64: exp(x) is +0 for
// x < -745.14; -760 leaves a wide margin.
constexpr double kSkipF32 = 88.0;
constexpr double kSkipF64 = 760.0;

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
};

void split_float(double x, float& hi, float& lo) {
    hi = (float)x;
    lo = (float)(x - (double)hi);
}

// Exponent offset that removes the mean bias of ex2.approx.ftz.f32, measured
// once per device (2^20 arguments over [-16, 0)) and cached.
constexpr int kMaxDevices = 64;
constexpr int kEx2Samples = 1 << 20;
std::mutex gEx2Mutex;
bool gEx2Done[kMaxDevices] = {};
float gEx2Fix[kMaxDevices] = {};
double gEx2Bias[kMaxDevices] = {};

cudaError_t ex2_fix_for_device(int device, cudaStream_t stream, float* fix, double* bias) {
    std::lock_guard<std::mutex> lock(gEx2Mutex);
    if (device >= 0 && device < kMaxDevices && gEx2Done[device]) {
        *fix = gEx2Fix[device];
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
    const double beta = s / kEx2Samples;
    *bias = beta;
    *fix = (float)(-std::log2(1.0 + beta));
    if (device >= 0 && device < kMaxDevices) {
        gEx2Fix[device] = *fix;
        gEx2Bias[device] = beta;
        gEx2Done[device] = true;
    }
    return cudaSuccess;
}

// Autotuned sweep shapes, per process: key (size bucket, D, precision,
// variant) -> (events per thread, items per SM).
std::mutex gTuneMutex;
std::map<long, std::pair<int, int>> gTuneCache;

}  // namespace

struct hphc_engine {
    int D = 0, N = 0;
    long flags = 0;
    int device = 0;
    int precision = HPHC_PRECISION_FP64;
    bool underflowSkip = true;
    int numSMs = 148;
    std::string lastError;

    cudaStream_t stream = nullptr;

    // state (src/NewHawkes.hpp:851-866)
    double params[6] = {0, 0, 0, 0, 0, 0};
    double storedParams[6] = {0, 0, 0, 0, 0, 0};
    double sumOfLikContribs = 0.0, storedSumOfLikContribs = 0.0;
    HostBuf<double> hLoc[2];  // double-buffered location mirrors (src/NewHawkes.hpp:869-873)
    int curLoc = 0;
    HostBuf<double> hTimes;
    HostBuf<int32_t> hRanks;
    HostBuf<double> hOut;
    bool dirty = true;

    // device data
    DevBuf<double> dLoc, dTimes, dRecF64, dTileMin, dTileMax;
    DevBuf<float> dRecF32;
    DevBuf<int32_t> dRanks;
    // scratch
    DevBuf<double> dPartials, dBlockSums, dOut, dProbs;

    // plan (sweep shape); fixedR / fixedItems = 0 lets the autotuner choose
    int R = 2, itemsPerSM = 8;
    int fixedR = 0, fixedItems = 0;
    bool tuned = false;
    SweepGeometry geom{};

    // FP32 variant (bit 0: coordinate lo parts, bit 1: software exponential)
    int f32Variant = 1;
    // scales the FP32 records were last packed with (-1: not packed)
    double packedX = -1.0, packedT = -1.0;
    // FP32 exponential bias correction (see PairConsts::ex2Fix)
    float ex2Fix = 0.0f;
    double ex2Bias = 0.0;

    // optional kernel timing (CUDA events on the engine stream)
    bool kernelTiming = false;
    bool timedValid = false;
    cudaEvent_t evSweep0 = nullptr, evSweep1 = nullptr, evFinish1 = nullptr;

    // launch accounting of the last evaluation
    int lastLaunches = 0;
    PairConsts lastConsts{};

    int fail(int status, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        lastError = buf;
        return status;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        return fail(e == cudaErrorMemoryAllocation ? HPHC_ERR_OUT_OF_MEMORY : HPHC_ERR_CUDA,
                    "%s: %s", what, cudaGetErrorString(e));
    }

    // Geometry for R events per thread and `items` (strip, j-range) CTAs per
    // SM (several waves, so the hardware scheduler balances uneven items).
    SweepGeometry plan_for(int r, int items) const {
        SweepGeometry g{};
        const int stripEvents = kSweepThreads * r;
        g.N = N;
        g.nTiles = (N + kTile - 1) / kTile;
        g.nStrips = (N + stripEvents - 1) / stripEvents;
        g.Npad = g.nStrips * stripEvents;
        const int target = numSMs * items;
        int nChunks = std::max(1, (target + g.nStrips - 1) / g.nStrips);
        nChunks = std::min(nChunks, g.nTiles);
        g.chunkTiles = (g.nTiles + nChunks - 1) / nChunks;
        g.nChunks = (g.nTiles + g.chunkTiles - 1) / g.chunkTiles;
        return g;
    }

    int set_plan(int r, int items) {
        const SweepGeometry g = plan_for(r, items);
        cudaError_t e = dPartials.reserve((size_t)g.nChunks * kNumAcc * g.Npad);
        if (e != cudaSuccess) return cuda_fail(e, "device allocation");
        R = r;
        itemsPerSM = items;
        geom = g;
        return HPHC_OK;
    }

    int launch_sweep(const PairConsts& c) {
        cudaError_t e;
        if (precision == HPHC_PRECISION_FP64)
            e = launch_sweep_f64(D, R, geom, dRecF64.p, dTileMin.p, dTileMax.p, c, dPartials.p,
                                 stream);
        else
            e = launch_sweep_f32c(D, R, f32Variant, geom, dRecF32.p, dTileMin.p, dTileMax.p, c,
                                  dPartials.p, stream);
        if (e != cudaSuccess) return cuda_fail(e, "sweep kernel");
        return HPHC_OK;
    }

    // Autotuner: time every candidate shape on this engine's data (one warm
    // and one timed sweep each), keep the fastest, cache it per process.
    int autotune(const PairConsts& c) {
        const long key = tune_key();
        {
            std::lock_guard<std::mutex> lock(gTuneMutex);
            auto it = gTuneCache.find(key);
            if (it != gTuneCache.end()) {
                tuned = true;
                return set_plan(fixedR ? fixedR : it->second.first,
                                fixedItems ? fixedItems : it->second.second);
            }
        }
        std::vector<int> rs, its;
        if (fixedR) rs = {fixedR};
        else if (precision == HPHC_PRECISION_FP64) rs = {1, 2};
        else rs = {2, 4};
        if (fixedItems) its = {fixedItems};
        else its = {8, 16, 32, 64};
        float best = 1e30f;
        int bestR = rs[0], bestI = its[0];
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        int st = HPHC_OK;
        for (int r : rs) {
            for (int it : its) {
                if ((st = set_plan(r, it))) break;
                if ((st = launch_sweep(c))) break;  // warm
                cudaEventRecord(e0, stream);
                if ((st = launch_sweep(c))) break;
                cudaEventRecord(e1, stream);
                lastLaunches += 2;
                cudaError_t err = cudaEventSynchronize(e1);
                if (err != cudaSuccess) {
                    st = cuda_fail(err, "autotune");
                    break;
                }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) {
                    best = ms;
                    bestR = r;
                    bestI = it;
                }
            }
            if (st) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st) return st;
        {
            std::lock_guard<std::mutex> lock(gTuneMutex);
            gTuneCache[key] = {bestR, bestI};
        }
        tuned = true;
        return set_plan(bestR, bestI);
    }

    long tune_key() const {
        int lg = 0;
        while ((1 << lg) < N) ++lg;  // power-of-two size bucket
        return ((long)lg << 16) | ((long)D << 8) | ((long)precision << 4) | (long)f32Variant;
    }

    // Record scales of the FP32 path: x' = x sX, t' = t sT make the background
    // exponent (log2 units) -(|dx'|^2 + dt'^2).
    static double record_scale(double precisionParam) {
        return std::fabs(precisionParam) * std::sqrt(0.5 * kLog2e);
    }

    PairConsts pair_consts(const double* p) const {
        const double sigma = p[0], a = p[1], b = p[2], omega = p[3];
        PairConsts c{};
        c.cA = -0.5 * a * a;
        c.cB = -0.5 * b * b;
        c.cS = -0.5 * sigma * sigma;
        c.cW = -omega;
        if (precision != HPHC_PRECISION_FP64) {
            const double sT = record_scale(b);
            split_float(-(sigma * sigma) / (a * a), c.fSh, c.fSl);
            split_float(-omega * kLog2e / sT, c.fWh, c.fWl);
        }
        c.ex2Fix = (precision == HPHC_PRECISION_FP64 || (f32Variant & 2)) ? 0.0f : ex2Fix;
        const double thr = precision == HPHC_PRECISION_FP64 ? kSkipF64 : kSkipF32;
        c.skipB = (underflowSkip && c.cB < 0.0 && c.cA <= 0.0) ? thr : -1.0;
        c.skipS = (underflowSkip && c.cW < 0.0 && c.cS <= 0.0) ? thr : -1.0;
        return c;
    }

    FinishConsts finish_consts(const double* p) const {
        FinishConsts f{};
        f.sigma = p[0];
        f.a = p[1];
        f.b = p[2];
        f.omega = p[3];
        f.theta = p[4];
        f.mu0 = p[5];
        f.bgScale = std::pow(f.a, D) * f.b / kTwoPi;
        f.seScale = f.omega * std::pow(f.sigma, D) * kInvSqrt2Pi;
        f.prefB = f.mu0 * f.bgScale;
        f.prefS = f.theta * f.seScale;
        for (int q = 0; q < kNumAcc; ++q) f.accScale[q] = 1.0;
        if (precision != HPHC_PRECISION_FP64) {
            const double sX = record_scale(f.a), sT = record_scale(f.b);
            f.accScale[1] = f.accScale[4] = 1.0 / (sX * sX);  // sums of d'^2
            f.accScale[2] = 1.0 / (sT * sT);                  // sum of dt'^2
            f.accScale[5] = 1.0 / sT;                         // sum of dt'
        }
        f.T = hTimes.p[N - 1];
        // src/NewHawkes.hpp:659: locationCount * (embeddingDimension - 1) * log(M_1_SQRT_2PI)
        f.constant = (double)(N * (D - 1)) * std::log(kInvSqrt2Pi);
        f.D = D;
        return f;
    }

    int upload_if_dirty() {
        if (!dirty) return HPHC_OK;
        cudaError_t e;
        const size_t nl = (size_t)N * D;
        if ((e = cudaMemcpyAsync(dLoc.p, hLoc[curLoc].p, nl * sizeof(double),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return cuda_fail(e, "upload locations");
        if ((e = cudaMemcpyAsync(dTimes.p, hTimes.p, (size_t)N * sizeof(double),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return cuda_fail(e, "upload times");
        if (precision == HPHC_PRECISION_FP64) {
            e = launch_pack_f64(D, N, dLoc.p, dTimes.p, dRecF64.p, dTileMin.p, dTileMax.p, stream);
            lastLaunches += 2;
        } else {
            if ((e = cudaMemcpyAsync(dRanks.p, hRanks.p, (size_t)N * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, stream)) != cudaSuccess)
                return cuda_fail(e, "upload ranks");
            e = launch_tile_bounds(N, dTimes.p, dTileMin.p, dTileMax.p, stream);
            lastLaunches += 1;
            packedX = packedT = -1.0;  // records must be rebuilt
        }
        if (e != cudaSuccess) return cuda_fail(e, "pack kernel");
        dirty = false;
        return HPHC_OK;
    }

    // FP32 records are scaled by the current background precisions: rebuild
    // them when those change.
    int pack_f32_for(const double* p) {
        if (!(p[1] != 0.0 && p[2] != 0.0 && std::isfinite(p[1]) && std::isfinite(p[2])))
            return fail(HPHC_ERR_UNSUPPORTED,
                        "FP32-compensated mode needs finite non-zero tauXprec and tauTprec "
                        "(got %g, %g); use the FP64 mode", p[1], p[2]);
        const double sX = record_scale(p[1]), sT = record_scale(p[2]);
        if (sX == packedX && sT == packedT) return HPHC_OK;
        cudaError_t e = launch_pack_f32(D, N, dLoc.p, dTimes.p, dRanks.p, sX, sT, dRecF32.p, stream);
        if (e != cudaSuccess) return cuda_fail(e, "pack kernel");
        lastLaunches += 1;
        packedX = sX;
        packedT = sT;
        return HPHC_OK;
    }

    // Enqueue sweep + finish + final for parameter vector p; results land in
    // dOut[slot*8 .. slot*8+7] (and dProbs if wantProbs).
    int enqueue_eval(const double* p, int slot, bool wantProbs) {
        if (precision != HPHC_PRECISION_FP64) {
            const int st = pack_f32_for(p);
            if (st) return st;
        }
        const PairConsts c = pair_consts(p);
        const FinishConsts f = finish_consts(p);
        lastConsts = c;
        if (!tuned) {
            const int st = autotune(c);
            if (st) return st;
        }
        cudaError_t e;
        if (kernelTiming) cudaEventRecord(evSweep0, stream);
        if (const int st = launch_sweep(c)) return st;
        if (kernelTiming) cudaEventRecord(evSweep1, stream);
        e = launch_finish(geom, dPartials.p, dTimes.p, f, dBlockSums.p,
                          wantProbs ? dProbs.p : nullptr, stream);
        if (e != cudaSuccess) return cuda_fail(e, "finish kernel");
        e = launch_final(finish_blocks(N), dBlockSums.p, f, dOut.p + (size_t)slot * 8, stream);
        if (e != cudaSuccess) return cuda_fail(e, "final kernel");
        if (kernelTiming) cudaEventRecord(evFinish1, stream);
        timedValid = kernelTiming;
        lastLaunches += 3;
        return HPHC_OK;
    }

    int evaluate(const double* p, double* loglik, double* grad, double* probs) {
        DeviceGuard g(device);
        if (!g.ok) return fail(HPHC_ERR_CUDA, "cannot select device %d", device);
        lastLaunches = 0;
        int st = upload_if_dirty();
        if (st) return st;
        if ((st = enqueue_eval(p, 0, probs != nullptr))) return st;
        cudaError_t e = cudaMemcpyAsync(hOut.p, dOut.p, 8 * sizeof(double),
                                        cudaMemcpyDeviceToHost, stream);
        if (e != cudaSuccess) return cuda_fail(e, "read results");
        if (probs) {
            e = cudaMemcpyAsync(probs, dProbs.p, (size_t)N * sizeof(double),
                                cudaMemcpyDeviceToHost, stream);
            if (e != cudaSuccess) return cuda_fail(e, "read probabilities");
        }
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "evaluation");
        if (loglik) *loglik = hOut.p[0];
        if (grad)
            for (int k = 0; k < 6; ++k) grad[k] = hOut.p[1 + k];
        return HPHC_OK;
    }

    int init(int dim, int n, long fl, int dev) {
        D = dim;
        N = n;
        flags = fl;
        precision = (fl & (HPHC_FLAG_FLOAT | HPHC_FLAG_COMPENSATED)) ? HPHC_PRECISION_FP32_COMP
                                                                      : HPHC_PRECISION_FP64;
        underflowSkip = !(fl & HPHC_FLAG_NO_UNDERFLOW_SKIP);
        f32Variant = ((fl & HPHC_FLAG_FP32_SPACE_HILO) ? 1 : 0) | ((fl & HPHC_FLAG_FP32_FAST_EXP) ? 0 : 2);
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1)
            return fail(HPHC_ERR_NO_DEVICE, "no CUDA device visible");
        device = (dev < 0 || dev >= count) ? 0 : dev;
        DeviceGuard g(device);
        if (!g.ok) return fail(HPHC_ERR_CUDA, "cannot select device %d", device);
        cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device);
        cudaError_t e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e, "create stream");
        if ((e = cudaEventCreate(&evSweep0)) || (e = cudaEventCreate(&evSweep1)) ||
            (e = cudaEventCreate(&evFinish1)))
            return cuda_fail(e, "create events");
        if (precision != HPHC_PRECISION_FP64 && !(f32Variant & 2) &&
            (e = ex2_fix_for_device(device, stream, &ex2Fix, &ex2Bias)) != cudaSuccess)
            return cuda_fail(e, "exponential calibration");
        if (int st = set_plan(2, 8)) return st;
        const size_t nl = (size_t)N * D;
        if ((e = hLoc[0].reserve(nl)) || (e = hLoc[1].reserve(nl)) || (e = hTimes.reserve(N)) ||
            (e = hRanks.reserve(N)) || (e = hOut.reserve(8)))
            return cuda_fail(e, "pinned host allocation");
        std::memset(hLoc[0].p, 0, nl * sizeof(double));
        std::memset(hLoc[1].p, 0, nl * sizeof(double));
        std::memset(hTimes.p, 0, (size_t)N * sizeof(double));
        std::memset(hRanks.p, 0, (size_t)N * sizeof(int32_t));
        if ((e = dLoc.reserve(nl)) || (e = dTimes.reserve(N)) ||
            (e = dTileMin.reserve(geom.nTiles)) || (e = dTileMax.reserve(geom.nTiles)) ||
            (e = dBlockSums.reserve((size_t)finish_blocks(N) * 8)) || (e = dOut.reserve(8)) ||
            (e = dProbs.reserve(N)))
            return cuda_fail(e, "device allocation");
        if (precision == HPHC_PRECISION_FP64) {
            if ((e = dRecF64.reserve((size_t)N * 10))) return cuda_fail(e, "device allocation");
        } else {
            if ((e = dRecF32.reserve((size_t)N * 20)) || (e = dRanks.reserve(N)))
                return cuda_fail(e, "device allocation");
        }
        dirty = true;
        return HPHC_OK;
    }

    void destroy() {
        DeviceGuard g(device);
        if (stream) cudaStreamSynchronize(stream);
        hLoc[0].release();
        hLoc[1].release();
        hTimes.release();
        hRanks.release();
        hOut.release();
        dLoc.release();
        dTimes.release();
        dRecF64.release();
        dRecF32.release();
        dRanks.release();
        dTileMin.release();
        dTileMax.release();
        dPartials.release();
        dBlockSums.release();
        dOut.release();
        dProbs.release();
        if (evSweep0) cudaEventDestroy(evSweep0);
        if (evSweep1) cudaEventDestroy(evSweep1);
        if (evFinish1) cudaEventDestroy(evFinish1);
        evSweep0 = evSweep1 = evFinish1 = nullptr;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    // Dense rank of each time (equal times share a rank), for the exact
    // strict-causality mask of the FP32 records.
    void compute_ranks() {
        bool sorted = true;
        for (int i = 1; i < N && sorted; ++i) sorted = hTimes.p[i - 1] <= hTimes.p[i];
        if (sorted) {
            int r = 0;
            for (int i = 0; i < N; ++i) {
                if (i > 0 && hTimes.p[i] != hTimes.p[i - 1]) ++r;
                hRanks.p[i] = r;
            }
            return;
        }
        std::vector<int> idx(N);
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(),
                         [&](int x, int y) { return hTimes.p[x] < hTimes.p[y]; });
        int r = 0;
        for (int k = 0; k < N; ++k) {
            if (k > 0 && hTimes.p[idx[k]] != hTimes.p[idx[k - 1]]) ++r;
            hRanks.p[idx[k]] = r;
        }
    }

    // Host replay of the kernels' tile-pair decisions for launch accounting.
    void count_terms(double& bTerms, double& sTerms) const {
        const int nT = geom.nTiles;
        std::vector<double> tmin(nT, INFINITY), tmax(nT, -INFINITY);
        for (int j = 0; j < N; ++j) {
            const int t = j / kTile;
            tmin[t] = std::min(tmin[t], hTimes.p[j]);
            tmax[t] = std::max(tmax[t], hTimes.p[j]);
        }
        const PairConsts& c = lastConsts;
        const int stripEvents = kSweepThreads * R;
        double nb = 0.0, ns = 0.0;
        for (int s = 0; s < geom.nStrips; ++s) {
            double lo = INFINITY, hi = -INFINITY;
            for (int r = 0; r < R; ++r) {
                const int t = s * stripEvents / kTile + r;
                if (t < nT) {
                    lo = std::min(lo, tmin[t]);
                    hi = std::max(hi, tmax[t]);
                }
            }
            const double ni = std::min(stripEvents, N - s * stripEvents);
            for (int t = 0; t < nT; ++t) {
                const double nj = std::min(kTile, N - t * kTile);
                const double dtLo = lo - tmax[t], dtHi = hi - tmin[t];
                const double minAbs = dtLo > 0.0 ? dtLo : (dtHi < 0.0 ? -dtHi : 0.0);
                const bool doB = !(c.skipB >= 0.0 && -c.cB * minAbs * minAbs >= c.skipB);
                const bool allCausal = dtLo > 0.0;
                const bool doS =
                    dtHi > 0.0 && !(c.skipS >= 0.0 && allCausal && -c.cW * dtLo >= c.skipS);
                if (doB) nb += ni * nj;
                if (doS) ns += ni * nj;
            }
        }
        bTerms = nb;
        sTerms = ns;
    }
};

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
    for (size_t i = 0; i < length; ++i)
        if (!std::isfinite(data[i]))
            return e->fail(HPHC_ERR_NONFINITE, "times: entry %zu is not finite", i);
    std::memcpy(e->hTimes.p, data, length * sizeof(double));
    e->compute_ranks();
    e->dirty = true;
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
    for (size_t i = 0; i < length; ++i)
        if (!std::isfinite(location[i]))
            return e->fail(HPHC_ERR_NONFINITE, "locations: entry %zu is not finite", i);
    std::memcpy(e->hLoc[e->curLoc].p + offset, location, length * sizeof(double));
    e->dirty = true;
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
    return HPHC_OK;
}

int hphc_restore_state(hphc_engine* e) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    e->sumOfLikContribs = e->storedSumOfLikContribs;
    std::memcpy(e->params, e->storedParams, sizeof e->params);
    e->curLoc = 1 - e->curLoc;
    e->dirty = true;
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
    for (int k = 0; k < K; ++k) {
        const int st = e->evaluate(params + (size_t)6 * k, loglik + k,
                                   gradient ? gradient + (size_t)6 * k : nullptr, nullptr);
        if (st) return st;
    }
    return HPHC_OK;
}

int hphc_get_precision(hphc_engine* e, int* out) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!out) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    *out = e->precision;
    return HPHC_OK;
}

int hphc_get_stream(hphc_engine* e, void** stream) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!stream) return e->fail(HPHC_ERR_BAD_ARGUMENT, "null output");
    *stream = (void*)e->stream;
    return HPHC_OK;
}

int hphc_enqueue_log_likelihood_and_gradient(hphc_engine* e) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    DeviceGuard g(e->device);
    if (!g.ok) return e->fail(HPHC_ERR_CUDA, "cannot select device %d", e->device);
    e->lastLaunches = 0;
    int st = e->upload_if_dirty();
    if (st) return st;
    return e->enqueue_eval(e->params, 0, false);
}

int hphc_read_results(hphc_engine* e, double* loglik, double* gradient, size_t length) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (gradient && length != 6)
        return e->fail(HPHC_ERR_BAD_LENGTH, "gradient: length %zu != 6", length);
    DeviceGuard g(e->device);
    cudaError_t err = cudaMemcpyAsync(e->hOut.p, e->dOut.p, 8 * sizeof(double),
                                      cudaMemcpyDeviceToHost, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return e->cuda_fail(err, "read results");
    if (loglik) *loglik = e->hOut.p[0];
    if (gradient)
        for (int k = 0; k < 6; ++k) gradient[k] = e->hOut.p[1 + k];
    return HPHC_OK;
}

int hphc_get_last_launch_stats(hphc_engine* e, int* kernelLaunches, double* backgroundTerms,
                               double* selfExciteTerms) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (kernelLaunches) *kernelLaunches = e->lastLaunches;
    if (backgroundTerms || selfExciteTerms) {
        double nb = 0.0, ns = 0.0;
        e->count_terms(nb, ns);
        if (backgroundTerms) *backgroundTerms = nb;
        if (selfExciteTerms) *selfExciteTerms = ns;
    }
    return HPHC_OK;
}

int hphc_set_sweep_shape(hphc_engine* e, int eventsPerThread, int itemsPerSM) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    const bool fp64 = e->precision == HPHC_PRECISION_FP64;
    const bool okR = eventsPerThread == 0 ||
                     (fp64 ? (eventsPerThread == 1 || eventsPerThread == 2)
                           : (eventsPerThread == 2 || eventsPerThread == 4));
    if (!okR) return e->fail(HPHC_ERR_BAD_ARGUMENT, "events per thread %d not supported",
                             eventsPerThread);
    if (itemsPerSM < 0 || itemsPerSM > 1024)
        return e->fail(HPHC_ERR_BAD_ARGUMENT, "items per SM %d out of range", itemsPerSM);
    e->fixedR = eventsPerThread;
    e->fixedItems = itemsPerSM;
    e->tuned = false;
    if (eventsPerThread && itemsPerSM) {
        DeviceGuard g(e->device);
        e->tuned = true;
        return e->set_plan(eventsPerThread, itemsPerSM);
    }
    return HPHC_OK;
}

int hphc_get_sweep_shape(hphc_engine* e, int* eventsPerThread, int* itemsPerSM) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (eventsPerThread) *eventsPerThread = e->R;
    if (itemsPerSM) *itemsPerSM = e->itemsPerSM;
    return HPHC_OK;
}

int hphc_set_kernel_timing(hphc_engine* e, int enable) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    e->kernelTiming = enable != 0;
    return HPHC_OK;
}

int hphc_get_kernel_times(hphc_engine* e, float* sweepMs, float* finishMs) {
    if (!e) return HPHC_ERR_INVALID_HANDLE;
    if (!e->timedValid)
        return e->fail(HPHC_ERR_NOT_READY, "no evaluation with kernel timing enabled yet");
    DeviceGuard g(e->device);
    cudaError_t err = cudaEventSynchronize(e->evFinish1);
    if (err != cudaSuccess) return e->cuda_fail(err, "kernel timing");
    float a = 0.f, b = 0.f;
    if ((err = cudaEventElapsedTime(&a, e->evSweep0, e->evSweep1)) != cudaSuccess ||
        (err = cudaEventElapsedTime(&b, e->evSweep1, e->evFinish1)) != cudaSuccess)
        return e->cuda_fail(err, "kernel timing");
    if (sweepMs) *sweepMs = a;
    if (finishMs) *finishMs = b;
    return HPHC_OK;
}

}  // extern "C"
