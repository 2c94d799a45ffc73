// hphc_loglik_grad_fp64_static: log-likelihood and gradient without any
// device or host allocation.
//
// Who needs it: callers that must not allocate GPU memory while they run --
// code inside a host framework that owns all device memory through its own
// pool (a cudaMalloc behind its back breaks its accounting or fails under its
// memory cap), real-time or embedded loops where an allocation's implicit
// device synchronisation and latency are not acceptable, and processes whose
// GPU memory is pinned down to a fixed budget at start-up.  They hand in
// device-resident inputs and an output buffer and get the FP64 result.
//
// How: every intermediate (packed event records, tile time bounds, per-chunk
// pair sums, per-CTA sums) lives in one file-scope static __device__ array of
// kStaticScratchBytes (16 MiB).  A CUDA module's static device memory is
// allocated when the module is loaded on a device and held until the process
// exits, on every GPU that loads this library.  In host code the array's name
// is only a host-side stand-in, so its device address is looked up once per
// device with cudaGetSymbolAddress (with that device current) and passed to
// the kernels.  That lookup happens in the first call on each device, which
// is why the first call should come before any stream capture.  A device
// whose context was destroyed (cudaDeviceReset) gets a new context and a
// new copy of the array on its next use, so the address is cached together
// with the context's unique id and looked up again when that id changes.
//
// Device inputs are used as given: they are not checked for non-finite
// values or for ordering (times need not be sorted; T is t[N-1], as in the
// reference).  A NaN or infinity in them gives a non-finite result.
//
// Sharing: all calls in the process use the same array.  Every scratch word a
// call reads is written earlier in the same call, so nothing has to start at
// zero; but two calls whose work overlaps on the GPU (different streams,
// different host threads) race on the array and corrupt each other's results.
// Serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "hphc.h"
#include "hphc_kernels.cuh"

using namespace hphc;

namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;
constexpr size_t kScratchDoubles = kStaticScratchBytes / sizeof(double);
constexpr int kStaticR = 2;        // target events per thread (FP64 sweep)
constexpr int kStaticItemsPerSM = 16;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_hphc_static_scratch[kScratchDoubles];

std::mutex gScratchMutex;
double* gScratchAddress[kMaxDevices] = {};
unsigned long long gScratchContext[kMaxDevices] = {};

// Unique id of the current context (cuCtxGetCurrent + cuCtxGetId through the
// runtime's driver entry points, so the library needs no link against the
// driver library); 0 if it cannot be read.  Called with gScratchMutex held.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent getCurrent = nullptr;
    static GetId getId = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getCurrent = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getId = reinterpret_cast<GetId>(f);
    }
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!getCurrent || !getId || getCurrent(&ctx) != 0 || !ctx || getId(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the static scratch on the current device: looked up on
// the first call on the device, and again after its context was recreated.
cudaError_t static_scratch_address(int device, double** out) {
    std::lock_guard<std::mutex> lock(gScratchMutex);
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    const unsigned long long ctx = current_context_id();
    if (!gScratchAddress[device] || ctx == 0 || ctx != gScratchContext[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_hphc_static_scratch);
        if (e != cudaSuccess) return e;
        gScratchAddress[device] = static_cast<double*>(p);
        gScratchContext[device] = ctx;
    }
    *out = gScratchAddress[device];
    return cudaSuccess;
}

size_t round_up_256(size_t doubles) { return (doubles + 31) / 32 * 32; }  // 256-byte multiples

struct StaticPlan {
    SweepGeometry g;
    size_t rec, tmin, tmax, partials, blocks, total;  // offsets / size in doubles
};

// Same sweep geometry rules as the engine's planner, with the chunk count
// reduced until the scratch fits.
bool static_plan(int D, int N, int numSMs, StaticPlan* p) {
    const int stride = D <= 1 ? Layout<1>::kF64Stride
                     : D == 2 ? Layout<2>::kF64Stride
                     : D == 3 ? Layout<3>::kF64Stride
                     : D == 4 ? Layout<4>::kF64Stride
                     : D == 5 ? Layout<5>::kF64Stride
                     : D == 6 ? Layout<6>::kF64Stride
                     : D == 7 ? Layout<7>::kF64Stride
                              : Layout<8>::kF64Stride;
    SweepGeometry g{};
    const int stripEvents = kSweepThreads * kStaticR;
    g.N = N;
    g.nTiles = (N + kTile - 1) / kTile;
    g.nStrips = (N + stripEvents - 1) / stripEvents;
    g.Npad = g.nStrips * stripEvents;
    int nChunks = std::max(1, (numSMs * kStaticItemsPerSM + g.nStrips - 1) / g.nStrips);
    nChunks = std::min(nChunks, g.nTiles);
    for (;;) {
        g.chunkTiles = (g.nTiles + nChunks - 1) / nChunks;
        g.nChunks = (g.nTiles + g.chunkTiles - 1) / g.chunkTiles;
        p->rec = 0;
        p->tmin = p->rec + round_up_256((size_t)N * stride);
        p->tmax = p->tmin + round_up_256(g.nTiles);
        p->partials = p->tmax + round_up_256(g.nTiles);
        p->blocks = p->partials + round_up_256((size_t)g.nChunks * kNumAcc * g.Npad);
        p->total = p->blocks + round_up_256((size_t)finish_blocks(N) * 8);
        if (p->total <= kScratchDoubles) {
            p->g = g;
            return true;
        }
        if (nChunks == 1) return false;
        nChunks = std::max(1, nChunks / 2);
    }
}

bool is_device_pointer(const void* ptr, int device) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();  // the query's error is not sticky; clear it
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) &&
           a.device == device;
}

}  // namespace

extern "C" int hphc_loglik_grad_fp64_static(int embeddingDimension, int locationCount,
                                            const double* deviceLocations,
                                            const double* deviceTimes, const double* params,
                                            double* deviceOut, void* stream) {
    const int D = embeddingDimension, N = locationCount;
    if (D < 1 || D > kMaxDim) return HPHC_ERR_UNSUPPORTED;
    if (N < 1 || !deviceLocations || !deviceTimes || !params || !deviceOut)
        return HPHC_ERR_BAD_ARGUMENT;
    for (int k = 0; k < 6; ++k)
        if (!std::isfinite(params[k])) return HPHC_ERR_NONFINITE;

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return HPHC_ERR_NO_DEVICE;
    int numSMs = 0;
    if (cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return HPHC_ERR_CUDA;
    StaticPlan plan{};
    if (!static_plan(D, N, numSMs, &plan)) return HPHC_ERR_SCRATCH_TOO_SMALL;
    if (!is_device_pointer(deviceLocations, device) || !is_device_pointer(deviceTimes, device) ||
        !is_device_pointer(deviceOut, device))
        return HPHC_ERR_BAD_ARGUMENT;

    double* scratch = nullptr;
    if (static_scratch_address(device, &scratch) != cudaSuccess) return HPHC_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // T = t[N-1] (src/NewHawkes.hpp:653) is needed by the finish constants.
    double T = 0.0;
    if (cudaMemcpyAsync(&T, deviceTimes + (N - 1), sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return HPHC_ERR_CUDA;

    // The same constants as the engine's FP64 mode (hphc::param_consts),
    // with the tile-level underflow skip only: no tail truncation, no far
    // tail on the hardware exponential.
    ConstsSpec spec{};
    spec.precision = 0;
    spec.D = D;
    spec.variant = 0;
    spec.skip = 1;
    spec.truncate = 0;
    spec.ex2Bias = 0.0;
    spec.fastTail = 0;
    spec.noB = 0;
    PairConsts c{};
    FinishConsts f{};
    param_consts(params, spec, c, f);
    const double kInvSqrt2Pi = 0.398942280401432677939946059934;
    f.T = T;
    f.constant = (double)(N * (D - 1)) * std::log(kInvSqrt2Pi);

    double* rec = scratch + plan.rec;
    double* tmin = scratch + plan.tmin;
    double* tmax = scratch + plan.tmax;
    double* partials = scratch + plan.partials;
    double* blockSums = scratch + plan.blocks;
    if (launch_pack_f64(D, N, deviceLocations, deviceTimes, rec, tmin, tmax, s) != cudaSuccess ||
        launch_sweep_f64(D, kStaticR, plan.g, rec, tmin, tmax, c, partials, s) != cudaSuccess ||
        launch_finish(plan.g, partials, deviceTimes, f, blockSums, nullptr, s) != cudaSuccess ||
        launch_final(finish_blocks(N), blockSums, f, deviceOut, s) != cudaSuccess)
        return HPHC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HPHC_ERR_CUDA;
    return HPHC_OK;
}
