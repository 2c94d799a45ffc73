// Multi-chain random-scan Metropolis-Hastings sampler over the Hawkes
// parameters: the caller of the likelihood in the reference's production path,
// the R function sampler() (R/Untitled.R:254-422), for K independent chains
// whose proposals are evaluated together.  The chain step (proposal,
// truncated-normal densities, prior, acceptance, radius adaptation) is
// hphc_mh.cuh, shared by the two drivers here:
//
//   host driver    hphc_sampler_run / hphc_sampler_run_with: each iteration
//                  proposes on the host, evaluates the K proposals in one
//                  batched likelihood run (hphc_batch_log_likelihood_and_
//                  gradient: one launch per stage for all K, replayed from a
//                  CUDA graph) or by a caller-supplied evaluator, and accepts
//                  on the host;
//   device driver  hphc_sampler_run_device: the chains live in device memory
//                  and one iteration -- a proposal kernel that also rewrites
//                  each problem's parameter constants in the engine's device
//                  tables, the pair sweep, finish and final kernels, and an
//                  acceptance kernel -- is captured once into a CUDA graph and
//                  replayed for every iteration, with no host work or
//                  transfer in between.
//
// Both drivers draw the same random numbers (one splitmix64 stream per chain)
// and evaluate with the same kernels; their chains differ only where the host
// and device math libraries round log, cos, erfc, exp or pow differently in
// the last bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <new>
#include <string>
#include <vector>

#include "hphc.h"
#include "hphc_internal.h"
#include "hphc_mh.cuh"

using hphc::mh::Chain;
using hphc::mh::kParams;

namespace {

// Parameter indices proposed from, by value for the device kernels.
struct SampledSet {
    int idx[kParams];
    int n;
};

constexpr int kChainThreads = 128;

// Proposal of every chain; the problem k constants in the engine's device
// tables are rewritten for the proposal (the fields that depend on the event
// set only, T and constant, are kept).  Thread 0 also advances the
// iteration counter.
__global__ void __launch_bounds__(kChainThreads)
mh_propose_kernel(Chain* __restrict__ chains, int K, SampledSet sampled,
                  double* __restrict__ prop, hphc::SweepProblem* __restrict__ sp,
                  hphc::FinishProblem* __restrict__ fp, hphc::ConstsSpec spec,
                  int* __restrict__ iteration) {
    const int k = blockIdx.x * kChainThreads + threadIdx.x;
    if (k == 0) ++*iteration;
    if (k >= K) return;
    double* p = prop + (size_t)k * kParams;
    hphc::mh::propose(chains[k], sampled.idx, sampled.n, p);
    hphc::PairConsts c = sp[k].c;
    hphc::FinishConsts f = fp[k].f;
    hphc::param_consts(p, spec, c, f);
    sp[k].c = c;
    fp[k].f = f;
}

// Acceptance of every chain from its proposal's log-likelihood (results:
// K x 8, [0] = log-likelihood) and, after burn-in, the chain's state into
// samples (K x saved x 6) and targets (K x saved).
__global__ void __launch_bounds__(kChainThreads)
mh_accept_kernel(Chain* __restrict__ chains, int K, const double* __restrict__ prop,
                 const double* __restrict__ results, const int* __restrict__ iteration,
                 int burnIn, int saved, double* __restrict__ samples,
                 double* __restrict__ targets) {
    const int k = blockIdx.x * kChainThreads + threadIdx.x;
    if (k >= K) return;
    Chain& c = chains[k];
    hphc::mh::accept(c, prop + (size_t)k * kParams, results[(size_t)8 * k]);
    const int it = *iteration;  // 1-based, advanced by this iteration's proposal kernel
    if (it > burnIn && it - burnIn <= saved) {
        const size_t s = (size_t)k * saved + (it - burnIn - 1);
        for (int q = 0; q < kParams; ++q) samples[s * kParams + q] = c.params[q];
        targets[s] = c.potential;
    }
}

}  // namespace

struct hphc_sampler {
    std::vector<Chain> chains;
    std::vector<int> sampled;  // parameter indices proposed from
    bool initialised = false;  // potentials of the current parameters known
    std::string lastError;

    int fail(int status, const char* f, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, f);
        vsnprintf(buf, sizeof buf, f, ap);
        va_end(ap);
        lastError = buf;
        return status;
    }

    std::vector<double> current_params() const {
        std::vector<double> p(chains.size() * kParams);
        for (size_t k = 0; k < chains.size(); ++k)
            for (int q = 0; q < kParams; ++q) p[k * kParams + q] = chains[k].params[q];
        return p;
    }

    // Potentials of the current parameters (one batched evaluation).
    template <typename Eval>
    int initialise(Eval&& eval) {
        if (initialised) return HPHC_OK;
        const int K = (int)chains.size();
        std::vector<double> p = current_params(), ll(K);
        const int st = eval(p.data(), K, ll.data());
        if (st) return st;
        for (int k = 0; k < K; ++k)
            chains[k].potential = -ll[k] - hphc::mh::log_prior(chains[k].params);
        initialised = true;
        return HPHC_OK;
    }

    template <typename Eval>
    int run(Eval&& eval, int iterations, int burnIn, double* samples, double* targets) {
        const int K = (int)chains.size();
        int st = initialise(eval);
        if (st) return st;
        std::vector<double> prop((size_t)K * kParams), ll(K);
        const int saved = iterations - burnIn;
        for (int it = 1; it <= iterations; ++it) {
            for (int k = 0; k < K; ++k)
                hphc::mh::propose(chains[k], sampled.data(), (int)sampled.size(),
                                  &prop[(size_t)k * kParams]);
            if ((st = eval(prop.data(), K, ll.data()))) return st;
            for (int k = 0; k < K; ++k) {
                Chain& c = chains[k];
                hphc::mh::accept(c, &prop[(size_t)k * kParams], ll[k]);
                if (it > burnIn) {
                    const size_t s = (size_t)k * saved + (it - burnIn - 1);
                    if (samples)
                        for (int q = 0; q < kParams; ++q) samples[s * kParams + q] = c.params[q];
                    if (targets) targets[s] = c.potential;
                }
            }
        }
        return HPHC_OK;
    }
};

namespace {

// Device buffers of one device run, released on every path.
struct DeviceRun {
    Chain* chains = nullptr;
    double* prop = nullptr;
    double* samples = nullptr;
    double* targets = nullptr;
    int* iteration = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~DeviceRun() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaFree(chains);
        cudaFree(prop);
        cudaFree(samples);
        cudaFree(targets);
        cudaFree(iteration);
    }
};

}  // namespace

extern "C" {

int hphc_sampler_create(int numChains, const double* initialParams, double radius,
                        int sampledMask, unsigned long long seed, hphc_sampler** out) {
    if (!out) return HPHC_ERR_BAD_ARGUMENT;
    *out = nullptr;
    if (numChains < 1 || !initialParams || !(radius > 0.0) || !std::isfinite(radius))
        return HPHC_ERR_BAD_ARGUMENT;
    if (sampledMask == 0) sampledMask = (1 << 0) | (1 << 3) | (1 << 4) | (1 << 5);
    if (sampledMask < 0 || sampledMask >= (1 << kParams)) return HPHC_ERR_BAD_ARGUMENT;
    for (int i = 0; i < numChains * kParams; ++i)
        if (!(initialParams[i] >= 0.0) || !std::isfinite(initialParams[i]))
            return HPHC_ERR_BAD_ARGUMENT;
    auto* s = new (std::nothrow) hphc_sampler();
    if (!s) return HPHC_ERR_OUT_OF_MEMORY;
    for (int q = 0; q < kParams; ++q)
        if (sampledMask & (1 << q)) s->sampled.push_back(q);
    s->chains.resize(numChains);
    for (int k = 0; k < numChains; ++k)
        hphc::mh::init_chain(s->chains[k], initialParams + (size_t)k * kParams, radius, seed, k);
    *out = s;
    return HPHC_OK;
}

void hphc_sampler_destroy(hphc_sampler* s) { delete s; }

const char* hphc_sampler_last_error(const hphc_sampler* s) {
    return s ? s->lastError.c_str() : "invalid handle";
}

int hphc_sampler_run(hphc_sampler* s, hphc_engine* engine, int iterations, int burnIn,
                     double* samples, double* targets) {
    if (!s) return HPHC_ERR_INVALID_HANDLE;
    if (!engine) return s->fail(HPHC_ERR_INVALID_HANDLE, "null engine");
    if (iterations < 0 || burnIn < 0 || burnIn > iterations)
        return s->fail(HPHC_ERR_BAD_ARGUMENT, "iterations %d, burnIn %d", iterations, burnIn);
    hphc::NvtxRange range("hphc sampler run (host driver)");
    auto eval = [&](const double* p, int K, double* ll) -> int {
        const int st = hphc_batch_log_likelihood_and_gradient(engine, p, K, ll, nullptr);
        if (st) s->fail(st, "likelihood evaluation: %s", hphc_last_error(engine));
        return st;
    };
    return s->run(eval, iterations, burnIn, samples, targets);
}

int hphc_sampler_run_with(hphc_sampler* s, hphc_batch_loglik_fn fn, void* user, int iterations,
                          int burnIn, double* samples, double* targets) {
    if (!s) return HPHC_ERR_INVALID_HANDLE;
    if (!fn) return s->fail(HPHC_ERR_BAD_ARGUMENT, "null evaluator");
    if (iterations < 0 || burnIn < 0 || burnIn > iterations)
        return s->fail(HPHC_ERR_BAD_ARGUMENT, "iterations %d, burnIn %d", iterations, burnIn);
    auto eval = [&](const double* p, int K, double* ll) -> int {
        const int st = fn(user, p, K, ll);
        if (st) s->fail(st, "likelihood evaluation returned %d", st);
        return st;
    };
    return s->run(eval, iterations, burnIn, samples, targets);
}

int hphc_sampler_run_device(hphc_sampler* s, hphc_engine* engine, int iterations, int burnIn,
                            double* samples, double* targets) {
    if (!s) return HPHC_ERR_INVALID_HANDLE;
    if (!engine) return s->fail(HPHC_ERR_INVALID_HANDLE, "null engine");
    if (iterations < 0 || burnIn < 0 || burnIn > iterations)
        return s->fail(HPHC_ERR_BAD_ARGUMENT, "iterations %d, burnIn %d", iterations, burnIn);
    for (int q : s->sampled)
        if (q == 1 || q == 2)
            return s->fail(HPHC_ERR_UNSUPPORTED,
                           "the device driver keeps tauXprec and tauTprec fixed (they set the "
                           "record scaling and the work list); use hphc_sampler_run");
    hphc::NvtxRange range("hphc sampler run (device driver)");
    auto eval = [&](const double* p, int K, double* ll) -> int {
        const int st = hphc_batch_log_likelihood_and_gradient(engine, p, K, ll, nullptr);
        if (st) s->fail(st, "likelihood evaluation: %s", hphc_last_error(engine));
        return st;
    };
    int st = s->initialise(eval);
    if (st) return st;
    if (iterations == 0) return HPHC_OK;

    const int K = (int)s->chains.size();
    const int saved = iterations - burnIn;
    hphc::EngineLoop loop;
    std::string err;
    const std::vector<double> params = s->current_params();
    if ((st = hphc::engine_loop_setup(engine, params.data(), K, &loop, &err)))
        return s->fail(st, "device loop set-up: %s", err.c_str());
    int prevDevice = -1;
    cudaGetDevice(&prevDevice);
    if (prevDevice != loop.device) cudaSetDevice(loop.device);
    struct Restore {
        int dev;
        ~Restore() {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prevDevice};

    SampledSet sampled{};
    sampled.n = (int)s->sampled.size();
    for (int i = 0; i < sampled.n; ++i) sampled.idx[i] = s->sampled[i];

    DeviceRun run;
    cudaError_t e;
    auto cuda_fail = [&](const char* what) {
        return s->fail(e == cudaErrorMemoryAllocation ? HPHC_ERR_OUT_OF_MEMORY : HPHC_ERR_CUDA,
                       "%s: %s", what, cudaGetErrorString(e));
    };
    const size_t nSaved = (size_t)K * (size_t)(saved > 0 ? saved : 1);
    if ((e = cudaMalloc(&run.chains, sizeof(Chain) * K)) ||
        (e = cudaMalloc(&run.prop, sizeof(double) * kParams * K)) ||
        (e = cudaMalloc(&run.samples, sizeof(double) * kParams * nSaved)) ||
        (e = cudaMalloc(&run.targets, sizeof(double) * nSaved)) ||
        (e = cudaMalloc(&run.iteration, sizeof(int))))
        return cuda_fail("device allocation");
    cudaStream_t stream = loop.stream;
    if ((e = cudaMemcpyAsync(run.chains, s->chains.data(), sizeof(Chain) * K,
                             cudaMemcpyHostToDevice, stream)) ||
        (e = cudaMemsetAsync(run.iteration, 0, sizeof(int), stream)))
        return cuda_fail("upload chains");

    // one iteration, captured once
    const int blocks = (K + kChainThreads - 1) / kChainThreads;
    if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)))
        return cuda_fail("begin graph capture");
    mh_propose_kernel<<<blocks, kChainThreads, 0, stream>>>(
        run.chains, K, sampled, run.prop, loop.ex->device_sweep_problems(),
        loop.ex->device_finish_problems(), loop.spec, run.iteration);
    st = loop.ex->enqueue_device_body();
    mh_accept_kernel<<<blocks, kChainThreads, 0, stream>>>(
        run.chains, K, run.prop, loop.ex->device_results(), run.iteration, burnIn, saved,
        run.samples, run.targets);
    cudaError_t launchErr = cudaGetLastError();
    e = cudaStreamEndCapture(stream, &run.graph);
    if (st) return s->fail(st, "device loop: %s", loop.ex->error.c_str());
    if (e == cudaSuccess) e = launchErr;
    if (e != cudaSuccess) return cuda_fail("capture iteration");
    if ((e = cudaGraphInstantiate(&run.exec, run.graph, 0))) return cuda_fail("instantiate graph");
    for (int it = 0; it < iterations; ++it)
        if ((e = cudaGraphLaunch(run.exec, stream))) return cuda_fail("launch iteration");

    std::vector<Chain> back(K);
    if ((e = cudaMemcpyAsync(back.data(), run.chains, sizeof(Chain) * K, cudaMemcpyDeviceToHost,
                             stream)))
        return cuda_fail("read chains");
    if (saved > 0 && samples &&
        (e = cudaMemcpyAsync(samples, run.samples, sizeof(double) * kParams * nSaved,
                             cudaMemcpyDeviceToHost, stream)))
        return cuda_fail("read samples");
    if (saved > 0 && targets &&
        (e = cudaMemcpyAsync(targets, run.targets, sizeof(double) * nSaved,
                             cudaMemcpyDeviceToHost, stream)))
        return cuda_fail("read targets");
    if ((e = cudaStreamSynchronize(stream))) return cuda_fail("device iterations");
    s->chains = back;
    return HPHC_OK;
}

int hphc_sampler_get_state(const hphc_sampler* s, double* params, double* potential,
                           double* radii, long long* accepted, long long* proposed) {
    if (!s) return HPHC_ERR_INVALID_HANDLE;
    const int K = (int)s->chains.size();
    for (int k = 0; k < K; ++k) {
        const Chain& c = s->chains[k];
        for (int q = 0; q < kParams; ++q) {
            if (params) params[(size_t)k * kParams + q] = c.params[q];
            if (radii) radii[(size_t)k * kParams + q] = c.radii[q];
        }
        if (potential) potential[k] = s->initialised ? c.potential : NAN;
        if (accepted) accepted[k] = c.accepted;
        if (proposed) proposed[k] = c.proposed;
    }
    return HPHC_OK;
}

}  // extern "C"
