// Multi-chain random-scan Metropolis-Hastings sampler over the Hawkes
// parameters: the caller of the likelihood in the reference's production path,
// the R function sampler() (R/Untitled.R:254-422), restated in C++ for K
// independent chains whose proposals are evaluated together, one batched
// likelihood run per iteration (hphc_batch_log_likelihood_and_gradient: one
// launch per stage for all K, replayed from a CUDA graph).
//
// Per chain and iteration, as in the reference loop (R/Untitled.R:318-414):
//   - pick one parameter index uniformly from the sampled set (the reference
//     samples sigma, omega, theta, mu0: sample(c(1,4:6)), :328);
//   - propose it from a normal truncated to (0, inf) centred on the current
//     value with that index's radius (truncnorm::rtruncnorm, :332);
//   - potential U = -logL - log prior, the prior being independent normals
//     truncated to (0, inf) with sd 10 for the first five parameters and sd 1
//     for mu0 (Potential, :225-231);
//   - accept when -(U' - log q(x | x')) + (U - log q(x' | x)) > log(u),
//     u ~ U(0, 1), q the truncated-normal proposal density (:336-354);
//   - adapt the index's radius every SampBound proposals of that index by the
//     acceptance ratio over 0.44, clamped to [0.5, 2], and grow SampBound to
//     ceil(SampBound^1.1) (:362-374);
//   - after burn-in, save the current parameters and potential (:377-380).
//
// The reference draws from R's generator; here each chain has its own
// splitmix64 stream (Steele, Lea and Flood 2014), seeded from the caller's
// seed and the chain index, so a run is reproducible and chains are
// independent.  Truncated-normal draws use Robert's (1995) rejection samplers:
// normal rejection when the truncation point is at or below the mean, the
// translated-exponential proposal otherwise.  Normal variates come from the
// Box-Muller transform (one variate per pair of uniforms).
//
// The likelihood is evaluated through a batched evaluator: the engine's batch
// entry point for hphc_sampler_run, or a caller-supplied function for
// hphc_sampler_run_with.  The sampler's own work is O(K) host arithmetic per
// iteration.
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "hphc.h"

namespace {

constexpr int kParams = 6;
constexpr double kLogSqrt2Pi = 0.918938533204672741780329736406;
constexpr double kSqrtHalf = 0.707106781186547524400844362105;
constexpr double kTwoPi = 6.28318530717958647692528676655900577;
constexpr double kTargetAcceptance = 0.44;  // R/Untitled.R:366

struct SplitMix64 {
    uint64_t state = 0;
    uint64_t next() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    // Uniform on (0, 1): 53 random bits, offset by half a step.
    double uniform() { return ((double)(next() >> 11) + 0.5) * 0x1.0p-53; }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(kTwoPi * u2);
    }
};

// Draw from N(mean, sd^2) truncated to [0, inf) (Robert 1995).
double truncated_normal(SplitMix64& g, double mean, double sd) {
    const double alpha = -mean / sd;  // standardised truncation point
    if (alpha <= 0.0) {
        for (;;) {
            const double z = g.normal();
            if (z >= alpha) return mean + sd * z;
        }
    }
    const double lambda = 0.5 * (alpha + std::sqrt(alpha * alpha + 4.0));
    for (;;) {
        const double z = alpha - std::log(g.uniform()) / lambda;
        const double d = z - lambda;
        if (g.uniform() <= std::exp(-0.5 * d * d)) return mean + sd * z;
    }
}

// log density of N(mean, sd^2) truncated to [0, inf) at x (truncnorm::dtruncnorm
// with a = 0: zero below the truncation point).
double log_truncated_normal(double x, double mean, double sd) {
    if (!(x >= 0.0)) return -INFINITY;
    const double z = (x - mean) / sd;
    const double alpha = -mean / sd;
    const double tail = 0.5 * std::erfc(alpha * kSqrtHalf);  // P(Z > alpha)
    return -0.5 * z * z - std::log(sd) - kLogSqrt2Pi - std::log(tail);
}

// Log prior of the reference's Potential (R/Untitled.R:226-227).
double log_prior(const double* p) {
    double s = 0.0;
    for (int k = 0; k < 5; ++k) s += log_truncated_normal(p[k], 0.0, 10.0);
    return s + log_truncated_normal(p[5], 0.0, 1.0);
}

struct Chain {
    double params[kParams];
    double potential = 0.0;
    double radii[kParams];
    int acceptances[kParams], sampBound[kParams], sampCount[kParams];
    long long accepted = 0, proposed = 0;
    SplitMix64 rng;
};

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

    template <typename Eval>
    int run(Eval&& eval, int iterations, int burnIn, double* samples, double* targets) {
        const int K = (int)chains.size();
        std::vector<double> prop((size_t)K * kParams), ll(K);
        if (!initialised) {
            for (int k = 0; k < K; ++k)
                for (int q = 0; q < kParams; ++q) prop[(size_t)k * kParams + q] = chains[k].params[q];
            const int st = eval(prop.data(), K, ll.data());
            if (st) return st;
            for (int k = 0; k < K; ++k)
                chains[k].potential = -ll[k] - log_prior(chains[k].params);
            initialised = true;
        }
        std::vector<int> index(K);
        std::vector<double> former(K);
        const int saved = iterations - burnIn;
        for (int it = 1; it <= iterations; ++it) {
            for (int k = 0; k < K; ++k) {
                Chain& c = chains[k];
                double* p = &prop[(size_t)k * kParams];
                for (int q = 0; q < kParams; ++q) p[q] = c.params[q];
                const int n = (int)sampled.size();
                int pick = (int)(c.rng.uniform() * n);
                if (pick >= n) pick = n - 1;
                const int idx = sampled[pick];
                index[k] = idx;
                former[k] = p[idx];
                p[idx] = truncated_normal(c.rng, former[k], c.radii[idx]);
            }
            const int st = eval(prop.data(), K, ll.data());
            if (st) return st;
            for (int k = 0; k < K; ++k) {
                Chain& c = chains[k];
                const double* p = &prop[(size_t)k * kParams];
                const int idx = index[k];
                const double r = c.radii[idx];
                const double propU = -ll[k] - log_prior(p);
                const double curH = c.potential - log_truncated_normal(p[idx], former[k], r);
                const double propH = propU - log_truncated_normal(former[k], p[idx], r);
                const double ratio = -propH + curH;
                const double logU = std::log(c.rng.uniform());
                ++c.proposed;
                if (ratio > logU) {  // a NaN ratio rejects
                    for (int q = 0; q < kParams; ++q) c.params[q] = p[q];
                    c.potential = propU;
                    ++c.accepted;
                    ++c.acceptances[idx];
                }
                if (++c.sampCount[idx] == c.sampBound[idx]) {
                    double adapt = (double)c.acceptances[idx] / c.sampBound[idx] /
                                   kTargetAcceptance;
                    adapt = std::fmin(2.0, std::fmax(0.5, adapt));
                    c.radii[idx] *= adapt;
                    c.sampCount[idx] = 0;
                    c.sampBound[idx] = (int)std::ceil(std::pow((double)c.sampBound[idx], 1.1));
                    c.acceptances[idx] = 0;
                }
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
    for (int k = 0; k < numChains; ++k) {
        Chain& c = s->chains[k];
        for (int q = 0; q < kParams; ++q) {
            c.params[q] = initialParams[(size_t)k * kParams + q];
            c.radii[q] = radius;   // Radii = rep(radius, 6)
            c.acceptances[q] = 0;  // Acceptances = rep(0, 6)
            c.sampBound[q] = 5;    // SampBound = rep(5, 6)
            c.sampCount[q] = 0;    // SampCount = rep(0, 6)
        }
        c.rng.state = (uint64_t)seed ^ (0x632BE59BD9B4E019ULL * (uint64_t)(k + 1));
    }
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
