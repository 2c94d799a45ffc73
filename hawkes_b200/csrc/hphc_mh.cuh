// One chain of the random-scan Metropolis-Hastings sampler, written once for
// the host driver and the device-resident driver (hphc_sampler.cu).
//
// It restates the reference's R sampler() loop (R/Untitled.R:318-414):
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
//     ceil(SampBound^1.1) (:362-374).
//
// The reference draws from R's generator; here each chain has its own
// splitmix64 stream (Steele, Lea and Flood 2014).  Truncated-normal draws use
// Robert's (1995) rejection samplers: normal rejection when the truncation
// point is at or below the mean, the translated-exponential proposal
// otherwise.  Normal variates come from the Box-Muller transform (one
// variate per pair of uniforms).
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define HPHC_HD __host__ __device__
#else
#define HPHC_HD
#endif

namespace hphc {
namespace mh {

constexpr int kParams = 6;
constexpr double kLogSqrt2Pi = 0.918938533204672741780329736406;
constexpr double kSqrtHalf = 0.707106781186547524400844362105;
constexpr double kTwoPi = 6.28318530717958647692528676655900577;
constexpr double kTargetAcceptance = 0.44;  // R/Untitled.R:366
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;
constexpr uint64_t kChainSeedMix = 0x632BE59BD9B4E019ULL;

struct Rng {
    uint64_t state;
    HPHC_HD uint64_t next() {
        uint64_t z = (state += kGolden);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    // Uniform on (0, 1): 53 random bits, offset by half a step.
    HPHC_HD double uniform() { return ((double)(next() >> 11) + 0.5) * 0x1.0p-53; }
    HPHC_HD double normal() {
        const double u1 = uniform(), u2 = uniform();
        return sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
    }
};

// Initial generator state of chain k.
HPHC_HD inline uint64_t chain_seed(uint64_t seed, int k) {
    return seed ^ (kChainSeedMix * (uint64_t)(k + 1));
}

// Draw from N(mean, sd^2) truncated to [0, inf).
HPHC_HD inline double truncated_normal(Rng& g, double mean, double sd) {
    const double alpha = -mean / sd;  // standardised truncation point
    if (alpha <= 0.0) {
        for (;;) {
            const double z = g.normal();
            if (z >= alpha) return mean + sd * z;
        }
    }
    const double lambda = 0.5 * (alpha + sqrt(alpha * alpha + 4.0));
    for (;;) {
        const double z = alpha - log(g.uniform()) / lambda;
        const double d = z - lambda;
        if (g.uniform() <= exp(-0.5 * d * d)) return mean + sd * z;
    }
}

// log density of N(mean, sd^2) truncated to [0, inf) at x (truncnorm::dtruncnorm
// with a = 0: zero below the truncation point).
HPHC_HD inline double log_truncated_normal(double x, double mean, double sd) {
    if (!(x >= 0.0)) return -INFINITY;
    const double z = (x - mean) / sd;
    const double alpha = -mean / sd;
    const double tail = 0.5 * erfc(alpha * kSqrtHalf);  // P(Z > alpha)
    return -0.5 * z * z - log(sd) - kLogSqrt2Pi - log(tail);
}

// Log prior of the reference's Potential (R/Untitled.R:226-227).
HPHC_HD inline double log_prior(const double* p) {
    double s = 0.0;
    for (int k = 0; k < 5; ++k) s += log_truncated_normal(p[k], 0.0, 10.0);
    return s + log_truncated_normal(p[5], 0.0, 1.0);
}

struct Chain {
    double params[kParams];
    double potential;
    double radii[kParams];
    int acceptances[kParams], sampBound[kParams], sampCount[kParams];
    long long accepted, proposed;
    Rng rng;
    int index;      // parameter proposed in the current iteration
    double former;  // its value before the proposal
};

// The reference's initial state (R/Untitled.R:300-307) for chain k.
HPHC_HD inline void init_chain(Chain& c, const double* params, double radius, uint64_t seed,
                               int k) {
    for (int q = 0; q < kParams; ++q) {
        c.params[q] = params[q];
        c.radii[q] = radius;   // Radii = rep(radius, 6)
        c.acceptances[q] = 0;  // Acceptances = rep(0, 6)
        c.sampBound[q] = 5;    // SampBound = rep(5, 6)
        c.sampCount[q] = 0;    // SampCount = rep(0, 6)
    }
    c.potential = 0.0;
    c.accepted = c.proposed = 0;
    c.rng.state = chain_seed(seed, k);
    c.index = 0;
    c.former = 0.0;
}

// Proposal of one iteration: prop = the chain's parameters with one sampled
// index redrawn.
HPHC_HD inline void propose(Chain& c, const int* sampled, int nSampled, double* prop) {
    for (int q = 0; q < kParams; ++q) prop[q] = c.params[q];
    int pick = (int)(c.rng.uniform() * nSampled);
    if (pick >= nSampled) pick = nSampled - 1;
    const int idx = sampled[pick];
    c.index = idx;
    c.former = prop[idx];
    prop[idx] = truncated_normal(c.rng, c.former, c.radii[idx]);
}

// Accept or reject the proposal given its log-likelihood, then adapt.
HPHC_HD inline void accept(Chain& c, const double* prop, double loglik) {
    const int idx = c.index;
    const double r = c.radii[idx];
    const double propU = -loglik - log_prior(prop);
    const double curH = c.potential - log_truncated_normal(prop[idx], c.former, r);
    const double propH = propU - log_truncated_normal(c.former, prop[idx], r);
    const double ratio = -propH + curH;
    const double logU = log(c.rng.uniform());
    ++c.proposed;
    if (ratio > logU) {  // a NaN ratio rejects
        for (int q = 0; q < kParams; ++q) c.params[q] = prop[q];
        c.potential = propU;
        ++c.accepted;
        ++c.acceptances[idx];
    }
    if (++c.sampCount[idx] == c.sampBound[idx]) {
        double adapt = (double)c.acceptances[idx] / c.sampBound[idx] / kTargetAcceptance;
        adapt = fmin(2.0, fmax(0.5, adapt));
        c.radii[idx] *= adapt;
        c.sampCount[idx] = 0;
        c.sampBound[idx] = (int)ceil(pow((double)c.sampBound[idx], 1.1));
        c.acceptances[idx] = 0;
    }
}

}  // namespace mh
}  // namespace hphc
