// Kernels of the B200 Hawkes likelihood engine other than the pair sweeps:
// record packing, tile time bounds, dense time ranks, the strip row order,
// the per-event finish and fixed-order totals, the exponential calibration
// and the incremental single-event updates, plus the launchers that dispatch
// the pair sweeps (hphc_sweep.cuh) by embedding dimension to the
// hphc_sweep_d<D>.cu compilation units.
#include <limits.h>
#include <math.h>

#include "hphc_kernels.cuh"
#include "hphc_sweep.cuh"

namespace hphc {
namespace {

constexpr double kInvSqrt2Pi = 0.398942280401432677939946059934;
constexpr double kSqrtHalf = 0.707106781186547524400844362105;


// ---------------------------------------------------------------- packing --

template <int D>
__global__ void pack_f64_kernel(int N, const double* __restrict__ loc,
                                const double* __restrict__ times, double* __restrict__ rec) {
    constexpr int S = Layout<D>::kF64Stride;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double* r = rec + (size_t)i * S;
#pragma unroll
    for (int k = 0; k < D; ++k) r[k] = loc[(size_t)i * D + k];
    r[D] = times[i];
#pragma unroll
    for (int k = D + 1; k < S; ++k) r[k] = 0.0;
}

// FP32 records for many problems in one launch: blockIdx.y = job.
template <int D>
__global__ void pack_f32_jobs_kernel(const PackJob* __restrict__ jobs) {
    constexpr int S = Layout<D>::kF32Stride;
    const PackJob J = jobs[blockIdx.y];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= J.N) return;
    float* r = J.rec + (size_t)i * S;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const double v = J.loc[(size_t)i * D + k] * J.sX;
        const float h = (float)v;
        r[k] = h;
        r[D + 1 + k] = (float)(v - (double)h);
    }
    const double v = J.times[i] * J.sT;
    const float h = (float)v;
    r[D] = h;
    r[2 * D + 1] = (float)(v - (double)h);
    r[2 * D + 2] = __int_as_float(J.ranks[i]);
#pragma unroll
    for (int k = 2 * D + 3; k < S; ++k) r[k] = 0.0f;
}

// 1 where event j's time differs from event j-1's (j > 0): for sorted times
// the dense rank of t_j is the number of such events in 1..j.
// (floatTimes: of the times rounded to FP32, the plain single-precision mode's
// causality, as in the reference's float engine.)
__device__ __forceinline__ int time_changes(int N, const double* __restrict__ times, int j,
                                            bool floatTimes) {
    if (j <= 0 || j >= N) return 0;
    return (floatTimes ? (float)times[j] != (float)times[j - 1] : times[j] != times[j - 1]) ? 1
                                                                                              : 0;
}

// One CTA of kTile threads per tile: min and max of t over the tile, and
// (tileChanges non-null) the tile's count of time changes.
__global__ void __launch_bounds__(kTile)
tile_bounds_kernel(int N, const double* __restrict__ times, double* __restrict__ tileMin,
                   double* __restrict__ tileMax, int* __restrict__ tileChanges, bool floatTimes) {
    __shared__ double sMin[kTile / 32], sMax[kTile / 32];
    __shared__ int sChanges[kTile / 32];
    const int j = blockIdx.x * kTile + threadIdx.x;
    double lo = INFINITY, hi = -INFINITY;
    if (j < N) lo = hi = times[j];
    if (tileChanges) {
        const int c = __reduce_add_sync(0xffffffffu, time_changes(N, times, j, floatTimes));
        if ((threadIdx.x & 31) == 0) sChanges[threadIdx.x >> 5] = c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sMin[w] = lo;
        sMax[w] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kTile / 32; ++k) {
            lo = fmin(lo, sMin[k]);
            hi = fmax(hi, sMax[k]);
        }
        tileMin[blockIdx.x] = lo;
        tileMax[blockIdx.x] = hi;
        if (tileChanges) {
            int c = 0;
            for (int k = 0; k < kTile / 32; ++k) c += sChanges[k];
            tileChanges[blockIdx.x] = c;
        }
    }
}

// One CTA of 1024 threads: v[0..n) replaced by its exclusive prefix sums
// (the first time change of each tile), in chunks of 1024 with a carry.
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(int n, int* __restrict__ v) {
    __shared__ int sWarp[32];
    __shared__ int sTotal;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int carry = 0;
    for (int base = 0; base < n; base += 1024) {
        const int i = base + threadIdx.x;
        const int x = i < n ? v[i] : 0;
        int s = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane == 31) sWarp[w] = s;
        __syncthreads();
        if (w == 0) {
            const int ws = sWarp[lane];
            int t = ws;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            sWarp[lane] = t - ws;  // this warp's offset within the chunk
            if (lane == 31) sTotal = t;
        }
        __syncthreads();
        if (i < n) v[i] = carry + sWarp[w] + s - x;
        carry += sTotal;
        __syncthreads();  // sWarp and sTotal are rewritten by the next chunk
    }
}

// One CTA of kTile threads per tile: rank[j] = tileOffset[tile] (the time
// changes before the tile) + the changes at the tile's events up to j (an
// inclusive scan within the tile).
__global__ void __launch_bounds__(kTile)
sorted_ranks_kernel(int N, const double* __restrict__ times, const int* __restrict__ tileOffset,
                    int32_t* __restrict__ ranks, bool floatTimes) {
    __shared__ int sWarp[kTile / 32];
    const int j = blockIdx.x * kTile + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int s = time_changes(N, times, j, floatTimes);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
    }
    if (lane == 31) sWarp[w] = s;
    __syncthreads();
    int before = 0;
    for (int k = 0; k < w; ++k) before += sWarp[k];
    if (j < N) ranks[j] = tileOffset[blockIdx.x] + before + s;
}

// ------------------------------------------------------ strip row order --
//
// Order of the target rows inside each full strip of S = 128 R events for
// the FP32 symmetric sweep.  A thread holds R rows and sums their terms for
// each earlier column in FP32 before the cross-lane reduction; rows far
// apart in space give terms of very different size, and FP32 addition drops
// a term below half an ulp of its partner entirely, so those partial sums
// come out low on average.  Rows sorted along a Morton (Z-order) curve of
// their first two coordinates and dealt to threads in consecutive runs of R
// put spatial neighbours in each thread (and neighbouring threads in each
// warp), whose terms for any column are of similar size.  Only the order of
// the rows changes: every row is still summed over the same columns.
//
// order[stripBase + r * 128 + t] = the event of row r of thread t.  One CTA
// of 256 threads per full strip: Morton keys from the strip's coordinates
// quantised to 16 bits over the strip's bounding box (one coordinate for
// D = 1), a bitonic sort of (key, position) pairs in shared memory, then the
// sorted events dealt out.  The last, partial strip keeps the identity order
// (the sweep does not read it).
constexpr int kOrderThreads = 256;

__device__ __forceinline__ unsigned spread16(unsigned v) {  // bits 0..15 -> even bits
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

template <int S>
__global__ void __launch_bounds__(kOrderThreads)
strip_order_kernel(int D, const double* __restrict__ loc, int32_t* __restrict__ order) {
    static_assert(S % kOrderThreads == 0 && (S & (S - 1)) == 0, "strip size");
    constexpr int R = S / kSweepThreads;
    __shared__ unsigned long long sKey[S];
    __shared__ double sLo[2][kOrderThreads / 32], sHi[2][kOrderThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int base = blockIdx.x * S;
    const int dims = D >= 2 ? 2 : 1;
    double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    for (int p = tid; p < S; p += kOrderThreads)
        for (int k = 0; k < dims; ++k) {
            const double v = loc[(size_t)(base + p) * D + k];
            lo[k] = fmin(lo[k], v);
            hi[k] = fmax(hi[k], v);
        }
    for (int k = 0; k < dims; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
        if (lane == 0) {
            sLo[k][warp] = lo[k];
            sHi[k][warp] = hi[k];
        }
    }
    __syncthreads();
    for (int k = 0; k < dims; ++k) {
        lo[k] = sLo[k][0];
        hi[k] = sHi[k][0];
        for (int w = 1; w < kOrderThreads / 32; ++w) {
            lo[k] = fmin(lo[k], sLo[k][w]);
            hi[k] = fmax(hi[k], sHi[k][w]);
        }
    }
    for (int p = tid; p < S; p += kOrderThreads) {
        unsigned q[2] = {0u, 0u};
        for (int k = 0; k < dims; ++k) {
            const double span = hi[k] - lo[k];
            const double u = span > 0.0 ? (loc[(size_t)(base + p) * D + k] - lo[k]) / span : 0.0;
            q[k] = (unsigned)fmin(65535.0, fmax(0.0, floor(u * 65536.0)));
        }
        const unsigned key = dims == 2 ? (spread16(q[0]) | (spread16(q[1]) << 1)) : (q[0] << 16);
        sKey[p] = ((unsigned long long)key << 32) | (unsigned)p;
    }
    __syncthreads();
    // bitonic sort, ascending
    for (int size = 2; size <= S; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int p = tid; p < S; p += kOrderThreads) {
                const int partner = p ^ stride;
                if (partner > p) {
                    const unsigned long long x = sKey[p], y = sKey[partner];
                    const bool up = (p & size) == 0;
                    if ((x > y) == up) {
                        sKey[p] = y;
                        sKey[partner] = x;
                    }
                }
            }
            __syncthreads();
        }
    for (int p = tid; p < S; p += kOrderThreads) {
        const int r = p / kSweepThreads, t = p % kSweepThreads;
        order[base + p] = base + (int)(sKey[R * t + r] & 0xffffffffu);
    }
}

__global__ void identity_order_kernel(int from, int N, int32_t* __restrict__ order) {
    const int i = from + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) order[i] = i;
}

// Device-resident loop: before each sweep, one thread per work item sets the
// item's first tile from the problem's current constants (a separate launch,
// so the sweep kernels themselves only read WorkItem::start).
__global__ void __launch_bounds__(kBandThreads)
band_starts_kernel(const SweepProblem* __restrict__ problems, WorkItem* __restrict__ items,
                   const int* __restrict__ nItems, int R) {
    const int it = blockIdx.x * kBandThreads + threadIdx.x;
    if (it >= *nItems) return;
    WorkItem w = items[it];
    const SweepProblem& P = problems[w.problem];
    items[it].start = P.searchBand ? first_tile_with_terms(P, R, w.strip, w.jt0, w.jt1) : w.jt0;
}

// ------------------------------------------------------------- finish --

// Deterministic CTA sum of NV values per thread; result valid in thread 0.
template <int NV, int THREADS>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
    __shared__ double sWarp[THREADS / 32][NV];
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sWarp[w][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = sWarp[0][q];
            for (int k = 1; k < THREADS / 32; ++k) s += sWarp[k][q];
            v[q] = s;
        }
    }
}

__device__ __forceinline__ double std_normal_cdf(double v) { return 0.5 * erfc(-v * kSqrtHalf); }

// Per-event finish in FP64 from the six unit pair sums s (already rescaled):
// v[0] = log lambda_i + compensator (src/NewHawkes.hpp:652-655), v[1..6] =
// the event's gradient contributions, *prob = P_i (src/NewHawkes.hpp:685).
__device__ __forceinline__ void event_contributions_f64(const FinishConsts& f,
                                                    const double (&s)[kNumAcc], double ti,
                                                    double (&v)[8], double* prob) {
    const double SB = f.prefB * s[0];
    const double SS = f.prefS * s[3];
    const double lam = SB + SS;
    const double inv = 1.0 / lam;
    const double Di = f.T - ti;
    const double eW = exp(-f.omega * Di);
    const double cdf = std_normal_cdf(f.b * Di) - std_normal_cdf(-f.b * ti);
    v[0] = log(lam) + f.theta * (eW - 1.0) - f.mu0 * cdf;
    v[1] = ((double)f.D / f.sigma * SS - f.sigma * f.prefS * s[4]) * inv;
    v[2] = ((double)f.D / f.a * SB - f.a * f.prefB * s[1]) * inv;
    const double bD = f.b * Di, bt = f.b * ti;
    const double phiD = kInvSqrt2Pi * exp(-0.5 * bD * bD);
    const double phiT = kInvSqrt2Pi * exp(-0.5 * bt * bt);
    v[3] = (SB / f.b - f.b * f.prefB * s[2]) * inv - f.mu0 * (phiD * Di + phiT * ti);
    v[4] = (SS / f.omega - f.prefS * s[5]) * inv - f.theta * Di * eW;
    v[5] = f.seScale * s[3] * inv + (eW - 1.0);
    v[6] = f.bgScale * s[0] * inv - cdf;
    if (prob) *prob = SS * inv;
}

// The same in FP32, for the plain single-precision mode: the unit sums, the
// rate, its log, the compensator (CDF) and the gradient contributions in
// float, as the reference's float engine forms its per-event terms
// (OpenCLHawkes.hpp:694-698, likContribs in REAL = float); the CTA and
// problem totals stay FP64 and fixed-order.
__device__ __forceinline__ float std_normal_cdf_f(float v) {
    return 0.5f * erfcf(-v * 0.70710678118654752f);
}

__device__ __forceinline__ void event_contributions_f32(const FinishConsts& f,
                                                        const double (&s)[kNumAcc], double tiD,
                                                        double (&v)[8], double* prob) {
    const float s0 = (float)s[0], s1 = (float)s[1], s2 = (float)s[2];
    const float s3 = (float)s[3], s4 = (float)s[4], s5 = (float)s[5];
    const float sigma = (float)f.sigma, a = (float)f.a, b = (float)f.b;
    const float omega = (float)f.omega, theta = (float)f.theta, mu0 = (float)f.mu0;
    const float prefB = (float)f.prefB, prefS = (float)f.prefS;
    const float ti = (float)tiD, T = (float)f.T;
    const float SB = prefB * s0, SS = prefS * s3;
    const float lam = SB + SS;
    const float inv = 1.0f / lam;
    const float Di = T - ti;
    const float eW = expf(-omega * Di);
    const float cdf = std_normal_cdf_f(b * Di) - std_normal_cdf_f(-b * ti);
    const float Df = (float)f.D;
    v[0] = logf(lam) + theta * (eW - 1.0f) - mu0 * cdf;
    v[1] = (Df / sigma * SS - sigma * prefS * s4) * inv;
    v[2] = (Df / a * SB - a * prefB * s1) * inv;
    const float bD = b * Di, bt = b * ti;
    const float phiD = 0.39894228040143268f * expf(-0.5f * bD * bD);
    const float phiT = 0.39894228040143268f * expf(-0.5f * bt * bt);
    v[3] = (SB / b - b * prefB * s2) * inv - mu0 * (phiD * Di + phiT * ti);
    v[4] = (SS / omega - prefS * s5) * inv - theta * Di * eW;
    v[5] = (float)f.seScale * s3 * inv + (eW - 1.0f);
    v[6] = (float)f.bgScale * s0 * inv - cdf;
    if (prob) *prob = SS * inv;
}

__device__ __forceinline__ void event_contributions(const FinishConsts& f,
                                                    const double (&s)[kNumAcc], double ti,
                                                    double (&v)[8], double* prob) {
    if (f.plain32)
        event_contributions_f32(f, s, ti, v, prob);
    else
        event_contributions_f64(f, s, ti, v, prob);
}

__global__ void __launch_bounds__(kFinishThreads)
finish_kernel(SweepGeometry g, const double* __restrict__ partials,
              const double* __restrict__ times, FinishConsts f, double* __restrict__ blockSums,
              double* __restrict__ probs) {
    const int i = blockIdx.x * kFinishThreads + threadIdx.x;
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = 0.0;
    if (i < g.N) {
        double s[kNumAcc];
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) {
            double acc = 0.0;
            for (int ch = 0; ch < g.nChunks; ++ch)
                acc += partials[((size_t)ch * kNumAcc + q) * g.Npad + i];
            s[q] = acc * f.accScale[q];
        }
        event_contributions(f, s, times[i], v, probs ? probs + i : nullptr);
    }
    block_sum<8, kFinishThreads>(v);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) blockSums[(size_t)blockIdx.x * 8 + q] = v[q];
    }
}

// The two exponentials of the FP32 sweep at arguments s[k] >= 0, for the
// direct test of their errors: poly[k] = 2^-s by exp2_poly_neg2 (the
// software exponential of near terms, two arguments per thread as in the
// sweep), hw[k] = ex2.approx.ftz(-s) (far-tail background terms).
__global__ void eval_exponentials_kernel(int n, const float* __restrict__ s,
                                         float* __restrict__ poly, float* __restrict__ hw) {
    const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= n) return;
    const bool two = k + 1 < n;
    const float a = s[k], b = two ? s[k + 1] : 0.0f;
    const float2 p = exp2_poly_neg2(make_float2(a, b));
    poly[k] = p.x;
    hw[k] = ex2_ftz(-a);
    if (two) {
        poly[k + 1] = p.y;
        hw[k + 1] = ex2_ftz(-b);
    }
}

// Mean relative error of ex2.approx.ftz.f32 against FP64 exp2 over arguments
// spread uniformly on [-16, 0) (uniform fractional parts): per-CTA sums of
// ex2(x) / 2^x - 1, added by the host in CTA order.
__global__ void __launch_bounds__(kFinishThreads)
ex2_bias_kernel(int n, double* __restrict__ blockSums) {
    const int i = blockIdx.x * kFinishThreads + threadIdx.x;
    double v[1] = {0.0};
    if (i < n) {
        const float x = (float)(-16.0 * ((double)i + 0.5) / (double)n);
        v[0] = (double)ex2_ftz(x) / exp2((double)x) - 1.0;
    }
    block_sum<1, kFinishThreads>(v);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = v[0];
}

constexpr int kFinalThreads = 256;

__global__ void __launch_bounds__(kFinalThreads)
final_kernel(int nBlocks, const double* __restrict__ blockSums, FinishConsts f,
             double* __restrict__ out) {
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = 0.0;
    for (int b = threadIdx.x; b < nBlocks; b += kFinalThreads)
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] += blockSums[(size_t)b * 8 + q];
    block_sum<8, kFinalThreads>(v);
    if (threadIdx.x == 0) {
        out[0] = v[0] + f.constant;
#pragma unroll
        for (int q = 1; q < 7; ++q) out[q] = v[q];
        out[7] = 0.0;
    }
}

// Finish over many problems: CTA b handles events [i0, i0 + kFinishThreads)
// of problem blocks[b].problem; each event sums its strip's slots in order.
__global__ void __launch_bounds__(kFinishThreads)
finish_list_kernel(const FinishProblem* __restrict__ problems,
                   const FinishBlock* __restrict__ blocks, double* __restrict__ blockSums) {
    const FinishBlock fb = blocks[blockIdx.x];
    const FinishProblem& P = problems[fb.problem];
    const FinishConsts f = P.f;
    const int N = P.N;
    const int i = fb.i0 + threadIdx.x;
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = 0.0;
    if (i < N) {
        const int nc = P.stripChunks[i / P.stripEvents];
        double s[kNumAcc];
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) {
            if (q < 3 && P.keptB) {
                s[q] = P.keptB[(size_t)q * N + i];  // unchanged: not written back
                continue;
            }
            double acc = 0.0;
            for (int ch = 0; ch < nc; ++ch)
                acc += P.partials[((size_t)ch * kNumAcc + q) * P.Npad + i];
            if (q < 3 && P.colAcc) {
                if (P.colWords == 2)  // FP64 sweep: two-word fixed point
                    acc += ldexp((double)P.colAcc[(size_t)(2 * q) * P.Npad + i], -P.colShift[q]) +
                           ldexp((double)P.colAcc[(size_t)(2 * q + 1) * P.Npad + i],
                                 -(P.colShift[q] + kColLoBits));
                else
                    acc += (double)P.colAcc[(size_t)q * P.Npad + i] * kColInv;
            }
            s[q] = acc * f.accScale[q];
            if (P.sums) P.sums[(size_t)q * N + i] = s[q];
        }
        event_contributions(f, s, P.times[i], v, P.probs ? P.probs + i : nullptr);
    }
    block_sum<8, kFinishThreads>(v);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) blockSums[(size_t)blockIdx.x * 8 + q] = v[q];
    }
}

// One CTA per problem: fixed-order sum of its finish CTAs' sums.
__global__ void __launch_bounds__(kFinalThreads)
final_list_kernel(const FinishProblem* __restrict__ problems, const double* __restrict__ blockSums,
                  double* __restrict__ out) {
    const FinishProblem& P = problems[blockIdx.x];
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = 0.0;
    for (int b = threadIdx.x; b < P.nBlocks; b += kFinalThreads)
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] += blockSums[(size_t)(P.blockBase + b) * 8 + q];
    block_sum<8, kFinalThreads>(v);
    if (threadIdx.x == 0) {
        double* o = out + (size_t)blockIdx.x * 8;
        o[0] = v[0] + P.f.constant;
#pragma unroll
        for (int q = 1; q < 7; ++q) o[q] = v[q];
        o[7] = 0.0;
    }
}

// ------------------------------------------------------- incremental --

constexpr int kMoveThreads = 256;

// Unit pair terms of target i against source j in natural units (FP64): the
// background weights exp(cA d^2 + cB dt^2) x {1, d^2, dt^2} and, for dt > 0,
// the self-excitation weights exp(cS d^2 + cW dt) x {1, d^2, dt}.
__device__ __forceinline__ void unit_terms(double d2, double dt, const PairConsts& c,
                                           double (&u)[kNumAcc]) {
    const double t2 = dt * dt;
    const double B = exp(fma(c.cA, d2, c.cB * t2));
    u[0] = B;
    u[1] = B * d2;
    u[2] = B * t2;
    const double S = dt > 0.0 ? exp(fma(c.cS, d2, c.cW * dt)) : 0.0;
    u[3] = S;
    u[4] = S * d2;
    u[5] = S * dt;
}

template <int D>
__global__ void __launch_bounds__(kMoveThreads)
move_event_kernel(int N, MovedEvent m, const double* __restrict__ loc,
                  const double* __restrict__ times, PairConsts c, double* __restrict__ sums,
                  double* __restrict__ rowPartials) {
    const int i = blockIdx.x * kMoveThreads + threadIdx.x;
    const int k = m.k;
    double row[kNumAcc];
#pragma unroll
    for (int q = 0; q < kNumAcc; ++q) row[q] = 0.0;
    if (i < N) {
        const double ti = times[i], tk = times[k];
        double d2New = 0.0, d2Old = 0.0;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const double xi = loc[(size_t)i * D + a];
            const double dn = xi - loc[(size_t)k * D + a];
            const double dOld = xi - m.oldLoc[a];
            d2New = fma(dn, dn, d2New);
            d2Old = fma(dOld, dOld, d2Old);
        }
        if (i != k) {
            // event i's sums: its pair with k moves from the old to the new location
            double un[kNumAcc], uo[kNumAcc];
            unit_terms(d2New, ti - tk, c, un);
            unit_terms(d2Old, ti - tk, c, uo);
#pragma unroll
            for (int q = 0; q < kNumAcc; ++q) sums[(size_t)q * N + i] += un[q] - uo[q];
        }
        // event k's new row: its pair with i (i == k: the j = i background term)
        unit_terms(d2New, tk - ti, c, row);
    }
    double v[kNumAcc];
#pragma unroll
    for (int q = 0; q < kNumAcc; ++q) v[q] = row[q];
    block_sum<kNumAcc, kMoveThreads>(v);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) rowPartials[(size_t)blockIdx.x * kNumAcc + q] = v[q];
}

__global__ void __launch_bounds__(kFinalThreads)
move_event_row_kernel(int N, int k, int nBlocks, const double* __restrict__ rowPartials,
                      double* __restrict__ sums) {
    double v[kNumAcc];
#pragma unroll
    for (int q = 0; q < kNumAcc; ++q) v[q] = 0.0;
    for (int b = threadIdx.x; b < nBlocks; b += kFinalThreads)
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) v[q] += rowPartials[(size_t)b * kNumAcc + q];
    block_sum<kNumAcc, kFinalThreads>(v);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) sums[(size_t)q * N + k] = v[q];
}

__global__ void __launch_bounds__(kFinishThreads)
finish_sums_kernel(int N, const double* __restrict__ sums, const double* __restrict__ times,
                   FinishConsts f, double* __restrict__ blockSums, double* __restrict__ probs) {
    const int i = blockIdx.x * kFinishThreads + threadIdx.x;
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = 0.0;
    if (i < N) {
        double s[kNumAcc];
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) s[q] = sums[(size_t)q * N + i];
        event_contributions(f, s, times[i], v, probs ? probs + i : nullptr);
    }
    block_sum<8, kFinishThreads>(v);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) blockSums[(size_t)blockIdx.x * 8 + q] = v[q];
    }
}

}  // namespace

#define HPHC_FOR_EACH_DIM(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8)

cudaError_t launch_pack_f64(int D, int N, const double* loc, const double* times, double* rec,
                            double* tileMin, double* tileMax, cudaStream_t s) {
    const int blocks = (N + 255) / 256;
    switch (D) {
#define X(d) \
    case d: pack_f64_kernel<d><<<blocks, 256, 0, s>>>(N, loc, times, rec); break;
        HPHC_FOR_EACH_DIM(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
    tile_bounds_kernel<<<(N + kTile - 1) / kTile, kTile, 0, s>>>(N, times, tileMin, tileMax,
                                                                  nullptr, false);
    return cudaGetLastError();
}

cudaError_t launch_tile_bounds(int N, const double* times, double* tileMin, double* tileMax,
                               int* tileChanges, cudaStream_t s, int floatTimes) {
    tile_bounds_kernel<<<(N + kTile - 1) / kTile, kTile, 0, s>>>(N, times, tileMin, tileMax,
                                                                  tileChanges, floatTimes != 0);
    return cudaGetLastError();
}

cudaError_t launch_sorted_ranks(int N, const double* times, int* tileChanges, int32_t* ranks,
                                cudaStream_t s, int floatTimes) {
    const int nTiles = (N + kTile - 1) / kTile;
    exclusive_scan_kernel<<<1, 1024, 0, s>>>(nTiles, tileChanges);
    sorted_ranks_kernel<<<nTiles, kTile, 0, s>>>(N, times, tileChanges, ranks, floatTimes != 0);
    return cudaGetLastError();
}

cudaError_t launch_strip_order(int D, int N, int R, const double* loc, int32_t* order,
                               cudaStream_t s) {
    const int S = kSweepThreads * R;
    const int full = N / S;
    if (full > 0) {
        if (R == 2)
            strip_order_kernel<2 * kSweepThreads><<<full, kOrderThreads, 0, s>>>(D, loc, order);
        else if (R == 4)
            strip_order_kernel<4 * kSweepThreads><<<full, kOrderThreads, 0, s>>>(D, loc, order);
        else
            return cudaErrorInvalidValue;
    }
    const int rest = N - full * S;
    if (rest > 0) identity_order_kernel<<<(rest + 255) / 256, 256, 0, s>>>(full * S, N, order);
    return cudaGetLastError();
}

cudaError_t launch_sweep_f64(int D, int R, const SweepGeometry& g, const double* rec,
                             const double* tileMin, const double* tileMax, const PairConsts& c,
                             double* partials, cudaStream_t s) {
    switch (D) {
#define X(d) \
    case d: return sweep_grid_f64_d##d(R, g, rec, tileMin, tileMax, c, partials, s);
        HPHC_FOR_EACH_DIM(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
}

namespace {

cudaError_t sweep_list_dispatch(int precision, int D, int R, int V, int grid,
                                const SweepProblem* problems, const WorkItem* items,
                                const int* nItems, int* counter, cudaStream_t s,
                                int* blocksPerSM) {
    switch (D) {
#define X(d) \
    case d: return sweep_list_d##d(precision, R, V, grid, problems, items, nItems, counter, s, \
                                   blocksPerSM);
        HPHC_FOR_EACH_DIM(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace


cudaError_t launch_sweep_list(int precision, int D, int R, int V, int grid,
                              const SweepProblem* problems, const WorkItem* items,
                              const int* nItems, int* counter, cudaStream_t s) {
    if (grid < 1) return cudaErrorInvalidValue;
    return sweep_list_dispatch(precision, D, R, V, grid, problems, items, nItems, counter, s,
                               nullptr);
}

int sweep_list_blocks_per_sm(int precision, int D, int R, int V) {
    int n = 0;
    if (sweep_list_dispatch(precision, D, R, V, 1, nullptr, nullptr, nullptr, nullptr, 0, &n) !=
        cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_pack_f32_jobs(int D, int nJobs, int maxN, const PackJob* jobs, cudaStream_t s) {
    const dim3 grid((maxN + 255) / 256, nJobs);
    switch (D) {
#define X(d) \
    case d: pack_f32_jobs_kernel<d><<<grid, 256, 0, s>>>(jobs); break;
        HPHC_FOR_EACH_DIM(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_band_starts(int maxItems, const SweepProblem* problems, WorkItem* items,
                               const int* nItems, int R, cudaStream_t s) {
    if (maxItems <= 0) return cudaSuccess;
    band_starts_kernel<<<(maxItems + kBandThreads - 1) / kBandThreads, kBandThreads, 0, s>>>(
        problems, items, nItems, R);
    return cudaGetLastError();
}

cudaError_t launch_finish_list(int nBlocks, const FinishProblem* problems,
                               const FinishBlock* blocks, double* blockSums, cudaStream_t s) {
    finish_list_kernel<<<nBlocks, kFinishThreads, 0, s>>>(problems, blocks, blockSums);
    return cudaGetLastError();
}

cudaError_t launch_final_list(int nProblems, const FinishProblem* problems,
                              const double* blockSums, double* out, cudaStream_t s) {
    final_list_kernel<<<nProblems, kFinalThreads, 0, s>>>(problems, blockSums, out);
    return cudaGetLastError();
}

cudaError_t launch_finish(const SweepGeometry& g, const double* partials, const double* times,
                          const FinishConsts& f, double* blockSums, double* probs,
                          cudaStream_t s) {
    finish_kernel<<<finish_blocks(g.N), kFinishThreads, 0, s>>>(g, partials, times, f, blockSums,
                                                                probs);
    return cudaGetLastError();
}

cudaError_t launch_ex2_bias(int n, double* blockSums, cudaStream_t s) {
    ex2_bias_kernel<<<(n + kFinishThreads - 1) / kFinishThreads, kFinishThreads, 0, s>>>(
        n, blockSums);
    return cudaGetLastError();
}

cudaError_t launch_eval_exponentials(int n, const float* s, float* poly, float* hw,
                                     cudaStream_t st) {
    const int pairs = (n + 1) / 2;
    eval_exponentials_kernel<<<(pairs + 255) / 256, 256, 0, st>>>(n, s, poly, hw);
    return cudaGetLastError();
}

cudaError_t launch_final(int nBlocks, const double* blockSums, const FinishConsts& f, double* out,
                         cudaStream_t s) {
    final_kernel<<<1, kFinalThreads, 0, s>>>(nBlocks, blockSums, f, out);
    return cudaGetLastError();
}

int move_event_blocks(int N) { return (N + kMoveThreads - 1) / kMoveThreads; }

cudaError_t launch_move_event(int D, int N, const MovedEvent& m, const double* loc,
                              const double* times, const PairConsts& c, double* sums,
                              double* rowPartials, cudaStream_t s) {
    const int blocks = move_event_blocks(N);
    switch (D) {
#define X(d)                                                                                     \
    case d:                                                                                      \
        move_event_kernel<d><<<blocks, kMoveThreads, 0, s>>>(N, m, loc, times, c, sums,          \
                                                              rowPartials);                      \
        break;
        HPHC_FOR_EACH_DIM(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_move_event_row(int N, int k, const double* rowPartials, double* sums,
                                  cudaStream_t s) {
    move_event_row_kernel<<<1, kFinalThreads, 0, s>>>(N, k, move_event_blocks(N), rowPartials,
                                                      sums);
    return cudaGetLastError();
}

cudaError_t launch_finish_sums(int N, const double* sums, const double* times,
                               const FinishConsts& f, double* blockSums, double* probs,
                               double* out, cudaStream_t s) {
    finish_sums_kernel<<<finish_blocks(N), kFinishThreads, 0, s>>>(N, sums, times, f, blockSums,
                                                                   probs);
    final_kernel<<<1, kFinalThreads, 0, s>>>(finish_blocks(N), blockSums, f, out);
    return cudaGetLastError();
}

}  // namespace hphc
