// Pair-sweep kernels of the B200 Hawkes likelihood engine: device code shared
// by the per-dimension compilation units hphc_sweep_d<D>.cu (each instantiates
// the sweeps of one D, so the eight are compiled in parallel) and by
// hphc_kernels.cu (tile-pair decisions for the device-resident band kernel).
//
// The reference evaluates, for every target event i, the rate
//   lambda_i = sum_j B_ij + S_ij   (src/NewHawkes.hpp:520-547)
// with one work-group of 128 threads per event striding over j
// (src/backend/opencl/OpenCLHawkes.hpp:632-702).  Here a CTA owns a strip of
// kSweepThreads * R target events (R per thread, in registers) and a range of
// j tiles; each kTile-event j tile is staged in shared memory with coalesced
// 16-byte loads and read back as broadcasts.  Per (strip, tile) the CTA
// decides from FP64 time bounds whether the tile pair has any background term
// above the skip threshold, any causal (t_j < t_i) self-excitation term,
// and whether the causal mask is needed, so the non-causal half of the
// self-excitation sum is skipped at tile level.  Skipped self-excitation terms
// are exactly zero in the working precision; skipped background terms are
// zero too, or with tail truncation (the default) each at most 2^-91 (FP64)
// or 2^-60 (FP32 modes) of the event's own background term, which moves its
// sums by under 2^-60 or 2^-33 (kNegligibleLog2).
//
// All sums are written per (chunk, event) and combined in chunk order, then
// reduced over events with fixed shuffle trees: results do not depend on
// scheduling.
#pragma once

#include <limits.h>
#include <math.h>

#include "hphc_kernels.cuh"

namespace hphc {

// Per-dimension entry points (hphc_sweep_d<D>.cu): the work-list sweep of
// precision (0 = FP64, 1 = FP32) with R events per thread and FP32 variant V
// (blocksPerSM non-null: resident CTAs per SM instead of a launch), and the
// FP64 grid-form sweep.
#define HPHC_DECLARE_SWEEP_DIM(d)                                                                \
    cudaError_t sweep_list_d##d(int precision, int R, int V, int grid,                          \
                                const SweepProblem* problems, const WorkItem* items,            \
                                const int* nItems, int* counter, cudaStream_t s,                \
                                int* blocksPerSM);                                               \
    cudaError_t sweep_grid_f64_d##d(int R, const SweepGeometry& g, const double* rec,            \
                                    const double* tileMin, const double* tileMax,               \
                                    const PairConsts& c, double* partials, cudaStream_t s);
HPHC_DECLARE_SWEEP_DIM(1)
HPHC_DECLARE_SWEEP_DIM(2)
HPHC_DECLARE_SWEEP_DIM(3)
HPHC_DECLARE_SWEEP_DIM(4)
HPHC_DECLARE_SWEEP_DIM(5)
HPHC_DECLARE_SWEEP_DIM(6)
HPHC_DECLARE_SWEEP_DIM(7)
HPHC_DECLARE_SWEEP_DIM(8)
#undef HPHC_DECLARE_SWEEP_DIM

namespace {

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ------------------------------------------------------ tile-pair decision --

struct TileMode {
    bool doB, doS, allCausal;
    bool fastB;  // every background term of the pair is in the far tail (FP32)
};

// dt = t_i - t_j over the tile pair lies in [tminI - tmaxJ, tmaxI - tminJ].
__device__ __forceinline__ TileMode tile_mode(double tminI, double tmaxI, double tminJ,
                                              double tmaxJ, const PairConsts& c) {
    const double dtLo = tminI - tmaxJ, dtHi = tmaxI - tminJ;
    const double minAbs = dtLo > 0.0 ? dtLo : (dtHi < 0.0 ? -dtHi : 0.0);
    TileMode m;
    m.doB = !c.noB && !(c.skipB >= 0.0 && -c.cB * minAbs * minAbs >= c.skipB);
    m.allCausal = dtLo > 0.0;
    const bool anyCausal = dtHi > 0.0;
    m.doS = anyCausal && !(c.skipS >= 0.0 && m.allCausal && -c.cW * dtLo >= c.skipS);
    // fastB > 0 when enabled (12 ln 2); zero-initialized constants keep it off
    m.fastB = c.fastB > 0.0 && -c.cB * minAbs * minAbs >= c.fastB;
    return m;
}

// ----------------------------------------------------------- FP64 sweep --

// FP64 background term exp(x): CUDA's exp(), or for far-tail tile pairs
// (every term at most 2^-60, see kFastTailLog2F64) the FP32 hardware
// exponential.
template <bool FAST>
__device__ __forceinline__ double background_f64(double x) {
    if (FAST) return (double)ex2_ftz((float)(x * 1.44269504088896340735992468100189214));
    return exp(x);
}

template <int D, int R, bool DO_B, bool DO_S, bool MASK, bool FAST = false>
__device__ __forceinline__ void body_f64(const double* __restrict__ sRec, int nj,
                                         const double (&xi)[R][D], const double (&ti)[R],
                                         const PairConsts& c, double (&acc)[R][kNumAcc]) {
    constexpr int S = Layout<D>::kF64Stride;
#pragma unroll 2
    for (int j = 0; j < nj; ++j) {
        double rj[S];
#pragma unroll
        for (int v = 0; v < S / 2; ++v) {
            const double2 q = reinterpret_cast<const double2*>(sRec + j * S)[v];
            rj[2 * v] = q.x;
            rj[2 * v + 1] = q.y;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double d2 = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                const double dd = xi[r][k] - rj[k];
                d2 = fma(dd, dd, d2);
            }
            const double dt = ti[r] - rj[D];
            if (DO_B) {
                const double t2 = dt * dt;
                const double B = background_f64<FAST>(fma(c.cA, d2, c.cB * t2));
                acc[r][0] += B;
                acc[r][1] = fma(B, d2, acc[r][1]);
                acc[r][2] = fma(B, t2, acc[r][2]);
            }
            if (DO_S) {
                double Sv = exp(fma(c.cS, d2, c.cW * dt));
                if (MASK) Sv = dt > 0.0 ? Sv : 0.0;
                acc[r][3] += Sv;
                acc[r][4] = fma(Sv, d2, acc[r][4]);
                acc[r][5] = fma(Sv, dt, acc[r][5]);
            }
        }
    }
}

// ---- symmetric FP64 background tiles ----
//
// As in the FP32 sweep, a tile before the strip evaluates each background
// pair once and adds its three weighted terms to the row (registers) and to
// the column.  Column partials are reduced per warp in groups of 4 columns:
// lane l visits the group's columns in the order m ^ p, p = (l >> 3) & 3, so
// after the loop cp[.][m] holds column m ^ p over the lane's R rows; shuffles
// at distances 16 and 8 each keep the half of the columns the lane ends with,
// then 4, 2 and 1 sum, leaving lanes 8p .. 8p + 7 with the warp total of
// column p.  The 4 warp totals are added in FP64 in warp order and added to
// the column's two-word fixed-point sum (see add_fixed2), so the result does
// not depend on CTA order and keeps FP64 accuracy.

constexpr int kSymGroup64 = 4;  // columns per warp exchange (FP64)

// Adds v >= 0 to a two-word fixed-point sum: hi counts units of 2^-shift,
// lo units of 2^-(shift + kColLoBits).  The host chooses shift so that no
// column total exceeds 2^62 units; the lo word takes at most 2^23 additions
// of values below 2^kColLoBits without overflowing.
__device__ __forceinline__ void add_fixed2(unsigned long long* hi, unsigned long long* lo,
                                           double v, int shift) {
    const double scaled = ldexp(v, shift);
    const double whole = floor(scaled);
    atomicAdd(hi, (unsigned long long)whole);
    atomicAdd(lo, (unsigned long long)rint(ldexp(scaled - whole, kColLoBits)));
}

template <int D, int R, bool DO_S, bool MASK, bool FAST = false>
__device__ __forceinline__ void tile_sym_f64(const double* __restrict__ sRec,
                                             const double (&xi)[R][D], const double (&ti)[R],
                                             const PairConsts& c, double (&acc)[R][kNumAcc],
                                             double* __restrict__ sCol,
                                             unsigned long long* __restrict__ colAcc, int Npad,
                                             int j0, const int (&shift)[3]) {
    static_assert(kSweepThreads == kTile, "one column per thread in the column flush");
    constexpr int S = Layout<D>::kF64Stride;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int p = (lane >> 3) & 3;
#pragma unroll 1
    for (int g = 0; g < kTile; g += kSymGroup64) {
        double cp[3][kSymGroup64];
#pragma unroll
        for (int m = 0; m < kSymGroup64; ++m) {
            const int j = g + (m ^ p);
            double rj[S];
#pragma unroll
            for (int v = 0; v < S / 2; ++v) {
                const double2 q = reinterpret_cast<const double2*>(sRec + j * S)[v];
                rj[2 * v] = q.x;
                rj[2 * v + 1] = q.y;
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                double d2 = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const double dd = xi[r][k] - rj[k];
                    d2 = fma(dd, dd, d2);
                }
                const double dt = ti[r] - rj[D];
                const double t2 = dt * dt;
                const double B = background_f64<FAST>(fma(c.cA, d2, c.cB * t2));
                const double Bd = B * d2, Bt = B * t2;
                acc[r][0] += B;
                acc[r][1] += Bd;
                acc[r][2] += Bt;
                if (r == 0) {
                    cp[0][m] = B;
                    cp[1][m] = Bd;
                    cp[2][m] = Bt;
                } else {
                    cp[0][m] += B;
                    cp[1][m] += Bd;
                    cp[2][m] += Bt;
                }
                if (DO_S) {
                    double Sv = exp(fma(c.cS, d2, c.cW * dt));
                    if (MASK) Sv = dt > 0.0 ? Sv : 0.0;
                    acc[r][3] += Sv;
                    acc[r][4] = fma(Sv, d2, acc[r][4]);
                    acc[r][5] = fma(Sv, dt, acc[r][5]);
                }
            }
        }
        constexpr unsigned kAll = 0xffffffffu;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double u0 = cp[q][0] + __shfl_xor_sync(kAll, cp[q][2], 16);
            const double u1 = cp[q][1] + __shfl_xor_sync(kAll, cp[q][3], 16);
            double w = u0 + __shfl_xor_sync(kAll, u1, 8);
            w += __shfl_xor_sync(kAll, w, 4);
            w += __shfl_xor_sync(kAll, w, 2);
            w += __shfl_xor_sync(kAll, w, 1);
            if ((lane & 7) == 0) sCol[(warp * 3 + q) * kTile + g + p] = w;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kSweepThreads / 32; ++w) v += sCol[(w * 3 + q) * kTile + tid];
        add_fixed2(colAcc + (size_t)(2 * q) * Npad + j0 + tid,
                   colAcc + (size_t)(2 * q + 1) * Npad + j0 + tid, v, shift[q]);
    }
}

// Where an item of a problem with searchBand set may start: the first tile
// in [jt0, min(jt1, strip's first tile)) that is not ruled out by its time
// gap to strip `strip` (R tiles of targets).  With sorted times the gap
// shrinks as jt grows, so "the background can be non-zero, or the gap does
// not make every self-excitation term underflow" turns on once and stays
// on, and bisection finds the start with ~log2(nTiles) reads of the tile
// bounds instead of one read per skipped tile.  The set it keeps contains
// every tile tile_mode would evaluate (its causality test only removes more),
// and the item still decides each tile with tile_mode.
__device__ __forceinline__ int first_tile_with_terms(const SweepProblem& P, int R, int strip,
                                                     int jt0, int jt1) {
    const int ts0 = strip * R, ts1 = min(ts0 + R, P.nTiles);
    double tminI = INFINITY, tmaxI = -INFINITY;
    for (int t = ts0; t < ts1; ++t) {
        tminI = fmin(tminI, P.tileMin[t]);
        tmaxI = fmax(tmaxI, P.tileMax[t]);
    }
    int lo = jt0, hi = min(jt1, ts0);
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        const TileMode m = tile_mode(tminI, tmaxI, P.tileMin[mid], P.tileMax[mid], P.c);
        const double dtLo = tminI - P.tileMax[mid];
        const bool sFar = P.c.skipS >= 0.0 && dtLo > 0.0 && -P.c.cW * dtLo >= P.c.skipS;
        if (m.doB || !sFar)
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo;
}

// One work item of the FP64 sweep: target strip `strip` (kSweepThreads * R
// events) against j tiles [jt0, jt1); unit pair sums to partial slot `slot`.
// sym: tiles before the strip are evaluated once per pair (rows + columns).
template <int D, int R>
__device__ __forceinline__ void f64_item(const double* __restrict__ rec,
                                         const double* __restrict__ tileMin,
                                         const double* __restrict__ tileMax,
                                         double* __restrict__ partials, int N, int nTiles,
                                         int Npad, const PairConsts& c, int strip, int jt0,
                                         int jt1, int slot, double* sRec, bool sym,
                                         unsigned long long* __restrict__ colAcc,
                                         const int (&shift)[3], double* sCol) {
    constexpr int S = Layout<D>::kF64Stride;
    const int tid = threadIdx.x;
    const int stripBase = strip * kSweepThreads * R;
    const int ts0 = stripBase / kTile, ts1 = min(ts0 + R, nTiles);

    double xi[R][D], ti[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int iRaw = stripBase + r * kSweepThreads + tid;
        const int i = min(iRaw, N - 1);
#pragma unroll
        for (int k = 0; k < D; ++k)
            // padding rows of the last strip sit 1e150 away: every background
            // term they form is exactly 0, so they add nothing to column sums
            xi[r][k] = iRaw < N ? rec[(size_t)i * S + k] : 1e150;
        ti[r] = rec[(size_t)i * S + D];
    }
    double tminI = INFINITY, tmaxI = -INFINITY;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int tt = stripBase / kTile + r;
        if (tt < nTiles) {
            tminI = fmin(tminI, tileMin[tt]);
            tmaxI = fmax(tmaxI, tileMax[tt]);
        }
    }
    double acc[R][kNumAcc];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) acc[r][q] = 0.0;

    for (int jt = jt0; jt < jt1; ++jt) {
        TileMode m = tile_mode(tminI, tmaxI, tileMin[jt], tileMax[jt], c);
        if (sym && jt >= ts1) m.doB = false;  // covered as columns by later strips
        if (!m.doB && !m.doS) continue;
        const int j0 = jt * kTile;
        const int nj = min(kTile, N - j0);
        __syncthreads();
        const double2* src = reinterpret_cast<const double2*>(rec + (size_t)j0 * S);
        double2* dst = reinterpret_cast<double2*>(sRec);
        for (int v = tid; v < nj * (S / 2); v += kSweepThreads) dst[v] = src[v];
        __syncthreads();
        // warm L1 with the next tile's records while this tile is evaluated
        if (jt + 1 < jt1) {
            const int nn = min(kTile, N - j0 - kTile) * S;  // doubles of the next tile
            for (int v = 16 * tid; v < nn; v += 16 * kSweepThreads)
                prefetch_l1(rec + (size_t)(j0 + kTile) * S + v);
        }
        // Far-tail tile pairs (every background term at most 2^-60) take them
        // from the FP32 hardware exponential; the choice depends on the
        // background bound alone, and such a pair needs no causality mask.
        if (sym && m.doB && jt < ts0 && m.fastB) {
            if (!m.doS)
                tile_sym_f64<D, R, false, false, true>(sRec, xi, ti, c, acc, sCol, colAcc, Npad,
                                                       j0, shift);
            else
                tile_sym_f64<D, R, true, false, true>(sRec, xi, ti, c, acc, sCol, colAcc, Npad,
                                                      j0, shift);
        } else if (m.doB && m.fastB && !(sym && jt < ts0)) {
            if (!m.doS)
                body_f64<D, R, true, false, false, true>(sRec, nj, xi, ti, c, acc);
            else
                body_f64<D, R, true, true, false, true>(sRec, nj, xi, ti, c, acc);
        } else if (sym && m.doB && jt < ts0) {
            // jt < ts0 <= nTiles - 1: a full tile
            if (!m.doS)
                tile_sym_f64<D, R, false, false>(sRec, xi, ti, c, acc, sCol, colAcc, Npad, j0,
                                                 shift);
            else if (m.allCausal)
                tile_sym_f64<D, R, true, false>(sRec, xi, ti, c, acc, sCol, colAcc, Npad, j0,
                                                shift);
            else
                tile_sym_f64<D, R, true, true>(sRec, xi, ti, c, acc, sCol, colAcc, Npad, j0,
                                               shift);
        } else if (m.doB) {
            if (!m.doS)
                body_f64<D, R, true, false, false>(sRec, nj, xi, ti, c, acc);
            else if (m.allCausal)
                body_f64<D, R, true, true, false>(sRec, nj, xi, ti, c, acc);
            else
                body_f64<D, R, true, true, true>(sRec, nj, xi, ti, c, acc);
        } else {
            if (m.allCausal)
                body_f64<D, R, false, true, false>(sRec, nj, xi, ti, c, acc);
            else
                body_f64<D, R, false, true, true>(sRec, nj, xi, ti, c, acc);
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = stripBase + r * kSweepThreads + tid;
        if (i < N) {
#pragma unroll
            for (int q = 0; q < kNumAcc; ++q)
                // a self-excitation-only sweep leaves the background rows to
                // the kept sums: they are neither written nor read
                if (q >= 3 || !c.noB) partials[((size_t)slot * kNumAcc + q) * Npad + i] = acc[r][q];
        }
    }
}

// Grid form: one CTA per (strip, chunk), chunks of g.chunkTiles tiles.
template <int D, int R>
__global__ void __launch_bounds__(kSweepThreads)
sweep_f64_kernel(SweepGeometry g, const double* __restrict__ rec,
                 const double* __restrict__ tileMin, const double* __restrict__ tileMax,
                 PairConsts c, double* __restrict__ partials) {
    __shared__ __align__(16) double sRec[kTile * Layout<D>::kF64Stride];
    const int strip = blockIdx.x / g.nChunks;
    const int chunk = blockIdx.x - strip * g.nChunks;
    const int jt0 = chunk * g.chunkTiles;
    const int jt1 = min(jt0 + g.chunkTiles, g.nTiles);
    const int noShift[3] = {0, 0, 0};
    f64_item<D, R>(rec, tileMin, tileMax, partials, g.N, g.nTiles, g.Npad, c, strip, jt0, jt1,
                   chunk, sRec, false, nullptr, noShift, nullptr);
}

// Takes the next work-list index for the CTA (all threads get the same one).
__device__ __forceinline__ int next_item(int* counter, int* sNext) {
    __syncthreads();
    if (threadIdx.x == 0) *sNext = atomicAdd(counter, 1);
    __syncthreads();
    return *sNext;
}

// Work-list form: persistent CTAs take items until the list is exhausted.
template <int D, int R>
__global__ void __launch_bounds__(kSweepThreads)
sweep_f64_list_kernel(const SweepProblem* __restrict__ problems,
                      const WorkItem* __restrict__ items, const int* __restrict__ nItems,
                      int* __restrict__ counter) {
    __shared__ __align__(16) double sRec[kTile * Layout<D>::kF64Stride];
    __shared__ __align__(16) double sCol[(kSweepThreads / 32) * 3 * kTile];
    __shared__ int sNext;
    const int n = *nItems;
    for (;;) {
        const int it = next_item(counter, &sNext);
        if (it >= n) break;
        const WorkItem w = items[it];
        const SweepProblem& P = problems[w.problem];
        const PairConsts c = P.c;
        const int shift[3] = {P.colShift[0], P.colShift[1], P.colShift[2]};
        f64_item<D, R>(static_cast<const double*>(P.rec), P.tileMin, P.tileMax, P.partials, P.N,
                       P.nTiles, P.Npad, c, w.strip, w.start, w.jt1, w.slot, sRec,
                       P.symmetric != 0, P.colAcc, shift, sCol);
    }
}

// ------------------------------------------------ FP32-compensated sweep --
//
// Records hold coordinates and times pre-scaled by the background kernel's
// precisions, x' = x a sqrt(log2(e)/2) and t' = t b sqrt(log2(e)/2), so the
// background exponent in log2 units is -(|dx'|^2 + dt'^2) with no coefficient
// at all (hence no coefficient rounding).  Times are formed from hi/lo float
// pairs, dt' = (hi_i - hi_j) + (lo_i - lo_j), so the FP32 representation error
// of the inputs (ulp(8760 h) ~ 1e-3 h) never enters dt; coordinates likewise
// when the variant keeps their lo parts.  The self-excitation exponent
// kS |dx'|^2 + kW dt' uses hi + lo coefficients so their FP32 rounding does
// not bias every term in the same direction.  The weighted sums come out in
// scaled units and the finish rescales them in FP64.  Each of a row's six sums
// is a compensated FP32 pair (hi, lo; see RowSums below) over a work item's
// whole j range, formed into FP64 when the item writes its partial sums; the
// cross-chunk sums and the per-event finish are FP64.
//
// Variant bits (template parameter V):
//   kSpaceLo  coordinate differences use the lo parts too (else hi only: the
//             coordinate rounding then acts as a fixed ~1e-7 relative
//             perturbation of each event's location, unbiased across events).
//   kPolyExp  exponentials by exp2_poly_neg2 (unbiased to ~3e-10) instead of
//             ex2.approx, whose measured mean relative error the finish
//             divides out of the sums.
//   kTimeHiOnly  background terms from the hi parts of the times only (far-tail
//             tile pairs, set by the sweep itself): the lo parts are at most
//             half an FP32 ulp of t' (~1e-6 in record units over the 8760 h
//             span at the base tauT), which moves a far-tail term (|dt'| >= 3.16,
//             at most 2^-10) by ~2.6e-6 |dt'| relative, with a sign that varies
//             with the pair.  Self-excitation terms of such a tile pair still
//             use the full hi + lo difference.
//   kPlain    FP32 throughout, the reference's single precision
//             (src/factory.cpp:45, OpenCLHawkes.hpp:616-630): times and
//             coordinates as single floats (hi parts), the hardware
//             exponential for every term, plain FP32 sums, and causality
//             from the times rounded to FP32 (ranks and tile decisions).
constexpr int kSpaceLo = 1;
constexpr int kPolyExp = 2;
constexpr int kTimeHiOnly = 4;
constexpr int kPlain = 8;

// Coefficients of p(f) ~ 2^f on [-1/2, 1/2], degree 7, fitted in relative
// error by tests/fit_exp2.py with sequential FP32 rounding: max relative
// error 3.4e-10 (mean +2.8e-11) with these FP32 values in FP64 evaluation,
// below the 6.3e-8 rounding of FP32 Horner evaluation itself.  Degree 6
// (3.3e-9, one FMA fewer) left an error that oscillates with the fraction of
// the argument, which sums weighted by dt'^2 and by 1 sample differently:
// the strongly cancelling d/d tauT gradient component showed it at ~1e-8.
constexpr float kP1 = 0x1.62e430p-1f;
constexpr float kP2 = 0x1.ebfbe0p-3f;
constexpr float kP3 = 0x1.c6b070p-5f;
constexpr float kP4 = 0x1.3b2a78p-7f;
constexpr float kP5 = 0x1.5da248p-10f;
constexpr float kP6 = 0x1.43ec02p-13f;
constexpr float kP7 = 0x1.e50106p-17f;

// ---- packed column pairs ----
//
// sm_100 executes FP32 add, multiply and fused multiply-add on float2
// operands (one instruction, two results).  The sweep is bound by
// instruction issue, so each thread evaluates two consecutive columns
// (j, j+1) of a target row in one float2 throughout: differences, exponents,
// the exponential's polynomial and the weighted sums.  The staged tile is a
// structure of arrays (one array per record field, column values negated so
// that differences are additions), so one 8-byte shared load yields a field
// of a column pair; row values are held duplicated in both halves.  A tile
// with an odd number of events is padded with one column whose coordinate
// and time are 1e18 away, so all its terms are exactly zero.

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// 2^(-s) for both halves by Cody-Waite reduction: m = rint(s), f = m - s in
// [-1/2, 1/2] (exact), p(f) by packed Horner on the FMA pipe, times the exact
// power 2^-m from ex2.approx.ftz on the integer -m.  That instruction returns
// exactly 2^n for every integer n (checked on the device for n in [-200,
// 130]), +0 for n <= -127 and +inf above 127, so the scale needs no clamp or
// exponent-field arithmetic and any |s| is safe (for |s| >= 2^23, f = 0).
// Arguments s above 126.5 give +0 as with ex2.approx.ftz, so the tile-level
// underflow skip stays exact.  The hardware approximation error never
// enters: only the exact power of two is taken from it, the fractional part
// is the polynomial's.
__device__ __forceinline__ float2 exp2_poly_neg2(float2 s) {
    const float2 m = make_float2(rintf(s.x), rintf(s.y));
    const float2 f = fma2(s, dup2(-1.0f), m);
    float2 p = fma2(dup2(kP7), f, dup2(kP6));
    p = fma2(p, f, dup2(kP5));
    p = fma2(p, f, dup2(kP4));
    p = fma2(p, f, dup2(kP3));
    p = fma2(p, f, dup2(kP2));
    p = fma2(p, f, dup2(kP1));
    p = fma2(p, f, dup2(1.0f));
    return mul2(p, make_float2(ex2_ftz(-m.x), ex2_ftz(-m.y)));
}

// Background unit terms 2^-(d2 + t2).  In the hardware-exponential variant its
// mean relative error is divided out of the sums in the FP64 finish; far-tail
// terms of the polynomial variant (at most 2^-10 each) keep it.
template <int V>
__device__ __forceinline__ float2 background2(float2 s) {
    if (V & kPolyExp) return exp2_poly_neg2(s);
    return make_float2(ex2_ftz(-s.x), ex2_ftz(-s.y));
}

// Unit self-excitation terms of a column pair, zeroed where t_j >= t_i when
// MASK (ranks: equal times share one).
template <int V, bool MASK>
__device__ __forceinline__ float2 self_excite2(float2 d2, float2 dt, int rank, int2 rj,
                                               const PairConsts& c) {
    const float2 e = fma2(dup2(c.fSh), d2,
                          fma2(dup2(c.fWh), dt, fma2(dup2(c.fSl), d2, mul2(dup2(c.fWl), dt))));
    const float ex = fminf(e.x, 127.0f), ey = fminf(e.y, 127.0f);
    float2 S;
    if (V & kPolyExp) S = exp2_poly_neg2(make_float2(-ex, -ey));
    else S = make_float2(ex2_ftz(ex), ex2_ftz(ey));
    if (MASK) {
        S.x = rank > rj.x ? S.x : 0.0f;
        S.y = rank > rj.y ? S.y : 0.0f;
    }
    return S;
}

// A staged tile: per field, kTile columns (+1 padding column), negated.
template <int D>
struct StagedTile {
    static constexpr int kCols = kTile + 2;  // even stride, room for the padding column
    float nx[D][kCols];   // -x'hi
    float nxl[D][kCols];  // -x'lo
    float nt[kCols];      // -t'hi
    float ntl[kCols];     // -t'lo
    int rank[kCols];
};

// Row values held duplicated for the packed arithmetic.
template <int D, int R>
struct Rows2 {
    float2 xh[R][D], xl[R][D], th[R], tl[R];
    int rk[R];
};

// Squared distance and time difference of row r against column pair p
// (columns 2p, 2p+1 of the staged tile).
template <int D, int R, int V>
__device__ __forceinline__ void geometry2(const StagedTile<D>& t, int p, const Rows2<D, R>& w,
                                          int r, float2& d2, float2& dt) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
        float2 dd = add2(w.xh[r][k], reinterpret_cast<const float2*>(t.nx[k])[p]);
        if (V & kSpaceLo) dd = add2(dd, add2(w.xl[r][k], reinterpret_cast<const float2*>(t.nxl[k])[p]));
        d2 = k == 0 ? mul2(dd, dd) : fma2(dd, dd, d2);
    }
    if (V & kTimeHiOnly)
        dt = add2(w.th[r], reinterpret_cast<const float2*>(t.nt)[p]);
    else
        dt = add2(add2(w.th[r], reinterpret_cast<const float2*>(t.nt)[p]),
                  add2(w.tl[r], reinterpret_cast<const float2*>(t.ntl)[p]));
}

// The time difference the self-excitation terms use: hi + lo always, added
// in the same order as geometry2's full difference.
template <int D, int R, int V>
__device__ __forceinline__ float2 self_dt2(const StagedTile<D>& t, int p, const Rows2<D, R>& w,
                                           int r, float2 dt) {
    if ((V & kTimeHiOnly) && !(V & kPlain))
        return add2(dt, add2(w.tl[r], reinterpret_cast<const float2*>(t.ntl)[p]));
    return dt;
}

// ---- compensated row sums ----
//
// Each of the six sums of a target row is carried as a pair of float2 (even
// and odd columns): hi takes the terms, lo the exact rounding error of every
// addition to hi (Fast2Sum: t = hi + x, error = (hi - t) + x, both steps exact
// when |hi| >= |x|).  The sums are non-negative, so that holds once hi has
// passed the incoming term; when a term larger than hi arrives the step
// rounds like a plain FP32 addition of two comparable numbers (an unbiased
// error of at most half an ulp of the new hi).  What the compensation removes
// is the systematic loss of plain FP32 accumulation: a term below half an ulp
// of the running sum is rounded away entirely, so sums of many small terms
// come out low (measured at N = 100k: about -2.5e-9 relative on every
// background sum, which the cancelling d/d tauX and d/d tauT gradient
// components amplify about 80-fold).
//
// hi starts from PairConsts::rowOffset, a power of two no smaller than any
// single term of the sum, so |hi| >= |x| holds at every addition and each
// error is exact whatever order the terms come in (starting from zero, a
// term larger than the sum so far -- the nearest neighbour arriving late in
// a chunk -- would round with an error Fast2Sum does not see: ~1e-8 of an
// event's sum, moving with the chunk bounds).  Terms far below the offset
// pass to lo whole, where they add up in plain FP32 at their own scale.
// The row value (hi - offset) + lo is formed in FP64 when the work item
// writes its partial sums (hi - offset is exact there: two FP32 values).
//
// Far-tail background terms (each at most 2^-10 of the event's own term, see
// kFastTailLog2) are added to lo directly: lo then carries them and the
// errors, both far below hi, and its own FP32 rounding is below 2^-24 of
// that.
template <int R>
struct RowSums {
    float2 hi[R][kNumAcc];
    float2 lo[R][kNumAcc];
};

template <int R>
__device__ __forceinline__ void start_rows(RowSums<R>& a, const PairConsts& c) {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < kNumAcc; ++q) {
            a.hi[r][q] = make_float2(c.rowOffset[q], c.rowOffset[q]);
            a.lo[r][q] = make_float2(0.0f, 0.0f);
        }
}

// hi += x with the rounding error added to lo.
__device__ __forceinline__ void add_comp(float2& hi, float2& lo, float2 x) {
    const float2 t = add2(hi, x);
    const float2 d = fma2(t, dup2(-1.0f), hi);  // hi - t
    lo = add2(lo, add2(d, x));
    hi = t;
}

// hi += u * v with the rounding error added to lo: t = fma(u, v, hi) rounds
// once; hi - t is exact under the same condition, and fma(u, v, hi - t) is
// that rounding error (the product is exact inside the FMA) rounded to FP32,
// i.e. to 2^-24 of itself.
__device__ __forceinline__ void fma_comp(float2& hi, float2& lo, float2 u, float2 v) {
    const float2 t = fma2(u, v, hi);
    const float2 d = fma2(t, dup2(-1.0f), hi);  // hi - t
    lo = add2(lo, fma2(u, v, d));
    hi = t;
}

// The three background terms of a pair into row r: compensated, or (FAR)
// straight into lo.
template <int R, bool FAR>
__device__ __forceinline__ void add_background(RowSums<R>& a, int r, float2 B, float2 d2,
                                               float2 t2) {
    if (FAR) {
        a.lo[r][0] = add2(a.lo[r][0], B);
        a.lo[r][1] = fma2(B, d2, a.lo[r][1]);
        a.lo[r][2] = fma2(B, t2, a.lo[r][2]);
    } else {
        add_comp(a.hi[r][0], a.lo[r][0], B);
        fma_comp(a.hi[r][1], a.lo[r][1], B, d2);
        fma_comp(a.hi[r][2], a.lo[r][2], B, t2);
    }
}

template <int R, bool PLAIN>
__device__ __forceinline__ void add_self_excite(RowSums<R>& a, int r, float2 S, float2 d2,
                                                float2 dt) {
    if (PLAIN) {  // plain FP32 sums
        a.lo[r][3] = add2(a.lo[r][3], S);
        a.lo[r][4] = fma2(S, d2, a.lo[r][4]);
        a.lo[r][5] = fma2(S, dt, a.lo[r][5]);
    } else {
        add_comp(a.hi[r][3], a.lo[r][3], S);
        fma_comp(a.hi[r][4], a.lo[r][4], S, d2);
        fma_comp(a.hi[r][5], a.lo[r][5], S, dt);
    }
}

// After a far-tail tile pair, lo holds that tile pair's far background terms
// (and the small compensation error carried in): scale them by farScale and
// fold them into hi, leaving lo with the rounding error of that addition.
template <int R>
__device__ __forceinline__ void fold_far(RowSums<R>& a, float farScale) {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float2 x = mul2(a.lo[r][q], dup2(farScale));
            a.lo[r][q] = make_float2(0.0f, 0.0f);
            add_comp(a.hi[r][q], a.lo[r][q], x);
        }
}

// Geometry variant of a tile pair: one that carries self-excitation terms
// takes the coordinate differences from hi + lo parts.  With hi parts alone
// each event's coordinates are off by up to half an FP32 ulp (~6e-7 record
// units), the same offset in every one of its terms; the self-excitation
// sums are short (a few near neighbours), so they would move by ~1e-7 and
// the sigma gradient collect ~1e-8 of that over 100,000 events.  Background
// sums average the offset over thousands of terms (~5e-8 per event, under
// 4e-9 on every gradient component at N = 100,000), so background-only tile
// pairs keep the cheaper hi-only differences.
// The plain FP32 mode uses hi parts only, for times too.
template <int V, bool DO_S>
struct GeomV {
    static constexpr int value = (V & kPlain) ? (V | kTimeHiOnly) : DO_S ? (V | kSpaceLo) : V;
};

// Row-order pass over column pairs [p0, p1) of the staged tile (broadcast
// reads shared by the R rows).  FAR: every background term of the tile pair
// is in the far tail.
template <int D, int R, int V, int VB, bool FAR, bool DO_B, bool DO_S, bool MASK>
__device__ __forceinline__ void body_f32(const StagedTile<D>& t, int p0, int p1,
                                         const Rows2<D, R>& w, const PairConsts& c,
                                         RowSums<R>& a) {
    constexpr int VG = GeomV<V, DO_S>::value;
#pragma unroll 2
    for (int p = p0; p < p1; ++p) {
        const int2 rj = MASK ? reinterpret_cast<const int2*>(t.rank)[p] : make_int2(0, 0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 d2, dt;
            geometry2<D, R, VG>(t, p, w, r, d2, dt);
            if (DO_B) {
                const float2 t2 = mul2(dt, dt);
                const float2 B = background2<VB>(add2(d2, t2));
                add_background<R, FAR || (V & kPlain) != 0>(a, r, B, d2, t2);
            }
            if (DO_S) {
                const float2 dts = self_dt2<D, R, VG>(t, p, w, r, dt);
                const float2 S = self_excite2<VG & ~kTimeHiOnly, MASK>(d2, dts, w.rk[r], rj, c);
                add_self_excite<R, (V & kPlain) != 0>(a, r, S, d2, dts);
            }
        }
    }
}

template <int D, int R, int V, int VB, bool FAR, bool DO_B, bool DO_S, bool MASK>
__device__ __forceinline__ void tile_f32(const StagedTile<D>& t, int nj, const Rows2<D, R>& w,
                                         const PairConsts& c, RowSums<R>& a) {
    body_f32<D, R, V, VB, FAR, DO_B, DO_S, MASK>(t, 0, (nj + 1) / 2, w, c, a);
}

// ---- symmetric background tiles ----
//
// For a tile J before the strip, each pair (i, j) is evaluated once and its
// background terms B, B d'^2, B dt'^2 go to row i (registers, as above) and
// to column j.  Column sums are formed per warp in groups of 8 columns (4
// column pairs): lane l visits the group's pairs in the order m ^ q, q =
// (l >> 3) & 3, so that after the loop its accumulator c[m] holds column pair
// m ^ q summed over the lane's R rows.  A transposing exchange -- float2
// shuffles at distances 16 and 8 that each keep the half of the pairs the
// lane ends with, a split of the pair at distance 4, then sums at 2 and 1 --
// leaves lane l with the warp total of column (l >> 2), with no selects in
// the loop.  The 4 warp totals of a column are added in FP64 in warp order
// and added to the column's fixed-point sum, so the result does not depend
// on CTA order.

constexpr int kSymGroup = 8;  // columns per warp exchange

__device__ __forceinline__ float2 shfl_xor2(float2 v, int d) {
    constexpr unsigned kAll = 0xffffffffu;
    return make_float2(__shfl_xor_sync(kAll, v.x, d), __shfl_xor_sync(kAll, v.y, d));
}

// Warp total of column (lane >> 2) of the group.
__device__ __forceinline__ float sym_exchange(const float2 (&cp)[kSymGroup / 2], bool hi) {
    constexpr unsigned kAll = 0xffffffffu;
    const float2 u0 = add2(cp[0], shfl_xor2(cp[2], 16));
    const float2 u1 = add2(cp[1], shfl_xor2(cp[3], 16));
    const float2 w = add2(u0, shfl_xor2(u1, 8));
    const float keep = hi ? w.y : w.x, give = hi ? w.x : w.y;
    float x = keep + __shfl_xor_sync(kAll, give, 4);
    x += __shfl_xor_sync(kAll, x, 2);
    x += __shfl_xor_sync(kAll, x, 1);
    return x;
}

template <int D, int R, int V, int VB, bool FAR, bool DO_S, bool MASK>
__device__ __forceinline__ void sym_group_f32(const StagedTile<D>& t, int g, int q,
                                              const Rows2<D, R>& w, const PairConsts& c,
                                              RowSums<R>& a, float2 (&cp)[3][kSymGroup / 2]) {
    constexpr int VG = GeomV<V, DO_S>::value;
#pragma unroll
    for (int m = 0; m < kSymGroup / 2; ++m) {
        const int p = g / 2 + (m ^ q);
        const int2 rj = MASK ? reinterpret_cast<const int2*>(t.rank)[p] : make_int2(0, 0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 d2, dt;
            geometry2<D, R, VG>(t, p, w, r, d2, dt);
            const float2 t2 = mul2(dt, dt);
            const float2 B = background2<VB>(add2(d2, t2));
            add_background<R, FAR || (V & kPlain) != 0>(a, r, B, d2, t2);
            if (r == 0) {
                cp[0][m] = B;
                cp[1][m] = mul2(B, d2);
                cp[2][m] = mul2(B, t2);
            } else {
                cp[0][m] = add2(cp[0][m], B);
                cp[1][m] = fma2(B, d2, cp[1][m]);
                cp[2][m] = fma2(B, t2, cp[2][m]);
            }
            if (DO_S) {
                const float2 dts = self_dt2<D, R, VG>(t, p, w, r, dt);
                const float2 S = self_excite2<VG & ~kTimeHiOnly, MASK>(d2, dts, w.rk[r], rj, c);
                add_self_excite<R, (V & kPlain) != 0>(a, r, S, d2, dts);
            }
        }
    }
}

// One full tile J (kTile columns, all real events) before the strip.
// sCol: [kSweepThreads / 32][3][kTile] floats of shared memory.
template <int D, int R, int V, int VB, bool FAR, bool DO_S, bool MASK>
__device__ __forceinline__ void tile_sym_f32(const StagedTile<D>& t, const Rows2<D, R>& w,
                                             const PairConsts& c, RowSums<R>& a,
                                             float* __restrict__ sCol,
                                             unsigned long long* __restrict__ colAcc, int Npad,
                                             int j0) {
    static_assert(kSweepThreads == kTile, "one column per thread in the column flush");
    static_assert(kTile % kSymGroup == 0, "group sizes");
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int q = (lane >> 3) & 3;
    const bool hi = (lane >> 2) & 1;
#pragma unroll 1
    for (int g = 0; g < kTile; g += kSymGroup) {
        float2 cp[3][kSymGroup / 2];
        sym_group_f32<D, R, V, VB, FAR, DO_S, MASK>(t, g, q, w, c, a, cp);
        const float c0 = sym_exchange(cp[0], hi);
        const float c1 = sym_exchange(cp[1], hi);
        const float c2 = sym_exchange(cp[2], hi);
        if ((lane & 3) == 0) {
            float* o = sCol + warp * 3 * kTile + g + (lane >> 2);
            o[0] = c0;
            o[kTile] = c1;
            o[2 * kTile] = c2;
        }
    }
    __syncthreads();
#pragma unroll
    for (int qq = 0; qq < 3; ++qq) {
        double v = 0.0;
#pragma unroll
        for (int wq = 0; wq < kSweepThreads / 32; ++wq)
            v += (double)sCol[(wq * 3 + qq) * kTile + tid];
        if (FAR) v *= (double)c.farScale;
        atomicAdd(colAcc + (size_t)qq * Npad + j0 + tid,
                  (unsigned long long)__double2ll_rn(v * kColScale));
    }
}

// One FP32 record (S floats, S a multiple of 4, rows 16-byte aligned) by
// coalesced 16-byte loads: consecutive threads read consecutive records.
template <int S>
__device__ __forceinline__ void load_record_f32(const float* __restrict__ rec, int i,
                                                float (&out)[S]) {
    static_assert(S % 4 == 0, "FP32 records are whole float4s");
    const float4* r4 = reinterpret_cast<const float4*>(rec + (size_t)i * S);
#pragma unroll
    for (int q = 0; q < S / 4; ++q) {
        const float4 v = __ldg(r4 + q);
        out[4 * q] = v.x;
        out[4 * q + 1] = v.y;
        out[4 * q + 2] = v.z;
        out[4 * q + 3] = v.w;
    }
}

// One work item of the FP32-compensated sweep (see f64_item).
template <int D, int R, int V>
__device__ __forceinline__ void f32c_item(const float* __restrict__ rec,
                                          const double* __restrict__ tileMin,
                                          const double* __restrict__ tileMax,
                                          double* __restrict__ partials,
                                          unsigned long long* __restrict__ colAcc, int N,
                                          int nTiles, int Npad, bool sym, const PairConsts& c,
                                          int strip, int jt0, int jt1, int slot,
                                          const int32_t* __restrict__ rowOrder,
                                          StagedTile<D>& st, float* sCol) {
    constexpr int S = Layout<D>::kF32Stride;
    const int tid = threadIdx.x;
    const int stripBase = strip * kSweepThreads * R;
    const int ts0 = stripBase / kTile, ts1 = min(ts0 + R, nTiles);
    // full strips read their rows through the spatial row order
    const bool ordered = rowOrder != nullptr && stripBase + kSweepThreads * R <= N;

    Rows2<D, R> w;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int iRaw = stripBase + r * kSweepThreads + tid;
        const int i = ordered ? rowOrder[iRaw] : min(iRaw, N - 1);
        float ri[S];
        load_record_f32<S>(rec, i, ri);
#pragma unroll
        for (int k = 0; k < D; ++k) {
            w.xh[r][k] = dup2(ri[k]);
            w.xl[r][k] = dup2(ri[D + 1 + k]);
        }
        w.th[r] = dup2(ri[D]);
        w.tl[r] = dup2(ri[2 * D + 1]);
        w.rk[r] = __float_as_int(ri[2 * D + 2]);
        if (iRaw >= N) {
            // Padding rows of the last strip: a time 1e18 away makes every
            // background term exactly +0 (exponent ~ -1e36, finite), so they
            // add nothing to the column sums; their own rows are discarded.
            w.th[r] = dup2(1e18f);
            w.tl[r] = dup2(0.0f);
        }
    }
    double tminI = INFINITY, tmaxI = -INFINITY;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int tt = stripBase / kTile + r;
        if (tt < nTiles) {
            tminI = fmin(tminI, tileMin[tt]);
            tmaxI = fmax(tmaxI, tileMax[tt]);
        }
    }
    RowSums<R> acc;
    start_rows<R>(acc, c);

    for (int jt = jt0; jt < jt1; ++jt) {
        TileMode m = tile_mode(tminI, tmaxI, tileMin[jt], tileMax[jt], c);
        // plain FP32: causal only where the FP32-rounded times differ, so a
        // tile pair with equal rounded bounds keeps the rank mask
        if (V & kPlain) m.allCausal = m.allCausal && (float)tminI > (float)tileMax[jt];
        if (sym && jt >= ts1) m.doB = false;  // covered as columns by later strips
        if (!m.doB && !m.doS) continue;
        const int j0 = jt * kTile;
        const int nj = min(kTile, N - j0);
        __syncthreads();
        // stage the tile: one thread per column, fields negated
        if (tid < nj) {
            float rj[S];
            load_record_f32<S>(rec, j0 + tid, rj);
#pragma unroll
            for (int k = 0; k < D; ++k) {
                st.nx[k][tid] = -rj[k];
                st.nxl[k][tid] = -rj[D + 1 + k];
            }
            st.nt[tid] = -rj[D];
            st.ntl[tid] = -rj[2 * D + 1];
            st.rank[tid] = __float_as_int(rj[2 * D + 2]);
        } else if (tid == nj && (nj & 1)) {
            // padding column of an odd tile: coordinate and time 1e18 away
#pragma unroll
            for (int k = 0; k < D; ++k) {
                st.nx[k][tid] = -1e18f;
                st.nxl[k][tid] = 0.0f;
            }
            st.nt[tid] = 1e18f;
            st.ntl[tid] = 0.0f;
            st.rank[tid] = INT_MAX;
        }
        __syncthreads();
        // Warm L1 with the next tile's records (one 128-byte line per four
        // threads) while this tile is evaluated: its staging then waits on L1
        // hits instead of L2 (1.3 % of the headline sweep).
        if (jt + 1 < jt1 && j0 + kTile + tid < N && (tid & 3) == 0)
            prefetch_l1(rec + (size_t)(j0 + kTile + tid) * S);
        // Far-tail tile pairs take their background terms from the hardware
        // exponential.  The choice depends on the background magnitude alone,
        // so the underflow skip (which may drop the pair's self-excitation
        // terms) never changes it.  A far-tail pair has min|dt| > 0: its j
        // events are all earlier than its i events or all later, so it needs
        // no causality mask.
        constexpr int VF = V & ~kPolyExp;         // background exponential of far tiles
        constexpr int VG = V | kTimeHiOnly;        // their geometry: hi parts of the times
        if (sym && m.doB && jt < ts0) {
            // jt < ts0 <= nTiles - 1: a full tile
            if (m.fastB && !m.doS)
                tile_sym_f32<D, R, VG, VF, true, false, false>(st, w, c, acc, sCol, colAcc, Npad,
                                                               j0);
            else if (m.fastB)
                tile_sym_f32<D, R, VG, VF, true, true, false>(st, w, c, acc, sCol, colAcc, Npad,
                                                              j0);
            else if (!m.doS)
                tile_sym_f32<D, R, V, V, false, false, false>(st, w, c, acc, sCol, colAcc, Npad,
                                                              j0);
            else if (m.allCausal)
                tile_sym_f32<D, R, V, V, false, true, false>(st, w, c, acc, sCol, colAcc, Npad,
                                                             j0);
            else
                tile_sym_f32<D, R, V, V, false, true, true>(st, w, c, acc, sCol, colAcc, Npad,
                                                            j0);
        } else if (m.doB) {
            if (m.fastB && !m.doS)
                tile_f32<D, R, VG, VF, true, true, false, false>(st, nj, w, c, acc);
            else if (m.fastB)
                tile_f32<D, R, VG, VF, true, true, true, false>(st, nj, w, c, acc);
            else if (!m.doS)
                tile_f32<D, R, V, V, false, true, false, false>(st, nj, w, c, acc);
            else if (m.allCausal)
                tile_f32<D, R, V, V, false, true, true, false>(st, nj, w, c, acc);
            else
                tile_f32<D, R, V, V, false, true, true, true>(st, nj, w, c, acc);
        } else {
            if (m.allCausal)
                tile_f32<D, R, V, V, false, false, true, false>(st, nj, w, c, acc);
            else
                tile_f32<D, R, V, V, false, false, true, true>(st, nj, w, c, acc);
        }
        if (m.doB && m.fastB) fold_far<R>(acc, c.farScale);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int iRaw = stripBase + r * kSweepThreads + tid;
        const int i = ordered ? rowOrder[iRaw] : iRaw;
        if (iRaw < N) {
#pragma unroll
            for (int q = 0; q < kNumAcc; ++q)
                // a self-excitation-only sweep leaves the background rows to
                // the kept sums: they are neither written nor read
                if (q >= 3 || !c.noB)
                    partials[((size_t)slot * kNumAcc + q) * Npad + i] =
                        (((double)acc.hi[r][q].x - (double)c.rowOffset[q]) +
                         ((double)acc.hi[r][q].y - (double)c.rowOffset[q])) +
                        ((double)acc.lo[r][q].x + (double)acc.lo[r][q].y);
        }
    }
}

// R = 2 fits 128 registers (4 CTAs per SM); R = 4 holds twice the rows and
// column partials and runs 2 CTAs per SM.
template <int D, int R, int V>
__global__ void __launch_bounds__(kSweepThreads, (R <= 2 ? 4 : 2))
sweep_f32c_list_kernel(const SweepProblem* __restrict__ problems,
                       const WorkItem* __restrict__ items, const int* __restrict__ nItems,
                       int* __restrict__ counter) {
    __shared__ __align__(16) StagedTile<D> sTile;
    __shared__ __align__(16) float sCol[(kSweepThreads / 32) * 3 * kTile];
    __shared__ int sNext;
    const int n = *nItems;
    for (;;) {
        const int it = next_item(counter, &sNext);
        if (it >= n) break;
        const WorkItem w = items[it];
        const SweepProblem& P = problems[w.problem];
        const PairConsts c = P.c;
        f32c_item<D, R, V>(static_cast<const float*>(P.rec), P.tileMin, P.tileMax, P.partials,
                           P.colAcc, P.N, P.nTiles, P.Npad, P.symmetric != 0, c, w.strip, w.start,
                           w.jt1, w.slot, P.rowOrder, sTile, sCol);
    }
}

template <int D, int R>
cudaError_t sweep_list_dispatch_v(int precision, int V, int grid, const SweepProblem* problems,
                                  const WorkItem* items, const int* nItems, int* counter,
                                  cudaStream_t s, int* blocksPerSM) {
    const void* fn = nullptr;
    if (precision == 0) {
        if (R > 2) return cudaErrorInvalidValue;
        fn = reinterpret_cast<const void*>(&sweep_f64_list_kernel<D, (R > 2 ? 2 : R)>);
    } else {
        if (R < 2) return cudaErrorInvalidValue;
        switch (V) {
            case 0: fn = reinterpret_cast<const void*>(&sweep_f32c_list_kernel<D, (R < 2 ? 2 : R), 0>); break;
            case 1: fn = reinterpret_cast<const void*>(&sweep_f32c_list_kernel<D, (R < 2 ? 2 : R), 1>); break;
            case 2: fn = reinterpret_cast<const void*>(&sweep_f32c_list_kernel<D, (R < 2 ? 2 : R), 2>); break;
            case 3: fn = reinterpret_cast<const void*>(&sweep_f32c_list_kernel<D, (R < 2 ? 2 : R), 3>); break;
            case kPlain: fn = reinterpret_cast<const void*>(&sweep_f32c_list_kernel<D, (R < 2 ? 2 : R), kPlain>); break;
            default: return cudaErrorInvalidValue;
        }
    }
    if (blocksPerSM) {
        *blocksPerSM = 0;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, fn, kSweepThreads, 0);
    }
    void* args[] = {(void*)&problems, (void*)&items, (void*)&nItems, (void*)&counter};
    return cudaLaunchKernel(fn, dim3(grid), dim3(kSweepThreads), args, 0, s);
}

template <int D>
cudaError_t sweep_list_dispatch_r(int precision, int R, int V, int grid,
                                  const SweepProblem* problems, const WorkItem* items,
                                  const int* nItems, int* counter, cudaStream_t s,
                                  int* blocksPerSM) {
    switch (R) {
        case 1: return sweep_list_dispatch_v<D, 1>(precision, V, grid, problems, items, nItems,
                                                   counter, s, blocksPerSM);
        case 2: return sweep_list_dispatch_v<D, 2>(precision, V, grid, problems, items, nItems,
                                                   counter, s, blocksPerSM);
        case 4: return sweep_list_dispatch_v<D, 4>(precision, V, grid, problems, items, nItems,
                                                   counter, s, blocksPerSM);
        default: return cudaErrorInvalidValue;
    }
}

template <int D>
cudaError_t sweep_grid_f64_dispatch(int R, const SweepGeometry& g, const double* rec,
                                    const double* tileMin, const double* tileMax,
                                    const PairConsts& c, double* partials, cudaStream_t s) {
    const int grid = g.nStrips * g.nChunks;
    if (R == 1)
        sweep_f64_kernel<D, 1><<<grid, kSweepThreads, 0, s>>>(g, rec, tileMin, tileMax, c,
                                                             partials);
    else if (R == 2)
        sweep_f64_kernel<D, 2><<<grid, kSweepThreads, 0, s>>>(g, rec, tileMin, tileMax, c,
                                                             partials);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace
}  // namespace hphc
