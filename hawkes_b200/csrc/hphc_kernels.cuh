// Device-side layout and launch interface of the Hawkes pair-sum kernels.
//
// Data layout in HBM (one event set of N events, D spatial dimensions):
//   FP64 records  : N x kF64Stride<D> doubles, {x_0..x_{D-1}, t, pad}, 16-byte rows.
//   FP32 records  : N x kF32Stride<D> floats,
//                   {xhi_0..xhi_{D-1}, thi, xlo_0..xlo_{D-1}, tlo, rank, pad},
//                   16-byte rows; hi = float(v), lo = float(v - hi) so that
//                   hi + lo carries v to ~2^-48 relative, and rank is the dense
//                   rank of t (equal times share a rank) stored as int bits, so
//                   the strict "t_j < t_i" self-excitation mask
//                   (src/NewHawkes.hpp:540) is an exact integer compare.
//   tile bounds   : per kTile-event tile, FP64 min and max of t.
//   partials      : [chunk][6][Npad] FP64 unit pair sums per target event i.
//   block partials: [block][8] FP64 per-block sums of the per-event
//                   log-likelihood and gradient contributions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hphc {

constexpr int kMaxDim = 8;
constexpr int kSweepThreads = 128;   // threads per sweep CTA
constexpr int kTile = 128;           // j events staged in shared memory per step
constexpr int kFinishThreads = 256;  // threads per finish CTA
constexpr int kNumAcc = 6;           // unit pair sums per target event

template <int D>
struct Layout {
    static constexpr int kF64Stride = ((D + 1) + 1) / 2 * 2;          // doubles per FP64 record
    static constexpr int kF32Used = 2 * (D + 1) + 1;                   // hi, lo, rank
    static constexpr int kF32Stride = (kF32Used + 3) / 4 * 4;          // floats per FP32 record
};

// Per-parameter-vector constants of the pair terms.  Unit terms (no
// prefactor):  B_u = exp(cA d^2 + cB dt^2) for every pair,
//              S_u = exp(cS d^2 + cW dt)   for dt > 0,
// with cA = -a^2/2, cB = -b^2/2, cS = -sigma^2/2, cW = -omega.
struct PairConsts {
    double cA, cB, cS, cW;                 // natural-log units (FP64 path)
    // FP32 path, on records scaled by sX = |a| sqrt(log2(e)/2), sT = |b| sqrt(log2(e)/2):
    // S exponent (log2 units) = kS |dx'|^2 + kW dt' with kS = -sigma^2 / a^2 and
    // kW = -omega log2(e) / sT, each split hi + lo.
    float fSh, fSl, fWh, fWl;
    // Tile-pair skips.  A tile pair is skipped for B when cA <= 0, cB < 0 and
    // -cB * min|dt|^2 >= skipB: every B_u in it is exactly zero in the working
    // precision, or (tail truncation) at most 2^-kNegligibleLog2.  S is
    // skipped only where every S_u underflows: -cW * min(dt) >= skipS.
    double skipB, skipS;                   // natural-log thresholds; < 0 disables
    // A tile pair whose background terms are all below exp(-fastB) (natural
    // log; <= 0 disables) takes them from the hardware ex2.approx: instead of
    // the polynomial in the FP32 mode (2^-10, kFastTailLog2), of CUDA's exp()
    // in the FP64 mode (2^-60, kFastTailLog2F64).
    double fastB;
    // Self-excitation-only sweep: no background term is evaluated (the
    // finish takes the background sums from an earlier sweep, which depend
    // on tauX and tauT only).
    int noB;
    // FP32 software-exponential mode: factor applied to the far-tail
    // background terms, which come from ex2.approx: 1 / (1 + its mean
    // relative error measured on the device).
    float farScale;
    // FP32-compensated mode: the value each row sum's hi part starts from, a
    // power of two at least as large as any single unit term of that sum
    // (B_u, S_u <= 1; B_u d'^2, B_u dt'^2 <= 1/(e ln 2); S_u d'^2 <=
    // 1/(e ln 2 |kS|); S_u dt' <= 1/(e ln 2 |kW|)), and at least 1.  Every
    // addition to hi then has |hi| >= |term|, so its Fast2Sum error is exact
    // whatever order the terms come in.  Zero in the other modes.
    float rowOffset[kNumAcc];
};

// Constants of the per-event finish (all FP64).
struct FinishConsts {
    double sigma, a, b, omega, theta, mu0;
    double prefB;     // mu0 a^D b / (2 pi)      : B_ij = prefB * B_u
    double prefS;     // theta omega sigma^D / sqrt(2 pi) : S_ij = prefS * S_u
    double bgScale;   // prefB / mu0
    double seScale;   // prefS / theta
    double accScale[6];  // multiplies the six unit pair sums: undoes the record scaling
                         // and, with the hardware exponential, divides out its mean
                         // relative error (1 + beta, measured on the device)
    double T;         // t[N-1]
    double constant;  // N (D-1) log(1/sqrt(2 pi))
    int D;
    int plain32;      // FP32 throughout: the per-event finish in float (the reference's
                      // single precision, src/factory.cpp:45)
};

// What param_consts needs besides the parameters: fixed per engine (mode)
// or per set.
struct ConstsSpec {
    int precision;    // HPHC_PRECISION_* (0 = FP64)
    int D;
    int variant;      // FP32 variant bits (2 = software exponential, 8 = plain FP32)
    int skip;         // tile-level underflow skip on
    int truncate;     // background tail truncation at 2^-kNegligibleLog2 (needs skip)
    double ex2Bias;   // mean relative error of ex2.approx (FP32 modes: divided out of the
                      // sums of the hardware-exponential variant, and of the far-tail
                      // terms of the software-exponential one)
    int fastTail;     // far-tail tile pairs use the hardware exponential (FP32 software-
                      // exponential variant, and FP64)
    int noB;          // self-excitation-only sweep (PairConsts::noB)
};

// Far background tail of the FP32 software-exponential mode.  A tile pair
// whose background terms are all at most 2^-kFastTailLog2 of an event's own
// term (B_ii = 1 unit) evaluates them with ex2.approx instead of the
// polynomial.  Such terms lie beyond 3.16 scale units of the time Gaussian
// (3.8 of its standard deviations).  At the headline density they carry
// about 1.7e-4 of an event's background sum and 2.8e-3 of its sum weighted
// by dt'^2 (4e-3 at most over 400 sampled events), so the hardware
// exponential's relative error (< 1e-7, its mean divided out) moves those
// sums by ~1e-10.  Measured at N = 100k against the oracle: 2^-10 is 2.4 %
// faster than 2^-12 with the d/d tauT error 3.8e-9 -> 2.8e-9 (and lower at
// N = 20k and 40k); 2^-8 is 5.7 % faster but puts d/d tauT at 2.8e-8.
constexpr double kFastTailLog2 = 10.0;

// FP64 mode: a tile pair whose background terms are all at most 2^-60 takes
// them from the FP32 hardware exponential (relative error ~1e-7; zero below
// 2^-126).  All such terms of one event add up to at most N 2^-60 of its own
// term, so their error moves its sums by under N * 1e-25: below FP64
// rounding for any N this engine holds.
constexpr double kFastTailLog2F64 = 60.0;

// Underflow thresholds (natural-log units) for the tile-pair skip.  FP32:
// both exponentials return +0 for any argument below -126.5 (log2 units); a
// true exponent <= -88 is <= -126.96 in log2 units, which the FP32 rounding
// of the computed exponent (relative ~1e-6) cannot lift above -126.5.  FP64:
// exp(x) is +0 for x < -745.14; -760 leaves a wide margin.
constexpr double kSkipF32 = 88.0;
constexpr double kSkipF64 = 760.0;

// Background tail truncation.  Every event's background sum holds its own
// term, B_ii = 1 unit, the largest of all its terms.  A tile pair whose
// background terms are all at most 2^-T units is skipped: the skipped terms
// of one event add up to at most N 2^-T of its sum, and those weighted by a
// squared scaled distance x (the gradient sums) to at most x e^-x <= T 2^-T
// each, since x >= T ln 2 there.  FP64 mode: T = 91, so N 2^-91 <= 2^-60
// (N < 2^31), below FP64 rounding of the sums; at b = 1/336 per hour the
// cut falls at |dt| = 11.2 / b = 3774 h (FP64 underflow never cuts inside an
// 8760 h span).  FP32 modes: T = 60, so N 2^-60 <= 2^-33 = 1.2e-10 for any
// N the symmetric sweep holds (2^27), far below their own rounding; the cut
// falls at |dt| = 9.1 / b = 3070 h, against 13.3 / b for FP32 underflow.
// The self-excitation sums have no such lower bound and keep the underflow
// skip only.
constexpr double kNegligibleLog2 = 91.0;
constexpr double kNegligibleLog2F32 = 60.0;

// The parameter-dependent constants of one problem: every PairConsts field
// and every FinishConsts field except T and constant (which depend on the
// event set only).  Written for host and device alike with products for the
// integer powers and the correctly rounded sqrt as the only library call, so
// both give the same bits (the device-resident sampler rewrites them there).
#ifdef __CUDACC__
__host__ __device__
#endif
inline void param_consts(const double* p, const ConstsSpec& s, PairConsts& c, FinishConsts& f) {
    const double kLog2eC = 1.44269504088896340735992468100189214;
    const double kTwoPiC = 6.28318530717958647692528676655900577;
    const double kInvSqrt2PiC = 0.398942280401432677939946059934;
    const double sigma = p[0], a = p[1], b = p[2], omega = p[3];
    const bool fp32 = s.precision != 0;
    c.cA = -0.5 * a * a;
    c.cB = -0.5 * b * b;
    c.cS = -0.5 * sigma * sigma;
    c.cW = -omega;
    const double recScale = sqrt(0.5 * kLog2eC);  // record scale per unit precision
    const double sX = fabs(a) * recScale, sT = fabs(b) * recScale;
    if (fp32) {
        const double kS = -(sigma * sigma) / (a * a), kW = -omega * kLog2eC / sT;
        c.fSh = (float)kS;
        c.fSl = (float)(kS - (double)c.fSh);
        c.fWh = (float)kW;
        c.fWl = (float)(kW - (double)c.fWh);
    } else {
        c.fSh = c.fSl = c.fWh = c.fWl = 0.0f;
    }
    const double kLn2 = 0.693147180559945309417232121458176568;
    const double thr = fp32 ? kSkipF32 : kSkipF64;
    const double thrB =
        s.truncate ? fmin(thr, (fp32 ? kNegligibleLog2F32 : kNegligibleLog2) * kLn2) : thr;
    c.skipB = (s.skip && c.cB < 0.0 && c.cA <= 0.0) ? thrB : -1.0;
    c.skipS = (s.skip && c.cW < 0.0 && c.cS <= 0.0) ? thr : -1.0;
    c.fastB = (s.fastTail && (!fp32 || (s.variant & 2)) && c.cB < 0.0 && c.cA <= 0.0)
                  ? (fp32 ? kFastTailLog2 : kFastTailLog2F64) * kLn2
                  : -1.0;
    c.noB = s.noB;
    c.farScale = (fp32 && (s.variant & 2)) ? (float)(1.0 / (1.0 + s.ex2Bias)) : 1.0f;
    for (int q = 0; q < kNumAcc; ++q) c.rowOffset[q] = 0.0f;
    if (fp32 && !(s.variant & 8)) {
        const double kMaxUe = 0.53071497680680994;  // max of u 2^-u over u >= 0: 1/(e ln 2)
        const double kS = fabs((double)c.fSh + (double)c.fSl);
        const double kW = fabs((double)c.fWh + (double)c.fWl);
        const double bound[kNumAcc] = {1.0, kMaxUe, kMaxUe, 1.0,
                                       kS > 0.0 ? kMaxUe / kS : 1e30,
                                       kW > 0.0 ? kMaxUe / kW : 1e30};
        for (int q = 0; q < kNumAcc; ++q) {
            double h = 1.0;
            while (h < bound[q] && h < 0x1p100) h *= 2.0;
            c.rowOffset[q] = (float)h;
        }
    }

    double aD = 1.0, sigmaD = 1.0;
    for (int k = 0; k < s.D; ++k) {
        aD *= a;
        sigmaD *= sigma;
    }
    f.sigma = sigma;
    f.a = a;
    f.b = b;
    f.omega = omega;
    f.theta = p[4];
    f.mu0 = p[5];
    f.bgScale = aD * b / kTwoPiC;
    f.seScale = omega * sigmaD * kInvSqrt2PiC;
    f.prefB = f.mu0 * f.bgScale;
    f.prefS = f.theta * f.seScale;
    for (int q = 0; q < kNumAcc; ++q) f.accScale[q] = 1.0;
    if (fp32) {
        f.accScale[1] = f.accScale[4] = 1.0 / (sX * sX);  // sums of d'^2
        f.accScale[2] = 1.0 / (sT * sT);                  // sum of dt'^2
        f.accScale[5] = 1.0 / sT;                         // sum of dt'
        if (!(s.variant & (2 | 8)))  // hardware exponential: divide out its mean relative
            for (int q = 0; q < kNumAcc; ++q) f.accScale[q] /= 1.0 + s.ex2Bias;  // error
    }
    f.D = s.D;
    f.plain32 = (fp32 && (s.variant & 8)) ? 1 : 0;
}

struct SweepGeometry {
    int N;            // events
    int Npad;         // stride of the partials arrays (>= N)
    int nTiles;       // ceil(N / kTile)
    int nChunks;      // j-ranges per strip
    int chunkTiles;   // tiles per j-range
    int nStrips;      // ceil(N / strip size)
};

// ---- launchers (return cudaError_t of the launch) ---------------------------

// Pack FP64 locations (N x D row-major) and times into the kernel records and
// compute per-tile time bounds.  ranks may be null for the FP64 layout.
cudaError_t launch_pack_f64(int D, int N, const double* loc, const double* times, double* rec,
                            double* tileMin, double* tileMax, cudaStream_t s);
// Per-tile time bounds; tileChanges (nullable) receives each tile's count of
// events whose time differs from the previous event's (floatTimes: after
// rounding both to FP32).
cudaError_t launch_tile_bounds(int N, const double* times, double* tileMin, double* tileMax,
                               int* tileChanges, cudaStream_t s, int floatTimes = 0);
// Dense time ranks of SORTED times from the tile counts of launch_tile_bounds
// (which it overwrites with their exclusive prefix sums): rank[j] = number of
// k in 1..j with t_k != t_{k-1}.  Two launches.
cudaError_t launch_sorted_ranks(int N, const double* times, int* tileChanges, int32_t* ranks,
                                cudaStream_t s, int floatTimes = 0);

// Target-row order of the FP32 symmetric sweep with R events per thread:
// within each full strip of 128 R events, rows sorted along a Morton curve of
// their first two coordinates and dealt to threads in runs of R (spatial
// neighbours share a thread); the last partial strip keeps its order.  One
// or two launches.
cudaError_t launch_strip_order(int D, int N, int R, const double* loc, int32_t* order,
                               cudaStream_t s);

// Pair sweep: fills partials[chunk][6][Npad] with unit pair sums.  R is the
// number of target events per thread (strip = kSweepThreads * R events).
cudaError_t launch_sweep_f64(int D, int R, const SweepGeometry& g, const double* rec,
                             const double* tileMin, const double* tileMax, const PairConsts& c,
                             double* partials, cudaStream_t s);


// Per-event finish: combines the chunk partials of each event in chunk order,
// forms lambda_i, the log-likelihood and gradient contributions and (if probs
// is non-null) P_i, and writes one 8-double block sum per finish CTA.
cudaError_t launch_finish(const SweepGeometry& g, const double* partials, const double* times,
                          const FinishConsts& f, double* blockSums, double* probs,
                          cudaStream_t s);

// Fixed-order reduction of the block sums: out[0] = log-likelihood (with the
// constant), out[1..6] = gradient.
cudaError_t launch_final(int nBlocks, const double* blockSums, const FinishConsts& f, double* out,
                         cudaStream_t s);

// Calibration of the FP32 exponential: writes ceil(n / kFinishThreads) CTA
// sums of (ex2.approx(x) / 2^x - 1) for n arguments spread over [-16, 0).
cudaError_t launch_ex2_bias(int n, double* blockSums, cudaStream_t s);

// Test of the FP32 sweep's exponentials: poly[k] = 2^-s[k] by the software
// exponential, hw[k] = ex2.approx.ftz(-s[k]); s[k] >= 0, device arrays of n.
cudaError_t launch_eval_exponentials(int n, const float* s, float* poly, float* hw,
                                     cudaStream_t st);

// Number of finish CTAs for N events.
inline int finish_blocks(int N) { return (N + kFinishThreads - 1) / kFinishThreads; }

// ---- work-list execution ---------------------------------------------------
//
// A "problem" is one event set evaluated at one parameter vector.  One launch
// of each stage serves any number of problems: a single evaluation, K
// parameter vectors on one set (MCMC proposals), or many sets of uneven size.

// Fixed-point scale of the column sums of the symmetric sweep (2^36): the
// sums are non-negative and below 2^27 (at most N terms of at most 1), so
// they fit an unsigned 64-bit integer, and integer addition makes them
// independent of the order in which CTAs add to them.
constexpr double kColScale = 68719476736.0;
constexpr double kColInv = 1.0 / 68719476736.0;
constexpr int kMaxSymmetricEvents = 1 << 27;
// FP64 symmetric sweep: each column sum is two unsigned 64-bit words, hi in
// units of 2^-colShift[q] and lo in units of 2^-(colShift[q] + kColLoBits),
// the shift chosen per problem so that a column total stays below 2^62
// units of hi (resolution of the pair ~2^-(colShift + 40), far below FP64
// rounding of the sums).
constexpr int kColLoBits = 40;

// Pair-sweep view of a problem.
//
// Symmetric sweeps (FP32 records): the background kernel B_ij is symmetric,
// so a strip of targets i evaluates each pair with an earlier tile once and
// adds it to both its own rows and, as fixed-point column sums in colAcc, to
// the rows of the earlier tile; pairs inside the strip's own tiles are
// evaluated in both orders, and tiles after the strip carry only
// self-excitation terms (zero for sorted times).
struct SweepProblem {
    const void* rec;        // FP64 or FP32 records (FP32: scaled for this problem)
    const double* tileMin;  // per kTile-event tile of the problem's set
    const double* tileMax;
    double* partials;       // [slot][6][Npad]
    unsigned long long* colAcc;  // background column sums, or null: FP32 [3][Npad] x kColScale;
                                 // FP64 [3][2][Npad] two-word fixed point (see kColLoBits)
    int N, nTiles, Npad, symmetric;
    int colShift[4];        // FP64 column sums: fixed-point shift per weighted sum
    // Items may start far before the first tile holding a term (plans built
    // for any sigma and omega, sorted times): the sweep finds that tile by
    // bisection on the tile time bounds instead of scanning to it.
    int searchBand, pad[3];
    // FP32 sweep: event of row r of thread t of a full strip, at
    // [stripBase + r * 128 + t] (launch_strip_order for the sweep's R), or
    // null for the identity order.
    const int32_t* rowOrder;
    PairConsts c;
};

// One unit of sweep work: target strip `strip` of problem `problem` against j
// tiles [jt0, jt1), written to partial-sum slot `slot` of that strip.  The
// host lists items largest first; CTAs take them in that order from an atomic
// counter, so slow and fast items balance across SMs, and every item writes
// fixed slots, so results do not depend on which CTA ran it.  The sweep
// starts at tile `start`: jt0, or in the device-resident loop the first tile
// not ruled out by its time gap for the current constants (band_starts).
struct WorkItem {
    int problem, strip, jt0, jt1, slot, start, pad1, pad2;
};

constexpr int kBandThreads = 256;

// Device-resident loop: items[k].start for the first *nItems items (maxItems
// bounds the grid), from each problem's current constants where searchBand is
// set, else jt0.
cudaError_t launch_band_starts(int maxItems, const SweepProblem* problems, WorkItem* items,
                               const int* nItems, int R, cudaStream_t s);

// Finish view of a problem.
struct FinishProblem {
    const double* partials;   // [slot][6][Npad]
    const unsigned long long* colAcc;  // [3][Npad] symmetric-sweep column sums, or null
    const int* stripChunks;   // slots used by each strip
    const double* times;      // the set's raw times
    double* probs;            // P_i output (may be null)
    double* sums;             // [6][N] unit pair sums out, natural units (may be null)
    const double* keptB;      // [3][N] background unit sums (natural units) of an earlier
                              // sweep on the same events and tauX, tauT, used instead of
                              // this sweep's (which then has no background terms), or null
    int N, Npad, stripEvents, blockBase;  // blockBase: first finish CTA of this problem
    int nBlocks, colWords, pad0, pad1;    // colWords: 1 = FP32 column format, 2 = FP64
    int colShift[4];
    FinishConsts f;
};

struct FinishBlock {
    int problem, i0;
};

// FP32 record build for one problem.
struct PackJob {
    const double* loc;
    const double* times;
    const int32_t* ranks;
    float* rec;
    double sX, sT;
    int N, pad;
};

cudaError_t launch_pack_f32_jobs(int D, int nJobs, int maxN, const PackJob* jobs, cudaStream_t s);

// Persistent sweep over a work list: `grid` CTAs take items from *counter
// (which must be 0 at launch) until *nItems are taken.  precision: 0 = FP64,
// 1 = FP32-compensated with variant V.
cudaError_t launch_sweep_list(int precision, int D, int R, int V, int grid,
                              const SweepProblem* problems, const WorkItem* items,
                              const int* nItems, int* counter, cudaStream_t s);

// Resident CTAs per SM of that sweep kernel (0 if the configuration is invalid).
int sweep_list_blocks_per_sm(int precision, int D, int R, int V);

cudaError_t launch_finish_list(int nBlocks, const FinishProblem* problems,
                               const FinishBlock* blocks, double* blockSums, cudaStream_t s);

// out[8p .. 8p+7] for every problem p: log-likelihood, gradient, 0.
cudaError_t launch_final_list(int nProblems, const FinishProblem* problems,
                              const double* blockSums, double* out, cudaStream_t s);

// ---- incremental evaluation ------------------------------------------------
//
// After an evaluation the engine can keep each event's six unit pair sums
// (natural units, FP64, [6][N]).  When one event k moves and the parameters
// are unchanged, every other event's sums change only by its pair with k, and
// k's own sums are one O(N) row: the update is O(N) instead of the O(N^2)
// sweep.

struct MovedEvent {
    double oldLoc[kMaxDim];  // the location the sums were computed with
    int k;                   // event index
    int pad;
};

// sums[q][i] += u_q(i, k at its new location) - u_q(i, k at oldLoc) for every
// i != k (one thread per event, FP64), and per-CTA partial sums of event k's
// new row over all j (rowPartials[cta][6]).  loc: N x D raw coordinates
// (event k already at its new location), times: N raw times.
cudaError_t launch_move_event(int D, int N, const MovedEvent& m, const double* loc,
                              const double* times, const PairConsts& c, double* sums,
                              double* rowPartials, cudaStream_t s);
// sums[q][k] = fixed-order sum of the launch's row partials.
cudaError_t launch_move_event_row(int N, int k, const double* rowPartials, double* sums,
                                  cudaStream_t s);
// Per-event finish from kept sums (natural units) and the fixed-order total:
// out[0] = log-likelihood, out[1..6] = gradient, out[7] = 0; probs may be null.
cudaError_t launch_finish_sums(int N, const double* sums, const double* times,
                               const FinishConsts& f, double* blockSums, double* probs,
                               double* out, cudaStream_t s);
// CTAs of launch_move_event for N events.
int move_event_blocks(int N);

}  // namespace hphc
