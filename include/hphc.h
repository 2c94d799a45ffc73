/*
 * hphc.h -- C ABI of the B200 CUDA Hawkes likelihood engine (libhawkes_b200.so).
 *
 * The engine evaluates the O(N^2) spatio-temporal Hawkes log-likelihood of
 * hpHawkes, its analytic parameter gradient and the per-event
 * self-excitation probabilities on one NVIDIA B200 (sm_100a).  These entry
 * points are what a binding of the reference's engine interface
 * hph::AbstractHawkes (src/AbstractHawkes.hpp:32-60) calls: the header-only
 * adapter include/hawkes_b200/CudaHawkes.hpp wraps them in a class deriving
 * from hph::AbstractHawkes, and Rcpp / JNI / ctypes bindings can call them
 * directly.
 *
 * Conventions
 *   - Every function returns an int status (HPHC_OK = 0).  On failure the
 *     handle keeps a message, read with hphc_last_error().  The reference
 *     reports errors with assert (compiled out), Rcpp::stop or exit(-1); the C
 *     ABI reports them instead of stopping the process.
 *   - The caller owns every pointer passed in; inputs are copied into the
 *     engine before the call returns and outputs are written before it
 *     returns (synchronous, like the reference's bufferedCopy,
 *     src/MemoryManagement.hpp:40-56).
 *   - An engine is not thread-safe: one caller thread per handle, as with the
 *     reference engines.  Separate handles may be used from separate threads.
 *   - Parameter vectors have 6 entries in the reference order
 *     (src/NewHawkes.hpp:331-339): sigma (sigmaXprec), a (tauXprec),
 *     b (tauTprec), omega, theta, mu0.  sigma, a and b are precisions.
 *   - Gradients have the same 6 entries, d logL / d p_k.
 */
#ifndef HPHC_H
#define HPHC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define HPHC_OK 0
#define HPHC_ERR_INVALID_HANDLE 1   /* null or destroyed handle                        */
#define HPHC_ERR_BAD_LENGTH 2       /* a length does not match N, D or 6               */
#define HPHC_ERR_BAD_ARGUMENT 3     /* null pointer, index out of range, N < 1 ...     */
#define HPHC_ERR_NONFINITE 4        /* NaN or infinity in times or locations           */
#define HPHC_ERR_UNSUPPORTED 5      /* D outside 1..8, unknown precision flags         */
#define HPHC_ERR_CUDA 6             /* a CUDA runtime call or kernel launch failed     */
#define HPHC_ERR_NOT_READY 7        /* times, locations or parameters not set yet     */
#define HPHC_ERR_DEVICE_TIMEOUT 8   /* a bounded device-side wait gave up              */
#define HPHC_ERR_NO_DEVICE 9        /* no CUDA device visible                          */
#define HPHC_ERR_OUT_OF_MEMORY 10   /* device or pinned host allocation failed         */
#define HPHC_ERR_SCRATCH_TOO_SMALL 11 /* a problem needs more scratch than provided    */

/* ---- flags: bit-compatible with hph::Flags (src/flags.h:6-13) ----------- */
#define HPHC_FLAG_FLOAT (1L << 2)     /* single precision: FP32 throughout, as the
                                         reference's float engine (with COMPENSATED:
                                         the FP32-compensated mode)                  */
#define HPHC_FLAG_TBB (1L << 3)       /* accepted and ignored (CPU threading flag)    */
#define HPHC_FLAG_OPENCL (1L << 4)    /* accepted: the GPU engine slot                */
#define HPHC_FLAG_SSE (1L << 5)       /* accepted and ignored                         */
#define HPHC_FLAG_AVX (1L << 6)       /* accepted and ignored                         */
#define HPHC_FLAG_AVX512 (1L << 7)    /* accepted and ignored                         */
#define HPHC_FLAG_CUDA (1L << 8)      /* new: select the CUDA engine                  */
#define HPHC_FLAG_COMPENSATED (1L << 9) /* new: FP32 pair terms, compensated, FP64 reductions */
#define HPHC_FLAG_NO_UNDERFLOW_SKIP (1L << 10) /* new: evaluate every tile pair, even those
                                                  whose terms all underflow to zero */
/* FP32-compensated mode only.  By default its exponentials are computed on the
 * FMA pipe (range reduction + polynomial, unbiased to ~3e-10) and coordinate
 * differences from FP32 coordinates (times always from hi/lo float pairs). */
#define HPHC_FLAG_FP32_FAST_EXP (1L << 11)   /* hardware ex2.approx with its mean bias
                                                (measured on the device) removed: ~1.6x
                                                faster; strongly cancelling gradient
                                                components lose accuracy (~1e-6) */
#define HPHC_FLAG_FP32_SPACE_HILO (1L << 12) /* coordinate differences from hi/lo float
                                                pairs (times always use hi/lo pairs) */
#define HPHC_FLAG_ORDERED (1L << 13)         /* evaluate both orders of every background
                                                pair, in either precision (by default each
                                                pair is evaluated once and added to both
                                                events' sums) */
#define HPHC_FLAG_FP32_ORDERED HPHC_FLAG_ORDERED /* earlier name of the same bit */
#define HPHC_FLAG_NO_INCREMENTAL (1L << 14)  /* always run the full pair sweep (by default
                                                an evaluation at unchanged parameters after
                                                a few single-event updateLocations calls
                                                updates the kept per-event sums in O(N)) */
#define HPHC_FLAG_NO_FAST_TAIL (1L << 15)    /* one exponential for every pair term (by
                                                default tile pairs whose background terms are
                                                all below 2^-10 (FP32-compensated mode) or
                                                2^-60 (FP64 mode) of an event's own term take
                                                those terms from ex2.approx) */
#define HPHC_FLAG_NO_TAIL_TRUNCATION (1L << 16) /* skip background tile pairs only where
                                                every term underflows (by default tile pairs
                                                whose background terms are all below 2^-91
                                                (FP64) or 2^-60 (FP32 modes) of an event's
                                                own term are skipped: together under 2^-60
                                                and 2^-33 of any event's sums) */

/* How the last evaluation was computed (hphc_get_last_evaluation_path). */
#define HPHC_PATH_SWEEP 0        /* the O(N^2) pair sweep                             */
#define HPHC_PATH_INCREMENTAL 1  /* kept sums updated for moved events, O(N) each     */
#define HPHC_PATH_KEPT_SUMS 2    /* nothing changed since the sums were kept: O(N) finish */
#define HPHC_PATH_SELF_EXCITATION 3 /* kept background sums (same events, tauX, tauT):
                                       only the self-excitation terms swept */

/* Precision modes reported by hphc_get_precision(). */
#define HPHC_PRECISION_FP64 0          /* plain FP64 pair terms and reductions           */
#define HPHC_PRECISION_FP32_COMP 1     /* FP32 pair terms, compensated; FP64 reductions  */
#define HPHC_PRECISION_FP32 2          /* FP32 throughout (the reference's float engine):
                                          pair terms, plain sums, log and CDF in float;
                                          event totals FP64 and fixed-order            */

typedef struct hphc_engine hphc_engine;

/* ---- lifetime ----------------------------------------------------------- */

/*
 * Create an engine for locationCount events in embeddingDimension (1..8)
 * spatial dimensions.  Replaces hph::factory (src/factory.cpp:32) for the GPU
 * slot and the OpenCLHawkes constructor (src/backend/opencl/instantiate.cpp:15-52).
 * flags: HPHC_FLAG_COMPENSATED selects the FP32-compensated mode (FP32 pair
 * terms, compensated sums, FP64 reductions; with or without HPHC_FLAG_FLOAT);
 * HPHC_FLAG_FLOAT alone the plain FP32 mode, the reference's single precision
 * (src/factory.cpp:34, :45); otherwise plain FP64.  device: CUDA device ordinal; a value < 0 or
 * beyond the device count selects device 0, as the OpenCL engine falls back to
 * the default device (src/backend/opencl/OpenCLHawkes.hpp:88-92).
 */
int hphc_create(int embeddingDimension, int locationCount, long flags, int device,
                hphc_engine** out);

/* Release every device and host resource of the engine.  Null is a no-op. */
void hphc_destroy(hphc_engine* engine);

/* Message of the last failed call on this handle ("" if none). */
const char* hphc_last_error(const hphc_engine* engine);

/* Fixed text for a status code. */
const char* hphc_status_string(int status);

/* ---- data and parameters (hph::AbstractHawkes) ------------------------- */

/* Replaces AbstractHawkes::setTimesData (src/AbstractHawkes.hpp:49;
 * src/NewHawkes.hpp:320-323).  length must equal N.  Times need not be sorted;
 * as in the reference, T = data[N-1]. */
int hphc_set_times_data(hphc_engine* engine, const double* data, size_t length);

/* Replaces AbstractHawkes::updateLocations (src/AbstractHawkes.hpp:43;
 * src/NewHawkes.hpp:244-276).  locationIndex == -1: all N rows, row-major,
 * length == D*N.  Otherwise one row, length == D. */
int hphc_update_locations(hphc_engine* engine, int locationIndex, const double* location,
                          size_t length);

/* Replaces AbstractHawkes::setParameters (src/AbstractHawkes.hpp:50;
 * src/NewHawkes.hpp:331-339).  length must be 6. */
int hphc_set_parameters(hphc_engine* engine, const double* data, size_t length);

/* ---- evaluation --------------------------------------------------------- */

/* Replaces AbstractHawkes::getSumOfLikContribs (src/AbstractHawkes.hpp:42;
 * src/NewHawkes.hpp:278-282, :636-660): the full log-likelihood, including
 * the N(D-1)log(1/sqrt(2 pi)) constant. */
int hphc_get_sum_of_lik_contribs(hphc_engine* engine, double* out);

/* The interface method the reference leaves commented out
 * (src/AbstractHawkes.hpp:44, src/NewHawkes.hpp:341-345): d logL / d p, 6
 * entries in parameter order.  length must be 6. */
int hphc_get_log_likelihood_gradient(hphc_engine* engine, double* out, size_t length);

/* Log-likelihood and gradient from one pair sweep.  No reference
 * counterpart as a single call; equals getSumOfLikContribs followed by
 * getLogLikelihoodGradient on the same state.  gradient may be null. */
int hphc_get_log_likelihood_and_gradient(hphc_engine* engine, double* loglik, double* gradient,
                                         size_t length);

/* Replaces AbstractHawkes::getProbsSelfExcite (src/AbstractHawkes.hpp:45;
 * src/NewHawkes.hpp:325-329, :662-719).  length must equal N. */
int hphc_get_probs_self_excite(hphc_engine* engine, double* out, size_t length);

/* ---- MCMC state (src/AbstractHawkes.hpp:46-48) ------------------------ */

/* Save parameters, locations and the last log-likelihood.  The reference's
 * NewHawkes::storeState copies in the wrong direction (src/NewHawkes.hpp:286-291);
 * this saves the current state, as OpenCLHawkes::storeState does
 * (src/backend/opencl/OpenCLHawkes.hpp:283-300).  The kept per-event sums (if
 * current) are saved too, so that an evaluation after restoreState needs no
 * sweep. */
int hphc_store_state(hphc_engine* engine);

/* Return to the saved state (src/NewHawkes.hpp:305-318).  The saved
 * locations are used by every later evaluation (the OpenCL engine kept
 * binding the unswapped buffer, src/backend/opencl/OpenCLHawkes.hpp:257, :382). */
int hphc_restore_state(hphc_engine* engine);

/* Accept the proposal (src/NewHawkes.hpp:297-303): keeps the current state. */
int hphc_accept_state(hphc_engine* engine);

/* Replaces AbstractHawkes::getInternalDimension (src/AbstractHawkes.hpp:51): D. */
int hphc_get_internal_dimension(hphc_engine* engine, int* out);

/* ---- batched evaluation (no reference counterpart) ---------------------
 *
 * Evaluate K parameter vectors (K x 6, row-major) on the engine's events in
 * one run: one launch per stage for all K (MCMC proposals or parallel chains),
 * replayed from a CUDA graph.  loglik has K entries; gradient (K x 6) may be
 * null.  The engine's own parameters are not changed. */
int hphc_batch_log_likelihood_and_gradient(hphc_engine* engine, const double* params, int K,
                                           double* loglik, double* gradient);

/* ---- many event sets at once (no reference counterpart) -------------------
 *
 * A multiset holds numSets independent event sets of uneven sizes (for
 * example many regions or many simulated data sets) and evaluates each at its
 * own parameter vector in one run: one launch per stage for all sets, the
 * sweep's work items taken largest first by persistent CTAs, the sequence
 * replayed from a CUDA graph.  Same precision flags as hphc_create. */
typedef struct hphc_multiset hphc_multiset;

int hphc_multiset_create(int embeddingDimension, int numSets, const int* setSizes, long flags,
                         int device, hphc_multiset** out);
void hphc_multiset_destroy(hphc_multiset* multiset);
const char* hphc_multiset_last_error(const hphc_multiset* multiset);

/* Locations (setSizes[set] x D, row-major) and times of one set. */
int hphc_multiset_set_data(hphc_multiset* multiset, int set, const double* locations,
                           size_t locLength, const double* times, size_t timesLength);

/* params: numSets x 6; loglik: numSets; gradient: numSets x 6 (may be null). */
int hphc_multiset_log_likelihood_and_gradient(hphc_multiset* multiset, const double* params,
                                              double* loglik, double* gradient);

int hphc_multiset_set_kernel_timing(hphc_multiset* multiset, int enable);
int hphc_multiset_get_kernel_times(hphc_multiset* multiset, float* sweepMs, float* finishMs,
                                   float* stepMs);
int hphc_multiset_get_last_launch_stats(hphc_multiset* multiset, int* kernelLaunches,
                                        double* backgroundTerms, double* selfExciteTerms);
int hphc_multiset_get_last_launch_evals(hphc_multiset* multiset, double* backgroundEvals);

/* ---- multi-chain Metropolis-Hastings sampler ----------------------------
 *
 * Replaces the reference's R sampler() (R/Untitled.R:254-422) and its
 * Potential() (:225-231) for numChains independent chains whose proposals are
 * evaluated together: one batched likelihood run per iteration.  Each chain
 * follows the reference loop: random-scan choice of one sampled parameter, a
 * proposal from a normal truncated to (0, inf) centred on the current value
 * (sd = that parameter's radius), truncated-normal priors (sd 10 for the first
 * five parameters, 1 for mu0), the Metropolis-Hastings test with the proposal
 * densities, radius adaptation towards 0.44 acceptance every SampBound
 * proposals (SampBound from 5, growing to ceil(SampBound^1.1)).  Random
 * numbers come from one splitmix64 stream per chain seeded from `seed` and the
 * chain index (the reference uses R's generator), so runs are reproducible.
 *
 * initialParams: numChains x 6.  radius: initial proposal sd of every
 * parameter (the reference's `radius`, default 2).  sampledMask: bit q set =
 * parameter q is proposed; 0 selects the reference's set {sigma, omega,
 * theta, mu0} (sample(c(1,4:6)), R/Untitled.R:328).  The sampler keeps its
 * state between runs. */
typedef struct hphc_sampler hphc_sampler;

/* Batched log-likelihood evaluator for hphc_sampler_run_with: K parameter
 * vectors (K x 6) in, K log-likelihoods out; returns 0 on success. */
typedef int (*hphc_batch_loglik_fn)(void* user, const double* params, int K, double* loglik);

int hphc_sampler_create(int numChains, const double* initialParams, double radius,
                        int sampledMask, unsigned long long seed, hphc_sampler** out);
void hphc_sampler_destroy(hphc_sampler* sampler);
const char* hphc_sampler_last_error(const hphc_sampler* sampler);

/* Run `iterations` iterations of every chain on the engine's events (the
 * engine's own parameters are not changed).  samples (numChains x
 * (iterations - burnIn) x 6) and targets (numChains x (iterations - burnIn),
 * the potential -logL - log prior, the reference's `target`) may be null. */
int hphc_sampler_run(hphc_sampler* sampler, hphc_engine* engine, int iterations, int burnIn,
                     double* samples, double* targets);

/* The same with a caller-supplied batched evaluator. */
int hphc_sampler_run_with(hphc_sampler* sampler, hphc_batch_loglik_fn evaluate, void* user,
                          int iterations, int burnIn, double* samples, double* targets);

/* The same iterations run entirely on the device: the chains live in device
 * memory and one iteration (proposal kernel, pair sweep, finish, acceptance
 * kernel) is captured once into a CUDA graph and replayed for every
 * iteration, with no host work or transfer in between; the samples come back
 * at the end.  The chains continue from, and return to, the sampler's state.
 * The sampled set must leave tauXprec and tauTprec fixed (they fix the record
 * scaling and the work list); otherwise HPHC_ERR_UNSUPPORTED.  Chains match
 * hphc_sampler_run's except where the device math library rounds log, cos,
 * erfc, exp or pow differently in the last bit. */
int hphc_sampler_run_device(hphc_sampler* sampler, hphc_engine* engine, int iterations,
                            int burnIn, double* samples, double* targets);

/* Current state per chain (each pointer may be null): parameters (numChains x
 * 6), potential (NaN before the first run), radii (numChains x 6), accepted
 * and proposed counts. */
int hphc_sampler_get_state(const hphc_sampler* sampler, double* params, double* potential,
                           double* radii, long long* accepted, long long* proposed);

/* ---- evaluation without allocation (no reference counterpart) -----------
 *
 * FP64 log-likelihood and gradient of one event set for callers that must not
 * allocate GPU memory while they run: code inside a framework that owns all
 * device memory through its own pool or memory cap, real-time loops that
 * cannot take an allocation's implicit synchronisation, processes with a GPU
 * memory budget fixed at start-up.  This function calls no cudaMalloc,
 * cudaFree or other allocating routine; all of its scratch is one 16 MiB
 * static device array inside libhawkes_b200.so (held on every GPU that loads
 * the library, until the process exits), enough for N up to about 200,000
 * events at D = 2 (fewer at higher D).  Larger problems return
 * HPHC_ERR_SCRATCH_TOO_SMALL without touching the GPU.
 *
 * Inputs are device memory of the current CUDA device: deviceLocations (N x D
 * row-major), deviceTimes (N); params are 6 host doubles in reference order.
 * deviceOut is 8 doubles of device memory: [0] log-likelihood, [1..6]
 * gradient, [7] zero.  The call runs on `stream` (a cudaStream_t, or null
 * for the default stream) and returns when the result is written.
 *
 * The first call on a device does a one-time set-up: it looks up the static
 * array's device address (cudaGetSymbolAddress), and looks it up again after
 * the device's context was destroyed and recreated (cudaDeviceReset).  Make
 * that first call before any stream capture begins.  Device inputs are not
 * checked: a NaN or infinity in them gives a non-finite result; times need
 * not be sorted (T = t[N-1], as in the reference).  Every call shares the one
 * array: calls that overlap on the GPU (other streams or threads) race and
 * corrupt each other's results. */
int hphc_loglik_grad_fp64_static(int embeddingDimension, int locationCount,
                                 const double* deviceLocations, const double* deviceTimes,
                                 const double* params, double* deviceOut, void* stream);

/* ---- sharded evaluation across GPUs ---------------------------------------
 * No reference counterpart (the reference evaluates on one device).  One
 * engine per GPU, every engine holding all events and the same parameters.
 * Each rank sweeps a disjoint set of target strips (whole strips, assigned
 * by the same deterministic balance on every rank) and writes its share of
 * every event's six unit pair sums; the shares of ranks 0..world-1 add up to
 * the sums of one unsharded sweep.  The caller moves the shares between GPUs
 * (one all-gather of 6 N doubles per rank, e.g. NCCL), then gives every rank
 * all of them: the engine adds them in rank order, so all ranks then hold the
 * same sums, and its next getSumOfLikContribs / gradient /
 * getProbsSelfExcite at those parameters runs only the O(N) finish
 * (HPHC_PATH_KEPT_SUMS).  Needs the kept sums (no HPHC_FLAG_NO_INCREMENTAL).
 *
 * hphc_sweep_shard: rank's share into devicePart, device memory of the
 * engine's device holding length = 6 N doubles ([6][N], natural units).
 * Synchronous. */
int hphc_sweep_shard(hphc_engine* engine, int rank, int world, double* devicePart,
                     size_t length);

/* deviceParts: numParts shares back to back (length = numParts * 6 N doubles,
 * device memory of the engine's device), share r from rank r.  Fails with
 * HPHC_ERR_BAD_ARGUMENT if the events or parameters changed since this
 * engine's own hphc_sweep_shard. */
int hphc_set_unit_sums(hphc_engine* engine, const double* deviceParts, int numParts,
                       size_t length);

/* ---- fault injection (testing) --------------------------------------------
 * No reference counterpart.  Makes error handling testable without a GPU
 * fault: the next `count` calls of this handle that reach `stage` fail there
 * with a stand-in CUDA error instead of making the CUDA call (nothing is
 * uploaded or launched at that stage; at HPHC_FAULT_WAIT the launched work is
 * waited for first).  The call returns the status that error maps to, with
 * "injected" in hphc_last_error; the engine stays usable and its next calls
 * run normally.  count 0 clears.  Sampler runs on the engine see the same
 * faults. */
#define HPHC_FAULT_UPLOAD 1 /* host-to-device upload of events (HPHC_ERR_OUT_OF_MEMORY) */
#define HPHC_FAULT_LAUNCH 2 /* graph or kernel launch of an evaluation (HPHC_ERR_CUDA)  */
#define HPHC_FAULT_WAIT 3   /* completion wait of an evaluation (HPHC_ERR_CUDA)         */
int hphc_inject_fault(hphc_engine* engine, int stage, int count);

/* ---- introspection and device-resident timing --------------------------- */

/* No reference counterpart (the reference's exponentials are libm's).  The
 * two exponentials of the FP32 modes evaluated on `device` for n host
 * arguments s >= 0: poly[k] = 2^-s[k] by the software exponential (Cody-Waite
 * reduction, degree-7 polynomial, exact power of two; near terms), and
 * hardware[k] = ex2.approx.ftz(-s[k]) (far-tail background terms).  For
 * testing their error bounds against FP64.  Allocates device memory;
 * synchronous; n at most 2^28. */
int hphc_eval_exponentials(int device, const float* args, size_t n, float* poly,
                           float* hardware);

/* Precision mode in use (HPHC_PRECISION_*). */
int hphc_get_precision(hphc_engine* engine, int* out);

/* The cudaStream_t the engine launches on, as void*.  Callers may record CUDA
 * events on it to time the device work of hphc_enqueue_*. */
int hphc_get_stream(hphc_engine* engine, void** stream);

/* Enqueue one log-likelihood + gradient evaluation on the engine's stream
 * with the data already on the device, without waiting and without copying
 * results back.  hphc_read_results() waits and returns them.  Always the full
 * pair sweep (no kept sums are reused), so that it times the whole work. */
int hphc_enqueue_log_likelihood_and_gradient(hphc_engine* engine);

/* Wait for the last enqueued evaluation and copy its log-likelihood and
 * gradient (6, may be null) to the host. */
int hphc_read_results(hphc_engine* engine, double* loglik, double* gradient, size_t length);

/* Which path the most recent single evaluation took (HPHC_PATH_*).
 * Incremental evaluation (no reference counterpart; the reference recomputes
 * the O(N^2) sum on every call): after an evaluation the engine keeps each
 * event's six unit pair sums (of parameter vector 0 for a batched call).  The
 * background sums depend only on the events, tauX and tauT, the
 * self-excitation sums only on the events, sigma and omega; theta and mu0
 * enter only the O(N) finish.  So:
 *   - same sigma, tauX, tauT, omega (theta, mu0 free), no event moved:
 *     the O(N) finish only (HPHC_PATH_KEPT_SUMS);
 *   - the same, after a few events moved (hphc_update_locations with an
 *     index; at most max(1, min(64, N/512)) since the sums were formed):
 *     every event's sums are updated by its pair with each moved event and
 *     the moved events' rows recomputed, O(N) per moved event, then the
 *     finish (HPHC_PATH_INCREMENTAL);
 *   - same tauX and tauT in every parameter vector, sigma or omega changed,
 *     no event moved: only the self-excitation terms are swept (a narrow band
 *     near the diagonal for sorted times) and the kept background sums are
 *     reused (HPHC_PATH_SELF_EXCITATION) -- the steps of the reference's
 *     sampler, which keeps tauX and tauT fixed;
 *   - otherwise the full sweep (HPHC_PATH_SWEEP).
 * Changing the times or all locations (index -1) forces the sweep.  Results
 * agree with the sweep to FP64 rounding (FP64 mode) or to the FP32 mode's own
 * accuracy.  HPHC_FLAG_NO_INCREMENTAL keeps no sums. */
int hphc_get_last_evaluation_path(hphc_engine* engine, int* path);

/* Kernel launches made by the most recent evaluation call (for launch
 * accounting), and how many background and self-excitation pair terms its
 * sweep evaluated.  Of the 2 N^2 possible terms the rest were skipped at tile
 * level: the non-causal half of the self-excitation sum, tile pairs whose
 * terms all underflow to exactly zero in the working precision, and (tail
 * truncation) background tile pairs whose terms are all below 2^-91 (FP64) or
 * 2^-60 (FP32 modes) of an event's own term. */
int hphc_get_last_launch_stats(hphc_engine* engine, int* kernelLaunches,
                               double* backgroundTerms, double* selfExciteTerms);

/* Background exponentials the most recent evaluation's sweep computed.  In the
 * FP32-compensated mode each background pair (i, j) with j in a tile before
 * i's strip is evaluated once and counted once, but stands for two terms in
 * backgroundTerms above (B_ij in event i's sum, B_ji in event j's). */
int hphc_get_last_launch_evals(hphc_engine* engine, double* backgroundEvals);

/* Sweep shape: target events per thread (2 or 4; a CTA strip holds 128 times
 * as many) and the number of (strip, j-range) work items per SM the j range is
 * split into.  0 for either lets the engine's autotuner choose it (timed on the
 * engine's own data at the first evaluation, cached per process by problem
 * size and mode). */
int hphc_set_sweep_shape(hphc_engine* engine, int eventsPerThread, int itemsPerSM);
int hphc_get_sweep_shape(hphc_engine* engine, int* eventsPerThread, int* itemsPerSM);

/* Record CUDA events around the pair-sweep kernel and around the finish
 * kernels of every later evaluation (enable != 0), on the engine's stream. */
int hphc_set_kernel_timing(hphc_engine* engine, int enable);

/* Device durations (ms) of the most recent evaluation made with kernel timing
 * enabled, after it has been waited for (hphc_read_results or any
 * synchronous call): the pair sweep, the finish + final kernels and the whole
 * step (table upload, record build, sweep, finish, result copy). */
int hphc_get_kernel_times(hphc_engine* engine, float* sweepMs, float* finishMs, float* stepMs);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* HPHC_H */
