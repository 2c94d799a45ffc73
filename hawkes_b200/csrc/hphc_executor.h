// Work-list executor: evaluates any number of problems (an event set at a
// parameter vector) with one launch per stage.
//
//   stage   what                                          launch
//   H2D     problem tables, work items, finish tables    one cudaMemcpyAsync from pinned staging
//   pack    FP32 records scaled per problem (FP32 mode;   pack_f32_jobs_kernel, grid (N, jobs)
//           one copy per distinct set, tauX, tauT)
//   sweep   persistent CTAs over the work list            sweep_*_list_kernel
//   finish  per-event contributions, per-CTA sums        finish_list_kernel
//   final   per-problem fixed-order totals               final_list_kernel
//   D2H     P x 8 results                                 one cudaMemcpyAsync to pinned memory
//
// The sequence is captured once into a CUDA graph and replayed while buffer
// capacities and the sweep shape stay the same; only the staged tables change
// between runs.  Work items cover each strip's band of tiles that can hold a
// non-zero term (found on the host from per-tile time bounds with the same
// test the kernel applies), split into equal chunks and listed largest first.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "hphc_kernels.cuh"

namespace hphc {

// An event set resident on the device, with host copies used for planning.
struct SetView {
    int N = 0;
    const double* dLoc = nullptr;      // N x D raw coordinates
    const double* dTimes = nullptr;    // N raw times
    const int32_t* dRanks = nullptr;   // dense time ranks (FP32 mode)
    const int32_t* dOrder2 = nullptr;  // spatial row order of strips of R = 2 and 4 (FP32
    const int32_t* dOrder4 = nullptr;  //   mode, launch_strip_order), or null
    const double* dRecF64 = nullptr;   // FP64 records (FP64 mode)
    const double* dTileMin = nullptr;  // per-tile time bounds
    const double* dTileMax = nullptr;
    const double* hTimes = nullptr;    // host copies
    const double* hTileMin = nullptr;
    const double* hTileMax = nullptr;
    bool sorted = false;               // times ascending (bands are contiguous)
};

struct RunStats {
    int launches = 0;        // kernels launched by the last run
    double bTerms = 0.0;     // background pair terms the sweep accounted for
    double sTerms = 0.0;     // self-excitation pair terms the sweep evaluated
    double bEvals = 0.0;     // background exponentials evaluated (a symmetric pair: one)
};

class Executor {
public:
    // precision: HPHC_PRECISION_*; variant: FP32 variant bits (see
    // hphc_kernels.cu); ex2Bias: mean relative error of the hardware
    // exponential (divided out of the sums when the variant uses it).
    int init(int D, int precision, int variant, bool underflowSkip, int device, cudaStream_t stream,
             double ex2Bias);
    void release();

    // Plan and enqueue P problems (problem p = set setOf[p] at params[6p..6p+5])
    // without waiting.  dProbs: device buffer receiving P_i of problem 0, or null.
    int enqueue(const std::vector<SetView>& sets, const int* setOf, const double* params, int P,
                double* dProbs);
    // Wait for the last enqueue and copy its P x 8 results (log-likelihood,
    // gradient, 0) to hostOut.
    int wait(double* hostOut);

    // Device-resident loop (the on-device sampler): build the plan for P
    // problems once, with bands wide enough for any sigma, omega, theta and
    // mu0 at the problems' own tauX and tauT (all earlier tiles of sorted
    // times; the kernel still skips tile pairs whose terms all underflow),
    // upload its tables and pack the FP32 records.  enqueue_device_body()
    // then runs sweep, finish and final on those device tables, whose
    // per-problem constants a device kernel may rewrite between runs; the
    // P x 8 results are at device_results().  A later enqueue() replaces the
    // tables.
    int setup_device_loop(const std::vector<SetView>& sets, const int* setOf,
                          const double* params, int P);
    int enqueue_device_body();
    SweepProblem* device_sweep_problems() const;
    FinishProblem* device_finish_problems() const;
    const double* device_results() const { return dOut_; }
    int num_sms() const { return numSMs_; }

    // Pair terms the last run's sweep accounted for (replays the tile
    // decisions): background terms (both orders of a symmetric pair),
    // self-excitation terms, and background exponentials evaluated.
    void count_terms(const std::vector<SetView>& sets, double* bTerms, double* sTerms,
                     double* bEvals = nullptr) const;

    std::string error;
    int fixedR = 0, fixedItems = 0;  // sweep shape overrides; 0 = autotune
    int R = 2, itemsPerSM = 16;      // shape in use
    bool useGraph = true;
    bool kernelTiming = false;
    bool symmetric = false;  // symmetric background sweep (set before the first enqueue)
    bool fastTail = true;    // FP32 polynomial mode: far-tail tile pairs use ex2.approx
    bool truncateTail = true;  // skip background tile pairs below 2^-91 of B_ii (with the skip)
    // Sharded sweep: with shardWorld > 1 the plan keeps only the target
    // strips assigned to shardRank (whole strips, balanced by their tile
    // counts; every rank computes the same assignment), and the finish takes
    // the other strips' row sums as zero.  The unit sums written to sumsOut
    // are then this rank's share; the shares of all ranks add up to the sums
    // of the unsharded sweep.
    int shardRank = 0, shardWorld = 1;
    // Fault injection (HPHC_FAULT_LAUNCH / HPHC_FAULT_WAIT): the next
    // faultCount launches or waits fail with a stand-in error.
    int faultStage = 0, faultCount = 0;
    bool take_fault(int stage) {
        if (faultStage != stage || faultCount <= 0) return false;
        if (--faultCount == 0) faultStage = 0;
        return true;
    }
    double* sumsOut = nullptr;  // if set, problem 0's unit pair sums ([6][N], natural units)
    // If set: a self-excitation-only sweep.  keptB holds the background unit
    // sums ([3][N], natural units) of an earlier sweep of the same single
    // event set at the same tauX and tauT as every problem of this run (the
    // caller checks that); the finish uses them and the sweep evaluates no
    // background term.  Rows 0-2 of sumsOut are then not written.
    const double* keptB = nullptr;
    float lastSweepMs = 0.f, lastFinishMs = 0.f, lastStepMs = 0.f;
    bool timedValid = false;
    int lastLaunches = 0;

private:
    int D_ = 0, precision_ = 0, variant_ = 0, device_ = 0, numSMs_ = 148;
    bool skip_ = true;
    bool wideBands_ = false;  // build_plan: bands for any sampled parameters
    int loopGrid_ = 0;        // sweep grid of the device loop
    double ex2Bias_ = 0.0;
    std::string deviceName_;  // for the persistent tune cache
    cudaStream_t stream_ = nullptr;
    bool tuned_ = false;

    // plan of the last enqueue
    struct Plan {
        std::vector<SweepProblem> sp;
        std::vector<WorkItem> items;
        std::vector<int> stripChunks;   // concatenated over problems
        std::vector<FinishProblem> fp;
        std::vector<FinishBlock> fb;
        std::vector<PackJob> pj;
        std::vector<int> setOf;
        int P = 0, maxN = 0, nBlocks = 0;
    } plan_;

    // device / pinned buffers (capacities grow; a growth invalidates the graph)
    void* dTables_ = nullptr;
    size_t tablesCap_ = 0;
    void* hStaging_ = nullptr;
    size_t stagingCap_ = 0;
    float* dRecPool_ = nullptr;
    size_t recCap_ = 0;
    double* dPartials_ = nullptr;
    size_t partialsCap_ = 0;
    unsigned long long* dColAcc_ = nullptr;
    size_t colCap_ = 0;
    double* dBlockSums_ = nullptr;
    size_t blockCap_ = 0;
    double* dOut_ = nullptr;
    double* hOut_ = nullptr;
    size_t outCap_ = 0;
    int* dCounter_ = nullptr;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};

    // table layout inside dTables_ / hStaging_ (byte offsets)
    size_t offSP_ = 0, offItems_ = 0, offNItems_ = 0, offChunks_ = 0, offFP_ = 0, offFB_ = 0,
           offPJ_ = 0, tablesBytes_ = 0;
    size_t itemsCap_ = 0;
    size_t recNeed_ = 0, partialsNeed_ = 0;  // floats / doubles the last plan needs
    size_t colNeed_ = 0;                     // column-sum words the last plan needs

    // graph
    cudaGraphExec_t graphExec_ = nullptr;
    struct GraphKey {
        int P = -1, nJobs = -1, nBlocks = -1, maxN = -1, R = -1, grid = -1;
        size_t tablesBytes = 0, colNeed = 0;
        void* tables = nullptr;
        bool timing = false;
    } graphKey_;

    int build_plan(const std::vector<SetView>& sets, const int* setOf, const double* params, int P,
                   double* dProbs, int r, int items);
    int ensure_buffers();
    int launch_sequence(int grid);
    int sweep_grid(int r) const;
    int autotune(const std::vector<SetView>& sets, const int* setOf, const double* params, int P,
                 double* dProbs);
    int cuda_fail(cudaError_t e, const char* what);
    void drop_graph();
    cudaError_t record(cudaEvent_t ev);
    bool capturing_ = false;

public:
    ConstsSpec consts_spec() const;
    PairConsts pair_consts(const double* p) const;
    FinishConsts finish_consts(const double* p, const SetView& set) const;
};

}  // namespace hphc
