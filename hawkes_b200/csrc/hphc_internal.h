// Library-internal interface between the engine (hphc_engine.cpp) and the
// device-resident sampler driver (hphc_sampler.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>

#include "hphc.h"
#include "hphc_executor.h"
#include "hphc_kernels.cuh"

namespace hphc {

// NVTX range over a scope (header-only NVTX v3: a no-op unless a profiler
// is attached), so timelines and ncu --nvtx filters see the engine's phases.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// What the device-resident loop needs from an engine after set-up.
struct EngineLoop {
    int device = 0;
    cudaStream_t stream = nullptr;
    Executor* ex = nullptr;
    ConstsSpec spec{};
};

// Upload the engine's events if needed and prepare its executor's device
// loop for K problems on them at params (K x 6).  On failure returns a status
// and sets *err.
int engine_loop_setup(hphc_engine* engine, const double* params, int K, EngineLoop* out,
                      std::string* err);

// out[k] = parts[k] + parts[n + k] + ... + parts[(nParts - 1) n + k], added in
// that order (hphc_shard.cu).
cudaError_t launch_sum_parts(const double* parts, int nParts, size_t n, double* out, int numSMs,
                             cudaStream_t s);

}  // namespace hphc
