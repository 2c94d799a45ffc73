// Sharded evaluation support: the fixed-order sum of the ranks' shares of the
// per-event unit pair sums.  Each rank of a sharded evaluation sweeps its own
// target strips and writes a [6][N] share; the caller gathers every rank's
// share (one collective of 6N doubles per rank) and the engine adds them in
// rank order here, so every rank holds the same bits, whatever collective
// algorithm moved them.
#include <cuda_runtime.h>

#include <algorithm>

#include "hphc_internal.h"

namespace hphc {
namespace {

constexpr int kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads)
sum_parts_kernel(const double* __restrict__ parts, int nParts, size_t n, double* __restrict__ out) {
    for (size_t k = (size_t)blockIdx.x * kSumThreads + threadIdx.x; k < n;
         k += (size_t)gridDim.x * kSumThreads) {
        double s = parts[k];
        for (int r = 1; r < nParts; ++r) s += parts[(size_t)r * n + k];
        out[k] = s;
    }
}

}  // namespace

cudaError_t launch_sum_parts(const double* parts, int nParts, size_t n, double* out,
                             int numSMs, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t need = (n + kSumThreads - 1) / kSumThreads;
    const int grid = (int)std::min<size_t>(need, (size_t)numSMs * 8);
    sum_parts_kernel<<<grid, kSumThreads, 0, s>>>(parts, nParts, n, out);
    return cudaGetLastError();
}

}  // namespace hphc
