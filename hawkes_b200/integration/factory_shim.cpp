// Puts the CUDA engine in the GPU slot of the reference's hph::factory.
//
// src/factory.cpp, compiled with HAVE_OPENCL defined, sends every request with
// the OPENCL flag (set by the R glue for gpu > 0, src/hpHawkes.cpp:65-72, and by
// the benchmark CLI for --gpu, src/benchmark.cpp:83-87) to
// constructOpenCLHawkesDouble / constructOpenCLHawkesFloat (src/factory.cpp:41-47,
// :67-72).  Linking this file instead of src/backend/opencl/instantiate.cpp
// defines those two constructors to build hph::CudaHawkes, so the reference's
// factory, CLI and R entry points reach the CUDA engine without a source change.
// The FLOAT flag (single precision, src/factory.cpp:34) selects FP32
// throughout, as the reference's float engine; a caller that wants the
// FP32-compensated mode adds HPHC_FLAG_COMPENSATED to the flags.
#include "hawkes_b200/CudaHawkes.hpp"

namespace hph {

SharedPtr constructOpenCLHawkesDouble(int embeddingDimension, int locationCount, long flags,
                                      int device) {
    return constructCudaHawkes(embeddingDimension, locationCount, flags & ~long(HPHC_FLAG_FLOAT),
                               device);
}

SharedPtr constructOpenCLHawkesFloat(int embeddingDimension, int locationCount, long flags,
                                     int device) {
    return constructCudaHawkes(embeddingDimension, locationCount, flags | HPHC_FLAG_FLOAT, device);
}

}  // namespace hph
