// Scalar stand-in for the two xsimd 7.1.3 functions the hpHawkes CPU engine
// calls on its non-SIMD paths: xsimd::exp (src/NewHawkes.hpp:27, used by the
// FLOAT variant's adhoc::exp<float>) and xsimd::log (src/NewHawkes.hpp:652).
// xsimd is an un-vendored download (CMakeModules/build_xsimd.cmake:1) that is
// not present in this image; its scalar exp/log forward to the C library, and
// so does this stub.  The double-precision pair loop uses the reference's own
// in-tree FreeBSD exp (src/NewHawkes.hpp:53-104), which is compiled from source.
//
// Test infrastructure only: nothing in the product links it.
#ifndef HAWKES_ORACLE_XSIMD_STUB_HPP
#define HAWKES_ORACLE_XSIMD_STUB_HPP

#include <cmath>

namespace xsimd {
template <typename T>
inline T exp(T x) {
    return std::exp(x);
}
template <typename T>
inline T log(T x) {
    return std::log(x);
}
}  // namespace xsimd

#endif
