// ORACLE / TEST INFRASTRUCTURE -- not part of the product.
//
// A C wrapper around the reference hpHawkes CPU engine, compiled unmodified from
// the reference sources (src/NewHawkes.hpp, src/factory.cpp) against the stub
// tbb/xsimd headers under oracle/stubs.  It exposes the engine through plain C
// so Python tests (ctypes), the golden-fixture generator and the bench's CPU
// baseline can call it.  Only tests/, the smoke check and bench.py's CPU
// baseline load the resulting oracle/_ref/libhawkes_ref.so.
//
// Entry points mirror hph::AbstractHawkes (src/AbstractHawkes.hpp:32-60) and
// hph::factory (src/factory.cpp:32): create with (dim, N, flags, threads),
// setTimesData, updateLocations, setParameters, getSumOfLikContribs,
// getProbsSelfExcite, store/restore/acceptState.
#include <cstring>
#include <sstream>
#include <string>

#include "NewHawkes.hpp"
#include "factory.cpp"

namespace {
struct RefEngine {
    hph::SharedPtr engine;
    std::string variant;
};
}  // namespace

extern "C" {

// Returns an opaque engine or null.  The variant string the reference prints at
// construction ("DOUBLE, TBB PARALLEL, NO SIMD", src/NewHawkes.hpp:902-921) is
// captured instead of going to stdout; read it with ref_variant().
void* ref_create(int embeddingDimension, int locationCount, long flags, int threads) {
    std::ostringstream captured;
    auto* old = std::cout.rdbuf(captured.rdbuf());
    RefEngine* e = nullptr;
    try {
        e = new RefEngine{hph::factory(embeddingDimension, locationCount, flags, -1, threads), ""};
    } catch (...) {
        e = nullptr;
    }
    std::cout.rdbuf(old);
    if (e) {
        e->variant = captured.str();
        while (!e->variant.empty() && (e->variant.back() == '\n' || e->variant.back() == '\r'))
            e->variant.pop_back();
    }
    return e;
}

const char* ref_variant(void* h) { return static_cast<RefEngine*>(h)->variant.c_str(); }

void ref_destroy(void* h) { delete static_cast<RefEngine*>(h); }

void ref_set_times_data(void* h, const double* data, size_t length) {
    static_cast<RefEngine*>(h)->engine->setTimesData(const_cast<double*>(data), length);
}

void ref_update_locations(void* h, int index, const double* data, size_t length) {
    static_cast<RefEngine*>(h)->engine->updateLocations(index, const_cast<double*>(data), length);
}

void ref_set_parameters(void* h, const double* data, size_t length) {
    static_cast<RefEngine*>(h)->engine->setParameters(const_cast<double*>(data), length);
}

double ref_get_sum_of_lik_contribs(void* h) {
    return static_cast<RefEngine*>(h)->engine->getSumOfLikContribs();
}

void ref_get_probs_self_excite(void* h, double* out, size_t length) {
    static_cast<RefEngine*>(h)->engine->getProbsSelfExcite(out, length);
}

void ref_store_state(void* h) { static_cast<RefEngine*>(h)->engine->storeState(); }
void ref_restore_state(void* h) { static_cast<RefEngine*>(h)->engine->restoreState(); }
int ref_get_internal_dimension(void* h) {
    return static_cast<RefEngine*>(h)->engine->getInternalDimension();
}

}  // extern "C"
