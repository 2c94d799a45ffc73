// CudaHawkes: the B200 CUDA engine as an hph::AbstractHawkes.
//
// Header-only adapter for the reference code base: compile it with the
// reference's src/ directory on the include path (for AbstractHawkes.hpp) and
// this repository's include/ directory, and link libhawkes_b200.so.  It
// forwards every interface method (src/AbstractHawkes.hpp:32-60) to the C ABI
// in hphc.h and adds getLogLikelihoodGradient, whose declaration the reference
// keeps commented out (src/AbstractHawkes.hpp:44).
//
// Errors: a non-zero status becomes Rcpp::stop under RBUILD (as the R glue
// reports errors, src/hpHawkes.cpp:36-42) and std::runtime_error otherwise.
#ifndef HAWKES_B200_CUDA_HAWKES_HPP
#define HAWKES_B200_CUDA_HAWKES_HPP

#include <memory>
#include <stdexcept>
#include <string>

#include "AbstractHawkes.hpp"
#include "hphc.h"

#ifdef RBUILD
#include <Rcpp.h>
#endif

namespace hph {

class CudaHawkes : public AbstractHawkes {
public:
    // flags as in hph::Flags; FLOAT selects the FP32-compensated mode.
    CudaHawkes(int embeddingDimension, int locationCount, long flags, int device)
        : AbstractHawkes(embeddingDimension, locationCount, flags) {
        const int st = hphc_create(embeddingDimension, locationCount, flags, device, &engine);
        if (st != HPHC_OK) raise(std::string("CudaHawkes: ") + hphc_status_string(st));
        int precision = 0;
        hphc_get_precision(engine, &precision);
        std::cerr << "CUDA (sm_100a), "
                  << (precision == HPHC_PRECISION_FP64        ? "DOUBLE"
                      : precision == HPHC_PRECISION_FP32_COMP ? "SINGLE-COMPENSATED"
                                                              : "SINGLE")
                  << std::endl;
    }

    ~CudaHawkes() override { hphc_destroy(engine); }

    double getSumOfLikContribs() override {
        double v = 0.0;
        check(hphc_get_sum_of_lik_contribs(engine, &v));
        return v;
    }

    void updateLocations(int locationIndex, double* location, size_t length) override {
        check(hphc_update_locations(engine, locationIndex, location, length));
    }

    // Not an override: the base declaration is commented out in the reference.
    void getLogLikelihoodGradient(double* result, size_t length) {
        check(hphc_get_log_likelihood_gradient(engine, result, length));
    }

    void getProbsSelfExcite(double* result, size_t length) override {
        check(hphc_get_probs_self_excite(engine, result, length));
    }

    void storeState() override { check(hphc_store_state(engine)); }
    void restoreState() override { check(hphc_restore_state(engine)); }
    void acceptState() override { check(hphc_accept_state(engine)); }

    void setTimesData(double* data, size_t length) override {
        check(hphc_set_times_data(engine, data, length));
    }

    void setParameters(double* data, size_t length) override {
        check(hphc_set_parameters(engine, data, length));
    }

    int getInternalDimension() override {
        int d = 0;
        check(hphc_get_internal_dimension(engine, &d));
        return d;
    }

    hphc_engine* handle() { return engine; }

private:
    hphc_engine* engine = nullptr;

    void check(int status) {
        if (status != HPHC_OK) raise(std::string("CudaHawkes: ") + hphc_last_error(engine));
    }

    [[noreturn]] static void raise(const std::string& msg) {
#ifdef RBUILD
        Rcpp::stop(msg);
#else
        throw std::runtime_error(msg);
#endif
    }
};

// Constructor with the signature of the reference's engine constructors
// (e.g. constructOpenCLHawkesDouble, src/factory.cpp:6).
inline SharedPtr constructCudaHawkes(int embeddingDimension, int locationCount, long flags,
                                     int device) {
    return std::make_shared<CudaHawkes>(embeddingDimension, locationCount, flags, device);
}

}  // namespace hph

#endif  // HAWKES_B200_CUDA_HAWKES_HPP
