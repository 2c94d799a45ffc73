// ORACLE / TEST INFRASTRUCTURE: the data setters the reference's JNI glue
// leaves commented out (src/jni/dr_inference_hawkes_NativeHPHSingleton.cpp:23-33,
// updateLocations; no setTimesData at all), so that a test can give a JNI
// instance its events.  They act on the glue's own instance table, declared
// there as a global, and call the engine interface the glue already uses
// (hph::AbstractHawkes, src/AbstractHawkes.hpp:32-60).
#include <cstddef>
#include <memory>
#include <vector>

#include "AbstractHawkes.hpp"

extern std::vector<std::shared_ptr<hph::AbstractHawkes>> instances;

extern "C" __attribute__((visibility("default"))) int jni_harness_set_data(
    int instance, double* locations, size_t locationsLength, double* times, size_t n) {
    if (instance < 0 || (size_t)instance >= instances.size()) return -1;
    instances[instance]->setTimesData(times, n);
    instances[instance]->updateLocations(-1, locations, locationsLength);
    return 0;
}
