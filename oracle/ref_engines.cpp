// ORACLE / TEST INFRASTRUCTURE -- not part of the product.
//
// Pulls the reference CPU engine constructors (src/NewHawkes.hpp:899-922) into
// the reference CLI build (oracle/_ref/benchmark_ref).  hph::factory itself is
// compiled from the reference's src/factory.cpp as it is.
#include "NewHawkes.hpp"
