// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
#pragma once

#include "container/vector.hpp"

namespace num {

// clip negative entries to zero, then rescale to sum one; returns the total before rescaling
// (markovkit/distribution.hpp:62, tests/test_fsp.cpp:44-46)
inline real clip_and_normalize_nonnegative(array<real> &p) {
    real total = 0.0;
    for (real &v : p) {
        if (v < 0.0) {
            v = 0.0;
        }
        total += v;
    }
    if (total > 0.0) {
        for (real &v : p) {
            v /= total;
        }
    }
    return total;
}

} // namespace num
