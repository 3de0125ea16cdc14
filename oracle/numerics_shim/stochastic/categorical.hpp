// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
#pragma once

#include "container/vector.hpp"
#include "stochastic/rng.hpp"

namespace num {

// an index drawn with probability proportional to its weight (markovkit/ssa.hpp:63)
template <typename Rng>
idx sample_categorical(view<const real> weights, Rng &random) {
    real total = 0.0;
    for (real w : weights) {
        total += w;
    }
    const real u = std::uniform_real_distribution<real>(0.0, 1.0)(random) * total;
    real acc = 0.0;
    for (idx i = 0; i < weights.size(); ++i) {
        acc += weights[i];
        if (u < acc) {
            return i;
        }
    }
    return weights.size() - 1;
}

} // namespace num
