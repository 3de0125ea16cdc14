// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
#pragma once

#include "container/vector.hpp"
#include <algorithm>
#include <numeric>

namespace num {

// the indices of the `count` smallest values, ties broken by index (markovkit/fsp.hpp:169)
inline array<idx> smallest_indices(view<const real> values, idx count) {
    array<idx> order(values.size());
    std::iota(order.begin(), order.end(), 0);
    count = std::min(count, order.size());
    std::partial_sort(order.begin(), order.begin() + count, order.end(), [&](idx a, idx b) {
        return values[a] != values[b] ? values[a] < values[b] : a < b;
    });
    order.resize(count);
    return order;
}

} // namespace num
