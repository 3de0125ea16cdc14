// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
// The linear-operator concept the reference's tests assert (tests/test_rdme.cpp:104,163,216,232).
#pragma once

#include "container/vector.hpp"
#include <concepts>

namespace num {

template <typename Op, typename In, typename Out>
concept linear_operator = requires(const Op &op, const In &x, Out &y) {
    { op.rows() } -> std::convertible_to<idx>;
    { op.cols() } -> std::convertible_to<idx>;
    op.apply(x, y);
};

} // namespace num
