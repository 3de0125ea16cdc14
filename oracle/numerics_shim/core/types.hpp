// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Project-written stand-in for the numerics library that MarkovKit includes from its
// un-vendored git submodule `ext/numerics` (github.com/AdityaDendukuri/numerics; the
// submodule revision is not recorded in the reference tree). Only the API surface that
// MarkovKit's headers, tests and the resolvent/FSP examples use is provided, restated from
// those call sites. Nothing in the product may include this directory.
#pragma once

#include <cstddef>
#include <cstdint>

namespace num {

// 64-bit unsigned index: the reference compares idx values after casting to `long`
// (tests/test_rdme.cpp:131) and sizes containers with it.
using idx = std::size_t;
using real = double;

} // namespace num
