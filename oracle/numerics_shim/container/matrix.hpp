// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
// Dense row-major matrix, as used by population_multigrid::factor and fsp_solution::means.
#pragma once

#include "container/vector.hpp"

namespace num {

template <typename T>
class mat {
  public:
    mat() = default;
    mat(idx rows, idx cols, T value = T{}) : rows_(rows), cols_(cols), data_(rows * cols, value) {}

    [[nodiscard]] idx rows() const { return rows_; }
    [[nodiscard]] idx cols() const { return cols_; }
    T &operator()(idx i, idx j) { return data_[(i * cols_) + j]; }
    const T &operator()(idx i, idx j) const { return data_[(i * cols_) + j]; }
    [[nodiscard]] T *data() { return data_.data(); }
    [[nodiscard]] const T *data() const { return data_.data(); }

  private:
    idx rows_ = 0, cols_ = 0;
    std::vector<T> data_;
};

} // namespace num
