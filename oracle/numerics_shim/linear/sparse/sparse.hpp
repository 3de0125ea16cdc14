// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
// Compressed-row sparse matrix with triplet assembly (duplicates summed), as used by
// generator::assemble (markovkit/generator.hpp:93-107) and num::expv.
#pragma once

#include "container/vector.hpp"
#include "linear/operator.hpp"
#include <algorithm>
#include <cmath>
#include <numeric>

namespace num {

class spmat {
  public:
    using domain_type = vec<real>;
    using codomain_type = vec<real>;

    spmat() = default;
    spmat(idx rows, idx cols, array<real> values, array<idx> columns, array<idx> row_ptr)
        : rows_(rows), cols_(cols), value_(std::move(values)), column_(std::move(columns)),
          ptr_(std::move(row_ptr)) {}

    static spmat from_triplets(idx rows, idx cols, const array<idx> &row, const array<idx> &col,
                               const array<real> &value) {
        array<idx> order(row.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](idx a, idx b) {
            return row[a] != row[b] ? row[a] < row[b] : col[a] < col[b];
        });
        array<idx> ptr(rows + 1, 0), columns;
        array<real> values;
        columns.reserve(order.size());
        values.reserve(order.size());
        idx last_row = static_cast<idx>(-1), last_col = static_cast<idx>(-1);
        for (idx k : order) {
            if (row[k] == last_row && col[k] == last_col) {
                values.back() += value[k];
                continue;
            }
            columns.push_back(col[k]);
            values.push_back(value[k]);
            ++ptr[row[k] + 1];
            last_row = row[k];
            last_col = col[k];
        }
        for (idx i = 0; i < rows; ++i) {
            ptr[i + 1] += ptr[i];
        }
        return spmat(rows, cols, std::move(values), std::move(columns), std::move(ptr));
    }

    [[nodiscard]] idx rows() const { return rows_; }
    [[nodiscard]] idx cols() const { return cols_; }
    [[nodiscard]] idx nonzeros() const { return value_.size(); }
    [[nodiscard]] const array<idx> &row_ptr() const { return ptr_; }
    [[nodiscard]] const array<idx> &columns() const { return column_; }
    [[nodiscard]] const array<real> &values() const { return value_; }

    void apply(view<const real> x, view<real> y) const {
        for (idx i = 0; i < rows_; ++i) {
            real sum = 0.0;
            for (idx k = ptr_[i]; k < ptr_[i + 1]; ++k) {
                sum += value_[k] * x[column_[k]];
            }
            y[i] = sum;
        }
    }
    void apply(const vec<real> &x, vec<real> &y) const {
        apply(view<const real>(x), view<real>(y));
    }

    // max over rows of the absolute row sum
    [[nodiscard]] real norm_inf() const {
        real result = 0.0;
        for (idx i = 0; i < rows_; ++i) {
            real sum = 0.0;
            for (idx k = ptr_[i]; k < ptr_[i + 1]; ++k) {
                sum += std::abs(value_[k]);
            }
            result = std::max(result, sum);
        }
        return result;
    }

  private:
    idx rows_ = 0, cols_ = 0;
    array<real> value_;
    array<idx> column_;
    array<idx> ptr_;
};

} // namespace num
