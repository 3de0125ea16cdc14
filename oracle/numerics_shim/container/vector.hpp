// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
// Containers as MarkovKit uses them: growable arrays, numeric vectors and non-owning views.
#pragma once

#include "core/types.hpp"
#include <array>
#include <map>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace num {

template <typename T>
using array = std::vector<T>;

template <typename T>
using vec = std::vector<T>;

template <typename T, std::size_t N>
using static_array = std::array<T, N>;

template <typename K, typename V, typename C = std::less<K>>
using map = std::map<K, V, C>;

template <typename K, typename V, typename H = std::hash<K>, typename E = std::equal_to<K>>
using unordered_map = std::unordered_map<K, V, H, E>;

// a pointer and a length
template <typename T>
class view {
  public:
    using value_type = std::remove_const_t<T>;

    view() = default;
    view(T *data, idx size) : data_(data), size_(size) {}
    // from a vector: mutable views need a mutable vector, const views take either
    view(std::vector<value_type> &v) : data_(v.data()), size_(v.size()) {}
    template <typename U = T, typename = std::enable_if_t<std::is_const_v<U>>>
    view(const std::vector<value_type> &v) : data_(v.data()), size_(v.size()) {}
    template <typename U, typename = std::enable_if_t<std::is_const_v<T> &&
                                                      std::is_same_v<U, value_type>>>
    view(view<U> other) : data_(other.data()), size_(other.size()) {}

    [[nodiscard]] T *data() const { return data_; }
    [[nodiscard]] idx size() const { return size_; }
    [[nodiscard]] bool empty() const { return size_ == 0; }
    [[nodiscard]] T *begin() const { return data_; }
    [[nodiscard]] T *end() const { return data_ + size_; }
    T &operator[](idx i) const { return data_[i]; }

  private:
    T *data_ = nullptr;
    idx size_ = 0;
};

} // namespace num
