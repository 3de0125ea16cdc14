// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
// An explicit undirected weighted graph: add_edge(a, b, w) adds a -> b and b -> a
// (tests/test_rdme.cpp:35-43 reads both directions).
#pragma once

#include "container/vector.hpp"

namespace num {

template <typename W = double, typename I = idx>
class graph {
  public:
    using index_type = I;
    struct edge {
        I to;
        W weight;
    };

    explicit graph(I vertices = 0) : adjacency_(vertices) {}

    void add_edge(I a, I b, W weight) {
        adjacency_[a].push_back({b, weight});
        adjacency_[b].push_back({a, weight});
    }

    [[nodiscard]] idx n_vertices() const { return adjacency_.size(); }
    [[nodiscard]] view<const edge> neighbors(I v) const {
        return {adjacency_[v].data(), adjacency_[v].size()};
    }

  private:
    array<array<edge>> adjacency_;
};

} // namespace num
