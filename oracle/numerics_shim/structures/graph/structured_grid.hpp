// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
//
// Cartesian voxel grid as MarkovKit's RDME uses it (markovkit/rdme/multigrid.hpp:20-42,
// reaction_diffusion.hpp:14-56). Conventions restated from the reference's tests and the
// paper driver: vertices are numbered with axis 0 fastest (rdme/cpp/rdme_full_multigrid.cpp:
// 391-398,550-558); the boundary is closed, so a corner of a 2-D grid has two neighbours
// (tests/test_rdme.cpp:28); an edge along axis a has weight (face area) / h_a and the cell
// volume is the product of the spacings (tests/test_rdme.cpp:22-33). Neighbours are listed
// axis by axis, the lower one first.
#pragma once

#include "container/vector.hpp"
#include <cstdint>

namespace num {

enum class grid_boundary : std::uint8_t { closed };

template <std::size_t D>
class structured_grid_graph {
  public:
    using index_type = idx;
    struct edge {
        idx to;
        double weight;
    };

    structured_grid_graph(static_array<idx, D> dimensions, static_array<double, D> spacing = ones(),
                          static_array<grid_boundary, D> boundaries = closed())
        : dimensions_(dimensions), spacing_(spacing), boundaries_(boundaries) {
        n_ = 1;
        for (std::size_t a = 0; a < D; ++a) {
            stride_[a] = n_;
            n_ *= dimensions_[a];
        }
        first_.assign(n_ + 1, 0);
        for (idx v = 0; v < n_; ++v) {
            const auto c = coordinate(v);
            for (std::size_t a = 0; a < D; ++a) {
                double face = 1.0;
                for (std::size_t b = 0; b < D; ++b) {
                    if (b != a) {
                        face *= spacing_[b];
                    }
                }
                const double w = face / spacing_[a];
                if (c[a] > 0) {
                    edges_.push_back({v - stride_[a], w});
                }
                if (c[a] + 1 < dimensions_[a]) {
                    edges_.push_back({v + stride_[a], w});
                }
            }
            first_[v + 1] = edges_.size();
        }
    }

    [[nodiscard]] idx n_vertices() const { return n_; }
    [[nodiscard]] view<const edge> neighbors(idx v) const {
        return {edges_.data() + first_[v], first_[v + 1] - first_[v]};
    }
    [[nodiscard]] static_array<idx, D> coordinate(idx v) const {
        static_array<idx, D> c{};
        for (std::size_t a = 0; a < D; ++a) {
            c[a] = v % dimensions_[a];
            v /= dimensions_[a];
        }
        return c;
    }
    [[nodiscard]] idx vertex(const static_array<idx, D> &c) const {
        idx v = 0;
        for (std::size_t a = 0; a < D; ++a) {
            v += c[a] * stride_[a];
        }
        return v;
    }
    [[nodiscard]] const static_array<idx, D> &dimensions() const { return dimensions_; }
    [[nodiscard]] const static_array<double, D> &spacing() const { return spacing_; }
    [[nodiscard]] const static_array<grid_boundary, D> &boundaries() const { return boundaries_; }
    [[nodiscard]] double cell_volume() const {
        double v = 1.0;
        for (double h : spacing_) {
            v *= h;
        }
        return v;
    }

  private:
    static static_array<double, D> ones() {
        static_array<double, D> s{};
        s.fill(1.0);
        return s;
    }
    static static_array<grid_boundary, D> closed() {
        static_array<grid_boundary, D> b{};
        b.fill(grid_boundary::closed);
        return b;
    }

    static_array<idx, D> dimensions_;
    static_array<double, D> spacing_;
    static_array<grid_boundary, D> boundaries_;
    static_array<idx, D> stride_{};
    idx n_ = 0;
    array<idx> first_;
    array<edge> edges_;
};

} // namespace num
