// The bucket grid of the Voronoi builders (host code): its shape and the bucket offsets to visit, shared by the host
// builder (voronoi_build.cpp) and the device remesher (remesh.cu), which fill the buckets themselves.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "voronoi_cell.h"

namespace luna_voronoi {

struct GridShape {
    static constexpr int kReach = 8;  // buckets per axis the offsets reach
    int dim = 3;
    int nb[3] = {1, 1, 1};
    double w[3] = {1, 1, 1};
    int64_t buckets = 1;
    std::vector<int32_t> offsets;  // [k][3], by the lower bound of their distance
    std::vector<double> bound2;

    // About one point per bucket; offsets up to 8 buckets away per axis, stably sorted by the squared distance any point
    // of the offset bucket has at least (gaps of whole buckets between it and the centre bucket).
    void build(int d, int64_t n, const double* side) {
        dim = d;
        double vol = 1;
        for (int a = 0; a < d; ++a) vol *= side[a];
        const double spacing = std::pow(vol / static_cast<double>(n), 1.0 / d);
        buckets = 1;
        for (int a = 0; a < 3; ++a) {
            nb[a] = a < d ? std::max(1, static_cast<int>(std::floor(side[a] / spacing))) : 1;
            w[a] = a < d ? side[a] / nb[a] : 1.0;
            buckets *= nb[a];
        }
        const int K = kReach;
        std::vector<std::array<int, 3>> all;
        for (int x = -K; x <= K; ++x)
            for (int y = (d >= 2 ? -K : 0); y <= (d >= 2 ? K : 0); ++y)
                for (int z = (d >= 3 ? -K : 0); z <= (d >= 3 ? K : 0); ++z) all.push_back({x, y, z});
        auto lower = [&](const std::array<int, 3>& o) {
            double s = 0;
            for (int a = 0; a < d; ++a) {
                const double g = std::max(0, std::abs(o[a]) - 1) * w[a];
                s += g * g;
            }
            return s;
        };
        std::stable_sort(all.begin(), all.end(), [&](const auto& p, const auto& q) { return lower(p) < lower(q); });
        offsets.resize(3 * all.size());
        bound2.resize(all.size());
        for (size_t k = 0; k < all.size(); ++k) {
            for (int a = 0; a < 3; ++a) offsets[3 * k + a] = all[k][a];
            bound2[k] = lower(all[k]);
        }
    }
    Grid view(const int64_t* start, const int32_t* items, const int32_t* offsets_at, const double* bound2_at) const {
        Grid g;
        g.dim = dim;
        for (int a = 0; a < 3; ++a) {
            g.nb[a] = nb[a];
            g.w[a] = w[a];
        }
        g.start = start;
        g.items = items;
        g.offsets = offsets_at;
        g.bound2 = bound2_at;
        g.n_offsets = static_cast<int>(bound2.size());
        g.reach = kReach;
        return g;
    }
};

// A generator coordinate wrapped into [0, side).
LUNA_VC_HD double wrap_coordinate(double x, double side) {
    x -= side * floor(x / side);
    if (x >= side) x -= side;
    return x;
}

}  // namespace luna_voronoi
