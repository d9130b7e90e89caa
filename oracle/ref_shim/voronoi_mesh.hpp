// The part of voronoi-cpp's API that luna-cpp's src/hydro/finite_volume.hpp reads, over mesh arrays handed in by the
// caller: TEST INFRASTRUCTURE ONLY.
//
// voronoi-cpp is fetched at configure time by the reference's build and is not installed here. To run the reference's
// own FiniteVolume<D> as the CPU oracle, this header gives it a voronoi::Mesh<D, Exec, Geometry> whose arrays are the
// ones this repository's periodic Voronoi builder produces (the same arrays the CUDA path consumes), in the layout
// FiniteVolume::refresh() reads (finite_volume.hpp:353-364): owner and neighbour per face, per-cell CSR lists with the
// owner bit (~f for a face the cell does not own, Geometry::owned_at :318), area vectors owner -> neighbour, face
// centroids relative to the owner's generator, cell centroids relative to the generator, volumes, generators, box.
// A moving mesh's update(x) calls back into the caller, which builds the mesh of the new generators.
//
// exact_predicates (the snapping grid) and tet_mesh (nearest image, list entries) restate what finite_volume.hpp needs
// of them: the grid step is 2^-30 of the longest box side (the reference's README, "positions on a 2^-30 grid"), a
// coordinate's key is its nearest grid point wrapped into [0, period), a key difference is taken to the nearest periodic
// image; the nearest image of a separation is d - side * rint(d / side); a list entry e names face e, or ~e when negative.
#pragma once

#include <Kokkos_Core.hpp>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace exact_predicates {

template <int D>
struct BoxN {
    double side[D] = {}, inverse[D] = {};
    double step = 0, per_step = 0;
    long long period[D] = {};
};

template <int D>
BoxN<D> box_of(const double* sides) {
    BoxN<D> box;
    double longest = 0;
    for (int a = 0; a < D; ++a) longest = std::fmax(longest, sides[a]);
    box.step = std::ldexp(longest, -30);
    box.per_step = 1.0 / box.step;
    for (int a = 0; a < D; ++a) {
        box.side[a] = sides[a];
        box.inverse[a] = 1.0 / sides[a];
        box.period[a] = std::llround(sides[a] / box.step);
    }
    return box;
}

// The grid key of coordinate x on axis a, in [0, period).
template <int D>
KOKKOS_INLINE_FUNCTION int snap(double x, const BoxN<D>& box, int a) {
    const long long k = std::llround(x * box.per_step), p = box.period[a];
    return static_cast<int>(((k % p) + p) % p);
}
// k1 - k0 taken to the nearest periodic image.
KOKKOS_INLINE_FUNCTION int delta(long long k0, long long k1, long long p) {
    long long d = k1 - k0;
    if (d > p / 2) d -= p;
    if (d < -(p / 2)) d += p;
    return static_cast<int>(d);
}

}  // namespace exact_predicates

namespace tet_mesh {
KOKKOS_INLINE_FUNCTION double wrap(double d, double side, double inverse) { return d - side * std::rint(d * inverse); }
KOKKOS_INLINE_FUNCTION int list_face(int e) { return e >= 0 ? e : ~e; }
}  // namespace tet_mesh

namespace voronoi {

struct Layout {
    bool owner_bit = false, owner_faces = false, float_centroids = false;
    int every = 25, flips = 0, far = 0;
    bool resorts() const { return every > 0; }
};

struct Report {
    int resorted = 0;
    long long rebuilt = 0, stuck = 0, local_done = 0, local_cells = 0, host_flips = 0, flips = 0;
};

// One mesh's arrays as plain pointers (row-major, D = dim), valid for the duration of the call that hands them over.
struct MeshArrays {
    int dim;
    std::int64_t n, f;
    const std::int32_t *owner, *neighbour, *start, *list;
    const double *area, *face_centroid, *centroid, *volume, *positions;
    double box[3];
};
// Builds the mesh of `positions` ([n][dim]) into *out; returns 0 on success.
using RemeshFn = int (*)(void* user, const double* positions, MeshArrays* out);

template <int D, class ExecSpace = Kokkos::DefaultExecutionSpace, class Geometry = double>
class Mesh {
public:
    static constexpr int dimensions = D;
    using execution_space = ExecSpace;
    using Memory = typename ExecSpace::memory_space;
    static constexpr bool float_rows = std::is_same_v<Geometry, float>;
    using Rows = Kokkos::View<const double* [D], Kokkos::LayoutRight, Memory>;
    using FaceRows = Kokkos::View<const float* [8], Kokkos::LayoutRight, Memory>;
    using Positions = Kokkos::View<const double* [D], Kokkos::LayoutRight, Memory>;
    using Points = Kokkos::View<double* [D], Kokkos::LayoutRight, Memory>;

    Mesh(const MeshArrays& arrays, RemeshFn remesh = nullptr, void* user = nullptr) : remesh_(remesh), user_(user) {
        layout_.owner_bit = true;  // the lists carry the owner bit as built
        layout_.every = 0;
        take(arrays);
    }

    int particles() const { return n_; }
    int faces() const { return f_; }
    Kokkos::View<int*, Memory> owner() const { return owner_; }
    Kokkos::View<int*, Memory> neighbour() const { return neighbour_; }
    Kokkos::View<int*, Memory> cell_face_start() const { return start_; }
    Kokkos::View<int*, Memory> cell_face() const { return list_; }
    Rows area() const { return area_; }
    Rows face_centroid() const { return face_centroid_; }
    Rows centroid() const { return centroid_; }
    FaceRows face_rows() const { return FaceRows(); }
    Kokkos::View<double*, Memory> volume() const { return volume_; }
    Positions positions() const { return positions_; }
    exact_predicates::BoxN<D> sides() const { return box_; }
    Kokkos::View<const float* [3], Kokkos::LayoutRight, Memory> face_centroid32() const { return centroid32_; }
    const Layout& layout() const { return layout_; }
    void set_layout(const Layout& layout) { layout_ = layout; }
    void update_cells() {}
    // Face centroids as float relative to the owner (voronoi::Layout::float_centroids), as a mesh built with that layout.
    void use_float_centroids(bool on) {
        layout_.float_centroids = on;
        fill_centroid32();
    }

    // Spare bytes the solver borrows for its rows (kept between calls, grown to fit).
    Kokkos::View<char*, Memory> scratch(std::size_t bytes) {
        if (scratch_.extent(0) < bytes) scratch_ = Kokkos::View<char*, Memory>(Kokkos::view_alloc(Kokkos::WithoutInitializing, std::string("mesh_scratch")), bytes);
        return scratch_;
    }

    // The mesh of the moved generators, built by the caller's callback.
    Report update(const Points& x) {
        if (!remesh_) throw std::logic_error("voronoi::Mesh::update: no remesh callback");
        MeshArrays arrays{};
        if (remesh_(user_, x.data(), &arrays) != 0) throw std::runtime_error("voronoi::Mesh::update: the remesh callback failed");
        take(arrays);
        Report report;
        report.rebuilt = 1;
        return report;
    }
    template <class... A>
    void permute(A&...) const {}

private:
    void take(const MeshArrays& a) {
        if (a.dim != D) throw std::invalid_argument("voronoi::Mesh: dimension");
        n_ = static_cast<int>(a.n);
        f_ = static_cast<int>(a.f);
        owner_ = copy_of<int*>(a.owner, f_, 1);
        neighbour_ = copy_of<int*>(a.neighbour, f_, 1);
        start_ = copy_of<int*>(a.start, n_ + 1, 1);
        list_ = copy_of<int*>(a.list, 2 * f_, 1);
        area_ = copy_of<double* [D]>(a.area, f_, D);
        face_centroid_ = copy_of<double* [D]>(a.face_centroid, f_, D);
        centroid_ = copy_of<double* [D]>(a.centroid, n_, D);
        volume_ = copy_of<double*>(a.volume, n_, 1);
        positions_ = copy_of<double* [D]>(a.positions, n_, D);
        box_ = exact_predicates::box_of<D>(a.box);
        fill_centroid32();
    }
    void fill_centroid32() {
        if (!layout_.float_centroids || D != 3) {
            centroid32_ = {};
            return;
        }
        Kokkos::View<float* [3], Kokkos::LayoutRight, Memory> c("face_centroid32", f_);
        for (int f = 0; f < f_; ++f)
            for (int a = 0; a < 3; ++a) c(f, a) = static_cast<float>(face_centroid_(f, a < D ? a : 0));
        centroid32_ = c;
    }
    template <class T, class S>
    static Kokkos::View<T, Kokkos::LayoutRight, Memory> copy_of(const S* src, int rows, int width) {
        Kokkos::View<T, Kokkos::LayoutRight, Memory> v(Kokkos::view_alloc(Kokkos::WithoutInitializing, std::string("mesh")), rows);
        if (rows > 0) std::memcpy(v.data(), src, sizeof(S) * static_cast<std::size_t>(rows) * width);
        return v;
    }

    RemeshFn remesh_ = nullptr;
    void* user_ = nullptr;
    int n_ = 0, f_ = 0;
    Layout layout_;
    Kokkos::View<int*, Kokkos::LayoutRight, Memory> owner_, neighbour_, start_, list_;
    Kokkos::View<double* [D], Kokkos::LayoutRight, Memory> area_, face_centroid_, centroid_, positions_;
    Kokkos::View<double*, Kokkos::LayoutRight, Memory> volume_;
    Kokkos::View<const float* [3], Kokkos::LayoutRight, Memory> centroid32_;
    exact_predicates::BoxN<D> box_;
    Kokkos::View<char*, Memory> scratch_;
};

}  // namespace voronoi
