// The reference's own hydro::FiniteVolume<D> (luna-cpp src/hydro/finite_volume.hpp, euler.hpp, precision.hpp, compiled
// unmodified from the reference's tree) behind a C ABI: TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/Makefile into oracle/_ref/libluna_ref.so against ref_shim/ (a host-only Kokkos and the part of
// voronoi-cpp the solver reads, over mesh arrays from this repository's builder). The tests use it to pin the C
// restatement in luna_oracle.c, and through it the CUDA path, to the reference's own arithmetic; bench.py may time it
// as the reference's CPU path. Nothing in the product links it.
// Compiled as three objects (oracle/Makefile): LR_PART 2 and 3 instantiate the solvers of one dimension each (the
// heavy part, built in parallel), LR_PART 0 the C ABI.
#include "finite_volume.hpp"

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

namespace lr {

// A GeometryDerivative (mesh_derivative.hpp:10-29) whose tangent and adjoint are the caller's: the tests hand in their
// own 2D geometry derivative (as the reference's tests hand in theirs, src/test/reference_geometry_2d.hpp).
typedef void (*GeoTangent)(void* user, const double* dx, double* dV, double* dc, double* dA, double* dxf);
typedef void (*GeoAdjoint)(void* user, const double* Vbar, const double* cbar, const double* Abar, const double* xfbar, double* xbar);

struct Solver {
    virtual ~Solver() = default;
    virtual int cells() const = 0;
    virtual int faces() const = 0;
    virtual double* state() = 0;
    virtual double time_step(double courant) = 0;
    virtual void step(double dt) = 0;
    virtual long long fallbacks() = 0;
    virtual void step_adjoint(double dt, double* qbar) = 0;
    virtual double time_step_tangent(double courant, double* dq) = 0;
    virtual void step_tangent(double dt, double* dq) = 0;
    virtual const double* positions() = 0;
    virtual const double* point_velocities() = 0;
    virtual void density_gradients(double* out) = 0;
    virtual void set_positions(const double* x) = 0;
    virtual void step_moving_tangent(double dt, double* dq, double* dx, GeoTangent t, GeoAdjoint a, void* user, bool fixed) = 0;
    virtual void step_moving_adjoint(double dt, double* qbar, double* xbar, GeoTangent t, GeoAdjoint a, void* user, bool fixed) = 0;
};

template <class Base>
struct CallbackGeometry : Base {
    using typename Base::Points;
    using typename Base::Scalars;
    GeoTangent t;
    GeoAdjoint a;
    void* user;
    CallbackGeometry(GeoTangent t_, GeoAdjoint a_, void* u) : t(t_), a(a_), user(u) {}
    void tangent(const Points& dx, const Scalars& dV, const Points& dc, const Points& dA, const Points& dxf) const override {
        t(user, dx.data(), dV.data(), dc.data(), dA.data(), dxf.data());
    }
    void adjoint(const Scalars& Vbar, const Points& cbar, const Points& Abar, const Points& xfbar, const Points& xbar) const override {
        a(user, Vbar.data(), cbar.data(), Abar.data(), xfbar.data(), xbar.data());
    }
};

template <int D, class Riemann, class Precision>
struct SolverOf : Solver {
    using Exec = Kokkos::OpenMP;
    using FV = hydro::FiniteVolume<D, Exec, Riemann, Precision>;
    using Mesh = typename FV::Mesh;
    static constexpr int V = D + 2;

    Mesh mesh;
    FV fv;
    SolverOf(const voronoi::MeshArrays& arrays, voronoi::RemeshFn remesh, void* user, const hydro::Gas& gas, int order, hydro::Update update,
             hydro::Limiter limiter, hydro::Motion motion)
        : mesh(arrays, remesh, user), fv(Exec{}, mesh, gas, order, update, limiter, motion) {}

    int cells() const override { return mesh.particles(); }
    int faces() const override { return mesh.faces(); }
    double* state() override { return fv.state().data(); }
    double time_step(double courant) override { return fv.time_step(courant); }
    void step(double dt) override { fv.step(dt); }
    long long fallbacks() override { return fv.fallbacks(); }
    void step_adjoint(double dt, double* qbar) override {
        if constexpr (std::is_same_v<typename Precision::flux, double> && std::is_same_v<typename Precision::riemann, double>) {
            typename FV::Cells bar(qbar, static_cast<std::size_t>(cells()));
            fv.step_adjoint(dt, bar);
        } else {
            throw std::logic_error("step_adjoint: double flux rows and Riemann solve only");
        }
    }
    double time_step_tangent(double courant, double* dq) override {
        if constexpr (std::is_same_v<typename Precision::flux, double> && std::is_same_v<typename Precision::riemann, double>) {
            typename FV::Cells d(dq, static_cast<std::size_t>(cells()));
            return fv.time_step_tangent(courant, d);
        } else {
            throw std::logic_error("time_step_tangent: double flux rows and Riemann solve only");
        }
    }
    void step_tangent(double dt, double* dq) override {
        if constexpr (std::is_same_v<typename Precision::flux, double> && std::is_same_v<typename Precision::riemann, double>) {
            typename FV::Cells d(dq, static_cast<std::size_t>(cells()));
            fv.step_tangent(dt, d);
        } else {
            throw std::logic_error("step_tangent: double flux rows and Riemann solve only");
        }
    }
    const double* positions() override { return fv.motion() == hydro::Motion::moving ? fv.positions().data() : nullptr; }
    const double* point_velocities() override { return fv.motion() == hydro::Motion::moving ? fv.point_velocities().data() : nullptr; }
    void density_gradients(double* out) override {
        const auto rows = fv.density_gradients();
        std::memcpy(out, rows.data(), sizeof(double) * rows.size());
    }
    // Rollout::load_positions (rollout.cpp:146-152): the positions, the mesh of them, mesh_moved().
    void set_positions(const double* x) override {
        if (fv.motion() != hydro::Motion::moving) throw std::logic_error("set_positions: a moving mesh");
        std::memcpy(fv.positions().data(), x, sizeof(double) * D * static_cast<std::size_t>(cells()));
        mesh.update(fv.positions());
        mesh.update_cells();
        fv.mesh_moved();
    }
    void step_moving_tangent(double dt, double* dq, double* dx, GeoTangent t, GeoAdjoint a, void* user, bool fixed) override {
        if constexpr (std::is_same_v<typename Precision::flux, double> && std::is_same_v<typename Precision::riemann, double>) {
            typename FV::Cells q(dq, static_cast<std::size_t>(cells()));
            typename FV::Points x(dx, static_cast<std::size_t>(cells()));
            const CallbackGeometry<typename FV::Derivative> geometry(t, a, user);
            fv.step_moving_tangent(dt, q, x, geometry, fixed);
        } else {
            throw std::logic_error("step_moving_tangent: double flux rows and Riemann solve only");
        }
    }
    void step_moving_adjoint(double dt, double* qbar, double* xbar, GeoTangent t, GeoAdjoint a, void* user, bool fixed) override {
        if constexpr (std::is_same_v<typename Precision::flux, double> && std::is_same_v<typename Precision::riemann, double>) {
            typename FV::Cells q(qbar, static_cast<std::size_t>(cells()));
            typename FV::Points x(xbar, static_cast<std::size_t>(cells()));
            const CallbackGeometry<typename FV::Derivative> geometry(t, a, user);
            fv.step_moving_adjoint(dt, q, x, geometry, fixed);
        } else {
            throw std::logic_error("step_moving_adjoint: double flux rows and Riemann solve only");
        }
    }
};

#if LR_PART == 2 || LR_PART == 3
// precision: 0 Precision<> (double), 1 riemann32 = Precision<double, float, double, float> (hydro_sedov.cpp:422),
// 2 Grad32, 3 Grad16 = Precision<double, Half>, 4 single = Precision<double, float, float, float> (hydro_sedov.cpp:423).
template <int D>
Solver* make_solver(const voronoi::MeshArrays& m, voronoi::RemeshFn fn, void* user, const hydro::Gas& gas, int order, hydro::Update update,
             hydro::Limiter limiter, hydro::Motion motion, int riemann, int precision) {
    using hydro::Precision;
    if (riemann == 1) {
        if (precision != 0) throw std::invalid_argument("HLL: double precision only in this driver");
        return new SolverOf<D, hydro::HLL, Precision<>>(m, fn, user, gas, order, update, limiter, motion);
    }
    switch (precision) {
        case 0: return new SolverOf<D, hydro::HLLC, Precision<>>(m, fn, user, gas, order, update, limiter, motion);
        case 1: return new SolverOf<D, hydro::HLLC, Precision<double, float, double, float>>(m, fn, user, gas, order, update, limiter, motion);
        case 2: return new SolverOf<D, hydro::HLLC, hydro::Grad32>(m, fn, user, gas, order, update, limiter, motion);
        case 3: return new SolverOf<D, hydro::HLLC, Precision<double, hydro::Half>>(m, fn, user, gas, order, update, limiter, motion);
        case 4: return new SolverOf<D, hydro::HLLC, Precision<double, float, float, float>>(m, fn, user, gas, order, update, limiter, motion);
        default: throw std::invalid_argument("precision 0..4");
    }
}
template Solver* make_solver<LR_PART>(const voronoi::MeshArrays&, voronoi::RemeshFn, void*, const hydro::Gas&, int, hydro::Update,
                                     hydro::Limiter, hydro::Motion, int, int);
#else
template <int D>
Solver* make_solver(const voronoi::MeshArrays& m, voronoi::RemeshFn fn, void* user, const hydro::Gas& gas, int order, hydro::Update update,
                    hydro::Limiter limiter, hydro::Motion motion, int riemann, int precision);
#endif
}  // namespace lr

#if LR_PART == 0
namespace {
using lr::Solver;
thread_local std::string g_error;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

}  // namespace

extern "C" {

typedef voronoi::MeshArrays lr_mesh;

const char* lr_last_error(void) { return g_error.c_str(); }

int lr_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    return omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

// FiniteVolume(exec, mesh, gas, order, update, limiter, motion) (finite_volume.hpp:79-107). per_face: Update::per_face;
// limiter 0 face_centroid, 1 none; riemann 0 HLLC, 1 HLL; moving: Motion::moving (remesh builds each new mesh).
void* lr_fv_create(const lr_mesh* mesh, double gamma, int order, int per_face, int limiter, int riemann, int moving, int precision,
                   voronoi::RemeshFn remesh, void* user) {
    Solver* s = nullptr;
    const int rc = guarded([&] {
        const hydro::Gas gas(gamma);
        const auto update = per_face ? hydro::Update::per_face : hydro::Update::per_cell;
        const auto lim = limiter ? hydro::Limiter::none : hydro::Limiter::face_centroid;
        const auto motion = moving ? hydro::Motion::moving : hydro::Motion::static_mesh;
        if (mesh->dim == 3)
            s = lr::make_solver<3>(*mesh, remesh, user, gas, order, update, lim, motion, riemann, precision);
        else if (mesh->dim == 2)
            s = lr::make_solver<2>(*mesh, remesh, user, gas, order, update, lim, motion, riemann, precision);
        else
            throw std::invalid_argument("dim 2 or 3");
    });
    return rc == 0 ? s : nullptr;
}
void lr_fv_destroy(void* h) { delete static_cast<Solver*>(h); }
// state(): the extensive Q [N][D + 2]; taking it marks the primitive rows stale, so write it before the next step.
double* lr_fv_state(void* h) { return static_cast<Solver*>(h)->state(); }
int lr_fv_time_step(void* h, double courant, double* dt) {
    return guarded([&] { *dt = static_cast<Solver*>(h)->time_step(courant); });
}
int lr_fv_step(void* h, double dt) {
    return guarded([&] { static_cast<Solver*>(h)->step(dt); });
}
long long lr_fv_fallbacks(void* h) { return static_cast<Solver*>(h)->fallbacks(); }
// step_adjoint(dt, qbar) (:2201-2231): qbar [N][V] in and out; Q stays the state before the step.
int lr_fv_step_adjoint(void* h, double dt, double* qbar) {
    return guarded([&] { static_cast<Solver*>(h)->step_adjoint(dt, qbar); });
}
int lr_fv_time_step_tangent(void* h, double courant, double* dq, double* dt) {
    return guarded([&] { *dt = static_cast<Solver*>(h)->time_step_tangent(courant, dq); });
}
// step_tangent(dt, dq) (:2033-2062): dq [N][V] in and out; Q advances as step().
int lr_fv_step_tangent(void* h, double dt, double* dq) {
    return guarded([&] { static_cast<Solver*>(h)->step_tangent(dt, dq); });
}
const double* lr_fv_positions(void* h) { return static_cast<Solver*>(h)->positions(); }
const double* lr_fv_point_velocities(void* h) { return static_cast<Solver*>(h)->point_velocities(); }
int lr_fv_cells(void* h) { return static_cast<Solver*>(h)->cells(); }
int lr_fv_faces(void* h) { return static_cast<Solver*>(h)->faces(); }
int lr_fv_density_gradients(void* h, double* out) {
    return guarded([&] { static_cast<Solver*>(h)->density_gradients(out); });
}
// A moving mesh's positions [N][D] and the mesh of them (the state is kept).
int lr_fv_set_positions(void* h, const double* x) {
    return guarded([&] { static_cast<Solver*>(h)->set_positions(x); });
}
// step_moving_tangent / step_moving_adjoint (finite_volume.hpp:2431-3155) with the caller's geometry derivative; fixed: the
// order-1 derivatives' steps_fixed (the grid steps held).
int lr_fv_step_moving_tangent(void* h, double dt, double* dq, double* dx, lr::GeoTangent t, lr::GeoAdjoint a, void* user, int fixed) {
    return guarded([&] { static_cast<Solver*>(h)->step_moving_tangent(dt, dq, dx, t, a, user, fixed != 0); });
}
int lr_fv_step_moving_adjoint(void* h, double dt, double* qbar, double* xbar, lr::GeoTangent t, lr::GeoAdjoint a, void* user, int fixed) {
    return guarded([&] { static_cast<Solver*>(h)->step_moving_adjoint(dt, qbar, xbar, t, a, user, fixed != 0); });
}

}  // extern "C"
#endif
