// A host-only stand-in for the part of Kokkos's API that luna-cpp's solver headers use (src/hydro/euler.hpp,
// precision.hpp, finite_volume.hpp, mesh_derivative.hpp): TEST INFRASTRUCTURE ONLY.
//
// Kokkos 5.0 is not installed here, so the reference's own FiniteVolume<D> is compiled against this header to run it
// on the CPU as the oracle of the CUDA path. It implements the symbols those files name, with Kokkos's meaning, for one
// memory space (host memory) and two execution spaces: Serial, and OpenMP (parallel_for / parallel_reduce over a
// RangePolicy split across OpenMP threads; every reduction the solver runs is a minimum, a maximum or an integer sum, so
// the result does not depend on the split). Views are reference-counted, row-major (LayoutRight) arrays of rank 0 to 3
// with Kokkos's data-type syntax (T*, T**, T*[N], T[N]); a view built from a pointer does not own it.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]

namespace Kokkos {

// ---- spaces
struct HostSpace {
    using memory_space = HostSpace;
};
struct Serial {
    using memory_space = HostSpace;
    using execution_space = Serial;
    static constexpr bool parallel = false;
    void fence() const {}
    void fence(const std::string&) const {}
};
struct OpenMP {
    using memory_space = HostSpace;
    using execution_space = OpenMP;
    static constexpr bool parallel = true;
    void fence() const {}
    void fence(const std::string&) const {}
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

template <class A, class B>
struct SpaceAccessibility {
    static constexpr bool accessible = true;
    static constexpr bool assignable = true;
};

inline void fence() {}
inline void fence(const std::string&) {}

// ---- layouts and memory traits
struct LayoutRight {
    std::size_t dimension[3] = {0, 0, 0};
    LayoutRight() = default;
    explicit LayoutRight(std::size_t n0, std::size_t n1 = 0, std::size_t n2 = 0) : dimension{n0, n1, n2} {}
};
enum MemoryTraitsFlags : unsigned { Unmanaged = 1u, RandomAccess = 2u, Atomic = 4u, Restrict = 8u };
template <unsigned Flags>
struct MemoryTraits {
    static constexpr unsigned flags = Flags;
};
using MemoryUnmanaged = MemoryTraits<Unmanaged>;

// ---- allocation properties
struct WithoutInitializing_t {};
inline constexpr WithoutInitializing_t WithoutInitializing{};
struct ViewAllocProp {
    std::string label;
    bool initialize = true;
};
inline ViewAllocProp view_alloc_one(ViewAllocProp p, WithoutInitializing_t) {
    p.initialize = false;
    return p;
}
inline ViewAllocProp view_alloc_one(ViewAllocProp p, const std::string& label) {
    p.label = label;
    return p;
}
inline ViewAllocProp view_alloc_one(ViewAllocProp p, const char* label) {
    p.label = label;
    return p;
}
template <class E, std::enable_if_t<std::is_class_v<E> && !std::is_same_v<E, std::string> && !std::is_same_v<E, WithoutInitializing_t>, int> = 0>
inline ViewAllocProp view_alloc_one(ViewAllocProp p, const E&) {  // an execution space instance: ignored
    return p;
}
template <class... A>
ViewAllocProp view_alloc(const A&... a) {
    ViewAllocProp p;
    ((p = view_alloc_one(p, a)), ...);
    return p;
}

// ---- the data-type syntax of a view: dynamic extents (pointers) first, then static ones (arrays)
namespace impl {
template <class T>
struct Dims {
    using value_type = T;
    static constexpr int dynamic = 0, statics = 0;
    static constexpr std::size_t ext(int) { return 0; }
};
template <class T>
struct Dims<T*> {
    using value_type = typename Dims<T>::value_type;
    static constexpr int dynamic = Dims<T>::dynamic + 1, statics = Dims<T>::statics;
    static constexpr std::size_t ext(int s) { return Dims<T>::ext(s); }
};
template <class T, std::size_t N>
struct Dims<T[N]> {
    using value_type = typename Dims<T>::value_type;
    static constexpr int dynamic = Dims<T>::dynamic, statics = Dims<T>::statics + 1;
    static constexpr std::size_t ext(int s) { return s == 0 ? N : Dims<T>::ext(s - 1); }
};
template <class P, class... Ps>
struct HasUnmanaged {
    static constexpr bool value = false;
};
template <unsigned F, class... Ps>
struct HasUnmanaged<MemoryTraits<F>, Ps...> {
    static constexpr bool value = (F & Unmanaged) != 0;
};
template <class P, class Q, class... Ps>
struct HasUnmanaged<P, Q, Ps...> : HasUnmanaged<Q, Ps...> {};
inline void* allocate(std::size_t bytes, bool zero) {
    const std::size_t size = (std::max<std::size_t>(bytes, 1) + 63) / 64 * 64;
    void* p = std::aligned_alloc(64, size);
    if (!p) throw std::bad_alloc();
    if (zero) std::memset(p, 0, size);
    return p;
}
}  // namespace impl

struct ALL_t {};
inline constexpr ALL_t ALL{};

template <class DataType, class... Props>
class View {
    using dims = impl::Dims<DataType>;

public:
    using data_type = DataType;
    using value_type = typename dims::value_type;
    using non_const_value_type = std::remove_const_t<value_type>;
    using const_value_type = std::add_const_t<value_type>;
    using pointer_type = value_type*;
    using reference_type = value_type&;
    using array_layout = LayoutRight;
    using memory_space = HostSpace;
    using execution_space = DefaultExecutionSpace;
    using HostMirror = View;
    static constexpr int rank = dims::dynamic + dims::statics;
    static constexpr int rank_dynamic = dims::dynamic;
    static_assert(rank <= 3, "views of rank 0 to 3");

    static constexpr std::size_t static_extent(int r) { return r < dims::dynamic ? 0 : dims::ext(r - dims::dynamic); }

    View() { set_extents(0, 0, 0); }
    // Allocating constructors: a label (zero-filled), or view_alloc(label, WithoutInitializing).
    explicit View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0) {
        allocate(ViewAllocProp{label, true}, n0, n1, n2);
    }
    explicit View(const char* label, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0) {
        allocate(ViewAllocProp{label, true}, n0, n1, n2);
    }
    View(const ViewAllocProp& prop, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0) { allocate(prop, n0, n1, n2); }
    View(const ViewAllocProp& prop, const LayoutRight& layout) {
        allocate(prop, layout.dimension[0], layout.dimension[1], layout.dimension[2]);
    }
    // Unmanaged: a view of the caller's memory.
    View(value_type* data, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0) : data_(data) { set_extents(n0, n1, n2); }
    // From a view of the same shape with other properties, or of non-const to const values.
    template <class D2, class... P2,
              std::enable_if_t<std::is_convertible_v<typename View<D2, P2...>::value_type*, value_type*> &&
                                   View<D2, P2...>::rank == rank,
                               int> = 0>
    View(const View<D2, P2...>& other) : data_(other.data()), owner_(other.owner()), label_(other.label()) {
        for (int r = 0; r < 3; ++r) ext_[r] = r < rank ? other.extent(r) : 0;
        check_static();
    }

    std::size_t extent(int r) const { return r < rank ? ext_[r] : 1; }
    int extent_int(int r) const { return static_cast<int>(extent(r)); }
    std::size_t size() const {
        std::size_t s = 1;
        for (int r = 0; r < rank; ++r) s *= ext_[r];
        return s;
    }
    std::size_t span() const { return size(); }
    value_type* data() const { return data_; }
    const std::shared_ptr<void>& owner() const { return owner_; }
    const std::string& label() const { return label_; }
    LayoutRight layout() const { return LayoutRight(extent(0), extent(1), extent(2)); }
    bool is_allocated() const { return data_ != nullptr; }
    int use_count() const { return static_cast<int>(owner_.use_count()); }

    template <class... I>
    value_type& operator()(I... i) const {
        static_assert(sizeof...(I) == rank || (rank == 0 && sizeof...(I) == 0), "index count");
        return data_[offset(static_cast<std::size_t>(i)...)];
    }
    value_type& operator[](std::size_t i) const { return data_[i]; }

private:
    std::size_t offset() const { return 0; }
    std::size_t offset(std::size_t i) const { return i; }
    std::size_t offset(std::size_t i, std::size_t j) const { return i * ext_[1] + j; }
    std::size_t offset(std::size_t i, std::size_t j, std::size_t k) const { return (i * ext_[1] + j) * ext_[2] + k; }
    void set_extents(std::size_t n0, std::size_t n1, std::size_t n2) {
        const std::size_t given[3] = {n0, n1, n2};
        int next = 0;
        for (int r = 0; r < 3; ++r) {
            if (r >= rank)
                ext_[r] = 0;
            else if (r < dims::dynamic)
                ext_[r] = given[next++];
            else
                ext_[r] = dims::ext(r - dims::dynamic);
        }
    }
    void check_static() const {}
    void allocate(const ViewAllocProp& prop, std::size_t n0, std::size_t n1, std::size_t n2) {
        set_extents(n0, n1, n2);
        label_ = prop.label;
        void* p = impl::allocate(sizeof(value_type) * size(), true);  // zeroed either way: reproducible runs
        owner_ = std::shared_ptr<void>(p, [](void* q) { std::free(q); });
        data_ = static_cast<value_type*>(p);
        (void)prop.initialize;
    }
    template <class D2, class... P2>
    friend class View;

    value_type* data_ = nullptr;
    std::shared_ptr<void> owner_;
    std::size_t ext_[3] = {0, 0, 0};
    std::string label_;
};

// ---- subviews: fixed leading indices, then ALL
template <class DT, class... P>
View<typename View<DT, P...>::value_type, P...> subview(const View<DT, P...>& v, std::size_t i) {
    static_assert(View<DT, P...>::rank == 1, "subview(v, i): rank-1 view");
    using R = View<typename View<DT, P...>::value_type, P...>;
    return R(v.data() + i);
}
template <class DT, class... P>
View<typename View<DT, P...>::value_type*, P...> subview(const View<DT, P...>& v, std::size_t i, ALL_t) {
    static_assert(View<DT, P...>::rank == 2, "subview(v, i, ALL): rank-2 view");
    using R = View<typename View<DT, P...>::value_type*, P...>;
    return R(v.data() + i * v.extent(1), v.extent(1));
}

// ---- mirrors and copies (one memory space: a mirror is the view itself)
template <class DT, class... P>
View<DT, P...> create_mirror_view(const View<DT, P...>& v) {
    return v;
}
template <class S, class DT, class... P>
View<DT, P...> create_mirror_view(const S&, const View<DT, P...>& v) {
    return v;
}
template <class S, class DT, class... P>
View<DT, P...> create_mirror_view_and_copy(const S&, const View<DT, P...>& v) {
    return v;
}
template <class DT, class... P>
View<typename View<DT, P...>::non_const_value_type*, HostSpace> create_mirror(const View<DT, P...>& v) {
    View<typename View<DT, P...>::non_const_value_type*, HostSpace> out("mirror", v.size());
    return out;
}

template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
    if (dst.size() != src.size()) std::abort();
    if (dst.data() != src.data() && dst.size() > 0)
        std::memmove(static_cast<void*>(dst.data()), static_cast<const void*>(src.data()), sizeof(*dst.data()) * dst.size());
}
template <class D1, class... P1, class T, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
void deep_copy(const View<D1, P1...>& dst, const T& value) {
    const std::size_t n = dst.size();
    auto* p = dst.data();
    for (std::size_t i = 0; i < n; ++i) p[i] = static_cast<typename View<D1, P1...>::non_const_value_type>(value);
}
template <class T, class D2, class... P2, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
void deep_copy(T& value, const View<D2, P2...>& src) {
    static_assert(View<D2, P2...>::rank == 0, "deep_copy(scalar, view): rank-0 view");
    value = *src.data();
}
template <class E, class A, class B, std::enable_if_t<std::is_same_v<typename E::execution_space, E>, int> = 0>
void deep_copy(const E&, A& dst, const B& src) {
    deep_copy(dst, src);
}
template <class E, class A, class B, std::enable_if_t<std::is_same_v<typename E::execution_space, E>, int> = 0>
void deep_copy(const E&, const A& dst, const B& src) {
    deep_copy(dst, src);
}

// ---- small fixed arrays
template <class T, std::size_t N>
struct Array {
    T m_data[N > 0 ? N : 1];
    KOKKOS_INLINE_FUNCTION T& operator[](std::size_t i) { return m_data[i]; }
    KOKKOS_INLINE_FUNCTION const T& operator[](std::size_t i) const { return m_data[i]; }
    static constexpr std::size_t size() { return N; }
    T* data() { return m_data; }
    const T* data() const { return m_data; }
};

// ---- math
using std::abs;
using std::cbrt;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::round;
using std::sqrt;
using std::isfinite;
using std::isnan;
template <class T>
KOKKOS_INLINE_FUNCTION constexpr const T& min(const T& a, const T& b) {
    return b < a ? b : a;
}
template <class T>
KOKKOS_INLINE_FUNCTION constexpr const T& max(const T& a, const T& b) {
    return a < b ? b : a;
}
template <class T>
KOKKOS_INLINE_FUNCTION constexpr const T& clamp(const T& v, const T& lo, const T& hi) {
    return v < lo ? lo : hi < v ? hi : v;
}
template <class To, class From>
KOKKOS_INLINE_FUNCTION To bit_cast(const From& from) {
    static_assert(sizeof(To) == sizeof(From), "bit_cast: equal sizes");
    To to;
    std::memcpy(&to, &from, sizeof(To));
    return to;
}
namespace Experimental {
template <class T>
inline constexpr T infinity_v = std::numeric_limits<T>::infinity();
template <class T>
inline constexpr T finite_max_v = std::numeric_limits<T>::max();
template <class T>
inline constexpr T finite_min_v = std::numeric_limits<T>::lowest();
}  // namespace Experimental

// ---- timing
class Timer {
public:
    Timer() { reset(); }
    void reset() { start_ = std::chrono::steady_clock::now(); }
    double seconds() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count(); }

private:
    std::chrono::steady_clock::time_point start_;
};

// ---- policies
template <class E = DefaultExecutionSpace>
struct RangePolicy {
    using execution_space = E;
    long long begin_ = 0, end_ = 0;
    RangePolicy(long long b, long long e) : begin_(b), end_(e) {}
    RangePolicy(const E&, long long b, long long e) : begin_(b), end_(e) {}
    long long begin() const { return begin_; }
    long long end() const { return end_; }
};
struct AUTO_t {};
inline constexpr AUTO_t AUTO{};
template <class E = DefaultExecutionSpace>
struct TeamPolicy {
    using execution_space = E;
    int league = 0, team = 1, vector = 1;
    struct member_type {
        int league_rank_ = 0, team_rank_ = 0, team_size_ = 1, league_size_ = 0;
        int league_rank() const { return league_rank_; }
        int team_rank() const { return team_rank_; }
        int team_size() const { return team_size_; }
        int league_size() const { return league_size_; }
        void team_barrier() const {}
    };
    TeamPolicy(const E&, int l, int t, int v = 1) : league(l), team(t), vector(v) {}
    TeamPolicy(const E&, int l, AUTO_t) : league(l), team(1) {}
    TeamPolicy(int l, int t, int v = 1) : league(l), team(t), vector(v) {}
};
// Nested ranges run by the one thread of a serial team member.
template <class M>
struct NestedRange {
    long long begin, end;
};
template <class M>
NestedRange<M> ThreadVectorRange(const M&, long long n) {
    return {0, n};
}
template <class M>
NestedRange<M> ThreadVectorRange(const M&, long long b, long long e) {
    return {b, e};
}
template <class M>
NestedRange<M> TeamThreadRange(const M&, long long n) {
    return {0, n};
}
template <class M>
NestedRange<M> TeamThreadRange(const M&, long long b, long long e) {
    return {b, e};
}
template <class M>
NestedRange<M> TeamVectorRange(const M&, long long b, long long e) {
    return {b, e};
}
template <class M>
struct PerThreadTag {
    const M& m;
};
template <class M>
struct PerTeamTag {
    const M& m;
};
template <class M>
PerThreadTag<M> PerThread(const M& m) {
    return {m};
}
template <class M>
PerTeamTag<M> PerTeam(const M& m) {
    return {m};
}
template <class Tag, class F>
void single(const Tag&, const F& f) {
    f();
}

// ---- reducers: init / join / reference, as Kokkos's
template <class T>
struct Min {
    using reducer = Min;
    using value_type = T;
    T* value;
    explicit Min(T& v) : value(&v) {}
    void join(T& dest, const T& src) const {
        if (src < dest) dest = src;
    }
    void init(T& v) const { v = std::numeric_limits<T>::has_infinity ? std::numeric_limits<T>::infinity() : std::numeric_limits<T>::max(); }
    T& reference() const { return *value; }
};
template <class T>
struct Max {
    using reducer = Max;
    using value_type = T;
    T* value;
    explicit Max(T& v) : value(&v) {}
    void join(T& dest, const T& src) const {
        if (dest < src) dest = src;
    }
    void init(T& v) const { v = std::numeric_limits<T>::has_infinity ? -std::numeric_limits<T>::infinity() : std::numeric_limits<T>::lowest(); }
    T& reference() const { return *value; }
};
template <class T>
struct Sum {
    using reducer = Sum;
    using value_type = T;
    T* value;
    explicit Sum(T& v) : value(&v) {}
    void join(T& dest, const T& src) const { dest += src; }
    void init(T& v) const { v = T(0); }
    T& reference() const { return *value; }
};
template <class T, class I>
struct ValLocScalar {
    T val;
    I loc;
};
template <class T, class I>
struct MinLoc {
    using reducer = MinLoc;
    using value_type = ValLocScalar<T, I>;
    value_type* value;
    explicit MinLoc(value_type& v) : value(&v) {}
    void join(value_type& dest, const value_type& src) const {
        if (src.val < dest.val || (src.val == dest.val && src.loc < dest.loc)) dest = src;
    }
    void init(value_type& v) const {
        v.val = std::numeric_limits<T>::has_infinity ? std::numeric_limits<T>::infinity() : std::numeric_limits<T>::max();
        v.loc = std::numeric_limits<I>::max();
    }
    value_type& reference() const { return *value; }
};

namespace impl {
template <class R, class = void>
struct IsReducer : std::false_type {};
template <class R>
struct IsReducer<R, std::void_t<typename R::reducer>> : std::true_type {};
template <class R, class = void>
struct IsView : std::false_type {};
template <class R>
struct IsView<R, std::void_t<typename R::array_layout, typename R::data_type>> : std::true_type {};

// The result argument of parallel_reduce: a reducer, a rank-0 view (summed into), or a scalar (summed into).
template <class R>
struct Result {
    using reducer = Sum<R>;
};
template <class R, class Fn>
void reduce_range(long long b, long long e, bool parallel, const Fn& fn, const R& reducer) {
    using T = typename R::value_type;
    T total;
    reducer.init(total);
#ifdef _OPENMP
    if (parallel && e - b > 1) {
        const int threads = omp_get_max_threads();
        std::unique_ptr<T[]> part(new T[threads]);
#pragma omp parallel num_threads(threads)
        {
            const int t = omp_get_thread_num();
            T local;
            reducer.init(local);
#pragma omp for schedule(static)
            for (long long i = b; i < e; ++i) fn(i, local);
            part[t] = local;
        }
        for (int t = 0; t < threads; ++t) reducer.join(total, part[t]);
        reducer.reference() = total;
        return;
    }
#endif
    (void)parallel;
    for (long long i = b; i < e; ++i) fn(i, total);
    reducer.reference() = total;
}
}  // namespace impl

// ---- parallel_for
template <class E, class F>
void parallel_for(const RangePolicy<E>& policy, const F& f) {
#ifdef _OPENMP
    if (E::parallel) {
#pragma omp parallel for schedule(static)
        for (long long i = policy.begin(); i < policy.end(); ++i) f(static_cast<int>(i));
        return;
    }
#endif
    for (long long i = policy.begin(); i < policy.end(); ++i) f(static_cast<int>(i));
}
template <class E, class F>
void parallel_for(const std::string&, const RangePolicy<E>& policy, const F& f) {
    parallel_for(policy, f);
}
template <class F>
void parallel_for(const std::string& label, long long n, const F& f) {
    parallel_for(label, RangePolicy<DefaultExecutionSpace>(0, n), f);
}
template <class E, class F>
void parallel_for(const std::string&, const TeamPolicy<E>& policy, const F& f) {
    for (int l = 0; l < policy.league; ++l)
        for (int t = 0; t < policy.team; ++t) {
            typename TeamPolicy<E>::member_type m;
            m.league_rank_ = l;
            m.team_rank_ = t;
            m.team_size_ = policy.team;
            m.league_size_ = policy.league;
            f(m);
        }
}
template <class M, class F>
void parallel_for(const NestedRange<M>& r, const F& f) {
    for (long long i = r.begin; i < r.end; ++i) f(static_cast<int>(i));
}

// ---- parallel_reduce
template <class E, class F, class R>
void parallel_reduce(const std::string&, const RangePolicy<E>& policy, const F& f, const R& result) {
    auto call = [&](long long i, auto& value) { f(static_cast<int>(i), value); };
    if constexpr (impl::IsReducer<R>::value) {
        impl::reduce_range(policy.begin(), policy.end(), E::parallel, call, result);
    } else if constexpr (impl::IsView<R>::value) {
        using T = typename R::non_const_value_type;
        T total = 0;
        impl::reduce_range(policy.begin(), policy.end(), E::parallel, call, Sum<T>(total));
        *result.data() = total;
    } else {
        static_assert(impl::IsView<R>::value || impl::IsReducer<R>::value, "parallel_reduce: a reducer or a view (scalars: by reference)");
    }
}
template <class E, class F, class T, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
void parallel_reduce(const std::string&, const RangePolicy<E>& policy, const F& f, T& result) {
    auto call = [&](long long i, auto& value) { f(static_cast<int>(i), value); };
    T total = 0;
    impl::reduce_range(policy.begin(), policy.end(), E::parallel, call, Sum<T>(total));
    result = total;
}
template <class M, class F, class R>
void parallel_reduce(const NestedRange<M>& r, const F& f, const R& reducer) {
    if constexpr (impl::IsReducer<R>::value) {
        typename R::value_type total;
        reducer.init(total);
        for (long long i = r.begin; i < r.end; ++i) f(static_cast<int>(i), total);
        reducer.reference() = total;
    } else {
        static_assert(impl::IsReducer<R>::value, "nested parallel_reduce: a reducer");
    }
}
template <class M, class F, class T, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
void parallel_reduce(const NestedRange<M>& r, const F& f, T& result) {
    T total = 0;
    for (long long i = r.begin; i < r.end; ++i) f(static_cast<int>(i), total);
    result = total;
}

// ---- lifetime (nothing to set up on the host)
inline void initialize(int = 0, char** = nullptr) {}
inline void finalize() {}
inline bool is_initialized() { return true; }
struct ScopeGuard {
    ScopeGuard(int = 0, char** = nullptr) {}
};

}  // namespace Kokkos
