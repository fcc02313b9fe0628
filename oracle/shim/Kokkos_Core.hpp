// Test-infrastructure shim: the subset of the Kokkos API that the GR-ray-tracer
// reference headers use, implemented on the host with OpenMP.  It exists only so
// that the reference's own, unmodified headers (src/geodesic_integrate,
// src/metrics, src/radiative_transfer, ...) compile here as a CPU oracle; real
// Kokkos is not installable offline.  Semantics follow the Kokkos host backend:
//   * View is a reference-counted handle to zero-initialised LayoutRight storage;
//   * create_mirror_view on host memory returns the same allocation;
//   * parallel_for / parallel_reduce use an OpenMP static schedule;
//   * math functions forward to <cmath> (glibc), so the arithmetic of the
//     reference's functors is exactly what g++ produces for them.
// Nothing in the product links this file.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>

#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_FUNCTION
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_LAMBDA [=]

namespace Kokkos {

struct HostSpace {};
struct DefaultExecutionSpace {};

namespace shim_detail {
template <class T> struct view_traits {
    using value_type = T;
    static constexpr int rank = 0;
};
template <class T> struct view_traits<T*> {
    using value_type = typename view_traits<T>::value_type;
    static constexpr int rank = view_traits<T>::rank + 1;
};

// Counters the oracle driver reads after a run: how many functor invocations
// found a live photon, and how many of those advanced its coordinate time
// (i.e. took an integration step).
struct Stats {
    std::uint64_t live_invocations = 0;
    std::uint64_t stepped_invocations = 0;
};
inline Stats& stats() {
    static Stats s;
    return s;
}
}  // namespace shim_detail

template <class DataType, class... Props>
class View {
public:
    using value_type = typename shim_detail::view_traits<DataType>::value_type;
    using non_const_value_type = std::remove_const_t<value_type>;
    static constexpr int Rank = shim_detail::view_traits<DataType>::rank;

    View() = default;

    template <class... Extents,
              class = std::enable_if_t<(std::is_integral_v<Extents> && ...)>>
    explicit View(const std::string& /*label*/, Extents... extents) {
        static_assert(sizeof...(Extents) == Rank, "extent count must match view rank");
        std::size_t values[] = {static_cast<std::size_t>(extents)...};
        std::size_t total = 1;
        for (int r = 0; r < Rank; ++r) {
            extent_[r] = values[r];
            total *= values[r];
        }
        size_ = total;
        storage_ = std::shared_ptr<non_const_value_type[]>(new non_const_value_type[total > 0 ? total : 1]());
    }

    // Views differing only in memory-space tags share storage (host backend).
    template <class... OtherProps>
    View(const View<DataType, OtherProps...>& other)
        : storage_(other.storage_), size_(other.size_) {
        for (int r = 0; r < 8; ++r) extent_[r] = other.extent_[r];
    }
    template <class... OtherProps>
    View& operator=(const View<DataType, OtherProps...>& other) {
        storage_ = other.storage_;
        size_ = other.size_;
        for (int r = 0; r < 8; ++r) extent_[r] = other.extent_[r];
        return *this;
    }

    std::size_t extent(int r) const { return r < Rank ? extent_[r] : 1; }
    std::size_t size() const { return size_; }
    non_const_value_type* data() const { return storage_ ? storage_.get() : nullptr; }

    template <class... Indices>
    non_const_value_type& operator()(Indices... indices) const {
        static_assert(sizeof...(Indices) == Rank, "index count must match view rank");
        std::size_t idx[] = {static_cast<std::size_t>(indices)...};
        std::size_t flat = 0;
        for (int r = 0; r < Rank; ++r) flat = flat * extent_[r] + idx[r];
        return storage_.get()[flat];
    }

    std::shared_ptr<non_const_value_type[]> storage_;
    std::size_t size_ = 0;
    std::size_t extent_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

template <class D, class... P>
View<D, P...> create_mirror_view(const View<D, P...>& v) { return v; }

template <class D, class... P>
View<D, HostSpace> create_mirror_view_and_copy(HostSpace, const View<D, P...>& v) { return v; }

template <class D, class... P, class... Q>
void deep_copy(const View<D, P...>& dst, const View<D, Q...>& src) {
    if (dst.data() == src.data()) return;
    std::memcpy(static_cast<void*>(dst.data()), static_cast<const void*>(src.data()),
                sizeof(typename View<D, P...>::non_const_value_type) * dst.size());
}

template <class D, class... P, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
void deep_copy(const View<D, P...>& dst, const S& value) {
    using T = typename View<D, P...>::non_const_value_type;
    for (std::size_t i = 0; i < dst.size(); ++i) dst.data()[i] = static_cast<T>(value);
}

template <class... Args>
struct RangePolicy {
    std::int64_t begin = 0;
    std::int64_t end = 0;
    RangePolicy(std::int64_t b, std::int64_t e) : begin(b), end(e) {}
};

namespace shim_detail {
template <class F>
void run_range(std::int64_t begin, std::int64_t end, const F& f) {
    if constexpr (requires { f.photon_terminate; f.photon_x0; }) {
        // The reference's per-photon step functor: count live photons and
        // integration steps so throughput can be reported in RK steps.
        std::uint64_t live = 0, stepped = 0;
#pragma omp parallel for schedule(static) reduction(+ : live, stepped)
        for (std::int64_t i = begin; i < end; ++i) {
            const bool was_live = !f.photon_terminate(i);
            const double t_before = f.photon_x0(i);
            f(static_cast<int>(i));
            if (was_live) {
                ++live;
                if (f.photon_x0(i) != t_before) ++stepped;
            }
        }
        stats().live_invocations += live;
        stats().stepped_invocations += stepped;
    } else {
#pragma omp parallel for schedule(static)
        for (std::int64_t i = begin; i < end; ++i) f(static_cast<int>(i));
    }
}
}  // namespace shim_detail

template <class... A, class F>
void parallel_for(const std::string&, const RangePolicy<A...>& p, const F& f) {
    shim_detail::run_range(p.begin, p.end, f);
}
template <class F>
void parallel_for(const std::string&, std::int64_t n, const F& f) {
    shim_detail::run_range(0, n, f);
}
template <class... A, class F>
void parallel_for(const RangePolicy<A...>& p, const F& f) {
    shim_detail::run_range(p.begin, p.end, f);
}

template <class... A, class F, class T>
void parallel_reduce(const std::string&, const RangePolicy<A...>& p, const F& f, T& result) {
    T total{};
#pragma omp parallel
    {
        T local{};
#pragma omp for schedule(static)
        for (std::int64_t i = p.begin; i < p.end; ++i) f(static_cast<int>(i), local);
#pragma omp critical
        total += local;
    }
    result = total;
}

template <class... A, class F>
void parallel_scan(const std::string&, const RangePolicy<A...>& p, const F& f) {
    int partial = 0;
    for (std::int64_t i = p.begin; i < p.end; ++i) f(static_cast<int>(i), partial, false);
    partial = 0;
    for (std::int64_t i = p.begin; i < p.end; ++i) f(static_cast<int>(i), partial, true);
}

template <class T>
T atomic_fetch_add(T* target, T value) {
    return __atomic_fetch_add(target, value, __ATOMIC_SEQ_CST);
}

inline void initialize() {}
inline void initialize(int&, char**&) {}
inline void finalize() {}
inline void fence() {}

using std::abs;
using std::acos;
using std::atan2;
using std::cos;
using std::exp;
using std::fmax;
using std::fmin;
using std::fmod;
using std::isfinite;
using std::log;
using std::log10;
using std::pow;
using std::sin;
using std::sqrt;

}  // namespace Kokkos
