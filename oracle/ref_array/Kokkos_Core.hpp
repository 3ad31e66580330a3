// Oracle-only host stand-in for <Kokkos_Core.hpp> (test infrastructure): the
// per-cell pieces of oracle/ref_shim, the views of hcl_kokkos_view.hpp, and
// parallel dispatch on the host -- RangePolicy and 2-/3-D MDRangePolicy
// (Iterate::Left: index 0 innermost) as OpenMP loops over the outermost
// index, parallel_reduce with Sum / Min / Max reducers or plain sums, and a
// sequential parallel_scan.  It exists so that the reference's own array
// kernels run on the host cores as its Kokkos-OpenMP build would run them.
#pragma once

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "Kokkos_Array.hpp"
#include "Kokkos_Assert.hpp"
#include "Kokkos_Macros.hpp"
#include "Kokkos_MathematicalConstants.hpp"
#include "Kokkos_MathematicalFunctions.hpp"
#include "Kokkos_Printf.hpp"
#include "hcl_kokkos_view.hpp"

#ifndef KOKKOS_LAMBDA
#define KOKKOS_LAMBDA [=]
#endif
#ifndef KOKKOS_CLASS_LAMBDA
#define KOKKOS_CLASS_LAMBDA [=, *this]
#endif

namespace Kokkos {

using std::clamp;
using std::max;
using std::min;

inline void initialize(int&, char**) {}
inline void finalize() {}
inline void fence(const std::string& = std::string()) {}

namespace Profiling {
inline void pushRegion(const std::string&) {}
inline void popRegion() {}
class ScopedRegion {
public:
    explicit ScopedRegion(const std::string&) {}
};
} // namespace Profiling

template <class T>
struct IndexType {
};
enum class Iterate { Default, Left, Right };
template <unsigned N, Iterate Outer = Iterate::Default, Iterate Inner = Iterate::Default>
struct Rank {
    static constexpr unsigned rank = N;
};

namespace hcl_impl {
template <class... P>
struct mdrank {
    static constexpr unsigned value = 0;
};
template <class P0, class... P>
struct mdrank<P0, P...> {
    static constexpr unsigned value = mdrank<P...>::value;
};
template <unsigned N, Iterate O, Iterate I, class... P>
struct mdrank<Rank<N, O, I>, P...> {
    static constexpr unsigned value = N;
};
} // namespace hcl_impl

template <class... P>
struct RangePolicy {
    long begin, end;
    RangePolicy(long b, long e) : begin(b), end(e) {}
};

template <class... P>
struct MDRangePolicy {
    static constexpr unsigned rank = hcl_impl::mdrank<P...>::value;
    long lo[3] = {0, 0, 0};
    long hi[3] = {1, 1, 1};
    template <class A, class B>
    MDRangePolicy(const A& b, const B& e)
    {
        for (unsigned r = 0; r < rank; ++r) {
            lo[r] = (long)b[r];
            hi[r] = (long)e[r];
        }
    }
    MDRangePolicy(std::initializer_list<long> b, std::initializer_list<long> e)
    {
        unsigned r = 0;
        for (long x : b) {
            lo[r++] = x;
        }
        r = 0;
        for (long x : e) {
            hi[r++] = x;
        }
    }
};

// reducers: the result goes to a scalar or to a rank-0 view
template <class T>
struct Sum {
    T* ptr;
    explicit Sum(T& r) : ptr(&r) {}
    template <class DT, class... P>
    explicit Sum(const View<DT, P...>& v) : ptr(v.data())
    {
    }
    static T init() { return T(0); }
    static void join(T& dst, const T& src) { dst += src; }
};
template <class T>
struct Min {
    T* ptr;
    explicit Min(T& r) : ptr(&r) {}
    template <class DT, class... P>
    explicit Min(const View<DT, P...>& v) : ptr(v.data())
    {
    }
    static T init() { return std::numeric_limits<T>::max(); }
    static void join(T& dst, const T& src)
    {
        if (src < dst) {
            dst = src;
        }
    }
};
template <class T>
struct Max {
    T* ptr;
    explicit Max(T& r) : ptr(&r) {}
    template <class DT, class... P>
    explicit Max(const View<DT, P...>& v) : ptr(v.data())
    {
    }
    static T init() { return std::numeric_limits<T>::lowest(); }
    static void join(T& dst, const T& src)
    {
        if (src > dst) {
            dst = src;
        }
    }
};
template <class DT, class... P>
Sum(const View<DT, P...>&) -> Sum<typename View<DT, P...>::non_const_value_type>;
template <class DT, class... P>
Min(const View<DT, P...>&) -> Min<typename View<DT, P...>::non_const_value_type>;
template <class DT, class... P>
Max(const View<DT, P...>&) -> Max<typename View<DT, P...>::non_const_value_type>;

namespace hcl_impl {

// a reduction target: a reducer or a plain scalar (summed)
template <class R>
struct red {
    using value_type = std::remove_reference_t<R>;
    static value_type init() { return value_type(0); }
    static void join(value_type& d, const value_type& s) { d += s; }
    static value_type& target(R& r) { return r; }
};
template <class T>
struct red<Sum<T>> {
    using value_type = T;
    static T init() { return Sum<T>::init(); }
    static void join(T& d, const T& s) { Sum<T>::join(d, s); }
    static T& target(Sum<T>& r) { return *r.ptr; }
};
template <class T>
struct red<Min<T>> {
    using value_type = T;
    static T init() { return Min<T>::init(); }
    static void join(T& d, const T& s) { Min<T>::join(d, s); }
    static T& target(Min<T>& r) { return *r.ptr; }
};
template <class T>
struct red<Max<T>> {
    using value_type = T;
    static T init() { return Max<T>::init(); }
    static void join(T& d, const T& s) { Max<T>::join(d, s); }
    static T& target(Max<T>& r) { return *r.ptr; }
};

} // namespace hcl_impl

// ---- parallel_for -----------------------------------------------------------
template <class... P, class F>
void parallel_for(const std::string&, const RangePolicy<P...>& p, const F& f)
{
#pragma omp parallel for schedule(static)
    for (long i = p.begin; i < p.end; ++i) {
        f((int)i);
    }
}

template <class F>
void parallel_for(const std::string& label, long n, const F& f)
{
    parallel_for(label, RangePolicy<>(0, n), f);
}

template <class... P, class F>
void parallel_for(const std::string&, const MDRangePolicy<P...>& p, const F& f)
{
    constexpr unsigned R = MDRangePolicy<P...>::rank;
    if constexpr (R == 3) {
#pragma omp parallel for collapse(2) schedule(static)
        for (long k = p.lo[2]; k < p.hi[2]; ++k) {
            for (long j = p.lo[1]; j < p.hi[1]; ++j) {
                for (long i = p.lo[0]; i < p.hi[0]; ++i) {
                    f((int)i, (int)j, (int)k);
                }
            }
        }
    } else {
        static_assert(R == 2, "MDRangePolicy of rank 2 or 3");
#pragma omp parallel for schedule(static)
        for (long j = p.lo[1]; j < p.hi[1]; ++j) {
            for (long i = p.lo[0]; i < p.hi[0]; ++i) {
                f((int)i, (int)j);
            }
        }
    }
}

// ---- parallel_reduce ----------------------------------------------------------
// Each thread reduces its static share of the outermost index into its own
// accumulators; the shares are joined in thread order.
template <class... P, class F, class... Rs>
void parallel_reduce(const std::string&, const RangePolicy<P...>& p, const F& f, Rs&&... rs)
{
    using Tup = std::tuple<typename hcl_impl::red<std::remove_reference_t<Rs>>::value_type...>;
    const int nt = omp_get_max_threads();
    std::vector<Tup> part((size_t)nt, Tup{hcl_impl::red<std::remove_reference_t<Rs>>::init()...});
#pragma omp parallel num_threads(nt)
    {
        Tup mine = part[(size_t)omp_get_thread_num()];
#pragma omp for schedule(static)
        for (long i = p.begin; i < p.end; ++i) {
            std::apply([&](auto&... a) { f((int)i, a...); }, mine);
        }
        part[(size_t)omp_get_thread_num()] = mine;
    }
    Tup tot{hcl_impl::red<std::remove_reference_t<Rs>>::init()...};
    for (const Tup& t : part) {
        [&]<std::size_t... I>(std::index_sequence<I...>) {
            (hcl_impl::red<std::remove_reference_t<Rs>>::join(std::get<I>(tot), std::get<I>(t)), ...);
        }(std::index_sequence_for<Rs...>{});
    }
    [&]<std::size_t... I>(std::index_sequence<I...>) {
        ((hcl_impl::red<std::remove_reference_t<Rs>>::target(rs) = std::get<I>(tot)), ...);
    }(std::index_sequence_for<Rs...>{});
}

template <class... P, class F, class... Rs>
void parallel_reduce(const std::string&, const MDRangePolicy<P...>& p, const F& f, Rs&&... rs)
{
    constexpr unsigned R = MDRangePolicy<P...>::rank;
    using Tup = std::tuple<typename hcl_impl::red<std::remove_reference_t<Rs>>::value_type...>;
    const int nt = omp_get_max_threads();
    std::vector<Tup> part((size_t)nt, Tup{hcl_impl::red<std::remove_reference_t<Rs>>::init()...});
#pragma omp parallel num_threads(nt)
    {
        Tup mine = part[(size_t)omp_get_thread_num()];
        if constexpr (R == 3) {
#pragma omp for collapse(2) schedule(static)
            for (long k = p.lo[2]; k < p.hi[2]; ++k) {
                for (long j = p.lo[1]; j < p.hi[1]; ++j) {
                    for (long i = p.lo[0]; i < p.hi[0]; ++i) {
                        std::apply([&](auto&... a) { f((int)i, (int)j, (int)k, a...); }, mine);
                    }
                }
            }
        } else {
#pragma omp for schedule(static)
            for (long j = p.lo[1]; j < p.hi[1]; ++j) {
                for (long i = p.lo[0]; i < p.hi[0]; ++i) {
                    std::apply([&](auto&... a) { f((int)i, (int)j, a...); }, mine);
                }
            }
        }
        part[(size_t)omp_get_thread_num()] = mine;
    }
    Tup tot{hcl_impl::red<std::remove_reference_t<Rs>>::init()...};
    for (const Tup& t : part) {
        [&]<std::size_t... I>(std::index_sequence<I...>) {
            (hcl_impl::red<std::remove_reference_t<Rs>>::join(std::get<I>(tot), std::get<I>(t)), ...);
        }(std::index_sequence_for<Rs...>{});
    }
    [&]<std::size_t... I>(std::index_sequence<I...>) {
        ((hcl_impl::red<std::remove_reference_t<Rs>>::target(rs) = std::get<I>(tot)), ...);
    }(std::index_sequence_for<Rs...>{});
}

// ---- parallel_scan (sequential) ---------------------------------------------------
template <class... P, class F>
void parallel_scan(const std::string&, const RangePolicy<P...>& p, const F& f)
{
    double partial = 0;
    for (long i = p.begin; i < p.end; ++i) {
        f((int)i, partial, true);
    }
}

// ---- deep_copy --------------------------------------------------------------------
template <class DT, class... P, class DT2, class... P2>
void deep_copy(const View<DT, P...>& dst, const View<DT2, P2...>& src)
{
    static_assert(View<DT, P...>::Rank == View<DT2, P2...>::Rank, "deep_copy between views of one rank");
    constexpr int R = View<DT, P...>::Rank;
    const auto& e = dst.hcl_extents();
    const auto& sd = dst.hcl_strides();
    const auto& ss = src.hcl_strides();
    for (int r = 0; r < R; ++r) {
        assert(e[r] == src.hcl_extents()[r]);
    }
    long n = 1;
    for (int r = 0; r < R; ++r) {
        n *= e[r];
    }
    if (dst.span_is_contiguous() && src.span_is_contiguous()) {
        // both column-major and dense: one flat copy
        auto* d = dst.data();
        const auto* q = src.data();
#pragma omp parallel for schedule(static)
        for (long lin = 0; lin < n; ++lin) {
            d[lin] = q[lin];
        }
        return;
    }
#pragma omp parallel for schedule(static)
    for (long lin = 0; lin < n; ++lin) {
        long rem = lin, od = 0, os = 0;
        for (int r = 0; r < R; ++r) {
            const long ir = rem % e[r];
            rem /= e[r];
            od += ir * sd[r];
            os += ir * ss[r];
        }
        dst.data()[od] = src.data()[os];
    }
}

template <class DT, class... P, class T, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
void deep_copy(const View<DT, P...>& dst, const T& value)
{
    constexpr int R = View<DT, P...>::Rank;
    const auto& e = dst.hcl_extents();
    const auto& sd = dst.hcl_strides();
    long n = 1;
    for (int r = 0; r < R; ++r) {
        n *= e[r];
    }
    for (long lin = 0; lin < n; ++lin) {
        long rem = lin, od = 0;
        for (int r = 0; r < R; ++r) {
            const long ir = rem % e[r];
            rem /= e[r];
            od += ir * sd[r];
        }
        dst.data()[od] = value;
    }
}

template <class Space, class V1, class V2>
void deep_copy(const Space&, const V1& dst, const V2& src)
{
    deep_copy(dst, src);
}

} // namespace Kokkos
