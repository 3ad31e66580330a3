// Oracle-only host stand-in for the part of Kokkos::View that the reference's
// array code uses (test infrastructure: it lets the reference's own
// hydro/, mesh/, boundary*, gravity/ and analysis/ sources compile and run on
// the host so that the C restatement in oracle/hcl_oracle.c can be checked
// against them; nothing of the product links it).
//
// A view is a pointer, up to 6 extents and 6 element strides.  Managed views
// own a zero-initialised allocation (shared between copies, like Kokkos'
// reference counting); unmanaged views wrap a caller's pointer.  LayoutLeft
// views get column-major strides (index 0 fastest); subviews keep the parent's
// strides, so any layout tag converts to any other of the same rank.
#pragma once

#include <array>
#include <cassert>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>

namespace Kokkos {

// layouts carry their extents (Kokkos' layout objects do), so that
// View(label, other.layout()) allocates a view of the same shape
struct LayoutLeft {
    std::size_t dimension[8] = {1, 1, 1, 1, 1, 1, 1, 1};
};
struct LayoutRight {
    std::size_t dimension[8] = {1, 1, 1, 1, 1, 1, 1, 1};
};
struct LayoutStride {
    std::size_t dimension[8] = {1, 1, 1, 1, 1, 1, 1, 1};
};

struct OpenMP;
struct HostSpace {
    using memory_space = HostSpace;
    using execution_space = OpenMP;
};
using SharedHostPinnedSpace = HostSpace;
struct OpenMP {
    using memory_space = HostSpace;
    using execution_space = OpenMP;
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

template <unsigned T = 0>
struct MemoryTraits {
};

struct ALL_t {
};
inline constexpr ALL_t ALL{};

template <class A, class B>
struct pair {
    A first;
    B second;
};
template <class A, class B>
constexpr pair<A, B> make_pair(A a, B b)
{
    return pair<A, B>{a, b};
}

namespace hcl_impl {

// rank and value type of a Kokkos data type such as double const***
template <class T>
struct data_type_info {
    using value_type = T;
    static constexpr int rank = 0;
    template <class U>
    using rebind = U;
};
template <class T>
struct data_type_info<T*> {
    using value_type = typename data_type_info<T>::value_type;
    static constexpr int rank = data_type_info<T>::rank + 1;
    template <class U>
    using rebind = typename data_type_info<T>::template rebind<U>*;
};

// the data type of rank R over value type V (V*** for R = 3)
template <class V, int R>
struct make_data_type {
    using type = typename make_data_type<V, R - 1>::type*;
};
template <class V>
struct make_data_type<V, 0> {
    using type = V;
};

template <class... P>
struct first_layout {
    using type = LayoutRight; // Kokkos' default on host spaces
};
template <class P0, class... P>
struct first_layout<P0, P...> {
    using type = std::conditional_t<std::is_same_v<P0, LayoutLeft> || std::is_same_v<P0, LayoutRight> ||
                                        std::is_same_v<P0, LayoutStride>,
                                    P0, typename first_layout<P...>::type>;
};

} // namespace hcl_impl

template <class DataType, class... Props>
struct ViewTraits {
    using data_type = DataType;
    using value_type = typename hcl_impl::data_type_info<DataType>::value_type;
    using non_const_value_type = std::remove_const_t<value_type>;
    static constexpr int rank_ = hcl_impl::data_type_info<DataType>::rank;
    using const_data_type = typename hcl_impl::make_data_type<const non_const_value_type, rank_>::type;
    using non_const_data_type = typename hcl_impl::make_data_type<non_const_value_type, rank_>::type;
    using array_layout = typename hcl_impl::first_layout<Props...>::type;
    using memory_space = HostSpace;
    using execution_space = OpenMP;
    using memory_traits = MemoryTraits<>;
    struct host_mirror_space {
        using memory_space = HostSpace;
    };
    struct dimension {
        static constexpr unsigned rank = rank_;
        static constexpr unsigned rank_dynamic = rank_;
    };
};

template <class DataType, class... Props>
class View {
public:
    using traits = ViewTraits<DataType, Props...>;
    using data_type = DataType;
    using value_type = typename traits::value_type;
    using non_const_value_type = typename traits::non_const_value_type;
    using const_data_type = typename traits::const_data_type;
    using non_const_data_type = typename traits::non_const_data_type;
    using array_layout = typename traits::array_layout;
    using memory_space = HostSpace;
    using execution_space = OpenMP;
    using device_type = OpenMP;
    using pointer_type = value_type*;
    using reference_type = value_type&;
    using HostMirror = View<non_const_data_type, array_layout, HostSpace>;
    static constexpr int Rank = traits::rank_;
    static constexpr unsigned rank = traits::rank_;
    static constexpr unsigned rank_dynamic = traits::rank_;

    View() = default;

    // managed, zero-initialised: View("label", n0, ..., n_{rank-1})
    template <class... I, std::enable_if_t<(sizeof...(I) == Rank) && (std::is_integral_v<I> && ...), int> = 0>
    explicit View(const std::string& label, I... n) : m_label(label)
    {
        set_left_extents({static_cast<long>(n)...});
        const long count = span_count();
        m_alloc = std::shared_ptr<non_const_value_type[]>(new non_const_value_type[count > 0 ? count : 1]());
        m_ptr = m_alloc.get();
    }

    // managed view with the extents of a layout object
    View(const std::string& label, const LayoutLeft& l) : m_label(label)
    {
        std::array<long, 6> n{};
        for (int r = 0; r < 6; ++r) {
            n[r] = (long)l.dimension[r];
        }
        set_left_extents_n(n.data());
        const long count = span_count();
        m_alloc = std::shared_ptr<non_const_value_type[]>(new non_const_value_type[count > 0 ? count : 1]());
        m_ptr = m_alloc.get();
    }

    // unmanaged view of a caller's LayoutLeft array
    template <class... I, std::enable_if_t<(sizeof...(I) == Rank) && (std::is_integral_v<I> && ...), int> = 0>
    View(value_type* ptr, I... n) : m_ptr(ptr)
    {
        set_left_extents({static_cast<long>(n)...});
    }

    // conversion between layout tags and to const value types
    template <class DT2, class... P2,
              std::enable_if_t<(View<DT2, P2...>::Rank == Rank) &&
                                   std::is_convertible_v<typename View<DT2, P2...>::value_type*, value_type*>,
                               int> = 0>
    View(const View<DT2, P2...>& o)
        : m_alloc(o.m_alloc), m_ptr(o.m_ptr), m_ext(o.m_ext), m_str(o.m_str), m_label(o.m_label)
    {
    }

    template <class... I>
    reference_type operator()(I... i) const noexcept
    {
        static_assert(sizeof...(I) == Rank, "index count must equal the view's rank");
        return m_ptr[offset(std::index_sequence_for<I...>{}, i...)];
    }

    std::size_t extent(std::size_t r) const noexcept { return r < (std::size_t)Rank ? (std::size_t)m_ext[r] : 1; }
    int extent_int(std::size_t r) const noexcept { return (int)extent(r); }
    std::size_t stride(std::size_t r) const noexcept { return (std::size_t)m_str[r]; }
    pointer_type data() const noexcept { return m_ptr; }
    std::size_t size() const noexcept
    {
        std::size_t s = 1;
        for (int r = 0; r < Rank; ++r) {
            s *= (std::size_t)m_ext[r];
        }
        return s;
    }
    std::size_t span() const noexcept { return (std::size_t)span_count(); }
    bool span_is_contiguous() const noexcept
    {
        long expect = 1;
        for (int r = 0; r < Rank; ++r) {
            if (m_ext[r] > 1 && m_str[r] != expect) {
                return false;
            }
            expect *= m_ext[r];
        }
        return true;
    }
    std::string label() const { return m_label; }
    bool is_allocated() const noexcept { return m_ptr != nullptr; }
    int use_count() const noexcept { return (int)m_alloc.use_count(); }
    LayoutLeft layout() const noexcept
    {
        LayoutLeft l{};
        for (int r = 0; r < 8; ++r) {
            l.dimension[r] = r < Rank ? (std::size_t)m_ext[r] : 1;
        }
        return l;
    }

    // internal: build a view from explicit extents and strides (subviews)
    static View from_parts(const std::shared_ptr<non_const_value_type[]>& alloc, value_type* ptr,
                           const std::array<long, 6>& ext, const std::array<long, 6>& str, const std::string& label)
    {
        View v;
        v.m_alloc = alloc;
        v.m_ptr = ptr;
        v.m_ext = ext;
        v.m_str = str;
        v.m_label = label;
        return v;
    }

    const std::shared_ptr<non_const_value_type[]>& hcl_alloc() const noexcept { return m_alloc; }
    const std::array<long, 6>& hcl_extents() const noexcept { return m_ext; }
    const std::array<long, 6>& hcl_strides() const noexcept { return m_str; }

private:
    template <class DT2, class... P2>
    friend class View;

    template <std::size_t... R, class... I>
    long offset(std::index_sequence<R...>, I... i) const noexcept
    {
        return (0L + ... + (static_cast<long>(i) * m_str[R]));
    }
    void set_left_extents_n(const long* n)
    {
        long s = 1;
        for (int r = 0; r < 6; ++r) {
            m_ext[r] = r < Rank ? n[r] : 1;
            m_str[r] = s;
            s *= m_ext[r];
        }
    }
    void set_left_extents(std::initializer_list<long> n)
    {
        long s = 1;
        int r = 0;
        for (long e : n) {
            m_ext[r] = e;
            m_str[r] = s;
            s *= e;
            ++r;
        }
        for (; r < 6; ++r) {
            m_ext[r] = 1;
            m_str[r] = s;
        }
    }
    long span_count() const noexcept
    {
        long last = 0;
        for (int r = 0; r < Rank; ++r) {
            if (m_ext[r] == 0) {
                return 0;
            }
            last += (m_ext[r] - 1) * m_str[r];
        }
        return last + 1;
    }

    std::shared_ptr<non_const_value_type[]> m_alloc;
    value_type* m_ptr = nullptr;
    std::array<long, 6> m_ext{1, 1, 1, 1, 1, 1};
    std::array<long, 6> m_str{1, 1, 1, 1, 1, 1};
    std::string m_label;
};

template <class T>
struct is_view : std::false_type {
};
template <class DT, class... P>
struct is_view<View<DT, P...>> : std::true_type {
};
template <class T>
inline constexpr bool is_view_v = is_view<std::remove_cv_t<T>>::value;

namespace hcl_impl {

template <class A>
struct sub_arg {
    static constexpr bool keeps = false; // an integer index
};
template <>
struct sub_arg<ALL_t> {
    static constexpr bool keeps = true;
};
template <class A, class B>
struct sub_arg<pair<A, B>> {
    static constexpr bool keeps = true;
};
template <class A, class B>
struct sub_arg<std::pair<A, B>> {
    static constexpr bool keeps = true;
};

inline void apply_arg(ALL_t, long ext, long str, long& off, long& new_ext, long& new_str, bool& keep)
{
    new_ext = ext;
    new_str = str;
    keep = true;
    (void)off;
}
template <class A, class B>
void apply_arg(const pair<A, B>& p, long ext, long str, long& off, long& new_ext, long& new_str, bool& keep)
{
    (void)ext;
    off += (long)p.first * str;
    new_ext = (long)p.second - (long)p.first;
    new_str = str;
    keep = true;
}
template <class A, class B>
void apply_arg(const std::pair<A, B>& p, long ext, long str, long& off, long& new_ext, long& new_str, bool& keep)
{
    (void)ext;
    off += (long)p.first * str;
    new_ext = (long)p.second - (long)p.first;
    new_str = str;
    keep = true;
}
template <class I, std::enable_if_t<std::is_integral_v<I>, int> = 0>
void apply_arg(I i, long ext, long str, long& off, long& new_ext, long& new_str, bool& keep)
{
    (void)ext;
    off += (long)i * str;
    new_ext = 1;
    new_str = str;
    keep = false;
}

} // namespace hcl_impl

// subview(v, args...): an integer drops its dimension, ALL or a [first,
// second) pair keeps it
template <class DT, class... P, class... Args>
auto subview(const View<DT, P...>& v, Args... args)
{
    using V = View<DT, P...>;
    static_assert(sizeof...(Args) == V::Rank, "one subview argument per dimension");
    constexpr int R = (0 + ... + (hcl_impl::sub_arg<std::remove_cv_t<Args>>::keeps ? 1 : 0));
    using Out = View<typename hcl_impl::make_data_type<typename V::value_type, R>::type, LayoutStride, HostSpace>;
    std::array<long, 6> ext{1, 1, 1, 1, 1, 1};
    std::array<long, 6> str{1, 1, 1, 1, 1, 1};
    long off = 0;
    int r = 0;
    int out = 0;
    auto one = [&](const auto& a) {
        long ne = 1, ns = 1;
        bool keep = false;
        hcl_impl::apply_arg(a, v.hcl_extents()[r], v.hcl_strides()[r], off, ne, ns, keep);
        if (keep) {
            ext[out] = ne;
            str[out] = ns;
            ++out;
        }
        ++r;
    };
    (one(args), ...);
    return Out::from_parts(v.hcl_alloc(), v.data() + off, ext, str, v.label());
}

template <class V>
auto create_mirror_view(const V& v)
{
    return v;
}
template <class Space, class V>
auto create_mirror_view(const Space&, const V& v)
{
    return v;
}

} // namespace Kokkos
