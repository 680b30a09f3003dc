// Kokkos_Core.hpp -- a serial, single-threaded stand-in for the part of the
// Kokkos API that the reference's clustering sources use (src/*.cpp and
// interface/*.hpp of euphoricpoptarts/PennsylvaniaGPUGraphClustering).
//
// TEST INFRASTRUCTURE ONLY.  It lets the reference's own sources compile with
// g++ into oracle/_ref/, so that the CPU oracle and the CUDA library can be
// checked against the reference's code rather than only against a restatement.
// Execution model: every parallel construct runs its iterations in order on
// the calling thread; a team has exactly one member (team_size() == 1), so
// TeamThreadRange loops are plain loops, team barriers are no-ops and team
// reductions return the single member's value.  This is one legal schedule of
// the Kokkos programming model (the Serial back end behaves the same way), so
// the reference's results here are those of one particular execution.
//
// std::random_device, which the reference's refinement uses for its seeds
// (src/leidenR.cpp:289), is redirected to a stream the test harness controls.
#pragma once

#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

// math.h / stdlib.h above put the std::abs overloads (float and double as
// well as the integers) in the global namespace, as CUDA's headers do for the
// reference's device code: its unqualified abs(float) (src/local_mover.cpp:319)
// must not resolve to the C library's int abs.
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_FORCEINLINE_FUNCTION inline

// ---- seeds of std::random_device ------------------------------------------
namespace pggc_ref {
// next value of the harness-controlled seed stream (defined in the harness)
unsigned int next_random_seed();
struct seeded_random_device {
    using result_type = unsigned int;
    seeded_random_device() = default;
    explicit seeded_random_device(const std::string&) {}
    result_type operator()() { return next_random_seed(); }
    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return std::numeric_limits<result_type>::max(); }
    double entropy() const noexcept { return 0.0; }
};
}  // namespace pggc_ref
namespace std {
using pggc_ref_seeded_random_device = ::pggc_ref::seeded_random_device;
}
// <random> is included above, so the standard library's own declaration is
// not renamed; every later `std::random_device` becomes the seeded stand-in.
#define random_device pggc_ref_seeded_random_device

namespace Kokkos {

// ---- spaces -----------------------------------------------------------------
struct HostSpace {
    using memory_space = HostSpace;
};
struct SharedHostPinnedSpace {
    using memory_space = SharedHostPinnedSpace;
};
struct Serial {
    using execution_space = Serial;
    using memory_space = HostSpace;
    using device_type = Serial;
    void fence() const {}
    void fence(const std::string&) const {}
};
// the reference hard-wires Kokkos::Cuda (interface/core_types.h:16): here it
// is the serial space
using Cuda = Serial;
using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;
struct MemoryUnmanaged {};
inline void fence() {}
inline void fence(const std::string&) {}

template <class S>
struct Schedule {};
struct Dynamic {};
struct Static {};

struct Timer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    void reset() { t0 = std::chrono::steady_clock::now(); }
    double seconds() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

// ---- views ------------------------------------------------------------------
struct ViewAllocateWithoutInitializing {
    std::string label;
    explicit ViewAllocateWithoutInitializing(const std::string& l) : label(l) {}
    explicit ViewAllocateWithoutInitializing(const char* l) : label(l) {}
};

namespace Impl {
template <class T>
std::shared_ptr<T> alloc_array(size_t n, bool zero) {
    // value-initialised storage (zeros) whether or not the caller asked for
    // initialisation: uninitialised Kokkos memory has unspecified contents,
    // and zeros are one legal value of it
    (void)zero;
    std::shared_ptr<T> p(new T[n > 0 ? n : 1](), std::default_delete<T[]>());
    return p;
}
}  // namespace Impl

// rank-0 view
template <class D, class... P>
class View {
  public:
    using value_type = D;
    using non_const_value_type = std::remove_const_t<D>;
    std::shared_ptr<non_const_value_type> mem;
    non_const_value_type* ptr = nullptr;
    std::string lbl;
    View() = default;
    explicit View(const std::string& label) : mem(Impl::alloc_array<non_const_value_type>(1, true)), lbl(label) {
        ptr = mem.get();
    }
    explicit View(const char* label) : View(std::string(label)) {}
    explicit View(const ViewAllocateWithoutInitializing& a) : View(a.label) {}
    explicit View(non_const_value_type* p) : ptr(p) {}
    non_const_value_type& operator()() const { return *ptr; }
    non_const_value_type* data() const { return ptr; }
    size_t size() const { return 1; }
    size_t extent(int) const { return 1; }
    const std::string& label() const { return lbl; }
};

// rank-1 view: reference-counted, shallow copies, subviews alias
template <class T, class... P>
class View<T*, P...> {
  public:
    using value_type = T;
    using non_const_value_type = std::remove_const_t<T>;
    using data_type = T*;
    using size_type = size_t;
    std::shared_ptr<non_const_value_type> mem;
    non_const_value_type* ptr = nullptr;
    size_t n = 0;
    std::string lbl;

    View() = default;
    View(const std::string& label, size_t count)
        : mem(Impl::alloc_array<non_const_value_type>(count, true)), n(count), lbl(label) {
        ptr = mem.get();
    }
    View(const char* label, size_t count) : View(std::string(label), count) {}
    View(const ViewAllocateWithoutInitializing& a, size_t count) : View(a.label, count) {}
    // unmanaged view of caller memory
    View(non_const_value_type* p, size_t count) : ptr(p), n(count) {}
    // views of the same element type with other template arguments
    template <class... Q>
    View(const View<T*, Q...>& o) : mem(o.mem), ptr(o.ptr), n(o.n), lbl(o.lbl) {}
    template <class... Q>
    View& operator=(const View<T*, Q...>& o) {
        mem = o.mem;
        ptr = o.ptr;
        n = o.n;
        lbl = o.lbl;
        return *this;
    }
    View(const View&) = default;
    View& operator=(const View&) = default;

    template <class I>
    non_const_value_type& operator()(I i) const {
        return ptr[i];
    }
    template <class I>
    non_const_value_type& operator[](I i) const {
        return ptr[i];
    }
    non_const_value_type* data() const { return ptr; }
    size_t size() const { return n; }
    size_t span() const { return n; }
    size_t extent(int) const { return n; }
    int extent_int(int) const { return (int)n; }
    const std::string& label() const { return lbl; }
    bool is_allocated() const { return ptr != nullptr; }
};

template <class T, class... P, class A, class B>
View<T*, P...> subview(const View<T*, P...>& v, const std::pair<A, B>& r) {
    View<T*, P...> s;
    s.mem = v.mem;
    s.ptr = v.ptr + r.first;
    s.n = (size_t)(r.second - r.first);
    s.lbl = v.lbl;
    return s;
}

// deep_copy: view <- view (element-wise, the shorter length), view <- scalar,
// rank-0 view <- scalar
template <class T, class... P, class U, class... Q>
void deep_copy(const View<T*, P...>& dst, const View<U*, Q...>& src) {
    const size_t k = std::min(dst.size(), src.size());
    for (size_t i = 0; i < k; i++) dst.ptr[i] = src.ptr[i];
}
template <class T, class... P, class S, std::enable_if_t<std::is_arithmetic<S>::value, int> = 0>
void deep_copy(const View<T*, P...>& dst, const S& value) {
    for (size_t i = 0; i < dst.size(); i++) dst.ptr[i] = (T)value;
}
template <class T, class... P, class S, std::enable_if_t<std::is_arithmetic<S>::value, int> = 0>
void deep_copy(const View<T, P...>& dst, const S& value) {
    *dst.ptr = (T)value;
}
template <class E, class A, class B>
void deep_copy(const E&, const A& dst, const B& src) {
    deep_copy(dst, src);
}

// ---- atomics (plain operations: one thread) ----------------------------------
template <class T, class U>
void atomic_add(T* p, const U& v) {
    *p += (T)v;
}
template <class T, class U>
T atomic_fetch_add(T* p, const U& v) {
    T old = *p;
    *p += (T)v;
    return old;
}
template <class T, class U>
void atomic_min(T* p, const U& v) {
    if ((T)v < *p) *p = (T)v;
}
template <class T, class U>
void atomic_max(T* p, const U& v) {
    if ((T)v > *p) *p = (T)v;
}
template <class T, class U, class V>
T atomic_compare_exchange(T* p, const U& expected, const V& desired) {
    T old = *p;
    if (old == (T)expected) *p = (T)desired;
    return old;
}

// ---- math -------------------------------------------------------------------
template <class T>
T abs(T x) {
    return x < 0 ? -x : x;
}
inline float abs(float x) { return std::fabs(x); }
inline double abs(double x) { return std::fabs(x); }
// Kokkos' pow follows std::pow's overloads: a float base with an integer
// exponent is computed in double
template <class A, class B>
auto pow(A a, B b) {
    return std::pow(a, b);
}
template <class T>
T max(T a, T b) {
    return a < b ? b : a;
}
template <class T>
T min(T a, T b) {
    return b < a ? b : a;
}

// ---- hashing ----------------------------------------------------------------
// pod_hash: MurmurHash3_x86_32 (Austin Appleby, public domain) of the key's
// bytes with seed 0
template <class T>
struct pod_hash {
    using argument_type = T;
    using result_type = uint32_t;
    uint32_t operator()(const T& key) const {
        static_assert(sizeof(T) % 4 == 0, "pod_hash stand-in hashes whole 32-bit words");
        const unsigned char* bytes = reinterpret_cast<const unsigned char*>(&key);
        const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
        uint32_t h = 0;
        for (size_t i = 0; i < sizeof(T); i += 4) {
            uint32_t k;
            std::memcpy(&k, bytes + i, 4);
            k *= c1;
            k = (k << 15) | (k >> 17);
            k *= c2;
            h ^= k;
            h = (h << 13) | (h >> 19);
            h = h * 5 + 0xe6546b64u;
        }
        h ^= (uint32_t)sizeof(T);
        h ^= h >> 16;
        h *= 0x85ebca6bu;
        h ^= h >> 13;
        h *= 0xc2b2ae35u;
        h ^= h >> 16;
        return h;
    }
};

// ---- reducers ----------------------------------------------------------------
template <class S, class I>
struct ValLocScalar {
    S val;
    I loc;
};

template <class T, class Space = HostSpace>
struct Sum {
    using reducer = Sum;
    using value_type = T;
    T& ref;
    explicit Sum(T& r) : ref(r) {}
    void join(T& d, const T& s) const { d += s; }
    void init(T& v) const { v = T(0); }
    T& reference() const { return ref; }
};
template <class T, class Space = HostSpace>
struct Max {
    using reducer = Max;
    using value_type = T;
    T& ref;
    explicit Max(T& r) : ref(r) {}
    void join(T& d, const T& s) const {
        if (s > d) d = s;
    }
    void init(T& v) const { v = std::numeric_limits<T>::lowest(); }
    T& reference() const { return ref; }
};
template <class T, class Space = HostSpace>
struct Min {
    using reducer = Min;
    using value_type = T;
    T& ref;
    explicit Min(T& r) : ref(r) {}
    void join(T& d, const T& s) const {
        if (s < d) d = s;
    }
    void init(T& v) const { v = std::numeric_limits<T>::max(); }
    T& reference() const { return ref; }
};
// the largest value; among equal values the smallest location
template <class S, class I, class Space = HostSpace>
struct MaxFirstLoc {
    using reducer = MaxFirstLoc;
    using value_type = ValLocScalar<S, I>;
    value_type& ref;
    explicit MaxFirstLoc(value_type& r) : ref(r) {}
    void join(value_type& d, const value_type& s) const {
        if (s.val > d.val || (s.val == d.val && s.loc < d.loc)) d = s;
    }
    void init(value_type& v) const {
        v.val = std::numeric_limits<S>::lowest();
        v.loc = std::numeric_limits<I>::max();
    }
    value_type& reference() const { return ref; }
};

namespace Impl {
template <class R, class = void>
struct is_reducer : std::false_type {};
template <class R>
struct is_reducer<R, std::void_t<typename R::reducer>> : std::true_type {};

// the value type of a reduction / scan functor: its value_type typedef, or
// the second parameter of its call operator
template <class F, class = void>
struct has_value_type : std::false_type {};
template <class F>
struct has_value_type<F, std::void_t<typename F::value_type>> : std::true_type {};
template <class M>
struct second_arg;
template <class C, class R, class A0, class A1, class... A>
struct second_arg<R (C::*)(A0, A1, A...) const> {
    using type = std::remove_cv_t<std::remove_reference_t<A1>>;
};
template <class C, class R, class A0, class A1, class... A>
struct second_arg<R (C::*)(A0, A1, A...)> {
    using type = std::remove_cv_t<std::remove_reference_t<A1>>;
};
template <class F, bool = has_value_type<F>::value>
struct functor_value {
    using type = typename second_arg<decltype(&F::operator())>::type;
};
template <class F>
struct functor_value<F, true> {
    using type = typename F::value_type;
};
template <class F, class V, class = void>
struct has_init : std::false_type {};
template <class F, class V>
struct has_init<F, V, std::void_t<decltype(std::declval<const F&>().init(std::declval<V&>()))>> : std::true_type {};
template <class F, class V>
void init_value(const F& f, V& v) {
    if constexpr (has_init<F, V>::value) f.init(v);
    else v = V();
}
}  // namespace Impl

// ---- policies and the team member ------------------------------------------------
template <class... P>
struct RangePolicy {
    int64_t b = 0, e = 0;
    RangePolicy(int64_t begin, int64_t end) : b(begin), e(end) {}
};

struct AUTO_t {};
constexpr AUTO_t AUTO{};

struct PerTeamValue {
    size_t bytes;
};
inline PerTeamValue PerTeam(size_t bytes) { return PerTeamValue{bytes}; }

class TeamScratch {
  public:
    std::vector<unsigned char>* buf = nullptr;
    size_t top = 0;
    void* get_shmem(size_t bytes) {
        // 8-byte alignment of every chunk
        size_t at = (top + 7) & ~(size_t)7;
        if (at + bytes > buf->size()) buf->resize(at + bytes);
        top = at + bytes;
        return buf->data() + at;
    }
};

class TeamMember {
  public:
    int64_t league = 0, league_n = 0;
    mutable TeamScratch scratch;
    int64_t league_rank() const { return league; }
    int64_t league_size() const { return league_n; }
    int team_rank() const { return 0; }
    int team_size() const { return 1; }
    void team_barrier() const {}
    TeamScratch& team_shmem() const { return scratch; }
    TeamScratch& team_scratch(int) const { return scratch; }
    template <class R>
    void team_reduce(const R& r, const typename R::value_type& v) const {
        r.reference() = v;
    }
};

template <class... P>
struct TeamPolicy {
    using member_type = TeamMember;
    int64_t league = 0;
    size_t scratch_bytes = 0;
    TeamPolicy(int64_t l, AUTO_t) : league(l) {}
    TeamPolicy(int64_t l, int) : league(l) {}
    TeamPolicy(int64_t l, AUTO_t, int) : league(l) {}
    TeamPolicy(int64_t l, int, int) : league(l) {}
    TeamPolicy& set_scratch_size(int, PerTeamValue v) {
        scratch_bytes = v.bytes;
        return *this;
    }
};

template <class I>
struct TeamThreadRangeBounds {
    I b, e;
};
template <class A, class B>
auto TeamThreadRange(const TeamMember&, A b, B e) {
    using I = std::common_type_t<A, B>;
    return TeamThreadRangeBounds<I>{(I)b, (I)e};
}
template <class A>
auto TeamThreadRange(const TeamMember&, A e) {
    return TeamThreadRangeBounds<A>{A(0), e};
}
struct PerTeamSingle {};
inline PerTeamSingle PerTeam(const TeamMember&) { return PerTeamSingle{}; }
template <class F>
void single(PerTeamSingle, const F& f) {
    f();
}

// ---- parallel_for ---------------------------------------------------------------
template <class... P, class F>
void parallel_for(const std::string&, const RangePolicy<P...>& p, const F& f) {
    for (int64_t i = p.b; i < p.e; i++) f(i);
}
template <class F>
void parallel_for(const std::string& name, int64_t n, const F& f) {
    parallel_for(name, RangePolicy<>(0, n), f);
}
template <class... P, class F>
void parallel_for(const std::string&, const TeamPolicy<P...>& p, const F& f) {
    std::vector<unsigned char> buf(p.scratch_bytes);
    TeamMember m;
    m.league_n = p.league;
    m.scratch.buf = &buf;
    for (int64_t r = 0; r < p.league; r++) {
        m.league = r;
        m.scratch.top = 0;
        f(m);
    }
}
template <class I, class F>
void parallel_for(const TeamThreadRangeBounds<I>& r, const F& f) {
    for (I i = r.b; i < r.e; i++) f(i);
}

// ---- parallel_reduce --------------------------------------------------------------
template <class... P, class F, class R>
void parallel_reduce(const std::string&, const RangePolicy<P...>& p, const F& f, R&& result) {
    using RR = std::remove_cv_t<std::remove_reference_t<R>>;
    if constexpr (Impl::is_reducer<RR>::value) {
        typename RR::value_type v;
        result.init(v);
        for (int64_t i = p.b; i < p.e; i++) f(i, v);
        result.reference() = v;
    } else {
        RR v;
        Impl::init_value(f, v);
        for (int64_t i = p.b; i < p.e; i++) f(i, v);
        result = v;
    }
}
template <class I, class F, class R>
void parallel_reduce(const TeamThreadRangeBounds<I>& r, const F& f, R&& result) {
    using RR = std::remove_cv_t<std::remove_reference_t<R>>;
    if constexpr (Impl::is_reducer<RR>::value) {
        typename RR::value_type v;
        result.init(v);
        for (I i = r.b; i < r.e; i++) f(i, v);
        result.reference() = v;
    } else {
        RR v = RR();
        for (I i = r.b; i < r.e; i++) f(i, v);
        result = v;
    }
}

// ---- parallel_scan ------------------------------------------------------------------
// one pass with final = true: the functor sees the exclusive prefix
template <class... P, class F>
void parallel_scan(const std::string&, const RangePolicy<P...>& p, const F& f) {
    using V = typename Impl::functor_value<F>::type;
    V v;
    Impl::init_value(f, v);
    for (int64_t i = p.b; i < p.e; i++) f(i, v, true);
}
template <class... P, class F, class R>
void parallel_scan(const std::string&, const RangePolicy<P...>& p, const F& f, R& result) {
    using V = typename Impl::functor_value<F>::type;
    V v;
    Impl::init_value(f, v);
    for (int64_t i = p.b; i < p.e; i++) f(i, v, true);
    if constexpr (std::is_arithmetic<R>::value) result = v;
    else result() = v;
}

}  // namespace Kokkos
