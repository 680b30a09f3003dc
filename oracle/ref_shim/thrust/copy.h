// thrust stand-in for the reference's contraction (src/contract.cpp:310-328):
// execution-policy tags, counting_iterator and copy_if with a stencil, run
// serially in order.  TEST INFRASTRUCTURE ONLY (see Kokkos_Core.hpp one
// directory up).
#pragma once
#include <cstdint>
#include <iterator>

namespace thrust {

struct host_policy_t {};
struct device_policy_t {};
constexpr host_policy_t host{};
constexpr device_policy_t device{};

template <class T>
struct counting_iterator {
    T v;
    explicit counting_iterator(T x) : v(x) {}
    T operator*() const { return v; }
    counting_iterator operator+(int64_t k) const { return counting_iterator(v + (T)k); }
    counting_iterator& operator++() {
        ++v;
        return *this;
    }
    bool operator!=(const counting_iterator& o) const { return v != o.v; }
    int64_t operator-(const counting_iterator& o) const { return (int64_t)v - (int64_t)o.v; }
};

// copies *first.. for which pred(stencil[k]) holds, in order; returns the end
// of the output
template <class Policy, class In, class Stencil, class Out, class Pred>
Out copy_if(const Policy&, In first, In last, Stencil stencil, Out result, Pred pred) {
    for (; first != last; ++first, ++stencil)
        if (pred(*stencil)) *result++ = *first;
    return result;
}

}  // namespace thrust
