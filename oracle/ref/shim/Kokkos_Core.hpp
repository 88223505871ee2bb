// Minimal host-only stand-in for the parts of Kokkos that the reference
// GRMHD numerics touch (math wrappers, function-attribute macros, a
// fixed-size View).  Used only to compile the reference's per-cell code in
// place as a CPU checker; never linked into the CUDA library.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <algorithm>
#include <stdexcept>
#include <array>
#include <utility>
#include <vector>
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]
namespace Kokkos {
using std::fabs; using std::sqrt; using std::pow; using std::exp; using std::log;
using std::copysign; using std::isfinite; using std::fmin; using std::fmax;
template <class T> inline T min(T a, T b) { return a < b ? a : b; }
template <class T> inline T max(T a, T b) { return a > b ? a : b; }
[[noreturn]] inline void abort(const char* m) { throw std::runtime_error(m); }
struct HostSpace {};
struct LayoutLeft {};
// Fixed-extent 1-D view backed by owned storage (View<double[N], Space>).
template <class T, class... P> struct View;
template <class T, std::size_t N, class... P> struct View<T[N], P...> {
  T d[N] = {};
  View() = default;
  explicit View(const char*) {}
  T& operator()(std::size_t i) { return d[i]; }
  const T& operator()(std::size_t i) const { return d[i]; }
};
// Pointer-backed 1-D view (View<T*, Space[, MemoryTraits]>) over storage the
// checker owns, convertible to its const-element form.
template <unsigned> struct MemoryTraits {};
constexpr unsigned RandomAccess = 0;
template <class T, class... P> struct View<T*, P...> {
  T* p = nullptr;
  View() = default;
  explicit View(T* q) : p(q) {}
  template <class U, class... Q> View(const View<U*, Q...>& o) : p(o.p) {}
  T& operator()(std::size_t i) const { return p[i]; }
};
struct ALL_t {};
inline ALL_t ALL() { return {}; }
// subview(v, ALL, ALL, ALL, iv, q) for the checker's array adapters, which
// expose sub(iv, q) returning a 3-index accessor.
template <class V> auto subview(V const& v, ALL_t, ALL_t, ALL_t, int iv, int q) { return v.sub(iv, q); }
}  // namespace Kokkos
