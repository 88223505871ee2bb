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
template <class T, std::size_t N> using Array = std::array<T, N>;
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
// Pointer-backed 3-D view (View<T***>) with column-major indexing over
// storage the checker owns.
template <class T, class... P> struct View<T***, P...> {
  T* p = nullptr;
  std::size_t n0 = 0, n1 = 0;
  View() = default;
  View(T* q, std::size_t a, std::size_t b) : p(q), n0(a), n1(b) {}
  T& operator()(std::size_t i, std::size_t j, std::size_t k) const { return p[i + n0 * (j + n1 * k)]; }
};
struct ALL_t {};
inline ALL_t ALL() { return {}; }
// subview(v, ALL, ALL, ALL, iv, q) for the checker's array adapters, which
// expose sub(iv, q) returning a 3-index accessor, and subview(v, ALL, ALL,
// ALL, ALL, q), a 4-index accessor from sub4(q).
template <class V> auto subview(V const& v, ALL_t, ALL_t, ALL_t, int iv, int q) { return v.sub(iv, q); }
template <class V> auto subview(V const& v, ALL_t, ALL_t, ALL_t, ALL_t, std::size_t q) { return v.sub4(q); }
// Hierarchical parallelism run serially: a team is one element of a league,
// its thread range a plain nested loop.
template <unsigned N> struct Rank {};
struct SerialTeam {
  int rank = 0;
  int league_rank() const { return rank; }
  void team_barrier() const {}
};
template <class R, class Team> struct TeamThreadMDRange {
  std::size_t e[4];
  TeamThreadMDRange(const Team&, std::size_t a, std::size_t b, std::size_t c, std::size_t d) : e{a, b, c, d} {}
};
template <class R, class Team, class F> void parallel_for(const TeamThreadMDRange<R, Team>& r, F f) {
  for (std::size_t v = 0; v < r.e[3]; ++v)
    for (std::size_t k = 0; k < r.e[2]; ++k)
      for (std::size_t j = 0; j < r.e[1]; ++j)
        for (std::size_t i = 0; i < r.e[0]; ++i) f((int)i, (int)j, (int)k, (int)v);
}
}  // namespace Kokkos
