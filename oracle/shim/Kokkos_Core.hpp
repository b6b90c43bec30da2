// Minimal, project-written stand-in for the subset of the Kokkos Core API that the
// reference's hot-path sources use (views, range / multi-dimensional range
// policies, parallel_for / parallel_reduce, atomic_add, math forwarding).
//
// Test infrastructure only: it lets the reference's own src/*.cpp compile
// unmodified on the host with g++ and OpenMP so that they can serve as the
// pinned parity oracle and as the timed CPU baseline.  Nothing in the product
// library includes this header.
//
// Semantics kept from the Kokkos API as used by the reference:
//   * View allocations are zero-initialised (the reference relies on this for
//     freshly allocated proxy-target arrays in src/bve_time_step.cpp:335-338).
//   * Views are reference-counted handles; copying a View aliases its data.
//   * LayoutRight is row-major; LayoutStride carries explicit strides.
//   * HostSpace / the default space are the same memory (an OpenMP build).
#ifndef SBSLPM_ORACLE_SHIM_KOKKOS_CORE_HPP
#define SBSLPM_ORACLE_SHIM_KOKKOS_CORE_HPP

#include <algorithm>
#include <cmath>
// The C++ <math.h> / <stdlib.h> wrappers declare the floating-point ::abs
// overloads in the global namespace, as the real Kokkos headers' includes do;
// the reference calls unqualified abs() on doubles
// (src/initialize_cubed_sphere.cpp:305), which would otherwise bind to the
// C library's int abs(int).
#include <math.h>
#include <stdlib.h>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]

namespace Kokkos {

struct LayoutRight {};
struct LayoutLeft {};
struct LayoutStride {};
struct HostSpace {};
struct Unmanaged {};
template <class T> struct MemoryTraits {};

struct OpenMP {
  using memory_space = HostSpace;
  using execution_space = OpenMP;
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

struct ALL_t {};
static constexpr ALL_t ALL{};

namespace numbers {
static constexpr double pi = 3.141592653589793238462643383279502884;
}

namespace shim_detail {
template <class T> struct data_traits {
  using value_type = T;
  static constexpr int rank = 0;
};
template <class T> struct data_traits<T*> {
  using value_type = typename data_traits<T>::value_type;
  static constexpr int rank = data_traits<T>::rank + 1;
};
template <class T, std::size_t N> struct data_traits<T[N]> {
  using value_type = typename data_traits<T>::value_type;
  static constexpr int rank = data_traits<T>::rank + 1;
};

template <class... P> struct is_stride : std::false_type {};
template <class... P> struct is_stride<LayoutStride, P...> : std::true_type {};
template <class H, class... P> struct is_stride<H, P...> : is_stride<P...> {};
}  // namespace shim_detail

template <class DataType, class... Props>
class View {
 public:
  using traits = shim_detail::data_traits<DataType>;
  using value_type = typename traits::value_type;
  using non_const_value_type = typename std::remove_const<value_type>::type;
  static constexpr int rank = traits::rank;
  static constexpr int Rank = traits::rank;

  std::shared_ptr<non_const_value_type> m_alloc;
  value_type* m_ptr = nullptr;
  std::size_t m_ext[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::size_t m_str[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::string m_label;

  View() = default;

  View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    m_label = label;
    allocate(n0, n1, n2, n3);
  }
  View(const char* label, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    m_label = label;
    allocate(n0, n1, n2, n3);
  }
  // Unmanaged view over caller memory.
  View(value_type* ptr, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    m_ptr = ptr;
    set_extents(n0, n1, n2, n3);
    set_right_strides();
  }

  // Views of the same element type and rank alias each other across
  // layout / memory-space template arguments (one host memory space here).
  template <class D2, class... P2>
  View(const View<D2, P2...>& o) {
    static_assert(View<D2, P2...>::rank == rank, "rank mismatch");
    m_alloc = o.m_alloc;
    m_ptr = o.m_ptr;
    for (int i = 0; i < 8; i++) {
      m_ext[i] = o.m_ext[i];
      m_str[i] = o.m_str[i];
    }
    m_label = o.m_label;
  }

  void set_extents(std::size_t n0, std::size_t n1, std::size_t n2, std::size_t n3) {
    std::size_t n[4] = {n0, n1, n2, n3};
    for (int i = 0; i < 4; i++) m_ext[i] = (i < rank) ? n[i] : 1;
  }
  void set_right_strides() {
    std::size_t s = 1;
    for (int i = rank - 1; i >= 0; i--) {
      m_str[i] = s;
      s *= m_ext[i];
    }
  }
  void allocate(std::size_t n0, std::size_t n1, std::size_t n2, std::size_t n3) {
    set_extents(n0, n1, n2, n3);
    set_right_strides();
    std::size_t total = span_count();
    non_const_value_type* p = new non_const_value_type[total > 0 ? total : 1]();
    m_alloc = std::shared_ptr<non_const_value_type>(p, std::default_delete<non_const_value_type[]>());
    m_ptr = p;
  }
  std::size_t span_count() const {
    std::size_t t = 1;
    for (int i = 0; i < rank; i++) t *= m_ext[i];
    return t;
  }

  value_type& operator()(std::size_t i0) const { return m_ptr[i0 * m_str[0]]; }
  value_type& operator()(std::size_t i0, std::size_t i1) const {
    return m_ptr[i0 * m_str[0] + i1 * m_str[1]];
  }
  value_type& operator()(std::size_t i0, std::size_t i1, std::size_t i2) const {
    return m_ptr[i0 * m_str[0] + i1 * m_str[1] + i2 * m_str[2]];
  }
  value_type& operator[](std::size_t i0) const { return m_ptr[i0 * m_str[0]]; }

  std::size_t extent(int i) const { return i < rank ? m_ext[i] : 1; }
  int extent_int(int i) const { return static_cast<int>(extent(i)); }
  std::size_t stride(int i) const { return m_str[i]; }
  std::size_t size() const { return span_count(); }
  std::size_t span() const { return span_count(); }
  value_type* data() const { return m_ptr; }
  std::string label() const { return m_label; }
  bool is_allocated() const { return m_ptr != nullptr; }
};

template <class D, class... P>
void resize(View<D, P...>& v, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
            std::size_t n3 = 0) {
  View<D, P...> nv(v.m_label, n0, n1, n2, n3);
  constexpr int R = View<D, P...>::rank;
  if (v.m_ptr != nullptr) {
    std::size_t e0 = std::min(v.extent(0), nv.extent(0));
    std::size_t e1 = std::min(v.extent(1), nv.extent(1));
    std::size_t e2 = std::min(v.extent(2), nv.extent(2));
    for (std::size_t i = 0; i < e0; i++)
      for (std::size_t j = 0; j < (R > 1 ? e1 : 1); j++)
        for (std::size_t k = 0; k < (R > 2 ? e2 : 1); k++) {
          if (R == 1) nv(i) = v(i);
          else if (R == 2) nv(i, j) = v(i, j);
          else nv(i, j, k) = v(i, j, k);
        }
  }
  v = nv;
}

template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  constexpr int R = View<D1, P1...>::rank;
  for (std::size_t i = 0; i < dst.extent(0); i++)
    for (std::size_t j = 0; j < (R > 1 ? dst.extent(1) : 1); j++)
      for (std::size_t k = 0; k < (R > 2 ? dst.extent(2) : 1); k++) {
        if (R == 1) dst(i) = src(i);
        else if (R == 2) dst(i, j) = src(i, j);
        else dst(i, j, k) = src(i, j, k);
      }
}
template <class D1, class... P1>
void deep_copy(const View<D1, P1...>& dst, const typename View<D1, P1...>::value_type& val) {
  std::size_t n = dst.span_count();
  for (std::size_t i = 0; i < n; i++) dst.m_ptr[i] = val;
}
template <class D, class... P>
View<D, P...> create_mirror_view(const View<D, P...>& v) {
  return v;
}
template <class S, class D, class... P>
View<D, P...> create_mirror_view(const S&, const View<D, P...>& v) {
  return v;
}

// subview(v3, ALL, ALL, k): the only subview form used on the reference's path.
template <class D, class... P>
View<typename View<D, P...>::value_type**, LayoutStride, HostSpace> subview(const View<D, P...>& v, ALL_t,
                                                                            ALL_t, std::size_t k) {
  View<typename View<D, P...>::value_type**, LayoutStride, HostSpace> s;
  s.m_alloc = v.m_alloc;
  s.m_ptr = v.m_ptr + k * v.m_str[2];
  s.m_ext[0] = v.m_ext[0];
  s.m_ext[1] = v.m_ext[1];
  s.m_str[0] = v.m_str[0];
  s.m_str[1] = v.m_str[1];
  s.m_label = v.m_label;
  return s;
}

class RangePolicy {
 public:
  long m_begin, m_end;
  RangePolicy(long b, long e) : m_begin(b), m_end(e) {}
  template <class Space>
  RangePolicy(const Space&, long b, long e) : m_begin(b), m_end(e) {}
};

template <int N, class... Iter> struct Rank {};
namespace Iterate {
struct Left {};
struct Right {};
}  // namespace Iterate

class MDRangePolicy {
 public:
  int m_rank;
  long m_lo[3] = {0, 0, 0};
  long m_hi[3] = {1, 1, 1};
  MDRangePolicy(std::initializer_list<long> lo, std::initializer_list<long> hi) { init(lo, hi); }
  template <class Space>
  MDRangePolicy(const Space&, std::initializer_list<long> lo, std::initializer_list<long> hi) {
    init(lo, hi);
  }
  void init(std::initializer_list<long> lo, std::initializer_list<long> hi) {
    m_rank = static_cast<int>(lo.size());
    int i = 0;
    for (long v : lo) m_lo[i++] = v;
    i = 0;
    for (long v : hi) m_hi[i++] = v;
  }
};

template <class F>
void parallel_for(long n, const F& f) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) f(static_cast<int>(i));
}
template <class F>
void parallel_for(const RangePolicy& p, const F& f) {
#pragma omp parallel for schedule(static)
  for (long i = p.m_begin; i < p.m_end; i++) f(static_cast<int>(i));
}

namespace shim_detail {
template <class F>
auto call_md(const F& f, long i, long j, long, int) -> decltype(f(0, 0), void()) {
  f(static_cast<int>(i), static_cast<int>(j));
}
template <class F>
auto call_md(const F& f, long i, long j, long k, long) -> decltype(f(0, 0, 0), void()) {
  f(static_cast<int>(i), static_cast<int>(j), static_cast<int>(k));
}
}  // namespace shim_detail

template <class F>
void parallel_for(const MDRangePolicy& p, const F& f) {
  long n0 = p.m_hi[0] - p.m_lo[0];
  long n1 = p.m_hi[1] - p.m_lo[1];
  long n2 = (p.m_rank > 2) ? (p.m_hi[2] - p.m_lo[2]) : 1;
  if (n0 <= 0 || n1 <= 0 || n2 <= 0) return;
#pragma omp parallel for collapse(2) schedule(static)
  for (long i = 0; i < n0; i++)
    for (long j = 0; j < n1; j++)
      for (long k = 0; k < n2; k++)
        shim_detail::call_md(f, i + p.m_lo[0], j + p.m_lo[1], k + p.m_lo[2], 0);
}
template <class P, class F>
void parallel_for(const std::string&, const P& p, const F& f) {
  parallel_for(p, f);
}

template <class F, class V>
void parallel_reduce(const RangePolicy& p, const F& f, V& result) {
  V total;
  f.init(total);
#pragma omp parallel
  {
    V local;
    f.init(local);
#pragma omp for schedule(static)
    for (long i = p.m_begin; i < p.m_end; i++) f(static_cast<int>(i), local);
#pragma omp critical
    f.join(total, local);
  }
  result = total;
}

template <class T>
inline void atomic_add(T* dst, const T val) {
#pragma omp atomic
  *dst += val;
}
template <class T>
inline void atomic_add(volatile T* dst, const T val) {
#pragma omp atomic
  *dst += val;
}

inline void fence() {}
template <class S>
inline void fence(const S&) {}
inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}
inline int num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
inline int num_devices() { return 0; }
inline void abort(const char* msg) {
  std::fprintf(stderr, "Kokkos::abort (oracle shim): %s\n", msg);
  std::abort();
}
inline void* kokkos_malloc(std::size_t n) { return std::malloc(n); }
inline void kokkos_free(void* p) { std::free(p); }

using std::abs;
using std::acos;
using std::atan;
using std::atan2;
using std::cos;
using std::erf;
using std::exp;
using std::floor;
using std::fmax;
using std::fmin;
using std::fmod;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
using std::tan;
using std::min;
using std::max;

}  // namespace Kokkos

#endif
