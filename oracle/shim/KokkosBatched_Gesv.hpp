// Stand-in for KokkosBatched::SerialGesv as used by the reference's
// xyzvec_from_xietavec (src/cubed_sphere_transforms_impl.hpp:152-239): a 2x2
// dense solve A x = b by Cramer's rule.  Off the hot path; needed only so the
// reference sources compile (test infrastructure only).
#ifndef SBSLPM_ORACLE_SHIM_KOKKOSBATCHED_GESV_HPP
#define SBSLPM_ORACLE_SHIM_KOKKOSBATCHED_GESV_HPP
#include <Kokkos_Core.hpp>

namespace KokkosBatched {
namespace Gesv {
struct StaticPivoting {};
struct NoPivoting {};
}  // namespace Gesv

template <class Alg>
struct SerialGesv {
  template <class A, class X, class B, class T>
  static int invoke(const A& a, const X& x, const B& b, const T&) {
    double det = a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0);
    x(0) = (b(0) * a(1, 1) - a(0, 1) * b(1)) / det;
    x(1) = (a(0, 0) * b(1) - b(0) * a(1, 0)) / det;
    return 0;
  }
};
}  // namespace KokkosBatched

#endif
