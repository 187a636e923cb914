// TEST INFRASTRUCTURE ONLY: host stand-in for KokkosBatched::SerialGemv and
// SerialGemm with the unblocked algorithm, restated from KokkosKernels' published
// serial internals: y <- beta*y (0: set, 1: keep), then per output row
// t = sum_j A(i,j) x(j) in order of j and y(i) += alpha*t; for Gemm the same per
// output (i,j) with t = sum_p A(i,p) B(p,j).
#ifndef KFVM_REFSHIM_KOKKOSBATCHED_HPP
#define KFVM_REFSHIM_KOKKOSBATCHED_HPP

#include "Kokkos_Core.hpp"

namespace KokkosBatched {

struct Trans {
  struct NoTranspose {};
  struct Transpose {};
};
struct Algo {
  struct Gemv {
    struct Unblocked {};
  };
  struct Gemm {
    struct Unblocked {};
  };
};

template <class TransA, class AlgoT>
struct SerialGemv {
  template <class S, class AV, class XV, class YV>
  KOKKOS_INLINE_FUNCTION static int invoke(const S alpha, const AV &A, const XV &x,
                                           const S beta, const YV &y) {
    static_assert(std::is_same_v<TransA, Trans::NoTranspose>, "shim: NoTranspose only");
    const int m = int(A.extent(0)), n = int(A.extent(1));
    if (beta == S(0)) {
      for (int i = 0; i < m; i++) y(i) = S(0);
    } else if (beta != S(1)) {
      for (int i = 0; i < m; i++) y(i) *= beta;
    }
    if (alpha != S(0)) {
      for (int i = 0; i < m; i++) {
        S t(0);
        for (int j = 0; j < n; j++) t += A(i, j) * x(j);
        y(i) += alpha * t;
      }
    }
    return 0;
  }
};

template <class TransA, class TransB, class AlgoT>
struct SerialGemm {
  template <class S, class AV, class BV, class CV>
  KOKKOS_INLINE_FUNCTION static int invoke(const S alpha, const AV &A, const BV &B,
                                           const S beta, const CV &C) {
    static_assert(std::is_same_v<TransA, Trans::NoTranspose> &&
                      std::is_same_v<TransB, Trans::NoTranspose>,
                  "shim: NoTranspose only");
    const int m = int(C.extent(0)), n = int(C.extent(1)), k = int(A.extent(1));
    if (beta == S(0)) {
      for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) C(i, j) = S(0);
    } else if (beta != S(1)) {
      for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) C(i, j) *= beta;
    }
    if (alpha != S(0)) {
      for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) {
          S t(0);
          for (int p = 0; p < k; p++) t += A(i, p) * B(p, j);
          C(i, j) += alpha * t;
        }
    }
    return 0;
  }
};

} // namespace KokkosBatched

#endif
