// stencil_weights.cpp -- host FP64 precompute of the stencil geometry and the
// kernel-based (SE Gaussian kernel + monomial) reconstruction weights.
//
// Replaces the reference's Stencil object (slug-cfd/kfvm-kokkos):
//   src/stencil/Stencil.H:105-135        Stencil::Stencil(lfac, geom)
//   src/stencil/Stencil.cpp:47-229       disc stencil and biased substencils
//   src/stencil/Stencil.cpp:281-846      findWeights (face, interior, derivative weights)
//   src/stencil/ReconVectors.cpp:14-86   saddle system [K P; P^T 0], LU by dgetrf/dgetrs
//   src/stencil/Monomials.cpp:14-58      monomial functionals
//   src/stencil/SEKernel.H:14-28         SE kernel functionals
//   src/stencil/StencilSymmetry.cpp      reuse of weights through reflections/rotations
//
// The weights are computed once on the host in FP64 and uploaded to the device;
// the GPU never recomputes them.  Because the saddle system is ill-conditioned
// at the usual lfac=5 (condition number ~1e7 in 2D), the arithmetic is kept in
// the reference's exact order (and compiled without FMA contraction), and the
// LU is LAPACK's dgetrf/dgetrs, so the weights are reproducible bit for bit.
// Weight vectors that the reference obtains through a symmetry map are copied
// through the same map (not re-solved), for the same reason.

#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "geometry.h"
#include "../../include/kfvm_b200.h"

extern "C" {
// LAPACK (OpenBLAS build bundled with scipy exports these names)
void scipy_dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info);
void scipy_dgetrs_(char *trans, int *n, int *nrhs, double *a, int *lda, int *ipiv,
                   double *b, int *ldb, int *info);
}

namespace kfvm {
namespace {

using Pt = std::array<double, 3>;
using PtSet = std::vector<Pt>;
using Deg = std::array<int64_t, 3>;

// ---- univariate functionals -----------------------------------------------------

// cell average of x^p over [x-1/2, x+1/2]
double avg_monomial(int64_t p, double x) {
  double ub = std::pow(x + 0.5, p + 1) / (p + 1);
  double lb = std::pow(x - 0.5, p + 1) / (p + 1);
  return ub - lb;
}

// N-th derivative functional of x^p.  The reference's recursion passes its
// arguments in swapped order (coordinate as the derivative order and vice versa);
// the result is kept as the reference computes it, since its smoothness
// indicators are defined by it.
double deriv_monomial(int64_t p, int64_t N, double x) {
  if (N == 0) return std::pow(x, p);
  if (N > p) return 0.0;
  return p * deriv_monomial(p - 1, static_cast<int64_t>(x), static_cast<double>(N - 1));
}

// cell average of the Gaussian kernel exp(-eps^2 x^2)
double avg_kernel(double eps, double x) {
  auto pf = std::sqrt(M_PI) / (2.0 * eps);
  return pf * (std::erf(eps * (x + 0.5)) - std::erf(eps * (x - 0.5)));
}

// N-th derivative of the Gaussian kernel, via Hermite polynomials
double deriv_kernel(double eps, int64_t N, double x) {
  const double sgn = N % 2 == 0 ? 1.0 : -1.0,
               Hn = sgn * std::pow(eps, N) * std::hermite(N, eps * x);
  return Hn * std::exp(-eps * eps * x * x);
}

std::vector<Deg> monomial_degrees(int dim, int total) {
  std::vector<Deg> d;
  for (int t = 0; t <= total; t++)
    for (int i = 0; i <= t; i++) {
      if (dim == 2) {
        d.push_back({i, t - i, 0});
      } else {
        for (int j = 0; j <= t - i; j++) d.push_back({i, j, t - i - j});
      }
    }
  return d;
}

// ---- symmetry maps ---------------------------------------------------------------
// A symmetry is a signed permutation of the axes; (dst) = S (ref) is tested with a
// 1e-6 tolerance.  Order and membership follow the reference's SymType list.
struct SignedPerm {
  int src[3];   // dst coordinate a is +-ref coordinate src[a]
  double sg[3]; // sign
  bool in2d;
};
// RefX RefY RefZ RefXY RefXZ RefYZ RefXYZ RotXY RotXZ RotYZ RotXYm RotXZm RotYZm
const SignedPerm kSym[13] = {
    {{0, 1, 2}, {-1, 1, 1}, true},   {{0, 1, 2}, {1, -1, 1}, true},
    {{0, 1, 2}, {1, 1, -1}, false},  {{0, 1, 2}, {-1, -1, 1}, true},
    {{0, 1, 2}, {-1, 1, -1}, false}, {{0, 1, 2}, {1, -1, -1}, false},
    {{0, 1, 2}, {-1, -1, -1}, false}, {{1, 0, 2}, {-1, 1, 1}, true},
    {{2, 1, 0}, {-1, 1, 1}, false},  {{0, 2, 1}, {1, -1, 1}, false},
    {{1, 0, 2}, {1, -1, 1}, true},   {{2, 1, 0}, {1, 1, -1}, false},
    {{0, 2, 1}, {1, 1, -1}, false}};

bool close(double a, double b) { return std::fabs(a - b) < 1.e-6; }

bool maps(int dim, int s, const Pt &d, const Pt &r) {
  const SignedPerm &p = kSym[s];
  if (dim == 2 && !p.in2d) return false;
  for (int a = 0; a < dim; a++)
    if (!close(d[a], p.sg[a] * r[p.src[a]])) return false;
  return true;
}

// For each destination query point: the reference query point it maps from (or -1)
// and the stencil index permutation of that map.
struct WeightMap {
  std::vector<int> from;
  std::vector<std::vector<int>> perm;

  WeightMap(int dim, bool self, const PtSet &stD, const PtSet &stR, const PtSet &qD,
            const PtSet &qR) {
    const int nP = (int)qD.size(), N = (int)stD.size();
    from.assign(nP, -1);
    perm.assign(nP, std::vector<int>(N, -1));
    std::vector<int> allowed, chosen(nP, -1);
    for (int s = 0; s < 13; s++) {
      bool all = true;
      for (int a = 0; a < N && all; a++) {
        bool any = false;
        for (int b = 0; b < N && !any; b++) any = maps(dim, s, stD[a], stR[b]);
        all = any;
      }
      if (all) allowed.push_back(s);
    }
    for (int a = 0; a < nP; a++) {
      const int lim = self ? a : nP;
      for (int b = 0; b < lim && from[a] < 0; b++)
        for (int s : allowed)
          if (maps(dim, s, qD[a], qR[b])) {
            from[a] = b;
            chosen[a] = s;
            break;
          }
    }
    for (int a = 0; a < nP; a++) {
      if (from[a] < 0) continue;
      for (int c = 0; c < N; c++)
        for (int e = 0; e < N; e++)
          if (maps(dim, chosen[a], stD[c], stR[e])) {
            perm[a][c] = e;
            break;
          }
    }
  }

  // dst[row][j] = ref[from[row]][perm[row][j]]
  void apply(double *dst, const double *ref, int ld) const {
    for (size_t r = 0; r < from.size(); r++)
      if (from[r] >= 0)
        for (size_t j = 0; j < perm[r].size(); j++) dst[r * ld + j] = ref[from[r] * ld + perm[r][j]];
  }
};

// ---- the saddle-point system of one (sub)stencil -----------------------------------
class Saddle {
 public:
  Saddle(int dim, double eps, int polyDeg, const PtSet &cells)
      : dim_(dim), eps_(eps), cells_(cells), n_((int)cells.size()),
        deg_(monomial_degrees(dim, polyDeg)) {
    m_ = n_ + (int)deg_.size();
    A_.assign((size_t)m_ * m_, 0.0);
    piv_.assign(m_, 0);
    for (int i = 0; i < n_; i++)
      for (int j = 0; j < n_; j++) {
        double d0 = cells_[i][0] - cells_[j][0], d1 = cells_[i][1] - cells_[j][1],
               d2 = cells_[i][2] - cells_[j][2];
        at(i, j) = dim_ == 2 ? avg_kernel(eps_, d0) * avg_kernel(eps_, d1)
                             : avg_kernel(eps_, d0) * avg_kernel(eps_, d1) * avg_kernel(eps_, d2);
      }
    for (int i = 0; i < n_; i++)
      for (int j = 0; j < (int)deg_.size(); j++) {
        at(i, j + n_) = dim_ == 2 ? avg_monomial(deg_[j][0], cells_[i][0]) *
                                        avg_monomial(deg_[j][1], cells_[i][1])
                                  : avg_monomial(deg_[j][0], cells_[i][0]) *
                                        avg_monomial(deg_[j][1], cells_[i][1]) *
                                        avg_monomial(deg_[j][2], cells_[i][2]);
        at(j + n_, i) = at(i, j + n_);
      }
    int M = m_;
    scipy_dgetrf_(&M, &M, A_.data(), &M, piv_.data(), &info_);
  }

  int info() const { return info_; }

  // weights reproducing the functional "derivative Nd at point q" from cell averages
  void solve(const Deg &Nd, const Pt &q, double *w) {
    std::vector<double> rhs(m_, 0.0);
    for (int i = 0; i < n_; i++) {
      double d0 = q[0] - cells_[i][0], d1 = q[1] - cells_[i][1], d2 = q[2] - cells_[i][2];
      rhs[i] = dim_ == 2 ? deriv_kernel(eps_, Nd[0], d0) * deriv_kernel(eps_, Nd[1], d1)
                         : deriv_kernel(eps_, Nd[0], d0) * deriv_kernel(eps_, Nd[1], d1) *
                               deriv_kernel(eps_, Nd[2], d2);
    }
    for (size_t i = 0; i < deg_.size(); i++)
      rhs[i + n_] = dim_ == 2 ? deriv_monomial(deg_[i][0], Nd[0], q[0]) *
                                    deriv_monomial(deg_[i][1], Nd[1], q[1])
                              : deriv_monomial(deg_[i][0], Nd[0], q[0]) *
                                    deriv_monomial(deg_[i][1], Nd[1], q[1]) *
                                    deriv_monomial(deg_[i][2], Nd[2], q[2]);
    char tr = 'N';
    int M = m_, one = 1, inf = 0;
    scipy_dgetrs_(&tr, &M, &one, A_.data(), &M, piv_.data(), rhs.data(), &M, &inf);
    if (inf) info_ = inf;
    std::memcpy(w, rhs.data(), sizeof(double) * n_);
  }

  // point-value weights at a set of query points, reusing symmetric rows
  void solve_points(const PtSet &qs, double *w, int ld) {
    WeightMap sym(dim_, true, cells_, cells_, qs, qs);
    const Deg zero{0, 0, 0};
    for (size_t r = 0; r < qs.size(); r++) {
      if (sym.from[r] < 0) {
        solve(zero, qs[r], w + r * ld);
      } else {
        for (int j = 0; j < n_; j++) w[r * ld + j] = w[sym.from[r] * ld + sym.perm[r][j]];
      }
    }
  }

 private:
  double &at(int i, int j) { return A_[(size_t)j * m_ + i]; }
  int dim_;
  double eps_;
  PtSet cells_;
  int n_, m_;
  std::vector<Deg> deg_;
  std::vector<double> A_;
  std::vector<int> piv_;
  int info_ = 0;
};

// ---- stencil geometry ---------------------------------------------------------------
void disc_stencil(int dim, kfvm_stencil *st) {
  const int R = KFVM_RAD;
  std::vector<std::array<int64_t, 3>> c;
  if (dim == 2) {
    c.push_back({0, 0, 0});
    for (int L = 1; L <= R; L++) {
      c.push_back({-L, 0, 0});
      c.push_back({L, 0, 0});
      c.push_back({0, -L, 0});
      c.push_back({0, L, 0});
      for (int d = 1; d <= L; d++) { // diagonals whose ring is L
        double rsq = 2.0 * d * d;
        if (rsq <= R * R && (int64_t)std::ceil(std::sqrt(rsq)) == L) {
          c.push_back({-d, -d, 0});
          c.push_back({-d, d, 0});
          c.push_back({d, -d, 0});
          c.push_back({d, d, 0});
        }
      }
      for (int a = 2; a <= R; a++) // remaining lattice points of the disc on ring L
        for (int b = 1; b < a; b++) {
          double rsq = (double)a * a + (double)b * b;
          if (rsq <= R * R && (int64_t)std::ceil(std::sqrt(rsq)) == L) {
            const int64_t s8[8][2] = {{-a, b}, {-a, -b}, {a, b}, {a, -b},
                                      {-b, a}, {-b, -a}, {b, a}, {b, -a}};
            for (auto &p : s8) c.push_back({p[0], p[1], 0});
          }
        }
    }
  } else {
    const int64_t rm = R - 1;
    for (int pass = 0; pass < 2; pass++) // inner ball first, then the shell
      for (int64_t i = -R; i <= R; i++)
        for (int64_t j = -R; j <= R; j++)
          for (int64_t k = -R; k <= R; k++) {
            const int64_t rsq = i * i + j * j + k * k;
            const bool inner = rsq <= rm * rm && std::abs(i) <= rm && std::abs(j) <= rm &&
                               std::abs(k) <= rm;
            const bool shell = rsq > rm * rm && rsq <= (int64_t)R * R;
            if ((pass == 0 && inner) || (pass == 1 && shell)) c.push_back({i, j, k});
          }
  }
  st->n_cells = (int)c.size();
  for (size_t n = 0; n < c.size(); n++)
    for (int a = 0; a < 3; a++) st->off[a][n] = c[n][a];

  auto find = [&](int64_t i, int64_t j, int64_t k) -> int64_t {
    for (int n = 0; n < st->n_cells; n++)
      if (c[n][0] == i && c[n][1] == j && c[n][2] == k) return n;
    return -1;
  };
  if (dim == 2) {
    int cnt[4] = {0, 0, 0, 0};
    for (int h = 0; h <= R; h++) { // on-axis cells first
      st->sub_idx[0][cnt[0]++] = find(-h, 0, 0);
      st->sub_idx[1][cnt[1]++] = find(h, 0, 0);
      st->sub_idx[2][cnt[2]++] = find(0, -h, 0);
      st->sub_idx[3][cnt[3]++] = find(0, h, 0);
    }
    for (int h = 0; h <= R; h++) // then off-axis pairs that lie in the disc
      for (int l = 1; l <= h; l++) {
        if (find(-h, -l, 0) < 0) continue;
        st->sub_idx[0][cnt[0]++] = find(-h, -l, 0);
        st->sub_idx[0][cnt[0]++] = find(-h, l, 0);
        st->sub_idx[1][cnt[1]++] = find(h, -l, 0);
        st->sub_idx[1][cnt[1]++] = find(h, l, 0);
        st->sub_idx[2][cnt[2]++] = find(-l, -h, 0);
        st->sub_idx[2][cnt[2]++] = find(l, -h, 0);
        st->sub_idx[3][cnt[3]++] = find(-l, h, 0);
        st->sub_idx[3][cnt[3]++] = find(l, h, 0);
      }
  } else {
    int cnt[6] = {0, 0, 0, 0, 0, 0};
    for (int n = 0; n < st->n_cells; n++) {
      const int64_t a = c[n][0], b = c[n][1], e = c[n][2];
      // cone of cells whose offset is dominated by the substencil's axis
      const int64_t axis[6] = {-a, a, -b, b, -e, e};
      const int64_t o1[6] = {b, b, a, a, a, a}, o2[6] = {e, e, e, e, b, b};
      for (int s = 0; s < 6; s++)
        if (axis[s] >= std::abs(o1[s]) && axis[s] >= std::abs(o2[s])) st->sub_idx[s][cnt[s]++] = n;
    }
  }
}

} // namespace

// Stencil::findWeights restated (Stencil.cpp:281-846)
int build_stencil(const kfvm_config *cfg, kfvm_stencil *st) {
  std::memset(st, 0, sizeof(*st));
  const int dim = cfg->dim, nq = cfg->nq;
  if ((dim != 2 && dim != 3) || nq < 1 || nq > 3) return KFVM_ERR_ARG;
  st->dim = dim;
  st->nq = nq;
  disc_stencil(dim, st);
  const int C = st->n_cells;
  st->n_cells_ctr = dim == 2 ? 5 : 7;
  st->n_cells_bias = dim == 2 ? 5 : 11;
  st->n_sub = dim == 2 ? 6 : 8;
  st->n_bias = dim == 2 ? 4 : 6;
  const int nDeriv = dim == 2 ? 2 : 3;
  const std::vector<Deg> dset = monomial_degrees(dim, nDeriv);
  st->n_indic = (int)dset.size() - 1;
  st->nqf = dim == 2 ? nq : nq * nq;
  st->nqc = dim == 2 ? nq * nq : nq * nq * nq;
  const int nqf = st->nqf, nqc = st->nqc;
  const int polyDeg[3] = {3, 1, 1};
  // the cell sizes of the whole domain (Geometry.H:28-31)
  const double dx = kfvm::cfg_dx(cfg, 0), dy = kfvm::cfg_dx(cfg, 1), dz = kfvm::cfg_dx(cfg, 2);
  const double eps = 1.0 / (cfg->lfac * std::sqrt(2.0));

  // Gauss-Legendre abscissae on (-1/2, 1/2) (src/numeric/Numeric.cpp:9-46)
  double ab[3];
  if (nq == 1) {
    ab[0] = 0.0;
  } else if (nq == 2) {
    ab[0] = -0.577350269189625764509148 / 2.0;
    ab[1] = 0.577350269189625764509148 / 2.0;
  } else {
    ab[0] = 0.0;
    ab[1] = -0.7745966692414833770358530 / 2.0;
    ab[2] = 0.7745966692414833770358530 / 2.0;
  }
  // face point sets in face order W,E,S,N,B,T; cell points; the centre point
  PtSet fq[6], cq(nqc), cen{{0.0, 0.0, 0.0}};
  for (int f = 0; f < 6; f++) fq[f].resize(nqf);
  for (int p = 0; p < nqf; p++) {
    const double a = dim == 2 ? ab[p] : ab[p / nq], b = dim == 2 ? 0.0 : ab[p % nq];
    fq[0][p] = {-0.5, a, b};
    fq[1][p] = {0.5, a, b};
    fq[2][p] = {a, -0.5, b};
    fq[3][p] = {a, 0.5, b};
    fq[4][p] = {a, b, -0.5};
    fq[5][p] = {a, b, 0.5};
  }
  for (int p = 0; p < nqc; p++)
    cq[p] = dim == 2 ? Pt{ab[p / nq], ab[p % nq], 0.0}
                     : Pt{ab[p / (nq * nq)], ab[(p / nq) % nq], ab[p % nq]};

  auto cells_of = [&](int s, int n) {
    PtSet p(n);
    for (int i = 0; i < n; i++) {
      const int idx = s < 2 ? i : (int)st->sub_idx[s - 2][i];
      p[i] = {(double)st->off[0][idx], (double)st->off[1][idx], (double)st->off[2][idx]};
    }
    return p;
  };
  auto FW = [&](int s, int f) { return &st->face_w[s][f][0][0]; };
  const int LD = KFVM_MAX_CELLS;
  auto derivs = [&](Saddle &sys, int s, int n) {
    for (int i = 0; i < st->n_indic; i++) {
      const Deg &d = dset[i + 1];
      sys.solve(d, cen[0], st->deriv_w[s][i]);
      double scl = std::pow(dx, d[0]);
      scl *= std::pow(dy, d[1]);
      if (dim == 3) scl *= std::pow(dz, d[2]);
      for (int c = 0; c < n; c++) st->deriv_w[s][i][c] *= scl;
    }
  };
  int bad = 0;
  const Deg zero{0, 0, 0};
  (void)zero;

  // full (s=0) and central (s=1) stencils: solve the west face, map the others
  for (int s = 0; s < 2; s++) {
    const int n = s == 0 ? C : st->n_cells_ctr;
    const PtSet xs = cells_of(s, n);
    Saddle sys(dim, eps, polyDeg[s], xs);
    sys.solve_points(fq[0], FW(s, 0), LD);
    WeightMap(dim, false, xs, xs, fq[1], fq[0]).apply(FW(s, 1), FW(s, 0), LD);
    WeightMap(dim, false, xs, xs, fq[2], fq[0]).apply(FW(s, 2), FW(s, 0), LD);
    WeightMap(dim, false, xs, xs, fq[3], fq[2]).apply(FW(s, 3), FW(s, 2), LD);
    if (dim == 3) {
      WeightMap(dim, false, xs, xs, fq[4], fq[0]).apply(FW(s, 4), FW(s, 0), LD);
      WeightMap(dim, false, xs, xs, fq[5], fq[4]).apply(FW(s, 5), FW(s, 4), LD);
    }
    sys.solve_points(cq, &st->cell_w[s][0][0], LD);
    derivs(sys, s, n);
    bad |= sys.info();
  }

  // west-biased stencil (s=2): solve W, E, S faces, map N (and B, T)
  const int nb = st->n_cells_bias;
  const PtSet xw = cells_of(2, nb);
  {
    Saddle sys(dim, eps, polyDeg[2], xw);
    sys.solve_points(fq[0], FW(2, 0), LD);
    sys.solve_points(fq[1], FW(2, 1), LD);
    sys.solve_points(fq[2], FW(2, 2), LD);
    WeightMap(dim, false, xw, xw, fq[3], fq[2]).apply(FW(2, 3), FW(2, 2), LD);
    if (dim == 3) {
      WeightMap(dim, false, xw, xw, fq[4], fq[2]).apply(FW(2, 4), FW(2, 2), LD);
      WeightMap(dim, false, xw, xw, fq[5], fq[4]).apply(FW(2, 5), FW(2, 4), LD);
    }
    sys.solve_points(cq, &st->cell_w[2][0][0], LD);
    derivs(sys, 2, nb);
    bad |= sys.info();
  }
  // the other biased stencils are rotations/reflections of the west one: face f of
  // stencil s takes the west stencil's face src[s][f]
  static const int src[6][6] = {{1, 0, 2, 3, 4, 5},  // east
                                {3, 2, 0, 1, 4, 5},  // south
                                {2, 3, 1, 0, 4, 5},  // north
                                {5, 4, 2, 3, 0, 1},  // bottom
                                {4, 5, 2, 3, 1, 0}}; // top
  for (int s = 3; s < st->n_sub; s++) {
    const PtSet xs = cells_of(s, nb);
    for (int f = 0; f < 2 * dim; f++) {
      const int rf = src[s - 3][f];
      WeightMap(dim, false, xs, xw, fq[f], fq[rf]).apply(FW(s, f), FW(2, rf), LD);
    }
    WeightMap(dim, false, xs, xw, cq, cq).apply(&st->cell_w[s][0][0], &st->cell_w[2][0][0], LD);
    WeightMap dm(dim, false, xs, xw, cen, cen);
    for (int i = 0; i < st->n_indic; i++) dm.apply(st->deriv_w[s][i], st->deriv_w[2][i], LD);
  }
  return bad ? KFVM_ERR_LAPACK : KFVM_OK;
}

} // namespace kfvm
