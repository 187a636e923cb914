// oracle_weights.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).  Never linked
// into, imported by, or called from the product path.
//
// CPU restatement of the reference's stencil geometry and reconstruction-weight
// precompute (slug-cfd/kfvm-kokkos):
//   src/stencil/Stencil.cpp:47-156     Core::findStencil
//   src/stencil/Stencil.cpp:158-229    Core::findSubStencils
//   src/stencil/Stencil.cpp:281-846    Stencil::findWeights
//   src/stencil/ReconVectors.{H,cpp}   SE-kernel + monomial saddle system, LU
//   src/stencil/Monomials.cpp:14-58    monomials (incl. the argument swap at :29)
//   src/stencil/SEKernel.H:14-28       Gaussian kernel functionals
//   src/stencil/StencilSymmetry.cpp    reflection/rotation weight reuse
// The LU uses LAPACK dgetrf/dgetrs (the reference's ReconVectors.cpp:55-86);
// here they resolve to the OpenBLAS build bundled with scipy (scipy_ prefix).
//
// Parity status: the reference ships no golden weights; this restatement is
// pinned by the reference's own self-checks (polynomial reproduction as in its
// testPV, Stencil.cpp:250-277, and symmetry consistency) -- see tests/.

#include <cmath>
#include <cstdint>
#include <array>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

#include "../include/kfvm_b200.h"
#include "oracle.h"

extern "C" {
void scipy_dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info);
void scipy_dgetrs_(char *trans, int *n, int *nrhs, double *a, int *lda, int *ipiv,
                   double *b, int *ldb, int *info);
}

namespace orc {

// ---------------- quadrature tables (src/numeric/Numeric.cpp:9-46) ----------------
void quad_rule(int nq, double *ab, double *wt) {
  switch (nq) {
  case 1:
    ab[0] = 0.0;
    wt[0] = 1.0;
    break;
  case 2:
    ab[0] = -0.577350269189625764509148 / 2.0;
    ab[1] = 0.577350269189625764509148 / 2.0;
    wt[0] = 1.0 / 2.0;
    wt[1] = 1.0 / 2.0;
    break;
  default: // 3
    ab[0] = 0.0;
    ab[1] = -0.7745966692414833770358530 / 2.0;
    ab[2] = 0.7745966692414833770358530 / 2.0;
    wt[0] = 0.8888888888888888888888888 / 2.0;
    wt[1] = 0.5555555555555555555555555 / 2.0;
    wt[2] = 0.5555555555555555555555555 / 2.0;
    break;
  }
}

namespace {

typedef std::vector<double> dvec;

// ---------------- monomials (Monomials.cpp:14-32) ----------------
double mono_avg(int64_t p, double x) {
  double ub = std::pow(x + 0.5, p + 1) / (p + 1);
  double lb = std::pow(x - 0.5, p + 1) / (p + 1);
  return ub - lb;
}

// Reproduces Monomials.cpp:29 exactly, including the swapped arguments of the
// recursive call (x is passed as the derivative order, N-1 as the coordinate).
double mono_nd(int64_t p, int64_t N, double x) {
  if (N == 0) {
    return std::pow(x, p);
  } else if (N > p) {
    return 0.0;
  } else {
    return p * mono_nd(p - 1, static_cast<int64_t>(x), static_cast<double>(N - 1));
  }
}

int num_monos(int dim, int t) {
  return dim == 2 ? (t + 1) * (t + 2) / 2 : (t + 1) * (t + 2) * (t + 3) / 6;
}

// MonomialEnum (Monomials.cpp:34-58)
std::vector<std::array<int64_t, 3>> mono_enum(int dim, int tDeg) {
  std::vector<std::array<int64_t, 3>> deg;
  if (dim == 2) {
    for (int t = 0; t <= tDeg; t++)
      for (int i = 0; i <= t; i++) deg.push_back({i, t - i, 0});
  } else {
    for (int t = 0; t <= tDeg; t++)
      for (int i = 0; i <= t; i++)
        for (int j = 0; j <= t - i; j++) deg.push_back({i, j, t - i - j});
  }
  return deg;
}

// ---------------- SE kernel (SEKernel.H:14-28) ----------------
double se_avg(double eps, double x) {
  auto pf = std::sqrt(M_PI) / (2.0 * eps);
  return pf * (std::erf(eps * (x + 0.5)) - std::erf(eps * (x - 0.5)));
}

double se_nd(double eps, int64_t N, double x) {
  const double sgn = N % 2 == 0 ? 1.0 : -1.0,
               Hn = sgn * std::pow(eps, N) * std::hermite(N, eps * x);
  return Hn * std::exp(-eps * eps * x * x);
}

// ---------------- symmetry (StencilSymmetry.cpp) ----------------
enum Sym { RefX, RefY, RefZ, RefXY, RefXZ, RefYZ, RefXYZ, RotXY, RotXZ, RotYZ,
           RotXYm, RotXZm, RotYZm, SymNone };
const Sym kSyms[14] = {RefX, RefY, RefZ, RefXY, RefXZ, RefYZ, RefXYZ,
                       RotXY, RotXZ, RotYZ, RotXYm, RotXZm, RotYZm, SymNone};

bool deq(double a, double b) { return std::fabs(a - b) < 1.e-6; }

bool test_sym(int dim, Sym st, const double *p1, const double *p2) {
  const double x1 = p1[0], y1 = p1[1], z1 = p1[2], x2 = p2[0], y2 = p2[1], z2 = p2[2];
  if (dim == 2) {
    switch (st) {
    case RefX: return deq(x1, -x2) && deq(y1, y2);
    case RefY: return deq(x1, x2) && deq(y1, -y2);
    case RefXY: return deq(x1, -x2) && deq(y1, -y2);
    case RotXY: return deq(x1, -y2) && deq(y1, x2);
    case RotXYm: return deq(x1, y2) && deq(y1, -x2);
    default: return false;
    }
  }
  switch (st) {
  case RefX: return deq(x1, -x2) && deq(y1, y2) && deq(z1, z2);
  case RefY: return deq(x1, x2) && deq(y1, -y2) && deq(z1, z2);
  case RefZ: return deq(x1, x2) && deq(y1, y2) && deq(z1, -z2);
  case RefXY: return deq(x1, -x2) && deq(y1, -y2) && deq(z1, z2);
  case RefXZ: return deq(x1, -x2) && deq(y1, y2) && deq(z1, -z2);
  case RefYZ: return deq(x1, x2) && deq(y1, -y2) && deq(z1, -z2);
  case RefXYZ: return deq(x1, -x2) && deq(y1, -y2) && deq(z1, -z2);
  case RotXY: return deq(x1, -y2) && deq(y1, x2) && deq(z1, z2);
  case RotXZ: return deq(x1, -z2) && deq(y1, y2) && deq(z1, x2);
  case RotYZ: return deq(x1, x2) && deq(y1, -z2) && deq(z1, y2);
  case RotXYm: return deq(x1, y2) && deq(y1, -x2) && deq(z1, z2);
  case RotXZm: return deq(x1, z2) && deq(y1, y2) && deq(z1, -x2);
  case RotYZm: return deq(x1, x2) && deq(y1, z2) && deq(z1, -y2);
  default: return false;
  }
}

// A point set: coordinates as [n][3]
typedef std::vector<std::array<double, 3>> Pts;

// StencilSymmetry constructor (StencilSymmetry.cpp:203-283)
struct SymMapper {
  int nPts = 0, N = 0;
  std::vector<std::pair<int, Sym>> symMap;
  std::vector<std::vector<int>> idxMap;

  SymMapper(int dim, bool isSelf, const Pts &offD, const Pts &offR, const Pts &qD,
            const Pts &qR) {
    nPts = (int)qD.size();
    N = (int)offD.size();
    symMap.assign(nPts, {-1, SymNone});
    idxMap.assign(nPts, std::vector<int>(N, -1));
    std::vector<Sym> stenSym;
    for (int i = 0; i < 14; i++) {
      bool hasSym = true;
      for (int nD = 0; nD < N; nD++) {
        bool dSym = false;
        for (int nR = 0; nR < N; nR++) {
          dSym = test_sym(dim, kSyms[i], offD[nD].data(), offR[nR].data());
          if (dSym) break;
        }
        hasSym = hasSym && dSym;
      }
      if (hasSym) stenSym.push_back(kSyms[i]);
    }
    for (int nD = 0; nD < nPts; nD++) {
      int refLim = isSelf ? nD : nPts;
      for (int nR = 0; nR < refLim; nR++) {
        bool hasSym = false;
        for (size_t i = 0; i < stenSym.size(); i++) {
          hasSym = test_sym(dim, stenSym[i], qD[nD].data(), qR[nR].data());
          if (hasSym) {
            symMap[nD] = {nR, stenSym[i]};
            break;
          }
        }
        if (hasSym) break;
      }
    }
    for (int nP = 0; nP < nPts; nP++) {
      if (symMap[nP].first < 0) continue;
      for (int nD = 0; nD < N; nD++) {
        for (int nR = 0; nR < N; nR++) {
          if (test_sym(dim, symMap[nP].second, offD[nD].data(), offR[nR].data())) {
            idxMap[nP][nD] = nR;
            break;
          }
        }
      }
    }
  }
};

// Row-major weight block [rows][C] view into a larger array
struct WView {
  double *p;
  int ld;
  double &operator()(int r, int c) const { return p[r * ld + c]; }
};

// mapWeights (StencilSymmetry.H:69-87); returns number of missing symmetries
int map_weights(const SymMapper &sm, WView dst, WView ref) {
  int missing = 0;
  for (int nP = 0; nP < sm.nPts; nP++) {
    if (sm.symMap[nP].first >= 0) {
      for (int j = 0; j < sm.N; j++) dst(nP, j) = ref(sm.symMap[nP].first, sm.idxMap[nP][j]);
    } else {
      missing++;
    }
  }
  return missing;
}

// ---------------- ReconVectors (ReconVectors.{H,cpp}) ----------------
struct Recon {
  int dim, n, nMono, sys;
  double eps;
  Pts xs;
  std::vector<std::array<int64_t, 3>> deg;
  std::vector<double> C; // column-major sys x sys
  std::vector<int> ipiv;
  int info = 0;

  Recon(int dim_, double eps_, int monoDeg, const Pts &xs_)
      : dim(dim_), n((int)xs_.size()), eps(eps_), xs(xs_) {
    deg = mono_enum(dim, monoDeg);
    nMono = (int)deg.size();
    sys = n + nMono;
    C.assign((size_t)sys * sys, 0.0);
    ipiv.assign(sys, 0);
    auto c = [&](int i, int j) -> double & { return C[(size_t)j * sys + i]; };
    for (int i = 0; i < n; i++) {
      for (int j = 0; j < n; j++) {
        double dx = xs[i][0] - xs[j][0], dy = xs[i][1] - xs[j][1], dz = xs[i][2] - xs[j][2];
        c(i, j) = dim == 2 ? se_avg(eps, dx) * se_avg(eps, dy)
                           : se_avg(eps, dx) * se_avg(eps, dy) * se_avg(eps, dz);
      }
    }
    for (int i = 0; i < n; i++) {
      for (int j = 0; j < nMono; j++) {
        c(i, j + n) = dim == 2 ? mono_avg(deg[j][0], xs[i][0]) * mono_avg(deg[j][1], xs[i][1])
                               : mono_avg(deg[j][0], xs[i][0]) * mono_avg(deg[j][1], xs[i][1]) *
                                     mono_avg(deg[j][2], xs[i][2]);
        c(j + n, i) = c(i, j + n);
      }
    }
    for (int i = n; i < sys; i++)
      for (int j = n; j < sys; j++) c(i, j) = 0.0;
    int M = sys;
    scipy_dgetrf_(&M, &M, C.data(), &M, ipiv.data(), &info);
  }

  // recVec (ReconVectors.H:95-113)
  void rec_vec(const int64_t *Nd, const double *q, double *rec) {
    std::vector<double> S(sys, 0.0);
    for (int i = 0; i < n; i++) {
      double dx = q[0] - xs[i][0], dy = q[1] - xs[i][1], dz = q[2] - xs[i][2];
      S[i] = dim == 2 ? se_nd(eps, Nd[0], dx) * se_nd(eps, Nd[1], dy)
                      : se_nd(eps, Nd[0], dx) * se_nd(eps, Nd[1], dy) * se_nd(eps, Nd[2], dz);
    }
    for (int i = 0; i < nMono; i++) {
      S[i + n] = dim == 2 ? mono_nd(deg[i][0], Nd[0], q[0]) * mono_nd(deg[i][1], Nd[1], q[1])
                          : mono_nd(deg[i][0], Nd[0], q[0]) * mono_nd(deg[i][1], Nd[1], q[1]) *
                                mono_nd(deg[i][2], Nd[2], q[2]);
    }
    char trans = 'N';
    int M = sys, one = 1, inf = 0;
    scipy_dgetrs_(&trans, &M, &one, C.data(), &M, ipiv.data(), S.data(), &M, &inf);
    if (inf != 0) info = inf;
    for (int j = 0; j < n; j++) rec[j] = S[j];
  }

  // recVecs over a set of query points (ReconVectors.H:120-145)
  void rec_vecs(const int64_t *Nd, const Pts &q, WView wts) {
    SymMapper sm(dim, true, xs, xs, q, q);
    std::vector<double> rec(n, 0.0);
    for (int nQ = 0; nQ < (int)q.size(); nQ++) {
      if (sm.symMap[nQ].first < 0) {
        rec_vec(Nd, q[nQ].data(), rec.data());
        for (int j = 0; j < n; j++) wts(nQ, j) = rec[j];
      } else {
        for (int j = 0; j < n; j++) wts(nQ, j) = wts(sm.symMap[nQ].first, sm.idxMap[nQ][j]);
      }
    }
  }
};

} // namespace

// ---------------- geometry (Stencil.cpp:47-229) ----------------
static void find_stencil(int dim, kfvm_stencil *st) {
  const int rad = KFVM_RAD;
  int64_t *l = st->off[0], *t = st->off[1], *tt = st->off[2];
  int nC = 0;
  if (dim == 2) {
    double mjRsq = rad * rad;
    nC = 1;
    l[0] = 0;
    t[0] = 0;
    tt[0] = 0;
    auto add = [&](int64_t a, int64_t b) {
      l[nC] = a;
      t[nC] = b;
      tt[nC] = 0;
      nC++;
    };
    for (int nL = 1; nL <= rad; nL++) {
      add(-nL, 0);
      add(nL, 0);
      add(0, -nL);
      add(0, nL);
      for (int nR = 1; nR <= nL; nR++) {
        double rsq = 2.0 * nR * nR;
        int64_t lyr = (int64_t)std::ceil(std::sqrt(rsq));
        if (rsq <= mjRsq && lyr == nL) {
          add(-nR, -nR);
          add(-nR, nR);
          add(nR, -nR);
          add(nR, nR);
        }
      }
      for (int i = 2; i <= rad; i++) {
        for (int j = 1; j < i; j++) {
          double cx = i, cy = j, rsq = cx * cx + cy * cy;
          int64_t lyr = (int64_t)std::ceil(std::sqrt(rsq));
          if (rsq <= mjRsq && lyr == nL) {
            add(-i, j);
            add(-i, -j);
            add(i, j);
            add(i, -j);
            add(-j, i);
            add(-j, -i);
            add(j, i);
            add(j, -i);
          }
        }
      }
    }
  } else {
    int64_t mjRsq = rad * rad, rm = rad - 1;
    for (int64_t i = -rm; i <= rm; i++)
      for (int64_t j = -rm; j <= rm; j++)
        for (int64_t k = -rm; k <= rm; k++)
          if (i * i + j * j + k * k <= rm * rm) {
            l[nC] = i;
            t[nC] = j;
            tt[nC] = k;
            nC++;
          }
    for (int64_t i = -rad; i <= rad; i++)
      for (int64_t j = -rad; j <= rad; j++)
        for (int64_t k = -rad; k <= rad; k++) {
          int64_t rsq = i * i + j * j + k * k;
          if (rsq > rm * rm && rsq <= mjRsq) {
            l[nC] = i;
            t[nC] = j;
            tt[nC] = k;
            nC++;
          }
        }
  }
  st->n_cells = nC;

  auto c2i = [&](int64_t i, int64_t j, int64_t k) -> int64_t {
    for (int n = 0; n < st->n_cells; n++)
      if (i == l[n] && j == t[n] && (dim == 2 || k == tt[n])) return n;
    return -1;
  };
  if (dim == 2) {
    int nN = 0, nS = 0, nE = 0, nW = 0;
    for (int h = 0; h <= rad; h++) {
      st->sub_idx[0][nW++] = c2i(-h, 0, 0);
      st->sub_idx[1][nE++] = c2i(h, 0, 0);
      st->sub_idx[2][nS++] = c2i(0, -h, 0);
      st->sub_idx[3][nN++] = c2i(0, h, 0);
    }
    for (int h = 0; h <= rad; h++) {
      for (int lo = 1; lo <= h; lo++) {
        int64_t idx = c2i(-h, -lo, 0), idxp = c2i(-h, lo, 0);
        if (idx >= 0) {
          st->sub_idx[0][nW++] = idx;
          st->sub_idx[0][nW++] = idxp;
          st->sub_idx[1][nE++] = c2i(h, -lo, 0);
          st->sub_idx[1][nE++] = c2i(h, lo, 0);
          st->sub_idx[2][nS++] = c2i(-lo, -h, 0);
          st->sub_idx[2][nS++] = c2i(lo, -h, 0);
          st->sub_idx[3][nN++] = c2i(-lo, h, 0);
          st->sub_idx[3][nN++] = c2i(lo, h, 0);
        }
      }
    }
  } else {
    int cnt[6] = {0, 0, 0, 0, 0, 0};
    for (int n = 0; n < st->n_cells; n++) {
      int64_t a = l[n], b = t[n], c = tt[n];
      if (-a >= std::abs(b) && -a >= std::abs(c)) st->sub_idx[0][cnt[0]++] = n;
      if (a >= std::abs(b) && a >= std::abs(c)) st->sub_idx[1][cnt[1]++] = n;
      if (-b >= std::abs(a) && -b >= std::abs(c)) st->sub_idx[2][cnt[2]++] = n;
      if (b >= std::abs(a) && b >= std::abs(c)) st->sub_idx[3][cnt[3]++] = n;
      if (-c >= std::abs(a) && -c >= std::abs(b)) st->sub_idx[4][cnt[4]++] = n;
      if (c >= std::abs(a) && c >= std::abs(b)) st->sub_idx[5][cnt[5]++] = n;
    }
  }
}

// Stencil::findWeights (Stencil.cpp:281-846).  Returns 0, or KFVM_ERR_LAPACK.
int build_stencil(const kfvm_config *cfg, kfvm_stencil *st) {
  std::memset(st, 0, sizeof(*st));
  const int dim = cfg->dim, nq = cfg->nq;
  st->dim = dim;
  st->nq = nq;
  find_stencil(dim, st);
  const int C = st->n_cells;
  st->n_cells_ctr = dim == 2 ? 5 : 7;
  st->n_cells_bias = dim == 2 ? 5 : 11;
  st->n_sub = dim == 2 ? 6 : 8;
  st->n_bias = dim == 2 ? 4 : 6;
  const int nDeriv = dim == 2 ? 2 : 3;
  st->n_indic = num_monos(dim, nDeriv) - 1;
  st->nqf = dim == 2 ? nq : nq * nq;
  st->nqc = dim == 2 ? nq * nq : nq * nq * nq;
  const int monoDeg[3] = {3, 1, 1};
  auto derivSet = mono_enum(dim, nDeriv);

  // geometry (Geometry.H:27-43): the whole domain's extents over its cells, nx nb
  auto nbk = [&](int d) { return cfg->nb[d] > 0 ? cfg->nb[d] : 1; };
  const double dx = (cfg->xup - cfg->xlo) / (cfg->nx * nbk(0)), dy = (cfg->yup - cfg->ylo) / (cfg->ny * nbk(1)),
               dz = (cfg->zup - cfg->zlo) / (cfg->nz * nbk(2));
  const double eps = 1.0 / (cfg->lfac * std::sqrt(2.0));

  double ab[3], wt[3];
  quad_rule(nq, ab, wt);
  const int nqf = st->nqf, nqc = st->nqc;
  Pts fW(nqf), fE(nqf), fS(nqf), fN(nqf), fB(nqf), fT(nqf), cq(nqc), dq(1);
  for (int idx = 0; idx < nqf; idx++) {
    double f1 = dim == 2 ? ab[idx] : ab[idx / nq];
    double f2 = dim == 2 ? 0.0 : ab[idx % nq];
    fW[idx] = {-0.5, f1, f2};
    fE[idx] = {0.5, f1, f2};
    fS[idx] = {f1, -0.5, f2};
    fN[idx] = {f1, 0.5, f2};
    fB[idx] = {f1, f2, -0.5};
    fT[idx] = {f1, f2, 0.5};
  }
  for (int idx = 0; idx < nqc; idx++) {
    if (dim == 2)
      cq[idx] = {ab[idx / nq], ab[idx % nq], 0.0};
    else
      cq[idx] = {ab[idx / (nq * nq)], ab[(idx / nq) % nq], ab[idx % nq]};
  }
  dq[0] = {0.0, 0.0, 0.0};
  const Pts *faceQ[6] = {&fW, &fE, &fS, &fN, &fB, &fT};

  auto face = [&](int s, int f) { return WView{&st->face_w[s][f][0][0], KFVM_MAX_CELLS}; };
  auto cellv = [&](int s) { return WView{&st->cell_w[s][0][0], KFVM_MAX_CELLS}; };
  auto sub_pts = [&](int s, int n) {
    Pts p(n);
    for (int i = 0; i < n; i++) {
      int idx = s < 2 ? i : (int)st->sub_idx[s - 2][i];
      p[i] = {(double)st->off[0][idx], (double)st->off[1][idx],
              dim == 3 ? (double)st->off[2][idx] : 0.0};
    }
    return p;
  };
  int64_t point0[3] = {0, 0, 0};
  int err = 0;
  auto derivs = [&](Recon &rv, int s, int subSize) {
    for (int nI = 0; nI < st->n_indic; nI++) {
      double *dW = st->deriv_w[s][nI];
      int64_t Nd[3] = {derivSet[nI + 1][0], derivSet[nI + 1][1], derivSet[nI + 1][2]};
      double q0[3] = {0.0, 0.0, 0.0};
      rv.rec_vec(Nd, q0, dW);
      double scl = std::pow(dx, derivSet[nI + 1][0]);
      scl *= std::pow(dy, derivSet[nI + 1][1]);
      if (dim == 3) scl *= std::pow(dz, derivSet[nI + 1][2]);
      for (int nC = 0; nC < subSize; nC++) dW[nC] *= scl;
    }
  };

  // centered substencils (Stencil.cpp:346-430)
  for (int nS = 0; nS < 2; nS++) {
    int subSize = nS == 0 ? C : st->n_cells_ctr;
    Pts xs = sub_pts(nS, subSize);
    Recon rv(dim, eps, monoDeg[nS], xs);
    if (rv.info) err = KFVM_ERR_LAPACK;
    rv.rec_vecs(point0, fW, face(nS, 0));
    map_weights(SymMapper(dim, false, xs, xs, fE, fW), face(nS, 1), face(nS, 0));
    map_weights(SymMapper(dim, false, xs, xs, fS, fW), face(nS, 2), face(nS, 0));
    map_weights(SymMapper(dim, false, xs, xs, fN, fS), face(nS, 3), face(nS, 2));
    if (dim == 3) {
      map_weights(SymMapper(dim, false, xs, xs, fB, fW), face(nS, 4), face(nS, 0));
      map_weights(SymMapper(dim, false, xs, xs, fT, fB), face(nS, 5), face(nS, 4));
    }
    rv.rec_vecs(point0, cq, cellv(nS));
    derivs(rv, nS, subSize);
    if (rv.info) err = KFVM_ERR_LAPACK;
  }

  // biased substencils (Stencil.cpp:432-820)
  {
    const int subSize = st->n_cells_bias;
    Pts xw = sub_pts(2, subSize);
    Recon rv(dim, eps, monoDeg[2], xw);
    if (rv.info) err = KFVM_ERR_LAPACK;
    rv.rec_vecs(point0, fW, face(2, 0));
    rv.rec_vecs(point0, fE, face(2, 1));
    rv.rec_vecs(point0, fS, face(2, 2));
    map_weights(SymMapper(dim, false, xw, xw, fN, fS), face(2, 3), face(2, 2));
    if (dim == 3) {
      map_weights(SymMapper(dim, false, xw, xw, fB, fS), face(2, 4), face(2, 2));
      map_weights(SymMapper(dim, false, xw, xw, fT, fB), face(2, 5), face(2, 4));
    }
    rv.rec_vecs(point0, cq, cellv(2));
    derivs(rv, 2, subSize);
    if (rv.info) err = KFVM_ERR_LAPACK;

    // destination face f of substencil s <- reference face rf of the west substencil
    // (the table of StencilSymmetry constructions in Stencil.cpp:492-820)
    static const int map2d[4][4] = {
        {1, 0, 2, 3}, // east:  W<-E, E<-W, S<-S, N<-N
        {3, 2, 0, 1}, // south: W<-N, E<-S, S<-W, N<-E
        {2, 3, 1, 0}, // north: W<-S, E<-N, S<-E, N<-W
        {0, 0, 0, 0}};
    static const int map3d[6][6] = {
        {1, 0, 2, 3, 4, 5}, // east
        {3, 2, 0, 1, 4, 5}, // south
        {2, 3, 1, 0, 4, 5}, // north
        {5, 4, 2, 3, 0, 1}, // bottom: W<-T, E<-B, S<-S, N<-N, B<-W, T<-E
        {4, 5, 2, 3, 1, 0}, // top:    W<-B, E<-T, S<-S, N<-N, B<-E, T<-W
        {0, 0, 0, 0, 0, 0}};
    for (int nS = 3; nS < st->n_sub; nS++) {
      Pts xs = sub_pts(nS, subSize);
      for (int f = 0; f < 2 * dim; f++) {
        int rf = dim == 2 ? map2d[nS - 3][f] : map3d[nS - 3][f];
        map_weights(SymMapper(dim, false, xs, xw, *faceQ[f], *faceQ[rf]), face(nS, f),
                    face(2, rf));
      }
      map_weights(SymMapper(dim, false, xs, xw, cq, cq), cellv(nS), cellv(2));
      SymMapper dsm(dim, false, xs, xw, dq, dq);
      for (int nI = 0; nI < st->n_indic; nI++) {
        if (dsm.symMap[0].first >= 0)
          for (int j = 0; j < dsm.N; j++) st->deriv_w[nS][nI][j] = st->deriv_w[2][nI][dsm.idxMap[0][j]];
      }
    }
  }
  return err ? KFVM_ERR_LAPACK : 0;
}

} // namespace orc
