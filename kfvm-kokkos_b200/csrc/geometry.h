// geometry.h -- cell size and block origin of a (possibly decomposed) domain, as
// the reference's Geometry computes them (src/Geometry.H:28-31): the extents in
// the configuration are the whole domain's, nx etc. one block's cells, so
//   dx = (xup - xlo) / (nx nb[0]),   this block's xlo = xlo + dx (block[0] nx).
// With nb = 1 these are (xup - xlo) / nx and xlo exactly.
#pragma once

#include <cstdint>

#include "../../include/kfvm_b200.h"

namespace kfvm {

inline int cfg_nb(const kfvm_config *c, int d) { return c->nb[d] > 0 ? c->nb[d] : 1; }

inline int64_t cfg_n(const kfvm_config *c, int d) { return d == 0 ? c->nx : (d == 1 ? c->ny : (c->dim == 3 ? c->nz : 1)); }

inline double cfg_dx(const kfvm_config *c, int d) {
  const double lo = d == 0 ? c->xlo : (d == 1 ? c->ylo : c->zlo);
  const double up = d == 0 ? c->xup : (d == 1 ? c->yup : c->zup);
  return (up - lo) / (double)(cfg_n(c, d) * (int64_t)cfg_nb(c, d));
}

// first face of this block along axis d
inline double cfg_lo(const kfvm_config *c, int d) {
  const double lo = d == 0 ? c->xlo : (d == 1 ? c->ylo : c->zlo);
  const int64_t bLo = (int64_t)(cfg_nb(c, d) > 1 ? c->block[d] : 0) * cfg_n(c, d);
  return bLo == 0 ? lo : lo + cfg_dx(c, d) * (double)bLo;
}

// global index of this block's first cell along axis d
inline int64_t cfg_offset(const kfvm_config *c, int d) {
  return (int64_t)(cfg_nb(c, d) > 1 ? c->block[d] : 0) * cfg_n(c, d);
}

} // namespace kfvm
