// TEST INFRASTRUCTURE ONLY: the PDI stand-in of the reference build (see pdi.h).
// Compiled with the problem's Definitions.H so that the variable count is known.
//
// Checkpoint file written for "write_ckpt_data" (little-endian), at the
// reference's chosen .h5 path with ".raw" appended:
//   char[8] "KFVMREF1"; int32 step, nvars, dim; int32 ncell_l[3], nghost[3];
//   double time, dt;
//   double cons_field[nvars][nz+2gz][ny+2gy][nx+2gx]   (x fastest: the
//          reference's LayoutLeft host mirror (i, j, k, v))
//   double weno_field[2][nz][ny][nx]
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include <Definitions.H>

#include "physics/EquationTypes.H"
#include "pdi.h"

namespace {
int g_ncell[3] = {1, 1, 1};
int g_nghost[3] = {0, 0, 0};

struct Item {
  const char *name;
  const void *data;
};

const void *find(Item *items, int n, const char *name) {
  for (int i = 0; i < n; i++)
    if (std::strcmp(items[i].name, name) == 0) return items[i].data;
  return nullptr;
}
} // namespace

PDI_status_t PDI_init(PC_tree_t) { return 0; }
PDI_status_t PDI_finalize(void) { return 0; }

PDI_status_t PDI_multi_expose(const char *event_name, const char *name, const void *data,
                              PDI_inout_t access, ...) {
  Item items[32];
  int n = 0;
  items[n++] = Item{name, data};
  (void)access;
  va_list ap;
  va_start(ap, access);
  for (;;) {
    const char *nm = va_arg(ap, const char *);
    if (nm == nullptr || n >= 32) break;
    const void *d = va_arg(ap, const void *);
    (void)va_arg(ap, int);
    items[n++] = Item{nm, d};
  }
  va_end(ap);

  const std::string ev(event_name ? event_name : "");
  if (ev.empty()) {
    if (auto p = static_cast<const int *>(find(items, n, "ncell_l")))
      std::memcpy(g_ncell, p, sizeof(g_ncell));
    if (auto p = static_cast<const int *>(find(items, n, "nghost")))
      std::memcpy(g_nghost, p, sizeof(g_nghost));
    return 0;
  }
  if (ev == "read_ckpt_data") {
    std::fprintf(stderr, "PDI stand-in: restart files are not supported\n");
    return 1;
  }
  if (ev != "write_ckpt_data") return 0;  // plot and statistics files are not needed

  const char *fname = static_cast<const char *>(find(items, n, "filename"));
  const int *step = static_cast<const int *>(find(items, n, "time_step"));
  const double *time = static_cast<const double *>(find(items, n, "time"));
  const double *dt = static_cast<const double *>(find(items, n, "time_step_size"));
  const double *cons = static_cast<const double *>(find(items, n, "cons_field"));
  const double *weno = static_cast<const double *>(find(items, n, "weno_field"));
  if (!fname || !step || !time || !dt || !cons || !weno) return 1;

  const int32_t nv = int32_t(KFVM::NUM_EQN_VARS[eqType]);
  const int32_t dim = SPACE_DIM;
  std::size_t halo = 1, cells = 1;
  for (int d = 0; d < 3; d++) {
    halo *= std::size_t(g_ncell[d] + 2 * g_nghost[d]);
    cells *= std::size_t(g_ncell[d]);
  }
  std::string out = std::string(fname) + ".raw";
  FILE *f = std::fopen(out.c_str(), "wb");
  if (!f) return 1;
  std::fwrite("KFVMREF1", 1, 8, f);
  int32_t hdr[9] = {*step, nv, dim, g_ncell[0], g_ncell[1], g_ncell[2],
                    g_nghost[0], g_nghost[1], g_nghost[2]};
  std::fwrite(hdr, sizeof(int32_t), 9, f);
  std::fwrite(time, sizeof(double), 1, f);
  std::fwrite(dt, sizeof(double), 1, f);
  std::fwrite(cons, sizeof(double), halo * nv, f);
  std::fwrite(weno, sizeof(double), cells * 2, f);
  std::fclose(f);
  return 0;
}
