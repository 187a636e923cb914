// plotfile.cpp -- plot and checkpoint files in the reference's XDMF layout, with
// raw little-endian binary datasets where the reference writes HDF5 through PDI
// (src/io/WriterPDI.cpp:100-330, user/pdi_euler_xdmf.yml, user/pdi_mhd_glm_xdmf.yml).
//
// One file set per output: <base>_<num:07d>.xmf (XDMF 2, a 3DRectMesh of nodal
// coordinates, one cell-centred attribute per dataset), <base>_<num:07d>.<name>.bin
// per dataset (FP64, [z][y][x] with x fastest, as the HDF5 datasets are) and
// <base>_<num:07d>.meta (time, time step, time step size, gamma and the grid, the
// scalars the reference stores in the HDF5 file).  Datasets:
//   conserved   dens momx momy momz etot (+ magx magy magz psi for GLM-MHD)
//   plot only   velx vely velz eint pres (GLM-MHD: eint prsg prsb; SRHydro: rho
//               velx vely velz lorz pres), as AuxVars computes them
//               (src/physics/hydro/Hydro_K.H:66-97, src/physics/mhd_glm/MHD_GLM_K.H:71-106,
//               src/physics/srhydro/SRHydro_K.H:59-88; WriterPDI.cpp:268-278)
//   both        weno (WENO applied, 0 or 1) and fomx (the positivity theta), the
//               two components of the reference's wenoFlag view
// Host code only; the solver-level calls in capi.cu download the state first.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "geometry.h"
#include "../../include/kfvm_b200.h"
#include "sr_eos.h"

namespace kfvm {
int set_last_error(int code, const std::string &msg);
}

namespace {

struct Grid3 {
  int64_t nx, ny, nz, n;
  int nv;
  bool glm, sr;
};

Grid3 grid_of(const kfvm_config *c) {
  Grid3 g;
  g.nx = c->nx;
  g.ny = c->ny;
  g.nz = c->dim == 3 ? c->nz : 1;
  g.n = g.nx * g.ny * g.nz;
  g.glm = c->eq == KFVM_EQ_MHD_GLM;
  g.sr = c->eq == KFVM_EQ_SRHYDRO;
  g.nv = g.glm ? 9 : 5;
  return g;
}

const char *const kConsNames[9] = {"dens", "momx", "momy", "momz", "etot", "magx", "magy", "magz", "psi"};

std::string stem_of(const char *dir, const char *base, int32_t num) {
  char b[32];
  std::snprintf(b, sizeof(b), "_%07d", (int)num);
  return (std::filesystem::path(dir) / (std::string(base) + b)).string();
}

bool write_raw(const std::string &path, const double *p, size_t count) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const size_t w = std::fwrite(p, sizeof(double), count, f);
  return std::fclose(f) == 0 && w == count;
}

bool read_raw(const std::string &path, double *p, size_t count) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  const size_t r = std::fread(p, sizeof(double), count, f);
  // the file must hold exactly count values
  const bool atEnd = std::fgetc(f) == EOF;
  std::fclose(f);
  return r == count && atEnd;
}

std::string file_name(const std::string &path) { return std::filesystem::path(path).filename().string(); }

void attr_scalar(std::ostream &o, const Grid3 &g, const std::string &stem, const char *name) {
  o << "      <Attribute Name=\"" << name << "\" AttributeType=\"Scalar\" Center=\"Cell\">\n"
    << "        <DataItem Format=\"Binary\" Endian=\"Little\" NumberType=\"Float\" Precision=\"8\" Dimensions=\""
    << g.nz << " " << g.ny << " " << g.nx << "\">\n"
    << "          " << file_name(stem) << "." << name << ".bin\n"
    << "        </DataItem>\n      </Attribute>\n";
}

void attr_vector(std::ostream &o, const Grid3 &g, const std::string &stem, const char *name, const char *x,
                 const char *y, const char *z) {
  o << "      <Attribute Name=\"" << name << "\" AttributeType=\"Vector\" Center=\"Cell\">\n"
    << "        <DataItem ItemType=\"Function\" Function=\"JOIN($0, $1, $2)\" Dimensions=\"" << g.nz << " "
    << g.ny << " " << g.nx << " 3\">\n";
  for (const char *c : {x, y, z})
    o << "          <DataItem Format=\"Binary\" Endian=\"Little\" NumberType=\"Float\" Precision=\"8\" "
         "Dimensions=\""
      << g.nz << " " << g.ny << " " << g.nx << "\">\n"
      << "            " << file_name(stem) << "." << c << ".bin\n"
      << "          </DataItem>\n";
  o << "        </DataItem>\n      </Attribute>\n";
}

int plotfile_write(const kfvm_config *cfg, const char *dir, const char *base, int32_t num, int32_t ckpt,
                   int32_t time_step, double time, double dt, const double *u, const uint8_t *weno,
                   const double *theta) {
  if (!cfg || !dir || !base || !u || !weno || !theta || num < 0)
    return kfvm::set_last_error(KFVM_ERR_ARG, "kfvm_plotfile_write: bad argument");
  const Grid3 g = grid_of(cfg);
  if (g.n <= 0) return kfvm::set_last_error(KFVM_ERR_ARG, "kfvm_plotfile_write: empty grid");
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  if (ec) return kfvm::set_last_error(KFVM_ERR_IO, std::string("cannot create ") + dir + ": " + ec.message());
  const std::string stem = stem_of(dir, base, num);
  const size_t n = (size_t)g.n;
  bool ok = true;
  // nodal coordinates (WriterPDI.cpp:38-52; z uses dmin in 2D)
  const double dx = kfvm::cfg_dx(cfg, 0), dy = kfvm::cfg_dx(cfg, 1);
  const double dz = cfg->dim == 3 ? kfvm::cfg_dx(cfg, 2) : std::fmin(dx, dy);
  const double x0 = kfvm::cfg_lo(cfg, 0), y0 = kfvm::cfg_lo(cfg, 1), z0 = cfg->dim == 3 ? kfvm::cfg_lo(cfg, 2) : 0.0;
  std::vector<double> xc(g.nx + 1), yc(g.ny + 1), zc(g.nz + 1);
  for (int64_t i = 0; i <= g.nx; i++) xc[i] = (double)i * dx + x0;
  for (int64_t j = 0; j <= g.ny; j++) yc[j] = (double)j * dy + y0;
  for (int64_t k = 0; k <= g.nz; k++) zc[k] = (double)k * dz + z0;
  ok = ok && write_raw(stem + ".xcoord.bin", xc.data(), xc.size());
  ok = ok && write_raw(stem + ".ycoord.bin", yc.data(), yc.size());
  ok = ok && write_raw(stem + ".zcoord.bin", zc.data(), zc.size());
  for (int v = 0; v < g.nv && ok; v++) ok = write_raw(stem + "." + kConsNames[v] + ".bin", u + (size_t)v * n, n);
  {
    std::vector<double> w(n);
    for (size_t c = 0; c < n; c++) w[c] = weno[c] ? 1.0 : 0.0;
    ok = ok && write_raw(stem + ".weno.bin", w.data(), n);
    ok = ok && write_raw(stem + ".fomx.bin", theta, n);
  }
  if (!ckpt && ok && g.sr) {
    // AuxVars<SRHydro>: the primitives by the pressure recovery
    std::vector<double> V(6 * n);
    for (size_t c = 0; c < n; c++) {
      double U[5], v[6];
      for (int q = 0; q < 5; q++) U[q] = u[(size_t)q * n + c];
      kfvm::sr::cons2prim(cfg->gamma, U, v);
      for (int q = 0; q < 6; q++) V[(size_t)q * n + c] = v[q];
    }
    const char *an[6] = {".rho.bin", ".velx.bin", ".vely.bin", ".velz.bin", ".pres.bin", ".lorz.bin"};
    for (int q = 0; q < 6 && ok; q++) ok = write_raw(stem + an[q], V.data() + (size_t)q * n, n);
  } else if (!ckpt && ok) {
    // auxiliary variables (AuxVars<Hydro> / AuxVars<MHD_GLM>)
    const double gm = cfg->gamma;
    std::vector<double> a(n);
    for (int comp = 0; comp < 3 && ok; comp++) {
      for (size_t c = 0; c < n; c++) a[c] = u[(size_t)(1 + comp) * n + c] / u[c];
      const char *vn = comp == 0 ? ".velx.bin" : comp == 1 ? ".vely.bin" : ".velz.bin";
      ok = write_raw(stem + vn, a.data(), n);
    }
    std::vector<double> ei(n), pb(g.glm ? n : 0);
    for (size_t c = 0; c < n; c++) {
      const double rho = u[c], mx = u[n + c], my = u[2 * n + c], mz = u[3 * n + c], et = u[4 * n + c];
      const double ekin = 0.5 * (mx * mx + my * my + mz * mz) / rho;
      if (g.glm) {
        const double bx = u[5 * n + c], by = u[6 * n + c], bz = u[7 * n + c], psi = u[8 * n + c];
        pb[c] = 0.5 * (bx * bx + by * by + bz * bz);
        ei[c] = et - pb[c] - ekin - 0.5 * psi * psi;
      } else {
        ei[c] = et - ekin;
      }
    }
    ok = ok && write_raw(stem + ".eint.bin", ei.data(), n);
    for (size_t c = 0; c < n; c++) a[c] = (gm - 1.0) * ei[c];
    ok = ok && write_raw(stem + (g.glm ? ".prsg.bin" : ".pres.bin"), a.data(), n);
    if (g.glm) ok = ok && write_raw(stem + ".prsb.bin", pb.data(), n);
  }
  if (!ok) return kfvm::set_last_error(KFVM_ERR_IO, "kfvm_plotfile_write: cannot write " + stem + ".*.bin");
  {
    // scalars and grid, read back by kfvm_plotfile_read
    std::ofstream m(stem + ".meta", std::ios::trunc);
    char b[512];
    std::snprintf(b, sizeof(b),
                  "kind %s\ndim %d\neq %d\nnx %lld\nny %lld\nnz %lld\nnv %d\ntime %.17g\ntime_step %d\n"
                  "time_step_size %.17g\ngamma %.17g\n",
                  ckpt ? "ckpt" : "plot", cfg->dim, cfg->eq, (long long)g.nx, (long long)g.ny, (long long)g.nz, g.nv,
                  time, (int)time_step, dt, cfg->gamma);
    m << b;
    if (!m) return kfvm::set_last_error(KFVM_ERR_IO, "kfvm_plotfile_write: cannot write " + stem + ".meta");
  }
  {
    // XDMF description (WriterPDI::writeXML, WriterPDI.cpp:170-330)
    std::ofstream o(stem + ".xmf", std::ios::trunc);
    char tb[64];
    std::snprintf(tb, sizeof(tb), "%.17g", time);
    o << "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n  <Domain>\n"
      << "    <Grid Name=\"Structured Grid\" GridType=\"Uniform\">\n"
      << "      <Time Value=\"" << tb << "\" />\n"
      << "      <Topology TopologyType=\"3DRectMesh\" NumberOfElements=\"" << (g.nz + 1) << " " << (g.ny + 1) << " "
      << (g.nx + 1) << "\"/>\n"
      << "      <Geometry GeometryType=\"VxVyVz\">\n";
    const int64_t nn[3] = {g.nx + 1, g.ny + 1, g.nz + 1};
    const char *cn[3] = {"xcoord", "ycoord", "zcoord"}, *vn[3] = {"Vx", "Vy", "Vz"};
    for (int d = 0; d < 3; d++)
      o << "        <DataItem Name=\"" << vn[d] << "\" Dimensions=\"" << nn[d]
        << "\" NumberType=\"Float\" Precision=\"8\" Format=\"Binary\" Endian=\"Little\">\n"
        << "          " << file_name(stem) << "." << cn[d] << ".bin\n        </DataItem>\n";
    o << "      </Geometry>\n";
    attr_scalar(o, g, stem, "dens");
    attr_vector(o, g, stem, "mom", "momx", "momy", "momz");
    if (g.glm) attr_vector(o, g, stem, "B", "magx", "magy", "magz");
    attr_scalar(o, g, stem, "etot");
    if (g.glm) attr_scalar(o, g, stem, "psi");
    if (!ckpt && g.sr) {
      attr_scalar(o, g, stem, "rho");
      attr_vector(o, g, stem, "vel", "velx", "vely", "velz");
      attr_scalar(o, g, stem, "lorz");
      attr_scalar(o, g, stem, "pres");
    } else if (!ckpt) {
      attr_vector(o, g, stem, "vel", "velx", "vely", "velz");
      attr_scalar(o, g, stem, "eint");
      if (g.glm) {
        attr_scalar(o, g, stem, "prsg");
        attr_scalar(o, g, stem, "prsb");
      } else {
        attr_scalar(o, g, stem, "pres");
      }
    }
    attr_scalar(o, g, stem, "weno");
    attr_scalar(o, g, stem, "fomx");
    o << "    </Grid>\n  </Domain>\n</Xdmf>\n";
    if (!o) return kfvm::set_last_error(KFVM_ERR_IO, "kfvm_plotfile_write: cannot write " + stem + ".xmf");
  }
  return KFVM_OK;
}

int plotfile_read(const kfvm_config *cfg, const char *xmf_path, double *u, uint8_t *weno, double *theta,
                  int32_t *time_step, double *time, double *dt) {
  if (!cfg || !xmf_path || !u || !weno || !theta || !time_step || !time || !dt)
    return kfvm::set_last_error(KFVM_ERR_ARG, "kfvm_plotfile_read: bad argument");
  std::string stem(xmf_path);
  if (stem.size() > 4 && stem.compare(stem.size() - 4, 4, ".xmf") == 0) stem.resize(stem.size() - 4);
  const Grid3 g = grid_of(cfg);
  std::ifstream m(stem + ".meta");
  if (!m) return kfvm::set_last_error(KFVM_ERR_IO, "kfvm_plotfile_read: cannot open " + stem + ".meta");
  long long nx = -1, ny = -1, nz = -1;
  int dim = -1, eq = -1, nv = -1, ts = -1;
  double t = NAN, h = NAN;
  std::string line;
  while (std::getline(m, line)) {
    std::istringstream ls(line);
    std::string k;
    ls >> k;
    if (k == "dim") ls >> dim;
    else if (k == "eq") ls >> eq;
    else if (k == "nx") ls >> nx;
    else if (k == "ny") ls >> ny;
    else if (k == "nz") ls >> nz;
    else if (k == "nv") ls >> nv;
    else if (k == "time") t = std::strtod(line.c_str() + 5, nullptr);
    else if (k == "time_step") ls >> ts;
    else if (k == "time_step_size") h = std::strtod(line.c_str() + 15, nullptr);
  }
  if (dim != cfg->dim || eq != cfg->eq || nx != g.nx || ny != g.ny || nz != g.nz || nv != g.nv)
    return kfvm::set_last_error(KFVM_ERR_ARG, "kfvm_plotfile_read: " + stem + " was written for another grid or system");
  const size_t n = (size_t)g.n;
  for (int v = 0; v < g.nv; v++)
    if (!read_raw(stem + "." + kConsNames[v] + ".bin", u + (size_t)v * n, n))
      return kfvm::set_last_error(KFVM_ERR_IO, "kfvm_plotfile_read: bad dataset " + stem + "." + kConsNames[v] + ".bin");
  std::vector<double> w(n);
  if (!read_raw(stem + ".weno.bin", w.data(), n) || !read_raw(stem + ".fomx.bin", theta, n))
    return kfvm::set_last_error(KFVM_ERR_IO, "kfvm_plotfile_read: bad weno/fomx datasets in " + stem);
  for (size_t c = 0; c < n; c++) weno[c] = w[c] != 0.0 ? 1 : 0;
  *time_step = ts;
  *time = t;
  *dt = h;
  return KFVM_OK;
}

} // namespace

extern "C" {

int kfvm_plotfile_write(const kfvm_config *cfg, const char *dir, const char *base, int32_t num, int32_t ckpt,
                        int32_t time_step, double time, double dt, const double *u, const uint8_t *weno,
                        const double *theta) {
  try {
    return plotfile_write(cfg, dir, base, num, ckpt, time_step, time, dt, u, weno, theta);
  } catch (const std::exception &e) {
    return kfvm::set_last_error(KFVM_ERR_NOMEM, std::string("kfvm_plotfile_write: ") + e.what());
  }
}

int kfvm_plotfile_read(const kfvm_config *cfg, const char *xmf_path, double *u, uint8_t *weno, double *theta,
                       int32_t *time_step, double *time, double *dt) {
  try {
    return plotfile_read(cfg, xmf_path, u, weno, theta, time_step, time, dt);
  } catch (const std::exception &e) {
    return kfvm::set_last_error(KFVM_ERR_NOMEM, std::string("kfvm_plotfile_read: ") + e.what());
  }
}

} // extern "C"
