// kfvm_host.cpp -- ProblemSetup (.init parsing) and Solver over the C ABI.
#include "kfvm_host.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace kfvm {

namespace {

// the reference parses reals with std::stof (float), ints with std::stoi / stod
double rf(const std::string &v) { return static_cast<double>(std::stof(v)); }

std::vector<std::string> words(const std::string &s) {
  std::istringstream is(s);
  std::vector<std::string> w;
  std::string t;
  while (std::getline(is, t, ' '))
    if (!t.empty()) w.push_back(t);
  return w;
}

} // namespace

ProblemSetup::ProblemSetup() { kfvm_default_config(&cfg); }

bool ProblemSetup::setFromFile(const std::string &path) {
  std::ifstream in(path);
  if (!in.is_open()) return false;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    std::string category, setting;
    std::getline(ls, category, ':');
    std::getline(ls, setting, ':');
    bool ok = false;
    try {
      if (category == "mesh") ok = setMesh(setting);
      else if (category == "stencil") ok = setStencil(setting);
      else if (category == "time") ok = setTime(setting);
      else if (category == "eos") ok = setEos(setting);
      else if (category == "io") ok = setIO(setting);
      else if (category == "setup") ok = setSetup(setting);
      else if (category == "user") ok = true; // problem parameters are built into the ICs
      else {
        warnings.push_back("Ignoring line from input file: " + line);
        ok = true;
      }
    } catch (const std::exception &) {
      ok = false;
    }
    if (!ok) warnings.push_back("Line could not be parsed: " + line);
  }
  if (cfg.dim == 2) cfg.nz = 1;
  if (cfg.eq == KFVM_EQ_MHD_GLM) cfg.have_sources = 1; // ProblemSetup.H:81
  if (forcing && !forceTOffSet)
    warnings.push_back("setup:forcing on without eos:forcetoff: no step is forced (forcetoff = 0)");
  return true;
}

bool ProblemSetup::setMesh(const std::string &setting) {
  auto w = words(setting);
  if (w.empty()) return false;
  if (w[0] == "resolution" && w.size() >= 3) {
    cfg.nx = std::stoi(w[1]);
    cfg.ny = std::stoi(w[2]);
    if (w.size() >= 4) cfg.nz = std::stoi(w[3]);
  } else if (w[0] == "numblocks") {
    for (size_t i = 1; i < w.size(); i++)
      if (std::stoi(w[i]) != 1) warnings.push_back("one block per axis: this build runs one rank");
  } else if (w[0] == "extent" && w.size() >= 5) {
    cfg.xlo = rf(w[1]);
    cfg.xup = rf(w[2]);
    cfg.ylo = rf(w[3]);
    cfg.yup = rf(w[4]);
    if (w.size() >= 7) {
      cfg.zlo = rf(w[5]);
      cfg.zup = rf(w[6]);
    }
  } else {
    return false;
  }
  return true;
}

bool ProblemSetup::setStencil(const std::string &setting) {
  auto w = words(setting);
  if (w.size() >= 2 && w[0] == "lfac") {
    cfg.lfac = rf(w[1]);
    return true;
  }
  return false;
}

bool ProblemSetup::setTime(const std::string &setting) {
  auto w = words(setting);
  if (w.size() < 2) return false;
  const std::string &k = w[0], &v = w[1];
  if (k == "mindt") cfg.min_dt = rf(v);
  else if (k == "final") cfg.final_time = rf(v);
  else if (k == "cfl") cfg.cfl = rf(v);
  else if (k == "atol") cfg.atol = rf(v);
  else if (k == "rtol") cfg.rtol = rf(v);
  else if (k == "rejectionthresh") cfg.rejection_thresh = rf(v);
  else if (k == "rejectionlimit") cfg.rejection_limit = (int32_t)std::stod(v);
  else if (k == "maxsteps") cfg.max_steps = (int32_t)std::stod(v);
  else return false;
  return true;
}

bool ProblemSetup::setEos(const std::string &setting) {
  auto w = words(setting);
  if (w.size() < 2) return false;
  const std::string &k = w[0], &v = w[1];
  if (k == "gamma") cfg.gamma = rf(v);
  else if (k == "reynolds") cfg.reynolds = rf(v);
  else if (k == "prandtl") cfg.prandtl = rf(v);
  else if (k == "wenothresh") cfg.weno_thresh = rf(v);
  else if (k == "forceedot") force.edot = rf(v);
  else if (k == "forceratio") force.ratio = rf(v);
  else if (k == "forcetoff") {
    force.t_off = rf(v);
    forceTOffSet = true;
  } else if (k == "forcestr") (void)rf(v); // computed every step, the value read is not used
  else return false;
  return true;
}

bool ProblemSetup::setIO(const std::string &setting) {
  auto w = words(setting);
  if (w.empty()) return false;
  if (w[0] == "basename" && w.size() >= 2) baseName = w[1];
  else if (w[0] == "datadir" && w.size() >= 2) dataDir = w[1];
  else if (w[0] == "verbose" && w.size() >= 2) verbose = std::stoi(w[1]);
  else if (w[0] == "dumpstate" && w.size() >= 2) dumpState = std::stoi(w[1]) != 0;
  else if (w[0] == "plotfreq" && w.size() >= 2) plotFreq = rf(w[1]);
  else if (w[0] == "ckptfreq" && w.size() >= 2) ckptFreq = std::stoi(w[1]);
  else if (w[0] == "restartfile" && w.size() >= 2) {
    restartFile = w[1];
    restart = true;
  } else if (w[0] == "statsfreq" && w.size() >= 2) {
    statsFreq = std::stoi(w[1]);
  } else if (w[0] == "pdiconf") {
    warnings.push_back("io:pdiconf has no effect in this build (PDI is not built; files are XDMF + raw binary)");
  } else {
    return false;
  }
  return true;
}

// compile-time choices of the reference's Definitions.H, as run-time settings
bool ProblemSetup::setSetup(const std::string &setting) {
  auto w = words(setting);
  if (w.size() < 2) return false;
  const std::string &k = w[0], &v = w[1];
  if (k == "dim") cfg.dim = std::stoi(v);
  else if (k == "quadpts") cfg.nq = std::stoi(v);
  else if (k == "equations") {
    if (v == "hydro") cfg.eq = KFVM_EQ_HYDRO;
    else if (v == "navierstokes") cfg.eq = KFVM_EQ_NAVIERSTOKES;
    else if (v == "mhd_glm") cfg.eq = KFVM_EQ_MHD_GLM;
    else if (v == "srhydro") cfg.eq = KFVM_EQ_SRHYDRO;
    else return false;
  } else if (k == "riemann") {
    if (v == "llf") cfg.rs = KFVM_RS_LLF;
    else if (v == "hll") cfg.rs = KFVM_RS_HLL;
    else if (v == "hllc") cfg.rs = KFVM_RS_HLLC;
    else return false;
  } else if (k == "rk") {
    if (v == "ssp4_3_2") cfg.rk = KFVM_RK_SSP4_3_2;
    else if (v == "threestarp") cfg.rk = KFVM_RK_THREESTARP;
    else if (v == "fourstarp") cfg.rk = KFVM_RK_FOURSTARP;
    else if (v == "ssp10_4_3") cfg.rk = KFVM_RK_SSP10_4_3;
    else return false;
  } else if (k == "bc") {
    // one word per face (west east south north [bottom top]) or one for all
    const int nf = (int)w.size() - 1;
    for (int f = 0; f < 6; f++) {
      const std::string &b = w[1 + (nf == 1 ? 0 : std::min(f, nf - 1))];
      if (b == "periodic") cfg.bc[f] = KFVM_BC_PERIODIC;
      else if (b == "outflow") cfg.bc[f] = KFVM_BC_OUTFLOW;
      else if (b == "reflecting") cfg.bc[f] = KFVM_BC_REFLECTING;
      else if (b == "noslip") cfg.bc[f] = KFVM_BC_NOSLIP;
      else return false;
    }
  } else if (k == "ic") {
    if (v == "isentropic_vortex") ic = KFVM_IC_ISENTROPIC_VORTEX;
    else if (v == "spherical_sod") ic = KFVM_IC_SPHERICAL_SOD;
    else if (v == "kelvin_helmholtz") ic = KFVM_IC_KELVIN_HELMHOLTZ;
    else if (v == "taylor_green") ic = KFVM_IC_TAYLOR_GREEN;
    else if (v == "orszag_tang") ic = KFVM_IC_ORSZAG_TANG;
    else if (v == "smooth_wave") ic = KFVM_IC_SMOOTH_WAVE;
    else if (v == "sr_shock_tube") ic = KFVM_IC_SR_SHOCK_TUBE;
    else if (v == "sr_riemann_2d") ic = KFVM_IC_SR_RIEMANN_2D;
    else if (v == "stir_turb") ic = KFVM_IC_STIR_TURB;
    else return false;
  } else if (k == "forcing") {
    if (v == "on") forcing = true;
    else if (v == "off") forcing = false;
    else return false;
  } else if (k == "seed") {
    seed = (uint64_t)std::stoull(v);
    force.seed = seed;
  } else if (k == "indicator") {
    if (v == "kxrcf") cfg.indicator = KFVM_IND_KXRCF;
    else if (v == "all") cfg.indicator = KFVM_IND_ALL;
    else if (v == "none") cfg.indicator = KFVM_IND_NONE;
    else return false;
  } else {
    return false;
  }
  return true;
}

std::string ProblemSetup::toJson() const {
  char b[2048];
  std::snprintf(b, sizeof(b),
                "{\"dim\": %d, \"eq\": %d, \"rs\": %d, \"rk\": %d, \"nq\": %d, \"indicator\": %d, "
                "\"nx\": %lld, \"ny\": %lld, \"nz\": %lld, \"extent\": [%.17g, %.17g, %.17g, %.17g, %.17g, "
                "%.17g], \"bc\": [%d, %d, %d, %d, %d, %d], \"gamma\": %.17g, \"reynolds\": %.17g, "
                "\"prandtl\": %.17g, \"weno_thresh\": %.17g, \"lfac\": %.17g, \"cfl\": %.17g, \"atol\": "
                "%.17g, \"rtol\": %.17g, \"rejection_thresh\": %.17g, \"min_dt\": %.17g, \"final_time\": "
                "%.17g, \"rejection_limit\": %d, \"max_steps\": %d, \"have_sources\": %d, \"ic\": %d, "
                "\"seed\": %llu, \"warnings\": %d, \"plot_freq\": %.17g, \"ckpt_freq\": %d, \"restart\": %d, "
                "\"forcing\": %d, \"force_edot\": %.17g, \"force_ratio\": %.17g, \"force_t_off\": %.17g, "
                "\"stats_freq\": %d}",
                cfg.dim, cfg.eq, cfg.rs, cfg.rk, cfg.nq, cfg.indicator, (long long)cfg.nx,
                (long long)cfg.ny, (long long)cfg.nz, cfg.xlo, cfg.xup, cfg.ylo, cfg.yup, cfg.zlo, cfg.zup,
                cfg.bc[0], cfg.bc[1], cfg.bc[2], cfg.bc[3], cfg.bc[4], cfg.bc[5], cfg.gamma, cfg.reynolds,
                cfg.prandtl, cfg.weno_thresh, cfg.lfac, cfg.cfl, cfg.atol, cfg.rtol, cfg.rejection_thresh,
                cfg.min_dt, cfg.final_time, cfg.rejection_limit, cfg.max_steps, cfg.have_sources, ic,
                (unsigned long long)seed, (int)warnings.size(), plotFreq, ckptFreq, restart ? 1 : 0, forcing ? 1 : 0,
                force.edot, force.ratio, force.t_off, statsFreq);
  return b;
}

// ---------------------------------------------------------------------------
Solver::Solver(const ProblemSetup &ps) : ps_(ps) {
  check(kfvm_create(&ps.cfg, &s_), "kfvm_create");
  if (!ps.restart) {
    check(kfvm_init_ic(s_, ps.ic, ps.seed), "kfvm_init_ic"); // setIC + FSAL priming + first dt
    if (ps.plotFreq > 0.0) {
      writePlot();
      plotNum_++;
    }
    if (ps.ckptFreq > 0) writeCkpt(0);
  } else {
    std::printf("Restarting from: %s\n", ps.restartFile.c_str());
    int32_t step = 0;
    check(kfvm_restart(s_, ps.restartFile.c_str(), &step), "kfvm_restart");
    nTS_ = step + 1;
  }
  if (ps.forcing) check(kfvm_set_forcing(s_, &ps.force), "kfvm_set_forcing");
  check(kfvm_get_time(s_, &time_, &dt_), "kfvm_get_time");
  if (ps.restart && ps.plotFreq > 0.0) plotNum_ = static_cast<int>(std::ceil(time_ / ps.plotFreq));
  check(kfvm_set_plot_freq(s_, ps.plotFreq, plotNum_), "kfvm_set_plot_freq");
}

std::string Solver::outputPrefix() const {
  const kfvm_config &c = ps_.cfg;
  std::string p = ps_.dataDir + "/R2_NX" + std::to_string(c.nx) + "_NY" + std::to_string(c.ny);
  if (c.dim == 3) p += "_NZ" + std::to_string(c.nz);
  return p + "/";
}

void Solver::writePlot() {
  const std::string dir = outputPrefix() + "plot";
  char b[32];
  std::snprintf(b, sizeof(b), "_%07d.xmf", plotNum_);
  std::printf("Writing file: %s/%s%s\n", dir.c_str(), ps_.baseName.c_str(), b);
  check(kfvm_write_plotfile(s_, dir.c_str(), ps_.baseName.c_str(), plotNum_, 0, plotNum_), "kfvm_write_plotfile");
}

void Solver::evalFlowStats() {
  double st[3];
  int32_t n = 0;
  check(kfvm_flow_stats(s_, st, &n), "kfvm_flow_stats");
  const std::string dir = outputPrefix();
  std::filesystem::create_directories(dir);
  FILE *f = std::fopen((dir + ps_.baseName + "_stats.dat").c_str(), statsRows_ == 0 ? "w" : "a");
  if (!f) throw std::runtime_error("cannot write " + dir + ps_.baseName + "_stats.dat");
  std::fprintf(f, "%.17g", time_);
  for (int q = 0; q < n; q++) std::fprintf(f, " %.17g", st[q]);
  std::fprintf(f, "\n");
  std::fclose(f);
  statsRows_++;
}

void Solver::writeCkpt(int step) {
  const std::string dir = outputPrefix() + "ckpt";
  char b[32];
  std::snprintf(b, sizeof(b), "_%07d.xmf", step);
  std::printf("Writing file: %s/%s%s\n", dir.c_str(), ps_.baseName.c_str(), b);
  check(kfvm_write_plotfile(s_, dir.c_str(), ps_.baseName.c_str(), step, 1, step), "kfvm_write_plotfile");
}

Solver::~Solver() { kfvm_destroy(s_); }

void Solver::check(int rc, const char *what) const {
  if (rc != KFVM_OK) throw std::runtime_error(std::string(what) + ": " + kfvm_last_error());
}

void Solver::TakeStep() {
  check(kfvm_take_step(s_, &info_), "kfvm_take_step");
  time_ = info_.time;
  dt_ = info_.dt;
  lastTimeStep_ = info_.last_step != 0;
  accepted_ += info_.accepted;
  const int rejected = info_.attempts - info_.accepted;
  if (rejected > 0) {
    if (info_.status == KFVM_TS_UNPHYSICAL) nRejectUnphys_ += rejected;
    else nRejectThresh_ += rejected;
  }
}

// Solver::Solve (src/Solver.cpp:84-140) with its plot and checkpoint cadence
void Solver::Solve() {
  const int maxSteps = ps_.cfg.max_steps;
  // flow statistics before stepping, every statsfreq steps and after the last
  // (Solver.cpp:87-91, 108-111, 124-126)
  if (ps_.statsFreq > 0) evalFlowStats();
  for (; nTS_ < maxSteps && !lastTimeStep_; ++nTS_) {
    if (ps_.verbose > 0) std::printf("Step %d: time = %.4g\n", nTS_, time_);
    // random forcing before the step while time < forcetoff (Solver.cpp:99-103)
    if (ps_.forcing && time_ < ps_.force.t_off) check(kfvm_apply_forcing(s_, nullptr, nullptr, nullptr), "kfvm_apply_forcing");
    TakeStep();
    if (ps_.statsFreq > 0 && nTS_ % ps_.statsFreq == 0) evalFlowStats();
    if (ps_.plotFreq > 0.0 && (info_.write_plot || lastTimeStep_ || nTS_ == maxSteps - 1)) {
      writePlot();
      plotNum_++;
      check(kfvm_set_plot_freq(s_, ps_.plotFreq, plotNum_), "kfvm_set_plot_freq");
    }
    if (ps_.ckptFreq > 0 && (nTS_ % ps_.ckptFreq == 0 || lastTimeStep_ || nTS_ == maxSteps - 1)) writeCkpt(nTS_);
    if (lastTimeStep_ && ps_.statsFreq > 0) evalFlowStats();
  }
  std::printf("Time stepping completed\n  %lld RHS evals and %lld/%lld rejected (accuracy/unphysical) steps\n",
              (long long)info_.n_rhs, (long long)nRejectThresh_, (long long)nRejectUnphys_);
}

double Solver::evalRHS(double t) {
  double mv = 0.0;
  check(kfvm_eval_rhs(s_, t, nullptr, &mv), "kfvm_eval_rhs");
  return mv;
}

std::vector<double> Solver::state() const {
  const int nv = ps_.cfg.eq == KFVM_EQ_MHD_GLM ? 9 : 5;
  const int64_t n = ps_.cfg.nx * ps_.cfg.ny * (ps_.cfg.dim == 3 ? ps_.cfg.nz : 1);
  std::vector<double> u((size_t)nv * n);
  check(kfvm_get_state(s_, u.data()), "kfvm_get_state");
  return u;
}

} // namespace kfvm
