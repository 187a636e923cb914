// kfvm_host.hpp -- C++ host layer over the C ABI: the reference's ProblemSetup
// (.init parsing, src/ProblemSetup.H:142-367) and Solver (src/Solver.H:118-160)
// for one rank on one GPU.  The reference selects dimension, equations, Riemann
// solver and RK scheme at compile time (exec/<problem>/Definitions.H); here they
// are read from a "setup" category of the same .init file, next to the
// reference's own categories (mesh, stencil, time, eos, user, io).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/kfvm_b200.h"

namespace kfvm {

struct ProblemSetup {
  kfvm_config cfg;
  int32_t ic = KFVM_IC_SMOOTH_WAVE;
  uint64_t seed = 12345;
  std::string baseName = "default", dataDir = "data";
  // plot / checkpoint output and restart (ProblemSetup.H:333-367)
  double plotFreq = 0.0;
  int ckptFreq = 0;
  int statsFreq = 0; // io:statsfreq: flow statistics every statsFreq steps
  std::string restartFile;
  bool restart = false;
  // random forcing (ENABLE_RANDOM_FORCING of the reference's Definitions.H as
  // setup:forcing on; eos:forceedot / forceratio / forcetoff, ParameterStructs.cpp:15-38)
  bool forcing = false, forceTOffSet = false;
  kfvm_forcing force{2.0, 1.0, 0.0, 12345};
  int verbose = 0;
  bool dumpState = false;
  std::vector<std::string> warnings;

  ProblemSetup();
  // Reads "category:key value..." lines; reals go through std::stof as in the
  // reference.  Returns false if the file cannot be opened.
  bool setFromFile(const std::string &path);
  std::string toJson() const;

 private:
  bool setMesh(const std::string &setting);
  bool setStencil(const std::string &setting);
  bool setTime(const std::string &setting);
  bool setEos(const std::string &setting);
  bool setIO(const std::string &setting);
  bool setSetup(const std::string &setting);
};

// Solver::Solver / Solve / TakeStep / evalRHS over the C ABI
class Solver {
 public:
  // Solver::Solver: initial condition (plus the first plot and checkpoint) or a
  // restart from ps.restartFile, then the FSAL priming evaluation
  explicit Solver(const ProblemSetup &ps);
  ~Solver();
  Solver(const Solver &) = delete;
  Solver &operator=(const Solver &) = delete;

  void Solve();
  void TakeStep();
  double evalRHS(double t);

  double time() const { return time_; }
  double dt() const { return dt_; }
  int64_t acceptedSteps() const { return accepted_; }
  const kfvm_step_info &lastInfo() const { return info_; }
  std::vector<double> state() const;

 private:
  void check(int rc, const char *what) const;
  // <dataDir>/R2_NX.._NY..[_NZ..]/ (WriterPDI.cpp:20-33)
  std::string outputPrefix() const;
  void writePlot();
  void writeCkpt(int step);
  // Solver::evalFlowStats: one row "time stats..." appended to <prefix><base>_stats.dat
  // (the reference appends the same row to <prefix><base>_stats.h5)
  void evalFlowStats();
  const ProblemSetup &ps_;
  kfvm_solver *s_ = nullptr;
  kfvm_step_info info_{};
  double time_ = 0.0, dt_ = 0.0;
  int64_t accepted_ = 0, nRejectThresh_ = 0, nRejectUnphys_ = 0;
  int nTS_ = 1;
  int plotNum_ = 0;
  int statsRows_ = 0;
  bool lastTimeStep_ = false;
};

} // namespace kfvm
