// kfvm_run -- command-line driver, the counterpart of the reference's
// `kfvm.ex <file.init>` (src/main.cpp:23-55) for one rank on one GPU.
//   kfvm_run <file.init>               run to final time / maxsteps
//   kfvm_run --parse-only <file.init>  print the parsed configuration as JSON
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

#include "kfvm_host.hpp"

int main(int argc, char **argv) {
  bool parseOnly = false;
  std::string path;
  for (int i = 1; i < argc; i++) {
    if (std::strcmp(argv[i], "--parse-only") == 0) parseOnly = true;
    else path = argv[i];
  }
  if (path.empty()) {
    std::fprintf(stderr, "usage: kfvm_run [--parse-only] <file.init>\n");
    return 2;
  }
  kfvm::ProblemSetup ps;
  if (!ps.setFromFile(path)) {
    std::fprintf(stderr, "Error: could not open input file: %s\n", path.c_str());
    return 1;
  }
  for (auto &w : ps.warnings) std::fprintf(stderr, "[Warning] %s\n", w.c_str());
  if (parseOnly) {
    std::printf("%s\n", ps.toJson().c_str());
    return 0;
  }
  try {
    std::printf("Setting options from input file: %s\n", path.c_str());
    kfvm::Solver solver(ps);
    solver.Solve();
    std::printf("final time %.17g, accepted steps %lld\n", solver.time(), (long long)solver.acceptedSteps());
    if (ps.dumpState) {
      const std::string out = ps.baseName + "_state.bin";
      auto u = solver.state();
      FILE *f = std::fopen(out.c_str(), "wb");
      if (f) {
        std::fwrite(u.data(), sizeof(double), u.size(), f);
        std::fclose(f);
        std::printf("state written to %s (float64 [v][z][y][x])\n", out.c_str());
      }
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "Error: %s\n", e.what());
    return 1;
  }
  return 0;
}
