// Drop-in executable for the reference's CalcNonstat3DLine (run in the
// Calculations directory by GeoCalculatorSP, GeoCalculatorSP.cpp:1656-1662).
//
//   tdem_calcnonstat3dline [--form A|E] [--scheme 2|3] [--device N] [workdir]
//
// Without flags the variant is taken from the program name when it ends in
// _A2, _A3, _E2 or _E3 (one name per reference build), else A-form, two-point.
// Unlike the reference, which always exits 0, the exit code is the tdem_status.
//
// Installed under a name containing CalcStat3D (or run with --stationary) it is
// the drop-in for CalcStat3D_3T_A instead: the stationary initial field
// (v3n.dat, v3a.dat, a0.dat) of the model in workdir.
//
// Installed under a name containing SumNonstat3DOnly (or run with
// --sum-nonstat-3d-only [workdir]) it is the drop-in for that module: the
// per-component files of the results in workdir (default the current directory,
// where GeoCalculatorSP.cpp:1673 runs it).  Installed under a name containing
// SummatorEDMN (or run with --summator-edmn) it takes that module's command line,
//   SummatorEDMN WithDDV profile place [--dir workdir]
// (SummatorEDMN/main.cpp:253-294) and writes the line voltages.  Under a name
// containing TimeDirectSolver or CorrectTimeMesh (or with --time-direct-solver /
// --correct-time-mesh [workdir]) it prepares the time grid as those modules do.
// With --pipeline (or under a name containing GeoCalculatorSP) it runs the
// direct-mode 3D-only module sequence in workdir (tdem_pipeline_directory): the
// time grid, the stationary field (--no-stationary skips it), the transient and
// the per-component split.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/tdem.h"

namespace {

// SumNonstat3DOnly [workdir] / SummatorEDMN WithDDV profile place [--dir workdir]
int post_main(bool summator, int argc, char** argv, int first) {
  std::string dir = ".";
  const char* pos[3] = {nullptr, nullptr, nullptr};
  int npos = 0;
  for (int i = first; i < argc; ++i) {
    if (!strcmp(argv[i], "--dir") && i + 1 < argc) {
      dir = argv[++i];
    } else if (summator && npos < 3) {
      pos[npos++] = argv[i];
    } else if (!summator && argv[i][0] != '-') {
      dir = argv[i];
    } else {
      fprintf(stderr, summator ? "usage: %s WithDDV profile place [--dir workdir]\n" : "usage: %s [workdir]\n",
              argv[0]);
      return (int)TDEM_ERR_ARGUMENT;
    }
  }
  char err[1024] = {0};
  tdem_status st;
  if (summator) {
    if (npos < 3) {
      fprintf(stderr, "usage: %s WithDDV profile place [--dir workdir]\n", argv[0]);
      return (int)TDEM_ERR_ARGUMENT;
    }
    st = tdem_summator_edmn(dir.c_str(), atoi(pos[0]), atoi(pos[1]), atoi(pos[2]), err, sizeof err);
    if (st != TDEM_OK) fprintf(stderr, "SummatorEDMN: %s\n", err);
  } else {
    st = tdem_sum_nonstat_3d_only(dir.c_str(), err, sizeof err);
    if (st != TDEM_OK) fprintf(stderr, "SumNonstat3DOnly: %s\n", err);
  }
  return (int)st;
}

// TimeDirectSolver [workdir] / CorrectTimeMesh [workdir]
int grid_main(bool correct, int argc, char** argv, int first) {
  std::string dir = ".";
  for (int i = first; i < argc; ++i) {
    if (argv[i][0] == '-') {
      fprintf(stderr, "usage: %s [workdir]\n", argv[0]);
      return (int)TDEM_ERR_ARGUMENT;
    }
    dir = argv[i];
  }
  char err[1024] = {0};
  const tdem_status st = correct ? tdem_correct_time_mesh(dir.c_str(), err, sizeof err)
                                 : tdem_time_direct_solver(dir.c_str(), err, sizeof err);
  if (st != TDEM_OK) fprintf(stderr, "%s: %s\n", correct ? "CorrectTimeMesh" : "TimeDirectSolver", err);
  return (int)st;
}

}  // namespace

int main(int argc, char** argv) {
  {
    const std::string prog = argv[0];
    if (prog.find("TimeDirectSolver") != std::string::npos) return grid_main(false, argc, argv, 1);
    if (prog.find("CorrectTimeMesh") != std::string::npos) return grid_main(true, argc, argv, 1);
    if (argc > 1 && !strcmp(argv[1], "--time-direct-solver")) return grid_main(false, argc, argv, 2);
    if (argc > 1 && !strcmp(argv[1], "--correct-time-mesh")) return grid_main(true, argc, argv, 2);
    if (prog.find("SummatorEDMN") != std::string::npos) return post_main(true, argc, argv, 1);
    if (prog.find("SumNonstat3DOnly") != std::string::npos) return post_main(false, argc, argv, 1);
    if (argc > 1 && !strcmp(argv[1], "--summator-edmn")) return post_main(true, argc, argv, 2);
    if (argc > 1 && !strcmp(argv[1], "--sum-nonstat-3d-only")) return post_main(false, argc, argv, 2);
  }
  int form = 0, scheme = 2, device = 0;
  bool stationary = false, pipeline = false, pipe_stat = true;
  std::string dir = ".";
  const std::string prog = argv[0];
  if (prog.find("CalcStat3D") != std::string::npos) stationary = true;
  if (prog.find("GeoCalculatorSP") != std::string::npos) pipeline = true;
  if (prog.size() >= 3) {
    const std::string tail = prog.substr(prog.size() - 3);
    if (tail == "_A2") { form = 0; scheme = 2; }
    if (tail == "_A3") { form = 0; scheme = 3; }
    if (tail == "_E2") { form = 1; scheme = 2; }
    if (tail == "_E3") { form = 1; scheme = 3; }
  }
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--form") && i + 1 < argc) {
      const char* v = argv[++i];
      form = (v[0] == 'E' || v[0] == 'e' || v[0] == '1') ? 1 : 0;
    } else if (!strcmp(argv[i], "--scheme") && i + 1 < argc) {
      scheme = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "--device") && i + 1 < argc) {
      device = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "--stationary")) {
      stationary = true;
    } else if (!strcmp(argv[i], "--pipeline")) {
      pipeline = true;
    } else if (!strcmp(argv[i], "--no-stationary")) {
      pipe_stat = false;
    } else if (argv[i][0] == '-') {
      fprintf(stderr, "usage: %s [--form A|E] [--scheme 2|3] [--stationary | --pipeline [--no-stationary]] "
              "[--device N] [workdir]\n", argv[0]);
      return (int)TDEM_ERR_ARGUMENT;
    } else {
      dir = argv[i];
    }
  }
  char err[1024] = {0};
  if (pipeline) {
    const int flags = TDEM_PIPE_TIME_GRID | TDEM_PIPE_SPLIT | (pipe_stat ? TDEM_PIPE_STATIONARY : 0);
    const tdem_status st = tdem_pipeline_directory(dir.c_str(), form, scheme, device, flags, err, sizeof err);
    if (st != TDEM_OK) fprintf(stderr, "pipeline (B200): %s\n", err);
    return (int)st;
  }
  if (stationary) {
    const tdem_status st = tdem_stationary_directory(dir.c_str(), device, err, sizeof err);
    if (st != TDEM_OK) fprintf(stderr, "CalcStat3D_3T_A (B200): %s\n", err);
    return (int)st;
  }
  const tdem_status st = tdem_run_directory(dir.c_str(), form, scheme, device, err, sizeof err);
  if (st != TDEM_OK) fprintf(stderr, "CalcNonstat3DLine (B200): %s\n", err);
  return (int)st;
}
