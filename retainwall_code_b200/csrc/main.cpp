// loquat <project> [gpu] : the reference's command line (src/main.cpp:23-28,
// src/loquat.cu:289-343, 511-565) on top of the C ABI.  Reads <project>.xml/.dat/.motion,
// writes output_N.xml, N.dat or <id>_N.vtu and time_history.txt into the folder <project>.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "../../include/retainwall.h"

static int fail(rw_ctx* ctx, rw_status s, const char* what) {
  std::fprintf(stderr, "%s failed: %s (%s)\n", what, rw_status_string(s), rw_last_error(ctx));
  if (ctx) rw_destroy(ctx);
  return EXIT_FAILURE;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "Error! Please give the project name!\n");
    return EXIT_FAILURE;
  }
  const std::string project = argv[1];
  const int device = argc >= 3 ? std::atoi(argv[2]) : 0;
  const int precision = std::getenv("RW_PRECISION") ? std::atoi(std::getenv("RW_PRECISION")) : 4;
  rw_ctx* ctx = nullptr;
  rw_status s = rw_create(project.c_str(), device, precision, &ctx);
  if (s) return fail(nullptr, s, "rw_create");
  // each save's files are written while the following steps run
  if ((s = rw_set_option(ctx, RW_OPT_ASYNC_SAVE, 1.0))) return fail(ctx, s, "rw_set_option");
  rw_info inf;
  rw_get_info(ctx, &inf);
  std::printf("LOQUAT-compatible SPH step on device %d: np=%d npb=%d npm=%d ncell=%d dt=%.3e\n", device, inf.np,
              inf.npb, inf.npm, inf.ncell, inf.dt);
  if ((s = rw_save(ctx, project.c_str()))) return fail(ctx, s, "rw_save");  // initial output
  // time-max and output-frequency come from the parameter file (src/loquat_io.cu:192-195);
  // RW_TIME_MAX overrides time-max (short runs).
  const char* tm = std::getenv("RW_TIME_MAX");
  const double time_max = tm ? std::atof(tm) : inf.time_max;
  const double out_freq = inf.output_frequency, dt = inf.dt;
  // The reference's loop (src/loquat.cu:548-561), one step per iteration: Saving runs
  // inside a step when output_time > output-frequency, then time and output_time
  // advance by dt.  The host counters are advanced the same way to find each save's
  // step; the steps between saves run as one rw_step call.
  double time = inf.time, output_time = 0.0;
  while (time < time_max) {
    int n = 0;
    bool save = false;
    while (time < time_max && !save) {
      ++n;
      save = output_time > out_freq;
      if (save) output_time = 0.0;
      time += dt;
      output_time += dt;
    }
    if ((s = rw_step(ctx, n))) return fail(ctx, s, "rw_step");
    if ((s = rw_synchronize(ctx))) return fail(ctx, s, "rw_synchronize");
    if (save) {
      if ((s = rw_save(ctx, project.c_str()))) return fail(ctx, s, "rw_save");
      std::printf("Time = %0.5f saved\n", time - dt);
    }
  }
  if ((s = rw_synchronize(ctx))) return fail(ctx, s, "rw_synchronize");  // the last save's files
  rw_destroy(ctx);
  return 0;
}
