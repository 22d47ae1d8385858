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
  rw_info inf;
  rw_get_info(ctx, &inf);
  std::printf("LOQUAT-compatible SPH step on device %d: np=%d npb=%d npm=%d ncell=%d dt=%.3e\n", device, inf.np,
              inf.npb, inf.npm, inf.ncell, inf.dt);
  // The reference reads time-max/output-frequency from the parameter file; they are
  // re-read here from output_0 of the case through rw_create's parameters.
  if ((s = rw_save(ctx, project.c_str()))) return fail(ctx, s, "rw_save");
  double time = inf.time, output_time = 0.0;
  const char* tm = std::getenv("RW_TIME_MAX");
  double time_max = tm ? std::atof(tm) : -1.0;
  double out_freq = -1.0;
  {  // time-max / output-frequency from the parameter file (src/loquat_io.cu:192-195)
    std::FILE* f = std::fopen((project + ".xml").c_str(), "r");
    if (f) {
      char line[512];
      while (std::fgets(line, sizeof line, f)) {
        std::string l(line);
        auto val = [&](const char* tag) {
          size_t a = l.find('>'), b = l.find("</");
          return std::atof(l.substr(a + 1, b - a - 1).c_str());
        };
        if (l.find("<time-max ") != std::string::npos && time_max < 0) time_max = val("time-max");
        if (l.find("<output-frequency ") != std::string::npos) out_freq = val("output-frequency");
      }
      std::fclose(f);
    }
  }
  // Run in chunks of whole steps between saves (src/loquat.cu:548-561).
  while (time < time_max) {
    int n = 1;
    if (out_freq > 0) {
      n = (int)((out_freq - output_time) / inf.dt);
      if (n < 1) n = 1;
    }
    if ((s = rw_step(ctx, n))) return fail(ctx, s, "rw_step");
    if ((s = rw_synchronize(ctx))) return fail(ctx, s, "rw_synchronize");
    time += n * inf.dt;
    output_time += n * inf.dt;
    if (out_freq > 0 && output_time > out_freq) {
      if ((s = rw_save(ctx, project.c_str()))) return fail(ctx, s, "rw_save");
      output_time = 0.0;
      std::printf("Time = %0.5f saved\n", time);
    }
  }
  rw_destroy(ctx);
  return 0;
}
