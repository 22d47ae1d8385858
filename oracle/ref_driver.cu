// Test infrastructure, not product code.
//
// Driver for the UNMODIFIED reference CUDA build (Xshuaizhang/Retainwall_code,
// src/*.cu compiled from where they lie, see oracle/build_ref.sh). It replaces
// the reference's src/main.cpp so that the private per-stage methods of
// LoquatSph (src/loquat.h:44-126) can be called one at a time:
//   * golden dumps of every device array after each stage or step,
//   * device-timed step loops (CUDA events) of the reference's own step,
//   * the reference's wall-force probe (src/utilities.cu:643-669),
//   * the reference's own output files (initial save and LoquatSph::Saving,
//     src/loquat.cu:439-482,533-537) at chosen steps.
// Nothing here changes the reference's arithmetic: the step sequence is the
// one of LoquatSph::RunSimulation (src/loquat.cu:511-565) minus file output.
//
// The reference keeps its stage methods private; the access specifier is
// lifted for this translation unit only (class layout is unchanged).
#define private public
#include "loquat.h"
#undef private
#include "utilities.h"
#include <helper_cuda.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <set>
#include <string>
#include <vector>

namespace {

// Arrays a dump writes (empty: all of them).
std::set<std::string> g_keys;
bool want_key(const char* k) { return g_keys.empty() || g_keys.count(k) > 0; }

struct DumpWriter {
  std::FILE* f = nullptr;
  int n = 0;
  long count_pos = 0;
  explicit DumpWriter(const std::string& path) {
    f = std::fopen(path.c_str(), "wb");
    if (!f) {
      std::fprintf(stderr, "cannot open %s\n", path.c_str());
      std::exit(2);
    }
    std::fwrite("RWD1", 1, 4, f);
    count_pos = std::ftell(f);
    int32_t zero = 0;
    std::fwrite(&zero, 4, 1, f);
  }
  void raw(const char* name, const void* host, int32_t elem, int64_t count) {
    char nm[32] = {0};
    std::strncpy(nm, name, 31);
    std::fwrite(nm, 1, 32, f);
    std::fwrite(&elem, 4, 1, f);
    std::fwrite(&count, 8, 1, f);
    std::fwrite(host, (size_t)elem, (size_t)count, f);
    ++n;
  }
  void dev(const char* name, const void* dptr, int32_t elem, int64_t count) {
    if (!want_key(name)) return;
    std::vector<char> h((size_t)elem * (size_t)count);
    if (count > 0) checkCudaErrors(cudaMemcpy(h.data(), dptr, h.size(), cudaMemcpyDeviceToHost));
    raw(name, h.data(), elem, count);
  }
  ~DumpWriter() {
    std::fseek(f, count_pos, SEEK_SET);
    int32_t nn = n;
    std::fwrite(&nn, 4, 1, f);
    std::fclose(f);
  }
};

void dump_state(LoquatSph& s, const std::string& path, int step) {
  checkCudaErrors(cudaDeviceSynchronize());
  Parameters* p = s.par_host;
  const int64_t np = p->np, npb = p->npb, ncell = p->ncell;
  DumpWriter w(path);
  double meta[10] = {s.time, (double)step, (double)p->npm, (double)p->np_delete_m, (double)p->dt,
                     (double)np, (double)npb, (double)ncell, (double)sizeof(scalar), (double)p->time};
  w.raw("meta", meta, 8, 10);
  w.dev("codes", s.codes, sizeof(int4), np);
  w.dev("cellpos", s.cellpos, sizeof(int4), np);
  w.dev("pospres", s.pospres, sizeof(scalar4), np);
  w.dev("pospres_ori", s.pospres_ori, sizeof(scalar4), np);
  w.dev("velrhop", s.velrhop, sizeof(scalar4), np);
  w.dev("idmassidx", s.idmassidx, sizeof(scalar4), np);
  w.dev("str", s.str, sizeof(tensor2d), np);
  w.dev("stn", s.stn, sizeof(tensor2d), np);
  w.dev("normal_m", s.normal_m, sizeof(scalar4), npb);
  w.dev("contact_mag", s.contact_mag, sizeof(tensor2dful), np);
  w.dev("contact_var", s.contact_var, sizeof(scalar4), np);
  w.dev("accad", s.accad, sizeof(scalar4), np);
  w.dev("spin", s.spin, sizeof(scalar4), np);
  w.dev("acestn", s.acestn, sizeof(tensor2d), np);
  w.dev("pospres_ini", s.pospres_ini, sizeof(scalar4), np);
  w.dev("velrhop_ini", s.velrhop_ini, sizeof(scalar4), np);
  w.dev("str_ini", s.str_ini, sizeof(tensor2d), np);
  w.dev("stn_ini", s.stn_ini, sizeof(tensor2d), np);
  w.dev("part_idx", s.grid->GetPartIdx(), sizeof(int), np);
  w.dev("part_cel", s.grid->GetPartCel(), sizeof(int), np);
  w.dev("cell_beg", s.grid->GetCellBeg(), sizeof(int), ncell);
  w.dev("cell_end", s.grid->GetCellEnd(), sizeof(int), ncell);
}

// Zero every state array once after allocation. cudaMalloc gives fresh
// (zero-filled) pages in a new process in practice; doing it explicitly makes
// the never-written slots (e.g. contact state of boundary slots) defined.
void zero_state(LoquatSph& s) {
  Parameters* p = s.par_host;
  const size_t np = p->np;
  checkCudaErrors(cudaMemset(s.contact_mag, 0, np * sizeof(tensor2dful)));
  checkCudaErrors(cudaMemset(s.contact_var, 0, np * sizeof(scalar4)));
  checkCudaErrors(cudaMemset(s.accad, 0, np * sizeof(scalar4)));
  checkCudaErrors(cudaMemset(s.spin, 0, np * sizeof(scalar4)));
  checkCudaErrors(cudaMemset(s.acestn, 0, np * sizeof(tensor2d)));
  checkCudaErrors(cudaMemset(s.pospres_ini, 0, np * sizeof(scalar4)));
  checkCudaErrors(cudaMemset(s.velrhop_ini, 0, np * sizeof(scalar4)));
  checkCudaErrors(cudaMemset(s.str_ini, 0, np * sizeof(tensor2d)));
  checkCudaErrors(cudaMemset(s.stn_ini, 0, np * sizeof(tensor2d)));
}

// One step, as RunSimulation's loop body (src/loquat.cu:548-561), with an
// optional dump after every stage (PredictorSection / CorrectorSection bodies
// of src/loquat.cu:376-436 spelled out).
void step_once(LoquatSph& s, const std::string& stage_dir, int step, std::ofstream* save_to) {
  s.StepCalculation();
  if (stage_dir.empty()) {
    s.PredictorSection();
    s.CorrectorSection();
  } else {
    auto d = [&](const char* tag) { dump_state(s, stage_dir + "/" + tag + ".rwd", step); };
    Parameters* p = s.par_host;
    s.grid->NeighborSearch(p, s.par_device, s.cellpos, s.idmassidx);
    s.SortArraysPrimary();
    cudaDeviceSynchronize();
    d("p0_sorted");
    if (p->n_motion > 0) s.RigidBodyUpdate();
    s.AdamiBoundary();
    cudaDeviceSynchronize();
    d("p1_adami");
    s.FindCornerParticle();
    cudaDeviceSynchronize();
    d("p2_corner");
    if (p->stress_shepard_filter != 0 && s.step % p->stress_shepard_filter == 0 && s.step != 0)
      s.StressRegularization();
    s.ParticleInteraction();
    cudaDeviceSynchronize();
    d("p3_interaction");
    s.Predictor();
    cudaDeviceSynchronize();
    d("p4_predictor");
    s.grid->NeighborSearch(p, s.par_device, s.cellpos, s.idmassidx);
    s.SortArraysAll();
    cudaDeviceSynchronize();
    d("c0_sorted");
    s.AdamiBoundary();
    cudaDeviceSynchronize();
    d("c1_adami");
    s.FindCornerParticle();
    cudaDeviceSynchronize();
    d("c2_corner");
    s.ParticleInteraction();
    cudaDeviceSynchronize();
    d("c3_interaction");
    s.Corrector();
    cudaDeviceSynchronize();
    d("c4_corrector");
  }
  // RunSimulation saves after the corrector section, before time and step advance.
  if (save_to) s.Saving(*save_to);
  s.time += static_cast<double>(s.par_host->dt);
  s.output_time += static_cast<double>(s.par_host->dt);
  s.step++;
}

void usage() {
  std::fprintf(stderr,
               "usage: ref_driver <project> [--steps N] [--warmup W] [--time] [--dump-dir D]\n"
               "                  [--dump-steps a,b,c] [--stage-step S] [--wall-force-every K]\n"
               "                  [--dump-keys k1,k2] [--save-steps a,b]\n"
               "  --save-steps: 0 = RunSimulation's initial output; s > 0 = Saving during step s\n"
               "  (after its corrector section); files go to <project>/ as the reference writes them\n");
  std::exit(2);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) usage();
  std::string project = argv[1];
  int steps = 10, warmup = 0, stage_step = -1, wf_every = 0;
  bool timed = false;
  std::string dump_dir;
  std::vector<int> dump_steps, save_steps;
  auto int_list = [](const std::string& v, std::vector<int>& out) {
    size_t p0 = 0;
    while (p0 < v.size()) {
      size_t p1 = v.find(',', p0);
      if (p1 == std::string::npos) p1 = v.size();
      out.push_back(std::stoi(v.substr(p0, p1 - p0)));
      p0 = p1 + 1;
    }
  };
  for (int a = 2; a < argc; ++a) {
    std::string k = argv[a];
    auto next = [&]() -> std::string {
      if (a + 1 >= argc) usage();
      return argv[++a];
    };
    if (k == "--steps") steps = std::stoi(next());
    else if (k == "--warmup") warmup = std::stoi(next());
    else if (k == "--time") timed = true;
    else if (k == "--dump-dir") dump_dir = next();
    else if (k == "--stage-step") stage_step = std::stoi(next());
    else if (k == "--wall-force-every") wf_every = std::stoi(next());
    else if (k == "--dump-steps") int_list(next(), dump_steps);
    else if (k == "--save-steps") int_list(next(), save_steps);
    else if (k == "--dump-keys") {
      std::string v = next();
      size_t p0 = 0;
      while (p0 < v.size()) {
        size_t p1 = v.find(',', p0);
        if (p1 == std::string::npos) p1 = v.size();
        g_keys.insert(v.substr(p0, p1 - p0));
        p0 = p1 + 1;
      }
    } else usage();
  }

  checkCudaErrors(cudaSetDevice(0));
  LoquatSph s(project);
  // Initialisation of RunSimulation (src/loquat.cu:514-531) without the
  // results-folder creation and the initial file output.
  s.io->LoadParameters();
  s.io->LoadParticles();
  s.par_host = s.io->GetParameters();
  s.InitializeParameters();
  s.AllocateGpuMemory();
  zero_state(s);
  s.CopyDataFromHostToDevice();
  checkCudaErrors(cudaMemcpy(s.par_device, s.par_host, sizeof(Parameters), cudaMemcpyHostToDevice));
  s.grid->GridConfig(s.par_host);
  s.grid->PositionFromAbsolute2Relative(s.par_host, s.par_device, s.cellpos, s.pospres);
  s.grid->NeighborSearch(s.par_host, s.par_device, s.cellpos, s.idmassidx);
  s.SortArraysPrimary();
  auto want_save = [&](int st) {
    for (int d : save_steps)
      if (d == st) return true;
    return false;
  };
  std::ofstream history;
  if (!save_steps.empty()) {
    std::filesystem::create_directories(project);
    if (want_save(0)) {  // RunSimulation's output of the initial configuration
      s.CopyDataFromDeviceToHost();
      s.io->SaveXml();
      s.io->SaveParticles();
    }
    history.open((project + "/time_history.txt").c_str());
  }
  s.TimerInitiation();
  checkCudaErrors(cudaDeviceSynchronize());

  std::ofstream wf;
  if (!dump_dir.empty()) {
    dump_state(s, dump_dir + "/init.rwd", 0);
    wf.open((dump_dir + "/time_history.txt").c_str());
  }

  auto want_dump = [&](int st) {
    for (int d : dump_steps)
      if (d == st) return true;
    return false;
  };

  for (int w = 0; w < warmup; ++w) step_once(s, "", s.step, nullptr);
  checkCudaErrors(cudaDeviceSynchronize());

  cudaEvent_t e0, e1;
  checkCudaErrors(cudaEventCreate(&e0));
  checkCudaErrors(cudaEventCreate(&e1));
  checkCudaErrors(cudaEventRecord(e0));
  for (int k = 0; k < steps; ++k) {
    const int st = s.step;
    std::string sd;
    if (!dump_dir.empty() && st == stage_step) {
      sd = dump_dir + "/stage";
      std::filesystem::create_directories(sd);
    }
    step_once(s, sd, st, want_save(st + 1) ? &history : nullptr);
    if (!dump_dir.empty()) {
      if (want_dump(s.step)) dump_state(s, dump_dir + "/step_" + std::to_string(s.step) + ".rwd", s.step);
      if (wf_every > 0 && s.step % wf_every == 0)
        GetValuesAtPoint(project, s.par_host, s.par_device, s.pospres, s.velrhop, s.idmassidx, s.contact_mag,
                         s.contact_var, s.str, s.cellpos, s.grid->GetCellBeg(), s.grid->GetCellEnd(), wf);
    }
  }
  checkCudaErrors(cudaEventRecord(e1));
  checkCudaErrors(cudaEventSynchronize(e1));
  float ms = 0.f;
  checkCudaErrors(cudaEventElapsedTime(&ms, e0, e1));
  if (timed) {
    const double sps = steps / (ms * 1e-3);
    std::printf("\n{\"impl\": \"reference-cuda\", \"scalar_bytes\": %d, \"np\": %d, \"npb\": %d, \"npm\": %d, "
                "\"steps\": %d, \"warmup\": %d, \"ms_per_step\": %.6f, \"steps_per_s\": %.4f, "
                "\"particle_updates_per_s\": %.6e}\n",
                (int)sizeof(scalar), s.par_host->np, s.par_host->npb, s.par_host->npm, steps, warmup, ms / steps, sps,
                sps * s.par_host->npm);
  }
  return 0;
}
