// Host side of the step: device state, per-stage launches (one per reference stage
// method), the CUDA-graph whole-step path, array export in the reference layouts,
// output writing, and the extern "C" ABI declared in include/retainwall.h.
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <future>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "../../include/retainwall.h"
#include "rw_io.h"
#include "rw_kernels.cuh"

namespace rw {

static thread_local std::string g_create_err;

struct Fail : std::runtime_error {
  int code;
  Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define RW_CU(call)                                                                         \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) throw Fail(e_ == cudaErrorMemoryAllocation ? RW_ENOMEM : RW_ECUDA, \
                                      std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

struct EngineBase {
  std::string err;
  int device = 0;
  // Bumped whenever an option or the closure changes what a captured step does; a batch
  // graph captured before the change is rebuilt before its next launch.
  unsigned generation = 0;
  virtual ~EngineBase() = default;
  virtual void begin_step() = 0;
  virtual void neighbor_search(int section) = 0;
  virtual void rigid() = 0;
  virtual void adami() = 0;
  virtual void corner() = 0;
  virtual void shepard() = 0;
  virtual void interaction() = 0;
  virtual void predictor() = 0;
  virtual void corrector() = 0;
  virtual void end_step() = 0;
  virtual void step(int n) = 0;
  virtual int sync() = 0;
  virtual void wall_force(int mode, int wall_id, const double* strip, double* out) = 0;
  virtual void save(const char* outdir) = 0;
  virtual void info(rw_info* out) = 0;
  virtual int set_option(int opt, double v) = 0;
  virtual int get_array(int which, void* dst, size_t bytes) = 0;
  virtual int set_array(int which, const void* src, size_t bytes) = 0;
  virtual void set_counters(double time, int step, int npm, int np_delete_m) = 0;
  virtual void profile(int nsteps, double* ms, int n, int* kps) = 0;
  virtual void wall_profile(double x_wall, double z_top, double dz, int nbins, double* out) = 0;
  virtual double step_timed(int n) = 0;
  virtual cudaGraph_t step_graph(bool gates) = 0;
  // Launches one whole step on this context's stream while that stream takes part in a
  // capture begun elsewhere (the batch's fork/join capture).
  virtual void launch_into_capture(bool gates) = 0;
  // Wall resultant computed on stream s into the device array d_out (3 doubles).
  virtual void wall_force_enqueue(cudaStream_t s, int mode, int wall_id, const double* strip, double* d_out) = 0;
  virtual cudaStream_t stream() const = 0;
  virtual int soil_count() = 0;
  virtual int set_closure(rw_mlp* net, double margin) = 0;
  virtual void closure_stats(double* out) = 0;
  virtual long long collect(rw_mlp* net, int stride, const Augment& aug) = 0;
  virtual void list_totals(long long* out) = 0;
};

static inline unsigned nblk(long n, int t) { return (unsigned)((n + t - 1) / t); }

// Status of a save's file writing (rw_save, RW_OPT_ASYNC_SAVE).
struct SaveResult {
  int rc;
  std::string msg;
};

template <class T> struct Engine final : EngineBase {
  Params<T> P{};
  DevState<T> S{};
  Dyn<T>* d_dyn = nullptr;
  cudaStream_t st = nullptr;
  std::vector<void*> allocs;
  int cpar = 0;  // live contact buffer
  bool compat_contact = true;
  cudaGraphExec_t gexec = nullptr;
  int g_cpar = -1;
  int ix_kernel = 0;     // 0: neighbours through L1/L2 (default); 1: chunked, shared-memory position tile
  int walk_threads = 128;   // RW_OPT_WALK_THREADS: block size of the walk launch
  int integ_threads = 256;  // RW_OPT_INTEGRATOR_THREADS: block size of the predictor and corrector
  bool strict_fp = false;  // interaction arithmetic: fused multiply-adds (default) or separately rounded
  int ncol = 0, max_chunks = 0;
  rw_case_params cparams{};
  int output_number = 0;
  int saves = 0;  // the first save is RunSimulation's initial output
  rw_mlp* cl_net = nullptr;  // learned closure (P.closure), its trust region and statistics
  ClosureTrust cl_trust{};
  double cl_err_max = 0.02;  // RW_OPT_CLOSURE_MAX_ERR
  double* d_clstats = nullptr;
  unsigned long long* d_count = nullptr;
  int nsm = 148;
  size_t near_wall_words = 0;
  // Step graphs captured with conditional nodes (gated()); st_body captures their bodies.
  bool allow_cond = false;
  bool graph_gates = true;  // RW_OPT_GRAPH_GATES
  // RW_OPT_ASYNC_SAVE: the files of a save are formatted and written by a background
  // task (at most one in flight) instead of by rw_save itself
  bool async_save = false;
  std::future<SaveResult> pending_save;
  unsigned char* stage_h = nullptr;  // page-locked staging of a save's arrays
  size_t stage_bytes = 0;
  bool graph_cond = false;  // the instantiated step graph has the gates
  cudaStream_t st_body = nullptr;

  ~Engine() override {
    wait_save();
    if (stage_h) cudaFreeHost(stage_h);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (st) cudaStreamSynchronize(st);
    for (void* p : allocs) cudaFree(p);
    if (st) cudaStreamDestroy(st);
    if (st_body) cudaStreamDestroy(st_body);
  }

  // Zeroed device buffers.  create() sizes everything it allocates in a measuring pass
  // and takes it from one arena (one cudaMalloc instead of about seventy), each buffer
  // 256-byte aligned; later allocations get their own cudaMalloc.
  char* arena = nullptr;
  size_t arena_cap = 0, arena_used = 0;
  bool measuring = false;
  template <class X> X* dalloc(size_t n) {
    const size_t bytes = (std::max<size_t>(n, 1) * sizeof(X) + 255) & ~(size_t)255;
    if (measuring) {
      arena_used += bytes;
      return nullptr;
    }
    if (arena && arena_used + bytes <= arena_cap) {
      X* p = reinterpret_cast<X*>(arena + arena_used);
      arena_used += bytes;
      return p;
    }
    void* p = nullptr;
    RW_CU(cudaMalloc(&p, bytes));
    allocs.push_back(p);
    RW_CU(cudaMemsetAsync(p, 0, bytes, st));
    return (X*)p;
  }
  template <class X> void up(X* d, const std::vector<X>& h) {
    if (!h.empty()) RW_CU(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(X), cudaMemcpyHostToDevice, st));
  }
  template <class X> std::vector<X> down(const X* d, size_t n) {
    std::vector<X> h(n);
    if (n) RW_CU(cudaMemcpyAsync(h.data(), d, n * sizeof(X), cudaMemcpyDeviceToHost, st));
    RW_CU(cudaStreamSynchronize(st));
    return h;
  }
  int* need_ptr() { return &d_dyn->need_sort; }
  Dyn<T> dyn_host() {
    Dyn<T> d;
    RW_CU(cudaMemcpyAsync(&d, d_dyn, sizeof(d), cudaMemcpyDeviceToHost, st));
    RW_CU(cudaStreamSynchronize(st));
    return d;
  }
  void check_launch() { RW_CU(cudaGetLastError()); }

  // Work that often has nothing to do.  While a step graph is being captured (with
  // conditional nodes allowed), body() goes into the body of an IF node and gate(h)
  // launches the one-thread kernel that sets its condition on the device, so a skipped
  // body costs one small launch instead of a launch per kernel.  Otherwise body() is
  // launched as it is and its kernels return at once on their own.
  template <class Gate, class Body> void gated(Gate gate, Body body) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    RW_CU(cudaStreamIsCapturing(st, &cs));
    if (!allow_cond || cs != cudaStreamCaptureStatusActive) {
      body();
      return;
    }
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    RW_CU(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphConditionalHandle h;
    RW_CU(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    gate(h);
    check_launch();
    RW_CU(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    RW_CU(cudaGraphAddNode(&node, g, deps, nd, &cp));
    if (!st_body) RW_CU(cudaStreamCreateWithFlags(&st_body, cudaStreamNonBlocking));
    RW_CU(cudaStreamBeginCaptureToGraph(st_body, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
    std::swap(st, st_body);  // the body's launches go to the body graph
    try {
      body();
    } catch (...) {
      std::swap(st, st_body);
      cudaGraph_t bg = nullptr;
      cudaStreamEndCapture(st_body, &bg);
      throw;
    }
    std::swap(st, st_body);
    cudaGraph_t bg = nullptr;
    RW_CU(cudaStreamEndCapture(st_body, &bg));  // the body graph belongs to the node
    RW_CU(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  }

  // ------------------------------------------------------------------------------
  // Set-up: InitializeParameters (src/loquat.cu:130-190), AllocateGpuMemory,
  // CopyDataFromHostToDevice, PositionFromAbsolute2Relative, first NeighborSearch +
  // SortArraysPrimary (src/loquat.cu:514-531).
  // ------------------------------------------------------------------------------
  void create(const rw_case* c, int dev) {
    device = dev;
    RW_CU(cudaSetDevice(dev));
    RW_CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const rw_case_params& q = c->params;
    cparams = q;
    output_number = q.output_number;
    if (q.dim != 3) throw Fail(RW_EINVAL, "only 3D cases are supported (dimension-of-problem must be 3)");
    if (q.periodbound) {
      const double nl = q.planeleft[0] * q.planeleft[0] + q.planeleft[1] * q.planeleft[1] + q.planeleft[2] * q.planeleft[2];
      const double nr = q.planeright[0] * q.planeright[0] + q.planeright[1] * q.planeright[1] +
                        q.planeright[2] * q.planeright[2];
      if (!(nl > 0.0) || !(nr > 0.0)) throw Fail(RW_EINVAL, "periodic plane with a zero normal");
    }
    if (q.np != q.npb + q.npm || q.np <= 0 || q.npb < 0 || q.npm < 0)
      throw Fail(RW_EINVAL, "Error! Wrong number of particles ...");
    if (q.np >= (1 << 27)) throw Fail(RW_EINVAL, "more than 2^27 particles");
    if (q.n_motion < 0 || q.n_motion > kMotionMax) throw Fail(RW_EINVAL, "number-of-motion out of range");
    if (q.n_model < 0 || q.n_model > kModelMax) throw Fail(RW_EINVAL, "number-of-model out of range");
    for (int i = 0; i < q.np; ++i) {  // indices the kernels use to address tables
      const int32_t* cc = c->codes + 4 * i;
      const bool nonfix = cc[1] == 1;
      if (i < q.npb) {
        if (nonfix && (cc[3] < 0 || cc[3] >= q.n_motion))
          throw Fail(RW_EINVAL, "moving boundary particle " + std::to_string(i) + " has motion index out of range");
      } else if (nonfix && (cc[3] < 0 || cc[3] >= kModelMax)) {
        throw Fail(RW_EINVAL, "material particle " + std::to_string(i) + " has material index out of range");
      }
    }
    P.dim = q.dim;
    P.periodbound = q.periodbound ? 1 : 0;
    P.n_motion = q.n_motion;
    P.n_model = q.n_model;
    P.np = q.np;
    P.npb = q.npb;
    P.npm0 = q.npm;
    for (int k = 0; k < 4; ++k) {
      P.planeleft[k] = (T)q.planeleft[k];
      P.planeright[k] = (T)q.planeright[k];
    }
    for (int k = 0; k < 3; ++k) {
      P.domain_size[k] = (T)q.domain_size[k];
      P.domain_min[k] = (T)q.domain_min[k];
      P.gravity[k] = (T)q.gravity[k];
    }
    P.dr = (T)q.dr;
    P.hdr = (T)q.hdr;
    P.rho0_m = (T)q.rho0_m;
    P.damping = (T)q.damping;
    for (int i = 0; i < kModelMax; ++i)
      for (int j = 0; j < kMatSize; ++j) P.model_par[i][j] = (T)q.model_par[i][j];
    P.stress_shepard_filter = q.stress_shepard_filter;
    P.viscosity_type = q.viscosity_type;
    P.output_format = q.output_format;
    P.alpha_m = (T)q.artificial_viscosity_alpha_m;
    P.cs_m = (T)q.cs_m;
    P.cfl = (T)q.cfl;
    P.art_coef = (T)q.artificial_pressure_coefficient_material;
    P.time_max = (T)q.time_max;
    P.output_frequency = (T)q.output_frequency;
    P.wall_fric = (T)q.wall_friction;
    P.h = P.dr * P.hdr;
    P.i_h = T(1.0f) / P.h;
    P.eta = T(0.01f) * P.h * P.h;
    P.bound_thickness = (T)(std::ceil(2.0 * (double)P.hdr) * (double)P.dr);
    const double h_d = (double)P.h;
    P.vol_def = (T)std::pow((double)P.dr, 3.0);
    P.cell_num[0] = (int)(T(0.5f) * P.i_h * P.domain_size[0]) + 1;
    P.cell_num[1] = (int)(T(0.5f) * P.i_h * P.domain_size[1]) + 1;
    P.cell_num[2] = (int)(T(0.5f) * P.i_h * P.domain_size[2]) + 1;
    P.knorm = (T)(42.0 / (256.0 * 3.14159265358979323846 * std::pow(h_d, 3.0)));
    P.kgrad = (T)(-5.0 * 42 / (256.0 * 3.14159265358979323846 * std::pow(h_d, 5.0)));
    const long one = (long)P.cell_num[0] * P.cell_num[1] * P.cell_num[2];
    if (one <= 0 || 2 * one + 1 > (1L << 30)) throw Fail(RW_EINVAL, "cell grid too large");
    P.ncell_material = (int)one;
    P.ncell_delete_m = (int)(2 * one);
    P.ncell = P.ncell_delete_m + 1;
    const T qq = P.dr * P.i_h;
    P.kernel_zero = P.knorm * T(2.0f) * T(2.0f) * T(2.0f) * T(2.0f) * T(0.5f);
    P.kernel_dr = P.knorm * (T(2.0f) - qq) * (T(2.0f) - qq) * (T(2.0f) - qq) * (T(2.0f) - qq) * (qq + T(0.5f));
    P.two_h = (T)(2.0 * (double)P.h);
    P.visc_k = P.alpha_m * P.cs_m * P.h;
    const double rpre = 2.0 * h_d * (1.0 + 1e-4);
    P.r2_prefilter = (T)(rpre * rpre);
    set_skin(0.02);
    P.dt = P.cfl * (P.h / P.cs_m);  // StepCalculation (src/loquat.cu:368-369)

    const size_t np = P.np, npb = P.npb;
    HypoC<T>* tab = nullptr;
    auto allocate = [&] {
      for (int b = 0; b < 2; ++b) {
        S.codes[b] = dalloc<int4>(np);
        S.cellpos[b] = dalloc<int4>(np);
        S.pos[b] = dalloc<V4<T>>(np);
        S.pos_ori[b] = dalloc<V4<T>>(np);
        S.vel[b] = dalloc<V4<T>>(np);
        S.idm[b] = dalloc<V4<T>>(np);
        S.str_a[b] = dalloc<V4<T>>(np);
        S.str_b[b] = dalloc<V2<T>>(np);
        S.stn_a[b] = dalloc<V4<T>>(np);
        S.stn_b[b] = dalloc<V2<T>>(np);
        S.normal[b] = dalloc<V4<T>>(npb);
        S.pos_ini[b] = dalloc<V4<T>>(np);
        S.vel_ini[b] = dalloc<V4<T>>(np);
        S.stri_a[b] = dalloc<V4<T>>(np);
        S.stri_b[b] = dalloc<V2<T>>(np);
        S.stni_a[b] = dalloc<V4<T>>(np);
        S.stni_b[b] = dalloc<V2<T>>(np);
        S.cv[b] = dalloc<V4<T>>(np);
        S.cf[b] = dalloc<V4<T>>(np);
        S.cmp_p[b] = dalloc<V4<T>>(np);
        S.cmp_v[b] = dalloc<V4<T>>(np);
        S.cmp_pi[b] = dalloc<V4<T>>(np);
        S.cmp_vi[b] = dalloc<V4<T>>(np);
      }
      S.accad = dalloc<V4<T>>(np);
      S.spin = dalloc<V4<T>>(np);
      S.ace_a = dalloc<V4<T>>(np);
      S.ace_b = dalloc<V2<T>>(np);
      S.cny = dalloc<V4<T>>(np);
      S.cvz = dalloc<V4<T>>(np);
      S.rec = dalloc<Rec<T>>(np);
      S.tc_a = dalloc<V4<T>>(np);
      S.tc_b = dalloc<V2<T>>(np);
      S.keys = dalloc<int>(np);
      S.vals = dalloc<int>(np);
      S.tk = dalloc<int>(np);
      S.tv = dalloc<int>(np);
      S.range = dalloc<int2>(P.ncell);
      S.ntiles = (int)nblk((long)np, RS_TILE);
      S.hist = dalloc<int>(256 * (size_t)S.ntiles);
      S.dtot = dalloc<int>(256);
      int bits = 1;
      while ((1L << bits) <= P.ncell_delete_m) ++bits;
      S.sort_passes = (bits + 7) / 8;
      S.skeys = (S.sort_passes & 1) ? S.tk : S.keys;
      S.sperm = (S.sort_passes & 1) ? S.tv : S.vals;
      S.wsum = dalloc<double>(3 * (WF_BLOCKS + 1));
      ncol = P.cell_num[0] * P.cell_num[1];
      max_chunks = P.npm0 / IX2_TB + ncol + 1;
      S.col_beg = dalloc<int>(ncol);
      S.col_len = dalloc<int>(ncol);
      S.col_cnt = dalloc<int>(ncol);
      S.col_off = dalloc<int>(ncol);
      near_wall_words = ((size_t)P.ncell_material + 3) / 4;
      S.near_wall = reinterpret_cast<unsigned char*>(dalloc<unsigned>(near_wall_words));
      S.chunks = dalloc<Chunk>(max_chunks);
      S.nbg_stride = (int)(np - npb);
      // kept candidate lists, two buffers each (a list update after a permutation reads
      // one and writes the other), their displacement bounds, and the marked cells
      for (int b = 0; b < 2; ++b) {
        if (lists_fit()) {  // list indices stay 32-bit
          S.nbg[b] = dalloc<unsigned>((size_t)IX_CAP * (np - npb));
          S.nbg_cnt[b] = dalloc<int>(np - npb);
        }
        S.dacc[b] = dalloc<float>(np);
        if (npb > 0 && (size_t)IX_CAP * npb < ((size_t)1 << 31)) {  // boundary lists (Adami)
          S.nbb[b] = dalloc<unsigned>((size_t)IX_CAP * npb);
          S.nbb_cnt[b] = dalloc<int>(npb);
        }
      }
      S.inv = dalloc<int>(np);
      S.queue = dalloc<int>(np + 1);
      S.cell_mark = dalloc<unsigned>(P.ncell_material);
      S.marks = dalloc<int>(RW_MARK_CAP);
      S.near_mark = dalloc<unsigned>(P.ncell_material);
      tab = dalloc<HypoC<T>>(kModelMax);
      d_clstats = dalloc<double>(4);
      d_count = dalloc<unsigned long long>(1);
      d_dyn = dalloc<Dyn<T>>(1);
    };
    measuring = true;
    arena_used = 0;
    allocate();
    measuring = false;
    arena_cap = arena_used;
    arena_used = 0;
    RW_CU(cudaMalloc(reinterpret_cast<void**>(&arena), arena_cap));
    allocs.push_back(arena);
    RW_CU(cudaMemsetAsync(arena, 0, arena_cap, st));
    allocate();
    {  // hypoplastic material constants, evaluated on the device as the kernels would
      k_hypo_table<T><<<1, 32, 0, st>>>(P, tab);
      RW_CU(cudaGetLastError());
      RW_CU(cudaMemcpyAsync(P.hypo, tab, sizeof(P.hypo), cudaMemcpyDeviceToHost, st));
      RW_CU(cudaStreamSynchronize(st));
    }
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);

    // The case arrays are uploaded as the caller holds them and converted on the device
    // (k_ingest).  The staging area is the candidate-list buffer, unused until the first
    // interaction builds the lists, or a temporary allocation when that is too small.
    {
      const size_t b_codes = np * 16, b4 = np * 4 * sizeof(double), b6 = np * 6 * sizeof(double);
      const size_t b_nrm = npb * 4 * sizeof(double);
      const size_t raw = b_codes + 3 * b4 + 2 * b6 + b_nrm;
      unsigned char* stage = nullptr;
      bool temp = false;
      if (S.nbg[0] && (size_t)IX_CAP * (np - npb) * sizeof(unsigned) >= raw) {
        stage = reinterpret_cast<unsigned char*>(S.nbg[0]);
      } else {
        RW_CU(cudaMalloc(reinterpret_cast<void**>(&stage), raw));
        temp = true;
      }
      size_t off = 0;
      auto put = [&](const void* h, size_t n) -> const void* {
        unsigned char* d = stage + off;
        if (n) RW_CU(cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, st));
        off += n;
        return d;
      };
      RawCase R;
      R.codes = static_cast<const int4*>(put(c->codes, b_codes));
      R.pospres = static_cast<const double*>(put(c->pospres, b4));
      R.velrhop = static_cast<const double*>(put(c->velrhop, b4));
      R.idmassidx = static_cast<const double*>(put(c->idmassidx, b4));
      R.stress = static_cast<const double*>(put(c->stress, b6));
      R.strain = static_cast<const double*>(put(c->strain, b6));
      R.normal = static_cast<const double*>(put(npb ? c->normal : nullptr, b_nrm));
      k_ingest<T><<<nblk((long)np, 256), 256, 0, st>>>(P, S, R, (T)(0.5 * (double)P.i_h));
      RW_CU(cudaGetLastError());
      if (temp) {
        RW_CU(cudaStreamSynchronize(st));
        RW_CU(cudaFree(stage));
      }
    }

    Dyn<T> d;
    std::memset(&d, 0, sizeof(d));
    d.mark_gen = 1;  // cell marks start at generation 0: unmarked
    d.time_d = q.time;
    d.time_f = (T)q.time;
    d.npm = q.npm;
    d.host_dirty = 1;  // soil neighbour records are first written by the corner search
    d.cells_dirty = 1;
    for (int i = 0; i < P.n_motion; ++i) {
      const rw_motion& m = q.motion[i];
      Table<T>& tb = d.tab[i];
      tb.is_translation = m.is_translation != 0;
      tb.is_rotation = m.is_rotation != 0;
      tb.n_trans = m.n_trans;
      tb.n_rot = m.n_rot;
      tb.pattern = m.pattern;
      if (m.n_trans < 0 || m.n_trans > kTableMax || m.n_rot < 0 || m.n_rot > kTableMax)
        throw Fail(RW_EINVAL, "motion table too long");
      for (int j = 0; j < kTableMax; ++j) {
        tb.trans_time[j] = (T)m.trans_time[j];
        tb.rotat_time[j] = (T)m.rotat_time[j];
        tb.trans_vel[j] = Vec3<T>{(T)m.trans_vel[j][0], (T)m.trans_vel[j][1], (T)m.trans_vel[j][2]};
        tb.trans_acc[j] = Vec3<T>{(T)m.trans_acc[j][0], (T)m.trans_acc[j][1], (T)m.trans_acc[j][2]};
        tb.rotat_acc[j] = Vec3<T>{(T)m.rotat_acc[j][0], (T)m.rotat_acc[j][1], (T)m.rotat_acc[j][2]};
      }
      tb.pos_rp = Vec3<T>{(T)m.pos_rp[0], (T)m.pos_rp[1], (T)m.pos_rp[2]};
      tb.rotat_vel = Vec3<T>{(T)m.rotat_vel[0], (T)m.rotat_vel[1], (T)m.rotat_vel[2]};
      Motion<T>& mv = d.mv[i];  // LoadParticles, src/loquat_io.cu:289-302
      mv.is_trans = tb.is_translation;
      mv.is_rotat = tb.is_rotation;
      mv.trans_vel = tb.is_translation ? tb.trans_vel[0] : Vec3<T>{T(0), T(0), T(0)};
      if (mv.is_rotat) {
        mv.pattern = tb.pattern;
        mv.pos_rp = tb.pos_rp;
        mv.rotat_vel = tb.rotat_vel;
      }
    }
    RW_CU(cudaMemcpyAsync(d_dyn, &d, sizeof(d), cudaMemcpyHostToDevice, st));
    RW_CU(cudaFuncSetAttribute(k_interaction<T, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               IX_CAP * IX_THREADS * (int)sizeof(unsigned)));
    RW_CU(cudaFuncSetAttribute(k_interaction<T, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               IX_CAP * IX_THREADS * (int)sizeof(unsigned)));
    RW_CU(cudaFuncSetAttribute(k_interaction2<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(Ix2Smem<T>)));
    RW_CU(cudaFuncSetAttribute(k_interaction2<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(Ix2Smem<T>)));
    search(0);  // the first cell sort; the lists are built with the first step's boundary stage
    RW_CU(cudaStreamSynchronize(st));
  }

  // ------------------------------------------------------------------------------
  // Stages.
  // ------------------------------------------------------------------------------
  void begin_step() override {
    k_begin<T><<<1, 1, 0, st>>>(d_dyn);
    check_launch();
  }
  void end_step() override {
    k_end<T><<<1, 1, 0, st>>>(P, d_dyn);
    check_launch();
  }
  // The search, then the candidate lists, built or updated (only when they do not
  // stand), before the boundary and corner stages so that the corner search walks them.
  void neighbor_search(int section) override {
    search(section);
    if (lists_kept()) {
      gated([&](cudaGraphConditionalHandle h) { k_build_gate<T><<<1, 1, 0, st>>>(P, S, d_dyn, h); },
            [&] {
              k_build_lists<T><<<nblk(P.np, 256), 256, 0, st>>>(P, S, d_dyn);
              k_rebuild_lists<T><<<4 * nsm, 256, 0, st>>>(P, S, d_dyn);
            });
      check_launch();
    }
  }
  // Soil candidate lists are kept only with the walk kernels.
  bool lists_kept() const { return ix_kernel == 0 && P.np > P.npb && S.nbg[0] && P.keep_lists; }
  void search(int section) {
    // Every kernel of the search returns at once when no particle changed cell since
    // the last one (Dyn::cells_dirty): keys, order, ranges and counts then stand.
    gated([&](cudaGraphConditionalHandle h) { k_search_gate<T><<<1, 1, 0, st>>>(d_dyn, h); },
          [&] {
            const int np = P.np;
            const int* dirty = &d_dyn->cells_dirty;
            k_keys<T><<<nblk(np, 256), 256, 0, st>>>(P, S, d_dyn);
            if (np > 1) k_check_sorted<<<nblk(np - 1, 256), 256, 0, st>>>(S.keys, np, need_ptr(), dirty);
            for (int pass = 0; pass < S.sort_passes; ++pass) {
              const int* ki = (pass & 1) ? S.tk : S.keys;
              const int* vi = (pass & 1) ? S.tv : S.vals;
              int* ko = (pass & 1) ? S.keys : S.tk;
              int* vo = (pass & 1) ? S.vals : S.tv;
              k_rs_upsweep<<<S.ntiles, RS_THREADS, 0, st>>>(ki, np, 8 * pass, S.hist, S.ntiles, need_ptr());
              k_rs_scan<<<256, RS_THREADS, 0, st>>>(S.hist, S.ntiles, S.dtot, need_ptr());
              k_rs_downsweep<<<S.ntiles, RS_THREADS, 0, st>>>(ki, vi, ko, vo, np, 8 * pass, S.hist, S.dtot, S.ntiles,
                                                              need_ptr());
            }
            k_clear_if<<<2 * nsm, 256, 0, st>>>(reinterpret_cast<unsigned*>(S.range), 2 * (size_t)P.ncell, dirty);
            k_ranges<T><<<nblk(np, 256), 256, 0, st>>>(P, S, d_dyn);
            k_count<T><<<1, 1, 0, st>>>(P, S, d_dyn);
            k_permute<T><<<nblk(np, 256), 256, 0, st>>>(P, S, d_dyn, section, compat_contact ? 1 : 0);
            if (P.npb > 0) {  // cells near contact walls, for the corner search
              k_clear_if<<<nsm, 256, 0, st>>>(reinterpret_cast<unsigned*>(S.near_wall), near_wall_words, dirty);
              k_mark_near_wall<T><<<nblk(P.npb, 256), 256, 0, st>>>(P, S, d_dyn);
            }
            // cells next to the cells particles entered or left, for a list update
            k_mark_dilate<T><<<nsm, 256, 0, st>>>(P, S, d_dyn);
          });
    k_flip<T><<<1, 1, 0, st>>>(P, d_dyn, section, 0, lists_kept() ? 1 : 0);
    if (ix_kernel == 1) chunk_list();
    check_launch();
  }

  // Column chunks of the chunked interaction kernel (rebuilt after every search while
  // that kernel is selected).
  void chunk_list() {
    if (ncol <= 0) return;
    k_col_count<T><<<nblk(ncol, 256), 256, 0, st>>>(P, S);
    k_col_scan<T><<<1, 1024, 0, st>>>(P, S, d_dyn);
    k_col_fill<T><<<nblk(ncol, 256), 256, 0, st>>>(P, S);
    check_launch();
  }
  void rigid() override {
    if (P.n_motion <= 0) return;
    k_flip<T><<<1, 1, 0, st>>>(P, d_dyn, -1, 1, 0);
    check_launch();
  }
  void adami() override {
    if (P.npb == 0) return;
    k_adami<T><<<nblk(P.npb, 128), 128, 0, st>>>(P, S, d_dyn);
    check_launch();
  }
  void corner() override {
    if (P.npm0 == 0) return;
    k_corner<T><<<nblk(P.npm0, 128), 128, 0, st>>>(P, S, d_dyn, cpar);
    check_launch();
  }
  void shepard_kernels(int only_filter_steps) {
    if (P.npm0 == 0) return;
    k_shepard<T><<<nblk(P.npm0, 128), 128, 0, st>>>(P, S, d_dyn, only_filter_steps);
    k_shepard_store<T><<<nblk(P.npm0, 256), 256, 0, st>>>(P, S, d_dyn, only_filter_steps);
    check_launch();
  }
  void shepard() override { shepard_kernels(0); }
  void interaction() override {
    const int n = P.np - P.npb;
    if (n > 0) {
      const size_t sm1 = IX_CAP * IX_THREADS * sizeof(unsigned);
      if (ix_kernel == 1) {
        const unsigned grid = (unsigned)std::max(max_chunks, (int)nblk(n, IX2_TB));
        if (strict_fp) k_interaction2<T, true><<<grid, IX2_TB, sizeof(Ix2Smem<T>), st>>>(P, S, d_dyn, cpar);
        else k_interaction2<T, false><<<grid, IX2_TB, sizeof(Ix2Smem<T>), st>>>(P, S, d_dyn, cpar);
      } else {
        const unsigned g = nblk(n, IX_THREADS);
        // the scan launch (only for particles without a list, and deleted slots), then
        // the walk (the lists were built or updated at the end of the search)
        gated([&](cudaGraphConditionalHandle h) { k_scan_gate<T><<<1, 1, 0, st>>>(P, S, d_dyn, h); },
              [&] {
                if (strict_fp) k_interaction<T, true, false><<<g, IX_THREADS, sm1, st>>>(P, S, d_dyn, cpar);
                else k_interaction<T, false, false><<<g, IX_THREADS, sm1, st>>>(P, S, d_dyn, cpar);
              });
        const unsigned gw = nblk(n, walk_threads);
        if (strict_fp) k_interaction<T, true, true><<<gw, walk_threads, 0, st>>>(P, S, d_dyn, cpar);
        else k_interaction<T, false, true><<<gw, walk_threads, 0, st>>>(P, S, d_dyn, cpar);
      }
      check_launch();
    }
    cpar ^= 1;
  }
  void predictor() override {
    if (P.closure) return integrate_closure(0);
    k_predictor<T><<<nblk(P.np, integ_threads), integ_threads, 0, st>>>(P, S, d_dyn);
    check_launch();
  }
  void corrector() override {
    if (P.closure) return integrate_closure(1);
    k_corrector<T><<<nblk(P.npb + P.npm0, integ_threads), integ_threads, 0, st>>>(P, S, d_dyn);
    check_launch();
  }
  // An integrator stage with the learned closure: one persistent launch, four 128-thread
  // blocks per SM, each looping over tiles of rows (k_integrate_cl).
  void integrate_closure(int stage) {
    const long tiles = nblk(P.npb, mlp::TILE) + nblk(P.np - P.npb, mlp::TILE);
    const unsigned grid = (unsigned)std::max(1L, std::min(tiles, 4L * nsm));
    const mlp::Net net = mlp::net_view(cl_net);
    if (stage == 0)
      k_integrate_cl<T, 0><<<grid, mlp::TILE, sizeof(mlp::FwdSmem), st>>>(P, S, d_dyn, net, cl_trust, d_clstats);
    else
      k_integrate_cl<T, 1><<<grid, mlp::TILE, sizeof(mlp::FwdSmem), st>>>(P, S, d_dyn, net, cl_trust, d_clstats);
    check_launch();
  }

  // ------------------------------------------------------------------------------
  // Learned closure.
  // ------------------------------------------------------------------------------
  int set_closure(rw_mlp* net, double margin) override {
    if (gexec) {  // the closure launches are part of the captured step
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
    ++generation;
    if (!net) {
      P.closure = 0;
      cl_net = nullptr;
      return RW_OK;
    }
    if (mlp::device_of(net) != device) {
      err = "rw_set_closure: the network lives on another device";
      return RW_EINVAL;
    }
    float lo[mlp::IN], hi[mlp::IN], tmax = 0.0f;
    const rw_status s = rw_mlp_feature_ranges(net, lo, hi, &tmax);
    if (s != RW_OK) {
      err = std::string("rw_set_closure: ") + rw_mlp_last_error(net);
      return s;
    }
    for (int k = 0; k < mlp::IN; ++k) {
      const float w = hi[k] - lo[k];
      cl_trust.lo[k] = lo[k] - (float)margin * w;
      cl_trust.hi[k] = hi[k] + (float)margin * w;
    }
    cl_trust.out_max = tmax * (1.0f + (float)margin);
    cl_trust.err_max = (float)cl_err_max;
    RW_CU(cudaSetDevice(device));
    RW_CU(cudaFuncSetAttribute(k_integrate_cl<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(mlp::FwdSmem)));
    RW_CU(cudaFuncSetAttribute(k_integrate_cl<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(mlp::FwdSmem)));
    RW_CU(cudaMemsetAsync(d_clstats, 0, 4 * sizeof(double), st));
    RW_CU(cudaStreamSynchronize(st));
    P.closure = 1;
    cl_net = net;
    return RW_OK;
  }
  void closure_stats(double* out) override {
    double s[4];
    RW_CU(cudaMemcpyAsync(s, d_clstats, sizeof(s), cudaMemcpyDeviceToHost, st));
    RW_CU(cudaStreamSynchronize(st));
    out[0] = s[0];
    out[1] = s[1];
    out[2] = s[1] > 0 ? s[2] / s[1] : 0.0;
    out[3] = s[3];
  }
  void list_totals(long long* out) override {
    out[0] = out[1] = 0;
    if (!S.nbg[0]) return;
    Dyn<T> d = dyn_host();
    if (!d.list_ok) return;
    unsigned long long* tot = nullptr;
    RW_CU(cudaMallocAsync((void**)&tot, 2 * sizeof(unsigned long long), st));
    RW_CU(cudaMemsetAsync(tot, 0, 2 * sizeof(unsigned long long), st));
    k_list_totals<<<2 * nsm, 256, 0, st>>>(S.nbg_cnt[d.lbuf], d.npm, tot);
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(tot, st);
    RW_CU(e);
    RW_CU(cudaStreamSynchronize(st));
    out[0] = (long long)h[0];
    out[1] = (long long)h[1];
  }
  long long collect(rw_mlp* net, int stride, const Augment& aug) override {
    if (mlp::device_of(net) != device) throw Fail(RW_EINVAL, "rw_mlp_collect: the network lives on another device");
    const long long avail = mlp::free_slots(net);
    if (avail <= 0) return 0;
    float *x = nullptr, *t = nullptr;
    mlp::next_slot(net, &x, &t);
    RW_CU(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st));
    const long n = (P.npm0 + stride - 1) / stride;
    k_collect<T><<<nblk(n, 256), 256, 0, st>>>(P, S, d_dyn, x, t, avail, d_count, stride, aug);
    check_launch();
    unsigned long long cnt = 0;
    RW_CU(cudaMemcpyAsync(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    RW_CU(cudaStreamSynchronize(st));
    const long long added = std::min((long long)cnt, avail);
    mlp::commit(net, added);
    return added;
  }

  // One whole step (RunSimulation's loop body, src/loquat.cu:548-561).
  void launch_step() {
    begin_step();
    neighbor_search(0);
    rigid();
    adami();
    corner();
    if (P.stress_shepard_filter != 0) shepard_kernels(1);
    interaction();
    predictor();
    neighbor_search(1);
    adami();
    corner();
    interaction();
    corrector();
    end_step();
  }

  void step(int n) override {
    if (n <= 0) return;
    ensure_graph();
    for (int k = 0; k < n; ++k) RW_CU(cudaGraphLaunch(gexec, st));
  }

  // One whole step captured as a graph (not instantiated); the caller owns it.
  // cond: gate the search, the list build and the scan launch with conditional nodes
  // (gated()).  The batch's fallback nests step graphs as child graphs, without.
  cudaGraph_t capture_step(bool cond = false) {
    cudaGraph_t g = nullptr;
    const int c0 = cpar;
    RW_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    allow_cond = cond;
    try {
      launch_step();
    } catch (...) {
      allow_cond = false;
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      cpar = c0;
      throw;
    }
    allow_cond = false;
    RW_CU(cudaStreamEndCapture(st, &g));
    cpar = c0;  // the step runs two interactions: parity is back where it started
    return g;
  }

  void ensure_graph() {
    if (!gexec || g_cpar != cpar) {
      if (gexec) {
        cudaGraphExecDestroy(gexec);
        gexec = nullptr;
      }
      cudaError_t e = cudaErrorNotSupported;
      if (graph_gates) {
        try {
          cudaGraph_t g = capture_step(true);
          e = cudaGraphInstantiate(&gexec, g, 0);
          cudaGraphDestroy(g);
        } catch (const Fail&) {  // capture with conditional nodes refused
          e = cudaErrorNotSupported;
        }
      }
      graph_cond = e == cudaSuccess;
      if (e != cudaSuccess) {  // gates off, or a driver without conditional nodes: plain step graph
        cudaGetLastError();
        gexec = nullptr;
        cudaGraph_t g = capture_step(false);
        e = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
      }
      RW_CU(e);
      g_cpar = cpar;
    }
  }

  // Kernels launched by one whole step (launch_step), for launch accounting.
  int kernels_per_step() const {
    // keys, check, sort, clear + ranges, count, permute, [clear + near-wall marks], mark
    // dilation, flip, [chunks]
    const int search = 2 + 3 * S.sort_passes + 6 + (P.npb > 0 ? 2 : 0) + (ncol > 0 && ix_kernel == 1 ? 3 : 0);
    // chunked, or [list build + rebuild (end of the search)] + scan + walk
    const int ix = ix_kernel == 1 ? 1 : (lists_kept() ? 4 : 2);
    int k = 1 + 2 * search + 2 * (2 + ix) + 1 + 1 + 1;  // begin, 2 searches, 2x(adami, corner, interaction), predictor, corrector, end
    if (P.n_motion > 0) k += 1;
    if (P.stress_shepard_filter != 0) k += 2;
    if (P.npb == 0) k -= 2;
    return k;
  }

  void profile(int nsteps, double* ms, int n, int* kps) override {
    cudaEvent_t ev[RW_STAGE_COUNT_ + 1];
    for (auto& e : ev) RW_CU(cudaEventCreate(&e));
    std::vector<double> acc(RW_STAGE_COUNT_, 0.0);
    for (int it = 0; it < nsteps; ++it) {
      begin_step();
      RW_CU(cudaEventRecord(ev[0], st));
      neighbor_search(0);
      RW_CU(cudaEventRecord(ev[1], st));
      rigid();
      RW_CU(cudaEventRecord(ev[2], st));
      adami();
      RW_CU(cudaEventRecord(ev[3], st));
      corner();
      if (P.stress_shepard_filter != 0) shepard_kernels(1);
      RW_CU(cudaEventRecord(ev[4], st));
      interaction();
      RW_CU(cudaEventRecord(ev[5], st));
      predictor();
      RW_CU(cudaEventRecord(ev[6], st));
      neighbor_search(1);
      RW_CU(cudaEventRecord(ev[7], st));
      adami();
      RW_CU(cudaEventRecord(ev[8], st));
      corner();
      RW_CU(cudaEventRecord(ev[9], st));
      interaction();
      RW_CU(cudaEventRecord(ev[10], st));
      corrector();
      RW_CU(cudaEventRecord(ev[11], st));
      end_step();
      RW_CU(cudaEventSynchronize(ev[11]));
      for (int k = 0; k < RW_STAGE_COUNT_; ++k) {
        float t = 0.f;
        RW_CU(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
        acc[k] += t;
      }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < n && k < RW_STAGE_COUNT_; ++k) ms[k] = nsteps > 0 ? acc[k] / nsteps : 0.0;
    if (kps) *kps = kernels_per_step();
  }

  double step_timed(int n) override {
    cudaEvent_t e0, e1;
    RW_CU(cudaEventCreate(&e0));
    RW_CU(cudaEventCreate(&e1));
    ensure_graph();  // capture outside the timed interval
    RW_CU(cudaEventRecord(e0, st));
    for (int k = 0; k < n; ++k) RW_CU(cudaGraphLaunch(gexec, st));
    RW_CU(cudaEventRecord(e1, st));
    RW_CU(cudaEventSynchronize(e1));
    float ms = 0.f;
    RW_CU(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (double)ms;
  }

  cudaGraph_t step_graph(bool gates) override { return capture_step(gates && graph_gates); }
  void launch_into_capture(bool gates) override {
    const int c0 = cpar;
    allow_cond = gates && graph_gates;
    try {
      launch_step();
    } catch (...) {
      allow_cond = false;
      cpar = c0;
      throw;
    }
    allow_cond = false;
    cpar = c0;  // the step runs two interactions: parity is back where it started
  }

  // Defaults of the reference's profile (src/utilities.cu:284-292,336): wall face at
  // 0.04 + bound_thickness - 0.005 t, top at 0.04 + 1.0 + bound_thickness, bins of dr,
  // (int)(1/dr) bins.  NaN arguments select them.
  void wall_profile(double x_wall, double z_top, double dz, int nbins, double* out) override {
    Dyn<T> d = dyn_host();
    if (x_wall != x_wall) x_wall = (double)(T(0.04f) + P.bound_thickness) - (double)d.time_f * 0.005;
    if (z_top != z_top) z_top = (double)(T(0.04f) + T(1.0f) + P.bound_thickness);
    if (dz != dz || dz <= 0) dz = (double)P.dr;
    if (nbins <= 0) nbins = (int)(T(1.0f) / P.dr);
    int* last = nullptr;
    double* dout = nullptr;
    RW_CU(cudaMallocAsync((void**)&last, 3 * (size_t)nbins * sizeof(int), st));
    RW_CU(cudaMallocAsync((void**)&dout, 4 * (size_t)nbins * sizeof(double), st));
    RW_CU(cudaMemsetAsync(last, 0xff, 3 * (size_t)nbins * sizeof(int), st));
    const int n = P.np - P.npb;
    if (n > 0) k_profile_claim<T><<<nblk(n, 256), 256, 0, st>>>(P, S, d_dyn, x_wall, z_top, dz, nbins, last);
    k_profile_read<T><<<nblk(nbins, 128), 128, 0, st>>>(P, S, cpar, nbins, last, dout);
    check_launch();
    RW_CU(cudaMemcpyAsync(out, dout, 4 * (size_t)nbins * sizeof(double), cudaMemcpyDeviceToHost, st));
    RW_CU(cudaFreeAsync(last, st));
    RW_CU(cudaFreeAsync(dout, st));
    RW_CU(cudaStreamSynchronize(st));
  }
  cudaStream_t stream() const override { return st; }
  int soil_count() override { return dyn_host().npm; }

  int sync() override {
    RW_CU(cudaStreamSynchronize(st));
    if (int rc = wait_save()) return rc;  // a save written in the background
    Dyn<T> d = dyn_host();
    if (d.err) {
      err = "device error word " + std::to_string(d.err);
      return RW_EDEVICE;
    }
    return RW_OK;
  }

  void info(rw_info* o) override {
    Dyn<T> d = dyn_host();
    std::memset(o, 0, sizeof(*o));
    o->np = P.np;
    o->npb = P.npb;
    o->npm = d.npm;
    o->np_delete_m = d.np_delete_m;
    o->ncell = P.ncell;
    o->step = d.step;
    o->scalar_bytes = (int)sizeof(T);
    o->device_err = (int)d.err;
    for (int k = 0; k < 3; ++k) o->cell_num[k] = P.cell_num[k];
    o->n_motion = P.n_motion;
    o->time = d.time_d;
    o->dt = (double)P.dt;
    o->h = (double)P.h;
    o->dr = (double)P.dr;
    o->n_sorts = d.n_sorts;
    o->n_list_reuse = d.n_reuse;
    o->n_search_skipped = d.n_search_skipped;
    o->n_scan_skipped = d.n_scan_skipped;
    o->n_build_skipped = d.n_build_skipped;
    // kernels of the captured step graph when every gated body runs: the plain step
    // plus one gate per search and two per interaction (list build, scan launch)
    const int ix_gates = ix_kernel == 0 && P.np > P.npb ? (lists_kept() ? 4 : 2) : 0;
    o->graph_kernels = kernels_per_step() + (graph_cond ? 2 + ix_gates : 0);
    o->search_body_kernels = 2 + 3 * S.sort_passes + 5 + (P.npb > 0 ? 2 : 0);
    o->build_body_kernels = 2;
    o->n_list_updates = d.n_updates;
    o->n_lists_rebuilt = d.n_rebuilt;
    o->time_max = cparams.time_max;
    o->output_frequency = cparams.output_frequency;
    o->ix_kernel = ix_kernel;
    o->walk_threads = walk_threads;
    o->integrator_threads = integ_threads;
  }

  bool lists_fit() const { return (size_t)IX_CAP * (size_t)(P.np - P.npb) < ((size_t)1 << 31); }
  // Kept candidate lists: radius 2h + skin; all rebuilt once any particle may have moved
  // 0.45 skin since the last full build (two particles then close in by at most 0.9
  // skin, so every pair within 2h is still listed by a list built since).
  void set_skin(double skin_h) {
    const double h_d = (double)P.h;
    const double skin = skin_h * h_d;
    const double rlist = (2.0 * h_d + skin) * (1.0 + 1e-4);
    P.keep_lists = (skin_h > 0.0 && lists_fit()) ? 1 : 0;
    P.r2_list = (T)(rlist * rlist);
    P.disp_lim = (float)(0.45 * skin);
    P.disp_eps = (float)(std::ldexp(2.0 * h_d, -20));
  }

  int set_option(int opt, double v) override {
    if (opt == RW_OPT_LIST_SKIN) {
      if (!(v >= 0.0 && v <= 1.0)) {
        err = "list skin must be within [0, 1] h";
        return RW_EINVAL;
      }
      set_skin(v);
      drop_lists();
    } else if (opt == RW_OPT_WALL_FRICTION) {
      P.wall_fric = (T)v;
    } else if (opt == RW_OPT_MIXED_PRECISION) {
      if (sizeof(T) != 4 && v != 0.0) {
        err = "the precision form applies to float contexts";
        return RW_EINVAL;
      }
      P.mixed = v != 0.0 ? 1 : 0;
    } else if (opt == RW_OPT_STRICT_FP) {
      strict_fp = v != 0.0;
    } else if (opt == RW_OPT_GRAPH_GATES) {
      graph_gates = v != 0.0;
    } else if (opt == RW_OPT_ASYNC_SAVE) {
      if (int rc = wait_save()) return rc;
      async_save = v != 0.0;
    } else if (opt == RW_OPT_CLOSURE_MAX_ERR) {
      if (!(v >= 0.0)) {
        err = "closure error bound must be >= 0";
        return RW_EINVAL;
      }
      cl_err_max = v;
      cl_trust.err_max = (float)v;
    } else if (opt == RW_OPT_INTERACTION_KERNEL) {
      if (v != 0.0 && v != 1.0) return RW_EINVAL;
      const int was = ix_kernel;
      ix_kernel = (int)v;
      if (ix_kernel == 1 && was != 1) chunk_list();  // chunks of the current ordering
    } else if (opt == RW_OPT_WALK_THREADS) {
      if (v != 64.0 && v != 128.0) {
        err = "walk threads per block must be 64 or 128";
        return RW_EINVAL;
      }
      walk_threads = (int)v;
    } else if (opt == RW_OPT_INTEGRATOR_THREADS) {
      if (v != 128.0 && v != 256.0) {
        err = "integrator threads per block must be 128 or 256";
        return RW_EINVAL;
      }
      integ_threads = (int)v;
    } else if (opt == RW_OPT_COMPAT_CONTACT) {
      if (v == 0.0) {
        err = "contact state following particles (RW_OPT_COMPAT_CONTACT=0) is not available";
        return RW_EINVAL;
      }
      compat_contact = true;
    } else {
      return RW_EINVAL;
    }
    if (gexec) {  // parameters are baked into the captured graph
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
    ++generation;
    return RW_OK;
  }

  // ------------------------------------------------------------------------------
  // Arrays in the reference's layouts.
  // ------------------------------------------------------------------------------
  static size_t row_bytes(int which) {
    switch (which) {
      case RW_ARR_CODES: case RW_ARR_CELLPOS: return 16;
      case RW_ARR_STR: case RW_ARR_STN: case RW_ARR_ACESTN: case RW_ARR_STR_INI: case RW_ARR_STN_INI: return 6 * sizeof(T);
      case RW_ARR_CONTACT_MAG: return 9 * sizeof(T);
      case RW_ARR_PART_IDX: case RW_ARR_CELL_BEG: case RW_ARR_CELL_END: return 4;
      default: return 4 * sizeof(T);
    }
  }
  size_t rows(int which) const {
    if (which == RW_ARR_NORMAL) return P.npb;
    if (which == RW_ARR_CELL_BEG || which == RW_ARR_CELL_END) return P.ncell;
    return P.np;
  }

  int get_array(int which, void* dst, size_t bytes) override {
    if (which < 0 || which >= RW_ARR_COUNT_) return RW_EINVAL;
    const size_t n = rows(which);
    if (bytes != n * row_bytes(which)) {
      err = "rw_get_array: expected " + std::to_string(n * row_bytes(which)) + " bytes";
      return RW_EINVAL;
    }
    RW_CU(cudaStreamSynchronize(st));
    Dyn<T> d = dyn_host();
    const int c = d.cur_main, cn = d.cur_nrm, ci = d.cur_ini;
    T* o = (T*)dst;
    auto put4 = [&](const V4<T>* src) {
      auto h = down(src, n);
      std::memcpy(dst, h.data(), n * sizeof(V4<T>));
    };
    auto put6 = [&](const V4<T>* a, const V2<T>* b) {
      auto ha = down(a, n);
      auto hb = down(b, n);
      for (size_t i = 0; i < n; ++i) {
        o[6 * i + 0] = ha[i].x; o[6 * i + 1] = ha[i].y; o[6 * i + 2] = ha[i].z;
        o[6 * i + 3] = ha[i].w; o[6 * i + 4] = hb[i].x; o[6 * i + 5] = hb[i].y;
      }
    };
    switch (which) {
      case RW_ARR_CODES: { auto h = down(S.codes[c], n); std::memcpy(dst, h.data(), bytes); break; }
      case RW_ARR_CELLPOS: { auto h = down(S.cellpos[c], n); std::memcpy(dst, h.data(), bytes); break; }
      case RW_ARR_POSPRES: put4(S.pos[c]); break;
      case RW_ARR_POSPRES_ORI: put4(S.pos_ori[c]); break;
      case RW_ARR_VELRHOP: put4(S.vel[c]); break;
      case RW_ARR_IDMASSIDX: put4(S.idm[c]); break;
      case RW_ARR_STR: put6(S.str_a[c], S.str_b[c]); break;
      case RW_ARR_STN: put6(S.stn_a[c], S.stn_b[c]); break;
      case RW_ARR_NORMAL: put4(S.normal[cn]); break;
      case RW_ARR_CONTACT_MAG: {
        auto hf = down(S.cf[cpar], n);
        auto hy = down(S.cny, n);
        auto hz = down(S.cvz, n);
        for (size_t i = 0; i < n; ++i) {
          o[9 * i + 0] = hf[i].x; o[9 * i + 1] = hf[i].y; o[9 * i + 2] = hf[i].z;
          o[9 * i + 3] = hy[i].x; o[9 * i + 4] = hy[i].y; o[9 * i + 5] = hy[i].z;
          o[9 * i + 6] = hz[i].x; o[9 * i + 7] = hz[i].y; o[9 * i + 8] = hz[i].z;
        }
        break;
      }
      case RW_ARR_CONTACT_VAR: put4(S.cv[cpar]); break;
      case RW_ARR_ACCAD: put4(S.accad); break;
      case RW_ARR_SPIN: put4(S.spin); break;
      case RW_ARR_ACESTN: put6(S.ace_a, S.ace_b); break;
      case RW_ARR_POSPRES_INI: put4(S.pos_ini[ci]); break;
      case RW_ARR_VELRHOP_INI: put4(S.vel_ini[ci]); break;
      case RW_ARR_STR_INI: put6(S.stri_a[ci], S.stri_b[ci]); break;
      case RW_ARR_STN_INI: put6(S.stni_a[ci], S.stni_b[ci]); break;
      case RW_ARR_PART_IDX: {
        int* oi = (int*)dst;
        if (d.need_sort) {
          auto h = down(S.sperm, n);
          std::memcpy(oi, h.data(), bytes);
        } else {
          for (size_t i = 0; i < n; ++i) oi[i] = (int)i;
        }
        break;
      }
      case RW_ARR_CELL_BEG: case RW_ARR_CELL_END: {
        auto h = down(S.range, n);
        int* oi = (int*)dst;
        for (size_t k = 0; k < n; ++k) {
          const bool occ = h[k].y > h[k].x;
          oi[k] = occ ? (which == RW_ARR_CELL_BEG ? h[k].x : h[k].y) : -1;
        }
        break;
      }
      case RW_ARR_POS_ABS: {
        auto hp = down(S.pos[c], n);
        auto hc = down(S.cellpos[c], n);
        for (size_t i = 0; i < n; ++i) {
          o[4 * i + 0] = hp[i].x + (T)hc[i].x * P.two_h;
          o[4 * i + 1] = hp[i].y + (T)hc[i].y * P.two_h;
          o[4 * i + 2] = hp[i].z + (T)hc[i].z * P.two_h;
          o[4 * i + 3] = hp[i].w;
        }
        break;
      }
      default: return RW_EINVAL;
    }
    return RW_OK;
  }

  int set_array(int which, const void* src, size_t bytes) override {
    if (which < 0 || which >= RW_ARR_COUNT_ || which == RW_ARR_POS_ABS || which == RW_ARR_PART_IDX ||
        which == RW_ARR_CELL_BEG || which == RW_ARR_CELL_END)
      return RW_EINVAL;
    const size_t n = rows(which);
    if (bytes != n * row_bytes(which)) {
      err = "rw_set_array: expected " + std::to_string(n * row_bytes(which)) + " bytes";
      return RW_EINVAL;
    }
    RW_CU(cudaStreamSynchronize(st));
    Dyn<T> d = dyn_host();
    const int c = d.cur_main, cn = d.cur_nrm, ci = d.cur_ini;
    const T* s = (const T*)src;
    auto get4 = [&](V4<T>* dstp) {
      std::vector<V4<T>> h(n);
      std::memcpy(h.data(), src, n * sizeof(V4<T>));
      up(dstp, h);
    };
    auto get6 = [&](V4<T>* a, V2<T>* b) {
      std::vector<V4<T>> ha(n);
      std::vector<V2<T>> hb(n);
      for (size_t i = 0; i < n; ++i) {
        ha[i] = V4<T>{s[6 * i], s[6 * i + 1], s[6 * i + 2], s[6 * i + 3]};
        hb[i] = V2<T>{s[6 * i + 4], s[6 * i + 5]};
      }
      up(a, ha);
      up(b, hb);
    };
    switch (which) {
      case RW_ARR_CODES: { std::vector<int4> h(n); std::memcpy(h.data(), src, bytes); up(S.codes[c], h); break; }
      case RW_ARR_CELLPOS: { std::vector<int4> h(n); std::memcpy(h.data(), src, bytes); up(S.cellpos[c], h); break; }
      case RW_ARR_POSPRES: get4(S.pos[c]); break;
      case RW_ARR_POSPRES_ORI: get4(S.pos_ori[c]); break;
      case RW_ARR_VELRHOP: get4(S.vel[c]); break;
      case RW_ARR_IDMASSIDX: get4(S.idm[c]); break;
      case RW_ARR_STR: get6(S.str_a[c], S.str_b[c]); break;
      case RW_ARR_STN: get6(S.stn_a[c], S.stn_b[c]); break;
      case RW_ARR_NORMAL: get4(S.normal[cn]); break;
      case RW_ARR_CONTACT_MAG: {
        std::vector<V4<T>> hf(n), hy(n), hz(n);
        for (size_t i = 0; i < n; ++i) {
          hf[i] = V4<T>{s[9 * i + 0], s[9 * i + 1], s[9 * i + 2], T(0)};
          hy[i] = V4<T>{s[9 * i + 3], s[9 * i + 4], s[9 * i + 5], T(0)};
          hz[i] = V4<T>{s[9 * i + 6], s[9 * i + 7], s[9 * i + 8], T(0)};
        }
        up(S.cf[cpar], hf);
        up(S.cny, hy);
        up(S.cvz, hz);
        break;
      }
      case RW_ARR_CONTACT_VAR: get4(S.cv[cpar]); break;
      case RW_ARR_ACCAD: get4(S.accad); break;
      case RW_ARR_SPIN: get4(S.spin); break;
      case RW_ARR_ACESTN: get6(S.ace_a, S.ace_b); break;
      case RW_ARR_POSPRES_INI: get4(S.pos_ini[ci]); break;
      case RW_ARR_VELRHOP_INI: get4(S.vel_ini[ci]); break;
      case RW_ARR_STR_INI: get6(S.stri_a[ci], S.stri_b[ci]); break;
      case RW_ARR_STN_INI: get6(S.stni_a[ci], S.stni_b[ci]); break;
      default: return RW_EINVAL;
    }
    drop_lists();
    return RW_OK;
  }

  // State written from the host: the kept candidate lists no longer describe it.
  void drop_lists() {
    Dyn<T> d = dyn_host();
    d.list_ok = 0;
    d.ix_mode = 0;
    d.host_dirty = 1;
    d.cells_dirty = 1;
    RW_CU(cudaMemcpyAsync(d_dyn, &d, sizeof(d), cudaMemcpyHostToDevice, st));
    RW_CU(cudaStreamSynchronize(st));
  }

  void set_counters(double time, int step_, int npm, int np_delete_m) override {
    Dyn<T> d = dyn_host();
    d.time_d = time;
    d.time_f = (T)time;
    d.step = step_;
    d.npm = npm;
    d.np_delete_m = np_delete_m;
    d.list_ok = 0;
    d.ix_mode = 0;
    d.host_dirty = 1;
    d.cells_dirty = 1;
    RW_CU(cudaMemcpyAsync(d_dyn, &d, sizeof(d), cudaMemcpyHostToDevice, st));
    RW_CU(cudaStreamSynchronize(st));
  }

  void wall_force(int mode, int wall_id, const double* strip, double* out) override {
    wall_force_kernels(st, mode, wall_id, strip);
    RW_CU(cudaMemcpyAsync(out, S.wsum + 3 * WF_BLOCKS, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    RW_CU(cudaStreamSynchronize(st));
  }
  void wall_force_enqueue(cudaStream_t s, int mode, int wall_id, const double* strip, double* d_out) override {
    wall_force_kernels(s, mode, wall_id, strip);
    RW_CU(cudaMemcpyAsync(d_out, S.wsum + 3 * WF_BLOCKS, 3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  void wall_force_kernels(cudaStream_t s, int mode, int wall_id, const double* strip) {
    double xmax, zmin, zmax;
    if (strip) {
      xmax = strip[0];
      zmin = strip[1];
      zmax = strip[2];
    } else {  // the reference's strip, src/utilities.cu:619-621
      xmax = (double)(T(0.04f) + P.bound_thickness + P.dr * T(3));
      zmin = (double)(P.bound_thickness + T(0.04f));
      zmax = (double)(P.bound_thickness + T(0.04f) + T(1.0f));
    }
    k_wall_force<T><<<WF_BLOCKS, WF_THREADS, 0, s>>>(P, S, d_dyn, cpar, mode, wall_id, xmax, zmin, zmax);
    k_wall_force_final<<<1, 32, 0, s>>>(S.wsum, WF_BLOCKS);
    check_launch();
  }

  // Saving (src/loquat.cu:439-482): output_N.xml + particles with the Shepard-smoothed
  // stress (StressSavingRegularization, src/field_smoothing.cu:103-111) + time history.
  void save(const char* outdir) override {
    if (int rc = wait_save()) throw Fail(rc, "the previous save: " + err);
    std::string dir = outdir ? outdir : ".";
    ::mkdir(dir.c_str(), 0755);
    Dyn<T> d = dyn_host();
    const int c = d.cur_main;
    const size_t np = P.np;
    // tensor2d_cache = str, then Shepard over material particles into the cache.
    RW_CU(cudaMemcpyAsync(S.tc_a, S.str_a[c], np * sizeof(V4<T>), cudaMemcpyDeviceToDevice, st));
    RW_CU(cudaMemcpyAsync(S.tc_b, S.str_b[c], np * sizeof(V2<T>), cudaMemcpyDeviceToDevice, st));
    if (P.npm0 > 0) {
      k_shepard<T><<<nblk(P.npm0, 128), 128, 0, st>>>(P, S, d_dyn, 0);
      check_launch();
    }
    // The arrays a save writes, copied into one page-locked staging block with
    // asynchronous copies and one wait; the conversion to the output values (absolute
    // positions formed in the context's precision, as rw_get_array forms them) is done
    // by the writing task, on several host threads.  The block stays in use until that
    // task ends; the next save waits for it first.
    const size_t npb = P.npb, n4 = sizeof(V4<T>), n2 = sizeof(V2<T>);
    size_t off = 0;
    auto take = [&](size_t b) {
      const size_t o = off;
      off += (b + 255) & ~(size_t)255;
      return o;
    };
    const size_t o_codes = take(np * 16), o_pos = take(np * n4), o_cell = take(np * 16), o_vel = take(np * n4),
                 o_acc = take(np * n4), o_idm = take(np * n4), o_nrm = take(npb * n4), o_ta = take(np * n4),
                 o_tb = take(np * n2), o_sa = take(np * n4), o_sb = take(np * n2);
    if (off > stage_bytes) {
      if (stage_h) cudaFreeHost(stage_h);
      stage_h = nullptr;
      stage_bytes = 0;
      RW_CU(cudaMallocHost(reinterpret_cast<void**>(&stage_h), off));
      stage_bytes = off;
    }
    auto get = [&](size_t o, const void* src, size_t b) {
      if (b) RW_CU(cudaMemcpyAsync(stage_h + o, src, b, cudaMemcpyDeviceToHost, st));
    };
    get(o_codes, S.codes[c], np * 16);
    get(o_pos, S.pos[c], np * n4);
    get(o_cell, S.cellpos[c], np * 16);
    get(o_vel, S.vel[c], np * n4);
    get(o_acc, S.accad, np * n4);
    get(o_idm, S.idm[c], np * n4);
    get(o_nrm, S.normal[d.cur_nrm], npb * n4);
    get(o_ta, S.tc_a, np * n4);
    get(o_tb, S.tc_b, np * n2);
    get(o_sa, S.stn_a[c], np * n4);
    get(o_sb, S.stn_b[c], np * n2);
    RW_CU(cudaStreamSynchronize(st));
    const unsigned char* sh = stage_h;
    const T two_h = P.two_h;
    const int npm_now = d.npm;
    auto make_frame = [=]() {
      Frame f;
      f.np = (int)np;
      f.npb = (int)npb;
      f.npm = npm_now;
      f.codes.resize(4 * np);
      f.pos.resize(4 * np);
      f.vel.resize(4 * np);
      f.acc.resize(4 * np);
      f.idm.resize(4 * np);
      f.normal.resize(4 * npb);
      f.str.resize(6 * np);
      f.stn.resize(6 * np);
      const auto* codes = reinterpret_cast<const int32_t*>(sh + o_codes);
      const auto* pos = reinterpret_cast<const V4<T>*>(sh + o_pos);
      const auto* cell = reinterpret_cast<const int4*>(sh + o_cell);
      const auto* vel = reinterpret_cast<const V4<T>*>(sh + o_vel);
      const auto* acc = reinterpret_cast<const V4<T>*>(sh + o_acc);
      const auto* idm = reinterpret_cast<const V4<T>*>(sh + o_idm);
      const auto* nrm = reinterpret_cast<const V4<T>*>(sh + o_nrm);
      const auto* ta = reinterpret_cast<const V4<T>*>(sh + o_ta);
      const auto* tb = reinterpret_cast<const V2<T>*>(sh + o_tb);
      const auto* sa = reinterpret_cast<const V4<T>*>(sh + o_sa);
      const auto* sb = reinterpret_cast<const V2<T>*>(sh + o_sb);
      auto put4 = [](double* o, const V4<T>& v) {
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
      };
      auto put6 = [](double* o, const V4<T>& a, const V2<T>& b) {
        o[0] = a.x;
        o[1] = a.y;
        o[2] = a.z;
        o[3] = a.w;
        o[4] = b.x;
        o[5] = b.y;
      };
      auto rows = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
          std::memcpy(&f.codes[4 * i], codes + 4 * i, 16);
          const V4<T> p = pos[i];
          const int4 cc = cell[i];
          const V4<T> pa{p.x + (T)cc.x * two_h, p.y + (T)cc.y * two_h, p.z + (T)cc.z * two_h, p.w};
          put4(&f.pos[4 * i], pa);
          put4(&f.vel[4 * i], vel[i]);
          put4(&f.acc[4 * i], acc[i]);
          put4(&f.idm[4 * i], idm[i]);
          if (i < npb) put4(&f.normal[4 * i], nrm[i]);
          put6(&f.str[6 * i], ta[i], tb[i]);
          put6(&f.stn[6 * i], sa[i], sb[i]);
        }
      };
      const int nth = np < 65536 ? 1 : (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
      std::vector<std::thread> th;
      for (int t = 1; t < nth; ++t) th.emplace_back(rows, np * t / nth, np * (t + 1) / nth);
      rows(0, np / nth);
      for (auto& x : th) x.join();
      return f;
    };
    // RunSimulation writes the initial configuration with the case's output number
    // (src/loquat.cu:533-537); every later Saving increments first (src/loquat.cu:456).
    const bool initial = saves++ == 0;
    if (!initial) output_number++;
    const int onum = output_number;
    // The time written is the reference's par_host->time: that of the last step begun
    // (StepCalculation, src/loquat.cu:366-374), the case's time before any step.
    // and the time step is the parameter file's until StepCalculation first sets it.
    const double dt_out = initial && d.step == 0 ? (double)(T)cparams.dt : (double)P.dt;
    const double time_out = (double)d.time_f;
    // stress_zz<N>.txt and the time history need the device: computed here, written below
    std::vector<double> prof;
    double wf[3] = {0.0, 0.0, 0.0};
    const int nb = (int)(T(1.0f) / P.dr);
    if (!initial) {
      prof.assign(4 * (size_t)std::max(nb, 1), 0.0);
      const double nan = std::numeric_limits<double>::quiet_NaN();
      wall_profile(nan, nan, nan, nb, prof.data());
      wall_force(1, 10, nullptr, wf);
    }
    // The files: formatted and written here, or by a background task with
    // RW_OPT_ASYNC_SAVE (one in flight; the next save, rw_synchronize or the context's
    // end waits for it and reports its status).
    auto job = [dir, onum, dt_out, time_out, initial, nb, fmt = P.output_format, cp = cparams, np = P.np,
                npb = P.npb, npm = d.npm, mk = std::move(make_frame), prof = std::move(prof),
                wfx = wf[0]]() -> SaveResult {
      const Frame f = mk();
      const std::string xmlp = dir + "/output_" + std::to_string(onum) + ".xml";
      int rc = write_output_xml(xmlp, cp, np, npb, npm, time_out, dt_out, onum);
      if (rc) return {rc, "cannot write " + xmlp};
      if (fmt == 1) rc = write_frame_dat(dir + "/" + std::to_string(onum) + ".dat", f);
      else rc = write_frame_vtu(dir, onum, f);
      if (rc) return {rc, "cannot write particle output in " + dir};
      if (initial) return {RW_OK, ""};
      {  // stress_zz<N>.txt: depth, then the three bands (GetValuesAlongLine, src/utilities.cu:324-367)
        std::FILE* fz = std::fopen((dir + "/stress_zz" + std::to_string(onum) + ".txt").c_str(), "w");
        if (!fz) return {RW_EIO, "cannot write stress_zz file"};
        for (int b = 0; b < nb; ++b)
          std::fprintf(fz, "%g %g %g %g\n", prof[4 * b], prof[4 * b + 1], prof[4 * b + 2], prof[4 * b + 3]);
        std::fclose(fz);
      }
      std::FILE* th = std::fopen((dir + "/time_history.txt").c_str(), "a");
      if (!th) return {RW_EIO, "cannot write time_history.txt"};
      std::fprintf(th, "%g %g\n", time_out, 0.001 * wfx);  // ostream's default 6 digits
      std::fclose(th);
      return {RW_OK, ""};
    };
    if (async_save) {
      pending_save = std::async(std::launch::async, std::move(job));
    } else {
      const SaveResult r = job();
      if (r.rc) throw Fail(r.rc, r.msg);
    }
  }

  // Waits for a save being written in the background; its status, and its message in err.
  int wait_save() {
    if (!pending_save.valid()) return RW_OK;
    const SaveResult r = pending_save.get();
    if (r.rc) err = r.msg;
    return r.rc;
  }
  void get6_cache(std::vector<T>& o) {
    const size_t n = P.np;
    auto ha = down(S.tc_a, n);
    auto hb = down(S.tc_b, n);
    for (size_t i = 0; i < n; ++i) {
      o[6 * i + 0] = ha[i].x; o[6 * i + 1] = ha[i].y; o[6 * i + 2] = ha[i].z;
      o[6 * i + 3] = ha[i].w; o[6 * i + 4] = hb[i].x; o[6 * i + 5] = hb[i].y;
    }
  }
};

// ===================================================================================
// Batch: many contexts on one device advanced by one graph launch per step
// ===================================================================================
struct Batch {
  std::vector<EngineBase*> engines;
  std::vector<unsigned> generations;  // the engines' generations when the graph was built
  int device = 0;
  cudaStream_t st = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool gated = false;      // the children carry their search / scan gates
  double* d_wf = nullptr;  // wall resultants of every context (3 each), device and pinned host
  double* h_wf = nullptr;
  std::string err;
  ~Batch() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    if (d_wf) cudaFree(d_wf);
    if (h_wf) cudaFreeHost(h_wf);
  }
  // One graph holding every context's step as an independent branch, so the executor
  // runs them concurrently.  First choice: a single capture forked from the batch's
  // stream onto each context's stream and joined back, which keeps each step's
  // conditional gates.  Otherwise a parent graph of per-context child graphs, gated
  // where the driver accepts conditional nodes in child graphs, plain if not.
  bool build_forked() {
    std::vector<cudaEvent_t> ev(engines.size() + 1, nullptr);
    for (auto& e : ev) RW_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaGraph_t g = nullptr;
    bool ok = false;
    RW_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      RW_CU(cudaEventRecord(ev[0], st));
      for (size_t k = 0; k < engines.size(); ++k) {
        cudaStream_t es = engines[k]->stream();
        RW_CU(cudaStreamWaitEvent(es, ev[0], 0));
        engines[k]->launch_into_capture(true);
        RW_CU(cudaEventRecord(ev[k + 1], es));
        RW_CU(cudaStreamWaitEvent(st, ev[k + 1], 0));
      }
      RW_CU(cudaStreamEndCapture(st, &g));
      ok = cudaGraphInstantiate(&gexec, g, 0) == cudaSuccess;
    } catch (const Fail&) {
      cudaStreamEndCapture(st, &g);  // ends the capture on every joined stream
      ok = false;
    }
    if (g) cudaGraphDestroy(g);
    for (auto& e : ev) cudaEventDestroy(e);
    if (!ok) {
      gexec = nullptr;
      cudaGetLastError();
    }
    gated = ok;
    return ok;
  }
  // Rebuilds the graph when an option of some context changed since it was captured.
  void refresh() {
    bool stale = !gexec;
    for (size_t k = 0; k < engines.size(); ++k) stale = stale || engines[k]->generation != generations[k];
    if (!stale) return;
    if (gexec) {
      cudaGraphExecDestroy(gexec);  // freed once launches in flight complete
      gexec = nullptr;
    }
    build();
  }
  void build() {
    generations.clear();
    for (EngineBase* e : engines) generations.push_back(e->generation);
    if (build_forked()) return;
    for (int attempt = 0; attempt < 2 && !gexec; ++attempt) {
      const bool gates = attempt == 0;
      cudaGraph_t parent = nullptr;
      RW_CU(cudaGraphCreate(&parent, 0));
      cudaError_t rc = cudaSuccess;
      try {
        for (EngineBase* e : engines) {
          cudaGraph_t child = e->step_graph(gates);
          cudaGraphNode_t node;
          rc = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child);
          cudaGraphDestroy(child);
          if (rc != cudaSuccess) break;
        }
        if (rc == cudaSuccess) rc = cudaGraphInstantiate(&gexec, parent, 0);
      } catch (const Fail&) {
        cudaGraphDestroy(parent);
        if (!gates) throw;
        rc = cudaErrorNotSupported;  // capture with conditional nodes refused: plain children
        parent = nullptr;
      } catch (...) {
        cudaGraphDestroy(parent);
        throw;
      }
      if (parent) cudaGraphDestroy(parent);
      if (rc != cudaSuccess) {
        gexec = nullptr;
        cudaGetLastError();
        if (!gates) RW_CU(rc);
      }
      gated = gates && gexec;
    }
  }
  // Every context's wall resultant with one copy back and one wait.
  void wall_force(int mode, int wall_id, const double* strip, double* out) {
    const size_t n = engines.size();
    if (!d_wf) {
      RW_CU(cudaMalloc(reinterpret_cast<void**>(&d_wf), 3 * n * sizeof(double)));
      RW_CU(cudaMallocHost(reinterpret_cast<void**>(&h_wf), 3 * n * sizeof(double)));
    }
    for (size_t k = 0; k < n; ++k) engines[k]->wall_force_enqueue(st, mode, wall_id, strip, d_wf + 3 * k);
    RW_CU(cudaMemcpyAsync(h_wf, d_wf, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    RW_CU(cudaStreamSynchronize(st));
    std::memcpy(out, h_wf, 3 * n * sizeof(double));
  }
};

}  // namespace rw

// ===================================================================================
// C ABI
// ===================================================================================
struct rw_ctx {
  std::unique_ptr<rw::EngineBase> eng;
};

using rw::Fail;

template <class F> static rw_status guarded(rw_ctx* ctx, F fn) {
  if (!ctx || !ctx->eng) return RW_EINVAL;
  try {
    cudaSetDevice(ctx->eng->device);
    return fn(*ctx->eng);
  } catch (const Fail& f) {
    ctx->eng->err = f.what();
    return f.code;
  } catch (const std::bad_alloc&) {
    ctx->eng->err = "host allocation failed";
    return RW_ENOMEM;
  } catch (const std::exception& e) {
    ctx->eng->err = e.what();
    return RW_EINVAL;
  }
}

extern "C" {

const char* rw_status_string(rw_status s) {
  static const char* names[] = {"RW_OK", "RW_EINVAL", "RW_ENOENT", "RW_EIO", "RW_EFORMAT",
                                "RW_ECUDA", "RW_ENOMEM", "RW_EDEVICE", "RW_ETIMEDOUT", "RW_ESTATE"};
  return (s >= 0 && s <= RW_ESTATE) ? names[s] : "RW_UNKNOWN";
}

const char* rw_last_error(const rw_ctx* ctx) {
  if (!ctx || !ctx->eng) return rw::g_create_err.c_str();
  return ctx->eng->err.c_str();
}

rw_status rw_create_from_case(const rw_case* c, int device, int precision, rw_ctx** out) {
  if (!c || !out) return RW_EINVAL;
  *out = nullptr;
  if (precision != 4 && precision != 8) {
    rw::g_create_err = "precision must be 4 or 8";
    return RW_EINVAL;
  }
  std::unique_ptr<rw::EngineBase> e;
  try {
    if (precision == 4) {
      auto p = std::make_unique<rw::Engine<float>>();
      p->create(c, device);
      e = std::move(p);
    } else {
      auto p = std::make_unique<rw::Engine<double>>();
      p->create(c, device);
      e = std::move(p);
    }
  } catch (const Fail& f) {
    rw::g_create_err = f.what();
    return f.code;
  } catch (const std::bad_alloc&) {
    rw::g_create_err = "host allocation failed";
    return RW_ENOMEM;
  } catch (const std::exception& ex) {
    rw::g_create_err = ex.what();
    return RW_EINVAL;
  }
  *out = new rw_ctx{std::move(e)};
  return RW_OK;
}

rw_status rw_create(const char* project, int device, int precision, rw_ctx** out) {
  if (!project || !out) return RW_EINVAL;
  rw::HostCase hc;
  std::string msg;
  int rc = rw::read_project(project, &hc, &msg);
  if (rc) {
    rw::g_create_err = msg;
    return rc;
  }
  rw_case view = hc.view();
  return rw_create_from_case(&view, device, precision, out);
}

rw_status rw_destroy(rw_ctx* ctx) {
  if (!ctx) return RW_EINVAL;
  if (ctx->eng) cudaSetDevice(ctx->eng->device);
  delete ctx;
  return RW_OK;
}

#define RW_STAGE(fn, body) \
  rw_status fn(rw_ctx* ctx) { return guarded(ctx, [&](rw::EngineBase& e) { body; return RW_OK; }); }

RW_STAGE(rw_begin_step, e.begin_step())
RW_STAGE(rw_rigid_body_update, e.rigid())
RW_STAGE(rw_adami_boundary, e.adami())
RW_STAGE(rw_find_corner, e.corner())
RW_STAGE(rw_shepard_filter, e.shepard())
RW_STAGE(rw_particle_interaction, e.interaction())
RW_STAGE(rw_predictor, e.predictor())
RW_STAGE(rw_corrector, e.corrector())
RW_STAGE(rw_end_step, e.end_step())

rw_status rw_neighbor_search(rw_ctx* ctx, int section) {
  if (section != 0 && section != 1) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { e.neighbor_search(section); return RW_OK; });
}

rw_status rw_step(rw_ctx* ctx, int nsteps) {
  if (nsteps < 0) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { e.step(nsteps); return RW_OK; });
}

rw_status rw_step_timed(rw_ctx* ctx, int nsteps, double* ms) {
  if (nsteps < 1 || !ms) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { *ms = e.step_timed(nsteps); return RW_OK; });
}

rw_status rw_synchronize(rw_ctx* ctx) {
  return guarded(ctx, [&](rw::EngineBase& e) { return e.sync(); });
}

rw_status rw_wall_force(rw_ctx* ctx, int mode, int wall_id, const double* strip, double out_xyz[3]) {
  if (!out_xyz || (mode != 0 && mode != 1)) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { e.wall_force(mode, wall_id, strip, out_xyz); return RW_OK; });
}

rw_status rw_save(rw_ctx* ctx, const char* outdir) {
  return guarded(ctx, [&](rw::EngineBase& e) { e.save(outdir); return RW_OK; });
}

rw_status rw_wall_profile(rw_ctx* ctx, double x_wall, double z_top, double dz, int nbins, double* out) {
  if (!out || nbins <= 0) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { e.wall_profile(x_wall, z_top, dz, nbins, out); return RW_OK; });
}

rw_status rw_get_info(rw_ctx* ctx, rw_info* out) {
  if (!out) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { e.info(out); return RW_OK; });
}

rw_status rw_set_option(rw_ctx* ctx, int option, double value) {
  return guarded(ctx, [&](rw::EngineBase& e) { return e.set_option(option, value); });
}

rw_status rw_get_array(rw_ctx* ctx, int which, void* host_dst, size_t bytes) {
  if (!host_dst) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { return e.get_array(which, host_dst, bytes); });
}

rw_status rw_set_array(rw_ctx* ctx, int which, const void* host_src, size_t bytes) {
  if (!host_src) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { return e.set_array(which, host_src, bytes); });
}

rw_status rw_profile(rw_ctx* ctx, int nsteps, double* ms_per_stage, int n_stages, int* kernels_per_step) {
  if (nsteps < 0 || (n_stages > 0 && !ms_per_stage)) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) {
    e.profile(nsteps, ms_per_stage, n_stages, kernels_per_step);
    return RW_OK;
  });
}

struct rw_batch {
  rw::Batch b;
};

rw_status rw_batch_create(rw_ctx* const* ctxs, int n, rw_batch** out) {
  if (!ctxs || n <= 0 || !out) return RW_EINVAL;
  *out = nullptr;
  auto bt = std::make_unique<rw_batch>();
  try {
    for (int k = 0; k < n; ++k) {
      if (!ctxs[k] || !ctxs[k]->eng) return RW_EINVAL;
      if (k > 0 && ctxs[k]->eng->device != ctxs[0]->eng->device) {
        rw::g_create_err = "all contexts of a batch must be on one device";
        return RW_EINVAL;
      }
      bt->b.engines.push_back(ctxs[k]->eng.get());
    }
    bt->b.device = ctxs[0]->eng->device;
    RW_CU(cudaSetDevice(bt->b.device));
    for (auto* e : bt->b.engines) RW_CU(cudaStreamSynchronize(e->stream()));
    RW_CU(cudaStreamCreateWithFlags(&bt->b.st, cudaStreamNonBlocking));
    bt->b.build();
  } catch (const Fail& f) {
    rw::g_create_err = f.what();
    return f.code;
  } catch (const std::exception& e) {
    rw::g_create_err = e.what();
    return RW_EINVAL;
  }
  *out = bt.release();
  return RW_OK;
}

rw_status rw_batch_wall_force(rw_batch* b, int mode, int wall_id, const double* strip, double* out_xyz) {
  if (!b || !out_xyz || (mode != 0 && mode != 1)) return RW_EINVAL;
  try {
    RW_CU(cudaSetDevice(b->b.device));
    b->b.wall_force(mode, wall_id, strip, out_xyz);
  } catch (const Fail& f) {
    b->b.err = f.what();
    return f.code;
  }
  return RW_OK;
}

namespace {
struct EventPair {  // destroyed on every path out of the timed region
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~EventPair() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};
}  // namespace

rw_status rw_batch_step(rw_batch* b, int nsteps, double* ms) {
  if (!b || nsteps < 0) return RW_EINVAL;
  try {
    RW_CU(cudaSetDevice(b->b.device));
    b->b.refresh();  // options changed on a context since the capture: capture again
    EventPair ev;
    if (ms) {
      RW_CU(cudaEventCreate(&ev.e0));
      RW_CU(cudaEventCreate(&ev.e1));
      RW_CU(cudaEventRecord(ev.e0, b->b.st));
    }
    for (int k = 0; k < nsteps; ++k) RW_CU(cudaGraphLaunch(b->b.gexec, b->b.st));
    if (ms) {
      RW_CU(cudaEventRecord(ev.e1, b->b.st));
      RW_CU(cudaEventSynchronize(ev.e1));
      float t = 0.f;
      RW_CU(cudaEventElapsedTime(&t, ev.e0, ev.e1));
      *ms = t;
    }
  } catch (const Fail& f) {
    b->b.err = f.what();
    return f.code;
  }
  return RW_OK;
}

rw_status rw_batch_synchronize(rw_batch* b) {
  if (!b) return RW_EINVAL;
  cudaSetDevice(b->b.device);
  return cudaStreamSynchronize(b->b.st) == cudaSuccess ? RW_OK : RW_ECUDA;
}

rw_status rw_batch_destroy(rw_batch* b) {
  if (!b) return RW_EINVAL;
  cudaSetDevice(b->b.device);
  delete b;
  return RW_OK;
}

rw_status rw_list_stats(rw_ctx* ctx, int64_t* out) {
  if (!out) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) {
    long long t[2];
    e.list_totals(t);
    out[0] = t[0];
    out[1] = t[1];
    return RW_OK;
  });
}

rw_status rw_set_closure(rw_ctx* ctx, rw_mlp* net, double margin) {
  if (!(margin >= 0.0)) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) { return (rw_status)e.set_closure(net, margin); });
}

rw_status rw_closure_stats(rw_ctx* ctx, double* out) {
  if (!out) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) {
    e.closure_stats(out);
    return RW_OK;
  });
}

rw_status rw_mlp_collect(rw_mlp* net, rw_ctx* ctx, int stride, const double* augment, uint64_t seed,
                         int64_t* added) {
  if (!net || stride < 1) return RW_EINVAL;
  rw::Augment aug{};
  if (augment) {
    if (!(augment[0] > 0.0 && augment[1] >= augment[0] && augment[1] < 90.0 && augment[2] > 0.0 &&
          augment[3] >= augment[2]))
      return RW_EINVAL;
    const double d2r = 3.14159265358979323846 / 180.0;
    aug = rw::Augment{(float)(augment[0] * d2r), (float)(augment[1] * d2r), (float)augment[2], (float)augment[3],
                      (unsigned long long)seed, 1};
  }
  return guarded(ctx, [&](rw::EngineBase& e) {
    const long long a = e.collect(net, stride, aug);
    if (added) *added = a;
    return RW_OK;
  });
}

rw_status rw_autotune(rw_ctx* ctx, int steps, int* chosen) {
  if (steps < 1) return RW_EINVAL;
  return guarded(ctx, [&](rw::EngineBase& e) {
    // Shapes by measurement: each candidate runs one step to capture its graph and
    // `steps` timed steps; the fastest stays selected.  First the interaction (the walk
    // kernel at 64 or 128 threads per block, or the chunked kernel), then the
    // integrators' block size.
    auto timed = [&]() {
      e.step(1);
      return e.step_timed(steps);
    };
    const int walk_cand[3][2] = {{0, 64}, {0, 128}, {1, 128}};
    double best = 1e300;
    int pick = 1;
    for (int c = 0; c < 3; ++c) {
      if (e.set_option(RW_OPT_INTERACTION_KERNEL, walk_cand[c][0]) != RW_OK ||
          e.set_option(RW_OPT_WALK_THREADS, walk_cand[c][1]) != RW_OK)
        continue;
      const double t = timed();
      if (t < best) {
        best = t;
        pick = c;
      }
    }
    e.set_option(RW_OPT_INTERACTION_KERNEL, walk_cand[pick][0]);
    e.set_option(RW_OPT_WALK_THREADS, walk_cand[pick][1]);
    const int integ_cand[2] = {256, 128};
    int ipick = 0;
    best = 1e300;
    for (int c = 0; c < 2; ++c) {
      e.set_option(RW_OPT_INTEGRATOR_THREADS, integ_cand[c]);
      const double t = timed();
      if (t < best) {
        best = t;
        ipick = c;
      }
    }
    e.set_option(RW_OPT_INTEGRATOR_THREADS, integ_cand[ipick]);
    if (chosen) *chosen = walk_cand[pick][0];
    return RW_OK;
  });
}

rw_status rw_set_counters(rw_ctx* ctx, double time, int step, int npm, int np_delete_m) {
  return guarded(ctx, [&](rw::EngineBase& e) { e.set_counters(time, step, npm, np_delete_m); return RW_OK; });
}

}  // extern "C"
