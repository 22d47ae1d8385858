/*
 * retainwall.h - C ABI of the B200-native SPH geomechanics step (librw.so).
 *
 * The reference (Xshuaizhang/Retainwall_code, a LOQUAT-derived solver) exposes its
 * step only as private methods of the C++ class LoquatSph (src/loquat.h:44-126),
 * driven by LoquatSph::RunSimulation (src/loquat.cu:511-565) from src/main.cpp.
 * Each entry point below replaces one of those methods (cited per function) so a
 * host program written against the reference's step sequence can call this library
 * instead.  Conventions:
 *   - plain C types only; every call returns an rw_status (0 = RW_OK) and never exits;
 *   - one context per host thread; a context owns its device memory and CUDA stream;
 *   - arrays crossing the ABI use the reference's per-particle layouts (see rw_array).
 */
#ifndef RETAINWALL_H_
#define RETAINWALL_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int rw_status;
enum {
  RW_OK = 0,
  RW_EINVAL = 1,     /* bad argument or inconsistent case                          */
  RW_ENOENT = 2,     /* project file missing                                         */
  RW_EIO = 3,        /* read/write error                                             */
  RW_EFORMAT = 4,    /* malformed XML/.dat/.motion, missing mandatory parameter      */
  RW_ECUDA = 5,      /* CUDA runtime error (message in rw_last_error)                */
  RW_ENOMEM = 6,     /* device or host allocation failed                             */
  RW_EDEVICE = 7,    /* a kernel raised the device error word (see rw_info.device_err) */
  RW_ETIMEDOUT = 8,  /* a bounded device wait gave up                                */
  RW_ESTATE = 9      /* call out of sequence (e.g. wrong section)                    */
};

/* Device error word bits (rw_info.device_err). */
enum {
  RW_DERR_CELL_RANGE = 1,   /* a live particle's cell left the grid (reference: out-of-bounds write) */
  RW_DERR_COUNT = 2,        /* particle-count invariant npb+npm+deleted != np (src/loquat_grid.cu:182-185) */
  RW_DERR_LIST = 4,         /* neighbour list exceeded its per-cell capacity (handled, reported)  */
  RW_DERR_PERM = 8,         /* sort produced an index outside [0, np) (guarded; never expected)  */
  RW_DERR_CLOSURE = 16      /* a tensor-core wait of the learned closure gave up                  */
};

#define RW_MODEL_MAX 10
#define RW_MATERIAL_SIZE 15
#define RW_MOTION_MAX 10
#define RW_TABLE_MAX 10

/* One rigid body's motion table (MotionTable, src/types.h:77-97; .motion file). */
typedef struct rw_motion {
  int32_t is_translation, n_trans;
  double trans_time[RW_TABLE_MAX], trans_vel[RW_TABLE_MAX][3], trans_acc[RW_TABLE_MAX][3];
  int32_t is_rotation, pattern, n_rot, pad_;
  double pos_rp[3], rotat_vel[3], rotat_time[RW_TABLE_MAX], rotat_acc[RW_TABLE_MAX][3];
} rw_motion;

/* The parameter file (<project>.xml, read by LoquatIo::LoadParameters,
 * src/loquat_io.cu:75-202).  Values are given as parsed (double); the library rounds
 * them to its arithmetic type exactly as the reference's (scalar)atof does. */
typedef struct rw_case_params {
  int32_t dim, periodbound, n_motion, np, npb, npm, n_model;
  int32_t stress_shepard_filter, dynamic_time_step, integration_method, viscosity_type;
  int32_t output_number, output_format, pad_;
  double planeleft[4], planeright[4];
  double domain_size[3], domain_min[3];
  double dr, hdr, gravity[3], rho0_m, damping;
  double model_par[RW_MODEL_MAX][RW_MATERIAL_SIZE];
  double artificial_viscosity_alpha_m, cs_m, cfl, artificial_pressure_coefficient_material;
  double time_max, time, dt, output_frequency;
  /* Wall-soil Coulomb coefficient of contact walls.  The reference hard-codes
   * 0.58108 (src/particle_interaction.cu:188-189); optional XML tag
   * "wall-friction-coefficient" (type scalar) sets it. */
  double wall_friction;
  rw_motion motion[RW_MOTION_MAX];
} rw_case_params;

/* A case in the reference's particle layout (.dat, src/loquat_io.cu:229-254):
 * np rows, boundary particles first.  Positions are absolute. */
typedef struct rw_case {
  rw_case_params params;
  const int32_t* codes;    /* np x 4: block id, status (0 Fix / 1 NonFix), model, material|motion */
  const double* pospres;   /* np x 4 */
  const double* velrhop;   /* np x 4 */
  const double* idmassidx; /* np x 4: id (100 material, 0 boundary), mass, (index), w */
  const double* stress;    /* np x 6: xx yy zz xy xz yz */
  const double* strain;    /* np x 6 */
  const double* normal;    /* npb x 4: unit normal, w = +1 free slip / -1 no slip */
} rw_case;

/* Arrays for rw_get_array / rw_set_array, in the reference's device layouts
 * (element = scalar of the context's precision unless noted). */
typedef enum rw_array {
  RW_ARR_CODES = 0,       /* np   x int4            codes                       */
  RW_ARR_CELLPOS = 1,     /* np   x int4            cellpos (cell x,y,z, key)   */
  RW_ARR_POSPRES = 2,     /* np   x 4               in-cell position + pressure */
  RW_ARR_POSPRES_ORI = 3, /* np   x 4               accumulated displacement    */
  RW_ARR_VELRHOP = 4,     /* np   x 4               velocity + density          */
  RW_ARR_IDMASSIDX = 5,   /* np   x 4               id, mass, index, M_crt      */
  RW_ARR_STR = 6,         /* np   x 6               stress                      */
  RW_ARR_STN = 7,         /* np   x 6               strain                      */
  RW_ARR_NORMAL = 8,      /* npb  x 4               wall normals                */
  RW_ARR_CONTACT_MAG = 9, /* np   x 9               contact force, normal, velocity */
  RW_ARR_CONTACT_VAR = 10,/* np   x 4               kernel integral, distance, slide flag, wall id */
  RW_ARR_ACCAD = 11,      /* np   x 4               acceleration + density rate */
  RW_ARR_SPIN = 12,       /* np   x 4                                           */
  RW_ARR_ACESTN = 13,     /* np   x 6               strain rate                 */
  RW_ARR_POSPRES_INI = 14,
  RW_ARR_VELRHOP_INI = 15,
  RW_ARR_STR_INI = 16,
  RW_ARR_STN_INI = 17,
  RW_ARR_PART_IDX = 18,   /* np   x int32           last sort permutation       */
  RW_ARR_CELL_BEG = 19,   /* ncell x int32          -1 for empty cells          */
  RW_ARR_CELL_END = 20,   /* ncell x int32                                      */
  RW_ARR_POS_ABS = 21,    /* np   x 4               absolute position (get only) */
  RW_ARR_COUNT_ = 22
} rw_array;

typedef struct rw_info {
  int32_t np, npb, npm, np_delete_m, ncell, step, scalar_bytes, device_err;
  int32_t cell_num[3], n_motion;
  double time, dt, h, dr;
  int32_t n_sorts;       /* neighbour-search sections whose sort permuted the particles     */
  int32_t n_list_reuse;  /* interactions that walked kept candidate lists                    */
  int32_t n_search_skipped; /* captured-step searches skipped whole (no particle changed cell)  */
  int32_t n_scan_skipped;   /* captured-step interactions whose scan launch was skipped (every
                               particle walked a kept list)                                      */
  int32_t n_build_skipped;     /* captured-step interactions whose list build was skipped (the
                                  kept lists stood)                                              */
  int32_t graph_kernels;       /* kernels of one captured step when no gated body is skipped     */
  int32_t search_body_kernels; /* kernels a skipped search does not launch                       */
  int32_t n_list_updates;      /* interactions that updated the kept lists in part: rebuilt those
                                  next to a cell that particles entered or left, carried the
                                  others through the section's permutation                        */
  double time_max;             /* time-max of the parameter file (src/loquat_io.cu:192)          */
  double output_frequency;     /* output-frequency of the parameter file (src/loquat_io.cu:195)  */
  int32_t ix_kernel;           /* RW_OPT_INTERACTION_KERNEL in use                               */
  int32_t walk_threads;        /* RW_OPT_WALK_THREADS in use                                     */
  int32_t integrator_threads;  /* RW_OPT_INTEGRATOR_THREADS in use                               */
  int32_t n_lists_rebuilt;     /* candidate lists (soil and boundary) rebuilt by those updates    */
  int32_t build_body_kernels;  /* kernels a skipped list build does not launch                    */
  int32_t pad_;
} rw_info;

typedef struct rw_ctx rw_ctx;

/* Options (rw_set_option). */
enum {
  RW_OPT_WALL_FRICTION = 0,  /* Coulomb coefficient of contact walls (default from the case) */
  RW_OPT_COMPAT_CONTACT = 1, /* 1 (default): contact state bound to array slots as in the reference
                                (src/loquat.cu:254-287 never permutes it); 0: follows the particle */
  RW_OPT_INTERACTION_KERNEL = 2, /* 0 (default): one thread per particle, neighbours through L1/L2;
                                   1: column chunks with the neighbour positions staged in shared memory.
                                   Bit-identical results. */
  RW_OPT_STRICT_FP = 3,         /* interaction arithmetic: 0 (default) fused multiply-adds at fixed places;
                                   1 every product and sum rounded separately, the written order of the
                                   reference's expressions (slower; for bit-level comparisons) */
  RW_OPT_MIXED_PRECISION = 4,   /* precision form (float contexts): 1 = compensated (Kahan) position and
                                   velocity integration and an FP64 strain-rate norm in the hypoplastic
                                   update; the wall resultant is always accumulated in FP64.  Set before
                                   stepping. */
  RW_OPT_LIST_SKIN = 5,         /* skin of the kept candidate lists, in units of h (default 0.02; 0 = scan
                                   the cells in every interaction).  The interaction keeps each particle's
                                   candidates within 2h + skin and walks them instead of the 27 cells.
                                   After particles change cell, the next predictor section rebuilds only
                                   the lists next to the cells they entered or left and carries the others
                                   through the sort's permutation; every list is rebuilt once a particle
                                   may have moved 0.45 skin since the last full build.  Results do not
                                   depend on it. */
  RW_OPT_GRAPH_GATES = 6,       /* 1 (default): the captured step graph skips a search with no cell change
                                   and an idle scan launch behind conditional nodes; 0: plain graph, every
                                   kernel launched (profilers that replay single graph kernels need it).
                                   Results do not depend on it. */
  RW_OPT_WALK_THREADS = 8,      /* threads per block of the interaction's walk launch: 64 or 128 (default);
                                   results do not depend on it */
  RW_OPT_INTEGRATOR_THREADS = 9, /* threads per block of the predictor and corrector: 128 or 256 (default);
                                   results do not depend on it */
  RW_OPT_CLOSURE_MAX_ERR = 7,   /* learned closure: a particle keeps the network's objective rate only while
                                   its judged relative error against the exact rate is at most this
                                   (default 0.02; 0: no bound, the trust region alone decides) */
  RW_OPT_ASYNC_SAVE = 10        /* 1: rw_save gathers the output state and returns while a background task
                                   formats and writes the files (one save in flight); the next rw_save,
                                   rw_synchronize or rw_destroy waits for it, and the first two report its
                                   status.  0 (default): rw_save returns once the files are written. */
};

const char* rw_status_string(rw_status s);
/* Last error message of a context (or of the last failed rw_create* when ctx is NULL). */
const char* rw_last_error(const rw_ctx* ctx);

/* LoquatSph(name) + RunSimulation's set-up (src/loquat.cu:514-531): reads
 * <project>.xml/.dat/.motion, initialises parameters (InitializeParameters,
 * src/loquat.cu:130-190), uploads the state, converts to in-cell positions and runs the
 * first neighbour search and sort.  precision: 4 (float, the reference default) or 8. */
rw_status rw_create(const char* project, int device, int precision, rw_ctx** out);
/* Same set-up from a case held in host memory (no files). */
rw_status rw_create_from_case(const rw_case* c, int device, int precision, rw_ctx** out);
/* ~LoquatSph (src/loquat.cu:72-99). */
rw_status rw_destroy(rw_ctx* ctx);

/* StepCalculation (src/loquat.cu:366-374): dt = cfl*h/cs, time of this step. */
rw_status rw_begin_step(rw_ctx* ctx);
/* LoquatGrid::NeighborSearch (src/loquat_grid.cu:147-191) followed by SortArraysPrimary
 * (section 0, src/loquat.cu:254-266) or SortArraysAll (section 1, src/loquat.cu:269-287). */
rw_status rw_neighbor_search(rw_ctx* ctx, int section);
/* LoquatSph::RigidBodyUpdate (src/adami_boundary.cu:175-203), on the device. */
rw_status rw_rigid_body_update(rw_ctx* ctx);
/* LoquatSph::AdamiBoundary (src/adami_boundary.cu:160-169). */
rw_status rw_adami_boundary(rw_ctx* ctx);
/* LoquatSph::FindCornerParticle (src/adami_boundary.cu:294-306). */
rw_status rw_find_corner(rw_ctx* ctx);
/* LoquatSph::StressRegularization (src/field_smoothing.cu:92-101). */
rw_status rw_shepard_filter(rw_ctx* ctx);
/* LoquatSph::ParticleInteraction (src/particle_interaction.cu:310-313). */
rw_status rw_particle_interaction(rw_ctx* ctx);
/* LoquatSph::Predictor (src/predictor_corrector.cu:87-103). */
rw_status rw_predictor(rw_ctx* ctx);
/* LoquatSph::Corrector (src/predictor_corrector.cu:201-213). */
rw_status rw_corrector(rw_ctx* ctx);
/* End of RunSimulation's loop body (src/loquat.cu:559-561): time += dt, step++. */
rw_status rw_end_step(rw_ctx* ctx);
/* nsteps whole steps (StepCalculation + PredictorSection + CorrectorSection,
 * src/loquat.cu:548-561) replayed from one captured CUDA graph, no host round trip. */
rw_status rw_step(rw_ctx* ctx, int nsteps);
/* rw_step with a CUDA event pair recorded on the context's stream around the nsteps
 * graph launches; *ms receives the device time (no reference counterpart). */
rw_status rw_step_timed(rw_ctx* ctx, int nsteps, double* ms);
/* Blocks until the context's stream is idle; reports RW_EDEVICE if a kernel flagged an error. */
rw_status rw_synchronize(rw_ctx* ctx);

/* Lateral wall force, FP64 accumulation, in N (not kN).
 * mode 0: sum of contact force over material particles whose nearest contact wall
 *         (contact_var.w) equals wall_id;
 * mode 1: the reference's strip (src/utilities.cu:619-624): x <= x_max, z in [z_min, z_max],
 *         with strip = {x_max, z_min, z_max}; strip may be NULL for the reference's values
 *         (0.04 + bound_thickness + 3 dr, bound_thickness + 0.04, bound_thickness + 1.04). */
rw_status rw_wall_force(rw_ctx* ctx, int mode, int wall_id, const double* strip, double out_xyz[3]);
/* Earth-pressure profile along the wall (GetValuesAlongLine, src/utilities.cu:266-367):
 * out[4*b] = depth b*dr where the 1st band has a particle in bin b (the reference
 * writes the depth together with that band's value; 0 otherwise), out[4*b+1..3] =
 * contact_mag.xx / dr of the last soil particle (index order, as the reference) in depth
 * bin b of the 1st, 2nd, 3rd dr-thick band from the wall face x_wall; bins of size dz
 * below z_top; 0 for empty bins (the reference leaves them unwritten).  NaN x_wall, z_top
 * or dz select the reference's hard-coded values (face 0.04 + bound_thickness - 0.005 t,
 * top 0.04 + 1.0 + bound_thickness, dz = dr). */
rw_status rw_wall_profile(rw_ctx* ctx, double x_wall, double z_top, double dz, int nbins, double* out);
/* The first call writes the initial configuration as RunSimulation does (output number
 * of the case, particles and parameters only, src/loquat.cu:533-537); later calls are
 * Saving (src/loquat.cu:439-482) through LoquatIo::SaveXml / SaveParticles: writes
 * <outdir>/output_N.xml and N.dat (format 1) or <id>_N.vtu (format 2) with the
 * Shepard-smoothed stress, stress_zzN.txt (rw_wall_profile with the reference's
 * defaults) and appends "time F[kN]" to <outdir>/time_history.txt. */
rw_status rw_save(rw_ctx* ctx, const char* outdir);
/* (The reference's Saving writes its files before the step loop goes on; with
 * RW_OPT_ASYNC_SAVE the files are written while later steps run.  Formatting uses every
 * host core either way.) */

/* The particle file <project>.dat of a case, as the reference's generator writes it
 * (SaveDatFile, src/GenCase.cu:70-116, read back by LoquatIo::LoadParticles,
 * src/loquat_io.cu:222-264): one row per particle, boundary rows first with their
 * normal; reals printed as %.9g, so a float case reads back exactly.  Host only. */
rw_status rw_write_case_dat(const rw_case* c, const char* path);

rw_status rw_get_info(rw_ctx* ctx, rw_info* out);
rw_status rw_set_option(rw_ctx* ctx, int option, double value);
/* Copy an array out (host_dst, bytes = rows x row size of the context's precision). */
rw_status rw_get_array(rw_ctx* ctx, int which, void* host_dst, size_t bytes);
/* Overwrite a state array (golden-state restarts); RW_ARR_POS_ABS is not settable. */
rw_status rw_set_array(rw_ctx* ctx, int which, const void* host_src, size_t bytes);
/* Overwrite time, step and the live/deleted counts after rw_set_array restarts. */
rw_status rw_set_counters(rw_ctx* ctx, double time, int step, int npm, int np_delete_m);

/* Stage timing (no reference counterpart; the reference's Timer buckets CPU clock per
 * phase, src/types.h:167-184).  Runs nsteps whole steps as per-stage launches with a
 * CUDA event pair around each stage on the context's stream and returns the mean time
 * per stage in ms, in the order of RW_STAGE_*.  *kernels_per_step receives the number of
 * kernels one whole step launches. */
enum {
  RW_STAGE_SEARCH_P = 0, RW_STAGE_RIGID = 1, RW_STAGE_ADAMI_P = 2, RW_STAGE_CORNER_P = 3,
  RW_STAGE_INTERACTION_P = 4, RW_STAGE_PREDICTOR = 5, RW_STAGE_SEARCH_C = 6, RW_STAGE_ADAMI_C = 7,
  RW_STAGE_CORNER_C = 8, RW_STAGE_INTERACTION_C = 9, RW_STAGE_CORRECTOR = 10, RW_STAGE_COUNT_ = 11
};
rw_status rw_profile(rw_ctx* ctx, int nsteps, double* ms_per_stage, int n_stages, int* kernels_per_step);

/* Batched cases (no reference counterpart; the reference runs one case per process).
 * Contexts on one device are advanced together: each context's whole step becomes an
 * independent branch of one graph (captured forked onto the contexts' streams), so one
 * graph launch per step runs every case and the executor overlaps their kernels.  rw_batch_step is asynchronous unless
 * ms is non-NULL (then it waits and returns the device time of the nsteps launches);
 * call rw_batch_synchronize before reading any context.  The contexts must outlive the
 * batch and must not be stepped individually while it is in use.  Options set on a
 * context after rw_batch_create (rw_set_option, rw_set_closure) take effect at the next
 * rw_batch_step, which captures the batch's graph again first. */
typedef struct rw_batch rw_batch;
rw_status rw_batch_create(rw_ctx* const* ctxs, int n, rw_batch** out);
rw_status rw_batch_step(rw_batch* b, int nsteps, double* ms);
rw_status rw_batch_synchronize(rw_batch* b);
rw_status rw_batch_destroy(rw_batch* b);
/* rw_wall_force of every context of the batch (same mode, wall_id and strip), after the
 * batch's steps: out_xyz receives 3 doubles per context, in creation order, with one
 * copy back and one wait for all of them. */
rw_status rw_batch_wall_force(rw_batch* b, int mode, int wall_id, const double* strip, double* out_xyz);
/* Kept candidate lists (RW_OPT_LIST_SKIN) as they stand: out[0] = entries over all soil
 * particles, out[1] = soil particles holding a list (both 0 when none is kept). */
rw_status rw_list_stats(rw_ctx* ctx, int64_t* out);
/* Autotuner: times the interaction shapes (the walk kernel at 64 and 128 threads per
 * block, and the chunked kernel) and then the integrators' block size (256, 128) on
 * this case, `steps` steps each (plus one capture step each; the case advances), and
 * keeps the fastest; *chosen receives the interaction kernel (RW_OPT_INTERACTION_KERNEL),
 * rw_get_info the shapes. */
rw_status rw_autotune(rw_ctx* ctx, int steps, int* chosen);

/* Allocation-free cell-key sort.  No counterpart in the reference (which sorts with
 * cub::DeviceRadixSort into buffers it cudaMallocs, src/loquat_grid.cu:98-113); for
 * callers that cannot allocate device memory.  Stable sort of n cell keys (device
 * array d_keys, values in [0, max_key]) into d_sorted_keys, with d_perm[i] = index of
 * the key that lands at position i: the permutation NeighborSearch applies.  Uses a
 * fixed scratch array inside the library (8,913,924 bytes: 8.9 MB, 8.5 MiB, reserved
 * on every GPU that loads the library until the process exits) instead of
 * allocating: n is limited to
 * RW_NOALLOC_MAX_KEYS and max_key to 2^24 - 1 (RW_EINVAL beyond).  Runs on `stream`
 * (a cudaStream_t, NULL = default stream) of the current device.  The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  All calls share the one scratch array: calls whose work
 * overlaps on the GPU (other streams, other threads) race and must be serialised by
 * the caller.  d_keys must not alias the outputs. */
#define RW_NOALLOC_MAX_KEYS (1 << 20)
rw_status rw_cell_sort_noalloc(const int32_t* d_keys, int32_t n, int32_t max_key, int32_t* d_sorted_keys,
                               int32_t* d_perm, void* stream);

/* ---------------------------------------------------------------------------------
 * Learned constitutive closure.  No counterpart in the reference: a surrogate of the
 * objective (Jaumann-free) part of the HypoCS stress rate (src/constitutive_model.h:269),
 * a 16-64-64-64-64-6 perceptron with SiLU hidden units, BF16 weights and activations and
 * FP32 accumulation, evaluated and trained on the tensor cores (tcgen05).
 *   features  x[16]: stress / p (6), strain rate / |D| (6), relative void ratio
 *             psi = (e - e_min) / (e_c(p) - e_min), (sin phi_c - 0.556) / 0.087,
 *             psi^alpha, 0;
 *   target    t[6]:  R / (p |D|) / 1000, R the objective stress rate.
 * Parameters (RW_MLP_NPARAM floats): W1[16][64] b1[64] W2[64][64] b2 W3 b3 W4 b4
 * W5[64][6] b5[6] (y = x W + b).  Host arrays are row-major.
 * --------------------------------------------------------------------------------- */
typedef struct rw_mlp rw_mlp;
#define RW_MLP_IN 16
#define RW_MLP_OUT 6
#define RW_MLP_NPARAM 13958
const char* rw_mlp_last_error(rw_mlp* m);
/* Xavier-uniform weights from `seed`, zero biases; room for sample_capacity samples. */
rw_status rw_mlp_create(int device, uint64_t seed, int64_t sample_capacity, rw_mlp** out);
rw_status rw_mlp_destroy(rw_mlp* m);
rw_status rw_mlp_get_params(rw_mlp* m, float* out, size_t n);
rw_status rw_mlp_set_params(rw_mlp* m, const float* in, size_t n);
/* y[n][6] = net(x[n][16]). */
rw_status rw_mlp_forward(rw_mlp* m, const float* x, int64_t n, float* y);
/* Mean squared error over n samples and 6 outputs, and its gradient (RW_MLP_NPARAM). */
rw_status rw_mlp_grad(rw_mlp* m, const float* x, const float* t, int64_t n, double* loss, float* grad);
/* Training samples kept on the device. */
rw_status rw_mlp_add_samples(rw_mlp* m, const float* x, const float* t, int64_t n);
rw_status rw_mlp_samples(rw_mlp* m, int64_t* count, float* x, float* t, int64_t n);
rw_status rw_mlp_clear_samples(rw_mlp* m);
/* Adam (beta 0.9 / 0.999) over the stored samples, shuffled per epoch, the step size
 * decaying from lr to lr / 20 (cosine) over the call; *last_loss = mean squared error
 * over the last epoch. */
rw_status rw_mlp_train(rw_mlp* m, int epochs, int batch, float lr, uint64_t seed, double* last_loss);
/* Per-feature minimum / maximum of the stored samples and the largest |target|. */
rw_status rw_mlp_feature_ranges(rw_mlp* m, float* lo, float* hi, float* tmax);
/* Appends training samples (features and exact targets) from a context's current state:
 * every `stride`-th soil particle with a HypoCS update; *added = samples kept (bounded by
 * the network's free capacity).  augment = {phi_c min, phi_c max [deg], e0 min, e0 max}
 * or NULL: with it, each sample's friction angle and initial void ratio are drawn
 * uniformly (seeded) from those ranges and its target is the exact rate of that material
 * at the solver's state.  The context and the network share a device. */
rw_status rw_mlp_collect(rw_mlp* m, rw_ctx* ctx, int stride, const double* augment, uint64_t seed, int64_t* added);
/* Uses the network for the objective stress rate of this context's HypoCS particles
 * (NULL: exact updates again).  A particle uses it only when all its features lie within
 * the ranges of the network's stored samples, each widened by `margin` times its width,
 * and every output within (1 + margin) times the largest stored |target|, and the
 * network's rate is within RW_OPT_CLOSURE_MAX_ERR of the exact one (which is computed
 * anyway to judge it); otherwise, and for the zero-stress reset, the exact update runs.  The Jaumann term, the tension
 * cut-off and the cone projection stay exact.  Ranges are taken at this call; the
 * weights are read at every step. */
rw_status rw_set_closure(rw_ctx* ctx, rw_mlp* m, double margin);
/* Since rw_set_closure: [0] HypoCS updates offered to the network, [1] updates that used
 * it, [2] mean and [3] largest relative error (L2 over the six components) of its
 * objective rate against the exact one, over the updates that used it. */
rw_status rw_closure_stats(rw_ctx* ctx, double* out);

#ifdef __cplusplus
}
#endif
#endif /* RETAINWALL_H_ */
