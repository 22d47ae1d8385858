// Parameter block and device-resident dynamic state of one case.
//
// Params<T> mirrors the reference's Parameters (src/types.h:100-165) after
// InitializeParameters (src/loquat.cu:130-190).  It is passed BY VALUE to every
// kernel (kernel-parameter constant bank), replacing the reference's per-TU
// __constant__ copies refreshed by cudaMemcpyToSymbolAsync before each launch.
// What changes during a run (time, live counts, rigid-body motion, buffer parity,
// error word) lives in Dyn<T> in device memory, so a whole step can be captured in a
// CUDA graph with no host round trip.
#pragma once
#include <stdint.h>

#define RW_MATERIAL_NUMBER 100.0f  // idmassidx.x >= 100: material (src/types.h:37)
#define RW_MODEL_RIGID 0
#define RW_MODEL_DP 1
#define RW_MODEL_MUIDP 2
#define RW_MODEL_HYPO_BASIC 3
#define RW_MODEL_HYPO_CS 4
#define RW_PATTERN_CIRCLE 1

namespace rw {

constexpr int kModelMax = 10, kMatSize = 15, kMotionMax = 10, kTableMax = 10;

template <class T> struct Vec3 { T x, y, z; };

template <class T> struct Motion {  // RigidMotion (src/types.h:66-75)
  int is_trans, is_rotat, pattern, pad_;
  Vec3<T> trans_vel, trans_acc, pos_rp, rotat_vel, rotat_acc;
};

template <class T> struct Table {  // MotionTable (src/types.h:77-97)
  int is_translation, is_rotation, n_trans, n_rot, pattern, pad_;
  T trans_time[kTableMax], rotat_time[kTableMax];
  Vec3<T> trans_vel[kTableMax], trans_acc[kTableMax], rotat_acc[kTableMax];
  Vec3<T> pos_rp, rotat_vel;
};

// Per-material constants of the hypoplastic update (see hypo_coef).
template <class T> struct HypoC {
  T C1, a, C2, C3, C4, fa, fb, fc;
  double t1;
};

template <class T> struct Params {
  int dim, periodbound, n_motion, n_model;
  int np, npb, npm0;        // particle counts at set-up (np, npb never change)
  int cell_num[3];
  int ncell, ncell_material, ncell_delete_m;
  int stress_shepard_filter, viscosity_type, output_format;
  T planeleft[4], planeright[4];
  T domain_size[3], domain_min[3], gravity[3];
  T h, i_h, two_h, dr, hdr, vol_def, bound_thickness;
  T rho0_m, damping;
  T model_par[kModelMax][kMatSize];
  T knorm, kgrad;            // Wendland normalisations (src/loquat.cu:163-166)
  T alpha_m, cs_m, eta, cfl, art_coef, kernel_zero, kernel_dr;
  T visc_k;                  // alpha_m * cs_m * h (artificial viscosity, one-division form)
  T time_max, dt, output_frequency;
  T wall_fric;               // wall-soil Coulomb coefficient
  T r2_prefilter;            // conservative (2h)^2 bound for the candidate pre-test
  T r2_list;                 // conservative (2h + skin)^2: radius of the kept candidate lists
  float disp_lim;            // a particle's displacement since the lists were built may not pass this
  float disp_eps;            // rounding allowance added per position update
  int keep_lists;            // 0: every interaction scans the cells
  int closure;               // 1: HypoCS stress updates by the learned closure (k_closure)
  HypoC<T> hypo[kModelMax];  // per-material constants, evaluated once on the device
  int mixed;                 // precision form: compensated integration, FP64 strain-rate norm
  int pad_m;
};

// Device-resident state that changes during a run.
template <class T> struct Dyn {
  double time_d;             // host-side `time` of RunSimulation, accumulated in double
  T time_f;                  // par.time (scalar copy of time_d, StepCalculation)
  T pad0_;
  int npm, np_delete_m;      // live / deleted material counts (src/loquat_grid.cu:164-181)
  int cur_main, cur_nrm, cur_ini;  // which ping-pong buffer holds each permuted group
  int need_sort;             // 1 when the new cell keys are not already in order
  unsigned err;              // RW_DERR_* bits
  int step;
  int nchunks;               // live entries of the interaction chunk list
  // Candidate lists kept across sections and steps: ix_mode 0 = build every list (then
  // walk them), 1 = walk the kept lists, 2 = update them: rebuild the lists of the
  // particles next to a cell that some particle entered or left (a marked cell), carry
  // the others through the section's permutation, then walk.  list_kill: some particle
  // moved too far since the last full build, or left the grid; build_kill: lists
  // built in this section are not to be kept (a corrector-section rebuild).
  int ix_mode, list_ok, list_kill, build_kill;
  int n_sorts, n_reuse;      // sections that permuted / interactions that walked kept lists
  // Marked cells since the last list update (distinct cells, listed in DevState::marks;
  // more than RW_MARK_CAP: the next update is a full build).  Marks carry a generation
  // number instead of being cleared: mark_gen is the one the integrators mark with,
  // near_gen the one a list update tests (k_flip hands mark_gen over and advances it).
  // lbuf: which of the two list / displacement-bound buffers is live (it flips with
  // every permutation).
  int n_marks, lbuf;
  unsigned mark_gen, near_gen;
  int n_updates, n_rebuilt;  // interactions that updated the lists / lists rebuilt by them
  int n_queue;               // lists queued for rebuilding by the current update
  // Soil neighbour records: the integrators rewrite them; the corner search rewrites
  // them after a permutation or a host write (rec_stale: set by the search, cleared by
  // the interaction that follows).
  int rec_stale, host_dirty;
  // Some particle changed cell (or the host wrote the state) since the last search:
  // keys, ranges and counts must be recomputed.  Set by the corrector, cleared at the
  // end of each search.
  int cells_dirty;
  int n_spill;  // kept lists of the last build that overflowed (those particles scan)
  // Work skipped by the gates of a captured step graph (conditional nodes): searches
  // with no cell change, scan launches with every particle on a list, list builds
  // while the kept lists stand.
  int n_search_skipped, n_scan_skipped, n_build_skipped;
  Motion<T> mv[kMotionMax];
  Table<T> tab[kMotionMax];
};

}  // namespace rw
