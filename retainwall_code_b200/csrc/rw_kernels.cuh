// Kernels of the SPH geomechanics step (sm_100a).  Layout in HBM: structure of
// arrays, one 16-byte (float) / 32-byte (double) vector per particle per field,
// particles sorted by cell key (boundary cells first, then material cells, then the
// deleted cell), so the 27 neighbour cells of a particle are 9 contiguous index runs
// per layer and neighbour reads of consecutive particles hit the same lines.
#pragma once
#include "rw_device.cuh"
#include "rw_mlp.cuh"
#include "rw_params.h"

namespace rw {

// Per-particle record consumed by the pair loop of the interaction: everything the
// reference recomputes per neighbour pair from j's state (mass, volume, sigma/rho^2),
// computed once per particle per section.  48 bytes in float: the contact-wall flag
// travels as the sign of the (always positive) volume.
template <class T> struct Rec {
  V4<T> p;   // in-cell position (w unused): one aligned 64-byte record per neighbour in float
  V4<T> vr;  // velocity xyz, density
  V4<T> a;   // mass, +-volume (negative: contact-wall particle), sigma/rho^2 xx, yy
  V4<T> b;   // sigma/rho^2 zz, xy, xz, yz
};

template <class T> struct DevState {
  // Permuted every section (ping-pong, Dyn::cur_main selects the live buffer).
  int4* codes[2];
  int4* cellpos[2];
  V4<T>* pos[2];
  V4<T>* pos_ori[2];
  V4<T>* vel[2];
  V4<T>* idm[2];
  V4<T>* str_a[2];
  V2<T>* str_b[2];
  V4<T>* stn_a[2];
  V2<T>* stn_b[2];
  // Permuted in the predictor section only (SortArraysPrimary), Dyn::cur_nrm.
  V4<T>* normal[2];
  // Permuted in the corrector section only (SortArraysAll), Dyn::cur_ini.
  V4<T>* pos_ini[2];
  V4<T>* vel_ini[2];
  V4<T>* stri_a[2];
  V2<T>* stri_b[2];
  V4<T>* stni_a[2];
  V2<T>* stni_b[2];
  // Compensation terms of the precision form (position xyz, velocity xyz+rho),
  // permuted with the particles; *_ini copies saved by the predictor.
  V4<T>* cmp_p[2];
  V4<T>* cmp_v[2];
  V4<T>* cmp_pi[2];
  V4<T>* cmp_vi[2];
  // Stage outputs, indexed like the live buffers.
  V4<T>* accad;
  V4<T>* spin;
  V4<T>* ace_a;
  V2<T>* ace_b;
  // Contact state bound to array slots, as in the reference (never permuted there).
  // contact_var and the contact force are double-buffered across the interaction so
  // that every particle reads the others' values as of the start of the stage.
  V4<T>* cv[2];   // kernel integral, distance along normal, slide flag, wall id
  V4<T>* cf[2];   // contact force xyz
  V4<T>* cny;     // contact normal (contact_mag.yx..yz)
  V4<T>* cvz;     // contact velocity (contact_mag.zx..zz)
  Rec<T>* rec;
  V4<T>* tc_a;    // Shepard result (tensor2d_cache)
  V2<T>* tc_b;
  // Cell list.
  int* keys;      // cell key per particle (unsorted order)
  int* vals;
  int* tk;        // radix-sort ping-pong
  int* tv;
  const int* skeys;  // sorted keys / permutation (one of keys|tk, vals|tv)
  const int* sperm;
  int2* range;    // [beg, end) per cell, (0,0) when empty
  int* hist;      // radix-sort digit counts, 256 x ntiles
  int* dtot;      // per-digit totals
  int ntiles, sort_passes;
  double* wsum;   // wall-force partial sums
  // Column chunks of the interaction (rebuilt after every sort).
  int* col_beg;
  int* col_len;
  int* col_cnt;
  int* col_off;
  struct Chunk* chunks;
  // Candidate lists of the soil particles (entry e of soil slot t at nbg[b][e * nbg_stride + t],
  // encoded like the shared-memory lists), count per slot (-1: not kept).  Two buffers
  // b, Dyn::lbuf the live one: a list update after a permutation reads the other.
  unsigned* nbg[2];
  int* nbg_cnt[2];
  int nbg_stride;
  // Per particle: bound on the distance moved since the last full build of the lists
  // (permuted with the particles, into the other buffer).
  float* dacc[2];
  unsigned* nbb[2];  // boundary particles' kept lists (entry e of particle i at nbb[b][e * npb + i])
  int* nbb_cnt[2];
  int* inv;          // inverse of the last permutation: new index of old index j
  int* queue;        // rows whose lists a list update rebuilds (Dyn::n_queue of them)
  unsigned* cell_mark;  // per cell: generation of its last mark (listed in marks when first marked)
  int* marks;           // the cells marked in the current generation (Dyn::n_marks, at most RW_MARK_CAP)
  unsigned* near_mark;  // per cell: generation of the last mark in its 27-cell neighbourhood
  unsigned char* near_wall;  // per cell: a contact-wall particle lies in its 27-cell neighbourhood
};

// Distinct cells one list update takes; more marked cells make it a full build.
constexpr int RW_MARK_CAP = 8192;

// Interaction block size; capacity of a kept candidate list (entries per particle).
constexpr int IX_THREADS = 128, IX_CAP = 96;
// The walk launch takes 64 or 128 (default) threads per block (RW_OPT_WALK_THREADS); a
// launch bound of 256 made the same code 14% slower.
constexpr int IX_WALK_MAX_THREADS = 128;

template <class T> RWD V3<T> ld3(const V4<T>* p, int i) { V4<T> v = p[i]; return {v.x, v.y, v.z}; }
template <class T> RWD S6<T> ld6(const V4<T>* a, const V2<T>* b, int i) {
  V4<T> x = a[i];
  V2<T> y = b[i];
  return {x.x, x.y, x.z, x.w, y.x, y.y};
}
template <class T> RWD void st6(V4<T>* a, V2<T>* b, int i, S6<T> s) {
  a[i] = V4<T>{s.xx, s.yy, s.zz, s.xy};
  b[i] = V2<T>{s.xz, s.yz};
}
template <class T> RWD bool in_grid(const Params<T>& P, I3 c) {
  return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < P.cell_num[0] && c.y < P.cell_num[1] && c.z < P.cell_num[2];
}
template <class T> RWD int key_of(const Params<T>& P, I3 c) {
  return c.x * P.cell_num[1] * P.cell_num[2] + c.y * P.cell_num[2] + c.z;
}
RWD I3 off_of(int oc) { return {oc % 3 - 1, (oc / 3) % 3 - 1, oc / 9 - 1}; }

RWD float mul_rn(float a, float b) { return __fmul_rn(a, b); }
RWD float rmul(float a, float b) { return __fmul_rn(a, b); }
RWD double rmul(double a, double b) { return __dmul_rn(a, b); }
RWD double mul_rn(double a, double b) { return __dmul_rn(a, b); }
RWD float add_rn(float a, float b) { return __fadd_rn(a, b); }
RWD double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Neighbour record of particle i (boundary: mass = V0 rho; material: idmassidx.y),
// with the reference's per-pair expressions (src/particle_interaction.cu:44-49,71).
template <class T> RWD void write_rec(const Params<T>& P, Rec<T>* rec, int i, V4<T> pos, V4<T> vr, S6<T> s, T mass,
                                      bool contact) {
  const T rho = vr.w;
  const S6<T> sor = s / rmul(rho, rho);
  const T vol = mass / rho;
  Rec<T> r;
  r.p = V4<T>{pos.x, pos.y, pos.z, T(0)};
  r.vr = vr;
  r.a = V4<T>{mass, contact ? -vol : vol, sor.xx, sor.yy};
  r.b = V4<T>{sor.zz, sor.xy, sor.xz, sor.yz};
  if constexpr (sizeof(T) == 4) {  // two 256-bit stores (sm_100)
    float* q = reinterpret_cast<float*>(rec + i);
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(q), "f"(r.p.x), "f"(r.p.y), "f"(r.p.z),
                 "f"(r.p.w), "f"(r.vr.x), "f"(r.vr.y), "f"(r.vr.z), "f"(r.vr.w)
                 : "memory");
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(q + 8), "f"(r.a.x), "f"(r.a.y),
                 "f"(r.a.z), "f"(r.a.w), "f"(r.b.x), "f"(r.b.y), "f"(r.b.z), "f"(r.b.w)
                 : "memory");
  } else {
    rec[i] = r;
  }
}

// The neighbour-side values one pair term needs.
template <class T> struct NbVals {
  V4<T> p, vr, a, b;
};
template <class T> RWD NbVals<T> load_nb(const Rec<T>* __restrict__ rec, int j) {
  NbVals<T> v;
  v.p = rec[j].p;
  v.vr = rec[j].vr;
  v.a = rec[j].a;
  v.b = rec[j].b;
  return v;
}
// Float records: two 256-bit loads (sm_100) instead of four 128-bit ones.  Half the load
// instructions and L1 requests per neighbour; the walk kernel's L1 request rate is what
// bounds it.  Records are 64 bytes from a 256-byte aligned cudaMalloc base.
static_assert(sizeof(Rec<float>) == 64, "float records are one 64-byte line");
template <> RWD NbVals<float> load_nb<float>(const Rec<float>* __restrict__ rec, int j) {
  NbVals<float> v;
  const float* q = reinterpret_cast<const float*>(rec + j);
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(v.p.x), "=f"(v.p.y), "=f"(v.p.z), "=f"(v.p.w), "=f"(v.vr.x), "=f"(v.vr.y), "=f"(v.vr.z), "=f"(v.vr.w)
      : "l"(q));
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(v.a.x), "=f"(v.a.y), "=f"(v.a.z), "=f"(v.a.w), "=f"(v.b.x), "=f"(v.b.y), "=f"(v.b.z), "=f"(v.b.w)
      : "l"(q + 8));
  return v;
}

// ---------------------------------------------------------------------------------
// Case ingest: the caller's arrays (array of structures, double) -> the device layout.
// ---------------------------------------------------------------------------------
struct RawCase {
  const int4* codes;
  const double* pospres;
  const double* velrhop;
  const double* idmassidx;
  const double* stress;
  const double* strain;
  const double* normal;
};

// One particle of LoadParticles' values with the absolute -> in-cell split of
// PositionFromAbsolute2Relative (src/loquat_grid.cu:253-271): cell = trunc(x * (0.5/h)),
// the product rounded on its own, in-cell position = x - cell * 2h with one rounding, as
// the reference's kernel computes them.
template <class T> __global__ void k_ingest(const Params<T> P, DevState<T> S, RawCase R, T half_ih) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)P.np) return;
  S.codes[0][i] = R.codes[i];
  const double* a = R.pospres + 4 * i;
  const V4<T> pa{(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
  S.pos_ori[0][i] = pa;
  const int cx = (int)rmul(pa.x, half_ih), cy = (int)rmul(pa.y, half_ih), cz = (int)rmul(pa.z, half_ih);
  S.cellpos[0][i] = int4{cx, cy, cz, 0};
  // x - c 2h as one fused multiply-add: the reference's kernel (cuPositionFromAbsolute2Relative,
  // src/loquat_grid.cu:253-261) is compiled with contraction, which fuses that product
  // into the subtraction
  S.pos[0][i] = V4<T>{f_fma(-(T)cx, P.two_h, pa.x), f_fma(-(T)cy, P.two_h, pa.y), f_fma(-(T)cz, P.two_h, pa.z), pa.w};
  a = R.velrhop + 4 * i;
  S.vel[0][i] = V4<T>{(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
  a = R.idmassidx + 4 * i;
  S.idm[0][i] = V4<T>{(T)a[0], (T)a[1], (T)i, (T)a[3]};
  a = R.stress + 6 * i;
  S.str_a[0][i] = V4<T>{(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
  S.str_b[0][i] = V2<T>{(T)a[4], (T)a[5]};
  a = R.strain + 6 * i;
  S.stn_a[0][i] = V4<T>{(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
  S.stn_b[0][i] = V2<T>{(T)a[4], (T)a[5]};
  if (i < (size_t)P.npb) {
    a = R.normal + 4 * i;
    S.normal[0][i] = V4<T>{(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
  }
}

// ---------------------------------------------------------------------------------
// Cell list: keys, stable radix sort, ranges, gather-permute
// (src/loquat_grid.cu:71-261, src/loquat.cu:254-287).
// ---------------------------------------------------------------------------------

// cuGetParticleCellIndex (src/loquat_grid.cu:71-95).  A live particle whose cell is
// outside the grid would make the reference write out of bounds; here its key is
// clamped into the grid and RW_DERR_CELL_RANGE is raised.
template <class T> __global__ void k_keys(const Params<T> P, DevState<T> S, Dyn<T>* dyn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) dyn->need_sort = 0;
  if (i >= P.np || !dyn->cells_dirty) return;  // no cell changed: keys, order and ranges stand
  const int c = dyn->cur_main;
  int4 cp = S.cellpos[c][i];
  int key;
  if (cp.w == P.ncell_delete_m) {
    key = P.ncell_delete_m;
  } else {
    I3 cc{cp.x, cp.y, cp.z};
    if (!in_grid(P, cc)) {
      atomicOr(&dyn->err, 1u);
      cc.x = min(max(cc.x, 0), P.cell_num[0] - 1);
      cc.y = min(max(cc.y, 0), P.cell_num[1] - 1);
      cc.z = min(max(cc.z, 0), P.cell_num[2] - 1);
    }
    key = key_of(P, cc);
    if (!(S.idm[c][i].x < T(RW_MATERIAL_NUMBER))) key += P.ncell_material;
    S.cellpos[c][i].w = key;
  }
  S.keys[i] = key;
  S.vals[i] = i;
}

static __global__ void k_check_sorted(const int* keys, int n, int* need_sort, const int* dirty = nullptr) {
  if (dirty && !*dirty) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const bool out_of_order = i < n && keys[i - 1] > keys[i];
  // one store per warp that found a key out of order: in an unsorted array every thread
  // would otherwise store to the same word (measured 50 us instead of 6 us at 0.96M)
  if (__any_sync(0xffffffffu, out_of_order) && (threadIdx.x & 31) == 0) *need_sort = 1;
}

// Clears n words when the cells changed since the last search.
static __global__ void k_clear_if(unsigned* p, size_t n, const int* dirty) {
  if (!*dirty) return;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) p[k] = 0u;
}

constexpr int RS_THREADS = 256, RS_ITEMS = 8, RS_TILE = RS_THREADS * RS_ITEMS;

// LSD radix sort, 8-bit digits, stable: upsweep (per-tile digit counts), scan
// (per digit over tiles), downsweep (stable in-tile ranks + scatter).  All three
// return immediately when the keys are already in order (the permutation is then
// the identity, exactly what a stable sort of sorted keys returns).
static __global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const int* keys, int n, int shift, int* hist, int ntiles,
                                                         const int* need) {
  if (!*need) return;
  __shared__ int h[256];
  const int t = threadIdx.x;
  h[t] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
#pragma unroll
  for (int k = 0; k < RS_ITEMS; ++k) {
    int idx = base + k * RS_THREADS + t;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255], 1);
  }
  __syncthreads();
  hist[t * ntiles + blockIdx.x] = h[t];
}

static __device__ __forceinline__ int block_excl_scan256(int v, int* total) {
  __shared__ int ws[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < 8 ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < 8) ws[lane] = s;
  }
  __syncthreads();
  int incl = x + (w > 0 ? ws[w - 1] : 0);
  if (total) *total = ws[7];
  __syncthreads();
  return incl - v;
}

// One block per digit: exclusive scan of that digit's per-tile counts.
static __global__ void __launch_bounds__(RS_THREADS) k_rs_scan(int* hist, int ntiles, int* dtot, const int* need) {
  if (!*need) return;
  int* row = hist + blockIdx.x * ntiles;
  const int per = (ntiles + RS_THREADS - 1) / RS_THREADS;
  const int b = threadIdx.x * per, e = min(ntiles, b + per);
  int s = 0;
  for (int k = b; k < e; ++k) s += row[k];
  int total;
  int off = block_excl_scan256(s, &total);
  for (int k = b; k < e; ++k) {
    int v = row[k];
    row[k] = off;
    off += v;
  }
  if (threadIdx.x == 0) dtot[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(RS_THREADS) k_rs_downsweep(const int* kin, const int* vin, int* kout, int* vout, int n,
                                                           int shift, const int* hist, const int* dtot, int ntiles,
                                                           const int* need) {
  if (!*need) return;
  __shared__ int base[256];
  __shared__ int wcnt[8][257];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int dt_excl = block_excl_scan256(dtot[t], nullptr);
  base[t] = dt_excl + hist[t * ntiles + blockIdx.x];
  const unsigned lt = (1u << lane) - 1u;
  const int tile0 = blockIdx.x * RS_TILE;
  for (int r = 0; r < RS_ITEMS; ++r) {
#pragma unroll
    for (int q = 0; q < 8; ++q) wcnt[q][t] = 0;
    __syncthreads();
    const int idx = tile0 + r * RS_THREADS + t;
    const bool valid = idx < n;
    int key = 0, d = 256;
    if (valid) {
      key = kin[idx];
      d = (key >> shift) & 255;
    }
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int rank = __popc(peers & lt);
    int leader = __ffs(peers) - 1;
    if (lane == leader && valid) wcnt[w][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pre = 0;
      for (int q = 0; q < w; ++q) pre += wcnt[q][d];
      int pos = base[d] + pre + rank;
      if (pos >= 0 && pos < n) {  // always true for consistent counts; guards the scatter
        kout[pos] = key;
        vout[pos] = vin[idx];
      }
    }
    __syncthreads();
    int add = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) add += wcnt[q][t];
    base[t] += add;
    __syncthreads();
  }
}

// cuFindBegEndInCell (src/loquat_grid.cu:116-144): [beg, end) of every occupied cell.
template <class T> __global__ void k_ranges(const Params<T> P, DevState<T> S, const Dyn<T>* dyn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.np || !dyn->cells_dirty) return;
  const int* K = dyn->need_sort ? S.skeys : S.keys;
  const int k = K[i];
  int* r = reinterpret_cast<int*>(S.range);
  if (i == 0 || K[i - 1] != k) r[2 * k] = i;
  if (i == P.np - 1 || K[i + 1] != k) r[2 * k + 1] = i + 1;
}

// Deleted-particle accounting (src/loquat_grid.cu:164-190), on the device.
template <class T> __global__ void k_count(const Params<T> P, DevState<T> S, Dyn<T>* dyn) {
  if (!dyn->cells_dirty) return;
  int2 d = S.range[P.ncell_delete_m];
  int cnt = d.y - d.x;
  if (cnt > 0) {
    int now = cnt - dyn->np_delete_m;
    if (now != 0) {
      dyn->npm -= now;
      dyn->np_delete_m += now;
    }
  }
  if (P.npb + dyn->npm + dyn->np_delete_m != P.np) atomicOr(&dyn->err, 2u);
}

// SortArraysPrimary (section 0) / SortArraysAll (section 1), src/loquat.cu:254-287,
// as one gather into the other ping-pong buffer.  Stress/strain beyond npb+npm are
// not part of the reference's sorted range; they keep their slot values.
template <class T> __global__ void k_permute(const Params<T> P, DevState<T> S, const Dyn<T>* dyn, int section,
                                             int compat_contact) {
  if (!dyn->need_sort) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.np) return;
  int j = S.sperm[i];
  if (j < 0 || j >= P.np) {  // a valid permutation never gets here
    atomicOr(&const_cast<Dyn<T>*>(dyn)->err, 8u);
    j = i;
  }
  const int c = dyn->cur_main, n = c ^ 1;
  S.codes[n][i] = S.codes[c][j];
  S.cellpos[n][i] = S.cellpos[c][j];
  S.pos[n][i] = S.pos[c][j];
  S.pos_ori[n][i] = S.pos_ori[c][j];
  S.vel[n][i] = S.vel[c][j];
  S.idm[n][i] = S.idm[c][j];
  if (P.mixed) {
    S.cmp_p[n][i] = S.cmp_p[c][j];
    S.cmp_v[n][i] = S.cmp_v[c][j];
  }
  // the lists' displacement bounds move with the particles (k_flip then flips lbuf), and
  // a list update maps the entries through the inverse
  const int lb = dyn->lbuf;
  S.dacc[lb ^ 1][i] = S.dacc[lb][j];
  S.inv[j] = i;
  const int npm = dyn->npm;
  const int nbm = P.npb + npm;
  const bool perm_str = (section == 0) || (npm != 0);
  const int ss = (perm_str && i < nbm) ? j : i;
  S.str_a[n][i] = S.str_a[c][ss];
  S.str_b[n][i] = S.str_b[c][ss];
  S.stn_a[n][i] = S.stn_a[c][ss];
  S.stn_b[n][i] = S.stn_b[c][ss];
  if (section == 0) {
    const int cn = dyn->cur_nrm;
    if (i < P.npb) S.normal[cn ^ 1][i] = S.normal[cn][j];
  } else {
    const int ci = dyn->cur_ini, ni = ci ^ 1;
    S.pos_ini[ni][i] = S.pos_ini[ci][j];
    S.vel_ini[ni][i] = S.vel_ini[ci][j];
    S.stri_a[ni][i] = S.stri_a[ci][ss];
    S.stri_b[ni][i] = S.stri_b[ci][ss];
    S.stni_a[ni][i] = S.stni_a[ci][ss];
    S.stni_b[ni][i] = S.stni_b[ci][ss];
    if (P.mixed) {
      S.cmp_pi[ni][i] = S.cmp_pi[ci][j];
      S.cmp_vi[ni][i] = S.cmp_vi[ci][j];
    }
  }
  (void)compat_contact;
}

// Buffer flip after a permute; in the predictor section also RigidBodyUpdate
// (src/adami_boundary.cu:175-203), which the reference runs right after the sort.
// Plain round-to-nearest products/sums, as the reference's host code computes.
template <class T> __global__ void k_flip(const Params<T> P, Dyn<T>* dyn, int section, int rigid, int lists) {
  if (section >= 0 && dyn->need_sort) {
    dyn->cur_main ^= 1;
    if (section == 0) dyn->cur_nrm ^= 1;
    else dyn->cur_ini ^= 1;
    dyn->n_sorts += 1;
    dyn->lbuf ^= 1;  // k_permute carried the displacement bounds into the other buffer
  }
  // Candidate lists.  An interaction walks the kept lists (mode 1) when nothing was
  // permuted and no particle changed cell since they were built or updated.  When
  // particles changed cell (marked cells) in the step before a predictor section, the
  // lists are updated (mode 2): the lists of particles next to a marked cell are
  // rebuilt, the others carried through the permutation.  Every list is built anew
  // (mode 0) when some particle moved more than the skin allows since the last full
  // build (list_kill, raised by the integrators), after a host write, with too many
  // marked cells, or in the corrector section: lists built there, from mid-step
  // positions, are not kept, and a displacement bound counted from the start of the
  // step does not cover them.  Without kept soil lists (lists = 0: lists off, or the
  // chunked kernel) every section is mode 0 and no list stands.
  if (section >= 0) {
    if (dyn->need_sort || dyn->host_dirty) dyn->rec_stale = 1;  // until the next interaction
    dyn->host_dirty = 0;
    dyn->cells_dirty = 0;  // the search is complete
    int mode = 1;
    if (!lists || !dyn->list_ok || dyn->list_kill || dyn->n_marks > RW_MARK_CAP) mode = 0;
    else if (dyn->need_sort || dyn->n_marks > 0) mode = section == 0 ? 2 : 0;
    dyn->ix_mode = mode;
    dyn->n_reuse += mode == 1;
    dyn->n_updates += mode == 2;
    // the marks are consumed: the update tests this generation, new marks take the next
    dyn->near_gen = dyn->mark_gen;
    dyn->mark_gen += 1;
    dyn->n_marks = 0;
    dyn->n_queue = 0;
    if (mode == 0) {
      dyn->list_ok = 0;
      dyn->list_kill = 0;
      dyn->build_kill = section;
      dyn->n_spill = 0;
    }
  }
  if (!rigid) return;
  const T dt = P.dt;
  const T time = dyn->time_f;
  for (int i = 0; i < P.n_motion; ++i) {
    Table<T>& tb = dyn->tab[i];
    Motion<T>& mv = dyn->mv[i];
    if (tb.is_rotation) {
      for (int j = 0; j < tb.n_rot; ++j) {
        if (time < tb.rotat_time[j]) {
          tb.rotat_vel.x = add_rn(tb.rotat_vel.x, mul_rn(tb.rotat_acc[j].x, dt));
          tb.rotat_vel.y = add_rn(tb.rotat_vel.y, mul_rn(tb.rotat_acc[j].y, dt));
          tb.rotat_vel.z = add_rn(tb.rotat_vel.z, mul_rn(tb.rotat_acc[j].z, dt));
          const T hdt = (T)(0.5 * (double)dt);
          Vec3<T> vel{add_rn(tb.trans_vel[j].x, mul_rn(tb.trans_acc[j].x, hdt)),
                      add_rn(tb.trans_vel[j].y, mul_rn(tb.trans_acc[j].y, hdt)),
                      add_rn(tb.trans_vel[j].z, mul_rn(tb.trans_acc[j].z, hdt))};
          tb.pos_rp.x = add_rn(tb.pos_rp.x, mul_rn(vel.x, dt));
          tb.pos_rp.y = add_rn(tb.pos_rp.y, mul_rn(vel.y, dt));
          tb.pos_rp.z = add_rn(tb.pos_rp.z, mul_rn(vel.z, dt));
          mv.rotat_acc = tb.rotat_acc[j];
          mv.rotat_vel = tb.rotat_vel;
          mv.pos_rp = tb.pos_rp;
          break;
        }
      }
    }
    if (tb.is_translation) {
      for (int j = 0; j < tb.n_trans; ++j) {
        if (time < tb.trans_time[j]) {
          tb.trans_vel[j].x = add_rn(tb.trans_vel[j].x, mul_rn(tb.trans_acc[j].x, dt));
          tb.trans_vel[j].y = add_rn(tb.trans_vel[j].y, mul_rn(tb.trans_acc[j].y, dt));
          tb.trans_vel[j].z = add_rn(tb.trans_vel[j].z, mul_rn(tb.trans_acc[j].z, dt));
          mv.trans_acc = tb.trans_acc[j];
          mv.trans_vel = tb.trans_vel[j];
          break;
        }
      }
    }
  }
}

// Gates of a captured step graph: one-thread kernels that set the condition of the IF
// node holding work that would otherwise launch only to return at once.
// Search: keys, sort, ranges, counts, permutation and contact-wall cells have nothing to
// do when no particle changed cell (what k_keys does then is clear need_sort).
template <class T> __global__ void k_search_gate(Dyn<T>* dyn, cudaGraphConditionalHandle h) {
  const int d = dyn->cells_dirty;
  if (!d) {
    dyn->need_sort = 0;
    dyn->n_search_skipped += 1;
  }
  cudaGraphSetConditional(h, d ? 1u : 0u);
}
// List build: needed when the lists are to be built or updated (modes 0 and 2, lists on).
template <class T>
__global__ void k_build_gate(const Params<T> P, DevState<T> S, Dyn<T>* dyn, cudaGraphConditionalHandle h) {
  const bool run = S.nbg[0] && P.keep_lists && dyn->ix_mode != 1;
  if (!run) dyn->n_build_skipped += 1;
  cudaGraphSetConditional(h, run ? 1u : 0u);
}
// Interaction scan launch: needed with lists off, when some list of the last build
// overflowed, or for deleted slots (their contact state is carried).
template <class T>
__global__ void k_scan_gate(const Params<T> P, DevState<T> S, Dyn<T>* dyn, cudaGraphConditionalHandle h) {
  const bool run = !(S.nbg[0] && P.keep_lists) || dyn->n_spill > 0 || dyn->npm < P.np - P.npb;
  if (!run) {
    dyn->rec_stale = 0;  // what the scan launch does first
    dyn->n_scan_skipped += 1;
  }
  cudaGraphSetConditional(h, run ? 1u : 0u);
}

template <class T> __global__ void k_begin(Dyn<T>* dyn) { dyn->time_f = (T)dyn->time_d; }
template <class T> __global__ void k_end(const Params<T> P, Dyn<T>* dyn) {
  dyn->time_d += (double)P.dt;
  dyn->step += 1;
}

// ---------------------------------------------------------------------------------
// Periodic planes (period-bound cases).  Dist2Plane / AbsDist2Plane
// (src/functions.h:134-139); every operation separately rounded, so the decisions and
// the image coordinates match the oracle bit for bit.
// ---------------------------------------------------------------------------------
template <class T> RWD T plane_dist(const T* pl, const V3<T> a) {
  using F = Fp<true>;
  const T num = F::mad(a.z, pl[2], F::mad(a.y, pl[1], F::mul(a.x, pl[0]))) + pl[3];
  return num / pair_r(pair_r2(pl[0], pl[1], pl[2]));
}

template <class T> RWD V3<T> abs_pos(const V3<T> p, const I3 c, T th) {
  using F = Fp<true>;
  return V3<T>{F::mad((T)c.x, th, p.x), F::mad((T)c.y, th, p.y), F::mad((T)c.z, th, p.z)};
}

// Absolute position pabs moved by one period along the plane pl, as a cell and an
// in-cell position.
template <class T> RWD void period_shift(const Params<T>& P, const V3<T> pabs, const T* pl, T len, I3& cpb,
                                         V3<T>& ppb) {
  using F = Fp<true>;
  const V3<T> pb{F::mad(pl[0], len, pabs.x), F::mad(pl[1], len, pabs.y), F::mad(pl[2], len, pabs.z)};
  const T s = F::mul(T(0.5f), P.i_h);
  cpb = I3{int(F::mul(pb.x, s)), int(F::mul(pb.y, s)), int(F::mul(pb.z, s))};
  ppb = V3<T>{F::msub((T)cpb.x, P.two_h, pb.x), F::msub((T)cpb.y, P.two_h, pb.y), F::msub((T)cpb.z, P.two_h, pb.z)};
}

// Periodic image of a particle within 2h of a periodic plane (the *LoopPeriod helpers:
// src/adami_boundary.cu:73-88, src/field_smoothing.cu:58-72,
// src/particle_interaction.cu:243-257).  The period is |D_left + D_right| in the Adami
// and Shepard loops (abs_len) and the signed sum in the interaction.
template <class T> RWD bool period_image(const Params<T>& P, const I3 celli, const V3<T> pos_i, bool abs_len,
                                         I3& cpb, V3<T>& ppb) {
  const V3<T> pabs = abs_pos(pos_i, celli, P.two_h);
  const bool left = f_abs(plane_dist(P.planeleft, pabs)) < P.two_h;
  const bool right = f_abs(plane_dist(P.planeright, pabs)) < P.two_h;
  if (!left && !right) return false;
  T len = P.planeleft[3] + P.planeright[3];
  if (abs_len) len = f_abs(len);
  period_shift(P, pabs, left ? P.planeleft : P.planeright, len, cpb, ppb);
  return true;
}

// A particle that left through a periodic plane re-enters through the other one
// (cuCheckOutDomainPeriod, src/predictor_corrector.cu:26-40).
template <class T> RWD void period_wrap(const Params<T>& P, int4& cp, V4<T>& ps) {
  const V3<T> pabs = abs_pos(xyz(ps), I3{cp.x, cp.y, cp.z}, P.two_h);
  const bool left = plane_dist(P.planeleft, pabs) < T(0.0);
  const bool right = plane_dist(P.planeright, pabs) < T(0.0);
  if (!left && !right) return;
  I3 c;
  V3<T> pr;
  period_shift(P, pabs, left ? P.planeleft : P.planeright, f_abs(P.planeleft[3] + P.planeright[3]), c, pr);
  cp = int4{c.x, c.y, c.z, cp.w};
  ps = V4<T>{pr.x, pr.y, pr.z, ps.w};
}

// A list update rebuilds the list of a particle in cell c when c lies next to a cell
// marked in the generation being consumed; a cell outside the grid (a wall particle
// moved out of it) always counts as marked.
template <class T> RWD bool near_marked(const Params<T>& P, const DevState<T>& S, const Dyn<T>* dyn, I3 c) {
  return !in_grid(P, c) || S.near_mark[key_of(P, c)] == dyn->near_gen;
}

// A kept list carried through a permutation: the list of old index o (column o of the
// other buffer) becomes the list of new index i, each entry's particle index mapped to
// its new index; the cell offsets and the order stand (a stable sort keeps the order
// inside every cell whose particles all stayed).
RWD void carry_list(const unsigned* __restrict__ src, const int* __restrict__ src_cnt, int o, unsigned* __restrict__ dst,
                    int* __restrict__ dst_cnt, int i, size_t stride, const int* __restrict__ inv) {
  constexpr unsigned kIdx = 0x7ffffffu;  // entry: particle index in the low 27 bits
  const int cnt = src_cnt[o];
  dst_cnt[i] = cnt;
  // eight entries at a time, their loads and index lookups issued together (a thread
  // waits for two loads per eight entries, not two per entry)
  for (int e0 = 0; e0 < cnt; e0 += 8) {
    unsigned v[8];
    int m[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = e0 + k < cnt ? __ldcs(src + (size_t)(e0 + k) * stride + o) : 0u;
#pragma unroll
    for (int k = 0; k < 8; ++k) m[k] = e0 + k < cnt ? inv[v[k] & kIdx] : 0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (e0 + k < cnt) __stcs(dst + (size_t)(e0 + k) * stride + i, (unsigned)m[k] | (v[k] & ~kIdx));
  }
}

// ---------------------------------------------------------------------------------
// Adami boundary (src/adami_boundary.cu:26-158).
// ---------------------------------------------------------------------------------
template <class T> __global__ void __launch_bounds__(128) k_adami(const Params<T> P, DevState<T> S, const Dyn<T>* dyn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.npb) return;
  if (dyn->ix_mode == 0) S.dacc[dyn->lbuf][i] = 0.0f;  // candidate lists are rebuilt from these positions
  if (dyn->npm == 0) return;
  const int c = dyn->cur_main;
  const V4<T>* __restrict__ pos = S.pos[c];
  const V4<T>* __restrict__ vel = S.vel[c];
  const V4<T>* __restrict__ idm = S.idm[c];
  const V4<T>* __restrict__ sa = S.str_a[c];
  const V2<T>* __restrict__ sb = S.str_b[c];
  const V3<T> pos_i = ld3(pos, i);
  const int4 cp = S.cellpos[c][i];
  const I3 celli{cp.x, cp.y, cp.z};
  const int4 code = S.codes[c][i];
  const bool contact = code.x >= 10;
  S6<T> rs = zero6<T>();
  V4<T> rps{T(0), T(0), T(0), T(0)}, rvr{T(0), T(0), T(0), T(0)};
  V3<T> n_i{T(0), T(0), T(0)};
  const T th = P.two_h;
  // One neighbour j at dr = (pos_i - pos_j) - offset 2h: boundary j (contact walls
  // only) feeds the wall normal, material j the extrapolation sums.
  // mat(v, m, s) supplies material j's velocity-density, mass and stress.
  auto pair = [&](int j, const V3<T> dr, const T r2, auto&& mat) {
    if (!(r2 < P.r2_prefilter)) return;  // conservative: q >= 2 beyond it
    const T r = pair_r(r2);
    const T q = r * P.i_h;
    if (!(q < T(2.0f))) return;
    if (j < P.npb) {
      T dwdr = kernel_f(P.kgrad, q);
      V3<T> gker = dr * dwdr;
      n_i = n_i - gker * P.vol_def;
    } else {
      T ker = kernel_w(P.knorm, q);
      V4<T> vj;
      T mj;
      S6<T> sj;
      mat(vj, mj, sj);
      T vol_j = mj / vj.w;
      T kv = ker * vol_j;
      rs = rs + sj * kv;
      rps = rps + v4(dr * (ker * mj), kv);
      rvr = rvr + vj * kv;
    }
  };
  auto mat_of = [&](int j) {
    return [&, j](V4<T>& v, T& m, S6<T>& s) {
      v = vel[j];
      m = idm[j].y;
      s = ld6(sa, sb, j);
    };
  };
  const int lb = dyn->lbuf;
  unsigned* __restrict__ nbb = S.nbb[lb];
  // The 27 cells in the reference's order; with `keep`, the candidates within the list
  // radius are recorded (same order) for later sections.
  auto scan = [&](const I3 cc, const V3<T> pp, bool keep) {
    int cnt = 0;
    for (int oc = 0; oc < 27; ++oc) {
      const I3 off = off_of(oc);
      const I3 cj{cc.x + off.x, cc.y + off.y, cc.z + off.z};
      if (!in_grid(P, cj)) continue;
      const int k = key_of(P, cj);
      const V3<T> o = mulI(off, th);
      for (int layer = contact ? 0 : 1; layer < 2; ++layer) {
        const int2 rg = S.range[layer ? k + P.ncell_material : k];
        for (int j = rg.x; j < rg.y; ++j) {
          V3<T> dr = pp - ld3(pos, j);
          dr = dr - o;
          const T r2 = pair_r2(dr.x, dr.y, dr.z);
          if (keep && r2 < P.r2_list) {
            if (cnt < IX_CAP) nbb[(size_t)cnt * P.npb + i] = (unsigned)j | ((unsigned)oc << 27);
            ++cnt;
          }
          pair(j, dr, r2, mat_of(j));
        }
      }
    }
    if (keep) S.nbb_cnt[lb][i] = cnt <= IX_CAP ? cnt : -1;
  };
  const bool keep = S.nbb[0] && P.keep_lists;
  const int mode = keep ? dyn->ix_mode : 0;
  // In a list update (mode 2) the lists next to a marked cell were rebuilt and the
  // others carried through this section's permutation, if any, before this kernel
  // (k_build_lists, k_rebuild_lists); only a full build (mode 0) keeps them here.
  const bool rebuild = mode == 0;
  const int kept = (mode != 0 && !rebuild) ? S.nbb_cnt[lb][i] : -1;
  if (kept >= 0) {
    // Walk the kept list four entries at a time, each batch's neighbour data loaded
    // together and the next batch's entries loaded while it is in flight: a thread next
    // to the soil waits for about one load per four entries instead of a chain of loads
    // per entry.
    constexpr unsigned kNone = 0x7ffffffu;  // index of no particle (np < 2^27)
    auto entries = [&](int e0, unsigned* ent) {
#pragma unroll
      for (int k = 0; k < 4; ++k) ent[k] = e0 + k < kept ? __ldcs(nbb + (size_t)(e0 + k) * P.npb + i) : kNone;
    };
    unsigned ent[4], nxt[4];
    entries(0, ent);
    for (int e0 = 0; e0 < kept; e0 += 4) {
      V4<T> pj[4], vj[4];
      T mj[4];
      S6<T> sj[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int j = (int)(ent[k] & kNone);
        if (j == (int)kNone) continue;
        pj[k] = pos[j];
        if (j >= P.npb) {
          vj[k] = vel[j];
          mj[k] = idm[j].y;
          sj[k] = ld6(sa, sb, j);
        }
      }
      entries(e0 + 4, nxt);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int j = (int)(ent[k] & kNone);
        if (j == (int)kNone) continue;
        V3<T> dr = pos_i - V3<T>{pj[k].x, pj[k].y, pj[k].z};
        dr = dr - mulI(off_of((int)(ent[k] >> 27)), th);
        pair(j, dr, pair_r2(dr.x, dr.y, dr.z), [&](V4<T>& v, T& m, S6<T>& s6) {
          v = vj[k];
          m = mj[k];
          s6 = sj[k];
        });
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) ent[k] = nxt[k];
    }
  } else {
    scan(celli, pos_i, rebuild && keep);
  }
  if (P.periodbound) {
    I3 cpb;
    V3<T> ppb;
    if (period_image(P, celli, pos_i, true, cpb, ppb)) scan(cpb, ppb, false);
  }
  if (enorm(n_i) > T(0)) {
    T nn = enorm(n_i);
    S.cny[i] = V4<T>{n_i.x / nn, n_i.y / nn, n_i.z / nn, T(0)};
  }
  V4<T> vr_out = vel[i];
  S6<T> str_out;
  if (rps.w > T(0.0f)) {
    const T kersum = rps.w;
    const V3<T> dr_ref = xyz(rps);
    const V4<T> nrm4 = S.normal[dyn->cur_nrm][i];
    const T fcoef = nrm4.w;
    const V3<T> nrm = xyz(nrm4);
    const V3<T> vel_ref = xyz(rvr) / kersum;
    const V3<T> vel_ref_n = nrm * dot(nrm, vel_ref);
    const V3<T> vel_ref_t = vel_ref - vel_ref_n;
    V3<T> vel_rb{T(0.0f), T(0.0f), T(0.0f)};
    if (code.y == 1) {
      const Motion<T>& mv = dyn->mv[code.w];
      vel_rb = V3<T>{mv.trans_vel.x, mv.trans_vel.y, mv.trans_vel.z};
      if (mv.is_rotat) {
        V3<T> pabs = pos_i + mulI(celli, T(2.0f) * P.h);
        V3<T> rp{mv.pos_rp.x, mv.pos_rp.y, mv.pos_rp.z};
        V3<T> w{mv.rotat_vel.x, mv.rotat_vel.y, mv.rotat_vel.z};
        vel_rb = vel_rb + cross(w, pabs - rp);
      }
    }
    const V3<T> vel_rb_n = nrm * dot(nrm, vel_rb);
    const V3<T> vel_rb_t = vel_rb - vel_rb_n;
    const V3<T> vel_ext_n = vel_rb_n * T(2.0f) - vel_ref_n;
    const V3<T> vel_ext_t = fcoef == T(-1.0f) ? vel_rb_t * T(2.0f) - vel_ref_t : vel_ref_t;
    const V3<T> vel_ext = vel_ext_n + vel_ext_t;
    const T rho = rvr.w / kersum;
    vr_out = v4(vel_ext, rho);
    if (contact) {
      vr_out = v4(vel_rb, rho);
      S.cvz[i] = V4<T>{vel_ext.x, vel_ext.y, vel_ext.z, T(0)};
    }
    const S6<T> str_ref = rs / kersum;
    const V3<T> g{P.gravity[0], P.gravity[1], P.gravity[2]};
    str_out = subdiag(str_ref, (g * dr_ref) / kersum);
    S.vel[c][i] = vr_out;
  } else {
    str_out = zero6<T>();
  }
  st6(S.str_a[c], S.str_b[c], i, str_out);
  write_rec(P, S.rec, i, S.pos[c][i], vr_out, str_out, P.vol_def * vr_out.w, contact);
}

// ---------------------------------------------------------------------------------
// Nearest contact-wall particle / corner rule (src/adami_boundary.cu:209-292), plus
// the material neighbour records for the interaction.
// ---------------------------------------------------------------------------------
// Cells within one cell of a contact-wall particle (codes.x >= 10): the only cells whose
// soil particles can find a contact wall in cuFindCornerParticleMaterial's 27-cell scan.
// near_wall is cleared before each search's marking.
template <class T> __global__ void k_mark_near_wall(const Params<T> P, DevState<T> S, const Dyn<T>* dyn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.npb || !dyn->cells_dirty) return;
  const int c = dyn->cur_main;
  if (S.codes[c][i].x < 10) return;
  const int4 cp = S.cellpos[c][i];
  for (int oc = 0; oc < 27; ++oc) {
    const I3 off = off_of(oc);
    const I3 cj{cp.x + off.x, cp.y + off.y, cp.z + off.z};
    if (in_grid(P, cj)) S.near_wall[key_of(P, cj)] = 1;
  }
}

// Cells next to a marked cell (its 27-cell neighbourhood), tagged with the current
// mark generation: a list update rebuilds the lists of the particles in them.
// Grid-stride over (marked cell, neighbour) pairs.
template <class T> __global__ void k_mark_dilate(const Params<T> P, DevState<T> S, const Dyn<T>* dyn) {
  const int n = dyn->n_marks;
  if (n > RW_MARK_CAP) return;  // a full build follows
  const unsigned gen = dyn->mark_gen;
  const int ny = P.cell_num[1], nz = P.cell_num[2];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 27 * n; k += gridDim.x * blockDim.x) {
    const int key = S.marks[k / 27];
    const I3 off = off_of(k % 27);
    const I3 cj{key / (ny * nz) + off.x, (key / nz) % ny + off.y, key % nz + off.z};
    if (in_grid(P, cj)) S.near_mark[key_of(P, cj)] = gen;
  }
}

template <class T> __global__ void __launch_bounds__(128) k_corner(const Params<T> P, DevState<T> S, const Dyn<T>* dyn,
                                                                  int cpar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int npm = dyn->npm;
  if (t >= npm) return;
  const int i = P.npb + t;
  const int c = dyn->cur_main;
  const V4<T>* __restrict__ pos = S.pos[c];
  const V3<T> pos_i = ld3(pos, i);
  const int4 cp = S.cellpos[c][i];
  const I3 celli{cp.x, cp.y, cp.z};
  V4<T> cv = S.cv[cpar][i];
  const bool near = P.npb > 0 && in_grid(P, celli) && S.near_wall[key_of(P, celli)];
  if (!near) {  // no contact-wall particle within the 27 cells: the scan would find nothing
    if (cv.x != T(0.0f) || cv.y != T(999)) {
      cv.x = T(0.0f);
      cv.y = T(999);
      S.cv[cpar][i] = cv;
    }
    if (dyn->rec_stale)
      write_rec(P, S.rec, i, S.pos[c][i], S.vel[c][i], ld6(S.str_a[c], S.str_b[c], i), S.idm[c][i].y,
                S.codes[c][i].x >= 10);
    return;
  }
  cv.x = T(0.0f);
  cv.y = T(999);
  T d_ij = T(999);
  V4<T> ny = S.cny[i];
  V4<T> vz = S.cvz[i];
  const T th = P.two_h;
  // One boundary candidate j at in-cell position pj, in the cell at offset off (the body
  // of the reference's scan).  contact(): j belongs to a contact wall; vel_of(): its
  // velocity.
  auto visit = [&](int j, const I3 off, const V3<T> pj, auto&& contact, auto&& vel_of) {
    V3<T> dr = pos_i - pj - mulI(off, th);
    const T r2 = pair_r2(dr.x, dr.y, dr.z);
    if (!(r2 < P.r2_prefilter)) return;
    T r = pair_r(r2);
    T q = r * P.i_h;
    if (!((double)q < 2.0)) return;
    if (!contact()) return;
    T dwdr = kernel_f(P.kgrad, q);
    V3<T> gker = dr * dwdr;
    if (r < d_ij && r > T(0)) {
      const V4<T> na4 = S.cny[j];
      const V3<T> n_ad{na4.x, na4.y, na4.z};
      const V3<T> n_mat = dr / r;
      d_ij = r;
      cv.y = f_abs(dot(dr, n_ad));
      cv.w = (T)S.codes[c][j].x;
      const V4<T> vj = vel_of();
      vz = V4<T>{vj.x, vj.y, vj.z, T(0)};
      const T cos_c = T(0.866f);
      const T cos_n = f_abs(dot(n_mat, n_ad));
      if (cos_n < cos_c) ny = V4<T>{n_mat.x, n_mat.y, n_mat.z, T(0)};
      else ny = V4<T>{n_ad.x, n_ad.y, n_ad.z, T(0)};
    }
    cv.x += f_abs((ny.x * gker.x + ny.y * gker.y + ny.z * gker.z) * P.vol_def);
  };
  // The candidate lists, current once the search has built, updated or kept them
  // (list_ok), hold every boundary particle within 2h of i in the scan's order (per cell
  // offset, the boundary range first, ascending index): walking their boundary entries
  // visits the same candidates that pass the q < 2 test, in the same order, without the
  // boundary cells' full ranges.  The boundary neighbour records (written by the Adami
  // kernel earlier in the section) carry j's position, velocity and contact flag in one
  // 64-byte line; entries are read four at a time and their records together, so a
  // near-wall thread waits for two loads per four entries instead of a chain of loads
  // per entry.
  const int kept = (S.nbg[0] && P.keep_lists && dyn->list_ok) ? S.nbg_cnt[dyn->lbuf][t] : -1;
  if (kept >= 0) {
    const Rec<T>* __restrict__ rec = S.rec;
    const unsigned* __restrict__ lst = S.nbg[dyn->lbuf] + t;
    const size_t stride = (size_t)S.nbg_stride;
    constexpr unsigned kNone = 0x7ffffffu;  // index of no particle (np < 2^27)
    auto entries = [&](int e0, unsigned* ent) {
#pragma unroll
      for (int k = 0; k < 4; ++k) ent[k] = e0 + k < kept ? __ldcs(lst + (size_t)(e0 + k) * stride) : kNone;
    };
    unsigned ent[4], nxt[4];
    entries(0, ent);
    for (int e0 = 0; e0 < kept; e0 += 4) {
      NbVals<T> nb[4];
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if ((int)(ent[k] & kNone) < P.npb) nb[k] = load_nb(rec, (int)(ent[k] & kNone));
      entries(e0 + 4, nxt);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int j = (int)(ent[k] & kNone);
        if (j >= P.npb) continue;
        const NbVals<T>& b = nb[k];
        visit(j, off_of((int)(ent[k] >> 27)), V3<T>{b.p.x, b.p.y, b.p.z}, [&] { return b.a.y < T(0); },
              [&] { return b.vr; });
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) ent[k] = nxt[k];
    }
  } else {
    for (int oc = 0; oc < 27; ++oc) {
      const I3 off = off_of(oc);
      const I3 cj{celli.x + off.x, celli.y + off.y, celli.z + off.z};
      if (!in_grid(P, cj)) continue;
      const int2 rg = S.range[key_of(P, cj)];
      for (int j = rg.x; j < rg.y; ++j)
        visit(j, off, ld3(pos, j), [&] { return S.codes[c][j].x >= 10; }, [&] { return S.vel[c][j]; });
    }
  }
  S.cv[cpar][i] = cv;
  S.cny[i] = ny;
  S.cvz[i] = vz;
  if (dyn->rec_stale)
    write_rec(P, S.rec, i, S.pos[c][i], S.vel[c][i], ld6(S.str_a[c], S.str_b[c], i), S.idm[c][i].y,
              S.codes[c][i].x >= 10);
}

// ---------------------------------------------------------------------------------
// Particle interaction (src/particle_interaction.cu:26-297).
//
// One thread per material particle.  Phase 1 scans the 27 neighbour cells in the
// reference's order (cz, cy, cx; boundary range then material range; ascending j)
// and appends every candidate passing a conservative distance test to a per-thread
// list in shared memory (column per thread: conflict-free).  Phase 2 walks the list
// in order and evaluates the exact q < 2 test and the pair terms, so every sum is
// accumulated in the reference's order while the expensive pair arithmetic runs with
// the warp converged.  A list that fills up is flushed and the rest of the scan is
// evaluated directly, still in order.
// ---------------------------------------------------------------------------------
template <class T> struct Acc {
  T accden;
  V3<T> s, av, as;
  F9<T> gv;
};

template <class T> struct IState {
  V3<T> pos, vel;
  T rho, ri;
  S6<T> sor;
  int shift;
};


// One pair (i, j) of cuParticleInteractionMaterialLoopSolution
// (src/particle_interaction.cu:29-114), given dr = (pos_i - pos_j) - offset * 2h.
// Strict: the reference's expressions, every operation separately rounded (the CPU
// restatement's order).  Default: the same terms in fewer instructions -- r from the
// hardware reciprocal square root, the velocity-gradient products with the neighbour
// volume folded into the kernel gradient, one approximate division in the artificial
// viscosity -- a few units in the last place from the reference's roundings.
template <bool Strict, class T> RWD void pair_eval(const Params<T>& P, const IState<T>& I, const V3<T> dr,
                                                   const NbVals<T>& nb, Acc<T>& A) {
  using F = Fp<Strict>;
  const T r2 = pair_r2(dr.x, dr.y, dr.z);
  T r;
  if constexpr (Strict) r = pair_r(r2);
  else r = r2 > T(0) ? r2 * f_rsqrt(r2) : T(0);
  T q = F::mul(r, P.i_h);
  if (!(q < T(2.0f))) return;
  const T t = T(2.0f) - q;
  T dwdr = F::mul(F::mul(F::mul(P.kgrad, t), t), t);
  const V3<T> gker{F::mul(dr.x, dwdr), F::mul(dr.y, dwdr), F::mul(dr.z, dwdr)};
  const T rho_j = nb.vr.w, mass_j = nb.a.x, vol_j = f_abs(nb.a.y);
  const bool contact_j = nb.a.y < T(0);
  V3<T> dvel{I.vel.x - nb.vr.x, I.vel.y - nb.vr.y, I.vel.z - nb.vr.z};
  if (contact_j && I.shift == 1) dvel = V3<T>{T(0), T(0), T(0)};
  // grad_vel -= (dvel (x) gker) * vol_j;  accden += rho_i (dvel . gker) vol_j
  if constexpr (Strict) {
    A.gv.xx = F::msub(F::mul(dvel.x, gker.x), vol_j, A.gv.xx);
    A.gv.xy = F::msub(F::mul(dvel.x, gker.y), vol_j, A.gv.xy);
    A.gv.xz = F::msub(F::mul(dvel.x, gker.z), vol_j, A.gv.xz);
    A.gv.yx = F::msub(F::mul(dvel.y, gker.x), vol_j, A.gv.yx);
    A.gv.yy = F::msub(F::mul(dvel.y, gker.y), vol_j, A.gv.yy);
    A.gv.yz = F::msub(F::mul(dvel.y, gker.z), vol_j, A.gv.yz);
    A.gv.zx = F::msub(F::mul(dvel.z, gker.x), vol_j, A.gv.zx);
    A.gv.zy = F::msub(F::mul(dvel.z, gker.y), vol_j, A.gv.zy);
    A.gv.zz = F::msub(F::mul(dvel.z, gker.z), vol_j, A.gv.zz);
    if (contact_j) return;
    const T dvg = F::dot3(dvel.x, dvel.y, dvel.z, gker.x, gker.y, gker.z);
    A.accden = F::mad(F::mul(I.rho, dvg), vol_j, A.accden);
  } else {
    const V3<T> gkv{F::mul(gker.x, vol_j), F::mul(gker.y, vol_j), F::mul(gker.z, vol_j)};
    A.gv.xx = f_fma(-dvel.x, gkv.x, A.gv.xx);
    A.gv.xy = f_fma(-dvel.x, gkv.y, A.gv.xy);
    A.gv.xz = f_fma(-dvel.x, gkv.z, A.gv.xz);
    A.gv.yx = f_fma(-dvel.y, gkv.x, A.gv.yx);
    A.gv.yy = f_fma(-dvel.y, gkv.y, A.gv.yy);
    A.gv.yz = f_fma(-dvel.y, gkv.z, A.gv.yz);
    A.gv.zx = f_fma(-dvel.z, gkv.x, A.gv.zx);
    A.gv.zy = f_fma(-dvel.z, gkv.y, A.gv.zy);
    A.gv.zz = f_fma(-dvel.z, gkv.z, A.gv.zz);
    if (contact_j) return;
    A.accden = f_fma(I.rho, F::dot3(dvel.x, dvel.y, dvel.z, gkv.x, gkv.y, gkv.z), A.accden);
  }
  const S6<T> st{I.sor.xx + nb.a.z, I.sor.yy + nb.a.w, I.sor.zz + nb.b.x,
                 I.sor.xy + nb.b.y, I.sor.xz + nb.b.z, I.sor.yz + nb.b.w};
  const T fx = F::dot3(st.xx, st.xy, st.xz, gker.x, gker.y, gker.z);
  const T fy = F::dot3(st.xy, st.yy, st.yz, gker.x, gker.y, gker.z);
  const T fz = F::dot3(st.xz, st.yz, st.zz, gker.x, gker.y, gker.z);
  A.s.x = F::mad(fx, mass_j, A.s.x);
  A.s.y = F::mad(fy, mass_j, A.s.y);
  A.s.z = F::mad(fz, mass_j, A.s.z);
  if (P.viscosity_type == 1) {
    T artv = T(0.0f);
    const T visc = F::dot3(dvel.x, dvel.y, dvel.z, dr.x, dr.y, dr.z);
    if (visc < T(0.0f)) {
      if constexpr (Strict) {
        const T phi = F::mul(P.h, visc) / F::mad(r, r, P.eta);
        artv = F::mul(F::mul(P.alpha_m, P.cs_m), phi) / F::mul(T(0.5f), I.rho + rho_j);
      } else {  // the same quotient with one approximate division
        artv = f_fastdiv(F::mul(P.visc_k, visc), F::mul(r2 + P.eta, F::mul(T(0.5f), I.rho + rho_j)));
      }
    }
    const T m = F::mul(mass_j, artv);
    A.av.x = F::mad(gker.x, m, A.av.x);
    A.av.y = F::mad(gker.y, m, A.av.y);
    A.av.z = F::mad(gker.z, m, A.av.z);
  }
  if (P.art_coef != T(0.f)) {
    T rj = nb.a.z + nb.a.w + nb.b.x;  // artificial-stress term of j (src/particle_interaction.cu:102-104)
    if (rj > T(0.0f)) rj = F::mul(rj, P.art_coef);
    else rj = T(0.0f);
    T artp = I.ri + rj;
    if (artp > T(0.0f)) {  // W itself is only needed here (a double expression, as GetKernel)
      const T ker = kernel_w(P.knorm, q);
      artp = F::mul(artp, f_pow(ker / P.kernel_dr, P.kernel_zero / P.kernel_dr));
      const T m = F::mul(mass_j, artp);
      A.as.x = F::msub(gker.x, m, A.as.x);
      A.as.y = F::msub(gker.y, m, A.as.y);
      A.as.z = F::msub(gker.z, m, A.as.z);
    }
  }
}

template <bool Strict, class T> RWD void pair_term(const Params<T>& P, const IState<T>& I, const V3<T> dr,
                                                   const Rec<T>* __restrict__ rec, int j, Acc<T>& A) {
  pair_eval<Strict>(P, I, dr, load_nb(rec, j), A);
}

// Particle i's own state at the start of cuParticleInteractionMaterial
// (src/particle_interaction.cu:264-277).
template <bool Strict, class T> RWD void ix_begin(const Params<T>& P, const DevState<T>& S, int c, int i,
                                                  const V4<T>& cv_i, IState<T>& I, Acc<T>& A) {
  using F = Fp<Strict>;
  I.pos = ld3(S.pos[c], i);
  const V4<T> vr_i = S.vel[c][i];
  I.vel = xyz(vr_i);
  I.rho = vr_i.w;
  I.sor = ld6(S.str_a[c], S.str_b[c], i) / F::mul(vr_i.w, vr_i.w);
  I.ri = T(0.0f);
  if (P.art_coef != T(0.f)) {
    I.ri = trace(I.sor);
    if (I.ri > T(0.0f)) I.ri = F::mul(I.ri, P.art_coef);
    else I.ri = T(0.0f);
  }
  I.shift = (int)cv_i.z;
  A.accden = T(0.f);
  A.s = A.av = A.as = V3<T>{T(0), T(0), T(0)};
  A.gv = F9<T>{T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0)};
}


// Exact float of a small integer (|v| < 2^22) without a conversion instruction.
template <class T> RWD T small_float(int v) {
  if constexpr (sizeof(T) == 4) return __int_as_float(0x4B400000 + v) - 12582912.0f;
  else return (T)v;
}

// Evaluates the listed candidates of particle i (entry k at my[k * stride]: index j |
// cell offset << 27) in list order.  The cell offset is decoded arithmetically (no
// table lookup, which would compete with the record gathers for the L1 data stage).
template <bool Strict, class T, bool Kept = false>
RWD void ix_list_eval(const Params<T>& P, const DevState<T>& S, int c, const IState<T>& I, const unsigned* my,
                      int stride, int cnt, Acc<T>& A) {
  const Rec<T>* __restrict__ rec = S.rec;
  if (cnt <= 0) return;
  // Kept lists (global memory) are read once per interaction: streaming loads, so they
  // do not push the neighbour records out of L2.
  auto entry = [&](int k) -> unsigned {
    if constexpr (Kept) return __ldcs(my + k);
    else return my[k];
  };
  // Entries are read two ahead and records one ahead, so a record's index is in hand
  // when its load is issued.
  unsigned ent = entry(0);
  unsigned ent1 = cnt > 1 ? entry(stride) : 0u;
  int oc = (int)(ent >> 27);
  NbVals<T> nb = load_nb(rec, (int)(ent & 0x7ffffffu));
#pragma unroll 2  // alternating record registers instead of copying the prefetched one
  for (int e = 0; e < cnt; ++e) {
    const NbVals<T> cur = nb;
    const int occ = oc;
    if (e + 1 < cnt) {
      oc = (int)(ent1 >> 27);
      nb = load_nb(rec, (int)(ent1 & 0x7ffffffu));
      if (e + 2 < cnt) ent1 = entry((e + 2) * stride);
    }
    // cell offset digits of occ = dx + 3 dy + 9 dz (each 0..2), without a table
    const int dz = (occ * 57) >> 9;
    const int rr = occ - 9 * dz;
    const int dy = (rr * 11) >> 5;
    const int dx = rr - 3 * dy;
    const T th = P.two_h;
    // (pos_i - p_j) - (d - 1) 2h with one rounding after the exact product: the same
    // value as subtracting the tabulated offset
    pair_eval<Strict>(P, I, V3<T>{f_fma(small_float<T>(1 - dx), th, I.pos.x - cur.p.x),
                                  f_fma(small_float<T>(1 - dy), th, I.pos.y - cur.p.y),
                                  f_fma(small_float<T>(1 - dz), th, I.pos.z - cur.p.z)}, cur, A);
  }
}

// Pair sums of particle i straight from global memory: phase 1 lists candidates in
// shared memory (my[k * stride]), phase 2 evaluates them in order.  A list that fills
// up is evaluated and emptied, and the scan resumes (order preserved).
template <bool Strict, class T> RWD void ix_sums_global(const Params<T>& P, const DevState<T>& S, int c, const I3 celli,
                                                        const IState<T>& I, unsigned* my, int stride, int cap,
                                                        Acc<T>& A) {
  const V4<T>* __restrict__ pos = S.pos[c];
  const T th = P.two_h;
  const T r2max = P.r2_prefilter;
  int cnt = 0;
  for (int oc = 0; oc < 27; ++oc) {
    const I3 off = off_of(oc);
    const I3 cj{celli.x + off.x, celli.y + off.y, celli.z + off.z};
    if (!in_grid(P, cj)) continue;
    const int k = key_of(P, cj);
    const V3<T> pmo = I.pos - mulI(off, th);  // conservative pre-test only
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      const int2 rg = S.range[pass ? k + P.ncell_material : k];
#pragma unroll 4
      for (int j = rg.x; j < rg.y; ++j) {
        const V4<T> pj = pos[j];
        const T dx = pmo.x - pj.x, dy = pmo.y - pj.y, dz = pmo.z - pj.z;
        if (dx * dx + dy * dy + dz * dz < r2max) {
          if (cnt == cap) {
            ix_list_eval<Strict>(P, S, c, I, my, stride, cnt, A);
            cnt = 0;
          }
          my[cnt * stride] = (unsigned)j | ((unsigned)oc << 27);
          ++cnt;
        }
      }
    }
  }
  ix_list_eval<Strict>(P, S, c, I, my, stride, cnt, A);
}

// Second pass of a particle within 2h of a periodic plane, over the neighbours of its
// periodic image (cuParticleInteractionMaterialLoopPeriod,
// src/particle_interaction.cu:243-257): same order, evaluated directly (few particles).
template <bool Strict, class T> RWD void ix_period(const Params<T>& P, const DevState<T>& S, int c, int i,
                                                   const I3 celli, IState<T>& I, Acc<T>& A) {
  I3 cpb;
  V3<T> ppb;
  if (!period_image(P, celli, I.pos, false, cpb, ppb)) return;
  const V4<T>* __restrict__ pos = S.pos[c];
  const V3<T> keep = I.pos;
  I.pos = ppb;
  for (int oc = 0; oc < 27; ++oc) {
    const I3 off = off_of(oc);
    const I3 cj{cpb.x + off.x, cpb.y + off.y, cpb.z + off.z};
    if (!in_grid(P, cj)) continue;
    const int k = key_of(P, cj);
    const V3<T> o = mulI(off, P.two_h);
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      const int2 rg = S.range[pass ? k + P.ncell_material : k];
#pragma unroll 1
      for (int j = rg.x; j < rg.y; ++j) {
        const V4<T> pj = pos[j];
        pair_term<Strict>(P, I, I.pos - V3<T>{pj.x, pj.y, pj.z} - o, S.rec, j, A);
      }
    }
  }
  I.pos = keep;
}

// End of cuParticleInteractionMaterial: provisional velocity, wall contact
// (cuParticleInteractionMaterialLoopContact, src/particle_interaction.cu:142-241) and
// the stage outputs (src/particle_interaction.cu:284-295).
template <bool Strict, class T> RWD void ix_finish(const Params<T>& P, const DevState<T>& S, int c, int cpar, int i,
                                                   const I3 celli, const IState<T>& I, const Acc<T>& A, V4<T> cv) {
  using F = Fp<Strict>;
  const V4<T>* __restrict__ cv_in = S.cv[cpar];
  const V4<T>* __restrict__ cf_in = S.cf[cpar];
  const V3<T> g{P.gravity[0], P.gravity[1], P.gravity[2]};
  const V3<T> damp{F::mul(I.vel.x, P.damping), F::mul(I.vel.y, P.damping), F::mul(I.vel.z, P.damping)};
  const V3<T> acc0{A.s.x + A.av.x + A.as.x - damp.x + g.x, A.s.y + A.av.y + A.as.y - damp.y + g.y,
                   A.s.z + A.av.z + A.as.z - damp.z + g.z};
  const V4<T> vr_new{F::mad(acc0.x, P.dt, I.vel.x), F::mad(acc0.y, P.dt, I.vel.y), F::mad(acc0.z, P.dt, I.vel.z),
                     F::mad(A.accden, P.dt, I.rho)};
  V3<T> acc_st{T(0.0f), T(0.0f), T(0.0f)};
  V4<T> fo = cf_in[i];
  const V4<T> ny = S.cny[i];
  const V4<T> vz = S.cvz[i];
  const T mass_i = S.idm[c][i].y;
  const T mrate = T(2.0f) / (T(2.0f) + T(0.0f));
  const V3<T> dv{F::mul(vz.x - vr_new.x, mrate), F::mul(vz.y - vr_new.y, mrate), F::mul(vz.z - vr_new.z, mrate)};
  const T dvn_s = F::dot3(dv.x, dv.y, dv.z, ny.x, ny.y, ny.z);
  if (cv.y <= F::mul(P.h, T(2)) && dvn_s > T(0)) {
    const V4<T>* __restrict__ pos = S.pos[c];
    const T fcoef = P.wall_fric;
    const V3<T> dvn{F::mul(ny.x, dvn_s), F::mul(ny.y, dvn_s), F::mul(ny.z, dvn_s)};
    const V3<T> fn{F::mul(dvn.x, mass_i) / P.dt, F::mul(dvn.y, mass_i) / P.dt, F::mul(dvn.z, mass_i) / P.dt};
    const V3<T> dvt{dv.x - dvn.x, dv.y - dvn.y, dv.z - dvn.z};
    V3<T> ft{F::mul(dvt.x, mass_i) / P.dt, F::mul(dvt.y, mass_i) / P.dt, F::mul(dvt.z, mass_i) / P.dt};
    const T afn = f_sqrt(F::dot3(fn.x, fn.y, fn.z, fn.x, fn.y, fn.z));
    const T aft = f_sqrt(F::dot3(ft.x, ft.y, ft.z, ft.x, ft.y, ft.z));
    const T cap = F::mul(fcoef, afn);
    if (aft > cap) {
      const T ratio = cap / aft;
      ft = V3<T>{F::mul(ft.x, ratio), F::mul(ft.y, ratio), F::mul(ft.z, ratio)};
      cv.z = T(1);
    } else {
      cv.z = T(0);
    }
    V3<T> fric{ft.x + fn.x, ft.y + fn.y, ft.z + fn.z};
    if (cv.y > F::mul(P.dr, T(1.0f))) {
      int count = 0;
      const T h2 = F::mul(T(2.0f), P.h);
      const V3<T> pabs_i{F::mad((T)celli.x, h2, I.pos.x), F::mad((T)celli.y, h2, I.pos.y),
                         F::mad((T)celli.z, h2, I.pos.z)};
      const T ylim = F::mul(P.dr, T(1.0001f));
      const T half_dr = P.dr / T(2);
      for (int oc = 0; oc < 27; ++oc) {
        const I3 off = off_of(oc);
        const I3 cj{celli.x + off.x, celli.y + off.y, celli.z + off.z};
        if (!in_grid(P, cj)) continue;
        const int2 rg = S.range[key_of(P, cj) + P.ncell_material];
        for (int j = rg.x; j < rg.y; ++j) {
          const V4<T> cvj = cv_in[j];
          if (cvj.y <= ylim) {
            const V4<T> pj = pos[j];
            const int4 cpj = S.cellpos[c][j];
            const V3<T> pabs_j{F::mad((T)cpj.x, h2, pj.x), F::mad((T)cpj.y, h2, pj.y), F::mad((T)cpj.z, h2, pj.z)};
            const V3<T> dc{pabs_i.x - pabs_j.x, pabs_i.y - pabs_j.y, pabs_i.z - pabs_j.z};
            const T rcol = f_abs(F::dot3(dc.x, dc.y, dc.z, ny.z, ny.y, ny.x));
            const T cvx_j0 = (j == i) ? cv.x : cvj.x;
            if (rcol <= half_dr && cvx_j0 != T(0)) {
              if (cv.x > cvx_j0) cv.x = cvx_j0;
              const T cvx_j = (j == i) ? cv.x : cvj.x;
              const V4<T> fj = cf_in[j];
              fric.x = F::mul(fj.x, cv.x) / cvx_j;
              fric.y = F::mul(fj.y, cv.x) / cvx_j;
              fric.z = F::mul(fj.z, cv.x) / cvx_j;
              count++;
            }
          }
        }
      }
      if (count == 0) fric = V3<T>{F::mul(fric.x, T(0)), F::mul(fric.y, T(0)), F::mul(fric.z, T(0))};
    }
    fo = V4<T>{fric.x, fric.y, fric.z, T(0)};
    const T im = T(1) / mass_i;
    acc_st = V3<T>{F::mul(fric.x, im), F::mul(fric.y, im), F::mul(fric.z, im)};
  }
  S.cv[cpar ^ 1][i] = cv;
  S.cf[cpar ^ 1][i] = fo;
  S.accad[i] = V4<T>{A.s.x + A.av.x + A.as.x + acc_st.x - damp.x + g.x, A.s.y + A.av.y + A.as.y + acc_st.y - damp.y + g.y,
                     A.s.z + A.av.z + A.as.z + acc_st.z - damp.z + g.z, A.accden};
  st6(S.ace_a, S.ace_b, i, full2sym(A.gv));
  S.spin[i] = v4(skewpart(A.gv), T(0.f));
}

// Candidate lists of the live soil particles: the 27 cells in the scan's order (cz,
// cy, cx; boundary range before material range; ascending j), every candidate within
// the list radius, written column-major to HBM.  Mode 0 builds every soil list here and
// starts the displacement bounds (the Adami kernel builds the boundary lists).  Mode 2
// (list update) queues the lists of particles next to a marked cell, soil and boundary
// rows alike, for k_rebuild_lists, and carries the others through the section's
// permutation; the bounds run on from the last full build (a list built since then
// moved no more than its particle's bound).  A list longer than IX_CAP is marked -1 and
// counted (n_spill): the scan launch then takes that particle.  Light (no pair
// arithmetic, no shared-memory list), so it runs at full occupancy; the walk kernel
// then evaluates the lists with the same pairs in the same order as a scan.  One thread
// per particle, boundary rows first, so that in an update the Adami kernel (many
// registers, few warps per SM) only walks lists.
template <class T> __global__ void __launch_bounds__(256) k_build_lists(const Params<T> P, DevState<T> S, Dyn<T>* dyn) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const int mode = dyn->ix_mode;
  if (!S.nbg[0] || !P.keep_lists || mode == 1) return;
  if (row == 0 && mode == 0) {
    dyn->list_ok = 1;
    dyn->list_kill = dyn->build_kill;
  }
  const int lb = dyn->lbuf;
  const int c = dyn->cur_main;
  // queues a row whose list k_rebuild_lists rebuilds (one warp per list), so that the
  // few lists an update rebuilds do not each wait on one thread's 27-cell scan
  auto enqueue = [&] {
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&dyn->n_queue, __popc(m));
    base = __shfl_sync(m, base, leader);
    S.queue[base + __popc(m & ((1u << lane) - 1u))] = row;
  };
  if (row < P.npb) {
    if (mode == 2 && S.nbb[0]) {
      const int4 cb = S.cellpos[c][row];
      if (near_marked(P, S, dyn, I3{cb.x, cb.y, cb.z})) enqueue();
      else if (dyn->need_sort)
        carry_list(S.nbb[lb ^ 1], S.nbb_cnt[lb ^ 1], S.sperm[row], S.nbb[lb], S.nbb_cnt[lb], row, P.npb, S.inv);
    }
    return;
  }
  const int t = row - P.npb;
  if (t >= dyn->npm) return;
  const int i = row;
  const int4 cp = S.cellpos[c][i];
  const I3 celli{cp.x, cp.y, cp.z};
  const size_t stride = (size_t)S.nbg_stride;
  if (mode == 2) {
    if (!near_marked(P, S, dyn, celli)) {
      if (dyn->need_sort)
        carry_list(S.nbg[lb ^ 1], S.nbg_cnt[lb ^ 1], S.sperm[i] - P.npb, S.nbg[lb], S.nbg_cnt[lb], t, stride, S.inv);
      return;
    }
    enqueue();  // next to a marked cell
    return;
  }
  S.dacc[lb][i] = 0.0f;
  const V4<T>* __restrict__ pos = S.pos[c];
  const V3<T> pos_i = ld3(pos, i);
  const T th = P.two_h;
  unsigned* __restrict__ out = S.nbg[lb] + t;
  int cnt = 0;
  for (int oc = 0; oc < 27; ++oc) {
    const I3 off = off_of(oc);
    const I3 cj{celli.x + off.x, celli.y + off.y, celli.z + off.z};
    if (!in_grid(P, cj)) continue;
    const int k = key_of(P, cj);
    const V3<T> pmo = pos_i - mulI(off, th);  // conservative pre-test only
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      const int2 rg = S.range[pass ? k + P.ncell_material : k];
#pragma unroll 4
      for (int j = rg.x; j < rg.y; ++j) {
        const V4<T> pj = pos[j];
        const T dx = pmo.x - pj.x, dy = pmo.y - pj.y, dz = pmo.z - pj.z;
        if (dx * dx + dy * dy + dz * dz < P.r2_list) {
          if (cnt < IX_CAP) __stcs(out + (size_t)cnt * stride, (unsigned)j | ((unsigned)oc << 27));
          ++cnt;
        }
      }
    }
  }
  if (cnt > IX_CAP) {
    S.nbg_cnt[lb][t] = -1;
    atomicAdd(&dyn->n_spill, 1);
  } else {
    S.nbg_cnt[lb][t] = cnt;
  }
}

// The lists queued by a list update (soil rows' interaction lists and boundary rows'
// Adami lists), one warp per list: the 27 cells x 2 ranges are 54 segments of
// candidates, flattened in the scan's order; the warp tests 32 consecutive candidates
// at a time and appends the hits in order (ballot + prefix count), so the list holds
// the pairs a full build lists, in the same order.  The displacement bounds run on.
template <class T> __global__ void __launch_bounds__(256) k_rebuild_lists(const Params<T> P, DevState<T> S, Dyn<T>* dyn) {
  constexpr int kSeg = 54, kWarps = 256 / 32;
  __shared__ int seg_beg[kWarps][kSeg + 1];  // first flattened candidate of each segment
  __shared__ int seg_j0[kWarps][kSeg];       // first particle index of each segment
  if (!S.nbg[0] || !P.keep_lists || dyn->ix_mode != 2) return;
  const int nq = dyn->n_queue;
  if (blockIdx.x == 0 && threadIdx.x == 0) dyn->n_rebuilt += nq;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lb = dyn->lbuf, c = dyn->cur_main;
  const V4<T>* __restrict__ pos = S.pos[c];
  const T th = P.two_h;
  int* beg = seg_beg[warp];
  int* j0 = seg_j0[warp];
  for (int q = blockIdx.x * kWarps + warp; q < nq; q += gridDim.x * kWarps) {
    // a soil row's list, or a boundary row's Adami list (without the boundary ranges
    // unless the particle belongs to a contact wall, as the Adami scan keeps it)
    const int i = S.queue[q];
    const bool bnd = i < P.npb;
    const bool with_bnd_range = !bnd || S.codes[c][i].x >= 10;
    const int4 cp = S.cellpos[c][i];
    const I3 celli{cp.x, cp.y, cp.z};
    const V3<T> pos_i = ld3(pos, i);
    int size[2], first[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int sg = lane + 32 * h;
      size[h] = 0;
      first[h] = 0;
      if (sg < kSeg && ((sg & 1) || with_bnd_range)) {
        const I3 off = off_of(sg >> 1);
        const I3 cj{celli.x + off.x, celli.y + off.y, celli.z + off.z};
        if (in_grid(P, cj)) {
          const int k = key_of(P, cj);
          const int2 rg = S.range[(sg & 1) ? k + P.ncell_material : k];
          size[h] = rg.y - rg.x;
          first[h] = rg.x;
        }
      }
    }
    int inc0 = size[0], inc1 = size[1];  // inclusive prefix sums over the lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int a = __shfl_up_sync(0xffffffffu, inc0, d), b = __shfl_up_sync(0xffffffffu, inc1, d);
      if (lane >= d) {
        inc0 += a;
        inc1 += b;
      }
    }
    const int tot0 = __shfl_sync(0xffffffffu, inc0, 31);
    const int total = tot0 + __shfl_sync(0xffffffffu, inc1, 31);
    beg[lane] = inc0 - size[0];
    j0[lane] = first[0];
    if (lane + 32 < kSeg) {
      beg[lane + 32] = tot0 + inc1 - size[1];
      j0[lane + 32] = first[1];
    }
    if (lane == 0) beg[kSeg] = total;
    __syncwarp();
    const size_t stride = bnd ? (size_t)P.npb : (size_t)S.nbg_stride;
    unsigned* __restrict__ out = bnd ? S.nbb[lb] + i : S.nbg[lb] + (i - P.npb);
    int* __restrict__ count = bnd ? S.nbb_cnt[lb] + i : S.nbg_cnt[lb] + (i - P.npb);
    int cnt = 0;
    for (int b0 = 0; b0 < total; b0 += 32) {
      const int ci = b0 + lane;
      bool hit = false;
      unsigned ent = 0u;
      if (ci < total) {
        int lo = 0, hi = kSeg;  // the last segment starting at or before ci (it is not empty)
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (beg[mid] <= ci) lo = mid;
          else hi = mid;
        }
        const int j = j0[lo] + (ci - beg[lo]);
        const int oc = lo >> 1;
        const V3<T> pmo = pos_i - mulI(off_of(oc), th);
        const V4<T> pj = pos[j];
        const T dx = pmo.x - pj.x, dy = pmo.y - pj.y, dz = pmo.z - pj.z;
        hit = dx * dx + dy * dy + dz * dz < P.r2_list;
        ent = (unsigned)j | ((unsigned)oc << 27);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (hit) {
        const int e = cnt + __popc(bal & ((1u << lane) - 1u));
        if (e < IX_CAP) __stcs(out + (size_t)e * stride, ent);
      }
      cnt += __popc(bal);
    }
    if (lane == 0) {
      *count = cnt > IX_CAP ? -1 : cnt;  // an overflowed boundary list: Adami scans for it
      if (cnt > IX_CAP && !bnd) atomicAdd(&dyn->n_spill, 1);
    }
    __syncwarp();  // before the next list overwrites the segment table
  }
}

// Interaction, one thread per soil particle, neighbours read from global memory, as
// two launches that split the particles between them:
//  - walk (Walk = true): walks the candidate lists, kept from an earlier section or
//    just built by k_build_lists.  It carries no scan state, so it runs with fewer
//    registers;
//  - scan (Walk = false): scans the 27 cells for the particles without a list (lists
//    off, or a list that overflowed) and carries the contact state of deleted slots.
#ifndef RW_WALK_MIN_BLOCKS
#define RW_WALK_MIN_BLOCKS 0  // resident blocks per SM the walk kernel's register budget aims at (0: none)
#endif
template <class T, bool Strict, bool Walk>
__global__ void __launch_bounds__(Walk ? IX_WALK_MAX_THREADS : IX_THREADS, Walk ? RW_WALK_MIN_BLOCKS : 0)
    k_interaction(const Params<T> P, DevState<T> S, const Dyn<T>* dyn, int cpar) {
  extern __shared__ unsigned nbl[];  // IX_CAP x blockDim, column per thread (scan only)
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (!Walk && t == 0) const_cast<Dyn<T>*>(dyn)->rec_stale = 0;  // the corner search has refreshed the records
  const int total = P.np - P.npb;
  if (t >= total) return;
  const int i = P.npb + t;
  const int npm = dyn->npm;
  const bool keep = S.nbg[0] && P.keep_lists;
  if (Walk) {
    if (!keep || t >= npm) return;
  } else if (t >= npm) {  // deleted slots keep their contact state
    S.cv[cpar ^ 1][i] = S.cv[cpar][i];
    S.cf[cpar ^ 1][i] = S.cf[cpar][i];
    return;
  }
  const int lb = dyn->lbuf;
  const int kept = keep ? S.nbg_cnt[lb][t] : -1;
  if (Walk != (kept >= 0)) return;  // the other launch takes this particle
  const int c = dyn->cur_main;
  const int4 cp = S.cellpos[c][i];
  const I3 celli{cp.x, cp.y, cp.z};
  const V4<T> cv = S.cv[cpar][i];
  IState<T> I;
  Acc<T> A;
  ix_begin<Strict>(P, S, c, i, cv, I, A);
  if (Walk) ix_list_eval<Strict, T, true>(P, S, c, I, S.nbg[lb] + t, S.nbg_stride, kept, A);
  else ix_sums_global<Strict>(P, S, c, celli, I, nbl + threadIdx.x, blockDim.x, IX_CAP, A);
  if (P.periodbound) ix_period<Strict>(P, S, c, i, celli, I, A);
  ix_finish<Strict>(P, S, c, cpar, i, celli, I, A, cv);
}

// ---------------------------------------------------------------------------------
// Chunked interaction with the neighbour tile staged in shared memory.
//
// The soil particles of one cell column (x, y) are contiguous and ordered by z, so a
// chunk of up to IX2_TB of them needs the 9 columns (x+-1, y+-1) over the z window
// [z_first - 1, z_last + 1], in both layers: 18 contiguous index runs.  The block
// copies those runs' positions into shared memory once; every candidate test of
// phase 1 then reads shared memory.  Lists are filled in warp-synchronous rounds of
// IX2_CAP entries (a round ends for the whole warp when any lane's list is full) and
// evaluated in order with the next neighbour record prefetched, so each particle's
// sums keep the reference's order exactly.  A chunk whose tile does not fit
// (more than IX2_SMAX particles or IX2_NZW cells in z) runs the global path.
// ---------------------------------------------------------------------------------
constexpr int IX2_TB = 128, IX2_SMAX = 2048, IX2_NZW = 30, IX2_CAP = 96;

// Run of a staged index: boundary runs are staged before material runs, so the layer
// is k >= base of the first material run; the column comes from the cell offset.
RWD int ix2_seg(int k, int oc, int base9) {
  const I3 off = off_of(oc);
  return (k >= base9 ? 9 : 0) + (off.y + 1) * 3 + (off.x + 1);
}

struct Chunk {
  int first, n, col, pad;
};

template <class T> struct Ix2Smem {
  V4<T> spos[IX2_SMAX];
  int2 tab[18][IX2_NZW];
  int delta[18];   // global index = staged index + delta
  int gbeg[18], glen[18], base[18];
  unsigned short list[IX2_CAP][IX2_TB];  // staged index (11 bits) | cell offset << 11
  int zl, nzw, total, fallback;
};

// Per-column soil runs and chunk counts (the chunk list is rebuilt after each sort).
template <class T> __global__ void k_col_count(const Params<T> P, DevState<T> S) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncol = P.cell_num[0] * P.cell_num[1];
  if (col >= ncol) return;
  const int nz = P.cell_num[2];
  const int base = P.ncell_material + col * nz;
  int beg = -1, end = -1;
  for (int z = 0; z < nz; ++z) {
    const int2 r = S.range[base + z];
    if (r.y > r.x) {
      if (beg < 0) beg = r.x;
      end = r.y;
    }
  }
  const int len = beg < 0 ? 0 : end - beg;
  S.col_beg[col] = beg < 0 ? 0 : beg;
  S.col_len[col] = len;
  S.col_cnt[col] = (len + IX2_TB - 1) / IX2_TB;
}

template <class T> __global__ void __launch_bounds__(1024) k_col_scan(const Params<T> P, DevState<T> S, Dyn<T>* dyn) {
  __shared__ int ws[32];
  const int ncol = P.cell_num[0] * P.cell_num[1];
  const int per = (ncol + 1023) / 1024;
  const int b = threadIdx.x * per, e = min(ncol, b + per);
  int s = 0;
  for (int k = b; k < e; ++k) s += S.col_cnt[k];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = s;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    int v = ws[lane];
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    ws[lane] = v;
  }
  __syncthreads();
  int off = x - s + (w > 0 ? ws[w - 1] : 0);
  for (int k = b; k < e; ++k) {
    const int n = S.col_cnt[k];
    S.col_off[k] = off;
    off += n;
  }
  if (threadIdx.x == 1023) dyn->nchunks = off;
}

template <class T> __global__ void k_col_fill(const Params<T> P, DevState<T> S) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncol = P.cell_num[0] * P.cell_num[1];
  if (col >= ncol) return;
  const int n = S.col_cnt[col];
  if (n == 0) return;
  const int len = S.col_len[col], beg = S.col_beg[col], off = S.col_off[col];
  for (int k = 0; k < n; ++k) {  // n nearly equal chunks
    const int a = beg + (int)((long)len * k / n);
    const int b = beg + (int)((long)len * (k + 1) / n);
    S.chunks[off + k] = Chunk{a, b - a, col, 0};
  }
}

template <class T, bool Strict> __global__ void __launch_bounds__(IX2_TB) k_interaction2(const Params<T> P, DevState<T> S,
                                                                                       const Dyn<T>* dyn, int cpar) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Ix2Smem<T>& sm = *reinterpret_cast<Ix2Smem<T>*>(smraw);
  const int tid = threadIdx.x;
  if (blockIdx.x == 0 && tid == 0) const_cast<Dyn<T>*>(dyn)->rec_stale = 0;  // records refreshed by the corner search
  // Deleted slots keep their contact state (the chunk list covers live particles only).
  {
    const int npm = dyn->npm;
    const int ndel = P.np - P.npb - npm;
    for (int t = blockIdx.x * IX2_TB + tid; t < ndel; t += gridDim.x * IX2_TB) {
      const int i = P.npb + npm + t;
      S.cv[cpar ^ 1][i] = S.cv[cpar][i];
      S.cf[cpar ^ 1][i] = S.cf[cpar][i];
    }
  }
  if ((int)blockIdx.x >= dyn->nchunks) return;
  const Chunk ch = S.chunks[blockIdx.x];
  const int c = dyn->cur_main;
  const int ny = P.cell_num[1], nz = P.cell_num[2];
  const int x = ch.col / ny, y = ch.col % ny;
  if (tid == 0) {
    const int z0 = S.cellpos[c][ch.first].z;
    const int z1 = S.cellpos[c][ch.first + ch.n - 1].z;
    const int zl = max(z0 - 1, 0), zh = min(z1 + 1, nz - 1);
    sm.zl = zl;
    sm.nzw = zh - zl + 1;
  }
  __syncthreads();
  const int zl = sm.zl, nzw = sm.nzw;
  const bool fits_z = nzw <= IX2_NZW;
  if (fits_z) {
    // Cell table (global ranges for now) of the 18 runs.
    for (int idx = tid; idx < 18 * nzw; idx += IX2_TB) {
      const int s = idx / nzw, zi = idx - s * nzw;
      const int lay = s / 9, c9 = s - lay * 9;
      const int xx = x + c9 % 3 - 1, yy = y + c9 / 3 - 1;
      int2 r{0, 0};
      if (xx >= 0 && yy >= 0 && xx < P.cell_num[0] && yy < ny)
        r = S.range[(lay ? P.ncell_material : 0) + xx * ny * nz + yy * nz + zl + zi];
      sm.tab[s][zi] = r;
    }
  }
  __syncthreads();
  if (tid < 18) {
    int gb = 0, ge = 0;
    bool any = false;
    if (fits_z)
      for (int zi = 0; zi < nzw; ++zi) {
        const int2 r = sm.tab[tid][zi];
        if (r.y > r.x) {
          if (!any) gb = r.x;
          ge = r.y;
          any = true;
        }
      }
    sm.gbeg[tid] = gb;
    sm.glen[tid] = any ? ge - gb : 0;
  }
  __syncthreads();
  if (tid == 0) {
    int tot = 0;
    for (int s = 0; s < 18; ++s) {
      sm.base[s] = tot;
      sm.delta[s] = sm.gbeg[s] - tot;
      tot += sm.glen[s];
    }
    sm.total = tot;
    sm.fallback = (!fits_z || tot > IX2_SMAX) ? 1 : 0;
  }
  __syncthreads();
  const bool fallback = sm.fallback != 0;
  if (!fallback) {
    // Staged coordinates for the table; copy the runs' positions.
    for (int idx = tid; idx < 18 * nzw; idx += IX2_TB) {
      const int s = idx / nzw, zi = idx - s * nzw;
      const int2 r = sm.tab[s][zi];
      sm.tab[s][zi] = (r.y > r.x) ? int2{r.x - sm.delta[s], r.y - sm.delta[s]} : int2{0, 0};
    }
    const V4<T>* __restrict__ pos = S.pos[c];
    for (int s = 0; s < 18; ++s) {
      const int n = sm.glen[s], gb = sm.gbeg[s], b = sm.base[s];
      for (int k = tid; k < n; k += IX2_TB) sm.spos[b + k] = pos[gb + k];
    }
  }
  __syncthreads();
  if (tid >= ch.n) return;
  const int i = ch.first + tid;
  const int4 cp = S.cellpos[c][i];
  const I3 celli{cp.x, cp.y, cp.z};
  const V4<T> cv = S.cv[cpar][i];
  IState<T> I;
  Acc<T> A;
  ix_begin<Strict>(P, S, c, i, cv, I, A);
  if (fallback) {
    // Too big for the tile: same arithmetic from global memory, list in the round buffer.
    ix_sums_global<Strict>(P, S, c, celli, I, reinterpret_cast<unsigned*>(&sm.list[0][0]) + tid, IX2_TB,
                           IX2_CAP / 2, A);
    if (P.periodbound) ix_period<Strict>(P, S, c, i, celli, I, A);
    ix_finish<Strict>(P, S, c, cpar, i, celli, I, A, cv);
    return;
  }
  const Rec<T>* __restrict__ rec = S.rec;
  const T th = P.two_h;
  const T r2max = P.r2_prefilter;
  const int zi_i = cp.z - zl;
  const unsigned lanes = __activemask();
  unsigned short* my = &sm.list[0][tid];
  int cnt = 0;
  // Evaluate the listed candidates in order (next neighbour record prefetched).
  auto flush = [&]() {
    if (cnt > 0) {
      int kk = my[0] & 0x7ff, oc = my[0] >> 11;
      NbVals<T> nb = load_nb(rec, kk + sm.delta[ix2_seg(kk, oc, sm.base[9])]);
      for (int e = 0; e < cnt; ++e) {
        const NbVals<T> cur = nb;
        const int kc = kk, occ = oc;
        if (e + 1 < cnt) {
          const unsigned short ent = my[(e + 1) * IX2_TB];
          kk = ent & 0x7ff;
          oc = ent >> 11;
          nb = load_nb(rec, kk + sm.delta[ix2_seg(kk, oc, sm.base[9])]);
        }
        const V3<T> o = mulI(off_of(occ), th);
        const V4<T> pj = sm.spos[kc];
        pair_eval<Strict>(P, I, I.pos - V3<T>{pj.x, pj.y, pj.z} - o, cur, A);
      }
    }
    cnt = 0;
  };
  // Phase 1 over the 54 (cell offset, layer) ranges in the reference's order; a range
  // that could overflow any lane's list first flushes every lane's list.
  for (int oc = 0; oc < 27; ++oc) {
    const I3 off = off_of(oc);
    const int zz = zi_i + off.z;
    const bool zin = zz >= 0 && zz < nzw;
    const V3<T> pmo = I.pos - mulI(off, th);
#pragma unroll 1
    for (int lay = 0; lay < 2; ++lay) {
      int2 r{0, 0};
      if (zin) r = sm.tab[lay * 9 + (off.y + 1) * 3 + (off.x + 1)][zz];
      if (__any_sync(lanes, cnt + (r.y - r.x) > IX2_CAP)) flush();
      for (int k = r.x; k < r.y; ++k) {
        const V4<T> pj = sm.spos[k];
        const T dx = pmo.x - pj.x, dy = pmo.y - pj.y, dz = pmo.z - pj.z;
        if (dx * dx + dy * dy + dz * dz < r2max) {
          if (cnt == IX2_CAP) flush();  // only a cell with more than IX2_CAP particles gets here
          my[cnt * IX2_TB] = (unsigned short)(k | (oc << 11));
          ++cnt;
        }
      }
    }
  }
  flush();
  if (P.periodbound) ix_period<Strict>(P, S, c, i, celli, I, A);
  ix_finish<Strict>(P, S, c, cpar, i, celli, I, A, cv);
}

// ---------------------------------------------------------------------------------
// Predictor (src/predictor_corrector.cu:52-103): saves the step-start state into the
// *_ini buffers (the reference's four D2D copies) and advances material half a step.
// ---------------------------------------------------------------------------------
// Both integrators are held to four 256-thread blocks per SM (64 registers, about
// 100 spilled bytes): they stream about 300 B per particle, and at the two blocks
// their natural 94 registers allow they wait on memory (measured 19% faster at
// three blocks, another 5% at four).
// One row of the predictor.  With the learned closure on, HypoCS rows keep their stress
// here and the closure's pass updates it (and writes their record).
template <class T> RWD void predictor_row(const Params<T>& P, const DevState<T>& S, const Dyn<T>* dyn, int i) {
  if (i >= P.np) return;
  const int c = dyn->cur_main, ci = dyn->cur_ini;
  const int npm = dyn->npm;
  V4<T> ps = S.pos[c][i];
  V4<T> vr = S.vel[c][i];
  S.pos_ini[ci][i] = ps;
  S.vel_ini[ci][i] = vr;
  V4<T> kp{T(0), T(0), T(0), T(0)}, kv{T(0), T(0), T(0), T(0)};
  if (P.mixed) {
    kp = S.cmp_p[c][i];
    kv = S.cmp_v[c][i];
    S.cmp_pi[ci][i] = kp;
    S.cmp_vi[ci][i] = kv;
  }
  if (npm == 0 || i >= P.npb + npm) return;
  S6<T> sg = ld6(S.str_a[c], S.str_b[c], i);
  S6<T> sn = ld6(S.stn_a[c], S.stn_b[c], i);
  st6(S.stri_a[ci], S.stri_b[ci], i, sg);
  st6(S.stni_a[ci], S.stni_b[ci], i, sn);
  if (i < P.npb) return;
  const int4 code = S.codes[c][i];
  if (code.y != 1) return;
  const T mass = S.idm[c][i].y;  // for the neighbour record (read early: the stores below may alias)
  const T hdt = T(0.5f) * P.dt;
  const V4<T> acc = S.accad[i];
  if (P.mixed) {  // compensated half step; the compensation itself is not kept
    kahan_add(vr.x, kv.x, acc.x * hdt);
    kahan_add(vr.y, kv.y, acc.y * hdt);
    kahan_add(vr.z, kv.z, acc.z * hdt);
    kahan_add(vr.w, kv.w, acc.w * hdt);
    kahan_add(ps.x, kp.x, vr.x * hdt);
    kahan_add(ps.y, kp.y, vr.y * hdt);
    kahan_add(ps.z, kp.z, vr.z * hdt);
  } else {
    vr = vr + acc * hdt;
    ps = add3(ps, xyz(vr) * hdt);
  }
  {  // distance since the lists were built, after this half step
    const float a = (float)(f_sqrt(vr.x * vr.x + vr.y * vr.y + vr.z * vr.z) * hdt);
    if (S.dacc[dyn->lbuf][i] + a + P.disp_eps > P.disp_lim) const_cast<Dyn<T>*>(dyn)->list_kill = 1;
  }
  const T* mp = P.model_par[code.w];
  vr.w = f_max(vr.w, mp[kMatSize - 2]);
  vr.w = f_min(vr.w, mp[kMatSize - 1]);
  const S6<T> D = ld6(S.ace_a, S.ace_b, i);
  sn = sn + D * hdt;
  bool yld = false;
  T mcrt = T(0);
  const bool by_closure = P.closure && code.z == RW_MODEL_HYPO_CS;  // the closure pass updates the stress
  const HypoC<T> hc = P.hypo[code.w];
  if (!by_closure) constitutive(code.z, mp, hdt, vr.w, xyz(S.spin[i]), D, sg, yld, mcrt, P.mixed != 0, &hc);
  S.pos[c][i] = ps;
  S.vel[c][i] = vr;
  st6(S.stn_a[c], S.stn_b[c], i, sn);
  st6(S.str_a[c], S.str_b[c], i, sg);
  if (!yld) S.idm[c][i].x = T(100);
  if (!by_closure) write_rec(P, S.rec, i, ps, vr, sg, mass, code.x >= 10);
}

template <class T>
__global__ void __launch_bounds__(256, 4) k_predictor(const Params<T> P, DevState<T> S, const Dyn<T>* dyn) {
  predictor_row(P, S, dyn, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------------
// Corrector (src/predictor_corrector.cu:109-213): rigid walls and material.
// ---------------------------------------------------------------------------------
// Rounding error of s = fl(a + b): exact(a + b) - s (Knuth's TwoSum).
template <class T> RWD T two_sum_err(T a, T b, T s) {
  const T bb = add_rn(s, -a);
  return add_rn(add_rn(a, -add_rn(s, -bb)), add_rn(b, -bb));
}

template <class T> RWD I3 rebin(V4<T>& ps, T th) {
  I3 dc{int(ps.x >= th) - int(ps.x < T(0)), int(ps.y >= th) - int(ps.y < T(0)), int(ps.z >= th) - int(ps.z < T(0))};
  ps = sub3(ps, mulI(dc, th));
  return dc;
}

// Marks a cell whose particles changed (once per generation: the first marker lists it).
template <class T> RWD void mark_cell(const Params<T>& P, const DevState<T>& S, const Dyn<T>* dyn, I3 c) {
  const int key = key_of(P, c);
  const unsigned gen = dyn->mark_gen;
  if (atomicExch(&S.cell_mark[key], gen) != gen) {
    const int k = atomicAdd(&const_cast<Dyn<T>*>(dyn)->n_marks, 1);
    if (k < RW_MARK_CAP) S.marks[k] = key;
  }
}

// Bookkeeping of the kept candidate lists for one particle's full step from cell `from`
// to cell `to`.  Its distance bound grows by the step (plus a rounding allowance) and
// must stay within the skin's share, else every list is rebuilt.  A cell change marks
// both cells (the next list update rebuilds the lists around them); leaving the grid
// (deletion) makes it a full build.
template <class T> RWD void list_account(const Params<T>& P, const DevState<T>& S, const Dyn<T>* dyn, int i, float step,
                                         I3 from, I3 to) {
  float* dacc = S.dacc[dyn->lbuf];
  const float d = dacc[i] + step + P.disp_eps;
  dacc[i] = d;
  Dyn<T>* w = const_cast<Dyn<T>*>(dyn);
  if (from.x != to.x || from.y != to.y || from.z != to.z) {
    w->cells_dirty = 1;
    if (!in_grid(P, from) || !in_grid(P, to)) {
      w->list_kill = 1;
    } else if (P.keep_lists) {
      mark_cell(P, S, dyn, from);
      mark_cell(P, S, dyn, to);
    }
  }
  if (d > P.disp_lim) w->list_kill = 1;
}

// One row of the corrector (moving boundary rows and soil rows); with the learned
// closure on, HypoCS rows keep their stress here, as in predictor_row.
template <class T> RWD void corrector_row(const Params<T>& P, const DevState<T>& S, const Dyn<T>* dyn, int i) {
  const int npm = dyn->npm;
  if (i >= P.npb + npm) return;
  const int c = dyn->cur_main, ci = dyn->cur_ini;
  const int4 code = S.codes[c][i];
  if (code.y != 1) return;
  const T th = P.two_h;
  if (i < P.npb) {
    if (P.n_motion <= 0) return;
    const Motion<T>& mv = dyn->mv[code.w];
    V3<T> vel{mv.trans_vel.x, mv.trans_vel.y, mv.trans_vel.z};
    int4 cp = S.cellpos[c][i];
    if (mv.is_rotat && mv.pattern != RW_PATTERN_CIRCLE) {
      const V3<T> pabs = ld3(S.pos[c], i) + mulI(I3{cp.x, cp.y, cp.z}, th);
      const V3<T> rp{mv.pos_rp.x, mv.pos_rp.y, mv.pos_rp.z};
      const V3<T> w{mv.rotat_vel.x, mv.rotat_vel.y, mv.rotat_vel.z};
      vel = vel + cross(w, pabs - rp);
      const F9<T> R = rodrigues(w * P.dt);
      const int cn = dyn->cur_nrm;
      const V4<T> n4 = S.normal[cn][i];
      const V3<T> n = dotFV(R, xyz(n4));
      S.normal[cn][i] = v4(n, n4.w);
    }
    V4<T> ps = add3(S.pos_ini[ci][i], vel * P.dt);
    const I3 dc = rebin(ps, th);
    S.pos[c][i] = ps;
    S.cellpos[c][i] = int4{cp.x + dc.x, cp.y + dc.y, cp.z + dc.z, cp.w};
    list_account(P, S, dyn, i, (float)(f_sqrt(dot(vel, vel)) * P.dt), I3{cp.x, cp.y, cp.z},
                 I3{cp.x + dc.x, cp.y + dc.y, cp.z + dc.z});
    return;
  }
  const V4<T> vri = S.vel_ini[ci][i];
  V4<T> id = S.idm[c][i];  // read early: the stores below may alias
  V4<T> vr, ps;
  V4<T> kp{T(0), T(0), T(0), T(0)}, kv{T(0), T(0), T(0), T(0)};
  if (P.mixed) {  // compensated full step (position and velocity keep their lost low bits)
    kp = S.cmp_pi[ci][i];
    kv = S.cmp_vi[ci][i];
    const V4<T> acc = S.accad[i];
    vr = vri;
    kahan_add(vr.x, kv.x, acc.x * P.dt);
    kahan_add(vr.y, kv.y, acc.y * P.dt);
    kahan_add(vr.z, kv.z, acc.z * P.dt);
    kahan_add(vr.w, kv.w, acc.w * P.dt);
    ps = S.pos_ini[ci][i];
    const T hdt = T(0.5f) * P.dt;
    kahan_add(ps.x, kp.x, (vr.x + vri.x) * hdt);
    kahan_add(ps.y, kp.y, (vr.y + vri.y) * hdt);
    kahan_add(ps.z, kp.z, (vr.z + vri.z) * hdt);
  } else {
    vr = vri + S.accad[i] * P.dt;
    ps = add3(S.pos_ini[ci][i], xyz(vr + vri) * (T(0.5f) * P.dt));
  }
  const T* mp = P.model_par[code.w];
  vr.w = f_max(vr.w, mp[kMatSize - 2]);
  vr.w = f_min(vr.w, mp[kMatSize - 1]);
  const V4<T> ps0 = ps;
  const I3 dc = rebin(ps, th);
  if (P.mixed) {  // re-binning adds -+2h: fold its rounding error into the compensation
    const V3<T> sh = mulI(dc, th);
    kp.x = add_rn(kp.x, -two_sum_err(ps0.x, -sh.x, ps.x));
    kp.y = add_rn(kp.y, -two_sum_err(ps0.y, -sh.y, ps.y));
    kp.z = add_rn(kp.z, -two_sum_err(ps0.z, -sh.z, ps.z));
    S.cmp_p[c][i] = kp;
    S.cmp_v[c][i] = kv;
  }
  const int4 cp0 = S.cellpos[c][i];
  int4 cp = int4{cp0.x + dc.x, cp0.y + dc.y, cp0.z + dc.z, cp0.w};
  if (P.periodbound) period_wrap(P, cp, ps);
  {
    const V3<T> inc = xyz(vr + vri) * (T(0.5f) * P.dt);
    list_account(P, S, dyn, i, (float)f_sqrt(dot(inc, inc)), I3{cp0.x, cp0.y, cp0.z}, I3{cp.x, cp.y, cp.z});
  }
  S6<T> sg = ld6(S.stri_a[ci], S.stri_b[ci], i);
  const S6<T> D = ld6(S.ace_a, S.ace_b, i);
  const S6<T> sn = ld6(S.stni_a[ci], S.stni_b[ci], i) + D * P.dt;
  bool yld = false;
  T mcrt = T(0);
  const bool by_closure = P.closure && code.z == RW_MODEL_HYPO_CS;  // the closure pass updates the stress
  const HypoC<T> hc = P.hypo[code.w];
  if (!by_closure) constitutive(code.z, mp, P.dt, vr.w, xyz(S.spin[i]), D, sg, yld, mcrt, P.mixed != 0, &hc);
  if (!yld) id.x = T(100);
  id.w = mcrt;
  if (!in_grid(P, I3{cp.x, cp.y, cp.z})) {
    cp.w = P.ncell_delete_m;
    id.x = T(999.0);
  }
  V4<T> po = S.pos_ori[c][i];
  if (dyn->time_f <= P.dt) po = V4<T>{T(0), T(0), T(0), T(0)};
  po = add3(po, xyz(vr) * P.dt);
  S.vel[c][i] = vr;
  S.pos[c][i] = ps;
  S.cellpos[c][i] = cp;
  st6(S.str_a[c], S.str_b[c], i, sg);
  st6(S.stn_a[c], S.stn_b[c], i, sn);
  S.idm[c][i] = id;
  S.pos_ori[c][i] = po;
  S.accad[i] = po;
  if (!by_closure) write_rec(P, S.rec, i, ps, vr, sg, id.y, code.x >= 10);
}

template <class T>
__global__ void __launch_bounds__(256, 4) k_corrector(const Params<T> P, DevState<T> S, const Dyn<T>* dyn) {
  corrector_row(P, S, dyn, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------------
// Shepard stress filter (src/field_smoothing.cu:26-111).  store != 0 copies the
// result back into the stress (StressRegularization) and refreshes the records.
// ---------------------------------------------------------------------------------
template <class T> __global__ void __launch_bounds__(128) k_shepard(const Params<T> P, DevState<T> S, const Dyn<T>* dyn,
                                                                   int only_filter_steps) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int npm = dyn->npm;
  if (t >= npm) return;
  if (only_filter_steps) {
    const int st = dyn->step;
    if (!(P.stress_shepard_filter != 0 && st % P.stress_shepard_filter == 0 && st != 0)) return;
  }
  const int i = P.npb + t;
  const int c = dyn->cur_main;
  const V4<T>* __restrict__ pos = S.pos[c];
  const V3<T> pos_i = ld3(pos, i);
  const int4 cp = S.cellpos[c][i];
  const I3 celli{cp.x, cp.y, cp.z};
  S6<T> sh = zero6<T>();
  T sumker = T(0.0f);
  const T th = P.two_h;
  auto scan = [&](const I3 cc, const V3<T> pp) {
    for (int oc = 0; oc < 27; ++oc) {
      const I3 off = off_of(oc);
      const I3 cj{cc.x + off.x, cc.y + off.y, cc.z + off.z};
      if (!in_grid(P, cj)) continue;
      const int2 rg = S.range[key_of(P, cj) + P.ncell_material];
      const V3<T> o = mulI(off, th);
      for (int j = rg.x; j < rg.y; ++j) {
        V3<T> dr = pp - ld3(pos, j) - o;
        const T r2 = pair_r2(dr.x, dr.y, dr.z);
        if (!(r2 < P.r2_prefilter)) continue;
        T r = pair_r(r2);
        T q = r * P.i_h;
        if (q < T(2.0f)) {
          T ker = kernel_w(P.knorm, q);
          T vol = S.idm[c][j].y / S.vel[c][j].w;
          sumker += ker * vol;
          sh = sh + ld6(S.str_a[c], S.str_b[c], j) * (ker * vol);
        }
      }
    }
  };
  // Inside the step (only_filter_steps) the filter runs after the corner search, where
  // the candidate lists are current (built, updated or kept at the end of the search)
  // and so are the neighbour records.  A list holds every material neighbour within
  // 2h in the scan's order (per cell offset, ascending index): walking its material
  // entries, with position, density and volume from the records, visits the same pairs
  // in the same order.  Entries four at a time, their data loaded together.
  const int kept = (only_filter_steps && S.nbg[0] && P.keep_lists && dyn->list_ok) ? S.nbg_cnt[dyn->lbuf][t] : -1;
  if (kept >= 0) {
    const Rec<T>* __restrict__ rec = S.rec;
    const unsigned* __restrict__ lst = S.nbg[dyn->lbuf] + t;
    const size_t stride = (size_t)S.nbg_stride;
    constexpr unsigned kNone = 0x7ffffffu;
    for (int e0 = 0; e0 < kept; e0 += 4) {
      unsigned ent[4];
      NbVals<T> nb[4];
      S6<T> sj[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) ent[k] = e0 + k < kept ? __ldcs(lst + (size_t)(e0 + k) * stride) : kNone;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int j = (int)(ent[k] & kNone);
        if (j == (int)kNone || j < P.npb) continue;
        nb[k] = load_nb(rec, j);
        sj[k] = ld6(S.str_a[c], S.str_b[c], j);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int j = (int)(ent[k] & kNone);
        if (j == (int)kNone || j < P.npb) continue;
        V3<T> dr = pos_i - V3<T>{nb[k].p.x, nb[k].p.y, nb[k].p.z};
        dr = dr - mulI(off_of((int)(ent[k] >> 27)), th);
        const T r2 = pair_r2(dr.x, dr.y, dr.z);
        if (!(r2 < P.r2_prefilter)) continue;
        T r = pair_r(r2);
        T q = r * P.i_h;
        if (q < T(2.0f)) {
          T ker = kernel_w(P.knorm, q);
          T vol = f_abs(nb[k].a.y);  // mass / density, as the record stores it
          sumker += ker * vol;
          sh = sh + sj[k] * (ker * vol);
        }
      }
    }
  } else {
    scan(celli, pos_i);
  }
  if (P.periodbound) {
    I3 cpb;
    V3<T> ppb;
    if (period_image(P, celli, pos_i, true, cpb, ppb)) scan(cpb, ppb);
  }
  if (sumker != T(0.f)) sh = sh / sumker;
  st6(S.tc_a, S.tc_b, i, sh);
}

template <class T> __global__ void k_shepard_store(const Params<T> P, DevState<T> S, const Dyn<T>* dyn,
                                                   int only_filter_steps) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int npm = dyn->npm;
  if (t >= npm) return;
  if (only_filter_steps) {
    const int st = dyn->step;
    if (!(P.stress_shepard_filter != 0 && st % P.stress_shepard_filter == 0 && st != 0)) return;
  }
  const int i = P.npb + t;
  const int c = dyn->cur_main;
  const S6<T> sh = ld6(S.tc_a, S.tc_b, i);
  st6(S.str_a[c], S.str_b[c], i, sh);
  write_rec(P, S.rec, i, S.pos[c][i], S.vel[c][i], sh, S.idm[c][i].y, S.codes[c][i].x >= 10);
}

// ---------------------------------------------------------------------------------
// Lateral wall force with FP64 accumulation (replaces the single-thread loop of
// src/utilities.cu:578-640): per-block sums in a fixed order, then one block adds
// the partial sums in block order, so the result is deterministic.
// ---------------------------------------------------------------------------------
constexpr int WF_THREADS = 256, WF_BLOCKS = 296;

// ---------------------------------------------------------------------------------
// Earth-pressure profile along the wall (cuGetValuesAlongLine, src/utilities.cu:266-322):
// three bands of thickness dr next to the wall, depth bins of size dz from z_top.  The
// reference's single loop keeps, per (band, bin), the value of the last particle in
// index order; here each particle claims its bin with atomicMax on its index and a
// second pass reads the winners' contact_mag.xx / dr, which is the same result.
// ---------------------------------------------------------------------------------
template <class T> __global__ void k_profile_claim(const Params<T> P, DevState<T> S, const Dyn<T>* dyn, double x_wall,
                                                   double z_top, double dz, int nbins, int* last) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  // The reference loops i over [npb, np): deleted particles take part too.
  if (t >= P.np - P.npb) return;
  const int i = P.npb + t;
  const int c = dyn->cur_main;
  const V4<T> ps = S.pos[c][i];
  const int4 cp = S.cellpos[c][i];
  const T h2 = (T)(2.0 * (double)P.h);
  const double px = (double)(ps.x + (T)cp.x * h2);
  const double pz = (double)(ps.z + (T)cp.z * h2);
  if (!(pz >= z_top - 1.0 && pz <= z_top)) return;
  const double dr = (double)P.dr;
  for (int band = 0; band < 3; ++band) {
    if (px >= x_wall + dr * band && px <= x_wall + dr * (band + 1)) {
      const int b = (int)((z_top - pz) / dz);
      if (b >= 0 && b < nbins) atomicMax(&last[band * nbins + b], i);
    }
  }
}

template <class T> __global__ void k_profile_read(const Params<T> P, DevState<T> S, int cpar, int nbins,
                                                  const int* last, double* out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  // the depth is written with the first band's value, as the reference's .xy
  out[4 * b] = last[b] >= 0 ? (double)b * (double)P.dr : 0.0;
  for (int band = 0; band < 3; ++band) {
    const int i = last[band * nbins + b];
    out[4 * b + 1 + band] = i >= 0 ? (double)(S.cf[cpar][i].x / P.dr) : 0.0;
  }
}

template <class T> __global__ void __launch_bounds__(WF_THREADS) k_wall_force(const Params<T> P, DevState<T> S,
                                                                             const Dyn<T>* dyn, int cpar, int mode,
                                                                             int wall_id, double xmax, double zmin,
                                                                             double zmax) {
  __shared__ double red[3][WF_THREADS / 32];
  const int npm = dyn->npm, c = dyn->cur_main;
  double a[3] = {0.0, 0.0, 0.0};
  for (int t = blockIdx.x * WF_THREADS + threadIdx.x; t < npm; t += gridDim.x * WF_THREADS) {
    const int i = P.npb + t;
    bool take;
    if (mode == 0) {
      const V4<T> cv = S.cv[cpar][i];
      take = (int)cv.w == wall_id && cv.y <= P.h * T(2);
    } else {
      const V4<T> ps = S.pos[c][i];
      const int4 cp = S.cellpos[c][i];
      const double px = (double)(ps.x + (T)cp.x * (T(2.0f) * P.h));
      const double pz = (double)(ps.z + (T)cp.z * (T(2.0f) * P.h));
      take = px <= xmax && pz >= zmin && pz <= zmax;
    }
    if (take) {
      const V4<T> f = S.cf[cpar][i];
      a[0] += (double)f.x;
      a[1] += (double)f.y;
      a[2] += (double)f.z;
    }
  }
  // warp-shuffle butterfly, then the warps' partials in warp order: a fixed order, so
  // the resultant does not change from run to run
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; ++k) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) red[k][warp] = a[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) {
      double v = 0.0;
      for (int w = 0; w < WF_THREADS / 32; ++w) v += red[k][w];
      S.wsum[3 * blockIdx.x + k] = v;
    }
}

static __global__ void k_wall_force_final(double* wsum, int nblocks) {
  if (threadIdx.x != 0) return;
  double a[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < nblocks; ++b)
    for (int k = 0; k < 3; ++k) a[k] += wsum[3 * b + k];
  for (int k = 0; k < 3; ++k) wsum[3 * nblocks + k] = a[k];
}

// Totals of the kept candidate lists: out[0] += entries, out[1] += soil particles with a list.
// Per-material constants of the hypoplastic update, once per case (rw_device.cuh).
template <class T> __global__ void k_hypo_table(const Params<T> P, HypoC<T>* out) {
  const int m = threadIdx.x;
  if (m < kModelMax) out[m] = hypo_coef(P.model_par[m][0], P.model_par[m][1], P.model_par[m][2], P.model_par[m][4]);
}

static __global__ void k_list_totals(const int* cnt, int n, unsigned long long* out) {
  unsigned long long e = 0, p = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    if (cnt[t] >= 0) {
      e += (unsigned long long)cnt[t];
      ++p;
    }
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    p += __shfl_xor_sync(0xffffffffu, p, o);
  }
  if ((threadIdx.x & 31) == 0 && p) {
    atomicAdd(&out[0], e);
    atomicAdd(&out[1], p);
  }
}

// ---------------------------------------------------------------------------------
// Learned constitutive closure (no counterpart in the reference): samples for its
// training and its use inside the step.  Features and target as in rw_mlp.cuh.
// ---------------------------------------------------------------------------------
struct ClosureTrust {
  float lo[mlp::IN], hi[mlp::IN];  // accepted feature ranges
  float out_max;                   // accepted |output|
  float err_max;                   // accepted judged relative error of the rate (<= 0: no bound)
};

template <class T> RWD void closure_features(const HypoPre<T>& h, const S6<T>& D, const T* mp, float* f) {
  const T ip = T(1) / h.p, inD = T(1) / h.nD;
  f[0] = (float)(h.str.xx * ip);
  f[1] = (float)(h.str.yy * ip);
  f[2] = (float)(h.str.zz * ip);
  f[3] = (float)(h.str.xy * ip);
  f[4] = (float)(h.str.xz * ip);
  f[5] = (float)(h.str.yz * ip);
  f[6] = (float)(D.xx * inD);
  f[7] = (float)(D.yy * inD);
  f[8] = (float)(D.zz * inD);
  f[9] = (float)(D.xy * inD);
  f[10] = (float)(D.xz * inD);
  f[11] = (float)(D.yz * inD);
  const T void_min = mp[9];
  f[12] = (float)((h.e - void_min) / (h.e_crt - void_min));
  f[13] = ((float)f_sin(mp[2]) - mlp::SIN_MID) / mlp::SIN_HALF;
  f[14] = (float)h.fd;  // the law's own void-ratio factor psi^alpha
  f[15] = 0.0f;
}

template <class T> RWD S6<T> closure_scale_out(const HypoPre<T>& h, const float* y) {
  const T sc = h.p * h.nD * (T)mlp::TARGET_SCALE;
  return S6<T>{(T)y[0] * sc, (T)y[1] * sc, (T)y[2] * sc, (T)y[3] * sc, (T)y[4] * sc, (T)y[5] * sc};
}

// Uniform in [0, 1) from a 64-bit key (splitmix64 finaliser).
RWD float hash_unit(unsigned long long k) {
  k += 0x9E3779B97F4A7C15ull;
  k = (k ^ (k >> 30)) * 0xBF58476D1CE4E5B9ull;
  k = (k ^ (k >> 27)) * 0x94D049BB133111EBull;
  k ^= k >> 31;
  return (float)(k >> 40) * (1.0f / 16777216.0f);
}

// Friction angle [rad] and initial void ratio ranges for augmented samples.
struct Augment {
  float phi_lo, phi_hi, e0_lo, e0_hi;
  unsigned long long seed;
  int on;
};

// Appends (features, exact normalised objective rate) of every stride-th soil particle
// with a HypoCS update, from the current stress, strain rate and density.  With
// augmentation each sample takes a friction angle and an initial void ratio drawn
// uniformly from the given ranges: the state comes from the solver, the target from the
// exact law for that material.
template <class T> __global__ void k_collect(const Params<T> P, DevState<T> S, const Dyn<T>* dyn, float* X, float* Tg,
                                             long long cap, unsigned long long* count, int stride, Augment aug) {
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) * stride;
  const int npm = dyn->npm, c = dyn->cur_main;
  bool ok = false;
  float f[mlp::IN], tg[mlp::OUT];
  if (t < npm) {
    const int i = P.npb + t;
    const int4 code = S.codes[c][i];
    if (code.y == 1 && code.z == RW_MODEL_HYPO_CS) {
      T mpa[kMatSize];
#pragma unroll
      for (int k = 0; k < kMatSize; ++k) mpa[k] = P.model_par[code.w][k];
      if (aug.on) {
        const unsigned long long key = aug.seed * 0x100000001B3ull + (unsigned long long)i;
        mpa[2] = (T)(aug.phi_lo + (aug.phi_hi - aug.phi_lo) * hash_unit(2 * key));
        mpa[11] = (T)(aug.e0_lo + (aug.e0_hi - aug.e0_lo) * hash_unit(2 * key + 1));
      }
      const T* mp = mpa;
      const S6<T> D = ld6(S.ace_a, S.ace_b, i);
      S6<T> sg = ld6(S.str_a[c], S.str_b[c], i);
      HypoPre<T> h;
      T mcrt;
      if (hypo_cs_pre(S.vel[c][i].w, V3<T>{T(0), T(0), T(0)}, D, sg, mp, mcrt, P.mixed != 0, h) && h.nD > T(0)) {
        closure_features(h, D, mp, f);
        const S6<T> R = hypo_cs_objective(h, D);
        const T sc = T(1) / (h.p * h.nD * (T)mlp::TARGET_SCALE);
        tg[0] = (float)(R.xx * sc);
        tg[1] = (float)(R.yy * sc);
        tg[2] = (float)(R.zz * sc);
        tg[3] = (float)(R.xy * sc);
        tg[4] = (float)(R.xz * sc);
        tg[5] = (float)(R.yz * sc);
        ok = true;
#pragma unroll
        for (int k = 0; k < mlp::IN; ++k) ok = ok && isfinite(f[k]);
#pragma unroll
        for (int o = 0; o < mlp::OUT; ++o) ok = ok && isfinite(tg[o]);
      }
    }
  }
  const unsigned mask = __ballot_sync(0xffffffffu, ok);
  if (!mask) return;
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (!ok) return;
  const long long idx = (long long)base + __popc(mask & ((1u << lane) - 1u));
  if (idx >= cap) return;
#pragma unroll
  for (int k = 0; k < mlp::IN; ++k) X[idx * mlp::IN + k] = f[k];
#pragma unroll
  for (int o = 0; o < mlp::OUT; ++o) Tg[idx * mlp::OUT + o] = tg[o];
}

// The HypoCS updates of one integrator stage (0: predictor half step, 1: corrector full
// step) with the learned objective rate: 128 soil slots per tile on the tensor cores;
// the Jaumann term, the cut-offs and every particle outside the trust region (or whose
// output leaves it) stay exact.  Every closure update is judged against the exact rate:
// stats = [offered, used, sum of relative errors, largest relative error].
// One tile of 128 soil slots (t = tile * 128 + thread); every thread of the block calls
// it for the same tile (the network runs on the whole tile).
template <class T>
RWD void closure_tile(const Params<T>& P, const DevState<T>& S, const Dyn<T>* dyn, mlp::FwdSmem& sm,
                      const ClosureTrust& tr, double* stats, int stage, int tile, uint32_t& phase) {
  const int npm = dyn->npm, c = dyn->cur_main;
  const int tid = threadIdx.x, lane = tid & 31;
  const T dt = stage == 0 ? T(0.5f) * P.dt : P.dt;
  {
    const int t = tile * mlp::TILE + tid, i = P.npb + t;
    bool mine = false, act = false;
    float f[mlp::IN];
#pragma unroll
    for (int k = 0; k < mlp::IN; ++k) f[k] = 0.0f;
    int4 code{0, 0, 0, 0};
    if (t < npm) {
      code = S.codes[c][i];
      mine = code.y == 1 && code.z == RW_MODEL_HYPO_CS;
      if (mine) {
        const T* mp = P.model_par[code.w];
        const S6<T> D = ld6(S.ace_a, S.ace_b, i);
        S6<T> sg = ld6(S.str_a[c], S.str_b[c], i);
        HypoPre<T> h;
        T mcrt;
        const HypoC<T> hc = P.hypo[code.w];
        if (hypo_cs_pre(S.vel[c][i].w, V3<T>{T(0), T(0), T(0)}, D, sg, mp, mcrt, P.mixed != 0, h, &hc) &&
            h.nD > T(0)) {
          closure_features(h, D, mp, f);
          act = true;
#pragma unroll
          for (int k = 0; k < mlp::IN; ++k) act = act && f[k] >= tr.lo[k] && f[k] <= tr.hi[k];
          if (!act)
#pragma unroll
            for (int k = 0; k < mlp::IN; ++k) f[k] = 0.0f;
        }
      }
    }
    float y[mlp::OUT];
#pragma unroll
    for (int o = 0; o < mlp::OUT; ++o) y[o] = 0.0f;
    if (__syncthreads_or(act)) {  // a tile without a trusted particle skips the network
      mlp::store_row<mlp::IN>(sm.x, tid, f);
      mlp::forward_tile(sm, 0, phase, y);
    }
    float used = 0.0f, offered = 0.0f, err = 0.0f;
    if (mine) {
      const T* mp = P.model_par[code.w];
      const S6<T> D = ld6(S.ace_a, S.ace_b, i);
      const V4<T> om4 = S.spin[i];
      S6<T> sg = ld6(S.str_a[c], S.str_b[c], i);
      HypoPre<T> h;
      T mcrt = T(0);
      const HypoC<T> hc = P.hypo[code.w];
      if (hypo_cs_pre(S.vel[c][i].w, V3<T>{om4.x, om4.y, om4.z}, D, sg, mp, mcrt, P.mixed != 0, h, &hc)) {
        S6<T> rate;
        bool use = act && !sm.err;
#pragma unroll
        for (int o = 0; o < mlp::OUT; ++o) use = use && fabsf(y[o]) <= tr.out_max;
        if (h.nD > T(0)) offered = 1.0f;
        if (use) {  // judged against the exact objective rate; kept within the error bound
          const S6<T> Rm = closure_scale_out(h, y);
          const S6<T> Rx = hypo_cs_objective(h, D);
          const S6<T> d = Rm - Rx;
          const T nx = f_sqrt(trace2(Rx, Rx)), nd = f_sqrt(trace2(d, d));
          err = (float)(nd / (nx + T(1e-30)));
          use = !(tr.err_max > 0.0f) || err <= tr.err_max;
        }
        if (use) {
          used = 1.0f;
          rate = h.jau + closure_scale_out(h, y);
        } else {
          err = 0.0f;
          rate = hypo_cs_rate(h, D);
        }
        hypo_cs_post(dt, h, rate, sg);
      }
      st6(S.str_a[c], S.str_b[c], i, sg);
      if (stage == 1) S.idm[c][i].w = mcrt;
      write_rec(P, S.rec, i, S.pos[c][i], S.vel[c][i], sg, S.idm[c][i].y, code.x >= 10);
    }
    // statistics: one atomic per warp and counter
    float so = offered, su = used, se = err, sx = err;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      so += __shfl_xor_sync(0xffffffffu, so, o);
      su += __shfl_xor_sync(0xffffffffu, su, o);
      se += __shfl_xor_sync(0xffffffffu, se, o);
      sx = fmaxf(sx, __shfl_xor_sync(0xffffffffu, sx, o));
    }
    if (lane == 0 && so > 0.0f) {
      atomicAdd(&stats[0], (double)so);
      atomicAdd(&stats[1], (double)su);
      atomicAdd(&stats[2], (double)se);
      atomicMax(reinterpret_cast<unsigned long long*>(&stats[3]), (unsigned long long)__double_as_longlong((double)sx));
    }
  }
}

// One integrator stage (0: predictor, 1: corrector) with the learned closure, in one
// persistent launch: the rows of a tile are advanced as predictor_row / corrector_row do
// (HypoCS stresses left to the closure), then the same block runs the closure on them.
// Tiles: the boundary rows first (integrator only), then the soil slots (in the predictor
// the deleted slots too, for their step-start copies).
template <class T, int Stage>
__global__ void __launch_bounds__(mlp::TILE) k_integrate_cl(const Params<T> P, DevState<T> S, Dyn<T>* dyn,
                                                             mlp::Net net, ClosureTrust tr, double* stats) {
  extern __shared__ __align__(128) unsigned char raw[];
  mlp::FwdSmem& sm = *reinterpret_cast<mlp::FwdSmem*>(raw);
  mlp::load_fwd(sm, net);
  if (threadIdx.x == 0) sm.err = 0;
  mlp::block_setup(&sm.bar, &sm.tmem, 64);
  const int nb_tiles = (P.npb + mlp::TILE - 1) / mlp::TILE;
  const int soil_rows = Stage == 0 ? P.np - P.npb : dyn->npm;
  const int n_tiles = nb_tiles + (soil_rows + mlp::TILE - 1) / mlp::TILE;
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {  // block-uniform
    if (tile < nb_tiles) {
      const int i = tile * mlp::TILE + threadIdx.x;
      if (i < P.npb) {
        if (Stage == 0) predictor_row(P, S, dyn, i);
        else corrector_row(P, S, dyn, i);
      }
      continue;
    }
    const int st = tile - nb_tiles, t = st * mlp::TILE + threadIdx.x;
    if (t < soil_rows) {
      if (Stage == 0) predictor_row(P, S, dyn, P.npb + t);
      else corrector_row(P, S, dyn, P.npb + t);
    }
    closure_tile(P, S, dyn, sm, tr, stats, Stage, st, phase);
  }
  __syncthreads();
  mlp::drain_after_timeout(&sm.bar, sm.err, phase);
  mlp::block_teardown(sm.tmem, 64);
  if (threadIdx.x == 0 && sm.err) atomicOr(&dyn->err, 16u);
}

}  // namespace rw
