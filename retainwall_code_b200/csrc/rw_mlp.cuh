// Learned constitutive closure: a 16-64-64-64-64-6 multilayer perceptron (SiLU hidden
// activations, BF16 weights and activations, FP32 accumulation) evaluated 128 samples at
// a time on the tcgen05 tensor cores.  Shared by the inference path inside the time step
// (rw_engine.cu) and by the training kernels (rw_mlp.cu).
//
// What it predicts: the objective (Jaumann-free) part of the HypoCS stress rate of
// cuMatModHypo (src/constitutive_model.h:269),
//     R = D (C1 tr s) + s (C2 tr D) + s (C3 tr(sD) / tr s) + (s + s_dev) (fd C4 |D|),
// normalised by p |D| and TARGET_SCALE, from the features
//     f[0..5]  = s / p                  (s = stress minus cohesion, p = -tr s / 3)
//     f[6..11] = D / |D|                (|D| = sqrt(D : D), as the reference's norm)
//     f[12]    = (e - e_min) / (e_c(p) - e_min)   (relative void ratio, fd = f[12]^alpha)
//     f[13]    = (sin phi_c - SIN_MID) / SIN_HALF (friction angle of the material)
//     f[14]    = f[12]^alpha            (the void-ratio factor fd of the law)
//     f[15]    = 0                      (padding to the MMA's K = 16)
// The Jaumann term, the tension cut-off and the cone projection stay exact.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "rw_tc.cuh"

struct rw_mlp;

namespace rw {
namespace mlp {

constexpr int IN = 16, HID = 64, OUT = 6, OUTP = 16, NHID = 4, TILE = 128;
constexpr float TARGET_SCALE = 1000.0f;
constexpr float SIN_MID = 0.556f, SIN_HALF = 0.087f;

// Flat FP32 parameters: W1 [IN x HID], b1, W2..W4 [HID x HID], b2..b4, W5 [HID x OUT], b5
// (W[in][out], y = x W + b).
constexpr int P_W1 = 0, P_B1 = P_W1 + IN * HID;
constexpr int P_W2 = P_B1 + HID, P_B2 = P_W2 + HID * HID;
constexpr int P_W3 = P_B2 + HID, P_B3 = P_W3 + HID * HID;
constexpr int P_W4 = P_B3 + HID, P_B4 = P_W4 + HID * HID;
constexpr int P_W5 = P_B4 + HID, P_B5 = P_W5 + HID * OUT;
constexpr int NPARAM = P_B5 + OUT;

// Packed BF16 operands (K-major, no swizzle, see rw_tc.cuh).
// Forward B operands W^T as [N = out x K = in]:
constexpr int FW1 = 0, FW2 = FW1 + HID * IN * 2, FW3 = FW2 + HID * HID * 2, FW4 = FW3 + HID * HID * 2;
constexpr int FW5 = FW4 + HID * HID * 2, FWBYTES = FW5 + OUTP * HID * 2;
// Backward-data B operands W as [N = in x K = out] (layers 2..5):
constexpr int BW2 = 0, BW3 = BW2 + HID * HID * 2, BW4 = BW3 + HID * HID * 2, BW5 = BW4 + HID * HID * 2;
constexpr int BWBYTES = BW5 + HID * OUTP * 2;
// Biases (FP32): b1..b4 at 64 l, b5 at 256 (16 entries, 6 used).
constexpr int NBIAS = NHID * HID + OUTP;

// Device view of one network's packed weights.
struct Net {
  const unsigned char* fw;
  const unsigned char* bw;
  const float* bias;
};

__device__ __forceinline__ float sigm(float z) { return 0.5f + 0.5f * tc::tanh_approx(0.5f * z); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = sigm(z);
  return s + z * s * (1.0f - s);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }

// Row r of a K-major tile with K columns, written from K floats (K multiple of 8).
template <int K>
__device__ __forceinline__ void store_row(unsigned char* tile, int r, const float* v) {
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 8) {
    uint4 q;
    q.x = pack_bf16(v[k0 + 0], v[k0 + 1]);
    q.y = pack_bf16(v[k0 + 2], v[k0 + 3]);
    q.z = pack_bf16(v[k0 + 4], v[k0 + 5]);
    q.w = pack_bf16(v[k0 + 6], v[k0 + 7]);
    *reinterpret_cast<uint4*>(tile + tc::kmajor_off(r, k0, K)) = q;
  }
}
// Columns [k0, k0 + 16) of row r of a K-major tile with K columns.
template <int K>
__device__ __forceinline__ void store_chunk16(unsigned char* tile, int r, int k0, const float* v) {
#pragma unroll
  for (int h = 0; h < 16; h += 8) {
    uint4 q;
    q.x = pack_bf16(v[h + 0], v[h + 1]);
    q.y = pack_bf16(v[h + 2], v[h + 3]);
    q.z = pack_bf16(v[h + 4], v[h + 5]);
    q.w = pack_bf16(v[h + 6], v[h + 7]);
    *reinterpret_cast<uint4*>(tile + tc::kmajor_off(r, k0 + h, K)) = q;
  }
}
// Element (r, k) of a K-major BF16 tile.
template <int K>
__device__ __forceinline__ float load_elem(const unsigned char* tile, int r, int k) {
  const unsigned short u = *reinterpret_cast<const unsigned short*>(tile + tc::kmajor_off(r, k, K));
  return __uint_as_float((uint32_t)u << 16);
}

// Shared memory of the forward pass of one 128-sample tile.
struct FwdSmem {
  alignas(128) unsigned char fw[FWBYTES];
  alignas(128) unsigned char x[TILE * IN * 2];
  alignas(128) unsigned char h[TILE * HID * 2];
  float bias[NBIAS];
  uint64_t bar;
  uint32_t tmem;
  int err;
};

// Copies the packed forward weights and biases into shared memory (all threads).
__device__ __forceinline__ void load_fwd(FwdSmem& sm, const Net& net) {
  const uint4* src = reinterpret_cast<const uint4*>(net.fw);
  uint4* dst = reinterpret_cast<uint4*>(sm.fw);
  for (int k = threadIdx.x; k < FWBYTES / 16; k += blockDim.x) dst[k] = src[k];
  for (int k = threadIdx.x; k < NBIAS; k += blockDim.x) sm.bias[k] = net.bias[k];
}

// Issues the MMAs of layer l (0..4) of one tile: A = x (l = 0) or h, B = packed W^T,
// D = TMEM columns [dcol, dcol + N).
__device__ __forceinline__ void issue_layer(const unsigned char* a_tile, int K, const unsigned char* b_tile, int N,
                                            uint32_t d_tmem) {
  const uint32_t a0 = tc::smem_u32(a_tile), b0 = tc::smem_u32(b_tile);
  const uint32_t sbo = (uint32_t)(K / 8) * 128u;
  const uint32_t idesc = tc::idesc_bf16(TILE, N);
  for (int ks = 0; ks < K / 16; ++ks)
    tc::mma_bf16(d_tmem, tc::sdesc(a0 + 256u * ks, 128u, sbo), tc::sdesc(b0 + 256u * ks, 128u, sbo), idesc,
                 ks > 0 ? 1u : 0u);
}

// Forward pass of the tile already in sm.x (rows = threads of this 128-thread block).
// TMEM: columns [tcol, tcol + 64) of the allocation at sm.tmem.  Each thread receives
// its row's six outputs (biases added).  phase counts the mbarrier phases used so far.
// A wait that times out sets sm.err: the outputs are then meaningless, and this and
// every later call issue no further MMAs (all threads see sm.err after the barrier at
// the top of a layer and return together).
__device__ __forceinline__ void forward_tile(FwdSmem& sm, int tcol, uint32_t& phase, float* out) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t tbase = sm.tmem + (uint32_t)tcol;
  const uint32_t tlane = tbase + ((uint32_t)(warp * 32) << 16);
  for (int l = 0; l <= NHID; ++l) {
    tc::fence_smem_to_async();
    __syncthreads();
    if (sm.err) return;
    if (tid == 0) {
      tc::fence_after_sync();
      if (l == 0) issue_layer(sm.x, IN, sm.fw + FW1, HID, tbase);
      else if (l < NHID) issue_layer(sm.h, HID, sm.fw + (l == 1 ? FW2 : l == 2 ? FW3 : FW4), HID, tbase);
      else issue_layer(sm.h, HID, sm.fw + FW5, OUTP, tbase);
      tc::mma_commit(&sm.bar);
    }
    if (!tc::mbar_wait(&sm.bar, phase & 1u)) sm.err = 1;
    ++phase;
    tc::fence_after_sync();
    if (l < NHID) {
      const float* b = sm.bias + l * HID;
#pragma unroll 1
      for (int c = 0; c < HID; c += 16) {
        float v[16];
        tc::tmem_ld16(tlane + (uint32_t)c, v);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = silu(v[k] + b[c + k]);
        store_chunk16<HID>(sm.h, tid, c, v);
      }
      tc::fence_before_sync();
    } else {
      float v[16];
      tc::tmem_ld16(tlane, v);
#pragma unroll
      for (int o = 0; o < OUT; ++o) out[o] = v[o] + sm.bias[NHID * HID + o];
      tc::fence_before_sync();
    }
  }
}

// One-time set-up of a block that runs tiles: mbarrier (thread 0) and TMEM (warp 0).
__device__ __forceinline__ void block_setup(uint64_t* bar, uint32_t* tmem_slot, uint32_t ncols) {
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(tmem_slot, ncols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}
// After a timed-out wait (err set), the MMAs of the phase that timed out (phase - 1)
// may still be running: one more bounded wait for it before the TMEM is released.
__device__ __forceinline__ void drain_after_timeout(uint64_t* bar, int err, uint32_t phase) {
  if (err && threadIdx.x == 0 && phase > 0) tc::mbar_wait(bar, (phase - 1u) & 1u);
}
__device__ __forceinline__ void block_teardown(uint32_t tmem, uint32_t ncols) {
  tc::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, ncols);
  }
}

// Host-side access of the time step to a network object (defined in rw_mlp.cu).
Net net_view(const rw_mlp* m);
int device_of(const rw_mlp* m);
long long free_slots(const rw_mlp* m);
// Device pointers of the next free sample slot.
void next_slot(rw_mlp* m, float** x, float** t);
void commit(rw_mlp* m, long long n);

}  // namespace mlp
}  // namespace rw
