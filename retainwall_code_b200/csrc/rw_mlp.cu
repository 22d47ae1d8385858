// Learned constitutive closure: the network object, its tcgen05 forward and training
// kernels and the C ABI (include/retainwall.h, rw_mlp_*).  The reference has no learned
// component; this is the surrogate of the HypoCS objective stress rate described in
// rw_mlp.cuh, trained on samples the plain solver generates.
//
// Training step (one launch per minibatch, one 128-sample tile per loop iteration):
//   forward  : five tcgen05 MMAs per tile (BF16 operands in shared memory, FP32 in
//              TMEM); the four hidden pre-activations stay in TMEM for the backward pass;
//   backward : dH(l-1) = G(l) W(l) on tcgen05 (G in BF16, as it feeds the MMA);
//              dW(l) = H(l-1)^T G(l) and db(l) = sum G(l) on the CUDA cores in FP32,
//              accumulated per block in shared memory (there is no TMEM or shared memory
//              left for a third set of transposed operand tiles), then added to the
//              global gradient once per launch;
//   update   : Adam on the FP32 master parameters, which also re-packs the BF16
//              operand tiles.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/retainwall.h"
#include "rw_mlp.cuh"

namespace rw {
namespace mlp {

// ---------------------------------------------------------------------------------
// Parameter packing: FP32 master value k -> its BF16 operand positions / bias slot.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void put_bf16(unsigned char* base, uint32_t off, float w) {
  *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(w);
}

__device__ void pack_param(int k, float w, unsigned char* fw, unsigned char* bw, float* bias) {
  if (k < P_B1) {
    put_bf16(fw, FW1 + tc::kmajor_off(k % HID, k / HID, IN), w);
  } else if (k < P_W2) {
    bias[k - P_B1] = w;
  } else if (k < P_B2 || (k >= P_W3 && k < P_B3) || (k >= P_W4 && k < P_B4)) {
    const int l = k < P_B2 ? 2 : k < P_B3 ? 3 : 4;
    const int q = k - (l == 2 ? P_W2 : l == 3 ? P_W3 : P_W4);
    const int i = q / HID, o = q % HID;
    put_bf16(fw, (l == 2 ? FW2 : l == 3 ? FW3 : FW4) + tc::kmajor_off(o, i, HID), w);
    put_bf16(bw, (l == 2 ? BW2 : l == 3 ? BW3 : BW4) + tc::kmajor_off(i, o, HID), w);
  } else if (k < P_W3) {
    bias[HID + (k - P_B2)] = w;
  } else if (k < P_W4) {
    bias[2 * HID + (k - P_B3)] = w;
  } else if (k < P_W5) {
    bias[3 * HID + (k - P_B4)] = w;
  } else if (k < P_B5) {
    const int q = k - P_W5;
    const int i = q / OUT, o = q % OUT;
    put_bf16(fw, FW5 + tc::kmajor_off(o, i, HID), w);
    put_bf16(bw, BW5 + tc::kmajor_off(i, o, OUTP), w);
  } else if (k < NPARAM) {
    bias[NHID * HID + (k - P_B5)] = w;
  }
}

__global__ void k_pack(const float* __restrict__ p, unsigned char* fw, unsigned char* bw, float* bias) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < NPARAM) pack_param(k, p[k], fw, bw, bias);
}

// Adam step on every parameter (bias-corrected), re-packing the operands; clears the
// gradient for the next minibatch.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       float lr, float b1, float b2, float eps, float bc1, float bc2, unsigned char* fw,
                       unsigned char* bw, float* bias) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NPARAM) return;
  const float gk = g[k];
  const float mk = b1 * m[k] + (1.0f - b1) * gk;
  const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
  m[k] = mk;
  v[k] = vk;
  const float w = p[k] - lr * (mk / bc1) / (sqrtf(vk / bc2) + eps);
  p[k] = w;
  g[k] = 0.0f;
  pack_param(k, w, fw, bw, bias);
}

// Sample index s of an epoch in shuffled order: s -> (a s + c) mod n with a coprime to n.
__device__ __forceinline__ int shuffled(long long s, long long n, long long a, long long c) {
  return (int)((a * s + c) % n);
}

// ---------------------------------------------------------------------------------
// Forward over arbitrary samples (X [n x IN] -> Y [n x OUT]).
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE) k_forward(Net net, const float* __restrict__ X, int n, float* __restrict__ Y,
                                                  int* err) {
  extern __shared__ __align__(128) unsigned char raw[];
  FwdSmem& sm = *reinterpret_cast<FwdSmem*>(raw);
  load_fwd(sm, net);
  if (threadIdx.x == 0) sm.err = 0;
  block_setup(&sm.bar, &sm.tmem, 64);
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile * TILE < n; tile += gridDim.x) {
    const int s = tile * TILE + threadIdx.x;
    float f[IN];
#pragma unroll
    for (int k = 0; k < IN; ++k) f[k] = s < n ? X[(size_t)s * IN + k] : 0.0f;
    store_row<IN>(sm.x, threadIdx.x, f);
    float out[OUT];
    forward_tile(sm, 0, phase, out);
    if (s < n)
#pragma unroll
      for (int o = 0; o < OUT; ++o) Y[(size_t)s * OUT + o] = out[o];
  }
  __syncthreads();
  drain_after_timeout(&sm.bar, sm.err, phase);
  block_teardown(sm.tmem, 64);
  if (threadIdx.x == 0 && sm.err) atomicExch(err, 1);
}

// ---------------------------------------------------------------------------------
// Training: forward + backward of a minibatch, gradient accumulated into grad.
// ---------------------------------------------------------------------------------
struct TrainSmem {
  alignas(128) unsigned char fw[FWBYTES];
  alignas(128) unsigned char bw[BWBYTES];
  alignas(128) unsigned char x[TILE * IN * 2];
  alignas(128) unsigned char h[NHID][TILE * HID * 2];
  alignas(128) unsigned char g[TILE * HID * 2];
  alignas(128) unsigned char g5[TILE * OUTP * 2];
  float acc[NPARAM];
  float bias[NBIAS];
  uint64_t bar;
  uint32_t tmem;
  int err;
};
constexpr uint32_t TRAIN_TMEM_COLS = 512;  // Z1..Z4 at 0..255, output at 256, dH at 320
constexpr int TCOL_Y = 256, TCOL_DH = 320;

// Weight gradients on the tensor cores.  For the tile's 128 samples b,
//   dW(l) = H(l-1)^T G(l)   (layers 2..5: M = 64 input features, N = the layer's outputs)
//   dW(1)^T = G(1)^T X      (layer 1: M = 64 outputs, N = 16 inputs)
// as D[64 x N] = A^T B with A and B the 128-row activation / signal tiles already in
// shared memory, read MN-major (no transposed copy).  Issued by one thread; K = 128 in
// eight steps of 16.
__device__ __forceinline__ void issue_wgrad(const unsigned char* a_tile, int Ka, const unsigned char* b_tile, int Kb,
                                            int N, uint32_t d_tmem) {
  const uint32_t a0 = tc::smem_u32(a_tile), b0 = tc::smem_u32(b_tile);
  const uint32_t idesc = tc::idesc_bf16_mn(64, N);
  for (int ks = 0; ks < TILE / 16; ++ks)
    tc::mma_bf16(d_tmem, tc::sdesc_mn(a0 + (uint32_t)(Ka * 32 * ks), Ka), tc::sdesc_mn(b0 + (uint32_t)(Kb * 32 * ks), Kb),
                 idesc, ks > 0 ? 1u : 0u);
}

// Adds a 64 x N accumulator (M = 64 layout: row r in TMEM lane 32 (r / 16) + r % 16, so
// lanes 0..15 of warp w hold rows 16 w .. 16 w + 15) into acc[base + col * 64 + row], for
// the columns col < ncols.  tcol: the accumulator's first column.  Every lane takes part
// in the TMEM loads; lanes 16..31 discard theirs.
template <int N>
__device__ __forceinline__ void add_wgrad(float* acc, uint32_t tmem, uint32_t tcol, int base, int ncols) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const uint32_t taddr = tmem + ((uint32_t)(w * 32) << 16) + tcol;
  const int r = 16 * w + l;
#pragma unroll
  for (int c = 0; c < N; c += 16) {
    float v[16];
    tc::tmem_ld16(taddr + (uint32_t)c, v);
    if (l < 16)
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (c + k < ncols) acc[base + (c + k) * 64 + r] += v[k];
  }
}

// acc[b0 + o] += sum over the tile's 128 rows of G[b][o], for o < NB (G: 128 x Kg tile).
// Thread o sums column o; the rows are visited in an order rotated by o / 8, so the four
// 8-column groups of a warp read different banks.
template <int Kg, int NB>
__device__ __forceinline__ void add_bias_grad(float* acc, int b0, const unsigned char* g) {
  const int o = threadIdx.x;
  if (o >= NB) return;
  float t = 0.0f;
#pragma unroll 8
  for (int k = 0; k < TILE; ++k) t += load_elem<Kg>(g, (k + (o >> 3)) & (TILE - 1), o);
  acc[b0 + o] += t;
}

// The accumulator layout of the weight gradients in shared memory: W1 as the parameters
// ([in][out]), W2..W5 transposed ([out][in], the rows of the tensor-core products).
__device__ __forceinline__ int acc_index(int k) {
  if (k >= P_W2 && k < P_B4 && !((k >= P_B2 && k < P_W3) || (k >= P_B3 && k < P_W4))) {
    const int w0 = k < P_B2 ? P_W2 : k < P_B3 ? P_W3 : P_W4;
    const int rel = k - w0;
    return w0 + (rel % HID) * HID + rel / HID;
  }
  if (k >= P_W5 && k < P_B5) {
    const int rel = k - P_W5;
    return P_W5 + (rel % OUT) * HID + rel / OUT;
  }
  return k;
}

__global__ void __launch_bounds__(TILE, 1) k_train(Net net, const float* __restrict__ X, const float* __restrict__ Tg,
                                                long long n_all, long long first, int n, long long sa, long long sc,
                                                float inv_count, float* __restrict__ grad, double* __restrict__ loss,
                                                int* err) {
  extern __shared__ __align__(128) unsigned char raw[];
  TrainSmem& sm = *reinterpret_cast<TrainSmem*>(raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  {
    const uint4* s1 = reinterpret_cast<const uint4*>(net.fw);
    uint4* d1 = reinterpret_cast<uint4*>(sm.fw);
    for (int k = tid; k < FWBYTES / 16; k += TILE) d1[k] = s1[k];
    const uint4* s2 = reinterpret_cast<const uint4*>(net.bw);
    uint4* d2 = reinterpret_cast<uint4*>(sm.bw);
    for (int k = tid; k < BWBYTES / 16; k += TILE) d2[k] = s2[k];
    for (int k = tid; k < NBIAS; k += TILE) sm.bias[k] = net.bias[k];
    for (int k = tid; k < NPARAM; k += TILE) sm.acc[k] = 0.0f;
    if (tid == 0) sm.err = 0;
  }
  block_setup(&sm.bar, &sm.tmem, TRAIN_TMEM_COLS);
  const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
  const uint32_t tl = sm.tmem + lane_off;
  uint32_t phase = 0;
  float lsum = 0.0f;
  // After a timed-out wait (sm.err, seen by every thread after the next barrier) no
  // MMA is issued and none is waited for; the tile loop ends at the next tile.
  auto wait_mma = [&]() {
    if (sm.err) return;
    if (!tc::mbar_wait(&sm.bar, phase & 1u)) sm.err = 1;
    ++phase;
    tc::fence_after_sync();
  };
  for (int tile = blockIdx.x; tile * TILE < n; tile += gridDim.x) {
    __syncthreads();  // the previous tile's first-layer weight gradient has read sm.x
    if (sm.err) break;
    const int r = tile * TILE + tid;
    const bool valid = r < n;
    const long long s = valid ? shuffled(first + r, n_all, sa, sc) : 0;
    float f[IN], t[OUT];
#pragma unroll
    for (int k = 0; k < IN; ++k) f[k] = valid ? X[s * IN + k] : 0.0f;
#pragma unroll
    for (int o = 0; o < OUT; ++o) t[o] = valid ? Tg[s * OUT + o] : 0.0f;
    store_row<IN>(sm.x, tid, f);
    // ---- forward: Z(l) kept in TMEM columns 64 (l - 1) -------------------------
    float y[OUT];
    for (int l = 0; l <= NHID; ++l) {
      tc::fence_smem_to_async();
      __syncthreads();
      if (tid == 0 && !sm.err) {
        tc::fence_after_sync();
        if (l == 0) issue_layer(sm.x, IN, sm.fw + FW1, HID, sm.tmem);
        else if (l < NHID)
          issue_layer(sm.h[l - 1], HID, sm.fw + (l == 1 ? FW2 : l == 2 ? FW3 : FW4), HID, sm.tmem + 64u * l);
        else issue_layer(sm.h[NHID - 1], HID, sm.fw + FW5, OUTP, sm.tmem + TCOL_Y);
        tc::mma_commit(&sm.bar);
      }
      wait_mma();
      if (l < NHID) {
        const float* b = sm.bias + l * HID;
#pragma unroll 1
        for (int c = 0; c < HID; c += 16) {
          float v[16];
          tc::tmem_ld16(tl + 64u * l + c, v);
#pragma unroll
          for (int k = 0; k < 16; ++k) v[k] = silu(v[k] + b[c + k]);
          store_chunk16<HID>(sm.h[l], tid, c, v);
        }
      } else {
        float v[16];
        tc::tmem_ld16(tl + TCOL_Y, v);
#pragma unroll
        for (int o = 0; o < OUT; ++o) y[o] = v[o] + sm.bias[NHID * HID + o];
      }
      tc::fence_before_sync();
    }
    // ---- loss (mean over samples and outputs) and its gradient -------------------
    {
      float g5[16];
#pragma unroll
      for (int o = 0; o < 16; ++o) g5[o] = 0.0f;
#pragma unroll
      for (int o = 0; o < OUT; ++o) {
        const float d = valid ? y[o] - t[o] : 0.0f;
        lsum += d * d;
        g5[o] = 2.0f * d * inv_count;
      }
      store_chunk16<OUTP>(sm.g5, tid, 0, g5);
    }
    tc::fence_smem_to_async();
    __syncthreads();
    if (tid == 0 && !sm.err) {  // dH4 = G5 W5 and dW5 = H4^T G5 (into the output's columns)
      tc::fence_after_sync();
      issue_layer(sm.g5, OUTP, sm.bw + BW5, HID, sm.tmem + TCOL_DH);
      issue_wgrad(sm.h[NHID - 1], HID, sm.g5, OUTP, OUTP, sm.tmem + TCOL_Y);
      tc::mma_commit(&sm.bar);
    }
    add_bias_grad<OUTP, OUT>(sm.acc, P_B5, sm.g5);
    wait_mma();
    add_wgrad<OUTP>(sm.acc, sm.tmem, TCOL_Y, P_W5, OUT);  // warp-wide loads: unconditional
    tc::fence_before_sync();
    // ---- hidden layers, last to first -------------------------------------------
    for (int l = NHID; l >= 1; --l) {
      __syncthreads();  // the previous bias gradient has finished reading sm.g
      const float* b = sm.bias + (l - 1) * HID;
#pragma unroll 1
      for (int c = 0; c < HID; c += 16) {
        float dh[16], z[16];
        tc::tmem_ld16(tl + TCOL_DH + c, dh);
        tc::tmem_ld16(tl + 64u * (l - 1) + c, z);
#pragma unroll
        for (int k = 0; k < 16; ++k) dh[k] *= silu_grad(z[k] + b[c + k]);
        store_chunk16<HID>(sm.g, tid, c, dh);
      }
      tc::fence_before_sync();
      tc::fence_smem_to_async();
      __syncthreads();
      // dH(l-1) = G(l) W(l) into the dH columns, and the weight gradient into Z(l)'s
      // columns (read above): dW(l) = H(l-1)^T G(l), for layer 1 dW(1)^T = G(1)^T X
      const uint32_t zcol = 64u * (l - 1);
      if (tid == 0 && !sm.err) {
        tc::fence_after_sync();
        if (l > 1) {
          issue_layer(sm.g, HID, sm.bw + (l == 2 ? BW2 : l == 3 ? BW3 : BW4), HID, sm.tmem + TCOL_DH);
          issue_wgrad(sm.h[l - 2], HID, sm.g, HID, HID, sm.tmem + zcol);
        } else {
          issue_wgrad(sm.g, HID, sm.x, IN, IN, sm.tmem + zcol);
        }
        tc::mma_commit(&sm.bar);
      }
      add_bias_grad<HID, HID>(sm.acc, l == 1 ? P_B1 : l == 2 ? P_B2 : l == 3 ? P_B3 : P_B4, sm.g);
      wait_mma();
      if (l > 1) add_wgrad<HID>(sm.acc, sm.tmem, zcol, l == 2 ? P_W2 : l == 3 ? P_W3 : P_W4, HID);
      else add_wgrad<IN>(sm.acc, sm.tmem, zcol, P_W1, IN);
      tc::fence_before_sync();
    }
  }
  __syncthreads();
  for (int k = tid; k < NPARAM; k += TILE) atomicAdd(&grad[k], sm.acc[acc_index(k)]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((tid & 31) == 0) atomicAdd(loss, (double)lsum);
  drain_after_timeout(&sm.bar, sm.err, phase);
  block_teardown(sm.tmem, TRAIN_TMEM_COLS);
  if (tid == 0 && sm.err) atomicExch(err, 1);
}

// Feature ranges of the stored samples (trust region of the closure): per feature
// min / max, and the largest |target|; one pass, block partials folded by atomics on
// the order-preserving integer image of the floats.
__device__ __forceinline__ unsigned f2ord(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__global__ void k_ranges(const float* __restrict__ X, const float* __restrict__ Tg, long long n, unsigned* lo,
                         unsigned* hi, unsigned* tmax) {
  __shared__ unsigned slo[IN], shi[IN], st;
  if (threadIdx.x < IN) {
    slo[threadIdx.x] = 0xFFFFFFFFu;
    shi[threadIdx.x] = 0u;
  }
  if (threadIdx.x == 0) st = 0u;
  __syncthreads();
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < IN; ++k) {
      const unsigned u = f2ord(X[s * IN + k]);
      atomicMin(&slo[k], u);
      atomicMax(&shi[k], u);
    }
    float m = 0.0f;
#pragma unroll
    for (int o = 0; o < OUT; ++o) m = fmaxf(m, fabsf(Tg[s * OUT + o]));
    atomicMax(&st, __float_as_uint(m));
  }
  __syncthreads();
  if (threadIdx.x < IN) {
    atomicMin(&lo[threadIdx.x], slo[threadIdx.x]);
    atomicMax(&hi[threadIdx.x], shi[threadIdx.x]);
  }
  if (threadIdx.x == 0) atomicMax(tmax, st);
}

}  // namespace mlp
}  // namespace rw

// =====================================================================================
// Host object and C ABI
// =====================================================================================
using namespace rw::mlp;

struct rw_mlp {
  int device = 0;
  cudaStream_t st = nullptr;
  float* params = nullptr;  // FP32 master
  float* grad = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  unsigned char* fw = nullptr;
  unsigned char* bw = nullptr;
  float* bias = nullptr;
  int* err = nullptr;
  double* loss = nullptr;
  unsigned* ranges = nullptr;  // lo[IN], hi[IN], tmax
  long long adam_t = 0;
  // samples
  float* sx = nullptr;
  float* stg = nullptr;
  long long cap = 0, n = 0;
  std::string msg;
  std::mutex mu;
};

namespace {

thread_local std::string g_mlp_err;

rw_status fail(rw_mlp* m, rw_status s, const std::string& what) {
  if (m) m->msg = what;
  g_mlp_err = what;
  return s;
}

#define MLP_CU(m, call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return fail(m, RW_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

Net net_of(const rw_mlp* m) { return Net{m->fw, m->bw, m->bias}; }

rw_status check_err(rw_mlp* m) {
  int e = 0;
  MLP_CU(m, cudaMemcpyAsync(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->st));
  MLP_CU(m, cudaStreamSynchronize(m->st));
  if (e) {
    MLP_CU(m, cudaMemsetAsync(m->err, 0, sizeof(int), m->st));
    return fail(m, RW_ETIMEDOUT, "a tensor-core completion wait gave up");
  }
  return RW_OK;
}

rw_status pack_all(rw_mlp* m) {
  k_pack<<<(NPARAM + 255) / 256, 256, 0, m->st>>>(m->params, m->fw, m->bw, m->bias);
  MLP_CU(m, cudaGetLastError());
  return RW_OK;
}

int num_sms(int dev) {
  int n = 148;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

// Forward of n samples already on the device.
rw_status forward_dev(rw_mlp* m, const float* dx, int n, float* dy) {
  if (n <= 0) return RW_OK;
  const int smem = (int)sizeof(FwdSmem);
  MLP_CU(m, cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int tiles = (n + TILE - 1) / TILE;
  const int grid = std::min(tiles, 4 * num_sms(m->device));
  k_forward<<<grid, TILE, smem, m->st>>>(net_of(m), dx, n, dy, m->err);
  MLP_CU(m, cudaGetLastError());
  return check_err(m);
}

// Gradient of the mean squared error over n samples (device arrays), into m->grad
// (added to what is there) and m->loss (sum of squared errors, added).
rw_status grad_dev(rw_mlp* m, const float* dx, const float* dt, long long n_all, long long first, int n,
                   long long sa, long long sc, float inv_count) {
  if (n <= 0) return RW_OK;
  const int smem = (int)sizeof(TrainSmem);
  MLP_CU(m, cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int tiles = (n + TILE - 1) / TILE;
  const int grid = std::min(tiles, num_sms(m->device));
  k_train<<<grid, TILE, smem, m->st>>>(net_of(m), dx, dt, n_all, first, n, sa, sc, inv_count, m->grad, m->loss,
                                       m->err);
  MLP_CU(m, cudaGetLastError());
  return RW_OK;
}

template <class F>
rw_status guarded_mlp(rw_mlp* m, F&& f) {
  if (!m) return fail(nullptr, RW_EINVAL, "null network");
  std::lock_guard<std::mutex> lk(m->mu);
  if (cudaSetDevice(m->device) != cudaSuccess) return fail(m, RW_ECUDA, "cudaSetDevice failed");
  try {
    return f();
  } catch (const std::bad_alloc&) {
    return fail(m, RW_ENOMEM, "host allocation failed");
  }
}

}  // namespace

extern "C" {

const char* rw_mlp_last_error(rw_mlp* m) { return m ? m->msg.c_str() : g_mlp_err.c_str(); }

rw_status rw_mlp_create(int device, uint64_t seed, int64_t sample_capacity, rw_mlp** out) {
  if (!out || sample_capacity < 0) return fail(nullptr, RW_EINVAL, "rw_mlp_create: bad arguments");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return fail(nullptr, RW_EDEVICE, "rw_mlp_create: no such CUDA device");
  rw_mlp* m = new rw_mlp();
  m->device = device;
  auto bad = [&](rw_status s) {
    rw_mlp_destroy(m);
    return s;
  };
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess)
    return bad(fail(nullptr, RW_ECUDA, "rw_mlp_create: stream"));
  bool ok = cudaMalloc(&m->params, NPARAM * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->grad, NPARAM * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->m, NPARAM * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->v, NPARAM * sizeof(float)) == cudaSuccess && cudaMalloc(&m->fw, FWBYTES) == cudaSuccess &&
            cudaMalloc(&m->bw, BWBYTES) == cudaSuccess &&
            cudaMalloc(&m->bias, NBIAS * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->err, sizeof(int)) == cudaSuccess && cudaMalloc(&m->loss, sizeof(double)) == cudaSuccess &&
            cudaMalloc(&m->ranges, (2 * IN + 1) * sizeof(unsigned)) == cudaSuccess;
  if (ok && sample_capacity > 0)
    ok = cudaMalloc(&m->sx, (size_t)sample_capacity * IN * sizeof(float)) == cudaSuccess &&
         cudaMalloc(&m->stg, (size_t)sample_capacity * OUT * sizeof(float)) == cudaSuccess;
  if (!ok) return bad(fail(nullptr, RW_ENOMEM, "rw_mlp_create: device allocation failed"));
  m->cap = sample_capacity;
  cudaMemsetAsync(m->grad, 0, NPARAM * sizeof(float), m->st);
  cudaMemsetAsync(m->m, 0, NPARAM * sizeof(float), m->st);
  cudaMemsetAsync(m->v, 0, NPARAM * sizeof(float), m->st);
  cudaMemsetAsync(m->fw, 0, FWBYTES, m->st);
  cudaMemsetAsync(m->bw, 0, BWBYTES, m->st);
  cudaMemsetAsync(m->bias, 0, NBIAS * sizeof(float), m->st);
  cudaMemsetAsync(m->err, 0, sizeof(int), m->st);
  // Xavier-uniform weights, zero biases.
  std::vector<float> p(NPARAM, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_in, int fan_out) {
    const double a = std::sqrt(6.0 / (fan_in + fan_out));
    std::uniform_real_distribution<double> U(-a, a);
    for (int k = 0; k < fan_in * fan_out; ++k) p[off + k] = (float)U(rng);
  };
  fill(P_W1, IN, HID);
  fill(P_W2, HID, HID);
  fill(P_W3, HID, HID);
  fill(P_W4, HID, HID);
  fill(P_W5, HID, OUT);
  if (cudaMemcpyAsync(m->params, p.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice, m->st) != cudaSuccess)
    return bad(fail(nullptr, RW_ECUDA, "rw_mlp_create: upload"));
  if (pack_all(m) != RW_OK || cudaStreamSynchronize(m->st) != cudaSuccess)
    return bad(fail(nullptr, RW_ECUDA, "rw_mlp_create: pack"));
  *out = m;
  return RW_OK;
}

rw_status rw_mlp_destroy(rw_mlp* m) {
  if (!m) return RW_OK;
  cudaSetDevice(m->device);
  if (m->st) cudaStreamSynchronize(m->st);
  for (void* p : {(void*)m->params, (void*)m->grad, (void*)m->m, (void*)m->v, (void*)m->fw, (void*)m->bw,
                  (void*)m->bias, (void*)m->err, (void*)m->loss, (void*)m->ranges, (void*)m->sx, (void*)m->stg})
    if (p) cudaFree(p);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
  return RW_OK;
}

rw_status rw_mlp_get_params(rw_mlp* m, float* out, size_t n) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (!out || n != (size_t)NPARAM) return fail(m, RW_EINVAL, "rw_mlp_get_params: expected RW_MLP_NPARAM floats");
    MLP_CU(m, cudaMemcpyAsync(out, m->params, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MLP_CU(m, cudaStreamSynchronize(m->st));
    return RW_OK;
  });
}

rw_status rw_mlp_set_params(rw_mlp* m, const float* in, size_t n) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (!in || n != (size_t)NPARAM) return fail(m, RW_EINVAL, "rw_mlp_set_params: expected RW_MLP_NPARAM floats");
    MLP_CU(m, cudaMemcpyAsync(m->params, in, NPARAM * sizeof(float), cudaMemcpyHostToDevice, m->st));
    MLP_CU(m, cudaMemsetAsync(m->m, 0, NPARAM * sizeof(float), m->st));
    MLP_CU(m, cudaMemsetAsync(m->v, 0, NPARAM * sizeof(float), m->st));
    m->adam_t = 0;
    rw_status s = pack_all(m);
    if (s != RW_OK) return s;
    MLP_CU(m, cudaStreamSynchronize(m->st));
    return RW_OK;
  });
}

rw_status rw_mlp_forward(rw_mlp* m, const float* x, int64_t n, float* y) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (n < 0 || n > (1LL << 30) || (n > 0 && (!x || !y))) return fail(m, RW_EINVAL, "rw_mlp_forward: bad arguments");
    if (n == 0) return RW_OK;
    float *dx = nullptr, *dy = nullptr;
    MLP_CU(m, cudaMallocAsync((void**)&dx, (size_t)n * IN * sizeof(float), m->st));
    MLP_CU(m, cudaMallocAsync((void**)&dy, (size_t)n * OUT * sizeof(float), m->st));
    MLP_CU(m, cudaMemcpyAsync(dx, x, (size_t)n * IN * sizeof(float), cudaMemcpyHostToDevice, m->st));
    rw_status s = forward_dev(m, dx, (int)n, dy);
    if (s == RW_OK) {
      MLP_CU(m, cudaMemcpyAsync(y, dy, (size_t)n * OUT * sizeof(float), cudaMemcpyDeviceToHost, m->st));
      MLP_CU(m, cudaStreamSynchronize(m->st));
    }
    cudaFreeAsync(dx, m->st);
    cudaFreeAsync(dy, m->st);
    cudaStreamSynchronize(m->st);
    return s;
  });
}

rw_status rw_mlp_grad(rw_mlp* m, const float* x, const float* t, int64_t n, double* loss, float* grad) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (n <= 0 || n > (1LL << 30) || !x || !t || !grad) return fail(m, RW_EINVAL, "rw_mlp_grad: bad arguments");
    float *dx = nullptr, *dt = nullptr;
    MLP_CU(m, cudaMallocAsync((void**)&dx, (size_t)n * IN * sizeof(float), m->st));
    MLP_CU(m, cudaMallocAsync((void**)&dt, (size_t)n * OUT * sizeof(float), m->st));
    MLP_CU(m, cudaMemcpyAsync(dx, x, (size_t)n * IN * sizeof(float), cudaMemcpyHostToDevice, m->st));
    MLP_CU(m, cudaMemcpyAsync(dt, t, (size_t)n * OUT * sizeof(float), cudaMemcpyHostToDevice, m->st));
    MLP_CU(m, cudaMemsetAsync(m->grad, 0, NPARAM * sizeof(float), m->st));
    MLP_CU(m, cudaMemsetAsync(m->loss, 0, sizeof(double), m->st));
    // identity order: a = 1, c = 0
    rw_status s = grad_dev(m, dx, dt, n, 0, (int)n, 1, 0, 1.0f / (float)(n * OUT));
    if (s == RW_OK) s = check_err(m);
    if (s == RW_OK) {
      double l = 0.0;
      MLP_CU(m, cudaMemcpyAsync(grad, m->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->st));
      MLP_CU(m, cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st));
      MLP_CU(m, cudaMemsetAsync(m->grad, 0, NPARAM * sizeof(float), m->st));
      MLP_CU(m, cudaStreamSynchronize(m->st));
      if (loss) *loss = l / (double)(n * OUT);
    }
    cudaFreeAsync(dx, m->st);
    cudaFreeAsync(dt, m->st);
    cudaStreamSynchronize(m->st);
    return s;
  });
}

rw_status rw_mlp_add_samples(rw_mlp* m, const float* x, const float* t, int64_t n) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (n < 0 || (n > 0 && (!x || !t))) return fail(m, RW_EINVAL, "rw_mlp_add_samples: bad arguments");
    if (m->n + n > m->cap) return fail(m, RW_ENOMEM, "rw_mlp_add_samples: sample capacity exceeded");
    MLP_CU(m, cudaMemcpyAsync(m->sx + m->n * IN, x, (size_t)n * IN * sizeof(float), cudaMemcpyHostToDevice, m->st));
    MLP_CU(m, cudaMemcpyAsync(m->stg + m->n * OUT, t, (size_t)n * OUT * sizeof(float), cudaMemcpyHostToDevice, m->st));
    MLP_CU(m, cudaStreamSynchronize(m->st));
    m->n += n;
    return RW_OK;
  });
}

rw_status rw_mlp_samples(rw_mlp* m, int64_t* count, float* x, float* t, int64_t n) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (count) *count = m->n;
    if (n <= 0) return RW_OK;
    if (n > m->n || !x || !t) return fail(m, RW_EINVAL, "rw_mlp_samples: bad arguments");
    MLP_CU(m, cudaMemcpyAsync(x, m->sx, (size_t)n * IN * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MLP_CU(m, cudaMemcpyAsync(t, m->stg, (size_t)n * OUT * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MLP_CU(m, cudaStreamSynchronize(m->st));
    return RW_OK;
  });
}

rw_status rw_mlp_clear_samples(rw_mlp* m) {
  return guarded_mlp(m, [&]() -> rw_status {
    m->n = 0;
    return RW_OK;
  });
}

rw_status rw_mlp_train(rw_mlp* m, int epochs, int batch, float lr, uint64_t seed, double* last_loss) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (epochs < 0 || batch < TILE || !(lr > 0.0f)) return fail(m, RW_EINVAL, "rw_mlp_train: bad arguments");
    if (m->n < batch) return fail(m, RW_ESTATE, "rw_mlp_train: fewer samples than one minibatch");
    const long long n = m->n;
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    double lsum_epoch = 0.0;
    long long nb = 0;
    const long long total = (long long)epochs * (n / batch);
    long long step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
      long long a;  // multiplier coprime to n: a shuffled order of the samples per epoch
      do {
        a = (long long)(rng() % (uint64_t)n) | 1;
      } while (std::gcd(a, n) != 1);
      const long long c = (long long)(rng() % (uint64_t)n);
      MLP_CU(m, cudaMemsetAsync(m->loss, 0, sizeof(double), m->st));
      nb = 0;
      for (long long first = 0; first + batch <= n; first += batch, ++nb) {
        rw_status s = grad_dev(m, m->sx, m->stg, n, first, batch, a, c, 1.0f / (float)(batch * OUT));
        if (s != RW_OK) return s;
        ++m->adam_t;
        const float bc1 = 1.0f - std::pow(b1, (float)m->adam_t), bc2 = 1.0f - std::pow(b2, (float)m->adam_t);
        // cosine decay from lr to lr / 20 over the call
        const double frac = total > 1 ? (double)step / (double)(total - 1) : 1.0;
        const float lr_t = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * frac))));
        ++step;
        k_adam<<<(NPARAM + 255) / 256, 256, 0, m->st>>>(m->params, m->grad, m->m, m->v, lr_t, b1, b2, eps, bc1, bc2,
                                                        m->fw, m->bw, m->bias);
        MLP_CU(m, cudaGetLastError());
      }
      rw_status s = check_err(m);
      if (s != RW_OK) return s;
      MLP_CU(m, cudaMemcpyAsync(&lsum_epoch, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st));
      MLP_CU(m, cudaStreamSynchronize(m->st));
    }
    if (last_loss) *last_loss = nb > 0 ? lsum_epoch / (double)(nb * batch * OUT) : 0.0;
    return RW_OK;
  });
}

rw_status rw_mlp_feature_ranges(rw_mlp* m, float* lo, float* hi, float* tmax) {
  return guarded_mlp(m, [&]() -> rw_status {
    if (!lo || !hi || !tmax) return fail(m, RW_EINVAL, "rw_mlp_feature_ranges: null output");
    if (m->n <= 0) return fail(m, RW_ESTATE, "rw_mlp_feature_ranges: no samples");
    std::vector<unsigned> init(2 * IN + 1, 0u);
    for (int k = 0; k < IN; ++k) init[k] = 0xFFFFFFFFu;
    MLP_CU(m, cudaMemcpyAsync(m->ranges, init.data(), init.size() * sizeof(unsigned), cudaMemcpyHostToDevice, m->st));
    k_ranges<<<4 * num_sms(m->device), 256, 0, m->st>>>(m->sx, m->stg, m->n, m->ranges, m->ranges + IN,
                                                         m->ranges + 2 * IN);
    MLP_CU(m, cudaGetLastError());
    std::vector<unsigned> r(2 * IN + 1);
    MLP_CU(m, cudaMemcpyAsync(r.data(), m->ranges, r.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, m->st));
    MLP_CU(m, cudaStreamSynchronize(m->st));
    auto back = [](unsigned u) {
      const unsigned b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
      float f;
      std::memcpy(&f, &b, 4);
      return f;
    };
    for (int k = 0; k < IN; ++k) {
      lo[k] = back(r[k]);
      hi[k] = back(r[IN + k]);
    }
    std::memcpy(tmax, &r[2 * IN], 4);
    return RW_OK;
  });
}

}  // extern "C"

// Access for the engine (closure inference, sample collection).
namespace rw {
namespace mlp {
Net net_view(const rw_mlp* m) { return net_of(m); }
int device_of(const rw_mlp* m) { return m->device; }
long long free_slots(const rw_mlp* m) { return m->cap - m->n; }
void next_slot(rw_mlp* m, float** x, float** t) {
  *x = m->sx + m->n * IN;
  *t = m->stg + m->n * OUT;
}
void commit(rw_mlp* m, long long n) { m->n += std::min(n, m->cap - m->n); }
}  // namespace mlp
}  // namespace rw
