// Allocation-free variant of the cell-key sort (stable LSD radix sort of cell keys
// with the particle permutation), for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not available or not allowed: a
// host program whose device allocator belongs to another framework, a real-time or
// interrupt-driven loop that must not block in the allocator, or a plugin whose host
// forbids device allocations after start-up.  Such a caller owns its input and output
// buffers; this entry point brings its own scratch memory: a fixed array in the
// library's device image, reserved on every GPU that loads the library for as long as
// the process lives.
#include <mutex>

#include "../../include/retainwall.h"
#include "rw_kernels.cuh"

namespace {

constexpr int kMaxKeys = RW_NOALLOC_MAX_KEYS;
constexpr int kMaxTiles = (kMaxKeys + rw::RS_TILE - 1) / rw::RS_TILE;

// Scratch: ping-pong keys/values, per-tile digit counts, digit totals, sort flag:
// 2 x 2^20 + 256 x 512 + 257 ints = 8,913,924 bytes (8.9 MB, 8.5 MiB).
struct Scratch {
  int tk[kMaxKeys];
  int tv[kMaxKeys];
  int hist[256 * kMaxTiles];
  int dtot[256];
  int need;
};
static __device__ __align__(256) Scratch g_scratch;

// Device addresses of g_scratch, looked up once per device.  In host code the name
// g_scratch is a host-side stand-in, not a device address.
constexpr int kMaxDevices = 64;
static Scratch* g_addr[kMaxDevices];
static std::mutex g_mu;

int scratch_for_current_device(Scratch** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return RW_ECUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return RW_ECUDA;
    g_addr[dev] = (Scratch*)p;
  }
  *out = g_addr[dev];
  return RW_OK;
}

__global__ void k_fill_iota(int* v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

__global__ void k_set_flag(int* f) { *f = 1; }

}  // namespace

extern "C" rw_status rw_cell_sort_noalloc(const int32_t* d_keys, int32_t n, int32_t max_key, int32_t* d_sorted_keys,
                                          int32_t* d_perm, void* stream) {
  if (n < 0 || n > kMaxKeys || max_key < 0 || max_key >= (1 << 24)) return RW_EINVAL;
  if (n == 0) return RW_OK;
  if (!d_keys || !d_sorted_keys || !d_perm) return RW_EINVAL;
  Scratch* s = nullptr;
  int rc = scratch_for_current_device(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int bits = 1;
  while ((1 << bits) <= max_key) ++bits;
  const int passes = (bits + 7) / 8;
  const int ntiles = (n + rw::RS_TILE - 1) / rw::RS_TILE;
  // The permutation starts as the identity in the output buffer; the sort flag is
  // set because every call sorts (the array keeps the previous call's contents).
  k_fill_iota<<<(n + 255) / 256, 256, 0, st>>>(d_perm, n);
  k_set_flag<<<1, 1, 0, st>>>(&s->need);
  // Ping-pong between (sorted_keys, perm) and the scratch pair, arranged so the last
  // pass writes the caller's outputs; the first pass reads the caller's keys.
  const int* kin = d_keys;
  const int* vin = d_perm;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    int* ko = to_out ? d_sorted_keys : s->tk;
    int* vo = to_out ? d_perm : s->tv;
    if (p == 0 && to_out) {  // odd pass count (1 or 3): pass 0 writes the caller's outputs, so
                             // its values come from an identity in the scratch (not in place)
      k_fill_iota<<<(n + 255) / 256, 256, 0, st>>>(s->tv, n);
      vin = s->tv;
    }
    rw::k_rs_upsweep<<<ntiles, rw::RS_THREADS, 0, st>>>(kin, n, 8 * p, s->hist, ntiles, &s->need);
    rw::k_rs_scan<<<256, rw::RS_THREADS, 0, st>>>(s->hist, ntiles, s->dtot, &s->need);
    rw::k_rs_downsweep<<<ntiles, rw::RS_THREADS, 0, st>>>(kin, vin, ko, vo, n, 8 * p, s->hist, s->dtot, ntiles,
                                                         &s->need);
    kin = ko;
    vin = vo;
  }
  return cudaGetLastError() == cudaSuccess ? RW_OK : RW_ECUDA;
}
