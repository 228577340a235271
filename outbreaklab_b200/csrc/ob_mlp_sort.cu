// ob_mlp_sort.cu — a canonical order for the recorded (state, tendency) pairs of the microphysics surrogate (sm_100a).
//
// The physics pass appends the pairs it samples with an atomic counter, so the pairs of one step land in an order
// that changes from run to run, and with it every training batch drawn by index. Each pair carries the model time of
// its step (pair float 23) and its texel offset (float 22, as bits): the two together are unique within one model's
// recording. ob_mlp_sort_pairs orders the buffer by (time, offset) with a stable least-significant-digit radix sort on
// the device (8-bit digits of a 64-bit key: the time's float bits above the offset), then gathers the 96-byte pairs
// into the new order. With it a run's recording, and so its trained network, no longer depends on the append order.
// A recording that ran past the buffer's capacity kept an arbitrary subset of its last step's pairs (those whose
// appends won the race); after the sort these are the tail of the buffer, and the sort drops them by setting the
// append counter to the first pair of that step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/ob.h"
#include "ob_mlp.cuh"

namespace ob {
void set_error(const char* fmt, ...);

namespace mlp {
namespace {
constexpr int RS_THREADS = 256, RS_ITEMS = 16, RS_CHUNK = RS_THREADS * RS_ITEMS;  // keys per block per pass

__global__ void k_make_keys(const float* __restrict__ pairs, long n, unsigned long long* __restrict__ key, unsigned* __restrict__ val) {
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
    const float* p = pairs + i * PAIR;
    key[i] = (static_cast<unsigned long long>(__float_as_uint(p[23])) << 32) | __float_as_uint(p[22]);
    val[i] = unsigned(i);
  }
}

// counts[d * nb + b] = keys of block b's chunk whose digit is d
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const unsigned long long* __restrict__ key, long n, int shift, int nb,
                                                         unsigned* __restrict__ counts) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long b0 = long(blockIdx.x) * RS_CHUNK;
  for (int i = threadIdx.x; i < RS_CHUNK; i += RS_THREADS) {
    const long j = b0 + i;
    if (j < n) atomicAdd(&h[unsigned(key[j] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[long(threadIdx.x) * nb + blockIdx.x] = h[threadIdx.x];
}

// per digit (one block each): exclusive scan of its nb block counts in place, and the digit's total
__global__ void __launch_bounds__(1024) k_rs_scan_digit(unsigned* __restrict__ counts, int nb, unsigned* __restrict__ total) {
  __shared__ unsigned s[1024];
  __shared__ unsigned carry;
  unsigned* c = counts + long(blockIdx.x) * nb;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const unsigned v = i < nb ? c[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {   // inclusive scan (Hillis-Steele)
      const unsigned t = threadIdx.x >= unsigned(o) ? s[threadIdx.x - o] : 0u;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) c[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) total[blockIdx.x] = carry;
}

// digit bases: exclusive scan of the 256 totals (one thread, in order)
__global__ void k_rs_scan_base(const unsigned* __restrict__ total, unsigned* __restrict__ base) {
  unsigned acc = 0;
  for (int d = 0; d < 256; d++) {
    base[d] = acc;
    acc += total[d];
  }
}

// stable scatter of block b's chunk: RS_ITEMS rounds of RS_THREADS consecutive keys; within a round a key's place
// among equal digits is (earlier rounds) + (earlier warps) + (earlier lanes of its warp)
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const unsigned long long* __restrict__ key_in, const unsigned* __restrict__ val_in,
                                                           long n, int shift, int nb, const unsigned* __restrict__ counts,
                                                           const unsigned* __restrict__ base, unsigned long long* __restrict__ key_out,
                                                           unsigned* __restrict__ val_out) {
  constexpr int NW = RS_THREADS / 32;
  __shared__ unsigned wcnt[NW][256];
  __shared__ unsigned run[256], off[256], rtot[256];
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  run[t] = 0;
  off[t] = base[t] + counts[long(t) * nb + blockIdx.x];
  const long b0 = long(blockIdx.x) * RS_CHUNK;
  for (int r = 0; r < RS_ITEMS; r++) {
#pragma unroll
    for (int q = 0; q < NW; q++) wcnt[q][t] = 0;
    __syncthreads();
    const long j = b0 + long(r) * RS_THREADS + t;
    const bool valid = j < n;
    const unsigned long long k = valid ? key_in[j] : 0ull;
    const unsigned d = valid ? unsigned(k >> shift) & 255u : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned below = __popc(peers & ((1u << lane) - 1u));
    if (valid && below == 0) wcnt[w][d] = __popc(peers);
    __syncthreads();
    {  // thread t: exclusive scan of digit t's counts over the warps, and the round's total
      unsigned acc = 0;
#pragma unroll
      for (int q = 0; q < NW; q++) {
        const unsigned c = wcnt[q][t];
        wcnt[q][t] = acc;
        acc += c;
      }
      rtot[t] = acc;
    }
    __syncthreads();
    if (valid) {
      const unsigned pos = off[d] + run[d] + wcnt[w][d] + below;
      key_out[pos] = k;
      val_out[pos] = val_in[j];
    }
    __syncthreads();
    run[t] += rtot[t];
    __syncthreads();
  }
}

__global__ void k_gather_pairs(const float4* __restrict__ src, const unsigned* __restrict__ order, long n, float4* __restrict__ dst) {
  constexpr int V = PAIR / 4;   // float4 per pair
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n * V; i += long(gridDim.x) * blockDim.x) {
    const long p = i / V;
    dst[i] = src[long(order[p]) * V + (i - p * V)];
  }
}
// count[0] = index of the first pair whose model time is the last pair's (the pairs are in time order)
__global__ void k_first_of_last_step(const float* __restrict__ pairs, long n, unsigned* __restrict__ count) {
  const unsigned last = __float_as_uint(pairs[(n - 1) * PAIR + 23]);
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    if (__float_as_uint(pairs[i * PAIR + 23]) == last && (i == 0 || __float_as_uint(pairs[(i - 1) * PAIR + 23]) != last))
      count[0] = unsigned(i);
}
}  // namespace

// sorts `n` pairs in place (`pairs` holds at least n * PAIR floats); with `overflowed` (the append counter passed the
// capacity) it then drops the last step's pairs by setting count[0] to the first of them. Allocates its scratch for
// the call.
int sort_pairs(float* pairs, long n, bool overflowed, unsigned* count, cudaStream_t s) {
  if (n <= 1) return OB_OK;
  const int nb = int((n + RS_CHUNK - 1) / RS_CHUNK);
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  unsigned *v0 = nullptr, *v1 = nullptr, *counts = nullptr, *tot = nullptr;
  float* tmp = nullptr;
  bool ok = cudaMalloc(&k0, size_t(n) * 8) == cudaSuccess && cudaMalloc(&k1, size_t(n) * 8) == cudaSuccess &&
            cudaMalloc(&v0, size_t(n) * 4) == cudaSuccess && cudaMalloc(&v1, size_t(n) * 4) == cudaSuccess &&
            cudaMalloc(&counts, size_t(nb) * 256 * 4) == cudaSuccess && cudaMalloc(&tot, 512 * 4) == cudaSuccess &&
            cudaMalloc(&tmp, size_t(n) * PAIR * 4) == cudaSuccess;
  int rc = OB_OK;
  if (!ok) {
    set_error("ob_mlp_sort_pairs: out of device memory for the sort's scratch");
    rc = OB_ERR_OOM;
  } else {
    k_make_keys<<<1184, 256, 0, s>>>(pairs, n, k0, v0);
    for (int pass = 0; pass < 8; pass++) {
      k_rs_hist<<<nb, RS_THREADS, 0, s>>>(k0, n, 8 * pass, nb, counts);
      k_rs_scan_digit<<<256, 1024, 0, s>>>(counts, nb, tot);
      k_rs_scan_base<<<1, 1, 0, s>>>(tot, tot + 256);
      k_rs_scatter<<<nb, RS_THREADS, 0, s>>>(k0, v0, n, 8 * pass, nb, counts, tot + 256, k1, v1);
      std::swap(k0, k1);
      std::swap(v0, v1);
    }
    k_gather_pairs<<<2368, 256, 0, s>>>(reinterpret_cast<const float4*>(pairs), v0, n, reinterpret_cast<float4*>(tmp));
    const cudaError_t e1 = cudaMemcpyAsync(pairs, tmp, size_t(n) * PAIR * 4, cudaMemcpyDeviceToDevice, s);
    if (overflowed && e1 == cudaSuccess) k_first_of_last_step<<<1184, 256, 0, s>>>(pairs, n, count);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
      set_error("ob_mlp_sort_pairs: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
      rc = OB_ERR_DEVICE;
    }
  }
  for (void* p : {(void*)k0, (void*)k1, (void*)v0, (void*)v1, (void*)counts, (void*)tot, (void*)tmp})
    if (p) cudaFree(p);
  return rc;
}

}  // namespace mlp
}  // namespace ob
