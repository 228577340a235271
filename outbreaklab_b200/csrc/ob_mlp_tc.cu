// ob_mlp_tc.cu — the microphysics surrogate inside the model step (sm_100a): a persistent tcgen05 kernel that runs
// the 12 -> 3 x 128 GELU -> 10 MLP on the cells the physics pass queued (those holding a hydrometeor), applies its
// process tendencies with positivity and total-water conservation enforced, closes with the scheme's saturation
// adjustment (thermodynamic equilibrium, not a process rate), and falls back to the whole scheme (micro_plain) for
// cells whose inputs lie outside the training range.
//
// One CTA per SM, 256 threads in two independent groups of 4 warps; each group takes tiles of 128 queued cells (one
// cell per thread = one TMEM lane) and runs the four layers as tcgen05.mma (M = 128 cells, BF16 operands, FP32
// accumulation in TMEM): the thread writes its cell's bf16 activations into a 128-byte-swizzled K-major tile in
// shared memory, one elected thread issues the MMAs against the weights (loaded once per CTA, 84 KB, the same
// swizzled layout), and the group reads the accumulator back with tcgen05.ld, adds the bias and applies GELU (tanh
// form with the hardware tanh approximation) for the next layer. While one group computes GELUs the other group's
// MMAs run. Every mbarrier wait is bounded (ob_tc.cuh).
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ob.h"
#include "ob_common.cuh"
#include "ob_micro.cuh"
#include "ob_mlp.cuh"
#include "ob_step.cuh"
#include "ob_tc.cuh"

namespace ob {
void set_error(const char* fmt, ...);

namespace mlp {

// shared-memory image of the weights (B operands, K-major, 128-byte swizzle, 1024-byte aligned tiles of 64 K-columns)
constexpr int W1_BYTES = NH * 128;        // 128 rows x 64 K (12 used)
constexpr int W2_BYTES = 2 * NH * 128;    // 128 rows x 128 K
constexpr int W4_ROWS = 16;               // 10 outputs padded to the MMA's N = 16
constexpr int W4_BYTES = 2 * W4_ROWS * 128;
constexpr int OFF_W1 = 0, OFF_W2 = OFF_W1 + W1_BYTES, OFF_W3 = OFF_W2 + W2_BYTES, OFF_W4 = OFF_W3 + W2_BYTES;
constexpr int WIMG_BYTES = OFF_W4 + W4_BYTES;  // 86016
constexpr int ACT_BYTES = 2 * 128 * 128;       // one group's activation tile: 128 cells x 128 K bf16
constexpr int SMEM_INFER = WIMG_BYTES + 2 * ACT_BYTES + 1024 + 64;
constexpr int NBIAS = 3 * NH + W4_ROWS;
constexpr float kNewSpeciesFloor = 1e-8f;  // kg/kg per step: gains of an empty species below this are noise

// byte offset of element (row r, column k) in a K-major 128-byte-swizzled operand of `rows` rows (64 columns per
// tile): rows of 128 bytes, the 16-byte chunk index XORed with the row index mod 8 (the layout TMA writes)
__host__ __device__ inline int swz(int r, int k, int rows) {
  return (k >> 6) * rows * 128 + r * 128 + ((((k & 63) >> 3) ^ (r & 7)) << 4) + ((k & 7) << 1);
}

struct Infer {
  const uint4* wimg;  // WIMG_BYTES
  const float* bias;  // b1, b2, b3 (NH each), b4 padded to 16
};

__device__ __forceinline__ float gelu_fast(float z) {
  float t;
  const float u = 0.7978845608f * (z + 0.044715f * z * z * z);
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return 0.5f * z * (1.f + t);
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void group_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// 32 lanes x 16 columns of fp32 from TMEM
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// bias + GELU of one accumulator row (this thread's cell) into the next layer's bf16 activation tile
__device__ __forceinline__ void hidden_to_smem(uint32_t tacc, const float* __restrict__ bias, uint8_t* act, int row) {
#pragma unroll 1
  for (int ch = 0; ch < NH / 32; ch++) {
    float v[32];
    tc::tmem_ld32(tacc + uint32_t(ch * 32), v);
#pragma unroll
    for (int c8 = 0; c8 < 4; c8++) {
      __align__(16) __nv_bfloat16 h[8];
#pragma unroll
      for (int e = 0; e < 8; e++) h[e] = __float2bfloat16_rn(gelu_fast(v[c8 * 8 + e] + __ldg(bias + ch * 32 + c8 * 8 + e)));
      *reinterpret_cast<uint4*>(act + swz(row, ch * 32 + c8 * 8, 128)) = *reinterpret_cast<const uint4*>(h);
    }
  }
}

// issue one layer: D[128 x N] = A[128 x K] W[N x K]^T with K in steps of 16
__device__ __forceinline__ void issue_layer(uint32_t tacc, uint32_t a_base, uint32_t w_base, int krows_w, int K, int N, uint64_t* bar) {
  const uint32_t idesc = tc::idesc_bf16_f32(128, N);
  for (int k = 0; k < K; k += 16) {
    const uint32_t ao = uint32_t((k >> 6) * 128 * 128 + ((k & 63) >> 3) * 16);
    const uint32_t wo = uint32_t((k >> 6) * krows_w * 128 + ((k & 63) >> 3) * 16);
    tc::mma_bf16(tacc, tc::desc_k_sw128(a_base + ao), tc::desc_k_sw128(w_base + wo), idesc, k > 0 ? 1u : 0u);
  }
  tc::mma_commit(bar);
}

// The inference of the queued cells of one model, or of several (an ensemble's grouped step: the members' queues are
// taken one after another, their tiles dealt round-robin to the CTAs' two groups as one sequence).
template <bool GROUP>
__device__ __forceinline__ void surrogate_run(const MemberC* __restrict__ members, int nmem, const Grid& g0, const Uni& U0,
                                              const Fields& F0, int par, const Infer& net, const Norm& nm, unsigned int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* wimg = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + WIMG_BYTES + 2 * ACT_BYTES);  // [2] one per group
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  const int tid = threadIdx.x, grp = tid >> 7, row = tid & 127, warp = tid >> 5;
  uint8_t* act = smem + WIMG_BYTES + grp * ACT_BYTES;

  for (int i = tid; i < WIMG_BYTES / 16; i += blockDim.x) reinterpret_cast<uint4*>(wimg)[i] = __ldg(net.wimg + i);
  if (tid == 0) {
    tc::mbar_init(&bars[0], 1);
    tc::mbar_init(&bars[1], 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, 512);
    tc::tmem_relinquish();
  }
  fence_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  // group g owns TMEM columns [256 g, 256 g + 256): the hidden accumulator at +0, the output at +128; warp w reads
  // lanes 32 (w % 4) .. +31, which holds this thread's row
  const uint32_t thid = *tmem_slot + uint32_t(grp * 256), tout = thid + 128;
  const uint32_t tbase = thid + (uint32_t((warp & 3) * 32) << 16);
  const uint32_t a_s = tc::smem_u32(act), w_s = tc::smem_u32(wimg);
  uint32_t phase = 0;
  // a timed-out wait marks this thread failed: it stops waiting and writing but keeps every group barrier, so the
  // kernel still ends (the host reads the error word)
  bool failed = false;
  const int start = blockIdx.x * 2 + grp, stride = gridDim.x * 2;
  int base = 0;
  for (int mi = 0; mi < (GROUP ? nmem : 1); mi++) {
    const Grid& g = GROUP ? members[mi].g : g0;
    const Uni& U = GROUP ? members[mi].U : U0;
    const Fields& F = GROUP ? members[mi].F : F0;
    const unsigned count = min(*F.mlp_count, F.mlp_cap);
    const unsigned* list = reinterpret_cast<const unsigned*>(F.mlp_buf);
    const float dt = U.step.x, tscale = nm.dt > 0.f ? dt / nm.dt : 1.f;
    const int ntiles = int((count + 127) / 128);
    int t0 = start;
    if (t0 < base) t0 += (base - t0 + stride - 1) / stride * stride;
    for (int tt = t0; tt < base + ntiles; tt += stride) {
      const int t = tt - base;
      const unsigned ci = unsigned(t) * 128u + unsigned(row);
      const bool valid = ci < count;
      const int o = valid ? int(list[ci]) : 0;
      const int k = o / g.plane, rem = o - k * g.plane, j = rem / g.px, i = rem - j * g.px;
      const float4 A = bsA(F.B, g.nz, k), Bb = bsB(F.B, g.nz, k);
      const float pi0 = Bb.x, p0 = Bb.y, rho = A.z;
      MCell m{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float ni = 0.f, w = 0.f;
      if (valid) {
        m.T = F.V[par][3][o] * pi0;
        m.qv = F.Q[0][0][o]; m.qc = F.Q[0][1][o]; m.qi = F.Q[0][2][o]; m.qr = F.Q[0][3][o];
        m.qs = F.Q[0][4][o]; m.qg = F.Q[0][5][o]; m.nr = F.Q[0][6][o];
        ni = F.Q[0][7][o];
        w = F.V[1 - par][2][o];
      }
      const float raw[NIN] = {m.T, p0, rho, m.qv, m.qc, m.qr, m.qi, m.qs, m.qg, m.nr, ni, w};
      bool inrange = true;
      __align__(16) __nv_bfloat16 xb[16];
  #pragma unroll
      for (int e = 0; e < NIN; e++) {
        inrange = inrange && raw[e] >= nm.in_lo[e] && raw[e] <= nm.in_hi[e];
        xb[e] = __float2bfloat16_rn((feature(e, raw[e]) - nm.in_mean[e]) * nm.in_scale[e]);
      }
  #pragma unroll
      for (int e = NIN; e < 16; e++) xb[e] = __float2bfloat16_rn(0.f);
      *reinterpret_cast<uint4*>(act + swz(row, 0, 128)) = *reinterpret_cast<const uint4*>(xb);
      *reinterpret_cast<uint4*>(act + swz(row, 8, 128)) = *reinterpret_cast<const uint4*>(xb + 8);
      // layers 1-3 into the hidden accumulator, layer 4 into the output accumulator
  #pragma unroll 1
      for (int layer = 0; layer < 4; layer++) {
        fence_async_smem();
        tc::tc_fence_before();
        group_sync(1 + grp);
        if (row == 0 && !failed) {
          tc::tc_fence_after();
          if (layer == 0) issue_layer(thid, a_s, w_s + OFF_W1, NH, 16, NH, &bars[grp]);
          else if (layer < 3) issue_layer(thid, a_s, w_s + (layer == 1 ? OFF_W2 : OFF_W3), NH, NH, NH, &bars[grp]);
          else issue_layer(tout, a_s, w_s + OFF_W4, W4_ROWS, NH, W4_ROWS, &bars[grp]);
        }
        if (!failed) failed = !tc::mbar_wait(&bars[grp], phase, err, 16u);
        phase ^= 1u;
        tc::tc_fence_after();
        if (layer < 3) hidden_to_smem(tbase, net.bias + layer * NH, act, row);
      }
      float y[16];
      tmem_ld16(tbase + 128, y);
      if (!valid || failed) continue;
      const float rs = __ldg(F.spz + 4 * k + 2);
      const float sl = fmaxf(__ldg(F.slx + 2 * i + 1), __ldg(F.sly + 2 * j + 1));
      bool finite = true;
  #pragma unroll
      for (int e = 0; e < NLOSS; e++) finite = finite && isfinite(y[e]);
      if (inrange && finite) {
        float d[NLOSS];
  #pragma unroll
        for (int e = 0; e < NLOSS; e++) d[e] = (y[e] + __ldg(net.bias + 3 * NH + e)) * nm.out_scale[e] * tscale;
        // no species appears from below the network's noise floor; no species loses more than it holds; the six
        // water tendencies sum to zero (total water), by shrinking whichever side, gains or losses, is larger
        float q[6] = {m.qv, m.qc, m.qi, m.qr, m.qs, m.qg};
        float gain = 0.f, loss = 0.f;
  #pragma unroll
        for (int s = 0; s < 6; s++) {
          if (q[s] == 0.f && d[1 + s] < kNewSpeciesFloor) d[1 + s] = 0.f;
          d[1 + s] = fmaxf(d[1 + s], -q[s]);
          if (d[1 + s] > 0.f) gain += d[1 + s]; else loss -= d[1 + s];
        }
        const float fg = gain > loss ? loss / gain : 1.f, fl = loss > gain ? gain / loss : 1.f;
  #pragma unroll
        for (int s = 0; s < 6; s++) q[s] += d[1 + s] * (d[1 + s] > 0.f ? fg : fl);
        m.qv = q[0]; m.qc = q[1]; m.qi = q[2]; m.qr = q[3]; m.qs = q[4]; m.qg = q[5];
        m.T += d[0];
        // the scheme's own bounds on the rain number (model.js:874-884): none without rain, else within the
        // mass-weighted limits
        const float nr = m.nr + d[7];
        m.nr = m.qr > 1e-9f ? clampf(nr, m.qr * 3.183e5f, m.qr * 3.183e11f) : 0.f;
        // the saturation adjustment is thermodynamic equilibrium, not a process rate: it runs as in the scheme
        sat_adjust(p0, m);
      } else {
        micro_plain(U, dt, p0, rho, rs, m);
        atomicAdd(F.mlp_count + 1, 1u);  // fallbacks of this step
      }
      const float keep = 1.f / (1.f + 2.f * dt * sl);
      float th = m.T / pi0;
      if (!(th == th)) {
        th = A.x;
        atomicAdd(F.flags, 1u);
      }
      F.V[par][3][o] = th;
      F.Q[0][0][o] = fmaxf(m.qv, 0.f);
      F.Q[0][1][o] = fmaxf(m.qc * keep, 0.f);
      F.Q[0][2][o] = fmaxf(m.qi * keep, 0.f);
      F.Q[0][3][o] = fmaxf(m.qr * keep, 0.f);
      F.Q[0][4][o] = fmaxf(m.qs * keep, 0.f);
      F.Q[0][5][o] = fmaxf(m.qg * keep, 0.f);
      F.Q[0][6][o] = fmaxf(m.nr * keep, 0.f);
  
    }
    base += ntiles;
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(*tmem_slot, 512);
  }
}

__global__ void __launch_bounds__(256, 1) k_surrogate(Grid g, Uni U, Fields F, int par, Infer net, Norm nm, unsigned int* err) {
  surrogate_run<false>(nullptr, 1, g, U, F, par, net, nm, err);
}
__global__ void __launch_bounds__(256, 1) k_surrogate_grp(const MemberC* __restrict__ members, int n, int par, Infer net, Norm nm,
                                                          unsigned int* err) {
  surrogate_run<true>(members, n, members[0].g, members[0].U, members[0].F, par, net, nm, err);
}

}  // namespace mlp

// ---------------------------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------------------------
const float* mlp_master(const ObMlp* n);
const mlp::Norm* mlp_norm(const ObMlp* n);

// the inference copy of a network: bf16 weights in the shared-memory image, fp32 biases and the normalisation
int surrogate_prepare(const ObMlp* net, void** d_image, mlp::Norm* norm) {
  using namespace mlp;
  std::vector<float> w(NPARAM);
  if (cudaMemcpy(w.data(), mlp_master(net), NPARAM * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("surrogate: reading the network failed");
    return OB_ERR_DEVICE;
  }
  std::vector<uint8_t> img(WIMG_BYTES + NBIAS * 4, 0);
  auto put = [&](int off, int rows, int r, int kcol, float v) {
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    std::memcpy(img.data() + off + swz(r, kcol, rows), &b, 2);
  };
  for (int r = 0; r < NH; r++)
    for (int k = 0; k < NIN; k++) put(OFF_W1, NH, r, k, w[OW1 + r * NIN + k]);
  for (int r = 0; r < NH; r++)
    for (int k = 0; k < NH; k++) {
      put(OFF_W2, NH, r, k, w[OW2 + r * NH + k]);
      put(OFF_W3, NH, r, k, w[OW3 + r * NH + k]);
    }
  for (int r = 0; r < NOUT; r++)
    for (int k = 0; k < NH; k++) put(OFF_W4, W4_ROWS, r, k, w[OW4 + r * NH + k]);
  float* bias = reinterpret_cast<float*>(img.data() + WIMG_BYTES);
  for (int i = 0; i < NH; i++) {
    bias[i] = w[OB1 + i];
    bias[NH + i] = w[OB2 + i];
    bias[2 * NH + i] = w[OB3 + i];
  }
  for (int i = 0; i < NOUT; i++) bias[3 * NH + i] = w[OB4 + i];
  if (!*d_image && cudaMalloc(d_image, img.size()) != cudaSuccess) {
    set_error("surrogate: out of device memory");
    return OB_ERR_OOM;
  }
  if (cudaMemcpy(*d_image, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("surrogate: upload failed");
    return OB_ERR_DEVICE;
  }
  *norm = *mlp_norm(net);
  return OB_OK;
}

void launch_surrogate(const Grid& g, const Uni& U, const Fields& F, int par, const void* d_image, const mlp::Norm& nm,
                      unsigned int* err, cudaStream_t s) {
  using namespace mlp;
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
    cudaFuncSetAttribute(k_surrogate, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_INFER);
  }
  Infer net{reinterpret_cast<const uint4*>(d_image), reinterpret_cast<const float*>(reinterpret_cast<const uint8_t*>(d_image) + WIMG_BYTES)};
  k_surrogate<<<nsm, 256, SMEM_INFER, s>>>(g, U, F, par, net, nm, err);
}

void launch_surrogate_grp(const MemberC* d_members, int n, int par, const void* d_image, const mlp::Norm& nm, unsigned int* err,
                          cudaStream_t s) {
  using namespace mlp;
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
    cudaFuncSetAttribute(k_surrogate_grp, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_INFER);
  }
  Infer net{reinterpret_cast<const uint4*>(d_image), reinterpret_cast<const float*>(reinterpret_cast<const uint8_t*>(d_image) + WIMG_BYTES)};
  k_surrogate_grp<<<nsm, 256, SMEM_INFER, s>>>(d_members, n, par, net, nm, err);
}

}  // namespace ob
