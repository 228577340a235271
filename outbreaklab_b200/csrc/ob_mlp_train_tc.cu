// ob_mlp_train_tc.cu — training of the microphysics surrogate on the 5th-generation tensor cores (sm_100a):
// BF16 operands, FP32 accumulation in TMEM, the elementwise work fused into the GEMM epilogues, every batch
// reduction in a fixed order (a seed fixes the trained network).
//
// One training step on a batch of B samples (B a multiple of 128) is eight tile GEMMs of one kernel, k_mlp_gemm
// (C[M][N] = A[M][K] B[N][K]^T, both operands K-major bf16 in global memory, TMA-loaded with a 128-byte swizzle into a
// 4-stage ring; one thread issues tcgen05.mma (M = 128, N = 16 / 128 / 144, K = 16 per instruction) into a TMEM
// accumulator; four warps drain it with tcgen05.ld and run the epilogue of the GEMM's role):
//   forward, layers 1-3   Z = H W^T; epilogue: + bias, GELU -> H (bf16, sample-major for the next layer and
//                         feature-major for the weight gradient), GELU'(Z) (fp32, for the backward pass)
//   forward, layer 4      Y = H3 W4^T; epilogue: + bias, the loss of the 8 scheme tendencies (FP64 partial per tile)
//                         and dY = 2 (Y - T) / (B * 8) (bf16, both layouts)
//   backward, layers 3-1  dH = dZ W (W transposed, kept as its own bf16 image); epilogue: dZ = dH * GELU'(Z) (bf16,
//                         both layouts)
//   weight gradients      dW = dZ^T [H, 1]: M = 128 output features (10 for layer 4, zero-padded), N = the input
//                         features plus a row of ones (so the last column is the bias gradient), K = the batch,
//                         split over CTAs into partial slices that k_grad_reduce adds in split order
// then k_adam_img updates the fp32 master parameters (Adam) and rewrites the bf16 weight images both ways.
// Every mbarrier wait is bounded (ob_tc.cuh): a timed-out wait sets a bit in the error word the host checks.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ob.h"
#include "ob_mlp.cuh"
#include "ob_tc.cuh"

namespace ob {
void set_error(const char* fmt, ...);

namespace mlp {

constexpr int GBM = 128, GBK = 64, GSTAGES = 4, GNMAX = 144;  // tile rows, K per stage, ring depth, widest N
constexpr int GA_BYTES = GBM * GBK * 2;                        // 16 KB
constexpr int GB_BYTES = GNMAX * GBK * 2;                      // 18 KB (a multiple of 1024)
constexpr int GSTAGE = GA_BYTES + GB_BYTES;
constexpr int GSMEM = GSTAGES * GSTAGE + 1024 + 256;
constexpr int GTHREADS = 192;
constexpr int NHX = NH + 16;   // feature-major activations: 128 features, a row of ones, 15 zero rows (N = 144)
constexpr int NXX = 16;        // feature-major inputs: 12 features, a row of ones, 3 zero rows
constexpr int KPAD = 64;       // sample-major inputs and dY: K padded to one 64-wide stage
constexpr int WSPLIT_MAX = 16; // batch splits of a weight-gradient GEMM

enum GemmRole { R_HIDDEN = 0, R_OUT = 1, R_BACK = 2, R_WGRAD = 3 };

struct Epi {
  long B;                    // batch
  const float* bias;         // R_HIDDEN: NH biases; R_OUT: NOUT biases
  __nv_bfloat16* s_out;      // sample-major output [B][ld_s] (H, dY or dZ; may be null for R_BACK)
  int ld_s;
  __nv_bfloat16* t_out;      // feature-major output [features][B]
  float* G;                  // R_HIDDEN: GELU' written [B][NH]; R_BACK: read
  const float* T;            // R_OUT: targets [B][NLOSS]
  double* lossp;             // R_OUT: per-tile loss partial (sum of squares)
  float inv;                 // R_OUT: 2 / (B * NLOSS)
};

// one weight-gradient GEMM of the grouped launch: A = dZ^T (or dY^T) [128][B], B = [H, 1]^T [N][B]
struct WgradSet {
  CUtensorMap a[4];
  CUtensorMap b[4];
  int N[4];
  float* part[4];            // [split][128][N]
};

__device__ __forceinline__ void tmem_ld16x(uint32_t taddr, float (&v)[16]) {
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

__device__ __forceinline__ void store8(__nv_bfloat16* dst, const float* v) {
  __align__(16) __nv_bfloat16 h[8];
#pragma unroll
  for (int e = 0; e < 8; e++) h[e] = __float2bfloat16_rn(v[e]);
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(h);
}

// The accumulator of one 128 x N tile: TMA producer (warp 0), MMA issuer (warp 1), the epilogue warps (2-5) wait for
// it. Returns the TMEM address of the accumulator (lane 0, column 0) to every thread; ok = false after a timeout.
__device__ __forceinline__ uint32_t gemm_mainloop(const CUtensorMap* tA, const CUtensorMap* tB, int arow0, int kel0, int ktiles, int N,
                                                  uint8_t* sm, unsigned int* err, bool& ok) {
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + GSTAGES * GSTAGE);
  uint64_t* empty = full + GSTAGES;
  uint64_t* accf = empty + GSTAGES;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(accf + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < GSTAGES; s++) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(accf, 1);
    tc::fence_mbar_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(tslot, 256);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t bytes = uint32_t(GA_BYTES + N * GBK * 2);
  ok = true;
  if (warp == 0 && lane == 0) {
    tc::prefetch_tmap(tA);
    tc::prefetch_tmap(tB);
    for (int t = 0; t < ktiles; t++) {
      const int s = t % GSTAGES;
      const uint32_t ph = uint32_t(t / GSTAGES) & 1u;
      if (!tc::mbar_wait(&empty[s], ph ^ 1u, err, 1u)) break;
      tc::mbar_expect_tx(&full[s], bytes);
      uint8_t* st = sm + s * GSTAGE;
      tc::tma_load_2d(st, tA, &full[s], kel0 + t * GBK, arow0);
      tc::tma_load_2d(st + GA_BYTES, tB, &full[s], kel0 + t * GBK, 0);
    }
  } else if (warp == 1 && lane == 0) {
    const uint32_t idesc = tc::idesc_bf16_f32(GBM, N);
    bool good = true;
    for (int t = 0; t < ktiles && good; t++) {
      const int s = t % GSTAGES;
      const uint32_t ph = uint32_t(t / GSTAGES) & 1u;
      if (!(good = tc::mbar_wait(&full[s], ph, err, 2u))) break;
      tc::tc_fence_after();
      const uint32_t a = tc::smem_u32(sm + s * GSTAGE), b = a + GA_BYTES;
#pragma unroll
      for (int kk = 0; kk < GBK / 16; kk++)
        tc::mma_bf16(tmem, tc::desc_k_sw128(a + kk * 32), tc::desc_k_sw128(b + kk * 32), idesc, (t > 0 || kk > 0) ? 1u : 0u);
      tc::mma_commit(&empty[s]);
    }
    tc::mma_commit(accf);
  }
  if (warp >= 2) {
    ok = tc::mbar_wait(accf, 0, err, 4u);
    tc::tc_fence_after();
  }
  return tmem;
}

__device__ __forceinline__ void gemm_teardown(uint32_t tmem) {
  tc::tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 1) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 256);
  }
}

// forward and backward-data tiles: rows are samples m0 .. m0 + 127
template <int ROLE>
__global__ void __launch_bounds__(GTHREADS, 1) k_mlp_gemm(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
                                                          int N, int ktiles, Epi ep, unsigned int* err) {
  extern __shared__ uint8_t smraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  __shared__ double lred[4];
  const int m0 = blockIdx.x * GBM;
  bool ok;
  const uint32_t tmem = gemm_mainloop(&tA, &tB, m0, 0, ktiles, N, sm, err, ok);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= 2) {
    const int q = warp & 3, row = q * 32 + lane;
    const long s = m0 + row;
    const uint32_t trow = tmem + (uint32_t(q * 32) << 16);
    if (ROLE == R_HIDDEN || ROLE == R_BACK) {
#pragma unroll 1
      for (int c0 = 0; c0 < NH; c0 += 32) {
        float v[32];
        tc::tmem_ld32(trow + uint32_t(c0), v);
        if (!ok) continue;
        if (ROLE == R_HIDDEN) {
          float gp[32];
#pragma unroll
          for (int e = 0; e < 32; e++) {
            const float z = v[e] + __ldg(ep.bias + c0 + e);
            v[e] = gelu(z);
            gp[e] = gelu_grad(z);
          }
#pragma unroll
          for (int e = 0; e < 32; e += 4) *reinterpret_cast<float4*>(ep.G + s * NH + c0 + e) = make_float4(gp[e], gp[e + 1], gp[e + 2], gp[e + 3]);
        } else {
#pragma unroll
          for (int e = 0; e < 32; e += 4) {
            const float4 g = *reinterpret_cast<const float4*>(ep.G + s * NH + c0 + e);
            v[e] *= g.x; v[e + 1] *= g.y; v[e + 2] *= g.z; v[e + 3] *= g.w;
          }
        }
        if (ep.s_out) {
#pragma unroll
          for (int e = 0; e < 32; e += 8) store8(ep.s_out + s * ep.ld_s + c0 + e, v + e);
        }
#pragma unroll
        for (int e = 0; e < 32; e++) ep.t_out[long(c0 + e) * ep.B + s] = __float2bfloat16_rn(v[e]);
      }
    } else {  // R_OUT: N = 16 columns, 10 outputs, the first NLOSS in the loss
      float y[16];
      tmem_ld16x(trow, y);
      double l = 0.0;
      if (ok) {
        float dy[16];
#pragma unroll
        for (int e = 0; e < 16; e++) {
          float d = 0.f;
          if (e < NLOSS) d = y[e] + __ldg(ep.bias + e) - __ldg(ep.T + s * NLOSS + e);
          l += double(d) * d;
          dy[e] = ep.inv * d;
        }
        store8(ep.s_out + s * ep.ld_s, dy);
        store8(ep.s_out + s * ep.ld_s + 8, dy + 8);
#pragma unroll
        for (int e = 0; e < 16; e++) ep.t_out[long(e) * ep.B + s] = __float2bfloat16_rn(dy[e]);
      }
      for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
      if (lane == 0) lred[q] = l;
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (warp == 2 && lane == 0) ep.lossp[blockIdx.x] = lred[0] + lred[1] + lred[2] + lred[3];
    }
  }
  gemm_teardown(tmem);
}

// the four weight gradients at once: blockIdx.y = problem, blockIdx.x = batch split (ktiles stages of 64 samples)
__global__ void __launch_bounds__(GTHREADS, 1) k_mlp_wgrad(const __grid_constant__ WgradSet S, int ktiles, unsigned int* err) {
  extern __shared__ uint8_t smraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const int p = blockIdx.y, z = blockIdx.x, N = S.N[p];
  bool ok;
  const uint32_t tmem = gemm_mainloop(&S.a[p], &S.b[p], 0, z * ktiles * GBK, ktiles, N, sm, err, ok);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= 2) {
    const int q = warp & 3, row = q * 32 + lane;
    const uint32_t trow = tmem + (uint32_t(q * 32) << 16);
    float* out = S.part[p] + (long(z) * GBM + row) * N;
#pragma unroll 1
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tmem_ld16x(trow + uint32_t(c0), v);
      if (!ok) continue;
#pragma unroll
      for (int e = 0; e < 16; e += 4) *reinterpret_cast<float4*>(out + c0 + e) = make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]);
    }
  }
  gemm_teardown(tmem);
}

// batch gather for the tensor-core step: inputs normalised to bf16, sample-major (K padded to 64, zeros past 12) and
// feature-major (rows 0-11; row 12 the ones, rows 13-15 zeros, both written once at allocation); targets fp32
__global__ void k_gather_tc(const float* __restrict__ pairs, const unsigned* __restrict__ idx, int B, Norm nm,
                            __nv_bfloat16* __restrict__ Xs, __nv_bfloat16* __restrict__ Xt, float* __restrict__ T) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const float* p = pairs + size_t(idx ? idx[s] : unsigned(s)) * PAIR;
#pragma unroll
  for (int i = 0; i < NIN; i++) {
    const __nv_bfloat16 x = __float2bfloat16_rn((feature(i, p[i]) - nm.in_mean[i]) * nm.in_scale[i]);
    Xs[size_t(s) * KPAD + i] = x;
    Xt[size_t(i) * B + s] = x;
  }
#pragma unroll
  for (int j = 0; j < NLOSS; j++) T[size_t(s) * NLOSS + j] = nm.out_scale[j] > 0.f ? p[NIN + j] / nm.out_scale[j] : 0.f;
}

// gradient of parameter t = sum over the splits, in split order, of its element of the partial slices
__global__ void k_grad_reduce(const float* __restrict__ p1, const float* __restrict__ p2, const float* __restrict__ p3,
                              const float* __restrict__ p4, int nsplit, float* __restrict__ g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NPARAM) return;
  const float* part;
  int N, j, n;
  if (t < OB1) { part = p1; N = NXX; j = t / NIN; n = t - j * NIN; }
  else if (t < OW2) { part = p1; N = NXX; j = t - OB1; n = NIN; }
  else if (t < OB2) { part = p2; N = NHX; j = (t - OW2) / NH; n = (t - OW2) % NH; }
  else if (t < OW3) { part = p2; N = NHX; j = t - OB2; n = NH; }
  else if (t < OB3) { part = p3; N = NHX; j = (t - OW3) / NH; n = (t - OW3) % NH; }
  else if (t < OW4) { part = p3; N = NHX; j = t - OB3; n = NH; }
  else if (t < OB4) { part = p4; N = NHX; j = (t - OW4) / NH; n = (t - OW4) % NH; }
  else { part = p4; N = NHX; j = t - OB4; n = NH; }
  float acc = 0.f;
  for (int z = 0; z < nsplit; z++) acc += part[(long(z) * GBM + j) * N + n];
  g[t] = acc;
}

// bf16 images of the weights, both ways: W1i [128][64], W2i / W3i [128][128], W4i [16][128] (forward, K-major over
// the inputs) and W2T / W3T [128][128], W4T [128][64] (backward, K-major over the outputs); padding stays zero
struct Images {
  __nv_bfloat16 *w1, *w2, *w3, *w4, *w2t, *w3t, *w4t;
};
__device__ __forceinline__ void put_image(const Images& im, int t, float w) {
  const __nv_bfloat16 b = __float2bfloat16_rn(w);
  if (t < OB1) { const int j = t / NIN, i = t - j * NIN; im.w1[j * KPAD + i] = b; }
  else if (t >= OW2 && t < OB2) { const int j = (t - OW2) / NH, i = (t - OW2) % NH; im.w2[j * NH + i] = b; im.w2t[i * NH + j] = b; }
  else if (t >= OW3 && t < OB3) { const int j = (t - OW3) / NH, i = (t - OW3) % NH; im.w3[j * NH + i] = b; im.w3t[i * NH + j] = b; }
  else if (t >= OW4 && t < OB4) { const int j = (t - OW4) / NH, i = (t - OW4) % NH; im.w4[j * NH + i] = b; im.w4t[i * KPAD + j] = b; }
}
__global__ void k_images(const float* __restrict__ w, Images im) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < NPARAM) put_image(im, t, w[t]);
}
__global__ void k_adam_img(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, float lr,
                           float b1, float b2, float eps, float c1, float c2, Images im) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  put_image(im, i, wi);
}
// loss += (the per-tile partials, summed in tile order) / (B * NLOSS)
__global__ void k_loss_tiles(const double* __restrict__ part, int n, long B, double* __restrict__ loss) {
  double t = 0.0;
  for (int i = 0; i < n; i++) t += part[i];
  *loss += t / double(B * NLOSS);
}
// random batch indices: a hash of (step, s) reduced to [0, n) (the same draw as the fp32 trainer's)
__global__ void k_draw_tc(unsigned* idx, int B, unsigned n, unsigned step, unsigned seed) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  unsigned h = unsigned(s) * 0x9E3779B1u ^ (step * 0x85EBCA77u + seed);
  h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
  idx[s] = unsigned((uint64_t(h) * n) >> 32);
}
__global__ void k_fill_bf16(__nv_bfloat16* p, long n, float v) {
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) p[i] = __float2bfloat16_rn(v);
}

}  // namespace mlp

// ---------------------------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------------------------
namespace {
typedef CUresult (*PFN_encode)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                               const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                               CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
PFN_encode encoder() {
  static PFN_encode fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_encode>(p);
  }
  return fn;
}
// K-major bf16 operand [rows][cols] (pitch cols), box 64 columns x box_rows, 128-byte swizzle
bool kmap(CUtensorMap* m, const void* base, long rows, long cols, int box_rows) {
  PFN_encode enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(cols * 2)};
  cuuint32_t box[2] = {cuuint32_t(mlp::GBK), cuuint32_t(box_rows)};
  cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

struct MlpTcTrainer {
  long cap = 0;   // batch capacity (a multiple of 128)
  long B = 0;     // batch the maps are made for
  __nv_bfloat16 *Xs = nullptr, *Xt = nullptr, *Hs[3] = {}, *Ht[3] = {}, *dYs = nullptr, *dYt = nullptr, *dZs[3] = {}, *dZt[3] = {};
  __nv_bfloat16* img = nullptr;
  mlp::Images im{};
  float *T = nullptr, *G[3] = {}, *part[4] = {};
  double* lossp = nullptr;
  unsigned* idx = nullptr;
  unsigned int* err = nullptr;
  int nsplit = 1, wktiles = 1;
  CUtensorMap fA[4], fB[4], bA[3], bB[3];
  mlp::WgradSet W{};
};

namespace mlp {
namespace {
int ok_or(bool ok, const char* what) {
  if (ok) return OB_OK;
  set_error("mlp tensor-core training: %s", what);
  return OB_ERR_DEVICE;
}
void free_all(MlpTcTrainer* t) {
  std::vector<void*> ps = {t->Xs, t->Xt, t->dYs, t->dYt, t->img, t->T, t->lossp, t->idx, t->err};
  for (int l = 0; l < 3; l++) { ps.push_back(t->Hs[l]); ps.push_back(t->Ht[l]); ps.push_back(t->dZs[l]); ps.push_back(t->dZt[l]); ps.push_back(t->G[l]); }
  for (int p = 0; p < 4; p++) ps.push_back(t->part[p]);
  for (void* p : ps)
    if (p) cudaFree(p);
  *t = MlpTcTrainer();
}
}  // namespace

// buffers and tensor maps for batches of B samples (B a multiple of 128)
int tc_train_prepare(MlpTcTrainer* t, long B, const float* d_w, cudaStream_t s) {
  if (B % GBM != 0 || B < GBM) { set_error("mlp tensor-core training: the batch must be a positive multiple of 128"); return OB_ERR_INVALID; }
  if (B == t->B) return OB_OK;
  free_all(t);
  bool ok = true;
  auto al = [&](void** p, size_t bytes) { ok = ok && cudaMalloc(p, bytes) == cudaSuccess && cudaMemsetAsync(*p, 0, bytes, s) == cudaSuccess; };
  const size_t b = size_t(B);
  al((void**)&t->Xs, b * KPAD * 2);
  al((void**)&t->Xt, NXX * b * 2);
  al((void**)&t->dYs, b * KPAD * 2);
  al((void**)&t->dYt, GBM * b * 2);
  for (int l = 0; l < 3; l++) {
    al((void**)&t->Hs[l], b * NH * 2);
    al((void**)&t->Ht[l], NHX * b * 2);
    al((void**)&t->dZt[l], GBM * b * 2);
    al((void**)&t->G[l], b * NH * 4);
  }
  al((void**)&t->dZs[1], b * NH * 2);
  al((void**)&t->dZs[2], b * NH * 2);
  const size_t img = size_t(NH) * KPAD + 2 * NH * NH + 16 * NH + 2 * NH * NH + NH * KPAD;
  al((void**)&t->img, img * 2);
  al((void**)&t->T, b * NLOSS * 4);
  al((void**)&t->lossp, (b / GBM) * 8);
  al((void**)&t->idx, b * 4);
  al((void**)&t->err, 16);
  // weight gradients: at most WSPLIT_MAX batch splits of whole 64-sample stages
  const int kt = int(B / GBK);
  t->nsplit = 1;
  for (int d = WSPLIT_MAX; d >= 1; d--)
    if (kt % d == 0) { t->nsplit = d; break; }
  t->wktiles = kt / t->nsplit;
  for (int p = 0; p < 4; p++) al((void**)&t->part[p], size_t(t->nsplit) * GBM * NHX * 4);
  if (!ok) { free_all(t); set_error("mlp tensor-core training: out of device memory"); return OB_ERR_OOM; }
  t->cap = t->B = B;
  __nv_bfloat16* q = t->img;
  t->im.w1 = q; q += NH * KPAD;
  t->im.w2 = q; q += NH * NH;
  t->im.w3 = q; q += NH * NH;
  t->im.w4 = q; q += 16 * NH;
  t->im.w2t = q; q += NH * NH;
  t->im.w3t = q; q += NH * NH;
  t->im.w4t = q;
  // the rows of ones that make the weight-gradient GEMMs return the bias gradients
  k_fill_bf16<<<64, 256, 0, s>>>(t->Xt + size_t(NIN) * b, long(b), 1.f);
  for (int l = 0; l < 3; l++) k_fill_bf16<<<64, 256, 0, s>>>(t->Ht[l] + size_t(NH) * b, long(b), 1.f);
  k_images<<<(NPARAM + 255) / 256, 256, 0, s>>>(d_w, t->im);
  // forward: A = X / H1 / H2 / H3 (sample-major), B = W1i / W2i / W3i / W4i
  ok = kmap(&t->fA[0], t->Xs, B, KPAD, GBM) && kmap(&t->fB[0], t->im.w1, NH, KPAD, NH);
  ok = ok && kmap(&t->fA[1], t->Hs[0], B, NH, GBM) && kmap(&t->fB[1], t->im.w2, NH, NH, NH);
  ok = ok && kmap(&t->fA[2], t->Hs[1], B, NH, GBM) && kmap(&t->fB[2], t->im.w3, NH, NH, NH);
  ok = ok && kmap(&t->fA[3], t->Hs[2], B, NH, GBM) && kmap(&t->fB[3], t->im.w4, 16, NH, 16);
  // backward data: dH3 = dY W4, dH2 = dZ3 W3, dH1 = dZ2 W2 (B = the transposed images)
  ok = ok && kmap(&t->bA[2], t->dYs, B, KPAD, GBM) && kmap(&t->bB[2], t->im.w4t, NH, KPAD, NH);
  ok = ok && kmap(&t->bA[1], t->dZs[2], B, NH, GBM) && kmap(&t->bB[1], t->im.w3t, NH, NH, NH);
  ok = ok && kmap(&t->bA[0], t->dZs[1], B, NH, GBM) && kmap(&t->bB[0], t->im.w2t, NH, NH, NH);
  // weight gradients: A = dZ^T / dY^T [128][B], B = [H, 1]^T / [X, 1]^T [N][B]
  ok = ok && kmap(&t->W.a[0], t->dZt[0], GBM, B, GBM) && kmap(&t->W.b[0], t->Xt, NXX, B, NXX);
  ok = ok && kmap(&t->W.a[1], t->dZt[1], GBM, B, GBM) && kmap(&t->W.b[1], t->Ht[0], NHX, B, NHX);
  ok = ok && kmap(&t->W.a[2], t->dZt[2], GBM, B, GBM) && kmap(&t->W.b[2], t->Ht[1], NHX, B, NHX);
  ok = ok && kmap(&t->W.a[3], t->dYt, GBM, B, GBM) && kmap(&t->W.b[3], t->Ht[2], NHX, B, NHX);
  t->W.N[0] = NXX; t->W.N[1] = t->W.N[2] = t->W.N[3] = NHX;
  for (int p = 0; p < 4; p++) t->W.part[p] = t->part[p];
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_mlp_gemm<R_HIDDEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, GSMEM);
    cudaFuncSetAttribute(k_mlp_gemm<R_OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, GSMEM);
    cudaFuncSetAttribute(k_mlp_gemm<R_BACK>, cudaFuncAttributeMaxDynamicSharedMemorySize, GSMEM);
    cudaFuncSetAttribute(k_mlp_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, GSMEM);
    attr = true;
  }
  return ok_or(ok, "tensor map encoding failed");
}

// forward + backward of the gathered batch (t->Xs, t->Xt, t->T): the loss partials and the gradient into g
void tc_forward_backward(MlpTcTrainer* t, const float* w, float* g, double* loss, cudaStream_t s) {
  const long B = t->B;
  const int tiles = int(B / GBM);
  Epi e{};
  e.B = B;
  // forward, hidden layers
  const int boff[3] = {OB1, OB2, OB3};
  const int kts[3] = {1, 2, 2};
  for (int l = 0; l < 3; l++) {
    e.bias = w + boff[l];
    e.s_out = t->Hs[l]; e.ld_s = NH; e.t_out = t->Ht[l]; e.G = t->G[l];
    k_mlp_gemm<R_HIDDEN><<<tiles, GTHREADS, GSMEM, s>>>(t->fA[l], t->fB[l], NH, kts[l], e, t->err);
  }
  // output layer: loss and dY
  e = Epi{};
  e.B = B; e.bias = w + OB4; e.s_out = t->dYs; e.ld_s = KPAD; e.t_out = t->dYt; e.T = t->T; e.lossp = t->lossp;
  e.inv = 2.f / float(B * NLOSS);
  k_mlp_gemm<R_OUT><<<tiles, GTHREADS, GSMEM, s>>>(t->fA[3], t->fB[3], 16, 2, e, t->err);
  k_loss_tiles<<<1, 1, 0, s>>>(t->lossp, tiles, B, loss);
  // backward data: dZ3 (from dY), dZ2, dZ1
  for (int l = 2; l >= 0; l--) {
    e = Epi{};
    e.B = B; e.G = t->G[l]; e.s_out = l > 0 ? t->dZs[l] : nullptr; e.ld_s = NH; e.t_out = t->dZt[l];
    k_mlp_gemm<R_BACK><<<tiles, GTHREADS, GSMEM, s>>>(t->bA[l], t->bB[l], NH, l == 2 ? 1 : 2, e, t->err);
  }
  // the four weight gradients in one launch, then their split sums in order
  k_mlp_wgrad<<<dim3(t->nsplit, 4), GTHREADS, GSMEM, s>>>(t->W, t->wktiles, t->err);
  k_grad_reduce<<<(NPARAM + 255) / 256, 256, 0, s>>>(t->part[0], t->part[1], t->part[2], t->part[3], t->nsplit, g);
}

// ---- entry points for ob_mlp.cu (the network's handle owns one trainer) ----
MlpTcTrainer* tc_trainer_new() { return new MlpTcTrainer(); }
void tc_trainer_delete(MlpTcTrainer* t) {
  if (!t) return;
  free_all(t);
  delete t;
}

static int tc_check_err(MlpTcTrainer* t, cudaStream_t s) {
  unsigned h = 0;
  if (cudaMemcpyAsync(&h, t->err, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
    set_error("mlp tensor-core training: %s", cudaGetErrorString(cudaGetLastError()));
    return OB_ERR_DEVICE;
  }
  if (h) {
    cudaMemsetAsync(t->err, 0, 4, s);
    set_error("mlp tensor-core training: a pipeline wait timed out (code %u)", h);
    return OB_ERR_TIMEOUT;
  }
  return OB_OK;
}

// `steps` Adam steps on random batches of `batch` recorded pairs; the loss of every step is added into *d_loss
int tc_train_run(MlpTcTrainer* t, float* w, float* g, float* m, float* v, int& adam_t, const float* pairs, unsigned npairs,
                 const Norm& nm, int batch, int steps, float lr, unsigned seed, double* d_loss, cudaStream_t s) {
  int rc = tc_train_prepare(t, batch, w, s);
  if (rc != OB_OK) return rc;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int st = 0; st < steps; st++) {
    k_draw_tc<<<(batch + 255) / 256, 256, 0, s>>>(t->idx, batch, npairs, unsigned(adam_t), seed);
    k_gather_tc<<<(batch + 127) / 128, 128, 0, s>>>(pairs, t->idx, batch, nm, t->Xs, t->Xt, t->T);
    tc_forward_backward(t, w, g, d_loss, s);
    adam_t++;
    const float c1 = 1.f - std::pow(b1, float(adam_t)), c2 = 1.f - std::pow(b2, float(adam_t));
    k_adam_img<<<(NPARAM + 255) / 256, 256, 0, s>>>(w, g, m, v, lr, b1, b2, 1e-8f, c1, c2, t->im);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("mlp tensor-core training launch: %s", cudaGetErrorString(e));
    return OB_ERR_DEVICE;
  }
  return tc_check_err(t, s);
}

// loss (added into *d_loss) and gradient g of `count` pairs in order (count a multiple of 128), at the parameters w
int tc_grad_run(MlpTcTrainer* t, const float* w, float* g, const float* pairs, int count, const Norm& nm, double* d_loss,
                cudaStream_t s) {
  int rc = tc_train_prepare(t, count, w, s);
  if (rc != OB_OK) return rc;
  k_images<<<(NPARAM + 255) / 256, 256, 0, s>>>(w, t->im);
  k_gather_tc<<<(count + 127) / 128, 128, 0, s>>>(pairs, nullptr, count, nm, t->Xs, t->Xt, t->T);
  tc_forward_backward(t, w, g, d_loss, s);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("mlp tensor-core gradient launch: %s", cudaGetErrorString(e));
    return OB_ERR_DEVICE;
  }
  return tc_check_err(t, s);
}

}  // namespace mlp
}  // namespace ob
