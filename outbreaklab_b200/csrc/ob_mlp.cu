// ob_mlp.cu — the C ABI of the microphysics surrogate (ob_mlp_*) and its fp32 SIMT training kernels (sm_100a):
// forward and backward kernels and Adam, the reference arithmetic for the gradient check and the path for batches that
// are not a multiple of 128. The default training runs on the tensor cores (ob_mlp_train_tc.cu); the inference kernel
// that runs inside the model step is in ob_mlp_tc.cu.
//
// One training step on a batch of B recorded pairs: gather + normalise (k_gather), three hidden layers
// Z = H W^T + b, H' = gelu(Z) and the output layer (k_gemm<false, true>), the mean squared error of the 8 scheme
// tendencies and its gradient (k_loss), the backward GEMMs dW = dZ^T H (split over the batch, k_gemm<true, false>)
// and dH = dZ W (k_gemm<false, false>), GELU derivatives, bias sums, and one Adam update of all parameters. The
// gradient of this chain is checked against a float64 restatement on the CPU in the tests.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ob.h"
#include "ob_mlp.cuh"

namespace ob {
void set_error(const char* fmt, ...);

namespace mlp {

constexpr int kMaxSplits = 64;   // batch splits of a weight-gradient GEMM (partial-sum slices of NH x NH floats)


// C[M][N] = op(A) op(B) (+ bias[n]) in fp32; AT: A is stored [K][M] (else [M][K]); BT: B is stored [N][K] (else
// [K][N]). 64 x 64 tiles, 256 threads, 4 x 4 outputs per thread; blockIdx.z splits K: with more than one split,
// split z writes its partial sum to its own slice C + z * M * ldc, and k_sum_slices adds the slices in split order,
// so the result does not depend on which block finishes first.
template <bool AT, bool BT>
__global__ void __launch_bounds__(256) k_gemm(const float* __restrict__ A, int lda, const float* __restrict__ B, int ldb,
                                              float* __restrict__ C, int ldc, int M, int N, int K, const float* __restrict__ bias,
                                              int ksplit) {
  __shared__ float As[16][64 + 4];
  __shared__ float Bs[16][64 + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const int kper = ((K + ksplit - 1) / ksplit + 15) / 16 * 16;
  const int kb = blockIdx.z * kper, ke = min(K, kb + kper);
  float acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk, mm;
      if (AT) { mm = e & 63; kk = e >> 6; } else { kk = e & 15; mm = e >> 4; }
      const int gk = k0 + kk, gm = m0 + mm;
      As[kk][mm] = (gk < ke && gm < M) ? (AT ? A[long(gk) * lda + gm] : A[long(gm) * lda + gk]) : 0.f;
      int kn, nn;
      if (BT) { kn = e & 15; nn = e >> 4; } else { nn = e & 63; kn = e >> 6; }
      const int gk2 = k0 + kn, gn = n0 + nn;
      Bs[kn][nn] = (gk2 < ke && gn < N) ? (BT ? B[long(gn) * ldb + gk2] : B[long(gk2) * ldb + gn]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      if (ksplit > 1) C[long(blockIdx.z) * M * ldc + long(m) * ldc + n] = acc[i][j];
      else C[long(m) * ldc + n] = acc[i][j] + (bias ? bias[n] : 0.f);
    }
  }
}

// out[i] = sum over z = 0 .. nsl-1 of part[z * n + i], in that order
__global__ void k_sum_slices(const float* __restrict__ part, int nsl, long n, float* __restrict__ out) {
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
    float acc = 0.f;
    for (int z = 0; z < nsl; z++) acc += part[z * n + i];
    out[i] = acc;
  }
}

// batch gather: sample s takes pair idx[s] (or s when idx is null), writes normalised inputs X[s][NIN] and scaled
// targets T[s][NOUT] (spare outputs 0)
__global__ void k_gather(const float* __restrict__ pairs, const unsigned* __restrict__ idx, int B, Norm nm, float* __restrict__ X,
                         float* __restrict__ T) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const float* p = pairs + size_t(idx ? idx[s] : unsigned(s)) * PAIR;
#pragma unroll
  for (int i = 0; i < NIN; i++) X[size_t(s) * NIN + i] = (feature(i, p[i]) - nm.in_mean[i]) * nm.in_scale[i];
#pragma unroll
  for (int j = 0; j < NOUT; j++) T[size_t(s) * NOUT + j] = nm.out_scale[j] > 0.f ? p[NIN + j] / nm.out_scale[j] : 0.f;
}

// random batch indices: a hash of (step, s) reduced to [0, n)
__global__ void k_draw(unsigned* idx, int B, unsigned n, unsigned step, unsigned seed) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  unsigned h = unsigned(s) * 0x9E3779B1u ^ (step * 0x85EBCA77u + seed);
  h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
  idx[s] = unsigned((uint64_t(h) * n) >> 32);
}

__global__ void k_gelu(const float* __restrict__ Z, float* __restrict__ H, long n) {
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) H[i] = gelu(Z[i]);
}
__global__ void k_gelu_back(const float* __restrict__ Z, float* __restrict__ dH, long n) {
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) dH[i] *= gelu_grad(Z[i]);
}

// loss = mean over the batch and the NLOSS scheme outputs of (Y - T)^2, accumulated in FP64; dY = dloss/dY. Each
// block writes its FP64 partial sum to part[blockIdx.x]; k_loss_total adds them in block order.
__global__ void __launch_bounds__(256) k_loss(const float* __restrict__ Y, const float* __restrict__ T, int B, float* __restrict__ dY,
                                              double* __restrict__ part) {
  __shared__ double red[8];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (s < B) {
    for (int j = 0; j < NOUT; j++) {
      const float d = j < NLOSS ? Y[size_t(s) * NOUT + j] - T[size_t(s) * NOUT + j] : 0.f;
      dY[size_t(s) * NOUT + j] = 2.f * d / float(B * NLOSS);
      l += double(d) * d;
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); w++) t += red[w];
    part[blockIdx.x] = t;
  }
}
// loss += (sum of the nb block partials, in order) / (B * NLOSS): one thread, once per training step
__global__ void k_loss_total(const double* __restrict__ part, int nb, int B, double* __restrict__ loss) {
  double t = 0.0;
  for (int b = 0; b < nb; b++) t += part[b];
  *loss += t / double(B * NLOSS);
}

// bias gradient: column sums of dZ[B][N]; row chunk y writes its partial column sums to part[y * N + n] (summed in
// chunk order by k_sum_slices)
__global__ void k_colsum(const float* __restrict__ dZ, int B, int N, float* __restrict__ part) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int rows = (B + gridDim.y - 1) / gridDim.y, r0 = blockIdx.y * rows, r1 = min(B, r0 + rows);
  float s = 0.f;
  for (int r = r0; r < r1; r++) s += dZ[size_t(r) * N + n];
  part[long(blockIdx.y) * N + n] = s;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, int n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace mlp
}  // namespace ob

// ---------------------------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------------------------
using namespace ob;
using namespace ob::mlp;

namespace ob {
struct MlpTcTrainer;
namespace mlp {
MlpTcTrainer* tc_trainer_new();
void tc_trainer_delete(MlpTcTrainer* t);
int tc_train_run(MlpTcTrainer* t, float* w, float* g, float* m, float* v, int& adam_t, const float* pairs, unsigned npairs,
                 const Norm& nm, int batch, int steps, float lr, unsigned seed, double* d_loss, cudaStream_t s);
int tc_grad_run(MlpTcTrainer* t, const float* w, float* g, const float* pairs, int count, const Norm& nm, double* d_loss,
                cudaStream_t s);
int sort_pairs(float* pairs, long n, bool overflowed, unsigned* count, cudaStream_t s);
}  // namespace mlp
}  // namespace ob

struct ObMlp {
  int train_mode = 1;    // 1: bf16 tcgen05 training kernels (batches that are multiples of 128), 0: fp32 SIMT kernels
  ob::MlpTcTrainer* tct = nullptr;
  float* d_w = nullptr;  // fp32 master parameters
  float* d_g = nullptr;  // gradient of the last batch
  float* d_m = nullptr;  // Adam moments
  float* d_v = nullptr;
  Norm norm{};
  int adam_t = 0;
  float* d_pairs = nullptr;  // recorded (state, tendency) pairs
  unsigned* d_count = nullptr;
  size_t cap = 0;
  int bcap = 0;  // training scratch for batches up to bcap
  float *X = nullptr, *T = nullptr, *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *Z3 = nullptr, *H3 = nullptr;
  float *Y = nullptr, *dY = nullptr, *dA = nullptr, *dB = nullptr, *hp = nullptr;
  unsigned* idx = nullptr;
  float* part = nullptr;       // split-K and bias partial sums (PART_FLOATS)
  double* lpart = nullptr;     // per-block loss partials
  double* d_loss = nullptr;
  cudaStream_t stream = nullptr;
};

namespace {
int cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return OB_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? OB_ERR_OOM : OB_ERR_DEVICE;
}
#define MLP_TRY(x) do { const int _r = (x); if (_r != OB_OK) return _r; } while (0)

void free_scratch(ObMlp* n) {
  for (float* p : {n->X, n->T, n->Z1, n->H1, n->Z2, n->H2, n->Z3, n->H3, n->Y, n->dY, n->dA, n->dB, n->hp})
    if (p) cudaFree(p);
  if (n->idx) cudaFree(n->idx);
  if (n->part) cudaFree(n->part);
  if (n->lpart) cudaFree(n->lpart);
  n->X = n->T = n->Z1 = n->H1 = n->Z2 = n->H2 = n->Z3 = n->H3 = n->Y = n->dY = n->dA = n->dB = n->hp = nullptr;
  n->idx = nullptr;
  n->part = nullptr;
  n->lpart = nullptr;
  n->bcap = 0;
}

int ensure_scratch(ObMlp* n, int B) {
  if (B <= n->bcap) return OB_OK;
  free_scratch(n);
  const size_t b = size_t(B);
  float** bufs[] = {&n->Z1, &n->H1, &n->Z2, &n->H2, &n->Z3, &n->H3, &n->dA, &n->dB};
  for (float** p : bufs) MLP_TRY(cuda_ok(cudaMalloc(p, b * NH * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->X, b * NIN * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->T, b * NOUT * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->Y, b * NOUT * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->dY, b * NOUT * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->hp, b * PAIR * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->idx, b * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->part, size_t(kMaxSplits) * NH * NH * 4), "mlp scratch"));
  MLP_TRY(cuda_ok(cudaMalloc(&n->lpart, ((b + 255) / 256) * 8), "mlp scratch"));
  n->bcap = B;
  return OB_OK;
}

inline dim3 ew(long n) { return dim3(unsigned(std::min<long>((n + 255) / 256, 4096))); }

template <bool AT, bool BT>
void gemm(const float* A, int lda, const float* B, int ldb, float* C, int ldc, int M, int N, int K, const float* bias, int ksplit,
          cudaStream_t s) {
  dim3 grid((N + 63) / 64, (M + 63) / 64, ksplit);
  k_gemm<AT, BT><<<grid, 256, 0, s>>>(A, lda, B, ldb, C, ldc, M, N, K, bias, ksplit);
}
// K splits of a weight-gradient GEMM (reduction over the batch): about two blocks per SM in total, at most kMaxSplits
int splits(int M, int N, int K) {
  const int tiles = ((M + 63) / 64) * ((N + 63) / 64);
  return std::min(kMaxSplits, std::max(2, std::min(std::max(1, K / 256), std::max(1, 296 / tiles))));
}
// weight gradient C[M][N] (pitch N) = A^T B over the batch, split over the batch into the partial-sum slices of
// n->part and added in split order
void weight_grad(ObMlp* n, const float* A, int lda, const float* B, int ldb, float* C, int M, int N, int K) {
  const int ks = splits(M, N, K);
  gemm<true, false>(A, lda, B, ldb, n->part, N, M, N, K, nullptr, ks, n->stream);
  k_sum_slices<<<ew(long(M) * N), 256, 0, n->stream>>>(n->part, ks, long(M) * N, C);
}
// bias gradient g[N] = column sums of dZ[B][N], in row-chunk order
void bias_grad(ObMlp* n, const float* dZ, int B, int N, float* g) {
  const int chunks = std::max(1, std::min(B / 512, 64));
  k_colsum<<<dim3((N + 127) / 128, chunks), 128, 0, n->stream>>>(dZ, B, N, n->part);
  k_sum_slices<<<ew(N), 256, 0, n->stream>>>(n->part, chunks, N, g);
}
// forward of B gathered samples (n->X) to n->Y
void forward(ObMlp* n, int B) {
  cudaStream_t s = n->stream;
  const float* w = n->d_w;
  gemm<false, true>(n->X, NIN, w + OW1, NIN, n->Z1, NH, B, NH, NIN, w + OB1, 1, s);
  k_gelu<<<ew(long(B) * NH), 256, 0, s>>>(n->Z1, n->H1, long(B) * NH);
  gemm<false, true>(n->H1, NH, w + OW2, NH, n->Z2, NH, B, NH, NH, w + OB2, 1, s);
  k_gelu<<<ew(long(B) * NH), 256, 0, s>>>(n->Z2, n->H2, long(B) * NH);
  gemm<false, true>(n->H2, NH, w + OW3, NH, n->Z3, NH, B, NH, NH, w + OB3, 1, s);
  k_gelu<<<ew(long(B) * NH), 256, 0, s>>>(n->Z3, n->H3, long(B) * NH);
  gemm<false, true>(n->H3, NH, w + OW4, NH, n->Y, NOUT, B, NOUT, NH, w + OB4, 1, s);
}

// loss and gradient (n->d_g) of the B gathered samples
void backward(ObMlp* n, int B) {
  cudaStream_t s = n->stream;
  const float* w = n->d_w;
  float* g = n->d_g;
  const int nb = (B + 255) / 256;
  k_loss<<<nb, 256, 0, s>>>(n->Y, n->T, B, n->dY, n->lpart);
  k_loss_total<<<1, 1, 0, s>>>(n->lpart, nb, B, n->d_loss);
  const long bh = long(B) * NH;
  // output layer
  weight_grad(n, n->dY, NOUT, n->H3, NH, g + OW4, NOUT, NH, B);
  bias_grad(n, n->dY, B, NOUT, g + OB4);
  gemm<false, false>(n->dY, NOUT, w + OW4, NH, n->dA, NH, B, NH, NOUT, nullptr, 1, s);
  k_gelu_back<<<ew(bh), 256, 0, s>>>(n->Z3, n->dA, bh);
  // layer 3
  weight_grad(n, n->dA, NH, n->H2, NH, g + OW3, NH, NH, B);
  bias_grad(n, n->dA, B, NH, g + OB3);
  gemm<false, false>(n->dA, NH, w + OW3, NH, n->dB, NH, B, NH, NH, nullptr, 1, s);
  k_gelu_back<<<ew(bh), 256, 0, s>>>(n->Z2, n->dB, bh);
  // layer 2
  weight_grad(n, n->dB, NH, n->H1, NH, g + OW2, NH, NH, B);
  bias_grad(n, n->dB, B, NH, g + OB2);
  gemm<false, false>(n->dB, NH, w + OW2, NH, n->dA, NH, B, NH, NH, nullptr, 1, s);
  k_gelu_back<<<ew(bh), 256, 0, s>>>(n->Z1, n->dA, bh);
  // layer 1
  weight_grad(n, n->dA, NH, n->X, NIN, g + OW1, NH, NIN, B);
  bias_grad(n, n->dA, B, NH, g + OB1);
}
}  // namespace

extern "C" {

int ob_mlp_create(unsigned seed, ObMlp** out) {
  if (!out) { set_error("ob_mlp_create: null argument"); return OB_ERR_INVALID; }
  *out = nullptr;
  ObMlp* n = new ObMlp();
  int rc = cuda_ok(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking), "mlp stream");
  for (float** p : {&n->d_w, &n->d_g, &n->d_m, &n->d_v})
    if (rc == OB_OK) rc = cuda_ok(cudaMalloc(p, NPARAM * 4), "mlp parameters");
  if (rc == OB_OK) rc = cuda_ok(cudaMalloc(&n->d_loss, 8), "mlp loss");
  if (rc == OB_OK) rc = cuda_ok(cudaMalloc(&n->d_count, 8), "mlp counter");
  if (rc != OB_OK) { ob_mlp_destroy(n); return rc; }
  // He-style initialisation, N(0, 2 / fan_in) weights (N(0, 1 / fan_in) for the linear output layer) and zero
  // biases, from a seeded host generator (xorshift64, Box-Muller)
  std::vector<float> w(NPARAM, 0.f);
  uint64_t st = 0x9E3779B97F4A7C15ull ^ (uint64_t(seed) * 0xD1B54A32D192ED03ull);
  auto uni = [&]() {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    return (double((st >> 11) & ((1ull << 53) - 1)) + 0.5) / double(1ull << 53);
  };
  auto normal = [&]() { return std::sqrt(-2.0 * std::log(uni())) * std::cos(6.283185307179586 * uni()); };
  const int offs[4] = {OW1, OW2, OW3, OW4}, fan[4] = {NIN, NH, NH, NH}, rows[4] = {NH, NH, NH, NOUT};
  for (int l = 0; l < 4; l++)
    for (int i = 0; i < rows[l] * fan[l]; i++) w[offs[l] + i] = float(normal() * std::sqrt((l == 3 ? 1.0 : 2.0) / fan[l]));
  cudaMemcpy(n->d_w, w.data(), NPARAM * 4, cudaMemcpyHostToDevice);
  cudaMemset(n->d_m, 0, NPARAM * 4);
  cudaMemset(n->d_v, 0, NPARAM * 4);
  cudaMemset(n->d_count, 0, 8);
  for (int i = 0; i < NIN; i++) { n->norm.in_scale[i] = 1.f; n->norm.in_lo[i] = -3e38f; n->norm.in_hi[i] = 3e38f; }
  for (int j = 0; j < NOUT; j++) n->norm.out_scale[j] = j < NLOSS ? 1.f : 0.f;
  n->norm.dt = 0.f;
  *out = n;
  return OB_OK;
}

int ob_mlp_destroy(ObMlp* n) {
  if (!n) return OB_OK;
  if (n->stream) cudaStreamSynchronize(n->stream);
  free_scratch(n);
  tc_trainer_delete(n->tct);
  for (void* p : {(void*)n->d_w, (void*)n->d_g, (void*)n->d_m, (void*)n->d_v, (void*)n->d_pairs, (void*)n->d_count, (void*)n->d_loss})
    if (p) cudaFree(p);
  if (n->stream) cudaStreamDestroy(n->stream);
  delete n;
  return OB_OK;
}

int ob_mlp_set_params(ObMlp* n, const float* host, int count) {
  if (!n || !host || count != NPARAM) { set_error("ob_mlp_set_params: expected %d parameters", NPARAM); return OB_ERR_INVALID; }
  n->adam_t = 0;
  cudaMemsetAsync(n->d_m, 0, NPARAM * 4, n->stream);
  cudaMemsetAsync(n->d_v, 0, NPARAM * 4, n->stream);
  MLP_TRY(cuda_ok(cudaMemcpyAsync(n->d_w, host, NPARAM * 4, cudaMemcpyHostToDevice, n->stream), "ob_mlp_set_params"));
  return cuda_ok(cudaStreamSynchronize(n->stream), "ob_mlp_set_params");
}

int ob_mlp_get_params(ObMlp* n, float* host, int count) {
  if (!n || !host || count != NPARAM) { set_error("ob_mlp_get_params: expected %d parameters", NPARAM); return OB_ERR_INVALID; }
  MLP_TRY(cuda_ok(cudaMemcpyAsync(host, n->d_w, NPARAM * 4, cudaMemcpyDeviceToHost, n->stream), "ob_mlp_get_params"));
  return cuda_ok(cudaStreamSynchronize(n->stream), "ob_mlp_get_params");
}

int ob_mlp_set_norm(ObMlp* n, const float* host, int count) {
  if (!n || !host || count != OB_MLP_NNORM) { set_error("ob_mlp_set_norm: expected %d floats", OB_MLP_NNORM); return OB_ERR_INVALID; }
  static_assert(sizeof(Norm) == OB_MLP_NNORM * sizeof(float), "norm layout");
  std::memcpy(&n->norm, host, sizeof(Norm));
  return OB_OK;
}

int ob_mlp_get_norm(ObMlp* n, float* host, int count) {
  if (!n || !host || count != OB_MLP_NNORM) { set_error("ob_mlp_get_norm: expected %d floats", OB_MLP_NNORM); return OB_ERR_INVALID; }
  std::memcpy(host, &n->norm, sizeof(Norm));
  return OB_OK;
}

int ob_mlp_reserve_pairs(ObMlp* n, long long cap) {
  if (!n || cap < 1 || cap > (1ll << 31)) { set_error("ob_mlp_reserve_pairs: bad capacity"); return OB_ERR_INVALID; }
  cudaStreamSynchronize(n->stream);
  if (n->d_pairs) cudaFree(n->d_pairs);
  n->d_pairs = nullptr;
  n->cap = 0;
  MLP_TRY(cuda_ok(cudaMalloc(&n->d_pairs, size_t(cap) * PAIR * 4), "ob_mlp_reserve_pairs"));
  n->cap = size_t(cap);
  return cuda_ok(cudaMemset(n->d_count, 0, 8), "ob_mlp_reserve_pairs");
}

int ob_mlp_pair_count(ObMlp* n, long long* count) {
  if (!n || !count) { set_error("ob_mlp_pair_count: null argument"); return OB_ERR_INVALID; }
  unsigned c = 0;
  MLP_TRY(cuda_ok(cudaDeviceSynchronize(), "ob_mlp_pair_count"));
  MLP_TRY(cuda_ok(cudaMemcpy(&c, n->d_count, 4, cudaMemcpyDeviceToHost), "ob_mlp_pair_count"));
  *count = std::min<long long>(c, (long long)n->cap);
  return OB_OK;
}

int ob_mlp_sort_pairs(ObMlp* n) {
  if (!n) { set_error("ob_mlp_sort_pairs: null network"); return OB_ERR_INVALID; }
  unsigned raw = 0;
  MLP_TRY(cuda_ok(cudaDeviceSynchronize(), "ob_mlp_sort_pairs"));
  MLP_TRY(cuda_ok(cudaMemcpy(&raw, n->d_count, 4, cudaMemcpyDeviceToHost), "ob_mlp_sort_pairs"));
  const long cnt = long(std::min<size_t>(raw, n->cap));
  return ob::mlp::sort_pairs(n->d_pairs, cnt, size_t(raw) > n->cap, n->d_count, n->stream);
}

int ob_mlp_read_pairs(ObMlp* n, long long first, long long count, float* host) {
  if (!n || !host || first < 0 || count < 0 || size_t(first + count) > n->cap) { set_error("ob_mlp_read_pairs: out of range"); return OB_ERR_INVALID; }
  MLP_TRY(cuda_ok(cudaDeviceSynchronize(), "ob_mlp_read_pairs"));
  return cuda_ok(cudaMemcpy(host, n->d_pairs + size_t(first) * PAIR, size_t(count) * PAIR * 4, cudaMemcpyDeviceToHost), "ob_mlp_read_pairs");
}

int ob_mlp_write_pairs(ObMlp* n, const float* host, long long count) {
  if (!n || !host || count < 0 || size_t(count) > n->cap) { set_error("ob_mlp_write_pairs: reserve a capacity first"); return OB_ERR_INVALID; }
  MLP_TRY(cuda_ok(cudaMemcpy(n->d_pairs, host, size_t(count) * PAIR * 4, cudaMemcpyHostToDevice), "ob_mlp_write_pairs"));
  const unsigned c = unsigned(count);
  return cuda_ok(cudaMemcpy(n->d_count, &c, 4, cudaMemcpyHostToDevice), "ob_mlp_write_pairs");
}

int ob_mlp_set_training(ObMlp* n, int mode) {
  if (!n || (mode != 0 && mode != 1)) { set_error("ob_mlp_set_training: mode must be 0 (fp32 SIMT) or 1 (bf16 tensor cores)"); return OB_ERR_INVALID; }
  n->train_mode = mode;
  return OB_OK;
}

// forward + backward on `count` host pairs in order: the batch loss and the gradient of every parameter
int ob_mlp_grad(ObMlp* n, const float* pairs, int count, double* loss, float* grad) {
  if (!n || !pairs || count < 1 || !loss || !grad) { set_error("ob_mlp_grad: bad arguments"); return OB_ERR_INVALID; }
  MLP_TRY(ensure_scratch(n, count));
  cudaStream_t s = n->stream;
  MLP_TRY(cuda_ok(cudaMemcpyAsync(n->hp, pairs, size_t(count) * PAIR * 4, cudaMemcpyHostToDevice, s), "ob_mlp_grad"));
  cudaMemsetAsync(n->d_loss, 0, 8, s);
  if (n->train_mode == 1 && count % 128 == 0) {
    if (!n->tct) n->tct = tc_trainer_new();
    MLP_TRY(tc_grad_run(n->tct, n->d_w, n->d_g, n->hp, count, n->norm, n->d_loss, s));
  } else {
    k_gather<<<(count + 127) / 128, 128, 0, s>>>(n->hp, nullptr, count, n->norm, n->X, n->T);
    forward(n, count);
    backward(n, count);
  }
  MLP_TRY(cuda_ok(cudaMemcpyAsync(grad, n->d_g, NPARAM * 4, cudaMemcpyDeviceToHost, s), "ob_mlp_grad"));
  MLP_TRY(cuda_ok(cudaMemcpyAsync(loss, n->d_loss, 8, cudaMemcpyDeviceToHost, s), "ob_mlp_grad"));
  return cuda_ok(cudaStreamSynchronize(s), "ob_mlp_grad");
}

// forward on `count` host pairs: the tendencies in physical units (count x OB_MLP_NOUT)
int ob_mlp_eval(ObMlp* n, const float* pairs, int count, float* out) {
  if (!n || !pairs || count < 1 || !out) { set_error("ob_mlp_eval: bad arguments"); return OB_ERR_INVALID; }
  MLP_TRY(ensure_scratch(n, count));
  cudaStream_t s = n->stream;
  MLP_TRY(cuda_ok(cudaMemcpyAsync(n->hp, pairs, size_t(count) * PAIR * 4, cudaMemcpyHostToDevice, s), "ob_mlp_eval"));
  k_gather<<<(count + 127) / 128, 128, 0, s>>>(n->hp, nullptr, count, n->norm, n->X, n->T);
  forward(n, count);
  std::vector<float> y(size_t(count) * NOUT);
  MLP_TRY(cuda_ok(cudaMemcpyAsync(y.data(), n->Y, y.size() * 4, cudaMemcpyDeviceToHost, s), "ob_mlp_eval"));
  MLP_TRY(cuda_ok(cudaStreamSynchronize(s), "ob_mlp_eval"));
  for (size_t i = 0; i < y.size(); i++) out[i] = y[i] * n->norm.out_scale[i % NOUT];
  return OB_OK;
}

// `steps` Adam steps, each on `batch` pairs drawn at random from the recorded pairs; mean loss over the steps
int ob_mlp_train(ObMlp* n, int batch, int steps, float lr, unsigned seed, double* mean_loss) {
  if (!n || batch < 1 || steps < 1 || !(lr > 0.f)) { set_error("ob_mlp_train: bad arguments"); return OB_ERR_INVALID; }
  long long cnt = 0;
  MLP_TRY(ob_mlp_pair_count(n, &cnt));
  if (cnt < 1) { set_error("ob_mlp_train: no recorded pairs"); return OB_ERR_INVALID; }
  cudaStream_t s = n->stream;
  if (n->train_mode == 1 && batch % 128 == 0) {
    if (!n->tct) n->tct = tc_trainer_new();
    cudaMemsetAsync(n->d_loss, 0, 8, s);
    MLP_TRY(tc_train_run(n->tct, n->d_w, n->d_g, n->d_m, n->d_v, n->adam_t, n->d_pairs, unsigned(cnt), n->norm, batch, steps, lr,
                         seed, n->d_loss, s));
    double l = 0.0;
    MLP_TRY(cuda_ok(cudaMemcpyAsync(&l, n->d_loss, 8, cudaMemcpyDeviceToHost, s), "ob_mlp_train"));
    MLP_TRY(cuda_ok(cudaStreamSynchronize(s), "ob_mlp_train"));
    if (mean_loss) *mean_loss = l / steps;
    return OB_OK;
  }
  MLP_TRY(ensure_scratch(n, batch));
  cudaMemsetAsync(n->d_loss, 0, 8, s);
  const float b1 = 0.9f, b2 = 0.999f;
  for (int st = 0; st < steps; st++) {
    k_draw<<<(batch + 255) / 256, 256, 0, s>>>(n->idx, batch, unsigned(cnt), unsigned(n->adam_t), seed);
    k_gather<<<(batch + 127) / 128, 128, 0, s>>>(n->d_pairs, n->idx, batch, n->norm, n->X, n->T);
    forward(n, batch);
    backward(n, batch);
    n->adam_t++;
    const float c1 = 1.f - std::pow(b1, float(n->adam_t)), c2 = 1.f - std::pow(b2, float(n->adam_t));
    k_adam<<<(NPARAM + 255) / 256, 256, 0, s>>>(n->d_w, n->d_g, n->d_m, n->d_v, NPARAM, lr, b1, b2, 1e-8f, c1, c2);
  }
  double l = 0.0;
  MLP_TRY(cuda_ok(cudaMemcpyAsync(&l, n->d_loss, 8, cudaMemcpyDeviceToHost, s), "ob_mlp_train"));
  MLP_TRY(cuda_ok(cudaStreamSynchronize(s), "ob_mlp_train"));
  if (mean_loss) *mean_loss = l / steps;
  return OB_OK;
}

}  // extern "C"

// internal: the pair buffer and counter a model records into, and what the surrogate copies for inference
namespace ob {
void mlp_record_target(ObMlp* n, float** buf, unsigned** count, unsigned* cap) {
  *buf = n ? n->d_pairs : nullptr;
  *count = n ? n->d_count : nullptr;
  *cap = n ? unsigned(std::min<size_t>(n->cap, 0xFFFFFFFFu)) : 0u;
}
const float* mlp_master(const ObMlp* n) { return n ? n->d_w : nullptr; }
const Norm* mlp_norm(const ObMlp* n) { return n ? &n->norm : nullptr; }
}  // namespace ob
