// ob_poisson.cu — exact anelastic pressure solve on the padded grid (solver.js:1-165), sm_100a.
//
//   rho_c(z) lap_h(phi) + d/dz(rho_w(z) d phi/dz) = rhs,  phi = 0 beyond the lateral faces, Neumann at ground / lid.
//
// Orthonormal DST-II in x and y (four dense transforms), one tridiagonal per horizontal mode (l, m) in z.
//   precision 0: fp32 SIMT transforms (tiled GEMM, 64 x 64 tiles, fp32 FMA) — the reference's own precision;
//   precision 1: bf16x3 tensor-core transforms (ob_dst_tc.cu) with fp32 accumulation; 2: plus a bf16x3
//   refinement sweep on the FP64-accumulated residual; 3: that sweep in plain bf16.
// The tridiagonals: fp32 Thomas with the forward-sweep coefficients in registers for every mode except the lowest
// 2 x 2 modes, which are near-singular (Neumann in z, shift ~ -(pi/L)^2) and run in FP64.
#include <cstdio>
#include <cmath>
#include <vector>

#include "ob_poisson.cuh"

namespace ob {

// ---------------------------------------------------------------------------------------------------------------
// fp32 SIMT batched GEMM: C(r, c) = sum_q A(r, q) B(q, c), C column-major (ldc), generic strides for A and B
// ---------------------------------------------------------------------------------------------------------------
constexpr int GBM = 64, GBN = 64, GBK = 16;
__global__ void __launch_bounds__(256) k_gemm_f32(int M, int N, int K, const float* __restrict__ A, long sar, long saq,
                                                  const float* __restrict__ B, long sbq, long sbc, float* __restrict__ C,
                                                  long ldc, long bA, long bB, long bC) {
  __shared__ float As[GBK][GBM + 4];
  __shared__ float Bs[GBK][GBN + 4];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int r0 = blockIdx.x * GBM, c0 = blockIdx.y * GBN;
  A += bA * blockIdx.z;
  B += bB * blockIdx.z;
  C += bC * blockIdx.z;
  float acc[4][4] = {};
  for (int q0 = 0; q0 < K; q0 += GBK) {
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const int e = tid + 256 * s;
      int r, q;
      if (saq == 1) { q = e % GBK; r = e / GBK; } else { r = e % GBM; q = e / GBM; }
      const int gr = r0 + r, gq = q0 + q;
      As[q][r] = (gr < M && gq < K) ? __ldg(A + gr * sar + gq * saq) : 0.f;
      int c, qb;
      if (sbq == 1) { qb = e % GBK; c = e / GBK; } else { c = e % GBN; qb = e / GBN; }
      const int gc = c0 + c, gqb = q0 + qb;
      Bs[qb][c] = (gc < N && gqb < K) ? __ldg(B + gqb * sbq + gc * sbc) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int t = 0; t < 4; t++) { a[t] = As[kk][tx + 16 * t]; b[t] = Bs[kk][ty + 16 * t]; }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = r0 + tx + 16 * i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = c0 + ty + 16 * j;
      if (c < N) C[r + c * ldc] = acc[i][j];
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------
// tridiagonal solves per mode (solver.js:70-103); zop = (lo, up, diag, rho_c) per level
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool low_mode(int l, int m) { return l < 2 && m < 2; }

template <int NZ>
__global__ void __launch_bounds__(128) k_tri_f32(int nx, int ny, const float* __restrict__ lam, const float4* __restrict__ zop,
                                                 float* __restrict__ hat) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x, m = blockIdx.y;
  if (l >= nx || low_mode(l, m)) return;
  const float shift = __ldg(lam + l) + __ldg(lam + nx + m);
  const long sxy = long(nx) * ny;
  float* h = hat + l + long(nx) * m;
  float cp[NZ];
  float cprev = 0.f, dprev = 0.f;
#pragma unroll
  for (int k = 0; k < NZ; k++) {
    const float4 o = __ldg(zop + k);
    const float den = o.z + shift * o.w - o.x * cprev;
    cprev = o.y / den;
    dprev = (h[sxy * k] - o.x * dprev) / den;
    cp[k] = cprev;
    h[sxy * k] = dprev;
  }
  float above = dprev;
#pragma unroll
  for (int k = NZ - 2; k >= 0; k--) {
    above = h[sxy * k] - cp[k] * above;
    h[sxy * k] = above;
  }
}
// any nz: forward-sweep coefficients in a global scratch column
__global__ void k_tri_f32_any(int nx, int ny, int nz, const float* __restrict__ lam, const float4* __restrict__ zop,
                              float* __restrict__ hat, float* __restrict__ cpbuf) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x, m = blockIdx.y;
  if (l >= nx || low_mode(l, m)) return;
  const float shift = __ldg(lam + l) + __ldg(lam + nx + m);
  const long sxy = long(nx) * ny;
  float* h = hat + l + long(nx) * m;
  float* cp = cpbuf + l + long(nx) * m;
  float cprev = 0.f, dprev = 0.f;
  for (int k = 0; k < nz; k++) {
    const float4 o = __ldg(zop + k);
    const float den = o.z + shift * o.w - o.x * cprev;
    cprev = o.y / den;
    dprev = (h[sxy * k] - o.x * dprev) / den;
    cp[sxy * k] = cprev;
    h[sxy * k] = dprev;
  }
  float above = dprev;
  for (int k = nz - 2; k >= 0; k--) {
    above = h[sxy * k] - cp[sxy * k] * above;
    h[sxy * k] = above;
  }
}
// the lowest 2 x 2 modes in FP64 (one warp)
__global__ void k_tri_f64_low(int nx, int ny, int nz, const float* __restrict__ lam, const float4* __restrict__ zop,
                              float* __restrict__ hat, double* __restrict__ cpbuf) {
  const int t = threadIdx.x;
  const int l = t & 1, m = t >> 1;
  if (t >= 4 || l >= nx || m >= ny) return;
  const double shift = double(lam[l]) + double(lam[nx + m]);
  const long sxy = long(nx) * ny;
  float* h = hat + l + long(nx) * m;
  double* cp = cpbuf + t * nz;
  double* dd = cpbuf + 4 * nz + t * nz;
  double cprev = 0.0, dprev = 0.0;
  for (int k = 0; k < nz; k++) {
    const float4 o = zop[k];
    const double den = double(o.z) + shift * double(o.w) - double(o.x) * cprev;
    cprev = double(o.y) / den;
    dprev = (double(h[sxy * k]) - double(o.x) * dprev) / den;
    cp[k] = cprev;
    dd[k] = dprev;
  }
  double above = dprev;
  h[sxy * (nz - 1)] = float(above);
  for (int k = nz - 2; k >= 0; k--) {
    above = dd[k] - cp[k] * above;
    h[sxy * k] = float(above);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------------------------------------------
static int ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? OB_ERR_OOM : OB_ERR_DEVICE;
  }
  return OB_OK;
}

int PoissonPlan::create(int nx_, int ny_, int nz_, double dx_, double dz_, int precision_) {
  nx = nx_; ny = ny_; nz = nz_; dx = dx_; dz = dz_; precision = precision_;
  if (nx < 2 || ny < 2 || nz < 2 || nz > 4096) { set_error("poisson: bad size %d x %d x %d", nx, ny, nz); return OB_ERR_INVALID; }
  const size_t n = size_t(nx) * ny * nz;
  // DST-II matrices (solver.js:115-125), computed in f64 and stored f32 as the reference does
  std::vector<float> M(2 * size_t(nx) * nx + 2 * size_t(ny) * ny);
  auto dst = [&](int N, float* q, float* qi) {
    for (int i = 0; i < N; i++)
      for (int l = 0; l < N; l++) {
        const double c = std::sqrt((l == N - 1 ? 1.0 : 2.0) / N);
        const double v = c * std::sin(M_PI * (l + 1) * (i + 0.5) / N);
        q[size_t(i) * N + l] = float(v);
        qi[size_t(l) * N + i] = float(v);
      }
  };
  ofs_qix = 0;
  ofs_qx = size_t(nx) * nx;
  ofs_qiy = 2 * size_t(nx) * nx;
  ofs_qy = 2 * size_t(nx) * nx + size_t(ny) * ny;
  dst(nx, M.data() + ofs_qx, M.data() + ofs_qix);
  dst(ny, M.data() + ofs_qy, M.data() + ofs_qiy);
  std::vector<float> lamh(nx + ny);
  for (int l = 0; l < nx; l++) lamh[l] = float(-4.0 / (dx * dx) * std::pow(std::sin(M_PI * (l + 1) / (2.0 * nx)), 2));
  for (int m = 0; m < ny; m++) lamh[nx + m] = float(-4.0 / (dx * dx) * std::pow(std::sin(M_PI * (m + 1) / (2.0 * ny)), 2));
  int rc;
  if ((rc = ck(cudaMalloc(&mats, M.size() * sizeof(float)), "poisson mats"))) return rc;
  if ((rc = ck(cudaMalloc(&lam, lamh.size() * sizeof(float)), "poisson eig"))) return rc;
  if ((rc = ck(cudaMalloc(&zop, size_t(nz) * sizeof(float4)), "poisson zop"))) return rc;
  if ((rc = ck(cudaMalloc(&tmp, n * sizeof(float)), "poisson tmp"))) return rc;
  if ((rc = ck(cudaMalloc(&hat, n * sizeof(float)), "poisson hat"))) return rc;
  if ((rc = ck(cudaMalloc(&cpd, size_t(8) * nz * sizeof(double)), "poisson low-mode scratch"))) return rc;
  if (nz != 40 && nz != 80 && nz != 16) {
    if ((rc = ck(cudaMalloc(&cpf, n * sizeof(float)), "poisson tri scratch"))) return rc;
  }
  if ((rc = ck(cudaMemcpy(mats, M.data(), M.size() * sizeof(float), cudaMemcpyHostToDevice), "poisson upload"))) return rc;
  if ((rc = ck(cudaMemcpy(lam, lamh.data(), lamh.size() * sizeof(float), cudaMemcpyHostToDevice), "poisson upload"))) return rc;
  std::vector<float> rc1(nz, 1.f), rw1(nz + 1, 1.f);
  if ((rc = set_density(rc1.data(), rw1.data()))) return rc;
  if (precision >= 1) {
    if ((rc = tc_create())) return rc;
  }
  return OB_OK;
}

int PoissonPlan::set_density(const float* rhoC, const float* rhoW) {  // solver.js:139-146
  std::vector<float4> zo(nz);
  const double a = 1.0 / (dz * dz);
  for (int k = 0; k < nz; k++) {
    const double lo = k > 0 ? double(rhoW[k]) * a : 0.0, up = k < nz - 1 ? double(rhoW[k + 1]) * a : 0.0;
    zo[k] = make_float4(float(lo), float(up), float(-(lo + up)), rhoC[k]);
  }
  const int rc = ck(cudaMemcpy(zop, zo.data(), zo.size() * sizeof(float4), cudaMemcpyHostToDevice), "poisson setDensity");
  if (rc != OB_OK || !tc) return rc;
  return tc_factor_low();
}

void PoissonPlan::destroy() {
  tc_destroy();
  for (void* p : {(void*)mats, (void*)lam, (void*)zop, (void*)tmp, (void*)hat, (void*)cpf, (void*)cpd})
    if (p) cudaFree(p);
  mats = lam = tmp = hat = cpf = nullptr;
  zop = nullptr;
  cpd = nullptr;
}

// x-transform (solver.js mode 0): dst(l, col) = sum_i M(l, i) src(i, col), col = j + ny k
void PoissonPlan::gemm_x(const float* Mx, const float* src, float* dst, cudaStream_t s) const {
  const int cols = ny * nz;
  dim3 grid((nx + GBM - 1) / GBM, (cols + GBN - 1) / GBN, 1);
  k_gemm_f32<<<grid, 256, 0, s>>>(nx, cols, nx, Mx, nx, 1, src, 1, nx, dst, nx, 0, 0, 0);
}
// y-transform (mode 1), per plane k: dst(i, m) = sum_j src(i, j) M(m, j)
void PoissonPlan::gemm_y(const float* My, const float* src, float* dst, cudaStream_t s) const {
  dim3 grid((nx + GBM - 1) / GBM, (ny + GBN - 1) / GBN, nz);
  const long pl = long(nx) * ny;
  k_gemm_f32<<<grid, 256, 0, s>>>(nx, ny, ny, src, 1, nx, My, 1, ny, dst, nx, pl, 0, pl);
}
void PoissonPlan::tri(float* h, cudaStream_t s) const {
  dim3 grid((nx + 127) / 128, ny, 1);
  switch (nz) {
    case 16: k_tri_f32<16><<<grid, 128, 0, s>>>(nx, ny, lam, zop, h); break;
    case 40: k_tri_f32<40><<<grid, 128, 0, s>>>(nx, ny, lam, zop, h); break;
    case 80: k_tri_f32<80><<<grid, 128, 0, s>>>(nx, ny, lam, zop, h); break;
    default: k_tri_f32_any<<<grid, 128, 0, s>>>(nx, ny, nz, lam, zop, h, cpf); break;
  }
  k_tri_f64_low<<<1, 32, 0, s>>>(nx, ny, nz, lam, zop, h, cpd);
}

int PoissonPlan::solve(const float* rhs, float* phi, cudaStream_t s) {
  if (precision >= 1) return tc_solve(rhs, phi, s);
  gemm_x(mats + ofs_qix, rhs, tmp, s);
  gemm_y(mats + ofs_qiy, tmp, hat, s);
  tri(hat, s);
  gemm_y(mats + ofs_qy, hat, tmp, s);
  gemm_x(mats + ofs_qx, tmp, phi, s);
  return ck(cudaGetLastError(), "poisson solve launch");
}

}  // namespace ob
