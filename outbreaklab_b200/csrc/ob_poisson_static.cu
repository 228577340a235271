// ob_poisson_static.cu — the pressure solve without any device allocation.
//
// Some hosts cannot call cudaMalloc: a plugin that runs inside another runtime's memory budget and has no right to
// grow it (a JavaScript engine's GPU process), or a real-time loop whose rules forbid blocking on the allocator once
// it has started.
// For them this file keeps the solver's working memory — the sine-transform matrices, eigenvalues, z-operator and
// the two intermediate spectra — in one file-scope device array of fixed size, and the entry point only launches
// kernels into it. The caller still owns and passes the right-hand side, the solution and the densities.
//
// Limits: nx, ny <= OB_STATIC_POISSON_MAX_SIDE, nz <= OB_STATIC_POISSON_MAX_NZ and nx*ny*nz <=
// OB_STATIC_POISSON_MAX_CELLS; the array (about 14 MB) is held by every GPU that loads the library until exit.
#include <cmath>
#include <mutex>

#include "ob_poisson.cuh"

namespace ob {

namespace {
constexpr size_t kMats = 4ull * OB_STATIC_POISSON_MAX_SIDE * OB_STATIC_POISSON_MAX_SIDE;
constexpr size_t kLam = 2ull * OB_STATIC_POISSON_MAX_SIDE;
constexpr size_t kZop = 4ull * OB_STATIC_POISSON_MAX_NZ;
constexpr size_t kCpd = 2ull * 8ull * OB_STATIC_POISSON_MAX_NZ;  // 8 * nz doubles, counted in floats
constexpr size_t kCells = size_t(OB_STATIC_POISSON_MAX_CELLS);
constexpr size_t round64(size_t n) { return (n + 63) / 64 * 64; }
constexpr size_t kOffLam = round64(kMats);
constexpr size_t kOffZop = kOffLam + round64(kLam);
constexpr size_t kOffCpd = kOffZop + round64(kZop);
constexpr size_t kOffTmp = kOffCpd + round64(kCpd);
constexpr size_t kOffHat = kOffTmp + kCells;
constexpr size_t kOffCpf = kOffHat + kCells;
constexpr size_t kTotal = kOffCpf + kCells;
}  // namespace

// The working memory. Host code must not hand this name to a kernel: on the host it is only a stand-in for the
// symbol, and its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) float g_poisson_scratch[kTotal];

// DST-II matrices (qix | qx | qiy | qy) and eigenvalues, the same values PoissonPlan::create computes on the host
__global__ void k_static_dst(int nx, int ny, double dx, float* mats, float* lam) {
  const size_t nxx = size_t(nx) * nx, nyy = size_t(ny) * ny;
  const size_t total = 2 * nxx + 2 * nyy;
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    int N;
    size_t base, e;
    bool inv;
    if (t < 2 * nxx) { N = nx; base = t < nxx ? 0 : nxx; e = t - base; inv = t < nxx; }
    else { N = ny; base = t < 2 * nxx + nyy ? 2 * nxx : 2 * nxx + nyy; e = t - base; inv = t < 2 * nxx + nyy; }
    // inv (forward) matrices are stored qi[l*N + i], the inverse ones q[i*N + l]; both hold v_l(i)
    const int r = int(e / N), c = int(e % N);
    const int l = inv ? r : c, i = inv ? c : r;
    const double cl = sqrt((l == N - 1 ? 1.0 : 2.0) / N);
    mats[t] = float(cl * sin(M_PI * (l + 1) * (i + 0.5) / N));
  }
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nx) { const double s = sin(M_PI * (t + 1) / (2.0 * nx)); lam[t] = float(-4.0 / (dx * dx) * s * s); }
  if (t < ny) { const double s = sin(M_PI * (t + 1) / (2.0 * ny)); lam[nx + t] = float(-4.0 / (dx * dx) * s * s); }
}

// z-operator from the caller's densities (solver.js:139-146)
__global__ void k_static_zop(int nz, double dz, const float* rhoC, const float* rhoW, float4* zop) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nz) return;
  const double a = 1.0 / (dz * dz);
  const double lo = k > 0 ? double(rhoW[k]) * a : 0.0, up = k < nz - 1 ? double(rhoW[k + 1]) * a : 0.0;
  zop[k] = make_float4(float(lo), float(up), float(-(lo + up)), rhoC[k]);
}

static std::mutex g_static_mu;
static float* g_static_ptr[256] = {};

}  // namespace ob

using namespace ob;

extern "C" int ob_poisson_solve_static(int nx, int ny, int nz, float dx, float dz, const float* d_rhoC, const float* d_rhoW,
                                       const float* d_rhs, float* d_phi, void* stream) {
  if (!d_rhoC || !d_rhoW || !d_rhs || !d_phi || !(dx > 0.f) || !(dz > 0.f)) {
    set_error("ob_poisson_solve_static: null pointer or non-positive spacing");
    return OB_ERR_INVALID;
  }
  if (nx < 2 || ny < 2 || nz < 2 || nx > OB_STATIC_POISSON_MAX_SIDE || ny > OB_STATIC_POISSON_MAX_SIDE ||
      nz > OB_STATIC_POISSON_MAX_NZ || double(nx) * ny * nz > double(OB_STATIC_POISSON_MAX_CELLS)) {
    set_error("ob_poisson_solve_static: %d x %d x %d exceeds the static limits (sides <= %d, nz <= %d, cells <= %d)",
              nx, ny, nz, OB_STATIC_POISSON_MAX_SIDE, OB_STATIC_POISSON_MAX_NZ, OB_STATIC_POISSON_MAX_CELLS);
    return OB_ERR_INVALID;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 256) {
    set_error("ob_poisson_solve_static: no current CUDA device (%s)", cudaGetErrorString(e));
    return OB_ERR_DEVICE;
  }
  float* base = nullptr;
  {
    // first call on this device: look up the array's device address (must happen before any stream capture)
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_ptr[dev]) {
      e = cudaGetSymbolAddress(reinterpret_cast<void**>(&base), g_poisson_scratch);
      if (e != cudaSuccess || !base) {
        set_error("ob_poisson_solve_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return OB_ERR_DEVICE;
      }
      g_static_ptr[dev] = base;
    }
    base = g_static_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // a plan whose every buffer points into the static array; nothing in the solve reads memory it has not first
  // written in the same call, so no part of the array has to start at zero
  PoissonPlan P;
  P.nx = nx; P.ny = ny; P.nz = nz; P.dx = dx; P.dz = dz; P.precision = 0;
  P.mats = base;
  P.ofs_qix = 0;
  P.ofs_qx = size_t(nx) * nx;
  P.ofs_qiy = 2 * size_t(nx) * nx;
  P.ofs_qy = 2 * size_t(nx) * nx + size_t(ny) * ny;
  P.lam = base + kOffLam;
  P.zop = reinterpret_cast<float4*>(base + kOffZop);
  P.cpd = reinterpret_cast<double*>(base + kOffCpd);
  P.tmp = base + kOffTmp;
  P.hat = base + kOffHat;
  P.cpf = base + kOffCpf;
  const size_t nmat = 2 * size_t(nx) * nx + 2 * size_t(ny) * ny;
  k_static_dst<<<int((nmat + 255) / 256), 256, 0, s>>>(nx, ny, double(dx), P.mats, P.lam);
  k_static_zop<<<(nz + 127) / 128, 128, 0, s>>>(nz, double(dz), d_rhoC, d_rhoW, P.zop);
  P.gemm_x(P.mats + P.ofs_qix, d_rhs, P.tmp, s);
  P.gemm_y(P.mats + P.ofs_qiy, P.tmp, P.hat, s);
  P.tri(P.hat, s);
  P.gemm_y(P.mats + P.ofs_qy, P.hat, P.tmp, s);
  P.gemm_x(P.mats + P.ofs_qx, P.tmp, d_phi, s);
  P.mats = nullptr;  // the plan does not own the array: keep destroy() away from it
  P.lam = P.tmp = P.hat = P.cpf = nullptr;
  P.zop = nullptr;
  P.cpd = nullptr;
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("ob_poisson_solve_static: launch failed: %s", cudaGetErrorString(e));
    return OB_ERR_DEVICE;
  }
  return OB_OK;
}
