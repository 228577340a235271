// ob_poisson.cuh — the pressure-solve plan (solver.js:105-165) shared by the model and the standalone C ABI.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "../../include/ob.h"

namespace ob {

void set_error(const char* fmt, ...);

struct PoissonPlan {
  int nx = 0, ny = 0, nz = 0, precision = 0;  // 0 fp32 SIMT, 1 bf16x3 tensor core, 2 bf16x3 + one refinement,
                                              // 3 refinement in plain bf16, 4 two bf16x3 refinements,
                                              // 5 a plain-bf16 pass refined by one bf16x3 sweep
  bool presplit = false;  // precision >= 1: the caller writes the split right-hand side (tc_rhs_split) itself
  double dx = 0, dz = 0;
  float* mats = nullptr;  // qix | qx | qiy | qy (fp32, solver.js:115-125)
  size_t ofs_qix = 0, ofs_qx = 0, ofs_qiy = 0, ofs_qy = 0;
  float* lam = nullptr;   // eigenvalues (nx + ny)
  float4* zop = nullptr;  // (lo, up, diag, rho_c) per level
  float* tmp = nullptr;
  float* hat = nullptr;
  float* cpf = nullptr;   // Thomas scratch for nz without a register specialisation
  double* cpd = nullptr;  // FP64 low-mode scratch
  // bf16x3 tensor-core path (ob_dst_tc.cu)
  void* tc = nullptr;

  int create(int nx, int ny, int nz, double dx, double dz, int precision);
  int set_density(const float* rhoC, const float* rhoW);
  int solve(const float* rhs, float* phi, cudaStream_t s);  // precision 1: rhs == nullptr -> pre-split input
  void destroy();

  void gemm_x(const float* Mx, const float* src, float* dst, cudaStream_t s) const;
  void gemm_y(const float* My, const float* src, float* dst, cudaStream_t s) const;
  void tri(float* h, cudaStream_t s) const;
  int tc_create();
  int tc_factor_low();
  int tc_solve(const float* rhs, float* phi, cudaStream_t s);
  int tc_check();  // OB_ERR_TIMEOUT if a tensor-core pipeline wait gave up since the last check
  int tc_set_pairs(bool on);  // transforms on tiles of 256 rows computed by SM pairs (bit-identical results)
  bool tc_pairs() const;
  int tc_set_tile_widths(int bnx, int bny);  // outputs per transform tile (multiples of 16, 32..256; 0: automatic)
  // where a producer writes the split right-hand side (bf16 hi/lo, [nz][ny][ld], x fastest) for tc_solve(nullptr, ...)
  void tc_rhs_split(__nv_bfloat16** hi, __nv_bfloat16** lo, int* ld) const;
  void tc_destroy();
};

// FP64 residual norms of phi for rhs (device arrays) under the solve's operator: rel = {max |r| / max |rhs|,
// ||r||_2 / ||rhs||_2}; scratch holds 4 * 1024 + 4 doubles
int poisson_residual(const PoissonPlan& P, const float* rhs, const float* phi, double* scratch, double rel[2], cudaStream_t s);

// grouped solve of an ensemble: every member's solve in the same few launches (ob_dst_tc.cu). The plans use the
// tensor-core path with the split right-hand side written by their divergence pass, share nz and precision;
// phi[i] is member i's output, rhs[i] its fp32 right-hand side (precision 2).
struct TcGroup;
int tc_group_create(PoissonPlan* const* plans, float* const* phi, const float* const* rhs, int n, TcGroup** out);
int tc_group_set_cap(TcGroup* G, int bn_cap);  // widest transform tile (16..256, multiple of 16)
int tc_group_cap(const TcGroup* G);
void tc_group_set_ctas(TcGroup* G, int ctas);  // CTAs per transform launch (0: one per SM)
int tc_group_solve(TcGroup* G, cudaStream_t s);
int tc_group_check(TcGroup* G);
void tc_group_destroy(TcGroup* G);

}  // namespace ob
