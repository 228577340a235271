// ob_step.cuh — host launchers of the step kernels (ob_step.cu) and the pressure solver (ob_poisson.cu).
#pragma once
#include "ob_common.cuh"

namespace ob {

struct Ptr8 {
  float* p[8];
};

void launch_lsf(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s);
void launch_ci(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s);
void launch_init(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s);
void launch_nut(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_advv(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_advq(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_activity(const Grid& g, const Fields& F, cudaStream_t s);
// sponge tables of the physics pass (Fields::spz/slx/sly) for the uniforms' sponge parameters and the base state
void launch_tables(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s);
// microphysics modes of the physics pass
enum { kMicroPlain = 0, kMicroRecord = 1, kMicroSurrogate = 2 };
void launch_phys(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s, int micro_mode = kMicroPlain);
void launch_div(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_proj(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_rain(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s);
void launch_maps(const Grid& g, const Uni& U, const Fields& F, int par, float4* out, cudaStream_t s);
void launch_tor_candidates(const Grid& g, float dx, const float4* maps, float zmin, float* out, int cap, unsigned* count, cudaStream_t s);
void launch_pack(const Grid& g, const Ptr8& src, int nch, int X, int Y, int Z, float* dst, cudaStream_t s);
void launch_unpack(const Grid& g, const Ptr8& dst, int nch, int X, int Y, int Z, const float* src, cudaStream_t s);

}  // namespace ob
