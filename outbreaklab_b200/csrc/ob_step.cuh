// ob_step.cuh — host launchers of the step kernels (ob_step.cu) and the pressure solver (ob_poisson.cu).
#pragma once
#include <vector>

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
// hurricane mode: the winds the advection carries (WGSL_M_PREP), the 2-dx filter into V[1-par] and Q slot 1
void launch_prep(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_filt(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_div(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_proj(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s);
void launch_rain(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s);
void launch_maps(const Grid& g, const Uni& U, const Fields& F, int par, float4* out, cudaStream_t s);
// grouped launches: one launch of a pass over every member of an ensemble (members in constant memory, uploaded from
// a device copy; the launch's grid is (x-y blocks of all members, 1, levels) and a block map gives each x-y block its
// member and block coordinates)
enum { kGroupLSF = 0, kGroupCI, kGroupNUT, kGroupADVV1, kGroupADVV2, kGroupADVQ1, kGroupADVQ2, kGroupPHYS, kGroupDIV, kGroupPROJ,
       kGroupRAIN, kGroupPasses };
enum { kGroupStag = 0, kGroupCell = 1, kGroup2D = 2 };
int group_kind(int pass);
dim3 group_default_block(int pass);
bool group_block_fixed(int pass);
// host: the block map of one launch of a pass over the members with grids[0..n-1] at table positions pos[0..n-1];
// returns the launch's z extent (levels), or -1 when the members' nz differ
int group_map(const Grid* grids, const int* pos, int n, int pass, dim3 block, std::vector<uint2>& map);
// copies the member table (n members) into constant memory on stream s
int group_upload_members(const MemberC* d_src, int n, cudaStream_t s);
void launch_group(int pass, const uint2* map, int nxy, int Z, dim3 block, int par, cudaStream_t s, int micro_mode = 0);
void launch_tor_candidates(const Grid& g, float dx, const float4* maps, float zmin, float* out, int cap, unsigned* count, cudaStream_t s);
void launch_pack(const Grid& g, const Ptr8& src, int nch, int X, int Y, int Z, float* dst, cudaStream_t s);
void launch_unpack(const Grid& g, const Ptr8& dst, int nch, int X, int Y, int Z, const float* src, cudaStream_t s);

}  // namespace ob
