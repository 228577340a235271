// ob_step.cu — the storm-model step kernels for sm_100a (one kernel per pass of model.js:1457-1472).
//
// Each kernel restates one WGSL pass of the reference (citations per kernel) over the structure-of-arrays layout of
// ob_common.cuh: one thread per texel, x fastest within a warp so that every stencil row is a coalesced 128-byte
// read, neighbours served from L1/L2. Semi-Lagrangian sampling is a software trilinear filter in fp32 (exact
// weights; WebGPU's hardware filter uses low-precision fixed-point weights, which are not reproduced).
#include <algorithm>
#include <vector>

#include "ob_common.cuh"
#include "ob_micro.cuh"
#include "ob_step.cuh"

namespace ob {

// members of the grouped launches (ensemble steps), uploaded by group_upload_members. A grouped launch's grid is
// (x-y blocks of all members, 1, levels): the members share nz, and blockIdx.x indexes a map that gives each x-y
// block its member and its block coordinates (one 8-byte load per thread, the same for the whole block).
__constant__ MemberC c_members[kMaxMembers];
#define OB_GROUP_RESOLVE                                                               \
  const uint2 gm__ = __ldg(map + blockIdx.x);                                         \
  const int mem = int(gm__.x), gbx = int(gm__.y & 0xffffu), gby = int(gm__.y >> 16u), \
            gbz = int(blockIdx.z);

// block coordinates: blockIdx for a launch over one model, or the (member, block) a grouped launch resolved
#define OB_BLOCKS_DIRECT const int BX = blockIdx.x, BY = blockIdx.y, BZ = blockIdx.z;
#define OB_TEXEL_LOOP_BEGIN(XMAX, YMAX, ZMAX)             \
  const int ci = BX * blockDim.x + threadIdx.x;           \
  const int cj = BY * blockDim.y + threadIdx.y;           \
  const int ck = BZ;                                      \
  if (ci > (XMAX) || cj > (YMAX) || ck > (ZMAX)) return;

// ---------------------------------------------------------------------------------------------------------------
// target state (model.js:121-134)
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ float tprof(float z, float H) { return 1.f - sstep(0.7f * H, 1.15f * H, z); }
__device__ __forceinline__ float4 l2d(const float4* __restrict__ m, const Grid& g, int i, int j) {
  return __ldg(m + clampi(j, 0, g.ny - 1) * g.nx + clampi(i, 0, g.nx - 1));
}
__device__ __forceinline__ float tgtTh(const float* B, const Grid& g, float dz, float4 A, int k) {
  float z = (float(k) + 0.5f) * dz;
  return bsA(B, g.nz, k).x + A.x / bsB(B, g.nz, k).x * tprof(z, A.y);
}
__device__ __forceinline__ float tgtQv(const float* B, const Grid& g, float dz, float4 A, int k) {
  float z = (float(k) + 0.5f) * dz;
  return bsA(B, g.nz, k).y * (1.f - A.z * tprof(z, A.w));
}
// with no boundary air masses (LSF over zero boundaries gives lsfA = (0, 100, 0, 100), lsfB = (0, 0, 100, 0) and
// phi_t = +-0), every target expression below reduces exactly to the base state: x + 0 * t == x, qv0 * (1 - 0 * t)
// == qv0, and +-0 differences of phi_t change nothing. The BND = false instantiations skip those loads.
template <bool BND>
__device__ __forceinline__ float tgtUb(const Fields& F, const Grid& g, float dz, int i, int j, int k);
template <bool BND>
__device__ __forceinline__ float tgtVb(const Fields& F, const Grid& g, float dz, int i, int j, int k);
__device__ __forceinline__ float tgtU(const Fields& F, const Grid& g, float dz, int i, int j, int k) {
  float z = (float(k) + 0.5f) * dz;
  float4 a = l2d(F.lsfB, g, i - 1, j), b = l2d(F.lsfB, g, i, j);
  return bsB(F.B, g.nz, k).z + 0.5f * (a.x * tprof(z, a.z) + b.x * tprof(z, b.z));
}
__device__ __forceinline__ float tgtV(const Fields& F, const Grid& g, float dz, int i, int j, int k) {
  float z = (float(k) + 0.5f) * dz;
  float4 a = l2d(F.lsfB, g, i, j - 1), b = l2d(F.lsfB, g, i, j);
  return bsB(F.B, g.nz, k).w + 0.5f * (a.y * tprof(z, a.z) + b.y * tprof(z, b.z));
}

template <>
__device__ __forceinline__ float tgtUb<true>(const Fields& F, const Grid& g, float dz, int i, int j, int k) { return tgtU(F, g, dz, i, j, k); }
template <>
__device__ __forceinline__ float tgtUb<false>(const Fields& F, const Grid& g, float, int, int, int k) { return bsB(F.B, g.nz, k).z; }
template <>
__device__ __forceinline__ float tgtVb<true>(const Fields& F, const Grid& g, float dz, int i, int j, int k) { return tgtV(F, g, dz, i, j, k); }
template <>
__device__ __forceinline__ float tgtVb<false>(const Fields& F, const Grid& g, float, int, int, int k) { return bsB(F.B, g.nz, k).w; }

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_LSF (model.js:142-244): per column, target anomalies of the boundaries' air masses + hydrostatic phi_t
// ---------------------------------------------------------------------------------------------------------------
__device__ void bpt(const float* bd, int i, float t, float& x, float& y) {
  const float* q = bd + 20 + 4 * i;
  x = q[0] + q[2] * t;
  y = q[1] + q[3] * t;
}
__device__ __forceinline__ void lsf_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  const int i = BX * blockDim.x + threadIdx.x, j = BY * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const float dx = U.dims.w, t = float(__ldg(F.clock));
  const float x = (float(i) + 0.5f) * dx, y = (float(j) + 0.5f) * dx;
  float sT = 0, sH = 0, sQ = 0, sHq = 0, sU = 0, sV = 0, sHw = 0, sw = 0, nud = 0;
  const int nb = int(U.cor.z);
  for (int b = 0; b < nb; b++) {
    const float* bd = F.bnd + b * 148;
    // signed distance to the moving polyline (model.js:157-179)
    const int np = int(bd[0]);
    float best = 1e30f, sg = 1.f, over = 0.f, along = 0.f, s0 = 0.f;
    for (int s = 0; s < np - 1; s++) {
      float ax, ay, ex, ey;
      bpt(bd, s, t, ax, ay);
      bpt(bd, s + 1, t, ex, ey);
      float abx = ex - ax, aby = ey - ay;
      float la = fmaxf(sqrtf(abx * abx + aby * aby), 1.f);
      float t0 = ((x - ax) * abx + (y - ay) * aby) / (la * la);
      float tt = t0;
      if (s > 0) tt = fmaxf(tt, 0.f);
      if (s < np - 2) tt = fminf(tt, 1.f);
      float ddx = x - (ax + tt * abx), ddy = y - (ay + tt * aby);
      float d = sqrtf(ddx * ddx + ddy * ddy);
      if (d < best) {
        best = d;
        sg = (abx * (y - ay) - aby * (x - ax) > 0.f) ? 1.f : -1.f;
        over = (s == 0 ? fmaxf(-t0, 0.f) * la : 0.f) + (s == np - 2 ? fmaxf(t0 - 1.f, 0.f) * la : 0.f);
        along = s0 + tt * la;
      }
      s0 += la;
    }
    const float d = best * sg * bd[15];
    const float w = sstep(-bd[3], bd[3], d) * (1.f - sstep(0.f, 60000.f, over));
    if (w <= 0.f) continue;
    const float vr = bd[16];
    const float fade = 1.f - sstep(30000.f, 90000.f, d);
    // along-front variation (model.js:183-187) and hot spots (model.js:191-206)
    float avv = 0.f;
    if (bd[16] > 0.f) avv = clampf(fbm2(along / bd[18], bd[17] + t / 5400.f, 2) * 1.6f, -1.f, 1.f);
    const float av = vr * avv * fade;
    float lift = 1.f;
    if (vr > 0.f) {
      const float L = bd[18];
      const int sd = int(bd[17] * 1000.f);
      const float ph = t / 4800.f;
      const int e = int(floorf(ph));
      const float fe = sstep(0.f, 1.f, ph - floorf(ph));
      const int k0 = int(floorf(along / L));
      float acc = 0.f;
      for (int k = k0 - 1; k <= k0 + 1; k++)
        for (int q = 0; q < 2; q++) {
          uint32_t h = hash3i(k, e + q, sd);
          float r1 = float(h & 0xffffu) / 65535.f, r2 = float((h >> 16u) & 0xffffu) / 65535.f;
          float z = (along - (float(k) + 0.5f + 0.7f * (r1 - 0.5f)) * L) / (0.17f * L);
          acc += (q == 1 ? fe : 1.f - fe) * (0.35f + 0.65f * r2) * expf(-z * z);
        }
      lift = mixf(1.f, mixf(1.f - 0.85f * vr, 1.f + 1.3f * vr, clampf(acc, 0.f, 1.f)), fade);
    }
    const float Hmin = bd[7] * clampf(lift, 0.15f, 3.f);
    const float H = fminf(fmaxf(bd[6] * fmaxf(d + bd[3], 0.f) * (1.f + 0.4f * av), Hmin), bd[5]);
    sT += w * bd[4] * expf(0.5f * av);
    sQ += w * bd[8];
    sU += w * bd[10] * lift;
    sV += w * bd[11] * lift;
    sH += w * H;
    sHq += w * H * bd[9];
    sHw += w * H * bd[12];
    sw += w;
    nud = fmaxf(nud, bd[13] * sstep(bd[14], bd[14] + 40000.f, d) * (1.f - sstep(0.f, 60000.f, over)));
  }
  const float iw = 1.f / fmaxf(sw, 1e-6f);
  const float4 A = make_float4(clampf(sT, -20.f, 10.f), fmaxf(sH * iw, 100.f), clampf(sQ, 0.f, 0.92f), fmaxf(sHq * iw, 100.f));
  F.lsfA[j * g.nx + i] = A;
  F.lsfB[j * g.nx + i] = make_float4(sU, sV, fmaxf(sHw * iw, 100.f), nud);
  const float dz = U.dzv.x;
  float ph = 0.f, bprev = 0.f;
  for (int k = g.nz - 1; k >= 0; k--) {
    const float z = (float(k) + 0.5f) * dz;
    const float4 a = bsA(F.B, g.nz, k), bb = bsB(F.B, g.nz, k);
    const float dth = A.x / bb.x * tprof(z, A.y);
    const float dqv = -a.y * A.z * tprof(z, A.w);
    const float bt = 9.81f * (dth / a.x + 0.608f * dqv);
    if (k == g.nz - 1) ph = -bt * 0.5f * dz;
    else ph -= 0.5f * (bt + bprev) * dz;
    bprev = bt;
    F.phT[g.at(i, j, k)] = ph;
  }
}
__global__ void k_lsf(Grid g, Uni U, Fields F) { lsf_body(g, U, F, 0, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void k_lsf_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  {
    const double t = *c_members[mem].F.clock, t0 = *c_members[mem].lsfT;
    if (!(t - t0 >= 60.0 || t == 0.0)) return;
  }
  lsf_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_CI (model.js:249-281): strongest active updraft-nudging event per column
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void ci_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  const int i = BX * blockDim.x + threadIdx.x, j = BY * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const float dx = U.dims.w, t = float(__ldg(F.clock));
  const float x = (float(i) + 0.5f) * dx, y = (float(j) + 0.5f) * dx;
  float4 best = make_float4(0.f, 0.f, 1500.f, 1500.f);
  const int ne = int(U.ci.x);
  for (int e = 0; e < ne; e++) {
    const float* E = F.ci + e * 12;
    if (t < E[6] || t > E[7]) continue;
    const float dxv = x - (E[0] + E[8] * (t - E[6])), dyv = y - (E[1] + E[9] * (t - E[6]));
    const float ang = atan2f(dyv, dxv);
    const float wob = 1.f + 0.25f * gnoise2(cosf(ang) * 1.6f + E[10], sinf(ang) * 1.6f + 3.7f * E[10]);
    const float gg = sstep(E[6], E[6] + fmaxf(E[11], 60.f), t);
    const float r = sqrtf(dxv * dxv + dyv * dyv) / (E[3] * wob * (0.35f + 0.65f * gg));
    if (r >= 1.f) continue;
    const float Lx = float(g.nx) * dx, Ly = float(g.ny) * dx;
    const float edge = fminf(fminf(x, Lx - x), fminf(y, Ly - y));
    const float h = sstep(E[6], E[6] + 60.f, t) * (1.f - sstep(E[7] - 180.f, E[7], t)) * sstep(U.sponge.x, U.sponge.x + 10000.f, edge);
    const float wt = E[5] * (0.4f + 0.6f * gg) * cosf(1.5707963f * r);
    if (h * wt > best.x * best.y) best = make_float4(h, wt, E[2], E[4]);
  }
  F.ciMap[j * g.nx + i] = best;
}
__global__ void k_ci(Grid g, Uni U, Fields F) { ci_body(g, U, F, 0, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void k_ci_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  if (gbx == 0 && gby == 0 && gbz == 0 && threadIdx.x == 0 && threadIdx.y == 0) {  // after the LSF pass of this step
    const double t = *c_members[mem].F.clock;
    double* t0 = c_members[mem].lsfT;
    if (t - *t0 >= 60.0 || t == 0.0) *t0 = t;
    if (c_members[mem].micro == kMicroSurrogate) {  // this step's surrogate queue and fallback count start empty
      c_members[mem].F.mlp_count[0] = 0u;
      c_members[mem].F.mlp_count[1] = 0u;
    }
  }
  ci_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_INIT (model.js:284-339), outbreak mode (no vortex)
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_init(Grid g, Uni U, Fields F) {
  OB_BLOCKS_DIRECT
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  const int k = min(ck, g.nz - 1);
  const float dz = U.dzv.x;
  const float4 A = l2d(F.lsfA, g, ci, cj);
  const float z = (float(k) + 0.5f) * dz;
  const float dx = U.dims.w;
  const bool vortex = U.vtx2.z > 0.5f && F.vx;
  float nz0 = sstep(800.f, 1500.f, z);
  // hurricane mode: the noise reaches up through the moist core (model.js:306-309)
  if (U.vtx2.z > 0.5f) {
    const float px = (float(ci) + 0.5f) * dx - U.vtx.x, py = (float(cj) + 0.5f) * dx - U.vtx.y;
    nz0 = sqrtf(px * px + py * py) < U.vtx2.x ? sstep(6000.f, 8000.f, z) : 1.f;
  }
  const float noise = U.misc.z * (rnd3(ci + 17, cj + 3, ck + 5) - 0.5f) * 2.f * (1.f - nz0);
  float th = tgtTh(F.B, g, dz, A, k) + noise;
  float u = (cj < g.ny && ck < g.nz) ? tgtU(F, g, dz, ci, cj, k) : 0.f;
  float v = (ci < g.nx && ck < g.nz) ? tgtV(F, g, dz, ci, cj, k) : 0.f;
  // the vortex table at radius r (model.js:292-297): (tangential wind, theta')
  auto vxAt = [&](float r) {
    const int nr = int(U.vtx.w);
    const float fr = r / U.vtx.z;
    const int i0 = int(floorf(fr));
    if (i0 >= nr - 1) return make_float2(0.f, 0.f);
    const int q = clampi(k, 0, g.nz - 1) * nr + i0;
    const float4 a = __ldg(F.vx + q), b = __ldg(F.vx + q + 1);
    const float t = fr - float(i0);
    return make_float2(a.x * (1.f - t) + b.x * t, a.y * (1.f - t) + b.y * t);
  };
  if (vortex) {  // a warm-core vortex in gradient-wind and hydrostatic balance (model.js:314-325)
    const float pux = float(ci) * dx - U.vtx.x, puy = (float(cj) + 0.5f) * dx - U.vtx.y;
    const float ru = fmaxf(sqrtf(pux * pux + puy * puy), 1.f);
    const float pvx = (float(ci) + 0.5f) * dx - U.vtx.x, pvy = float(cj) * dx - U.vtx.y;
    const float rv = fmaxf(sqrtf(pvx * pvx + pvy * pvy), 1.f);
    const float pcx = (float(ci) + 0.5f) * dx - U.vtx.x, pcy = (float(cj) + 0.5f) * dx - U.vtx.y;
    const float rc = sqrtf(pcx * pcx + pcy * pcy);
    u -= vxAt(ru).x * puy / ru;
    v += vxAt(rv).x * pvx / rv;
    th += vxAt(rc).y;
  }
  const float T = th * bsB(F.B, g.nz, k).x;
  float qv = fminf(tgtQv(F.B, g, dz, A, k), 0.95f * qvsat(T, bsB(F.B, g.nz, k).y, fIce(T)));
  if (vortex) {  // a nearly saturated core at the same density (model.js:328-335)
    const float pcx = (float(ci) + 0.5f) * dx - U.vtx.x, pcy = (float(cj) + 0.5f) * dx - U.vtx.y;
    const float f = (1.f - sstep(0.6f, 1.f, sqrtf(pcx * pcx + pcy * pcy) / U.vtx2.x)) * sstep(500.f, 1500.f, z) *
                    (1.f - sstep(7000.f, 10000.f, z));
    const float q2 = fmaxf(qv, f * U.vtx2.y * qvsat(T, bsB(F.B, g.nz, k).y, fIce(T)));
    const float dqv = q2 - qv;
    qv = q2;
    th -= 0.608f * dqv * bsA(F.B, g.nz, k).x;
  }
  const int o = g.at(ci, cj, ck);
  for (int p = 0; p < 2; p++) {  // both ping-pong slots (reset copies V0 to V1, model.js:1437)
    F.V[p][0][o] = u;
    F.V[p][1][o] = v;
    F.V[p][2][o] = 0.f;
    F.V[p][3][o] = th;
  }
  if (ci < g.nx && cj < g.ny && ck < g.nz) {
    F.Q[0][0][o] = qv;
#pragma unroll
    for (int c = 1; c < 8; c++) F.Q[0][c][o] = 0.f;
  }
}

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_NUT (model.js:342-389): Smagorinsky-Lilly viscosities with the Richardson correction
// ---------------------------------------------------------------------------------------------------------------
template <bool HUR = false>
__device__ __forceinline__ void nut_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  OB_TEXEL_LOOP_BEGIN(g.nx - 1, g.ny - 1, g.nz - 1)
  // a cell's +1 neighbours on the staggered box always exist; the -1 ones clamp to the edge (offset 0)
  const int o = g.at(ci, cj, ck);
  const int xm = ci > 0 ? -1 : 0, ym = cj > 0 ? -g.px : 0, zm = ck > 0 ? -g.plane : 0;
  const int xp = 1, yp = g.px, zp = g.plane;
  const float* __restrict__ u = F.V[par][0] + o;
  const float* __restrict__ v = F.V[par][1] + o;
  const float* __restrict__ w = F.V[par][2] + o;
  const float* __restrict__ th = F.V[par][3] + o;
  const float u0m = bsB(F.B, g.nz, ck - 1).z, u00 = bsB(F.B, g.nz, ck).z, u0p = bsB(F.B, g.nz, ck + 1).z;
  const float v0m = bsB(F.B, g.nz, ck - 1).w, v00 = bsB(F.B, g.nz, ck).w, v0p = bsB(F.B, g.nz, ck + 1).w;
  auto uc = [&](int off, float u0) { return 0.5f * (__ldg(u + off) + __ldg(u + off + xp)) - u0; };
  auto vc = [&](int off, float v0) { return 0.5f * (__ldg(v + off) + __ldg(v + off + yp)) - v0; };
  auto wc = [&](int off) { return 0.5f * (__ldg(w + off) + __ldg(w + off + zp)); };
  const float dx = U.dims.w, dz = U.dzv.x;
  // differences times the correctly rounded reciprocals 1/dx, 1/dz (and their exact halves) instead of divisions
  const float idx = U.dzv.y, idz = U.dzv.z, ih2x = 0.5f * idx, ih2z = 0.5f * idz;
  const float dudx = (__ldg(u + xp) - __ldg(u)) * idx;
  const float dvdy = (__ldg(v + yp) - __ldg(v)) * idx;
  const float dwdz = (__ldg(w + zp) - __ldg(w)) * idz;
  const float dudy = (uc(yp, u00) - uc(ym, u00)) * ih2x, dudz = (uc(zp, u0p) - uc(zm, u0m)) * ih2z;
  const float dvdx = (vc(xp, v00) - vc(xm, v00)) * ih2x, dvdz = (vc(zp, v0p) - vc(zm, v0m)) * ih2z;
  const float dwdx = (wc(xp) - wc(xm)) * ih2x, dwdy = (wc(yp) - wc(ym)) * ih2x;
  const float s12 = 0.5f * (dudy + dvdx), s13 = 0.5f * (dudz + dwdx), s23 = 0.5f * (dvdz + dwdy);
  const float S2 = 2.f * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + 4.f * (s12 * s12 + s13 * s13 + s23 * s23);
  const int kz0 = max(ck - 1, 0), kz1 = min(ck + 1, g.nz - 1);
  float N2 = 9.81f / bsA(F.B, g.nz, ck).x * (__ldg(th + (kz1 - ck) * g.plane) - __ldg(th + (kz0 - ck) * g.plane)) / (float(kz1 - kz0) * dz);
  if (U.cor.w > 0.5f && __ldg(F.Q[0][1] + o) + __ldg(F.Q[0][2] + o) > 1e-5f) N2 = fminf(N2, 0.f);
  const float Ri = N2 / fmaxf(S2, 1e-10f);
  const float fst = sqrtf(fmaxf(0.f, 1.f - Ri / 0.33f));
  const float sS = sqrtf(fmaxf(S2, 0.f));
  const float lh = U.turb.x * dx, lv = 0.18f * dz;
  const float dtc = fmaxf(U.step.x, 0.1f);
  F.aux[0][o] = fminf(lh * lh * sS * fst, 0.08f * dx * dx / dtc);
  float nuv = fminf(lv * lv * sS * fst, 0.15f * dz * dz / dtc);
  if (HUR) {  // hurricane mode: a K-profile boundary layer (model.js:377-386)
    const float zc = (float(ck) + 0.5f) * dz, h = U.hur2.z;
    if (zc < h) {
      const int o0 = g.at(ci, cj, 0);
      const float ua = 0.5f * (__ldg(F.V[par][0] + o0) + __ldg(F.V[par][0] + o0 + 1));
      const float va = 0.5f * (__ldg(F.V[par][1] + o0) + __ldg(F.V[par][1] + o0 + g.px));
      const float u1 = sqrtf(ua * ua + va * va);
      const float ust = sqrtf(cdSfc(U, u1, __ldg(F.sfc + cj * g.nx + ci).x)) * fmaxf(u1, U.hur3.y);
      const float q = 1.f - zc / h;
      nuv = fmaxf(nuv, fminf(0.4f * ust * zc * q * q, 0.15f * dz * dz / dtc));
    }
  }
  F.aux[1][o] = nuv;
}
__global__ void __launch_bounds__(128, 16) k_nut(Grid g, Uni U, Fields F, int par) { nut_body(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void k_nut_hur(Grid g, Uni U, Fields F, int par) { nut_body<true>(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void __launch_bounds__(128, 12) k_nut_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  nut_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---------------------------------------------------------------------------------------------------------------
// advection of the winds and theta (model.js:391-481)
// ---------------------------------------------------------------------------------------------------------------
struct Loc {
  float vu[3], vv[3], vw[3], vc[3];
};
__device__ __forceinline__ Loc localVel(const Fields& F, const Grid& g, int par, int i, int j, int k) {
  // clamp-to-edge neighbour offsets of the staggered box, once per texel
  const int o = g.at(i, j, k);
  const int xm = i > 0 ? -1 : 0, xp = i < g.nx ? 1 : 0;
  const int ym = j > 0 ? -g.px : 0, yp = j < g.ny ? g.px : 0;
  const int zm = k > 0 ? -g.plane : 0, zp = k < g.nz ? g.plane : 0;
  const float* __restrict__ u = F.V[par][0] + o;
  const float* __restrict__ v = F.V[par][1] + o;
  const float* __restrict__ w = F.V[par][2] + o;
  Loc L;
  const float pu = __ldg(u), pv = __ldg(v), pw = __ldg(w);
  const float xpu = __ldg(u + xp), ypv = __ldg(v + yp), zpw = __ldg(w + zp);
  L.vu[0] = pu;
  L.vu[1] = 0.25f * (__ldg(v + xm) + pv + __ldg(v + xm + yp) + ypv);
  L.vu[2] = 0.25f * (__ldg(w + xm) + pw + __ldg(w + xm + zp) + zpw);
  L.vv[0] = 0.25f * (__ldg(u + ym) + pu + __ldg(u + xp + ym) + xpu);
  L.vv[1] = pv;
  L.vv[2] = 0.25f * (__ldg(w + ym) + pw + __ldg(w + ym + zp) + zpw);
  L.vw[0] = 0.25f * (__ldg(u + zm) + pu + __ldg(u + xp + zm) + xpu);
  L.vw[1] = 0.25f * (__ldg(v + zm) + pv + __ldg(v + yp + zm) + ypv);
  L.vw[2] = pw;
  L.vc[0] = 0.5f * (pu + xpu);
  L.vc[1] = 0.5f * (pv + ypv);
  L.vc[2] = 0.5f * (pw + zpw);
  return L;
}
// departure (s = 1) or forward (s = -1) point, first-order trace clamped to the box (model.js:428-432)
__device__ __forceinline__ void traceV(const Grid& g, const float k[3], float px, float py, float pz, const float v[3], float s,
                                       float& x, float& y, float& z) {
  x = clampf(px - s * k[0] * v[0], 0.f, float(g.nx));
  y = clampf(py - s * k[1] * v[1], 0.f, float(g.ny));
  z = clampf(pz - s * k[2] * v[2], 0.f, float(g.nz));
}
// channel sample at a point in grid units (texel offsets of u, v, w, theta: model.js:419-422)
__device__ __forceinline__ float sampleVch(const float* f, const Grid& g, int ch, float x, float y, float z) {
  const float ox = ch == 0 ? 0.f : 0.5f, oy = ch == 1 ? 0.f : 0.5f, oz = ch == 2 ? 0.f : 0.5f;
  return trilerpB(f, g, g.nx + 1, g.ny + 1, g.nz + 1, x - ox, y - oy, z - oz);
}

// the departure-point sample of a channel, with the min / max of its 8 texels (ADVV2's limiter window: the
// reference's limiter traces the same point, model.js:455-479)
__device__ __forceinline__ void sampleVch_mm(const Fields& F, const Grid& g, int par, int ch, int o, float x, float y, float z) {
  const float ox = ch == 0 ? 0.f : 0.5f, oy = ch == 1 ? 0.f : 0.5f, oz = ch == 2 ? 0.f : 0.5f;
  float lo, hi;
  F.Vt[ch][o] = trilerpB_mm(F.V[par][ch], g, g.nx + 1, g.ny + 1, g.nz + 1, x - ox, y - oy, z - oz, lo, hi);
  F.Vlo[ch][o] = lo;
  F.Vhi[ch][o] = hi;
}
__device__ __forceinline__ void advv1_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  const Loc L = localVel(F, g, par, ci, cj, ck);
  const float kk[3] = {U.der.x, U.der.x, U.der.y};  // dt/dx, dt/dx, dt/dz
  const float fi = float(ci), fj = float(cj), fk = float(ck);
  const int o = g.at(ci, cj, ck);
  float x, y, z;
  traceV(g, kk, fi, fj + 0.5f, fk + 0.5f, L.vu, 1.f, x, y, z);
  sampleVch_mm(F, g, par, 0, o, x, y, z);
  traceV(g, kk, fi + 0.5f, fj, fk + 0.5f, L.vv, 1.f, x, y, z);
  sampleVch_mm(F, g, par, 1, o, x, y, z);
  traceV(g, kk, fi + 0.5f, fj + 0.5f, fk, L.vw, 1.f, x, y, z);
  sampleVch_mm(F, g, par, 2, o, x, y, z);
  traceV(g, kk, fi + 0.5f, fj + 0.5f, fk + 0.5f, L.vc, 1.f, x, y, z);
  sampleVch_mm(F, g, par, 3, o, x, y, z);
}
__global__ void k_advv1(Grid g, Uni U, Fields F, int par) { advv1_body(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void k_advv1_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  advv1_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

__device__ __forceinline__ float2 minmax8V(const float* __restrict__ f, const Grid& g, float x, float y, float z, float ox, float oy, float oz) {
  // the trace is clamped to the box, so each floor index lies in [-1, n] and one bound per corner clamps it
  const int i0 = __float2int_rd(x - ox), j0 = __float2int_rd(y - oy), k0 = __float2int_rd(z - oz);
  const int ia = max(i0, 0), ib = min(i0 + 1, g.nx), ja = max(j0, 0), jb = min(j0 + 1, g.ny), ka = max(k0, 0), kb = min(k0 + 1, g.nz);
  float lo = 1e30f, hi = -1e30f;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const float s = __ldg(f + g.at((q & 1) ? ib : ia, ((q >> 1) & 1) ? jb : ja, (q >> 2) ? kb : ka));
    lo = fminf(lo, s);
    hi = fmaxf(hi, s);
  }
  return make_float2(lo, hi);
}

__device__ __forceinline__ void advv2_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  const Loc L = localVel(F, g, par, ci, cj, ck);
  const float kk[3] = {U.der.x, U.der.x, U.der.y};  // dt/dx, dt/dx, dt/dz
  const float fi = float(ci), fj = float(cj), fk = float(ck);
  const float P[4][3] = {{fi, fj + 0.5f, fk + 0.5f}, {fi + 0.5f, fj, fk + 0.5f}, {fi + 0.5f, fj + 0.5f, fk}, {fi + 0.5f, fj + 0.5f, fk + 0.5f}};
  const float* vel[4] = {L.vu, L.vv, L.vw, L.vc};
  const float cx = L.vc[0] * kk[0], cy = L.vc[1] * kk[1], cz = L.vc[2] * kk[2];
  const float cour = sqrtf(cx * cx + cy * cy + cz * cz);
  const float sm = 0.5f * U.misc.y * clampf(cour / 0.35f, U.dzv.w, 1.f);
  const int o = g.at(ci, cj, ck);
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float x, y, z;
    traceV(g, kk, P[c][0], P[c][1], P[c][2], vel[c], -1.f, x, y, z);
    const float b = sampleVch(F.Vt[c], g, c, x, y, z);
    const float hat = __ldg(F.Vt[c] + o), old = __ldg(F.V[par][c] + o);
    const float r = hat + sm * (old - b);
    F.V[1 - par][c][o] = clampf(r, __ldg(F.Vlo[c] + o), __ldg(F.Vhi[c] + o));
  }
}
__global__ void __launch_bounds__(128, 12) k_advv2(Grid g, Uni U, Fields F, int par) { advv2_body(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void __launch_bounds__(128, 10) k_advv2_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  advv2_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---------------------------------------------------------------------------------------------------------------
// scalar advection with fall speeds (model.js:482-576)
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void cellVel(const Fields& F, const Grid& g, int par, int i, int j, int k, float v[3]) {
  const int o = g.at(i, j, k);
  v[0] = 0.5f * (__ldg(F.V[par][0] + o) + __ldg(F.V[par][0] + o + 1));
  v[1] = 0.5f * (__ldg(F.V[par][1] + o) + __ldg(F.V[par][1] + o + g.px));
  v[2] = 0.5f * (__ldg(F.V[par][2] + o) + __ldg(F.V[par][2] + o + g.plane));
}
__device__ __forceinline__ void traceQ(const Grid& g, const float k[3], const float p[3], const float v[3], float fall, float s,
                                       float& x, float& y, float& z) {
  x = clampf(p[0] - s * k[0] * v[0], 0.5f, float(g.nx) - 0.5f);
  y = clampf(p[1] - s * k[1] * v[1], 0.5f, float(g.ny) - 0.5f);
  z = clampf(p[2] - s * k[2] * (v[2] - fall), 0.5f, float(g.nz) - 0.5f);
}
// A trilinear tap on the cell-centred box: base offsets of the 2 x 2 x 2 neighbourhood (clamp-to-edge) and the
// weights; the same footprint is the 8-texel min/max window of the MacCormack limiter (model.js:537-540).
struct Tap {
  int i0, i1, r00, r10, r01, r11;
  float ax, ay, az;
};
__device__ __forceinline__ Tap tapQ(const Grid& g, float x, float y, float z) {
  // x, y, z come from traceQ, clamped to [0.5, n - 0.5]: the floor indices lie in [0, n - 1], so only the upper
  // corner needs its clamp-to-edge bound
  const float tx = x - 0.5f, ty = y - 0.5f, tz = z - 0.5f;
  const int i0 = __float2int_rd(tx), j0 = __float2int_rd(ty), k0 = __float2int_rd(tz);
  Tap t;
  t.ax = tx - float(i0);
  t.ay = ty - float(j0);
  t.az = tz - float(k0);
  const int j1 = min(j0 + 1, g.ny - 1), k1 = min(k0 + 1, g.nz - 1);
  t.i0 = i0;
  t.i1 = min(i0 + 1, g.nx - 1);
  t.r00 = g.px * (j0 + g.py * k0);
  t.r10 = g.px * (j1 + g.py * k0);
  t.r01 = g.px * (j0 + g.py * k1);
  t.r11 = g.px * (j1 + g.py * k1);
  return t;
}
__device__ __forceinline__ float gatherQ(const float* __restrict__ f, const Tap& t) {
  const float c00 = __ldg(f + t.r00 + t.i0) * (1.f - t.ax) + __ldg(f + t.r00 + t.i1) * t.ax;
  const float c10 = __ldg(f + t.r10 + t.i0) * (1.f - t.ax) + __ldg(f + t.r10 + t.i1) * t.ax;
  const float c01 = __ldg(f + t.r01 + t.i0) * (1.f - t.ax) + __ldg(f + t.r01 + t.i1) * t.ax;
  const float c11 = __ldg(f + t.r11 + t.i0) * (1.f - t.ax) + __ldg(f + t.r11 + t.i1) * t.ax;
  const float c0 = c00 * (1.f - t.ay) + c10 * t.ay;
  const float c1 = c01 * (1.f - t.ay) + c11 * t.ay;
  return c0 * (1.f - t.az) + c1 * t.az;
}
__device__ __forceinline__ float2 minmaxQ(const float* __restrict__ f, const Tap& t) {
  const float a = __ldg(f + t.r00 + t.i0), b = __ldg(f + t.r00 + t.i1), c = __ldg(f + t.r10 + t.i0), d = __ldg(f + t.r10 + t.i1);
  const float e = __ldg(f + t.r01 + t.i0), h = __ldg(f + t.r01 + t.i1), k = __ldg(f + t.r11 + t.i0), l = __ldg(f + t.r11 + t.i1);
  return make_float2(fminf(fminf(fminf(a, b), fminf(c, d)), fminf(fminf(e, h), fminf(k, l))),
                     fmaxf(fmaxf(fmaxf(a, b), fmaxf(c, d)), fmaxf(fmaxf(e, h), fmaxf(k, l))));
}

// Clear-air skip of the hydrometeor channels (qc, qi, qr, qs, qg, Nr) and of the spare fourth Q2 channel, which no
// scheme sets and physics only carries. A block (one brick of 32 x 4 x 1 cells) reads those channels only inside the
// footprints of its departure points; if every brick touching that region holds none of them (a hydrometeor or a
// nonzero spare), the semi-Lagrangian samples, the MacCormack correction, the limiter and the clip all give exactly
// +0, so the block writes zeros (once) instead of gathering. Falling hydrometeors shift a departure point vertically by
// at most dt/dz * fallmax, which widens the region in z.
struct Region {
  int x0, x1, y0, y1, z0, z1;
};
__device__ __forceinline__ bool region_active(const Grid& g, const Fields& F, Region r, const unsigned int* flagsA,
                                              const unsigned int* flagsB) {
  __shared__ int red[6];
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    red[0] = red[2] = red[4] = 1 << 30;
    red[1] = red[3] = red[5] = -(1 << 30);
  }
  __syncthreads();
  // warp-level min/max, then one shared atomic per warp
  const unsigned m = 0xffffffffu;
  const int a0 = __reduce_min_sync(m, r.x0), a1 = __reduce_max_sync(m, r.x1);
  const int b0 = __reduce_min_sync(m, r.y0), b1 = __reduce_max_sync(m, r.y1);
  const int c0 = __reduce_min_sync(m, r.z0), c1 = __reduce_max_sync(m, r.z1);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&red[0], a0); atomicMax(&red[1], a1);
    atomicMin(&red[2], b0); atomicMax(&red[3], b1);
    atomicMin(&red[4], c0); atomicMax(&red[5], c1);
  }
  __syncthreads();
  const int bx0 = clampi(red[0], 0, g.nx - 1) / 32, bx1 = clampi(red[1], 0, g.nx - 1) / 32;
  const int by0 = clampi(red[2], 0, g.ny - 1) / 4, by1 = clampi(red[3], 0, g.ny - 1) / 4;
  const int bz0 = clampi(red[4], 0, g.nz - 1), bz1 = clampi(red[5], 0, g.nz - 1);
  const int nxb = bx1 - bx0 + 1, nyb = by1 - by0 + 1, nzb = bz1 - bz0 + 1;
  const int count = nxb * nyb * nzb;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  unsigned any = 0;
  for (int t = tid; t < count; t += blockDim.x * blockDim.y) {
    const int bx = bx0 + t % nxb, by = by0 + (t / nxb) % nyb, bz = bz0 + t / (nxb * nyb);
    const int b = bx + F.nbx * (by + F.nby * bz);
    any |= __ldg(flagsA + b);
    if (flagsB) any |= __ldg(flagsB + b);
  }
  return __syncthreads_or(any != 0u) != 0;
}

// ---- ADVQ1 (model.js:500-529): semi-Lagrangian step of the 8 scalars, channels grouped by the fall speed of
// their trace (qv, qc, qi, spare [and Nr for Lin] at the air's speed; qr, qs, qg, Nr (Thompson) each their own) ----
__device__ __forceinline__ void advq1_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  const int ci = BX * blockDim.x + threadIdx.x, cj = BY * blockDim.y + threadIdx.y, ck = BZ;
  const bool in = ci < g.nx && cj < g.ny && ck < g.nz;
  const int o = in ? g.at(ci, cj, ck) : 0;
  const float kk[3] = {U.der.x, U.der.x, U.der.y};  // dt/dx, dt/dx, dt/dz
  float v[3] = {0.f, 0.f, 0.f};
  const float p[3] = {float(ci) + 0.5f, float(cj) + 0.5f, float(ck) + 0.5f};
  float x = 0.5f, y = 0.5f, z = 0.5f;
  Region r{ci, ci, cj, cj, ck, ck};
  if (in) {
    cellVel(F, g, par, ci, cj, ck, v);
    traceQ(g, kk, p, v, 0.f, 1.f, x, y, z);
    r.x0 = min(r.x0, int(floorf(x - 0.5f)));
    r.x1 = max(r.x1, int(floorf(x - 0.5f)) + 1);
    r.y0 = min(r.y0, int(floorf(y - 0.5f)));
    r.y1 = max(r.y1, int(floorf(y - 0.5f)) + 1);
    r.z0 = min(r.z0, int(floorf(z - 0.5f)));
    r.z1 = max(r.z1, int(floorf(fminf(z + kk[2] * F.fallmax, float(g.nz) - 0.5f) - 0.5f)) + 1);
  }
  const bool active = region_active(g, F, r, F.actQ0, nullptr);
  const int brick = BX + F.nbx * (BY + F.nby * BZ);
  if (in) {
    const Tap t0 = tapQ(g, x, y, z);
    F.Qt[0][o] = gatherQ(F.Q[0][0], t0);
    if (active) {
      F.Qt[1][o] = gatherQ(F.Q[0][1], t0);
      F.Qt[2][o] = gatherQ(F.Q[0][2], t0);
      F.Qt[7][o] = gatherQ(F.Q[0][7], t0);
      const float nr0 = gatherQ(F.Q[0][6], t0);
      const Fall fl{U.step.z, U.micro2.z > 0.5f};
      const float rho = bsA(F.B, g.nz, ck).z;
      const float2 fv = fl.vtRain(__ldg(F.Q[0][3] + o), __ldg(F.Q[0][6] + o), rho);
      const float fs = fl.vtS(__ldg(F.Q[0][4] + o), rho), fg = fl.vtGrau(__ldg(F.Q[0][5] + o), rho);
      traceQ(g, kk, p, v, fv.x, 1.f, x, y, z);
      F.Qt[3][o] = gatherQ(F.Q[0][3], tapQ(g, x, y, z));
      traceQ(g, kk, p, v, fs, 1.f, x, y, z);
      F.Qt[4][o] = gatherQ(F.Q[0][4], tapQ(g, x, y, z));
      traceQ(g, kk, p, v, fg, 1.f, x, y, z);
      F.Qt[5][o] = gatherQ(F.Q[0][5], tapQ(g, x, y, z));
      if (fl.thm) {
        traceQ(g, kk, p, v, fv.y, 1.f, x, y, z);
        F.Qt[6][o] = gatherQ(F.Q[0][6], tapQ(g, x, y, z));
      } else {
        F.Qt[6][o] = nr0;
      }
    } else if (!F.zeroQt[brick]) {
#pragma unroll
      for (int c = 1; c < 8; c++) F.Qt[c][o] = 0.f;
    }
  }
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    F.actQt[brick] = active ? 1u : 0u;
    F.zeroQt[brick] = active ? 0u : 1u;
  }
}
__global__ void __launch_bounds__(128, 12) k_advq1(Grid g, Uni U, Fields F, int par) { advq1_body(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void __launch_bounds__(128, 12) k_advq1_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  advq1_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---- ADVQ2 (model.js:530-576): MacCormack correction, limiter on the departure cell's 8 texels, clip >= 0 ----
__device__ __forceinline__ float advq2_channel(const Fields& F, const Grid& g, const float kk[3], const float p[3], const float v[3],
                                               float fall, float sm, float qc_, int c, int o) {
  float x, y, z;
  traceQ(g, kk, p, v, fall, -1.f, x, y, z);
  const float b = gatherQ(F.Qt[c], tapQ(g, x, y, z));
  const float r = __ldg(F.Qt[c] + o) + sm * (qc_ - b);
  traceQ(g, kk, p, v, fall, 1.f, x, y, z);
  const float2 m = minmaxQ(F.Q[0][c], tapQ(g, x, y, z));
  return fmaxf(clampf(r, m.x, m.y), 0.f);
}

__device__ __forceinline__ void advq2_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  const int ci = BX * blockDim.x + threadIdx.x, cj = BY * blockDim.y + threadIdx.y, ck = BZ;
  const bool in = ci < g.nx && cj < g.ny && ck < g.nz;
  const int o = in ? g.at(ci, cj, ck) : 0;
  const float kk[3] = {U.der.x, U.der.x, U.der.y};  // dt/dx, dt/dx, dt/dz
  float v[3] = {0.f, 0.f, 0.f};
  const float p[3] = {float(ci) + 0.5f, float(cj) + 0.5f, float(ck) + 0.5f};
  float xb = 0.5f, yb = 0.5f, zb = 0.5f, xf = 0.5f, yf = 0.5f, zf = 0.5f;
  Region r{ci, ci, cj, cj, ck, ck};
  if (in) {
    cellVel(F, g, par, ci, cj, ck, v);
    traceQ(g, kk, p, v, 0.f, -1.f, xb, yb, zb);
    traceQ(g, kk, p, v, 0.f, 1.f, xf, yf, zf);
    r.x0 = min(r.x0, int(floorf(fminf(xb, xf) - 0.5f)));
    r.x1 = max(r.x1, int(floorf(fmaxf(xb, xf) - 0.5f)) + 1);
    r.y0 = min(r.y0, int(floorf(fminf(yb, yf) - 0.5f)));
    r.y1 = max(r.y1, int(floorf(fmaxf(yb, yf) - 0.5f)) + 1);
    const float dzf = kk[2] * F.fallmax;
    r.z0 = min(r.z0, int(floorf(fmaxf(fminf(zb, zf) - dzf, 0.5f) - 0.5f)));
    r.z1 = max(r.z1, int(floorf(fminf(fmaxf(zb, zf) + dzf, float(g.nz) - 0.5f) - 0.5f)) + 1);
  }
  const bool active = region_active(g, F, r, F.actQ0, F.actQt);
  const int brick = BX + F.nbx * (BY + F.nby * BZ);
  if (in) {
    const float cx = v[0] * kk[0], cy = v[1] * kk[1], cz = v[2] * kk[2];
    const float cour = sqrtf(cx * cx + cy * cy + cz * cz);
    const float sm = 0.5f * U.misc.y * clampf(cour / 0.35f, U.dzv.w, 1.f);
    {  // the air-speed group: qv always; qc, qi and the spare channel where active
      const Tap tb = tapQ(g, xb, yb, zb), tf = tapQ(g, xf, yf, zf);
      {
        const float b = gatherQ(F.Qt[0], tb);
        const float rr = __ldg(F.Qt[0] + o) + sm * (__ldg(F.Q[0][0] + o) - b);
        const float2 m = minmaxQ(F.Q[0][0], tf);
        F.Q[1][0][o] = fmaxf(clampf(rr, m.x, m.y), 0.f);
      }
      if (active) {
        const Fall fl{U.step.z, U.micro2.z > 0.5f};
        constexpr int kAir[3] = {1, 2, 7};  // qc, qi, spare
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const int c = kAir[i];
          const float b = gatherQ(F.Qt[c], tb);
          const float rr = __ldg(F.Qt[c] + o) + sm * (__ldg(F.Q[0][c] + o) - b);
          const float2 m = minmaxQ(F.Q[0][c], tf);
          F.Q[1][c][o] = fmaxf(clampf(rr, m.x, m.y), 0.f);
        }
        if (!fl.thm) {
          const float b = gatherQ(F.Qt[6], tb);
          const float rr = __ldg(F.Qt[6] + o) + sm * (__ldg(F.Q[0][6] + o) - b);
          const float2 m = minmaxQ(F.Q[0][6], tf);
          F.Q[1][6][o] = fmaxf(clampf(rr, m.x, m.y), 0.f);
        }
      }
    }
    if (active) {
      const Fall fl{U.step.z, U.micro2.z > 0.5f};
      const float rho = bsA(F.B, g.nz, ck).z;
      const float q3 = __ldg(F.Q[0][3] + o), q4 = __ldg(F.Q[0][4] + o), q5 = __ldg(F.Q[0][5] + o), q6 = __ldg(F.Q[0][6] + o);
      const float2 fv = fl.vtRain(q3, q6, rho);
      F.Q[1][3][o] = advq2_channel(F, g, kk, p, v, fv.x, sm, q3, 3, o);
      F.Q[1][4][o] = advq2_channel(F, g, kk, p, v, fl.vtS(q4, rho), sm, q4, 4, o);
      F.Q[1][5][o] = advq2_channel(F, g, kk, p, v, fl.vtGrau(q5, rho), sm, q5, 5, o);
      if (fl.thm) F.Q[1][6][o] = advq2_channel(F, g, kk, p, v, fv.y, sm, q6, 6, o);
    } else if (!F.zeroQ1[brick]) {
#pragma unroll
      for (int c = 1; c < 8; c++) F.Q[1][c][o] = 0.f;
    }
  }
  if (threadIdx.x == 0 && threadIdx.y == 0) F.zeroQ1[brick] = active ? 0u : 1u;
}
__global__ void __launch_bounds__(128, 10) k_advq2(Grid g, Uni U, Fields F, int par) { advq2_body(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void __launch_bounds__(128, 9) k_advq2_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  advq2_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// hydrometeor flags of Q slot 0 per brick, from scratch (after a reset or a host upload of Q); the scratch-known-zero
// flags are cleared because the host may have written anywhere
__global__ void __launch_bounds__(128) k_activity(Grid g, Fields F) {
  const int ci = blockIdx.x * blockDim.x + threadIdx.x, cj = blockIdx.y * blockDim.y + threadIdx.y, ck = blockIdx.z;
  bool act = false;
  if (ci < g.nx && cj < g.ny && ck < g.nz) {
    const int o = g.at(ci, cj, ck);
#pragma unroll
    for (int c = 1; c < 8; c++) act |= F.Q[0][c][o] != 0.f;
  }
  const bool any = __syncthreads_or(act) != 0;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.x + F.nbx * (blockIdx.y + F.nby * blockIdx.z);
    F.actQ0[b] = any ? 1u : 0u;
    F.actQt[b] = 1u;
    F.zeroQt[b] = 0u;
    F.zeroQ1[b] = 0u;
  }
}

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_PHYS (model.js:578-907): forcing stencils + microphysics, outbreak mode
// ---------------------------------------------------------------------------------------------------------------
// lateral sponge of one distance to the nearest side wall, and the top sponge at height z (model.js:611-626)
__device__ __forceinline__ float spongeLat1(const Uni& U, float e) {
  const float d = clampf(1.f - e / U.sponge.x, 0.f, 1.f);
  return d * (0.3f + 0.7f * d) / U.sponge.y;
}
__device__ __forceinline__ float spongeTop(const Uni& U, const Grid& g, float z) {
  const float ztop = float(g.nz) * U.dzv.x;
  if (z < U.sponge.z) return 0.f;
  const float s = sinf(1.5707963f * (z - U.sponge.z) / (ztop - U.sponge.z));
  return s * s / U.sponge.w;
}
// sponge tables (Fields::spz/slx/sly) and the per-level rain-speed density factor sqrt(rho_sfc / rho) (spz[4k+2])
__global__ void k_tables(Grid g, Uni U, const float* B, float* spz, float* slx, float* sly) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const float dx = U.dims.w, dz = U.dzv.x;
  if (t <= g.nz) {
    spz[4 * t + 0] = spongeTop(U, g, (float(t) + 0.5f) * dz);
    spz[4 * t + 1] = spongeTop(U, g, float(t) * dz);
    spz[4 * t + 2] = sqrtf(U.step.z / bsA(B, g.nz, t).z);
    spz[4 * t + 3] = 0.f;
  }
  const float Lx = float(g.nx) * dx, Ly = float(g.ny) * dx;
  if (t <= g.nx) {
    const float xf = float(t) * dx, xc = (float(t) + 0.5f) * dx;
    slx[2 * t] = spongeLat1(U, fminf(xf, Lx - xf));
    slx[2 * t + 1] = spongeLat1(U, fminf(xc, Lx - xc));
  }
  if (t <= g.ny) {
    const float yf = float(t) * dx, yc = (float(t) + 0.5f) * dx;
    sly[2 * t] = spongeLat1(U, fminf(yf, Ly - yf));
    sly[2 * t + 1] = spongeLat1(U, fminf(yc, Ly - yc));
  }
}
__device__ __forceinline__ float bsV(const float* B, int nz, int k, int ch) {
  const int kk = clampi(k, 0, nz - 1);
  if (ch == 0) return bsB(B, nz, kk).z;
  if (ch == 1) return bsB(B, nz, kk).w;
  if (ch == 3) return bsA(B, nz, kk).x;
  return 0.f;
}

// one slot of an append-only list per calling thread: one atomic per warp, slots in lane order
__device__ __forceinline__ unsigned warp_append(unsigned* ctr) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(ctr, unsigned(__popc(mask)));
  base = __shfl_sync(mask, base, leader);
  return base + unsigned(__popc(mask & ((1u << lane) - 1u)));
}

// one texel of the physics pass; returns whether the cell's new state holds a hydrometeor. MM: microphysics as the
// scheme (kMicroPlain), the scheme plus sampled (state, tendency) pairs (kMicroRecord), or queued for the surrogate
// kernel where it can act (kMicroSurrogate).
// Neighbour reads clamp to the edge of their texture (textureLoad with clamped coordinates, model.js:596-606): the
// offsets below are the clamped index minus the texel's own, for the staggered box [0, n] (V) and the cell box
// [0, n-1] (Q, aux, phi_t), computed once per texel. BND: boundary air masses present (else the target state is the
// base state, see tgtUb).
template <bool BND, int MM, bool HUR = false>
__device__ __forceinline__ bool phys_texel(const Grid& g, const Uni& U, const Fields& F, int par, int ci, int cj, int ck, bool dry,
                                           bool was0) {
  bool hyd = false;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int o = g.at(ci, cj, ck);
  const float* __restrict__ Vu = F.V[1 - par][0] + o;
  const float* __restrict__ Vv = F.V[1 - par][1] + o;
  const float* __restrict__ Vw = F.V[1 - par][2] + o;
  const float* __restrict__ Vth = F.V[1 - par][3] + o;
  const float* __restrict__ A0 = F.aux[0] + o;
  const float* __restrict__ A1 = F.aux[1] + o;
  // staggered box
  const int xm = ci > 0 ? -1 : 0, xp = ci < nx ? 1 : 0;
  const int ym = cj > 0 ? -g.px : 0, yp = cj < ny ? g.px : 0;
  const int zm = ck > 0 ? -g.plane : 0, zp = ck < nz ? g.plane : 0;
  // cell box: own index and +-1, clamped to [0, n-1]
  const int xc0 = ci < nx ? 0 : -1, xcp = ci < nx - 1 ? 1 : xc0;
  const int yc0 = cj < ny ? 0 : -g.px, ycp = cj < ny - 1 ? g.px : yc0;
  auto LP = [&](int off) {
    if (!BND) return 0.f;
    return __ldg(F.phT + o + off);
  };
  const float dx = U.dims.w, dz = U.dzv.x, dt = U.step.x;
  float V[4] = {__ldg(Vu), __ldg(Vv), __ldg(Vw), __ldg(Vth)};
  float out[4] = {V[0], V[1], V[2], V[3]};
  const float ix2 = U.der.z, iz2 = U.der.w;
  const float fc = U.cor.x;
  const float* __restrict__ Vc[4] = {Vu, Vv, Vw, Vth};
  auto lapH = [&](int ch, float me) { return __ldg(Vc[ch] + xp) + __ldg(Vc[ch] + xm) + __ldg(Vc[ch] + yp) + __ldg(Vc[ch] + ym) - 4.f * me; };
  auto lapZp = [&](int ch, float me, bool lo, bool hi) {
    const float m0 = me - bsV(F.B, nz, ck, ch);
    const float a = lo ? m0 : __ldg(Vc[ch] + zm) - bsV(F.B, nz, ck - 1, ch);
    const float b = hi ? m0 : __ldg(Vc[ch] + zp) - bsV(F.B, nz, ck + 1, ch);
    return a + b - 2.f * m0;
  };
  const float4 spk = __ldg(reinterpret_cast<const float4*>(F.spz) + ck);  // (top sponge centre, face, rain factor, -)
  const float2 slx = __ldg(reinterpret_cast<const float2*>(F.slx) + ci);  // (face, centre)
  const float2 sly = __ldg(reinterpret_cast<const float2*>(F.sly) + cj);
  // u
  if (cj < ny && ck < nz) {
    const float nux = 0.5f * (__ldg(A0 + xm) + __ldg(A0 + xc0)) + U.turb.y;
    const float nuy = 0.5f * (__ldg(A1 + xm) + __ldg(A1 + xc0)) + U.turb.y;
    float du = nux * lapH(0, V[0]) * ix2 + nuy * lapZp(0, V[0], ck == 0, ck == nz - 1) * iz2;
    const float ut = tgtUb<BND>(F, g, dz, ci, cj, ck);
    const float vbar = 0.25f * (__ldg(Vv + xm) + V[1] + __ldg(Vv + xm + yp) + __ldg(Vv + yp));
    const float vtb = 0.5f * (tgtVb<BND>(F, g, dz, ci - 1, cj, ck) + tgtVb<BND>(F, g, dz, ci, cj + 1, ck));
    const float sp = fmaxf(slx.x, sly.y) + spk.x;
    if (BND) {
      const float nw = 0.5f * (l2d(F.lsfB, g, ci - 1, cj).w + l2d(F.lsfB, g, ci, cj).w);
      du += (sp + nw * (1.f / U.cor.y)) * (ut - V[0]);
    } else {
      du += sp * (ut - V[0]);
    }
    du += fc * (vbar - vtb);
    if (BND && ci > 0 && ci < nx) du -= (LP(0) - LP(-1)) / dx;
    if (ck == 0 && U.turb.w > 0.5f) {
      float cd = U.micro.w;
      if (HUR) {  // sea / land drag (model.js:649-652)
        const float land = 0.5f * (__ldg(F.sfc + cj * nx + max(ci - 1, 0)).x + __ldg(F.sfc + min(cj, ny - 1) * nx + min(ci, nx - 1)).x);
        cd = cdSfc(U, sqrtf(V[0] * V[0] + vbar * vbar), land);
      }
      du += cd * (-sqrtf(V[0] * V[0] + vbar * vbar) * V[0] + sqrtf(ut * ut + vtb * vtb) * ut) / dz;
    }
    out[0] = V[0] + dt * du;
  } else out[0] = 0.f;
  // v
  if (ci < nx && ck < nz) {
    const float nux = 0.5f * (__ldg(A0 + ym) + __ldg(A0 + yc0)) + U.turb.y;
    const float nuy = 0.5f * (__ldg(A1 + ym) + __ldg(A1 + yc0)) + U.turb.y;
    float dv = nux * lapH(1, V[1]) * ix2 + nuy * lapZp(1, V[1], ck == 0, ck == nz - 1) * iz2;
    const float vt = tgtVb<BND>(F, g, dz, ci, cj, ck);
    const float ubar = 0.25f * (__ldg(Vu + ym) + V[0] + __ldg(Vu + xp + ym) + __ldg(Vu + xp));
    const float utb = 0.5f * (tgtUb<BND>(F, g, dz, ci, cj - 1, ck) + tgtUb<BND>(F, g, dz, ci + 1, cj, ck));
    const float sp = fmaxf(slx.y, sly.x) + spk.x;
    if (BND) {
      const float nw = 0.5f * (l2d(F.lsfB, g, ci, cj - 1).w + l2d(F.lsfB, g, ci, cj).w);
      dv += (sp + nw * (1.f / U.cor.y)) * (vt - V[1]);
    } else {
      dv += sp * (vt - V[1]);
    }
    dv -= fc * (ubar - utb);
    if (BND && cj > 0 && cj < ny) dv -= (LP(0) - LP(-g.px)) / dx;
    if (ck == 0 && U.turb.w > 0.5f) {
      float cd = U.micro.w;
      if (HUR) {
        const float land = 0.5f * (__ldg(F.sfc + max(cj - 1, 0) * nx + ci).x + __ldg(F.sfc + min(cj, ny - 1) * nx + min(ci, nx - 1)).x);
        cd = cdSfc(U, sqrtf(ubar * ubar + V[1] * V[1]), land);
      }
      dv += cd * (-sqrtf(ubar * ubar + V[1] * V[1]) * V[1] + sqrtf(utb * utb + vt * vt) * vt) / dz;
    }
    out[1] = V[1] + dt * dv;
  } else out[1] = 0.f;
  // w
  if (ci < nx && cj < ny && ck > 0 && ck < nz) {
    const float nux = 0.5f * (__ldg(A0 - g.plane) + __ldg(A0)) + U.turb.y;
    const float nuy = 0.5f * (__ldg(A1 - g.plane) + __ldg(A1)) + U.turb.y;
    float dw = nux * lapH(2, V[2]) * ix2 + nuy * (__ldg(Vw - g.plane) + __ldg(Vw + g.plane) - 2.f * V[2]) * iz2;
    auto buoy = [&](int kk, int off) {
      const float4 A = bsA(F.B, nz, kk);
      float h[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
      if (!dry) {
#pragma unroll
        for (int c = 0; c < 5; c++) h[c] = __ldg(F.Q[1][1 + c] + o + off);
      }
      return 9.81f * ((__ldg(Vth + off) - A.x) / A.x + 0.608f * (__ldg(F.Q[1][0] + o + off) - A.y) -
                      (h[0] + h[1] + h[2] + h[3] + h[4]));
    };
    dw += 0.5f * (buoy(ck - 1, -g.plane) + buoy(ck, 0));
    if (BND) dw -= (LP(0) - LP(-g.plane)) / dz;
    dw += (fmaxf(slx.y, sly.y) + spk.y) * (0.f - V[2]);
    const float4 civ = __ldg(F.ciMap + cj * nx + ci);
    if (!HUR && civ.x > 0.f) {  // hurricane mode starts storms as warm bubbles instead (model.js:686-687)
      const float z = float(ck) * dz;
      const float zz = fabsf(z - civ.z) / civ.w;
      if (zz < 1.f) {
        const float cv = cosf(1.5707963f * zz);
        dw += U.misc.w * civ.x * cv * fmaxf(civ.y * cv - V[2], 0.f);
      }
    }
    out[2] = V[2] + dt * dw;
  } else out[2] = 0.f;
  // theta + microphysics at cell centres
  if (ci < nx && cj < ny && ck < nz) {
    const float4 A = bsA(F.B, nz, ck), Bb = bsB(F.B, nz, ck);
    const float4 LAv = BND ? l2d(F.lsfA, g, ci, cj) : make_float4(0.f, 100.f, 0.f, 100.f);
    const float tth = BND ? tgtTh(F.B, g, dz, LAv, ck) : A.x, tqv = BND ? tgtQv(F.B, g, dz, LAv, ck) : A.y;
    const float sl = fmaxf(slx.y, sly.y);
    const float relax = BND ? sl + l2d(F.lsfB, g, ci, cj).w * (1.f / U.cor.y) : sl;
    const float nux = __ldg(A0) * 3.f + U.turb.y, nuy = __ldg(A1) * 3.f + U.turb.y;
    float th = V[3] + dt * (nux * lapH(3, V[3]) * ix2 + nuy * lapZp(3, V[3], ck == 0, ck == nz - 1) * iz2 + (relax + spk.x) * (tth - V[3]));
    // hydrometeor and spare channels: exactly +0 throughout a dry block's reach, so not read there (the sums below
    // then see the same +0 operands the loads would have returned)
    float q1[4] = {__ldg(F.Q[1][0] + o), 0.f, 0.f, 0.f}, q2[4] = {0.f, 0.f, 0.f, 0.f};
    float l1[3] = {0.f, 0.f, 0.f}, l1z[3] = {0.f, 0.f, 0.f};
    if (!dry) {
#pragma unroll
      for (int c = 0; c < 4; c++) {
        if (c) q1[c] = __ldg(F.Q[1][c] + o);
        q2[c] = __ldg(F.Q[1][4 + c] + o);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (c && dry) continue;
      const float* __restrict__ q = F.Q[1][c] + o;
      l1[c] = __ldg(q + xcp) + __ldg(q + xm) + __ldg(q + ycp) + __ldg(q + ym) - 4.f * q1[c];
      l1z[c] = (ck == 0 ? q1[c] : __ldg(q + zm)) + (ck == nz - 1 ? q1[c] : __ldg(q + g.plane)) - 2.f * q1[c];
    }
    const float qvb = (ck == 0 ? A.y : bsA(F.B, nz, ck - 1).y) + (ck == nz - 1 ? A.y : bsA(F.B, nz, ck + 1).y) - 2.f * A.y;
    l1z[0] -= qvb;
#pragma unroll
    for (int c = 0; c < 3; c++) q1[c] = q1[c] + dt * (nux * l1[c] * ix2 + nuy * l1z[c] * iz2);
    q1[0] += dt * relax * (tqv - q1[0]);
    const float xmx = (float(ci) + 0.5f) * dx, xmy = (float(cj) + 0.5f) * dx;
    float envDecay = 0.f;
    if (HUR) {  // the warm sea and the tropical environment (model.js:713-774)
      const float z = (float(ck) + 0.5f) * dz;
      th += dt * clampf((tth - V[3]) / U.hur2.x, -U.hur2.y, U.hur2.y);
      const float4 cs = __ldg(F.ciMap + cj * nx + ci);
      if (cs.x > 0.f) {  // storm starts: a warm, moist bubble through the push's depth
        const float zz = fabsf(z - cs.z) / cs.w;
        if (zz < 1.f) {
          const float f = cs.x * cosf(1.5707963f * zz) * cs.y / 8.f;
          th += dt * 1.2e-3f * f;
          q1[0] += dt * f / 600.f * fmaxf(0.97f * qvsat(V[3] * Bb.x, Bb.y, 0.f) - q1[0], 0.f);
        }
      }
      const float dxh = xmx - U.hur4.x, dyh = xmy - U.hur4.y;
      const float rS = sqrtf(dxh * dxh + dyh * dyh);
      const float wEnv = sstep(U.hur4.w, 1.5f * U.hur4.w, rS) / 3600.f;  // the far field held to the sounding
      th += dt * wEnv * (tth - V[3]);
      q1[0] += dt * wEnv * (tqv - q1[0]);
      envDecay = sstep(U.hur4.w, 1.5f * U.hur4.w, rS) / 1800.f;
      if (z < U.hur2.z) {  // boundary-layer thermals: coherent ~6 km cells living ~15 min
        const int o0 = g.at(ci, cj, 0);
        const float ua = 0.5f * (__ldg(F.V[1 - par][0] + o0) + __ldg(F.V[1 - par][0] + o0 + 1));
        const float va = 0.5f * (__ldg(F.V[1 - par][1] + o0) + __ldg(F.V[1 - par][1] + o0 + g.px));
        const float u1 = sqrtf(ua * ua + va * va);
        const float e = float(__ldg(F.clock)) / 900.f, e0 = floorf(e);
        const float qx = xmx / 6000.f, qy = xmy / 6000.f;
        const float r = 0.5f * mixf(gnoise2(qx + 37.1f * e0, qy + 11.3f * e0), gnoise2(qx + 37.1f * (e0 + 1.f), qy + 11.3f * (e0 + 1.f)),
                                    sstep(0.f, 1.f, e - floorf(e)));
        const float fu = fminf(u1 * u1 / 225.f, 1.f) * (1.f - sstep(20.f, 32.f, u1)) * (1.f - sstep(U.hur4.z, 1.5f * U.hur4.z, rS));
        th += dt * U.hur3.z * 2.f * r * fu * (1.f - z / U.hur2.z);
      }
      if (ck == 0) {  // the sea's sensible and latent heat; dissipative heating
        const float4 sf = __ldg(F.sfc + cj * nx + ci);
        const float land = clampf(sf.x, 0.f, 1.f);
        const float ua = 0.5f * (V[0] + __ldg(Vu + 1)), va = 0.5f * (V[1] + __ldg(Vv + g.px));
        const float u1 = sqrtf(ua * ua + va * va);
        const float ch = U.hur.y * U.hur2.w * fmaxf(u1, U.hur3.y) / dz;
        const float ps = fmaxf(U.hur.w + A.z * U.cn.y * __ldg(F.phi + g.pidx(ci, cj, ck)), 50000.f);
        const float ths = sf.y * powf(1.0e5f / ps, 0.2854f);
        th += dt * ch * (1.f - land) * (ths - V[3]);
        if (U.hur5.y > 0.5f) {
          const float cdh = cdSfc(U, u1, land);
          th += dt * cdh * u1 * u1 * u1 / (1005.7f * dz) / Bb.x;
        }
        const float qsS = qvsat(sf.y, ps, 0.f);
        const float qsL = qvsat(V[3] * Bb.x, ps, 0.f);
        q1[0] += dt * ch * ((1.f - land) * (qsS - q1[0]) + land * U.hur.z * fmaxf(qsL - q1[0], 0.f));
      }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
      q1[c] = fmaxf(q1[c], 0.f);
      q2[c] = fmaxf(q2[c], 0.f);
    }
    const float pi0 = Bb.x, p0 = Bb.y, rho = A.z;
    float T = th * pi0;
    float qv = q1[0], qc = q1[1], qi = q1[2], qr = q1[3], qs = q2[0], qg = q2[1];
    const bool thm = U.micro2.z > 0.5f;
    MCell mc{T, qv, qc, qi, qr, qs, qg, fmaxf(q2[2], 0.f)};
    bool done = false;
    if (MM == kMicroSurrogate && surrogate_cell(mc)) {
      // surrogate cell: store the state before the microphysics and queue the cell; the surrogate kernel applies
      // the process tendencies, the saturation adjustment, the sponge removal and the clips (a full queue falls
      // through to the scheme here)
      const unsigned slot = warp_append(F.mlp_count);
      if (slot < F.mlp_cap) {
        reinterpret_cast<unsigned*>(F.mlp_buf)[slot] = unsigned(o);
        F.Q[0][0][o] = mc.qv; F.Q[0][1][o] = mc.qc; F.Q[0][2][o] = mc.qi; F.Q[0][3][o] = mc.qr;
        F.Q[0][4][o] = mc.qs; F.Q[0][5][o] = mc.qg; F.Q[0][6][o] = mc.nr; F.Q[0][7][o] = q2[3];
        out[3] = mc.T / pi0;
        hyd = true;
        done = true;
      }
    }
    if (!done) {
      const MCell pre = mc;
      // with every hydrometeor exactly +0 (a dry block) each process rate is zero and the block leaves the cell as it
      // is; the saturation adjustment below still runs (a supersaturated cell condenses)
      if (!dry) micro_processes(U, dt, p0, rho, spk.z, mc);
      if (MM == kMicroRecord && surrogate_cell(pre) &&
          float(hash3i(ci, cj, ck ^ int(__float_as_uint(float(__ldg(F.clock))) * 2654435761u)) >> 8u) * (1.f / 16777216.f) < F.mlp_rate) {
        // one (state, process tendency) pair of the scheme: 12 inputs, 10 tendencies (before the saturation
        // adjustment), the cell's texel offset (as bits), the model time of the step (the two order the pairs
        // canonically: ob_mlp_sort_pairs)
        const unsigned slot = warp_append(F.mlp_count);
        if (slot < F.mlp_cap) {
          float* r = F.mlp_buf + size_t(slot) * 24;
          const float x[12] = {pre.T, p0, rho, pre.qv, pre.qc, pre.qr, pre.qi, pre.qs, pre.qg, pre.nr, q2[3], V[2]};
          const float y[12] = {mc.T - pre.T, mc.qv - pre.qv, mc.qc - pre.qc, mc.qi - pre.qi, mc.qr - pre.qr, mc.qs - pre.qs,
                               mc.qg - pre.qg, mc.nr - pre.nr, 0.f, 0.f, __uint_as_float(unsigned(o)), float(__ldg(F.clock))};
#pragma unroll
          for (int e = 0; e < 12; e++) {
            r[e] = x[e];
            r[12 + e] = y[e];
          }
        }
      }
      sat_adjust(p0, mc);
      T = mc.T; qv = mc.qv; qc = mc.qc; qi = mc.qi; qr = mc.qr; qs = mc.qs; qg = mc.qg;
      float nr = mc.nr;
      th = T / pi0;
      // 1 / (1 + 0) == 1 exactly: no division outside the sponge (and, in hurricane mode, the far-field decay)
      const float keep = HUR ? 1.f / (1.f + 2.f * dt * sl + dt * envDecay) : (sl > 0.f ? 1.f / (1.f + 2.f * dt * sl) : 1.f);
      qc *= keep; qi *= keep; qr *= keep; qs *= keep; qg *= keep; nr *= keep;
      hyd = qc > 0.f || qi > 0.f || qr > 0.f || qs > 0.f || qg > 0.f || (thm ? nr : q2[2]) > 0.f || q2[3] > 0.f;
      F.Q[0][0][o] = fmaxf(qv, 0.f);
      if (hyd || !was0) {  // else the channels below are zero here and slot 0 already holds zeros
        F.Q[0][1][o] = fmaxf(qc, 0.f);
        F.Q[0][2][o] = fmaxf(qi, 0.f);
        F.Q[0][3][o] = fmaxf(qr, 0.f);
        F.Q[0][4][o] = fmaxf(qs, 0.f);
        F.Q[0][5][o] = fmaxf(qg, 0.f);
        F.Q[0][6][o] = thm ? fmaxf(nr, 0.f) : q2[2];
        F.Q[0][7][o] = q2[3];
      }
      out[3] = th;
    }
  }
  const float sp = sqrtf(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
  if (sp > U.misc.x) {
    const float s = U.misc.x / sp;
    out[0] *= s; out[1] *= s; out[2] *= s;
  }
  if (!(out[0] == out[0]) || !(out[1] == out[1]) || !(out[2] == out[2]) || !(out[3] == out[3])) {
    out[0] = bsB(F.B, nz, ck).z; out[1] = bsB(F.B, nz, ck).w; out[2] = 0.f; out[3] = bsA(F.B, nz, ck).x;
    atomicAdd(F.flags, 1u);
  }
#pragma unroll
  for (int c = 0; c < 4; c++) F.V[par][c][o] = out[c];
  return hyd;
}

// The clear-air flags of a physics block (one 32 x 4 brick of cells; blocks past the last brick hold only faces, which
// read and write no scalar), the same for all its threads: dry = Q slot 1 holds no hydrometeor and no nonzero spare in
// the brick and its six face neighbours (ADVQ2 wrote them as zeros), which bound every scalar read of the block; was0
// = the previous physics pass left slot 0's hydrometeor and spare channels zero in the brick (actQ0 clear), so a cell
// whose new values there are all zero need not store them again. Hurricane mode's 2-dx filter writes slot 0 between
// physics passes, so there was0 stays false.
template <bool HUR>
__device__ __forceinline__ void phys_flags(const Grid& g, const Fields& F, int BX, int BY, int ck, bool& dry, bool& was0) {
  dry = false;
  was0 = false;
  if (BX >= F.nbx || BY >= F.nby || ck >= g.nz) return;
  const int lane = threadIdx.x & 31;
  unsigned z = 1u;
  if (lane < 7) {
    const int bx = BX + (lane == 1 ? -1 : lane == 2 ? 1 : 0), by = BY + (lane == 3 ? -1 : lane == 4 ? 1 : 0);
    const int bz = ck + (lane == 5 ? -1 : lane == 6 ? 1 : 0);
    if (bx >= 0 && bx < F.nbx && by >= 0 && by < F.nby && bz >= 0 && bz < g.nz) z = F.zeroQ1[bx + F.nbx * (by + F.nby * bz)];
  }
  dry = __all_sync(0xffffffffu, z != 0u);
  if (!HUR) was0 = F.actQ0[BX + F.nbx * (BY + F.nby * ck)] == 0u;
}

// BND: 1 = boundary air masses present, 0 = none, -1 = decided per launch from the uniforms (U.cor.z)
template <int MM, bool HUR = false, int BND = -1>
__device__ __forceinline__ void phys_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  const int ci = BX * blockDim.x + threadIdx.x, cj = BY * blockDim.y + threadIdx.y, ck = BZ;
  bool dry, was0;
  phys_flags<HUR>(g, F, BX, BY, ck, dry, was0);
  bool hyd = false;
  if (ci <= g.nx && cj <= g.ny && ck <= g.nz)
    hyd = (BND == 1 || (BND < 0 && U.cor.z > 0.5f)) ? phys_texel<BND != 0, MM, HUR>(g, U, F, par, ci, cj, ck, dry, was0)
                                                    : phys_texel<false, MM, HUR>(g, U, F, par, ci, cj, ck, dry, was0);
  // hydrometeor flag of this block's brick for the next step's scalar advection
  const bool any = __syncthreads_or(hyd) != 0;
  if (threadIdx.x == 0 && threadIdx.y == 0 && int(BX) < F.nbx && int(BY) < F.nby && ck < g.nz)
    F.actQ0[BX + F.nbx * (BY + F.nby * ck)] = any ? 1u : 0u;
}
// one kernel per microphysics mode and per presence of boundary air masses: with one texel body per kernel, ten
// 128-thread blocks fit on an SM at 48 registers without spilling (the surrogate with boundaries keeps nine), where the
// kernel holding both bodies needed 56 registers at nine blocks; 0.64 -> 0.61 ms at 640 x 640 x 40
template <int MM, int BND>
__global__ void __launch_bounds__(128, (MM == kMicroSurrogate && BND == 1) ? 9 : 10) k_phys(Grid g, Uni U, Fields F, int par) {
  phys_body<MM, false, BND>(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z);
}
__global__ void __launch_bounds__(128) k_phys_hur(Grid g, Uni U, Fields F, int par) {
  phys_body<kMicroPlain, true>(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int MM>
__global__ void __launch_bounds__(128, 9) k_phys_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  phys_body<MM>(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_DIV (model.js:909-925): density-weighted divergence / dt on the padded solve grid
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void div_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  OB_TEXEL_LOOP_BEGIN(g.nx - 1, g.ny - 1, g.nz - 1)
  const int o = g.at(ci, cj, ck);
  const float* __restrict__ u = F.V[par][0];
  const float* __restrict__ v = F.V[par][1];
  const float* __restrict__ w = F.V[par][2];
  const float rc = bsA(F.B, g.nz, ck).z;
  const float wt = ck == g.nz - 1 ? 0.f : __ldg(w + o + g.plane);
  const float wb = ck == 0 ? 0.f : __ldg(w + o);
  // the reference divides by dx, dz and dt (model.js:909-925); multiplying by the host's reciprocals (1/dx, 1/dz in
  // dzv, 1/dt in der2) saves three IEEE divisions per cell and moves r by a few ulp
  const float d = rc * (__ldg(u + o + 1) - __ldg(u + o) + __ldg(v + o + g.px) - __ldg(v + o)) * U.dzv.y +
                  (rhoW(F.B, g.nz, ck + 1) * wt - rhoW(F.B, g.nz, ck) * wb) * U.dzv.z;
  const float r = d * U.der2.x;
  if (F.rhs_hi) {  // tensor-core solve: write the split directly in its [z][y][x] layout with pitch rhs_ld
    const long o2 = (long(ck) * g.nyp + (cj + g.pad)) * F.rhs_ld + (ci + g.pad);
    const __nv_bfloat16 h = __float2bfloat16_rn(r);
    F.rhs_hi[o2] = h;
    if (F.rhs_lo) F.rhs_lo[o2] = __float2bfloat16_rn(r - __bfloat162float(h));   // none when no pass reads it
  }
  if (F.rhs) F.rhs[g.pidx(ci, cj, ck)] = r;  // fp32 solve, or the residual of the refined solve
}
__global__ void k_div(Grid g, Uni U, Fields F, int par) { div_body(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void k_div_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  div_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_PROJ (model.js:927-946): u -= dt grad(phi), phi from the padded solve
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void proj_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  auto P = [&](int a, int b, int c) {
    return __ldg(F.phi + g.pidx(clampi(a, -g.pad, g.nx + g.pad - 1), clampi(b, -g.pad, g.ny + g.pad - 1), clampi(c, 0, g.nz - 1)));
  };
  const int o = g.at(ci, cj, ck);
  const float kx = U.der.x, kz = U.der.y;
  const float pc = P(ci, cj, ck);
  float u = __ldg(F.V[par][0] + o), v = __ldg(F.V[par][1] + o), w = __ldg(F.V[par][2] + o);
  if (cj < g.ny && ck < g.nz) u = u - kx * (pc - P(ci - 1, cj, ck));
  if (ci < g.nx && ck < g.nz) v = v - kx * (pc - P(ci, cj - 1, ck));
  if (ci < g.nx && cj < g.ny && ck > 0 && ck < g.nz) w = w - kz * (pc - P(ci, cj, ck - 1));
  else w = 0.f;
  F.V[1 - par][0][o] = u;
  F.V[1 - par][1][o] = v;
  F.V[1 - par][2][o] = w;
  F.V[1 - par][3][o] = __ldg(F.V[par][3] + o);
}
__global__ void k_proj(Grid g, Uni U, Fields F, int par) { proj_body(g, U, F, par, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void k_proj_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  proj_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// accumulated surface precipitation (no counterpart in the reference): rho(0) sum_x q_x vt_x at the lowest level
__device__ __forceinline__ void rain_body(const Grid& g, const Uni& U, const Fields& F, int par, const int BX, const int BY, const int BZ) {
  const int i = BX * blockDim.x + threadIdx.x, j = BY * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int o = g.at(i, j, 0);
  const Fall fl{U.step.z, U.micro2.z > 0.5f, U.hur3.w > 0.5f && U.micro2.z <= 0.5f};
  const float rho = bsA(F.B, g.nz, 0).z;
  const float qr = F.Q[0][3][o], qs = F.Q[0][4][o], qg = F.Q[0][5][o];
  const float2 fv = fl.vtRain(qr, F.Q[0][6][o], rho);
  const double flux = double(rho) * (double(qr) * double(fv.x) + double(qs) * double(fl.vtS(qs, rho)) + double(qg) * double(fl.vtGrau(qg, rho)));
  F.rain[j * g.nx + i] += flux * double(U.step.x);
  if (i == 0 && j == 0) *F.clock += double(U.step.x);  // the step's last pass advances the model time
}
__global__ void k_rain(Grid g, Uni U, Fields F) { rain_body(g, U, F, 0, blockIdx.x, blockIdx.y, blockIdx.z); }
__global__ void k_rain_grp(const uint2* __restrict__ map, int par) {
  OB_GROUP_RESOLVE
  rain_body(c_members[mem].g, c_members[mem].U, c_members[mem].F, par, gbx, gby, gbz);
}

// ---------------------------------------------------------------------------------------------------------------
// WGSL_M_MAP (model.js:1028-1100): 16 diagnostics per column
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_maps(Grid g, Uni U, Fields F, int par, float4* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const float* const* V = F.V[par];
  auto L = [&](int ch, int a, int b, int c) { return __ldg(V[ch] + g.at(clampi(a, 0, nx), clampi(b, 0, ny), clampi(c, 0, nz))); };
  auto cvel = [&](int a, int b, int c, float v[3]) {
    v[0] = 0.5f * (L(0, a, b, c) + L(0, a + 1, b, c));
    v[1] = 0.5f * (L(1, a, b, c) + L(1, a, b + 1, c));
    v[2] = 0.5f * (L(2, a, b, c) + L(2, a, b, c + 1));
  };
  const Fall fl{U.step.z, U.micro2.z > 0.5f, U.hur3.w > 0.5f && U.micro2.z <= 0.5f};
  auto dbz = [&](int k) {
    const int o = g.at(i, j, k);
    const float rho = bsA(F.B, nz, k).z;
    const float T = __ldg(V[3] + o) * bsB(F.B, nz, k).x;
    const float Zr = fl.zRain(__ldg(F.Q[0][3] + o), __ldg(F.Q[0][6] + o), rho);
    const float Zs = 9.80e8f * powf(fmaxf(rho * __ldg(F.Q[0][4] + o), 0.f), 1.75f) * 0.224f * 4.f;
    const float Zg = fl.zGrau(__ldg(F.Q[0][5] + o), rho, T);
    const float Z = Zr + Zs + Zg;
    return Z > 1e-3f ? 10.f * logf(Z) / 2.302585f : -30.f;
  };
  auto zeta = [&](int k) {
    float a[3], b[3], c[3], d[3];
    cvel(i + 1, j, k, a);
    cvel(i - 1, j, k, b);
    cvel(i, j + 1, k, c);
    cvel(i, j - 1, k, d);
    return (a[1] - b[1] - c[0] + d[0]) / (2.f * U.dims.w);
  };
  const float dz = U.dzv.x;
  float comp = -30.f, wmx = 0.f, uh = 0.f;
  const int k12 = min(int(12000.f / dz), nz - 1);
  for (int k = 0; k < k12; k++) {
    float v[3];
    cvel(i, j, k, v);
    wmx = fmaxf(wmx, v[2]);
    comp = fmaxf(comp, dbz(k));
    const float z = (float(k) + 0.5f) * dz;
    if (z > 2000.f && z < 5000.f && v[2] > 0.f) uh += v[2] * fmaxf(zeta(k), 0.f) * dz;
  }
  const int k1 = clampi(int(1000.f / dz), 1, nz - 2);
  float v0[3], v1[3];
  cvel(i, j, 0, v0);
  cvel(i, j, k1, v1);
  const float conv = -((L(0, i + 1, j, 0) - L(0, i, j, 0) + L(1, i, j + 1, 0) - L(1, i, j, 0)) / U.dims.w) * 1000.f;
  const int idx = j * nx + i, n2 = nx * ny;
  out[idx] = make_float4(comp, dbz(k1), L(3, i, j, 0) - bsA(F.B, nz, 0).x, zeta(k1));
  out[idx + n2] = make_float4(wmx, uh, conv, sqrtf(v0[0] * v0[0] + v0[1] * v0[1]));
  out[idx + 2 * n2] = make_float4(v0[0], v0[1], v1[0], v1[1]);
  float tr = 1.f, bt = 0.f;
  for (int k = nz - 1; k >= 0; k--) {
    const int o = g.at(i, j, k);
    const float dtau = (80.f * __ldg(F.Q[0][1] + o) + 60.f * __ldg(F.Q[0][2] + o) + 25.f * __ldg(F.Q[0][4] + o) + 4.f * __ldg(F.Q[0][5] + o) +
                        1.f * __ldg(F.Q[0][3] + o)) * bsA(F.B, nz, k).z * dz;
    const float a = 1.f - expf(-dtau);
    bt += tr * a * __ldg(V[3] + o) * bsB(F.B, nz, k).x;
    tr *= 1.f - a;
    if (tr < 1e-3f) break;
  }
  const float sst = F.sfc[idx].y;
  bt += tr * (sst > 200.f ? sst : L(3, i, j, 0) * bsB(F.B, nz, 0).x);
  const float ps = bsA(F.B, nz, 0).z * U.cn.z * __ldg(F.phi + (i + g.pad) + g.nxp * (j + g.pad)) / 100.f;
  const int k5 = clampi(int(5000.f / dz), 1, nz - 2);
  out[idx + 3 * n2] = make_float4(ps, bt, U.hur2.w * sqrtf(v0[0] * v0[0] + v0[1] * v0[1]), zeta(k5));
}

// ---------------------------------------------------------------------------------------------------------------
// layout conversion between the texel float4 layout of the C ABI and the device SoA layout
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_pack(Grid g, Ptr8 src, int nch, int X, int Y, int Z, float* dst) {
  OB_BLOCKS_DIRECT
  OB_TEXEL_LOOP_BEGIN(X - 1, Y - 1, Z - 1)
  const int o = g.at(ci, cj, ck);
  const size_t t = (size_t(ck) * Y + cj) * X + ci;
#pragma unroll
  for (int c = 0; c < 8; c++)
    if (c < nch) dst[t * nch + c] = src.p[c][o];
}
__global__ void k_unpack(Grid g, Ptr8 dst, int nch, int X, int Y, int Z, const float* src) {
  OB_BLOCKS_DIRECT
  OB_TEXEL_LOOP_BEGIN(X - 1, Y - 1, Z - 1)
  const int o = g.at(ci, cj, ck);
  const size_t t = (size_t(ck) * Y + cj) * X + ci;
#pragma unroll
  for (int c = 0; c < 8; c++)
    if (c < nch) dst.p[c][o] = src[t * nch + c];
}

// ---------------------------------------------------------------------------------------------------------------
// hurricane mode: the advection with midpoint trajectories and settling ice, the pressure force carried along the
// trajectories (WGSL_M_PREP) and the 2-dx filter (WGSL_M_FILT). Straight restatements, one thread per texel, no
// clear-air skip (these runs are the few, not the bench's).
// ---------------------------------------------------------------------------------------------------------------
// the winds at a point in grid units, from the true winds (model.js:420-423)
__device__ __forceinline__ void velAt(const Fields& F, const Grid& g, int par, float x, float y, float z, float v[3]) {
  v[0] = sampleVch(F.V[par][0], g, 0, x, y, z);
  v[1] = sampleVch(F.V[par][1], g, 1, x, y, z);
  v[2] = sampleVch(F.V[par][2], g, 2, x, y, z);
}
// departure (s = 1) or forward (s = -1) point: first order, or with the wind at the midpoint when cn.w (model.js:424-433)
__device__ __forceinline__ void traceH(const Uni& U, const Fields& F, const Grid& g, int par, const float k[3], float px, float py,
                                       float pz, const float v[3], float s, float& x, float& y, float& z) {
  if (U.cn.w < 0.5f) {
    traceV(g, k, px, py, pz, v, s, x, y, z);
    return;
  }
  float mx, my, mz, vm[3];
  traceV(g, k, px, py, pz, v, 0.5f * s, mx, my, mz);
  velAt(F, g, par, mx, my, mz, vm);
  traceV(g, k, px, py, pz, vm, s, x, y, z);
}
// the same for a cell centre and something falling at `fall` (model.js:494-499)
__device__ __forceinline__ void traceQH(const Uni& U, const Fields& F, const Grid& g, int par, const float k[3], const float p[3],
                                        const float v[3], float fall, float s, float& x, float& y, float& z) {
  if (U.cn.w < 0.5f) {
    traceQ(g, k, p, v, fall, s, x, y, z);
    return;
  }
  const float mx = clampf(p[0] - 0.5f * s * k[0] * v[0], 0.f, float(g.nx));
  const float my = clampf(p[1] - 0.5f * s * k[1] * v[1], 0.f, float(g.ny));
  const float mz = clampf(p[2] - 0.5f * s * k[2] * (v[2] - fall), 0.f, float(g.nz));
  float vm[3];
  velAt(F, g, par, mx, my, mz, vm);
  traceQ(g, k, p, vm, fall, s, x, y, z);
}

__global__ void k_prep(Grid g, Uni U, Fields F, int par) {
  OB_BLOCKS_DIRECT
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  auto P = [&](int a, int b, int c) {
    return __ldg(F.phi + g.pidx(clampi(a, -g.pad, g.nx + g.pad - 1), clampi(b, -g.pad, g.ny + g.pad - 1), clampi(c, 0, g.nz - 1)));
  };
  const int o = g.at(ci, cj, ck);
  const float f = U.cn.x * U.cn.y;
  const float kx = f * U.step.x / U.dims.w, kz = f * U.step.x / U.dzv.x;
  const float pc = P(ci, cj, ck);
  float u = __ldg(F.V[par][0] + o), v = __ldg(F.V[par][1] + o), w = __ldg(F.V[par][2] + o);
  if (cj < g.ny && ck < g.nz) u = u - kx * (pc - P(ci - 1, cj, ck));
  if (ci < g.nx && ck < g.nz) v = v - kx * (pc - P(ci, cj - 1, ck));
  if (ci < g.nx && cj < g.ny && ck > 0 && ck < g.nz) w = w - kz * (pc - P(ci, cj, ck - 1));
  F.Vp[0][o] = u;
  F.Vp[1][o] = v;
  F.Vp[2][o] = w;
  F.Vp[3][o] = __ldg(F.V[par][3] + o);
}

// 4th-order horizontal hyperdiffusion of V and Q into V[1-par], Q slot 1 (model.js:948-994)
__global__ void k_filt(Grid g, Uni U, Fields F, int par) {
  OB_BLOCKS_DIRECT
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  const float a = U.hur5.z;
  auto bih = [&](const float* __restrict__ f, int X, int Y) {
    auto L = [&](int i, int j) { return __ldg(f + g.at(clampi(i, 0, X), clampi(j, 0, Y), ck)); };
    return 20.f * L(ci, cj) - 8.f * (L(ci + 1, cj) + L(ci - 1, cj) + L(ci, cj + 1) + L(ci, cj - 1)) +
           2.f * (L(ci + 1, cj + 1) + L(ci + 1, cj - 1) + L(ci - 1, cj + 1) + L(ci - 1, cj - 1)) + L(ci + 2, cj) + L(ci - 2, cj) +
           L(ci, cj + 2) + L(ci, cj - 2);
  };
  const int o = g.at(ci, cj, ck);
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float val = __ldg(F.V[par][c] + o) - a * bih(F.V[par][c], g.nx, g.ny);
    if (c == 2 && (ck == 0 || ck >= g.nz)) val = 0.f;  // the lid / ground faces of w stay zero
    F.V[1 - par][c][o] = val;
  }
  if (ci < g.nx && cj < g.ny && ck < g.nz) {
#pragma unroll
    for (int c = 0; c < 8; c++) F.Q[1][c][o] = fmaxf(__ldg(F.Q[0][c] + o) - a * bih(F.Q[0][c], g.nx - 1, g.ny - 1), 0.f);
  }
}

// ADVV1/2 of hurricane mode (model.js:434-481): trajectories from the true winds, values carried from Vp
__global__ void k_advv1_hur(Grid g, Uni U, Fields F, int par) {
  OB_BLOCKS_DIRECT
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  const Loc L = localVel(F, g, par, ci, cj, ck);
  const float kk[3] = {U.der.x, U.der.x, U.der.y};
  const float fi = float(ci), fj = float(cj), fk = float(ck);
  const int o = g.at(ci, cj, ck);
  const float P[4][3] = {{fi, fj + 0.5f, fk + 0.5f}, {fi + 0.5f, fj, fk + 0.5f}, {fi + 0.5f, fj + 0.5f, fk}, {fi + 0.5f, fj + 0.5f, fk + 0.5f}};
  const float* vel[4] = {L.vu, L.vv, L.vw, L.vc};
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float x, y, z;
    traceH(U, F, g, par, kk, P[c][0], P[c][1], P[c][2], vel[c], 1.f, x, y, z);
    F.Vt[c][o] = sampleVch(F.Vp[c], g, c, x, y, z);
  }
}
__global__ void k_advv2_hur(Grid g, Uni U, Fields F, int par) {
  OB_BLOCKS_DIRECT
  OB_TEXEL_LOOP_BEGIN(g.nx, g.ny, g.nz)
  const Loc L = localVel(F, g, par, ci, cj, ck);
  const float kk[3] = {U.der.x, U.der.x, U.der.y};
  const float fi = float(ci), fj = float(cj), fk = float(ck);
  const float P[4][3] = {{fi, fj + 0.5f, fk + 0.5f}, {fi + 0.5f, fj, fk + 0.5f}, {fi + 0.5f, fj + 0.5f, fk}, {fi + 0.5f, fj + 0.5f, fk + 0.5f}};
  const float* vel[4] = {L.vu, L.vv, L.vw, L.vc};
  const float cx = L.vc[0] * kk[0], cy = L.vc[1] * kk[1], cz = L.vc[2] * kk[2];
  const float cour = sqrtf(cx * cx + cy * cy + cz * cz);
  const float sm = 0.5f * U.misc.y * clampf(cour / 0.35f, U.dzv.w, 1.f);
  const int o = g.at(ci, cj, ck);
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const float ox = c == 0 ? 0.f : 0.5f, oy = c == 1 ? 0.f : 0.5f, oz = c == 2 ? 0.f : 0.5f;
    float x, y, z;
    traceH(U, F, g, par, kk, P[c][0], P[c][1], P[c][2], vel[c], -1.f, x, y, z);
    const float b = sampleVch(F.Vt[c], g, c, x, y, z);
    const float hat = __ldg(F.Vt[c] + o), old = __ldg(F.Vp[c] + o);
    const float r = hat + sm * (old - b);
    traceH(U, F, g, par, kk, P[c][0], P[c][1], P[c][2], vel[c], 1.f, x, y, z);
    const float2 m = minmax8V(F.Vp[c], g, x, y, z, ox, oy, oz);
    F.V[1 - par][c][o] = clampf(r, m.x, m.y);
  }
}

// ADVQ1/2 of hurricane mode (model.js:500-576): every channel, maritime graupel, settling ice. The brick flags of the
// clear-air skip are left saying "may hold hydrometeors", so that a later run without the hurricane stays exact.
__device__ __forceinline__ void brick_flags_all(const Grid& g, const Fields& F, unsigned* a, unsigned* zq, unsigned* z1) {
  if (threadIdx.x == 0 && threadIdx.y == 0 && int(blockIdx.x) < F.nbx && int(blockIdx.y) < F.nby && int(blockIdx.z) < g.nz) {
    const int b = blockIdx.x + F.nbx * (blockIdx.y + F.nby * blockIdx.z);
    if (a) a[b] = 1u;
    if (zq) zq[b] = 0u;
    if (z1) z1[b] = 0u;
  }
}
__global__ void k_advq1_hur(Grid g, Uni U, Fields F, int par) {
  brick_flags_all(g, F, F.actQt, F.zeroQt, nullptr);
  const int ci = blockIdx.x * blockDim.x + threadIdx.x, cj = blockIdx.y * blockDim.y + threadIdx.y, ck = blockIdx.z;
  if (ci >= g.nx || cj >= g.ny || ck >= g.nz) return;
  const int o = g.at(ci, cj, ck);
  const float kk[3] = {U.der.x, U.der.x, U.der.y};
  const float p[3] = {float(ci) + 0.5f, float(cj) + 0.5f, float(ck) + 0.5f};
  float v[3];
  cellVel(F, g, par, ci, cj, ck, v);
  const float rho = bsA(F.B, g.nz, ck).z;
  const bool thm = U.micro2.z > 0.5f;
  const Fall fl{U.step.z, thm, U.hur3.w > 0.5f && !thm};
  const float2 fv = fl.vtRain(__ldg(F.Q[0][3] + o), __ldg(F.Q[0][6] + o), rho);
  const float fs = fl.vtS(__ldg(F.Q[0][4] + o), rho), fg = fl.vtGrau(__ldg(F.Q[0][5] + o), rho), fi = vtI(U, __ldg(F.Q[0][2] + o), rho);
  float x, y, z;
  auto at = [&](float fall, int c) {
    traceQH(U, F, g, par, kk, p, v, fall, 1.f, x, y, z);
    return gatherQ(F.Q[0][c], tapQ(g, x, y, z));
  };
  traceQH(U, F, g, par, kk, p, v, 0.f, 1.f, x, y, z);
  const Tap t0 = tapQ(g, x, y, z);
  F.Qt[0][o] = gatherQ(F.Q[0][0], t0);
  F.Qt[1][o] = gatherQ(F.Q[0][1], t0);
  F.Qt[2][o] = fi > 0.f ? at(fi, 2) : gatherQ(F.Q[0][2], t0);
  F.Qt[3][o] = at(fv.x, 3);
  F.Qt[4][o] = at(fs, 4);
  F.Qt[5][o] = at(fg, 5);
  F.Qt[6][o] = thm ? at(fv.y, 6) : gatherQ(F.Q[0][6], t0);
  F.Qt[7][o] = gatherQ(F.Q[0][7], t0);
}
__global__ void k_advq2_hur(Grid g, Uni U, Fields F, int par) {
  brick_flags_all(g, F, nullptr, nullptr, F.zeroQ1);
  const int ci = blockIdx.x * blockDim.x + threadIdx.x, cj = blockIdx.y * blockDim.y + threadIdx.y, ck = blockIdx.z;
  if (ci >= g.nx || cj >= g.ny || ck >= g.nz) return;
  const int o = g.at(ci, cj, ck);
  const float kk[3] = {U.der.x, U.der.x, U.der.y};
  const float p[3] = {float(ci) + 0.5f, float(cj) + 0.5f, float(ck) + 0.5f};
  float v[3];
  cellVel(F, g, par, ci, cj, ck, v);
  const float rho = bsA(F.B, g.nz, ck).z;
  const bool thm = U.micro2.z > 0.5f;
  const Fall fl{U.step.z, thm, U.hur3.w > 0.5f && !thm};
  float q[8];
#pragma unroll
  for (int c = 0; c < 8; c++) q[c] = __ldg(F.Q[0][c] + o);
  const float2 fv = fl.vtRain(q[3], q[6], rho);
  const float fs = fl.vtS(q[4], rho), fg = fl.vtGrau(q[5], rho), fi = vtI(U, q[2], rho);
  const float fn = thm ? fv.y : 0.f;
  const float cx = v[0] * kk[0], cy = v[1] * kk[1], cz = v[2] * kk[2];
  const float cour = sqrtf(cx * cx + cy * cy + cz * cz);
  const float sm = 0.5f * U.misc.y * clampf(cour / 0.35f, U.dzv.w, 1.f);
  // each channel's fall speed (0: the air's)
  const float fall[8] = {0.f, 0.f, fi, fv.x, fs, fg, fn, 0.f};
  float x, y, z;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    traceQH(U, F, g, par, kk, p, v, fall[c], -1.f, x, y, z);
    const float b = gatherQ(F.Qt[c], tapQ(g, x, y, z));
    const float r = __ldg(F.Qt[c] + o) + sm * (q[c] - b);
    traceQH(U, F, g, par, kk, p, v, fall[c], 1.f, x, y, z);
    const float2 m = minmaxQ(F.Q[0][c], tapQ(g, x, y, z));
    F.Q[1][c][o] = fmaxf(clampf(r, m.x, m.y), 0.f);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------------------------------
static inline dim3 grid3(int X, int Y, int Z, dim3 b) { return dim3((X + b.x - 1) / b.x, (Y + b.y - 1) / b.y, Z); }
static const dim3 kB3(32, 4, 1);
static const dim3 kB2(32, 8, 1);

void launch_lsf(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s) {
  k_lsf<<<grid3(g.nx, g.ny, 1, kB2), kB2, 0, s>>>(g, U, F);
}
void launch_ci(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s) {
  k_ci<<<grid3(g.nx, g.ny, 1, kB2), kB2, 0, s>>>(g, U, F);
}
void launch_init(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s) {
  k_init<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F);
}
void launch_nut(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s) {
  if (U.hur.x > 0.5f) k_nut_hur<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, U, F, par);
  else k_nut<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, U, F, par);
}
void launch_advv(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s) {
  if (U.hur.x > 0.5f && F.Vp[0]) {
    k_advv1_hur<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
    k_advv2_hur<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
    return;
  }
  k_advv1<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
  k_advv2<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
}
void launch_advq(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s) {
  if (U.hur.x > 0.5f) {
    k_advq1_hur<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, U, F, par);
    k_advq2_hur<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, U, F, par);
    return;
  }
  k_advq1<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, U, F, par);
  k_advq2<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, U, F, par);
}
void launch_prep(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s) {
  k_prep<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
}
void launch_filt(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s) {
  k_filt<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
}
void launch_activity(const Grid& g, const Fields& F, cudaStream_t s) {
  k_activity<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, F);
}
void launch_tables(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s) {
  const int n = std::max(g.nz, std::max(g.nx, g.ny)) + 1;
  k_tables<<<(n + 127) / 128, 128, 0, s>>>(g, U, F.B, const_cast<float*>(F.spz), const_cast<float*>(F.slx), const_cast<float*>(F.sly));
}
void launch_phys(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s, int micro_mode) {
  if (U.hur.x > 0.5f) {  // hurricane mode runs the scheme (model.js:578-907 with its hurricane branches)
    k_phys_hur<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
    return;
  }
  const dim3 grid = grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3);
  const bool bnd = U.cor.z > 0.5f;
  if (micro_mode == kMicroRecord) {
    if (bnd) k_phys<kMicroRecord, 1><<<grid, kB3, 0, s>>>(g, U, F, par);
    else k_phys<kMicroRecord, 0><<<grid, kB3, 0, s>>>(g, U, F, par);
  } else if (micro_mode == kMicroSurrogate) {
    if (bnd) k_phys<kMicroSurrogate, 1><<<grid, kB3, 0, s>>>(g, U, F, par);
    else k_phys<kMicroSurrogate, 0><<<grid, kB3, 0, s>>>(g, U, F, par);
  } else {
    if (bnd) k_phys<kMicroPlain, 1><<<grid, kB3, 0, s>>>(g, U, F, par);
    else k_phys<kMicroPlain, 0><<<grid, kB3, 0, s>>>(g, U, F, par);
  }
}
void launch_div(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s) {
  k_div<<<grid3(g.nx, g.ny, g.nz, kB3), kB3, 0, s>>>(g, U, F, par);
}
void launch_proj(const Grid& g, const Uni& U, const Fields& F, int par, cudaStream_t s) {
  k_proj<<<grid3(g.nx + 1, g.ny + 1, g.nz + 1, kB3), kB3, 0, s>>>(g, U, F, par);
}
void launch_rain(const Grid& g, const Uni& U, const Fields& F, cudaStream_t s) {
  k_rain<<<grid3(g.nx, g.ny, 1, kB2), kB2, 0, s>>>(g, U, F);
}
void launch_maps(const Grid& g, const Uni& U, const Fields& F, int par, float4* out, cudaStream_t s) {
  k_maps<<<grid3(g.nx, g.ny, 1, kB2), kB2, 0, s>>>(g, U, F, par, out);
}

// ---------------------------------------------------------------------------------------------------------------
// tornado candidates of the sub-grid tornado scheme (tornadoCandidates, app.js:1457-1472) on the device maps: on the
// stride-2 lattice 6 cells inside the edges, a point whose 1-km vorticity (map0.w) is at least zmin and whose
// low-level theta' (map0.z) is not below -4.5 K, that has the largest vorticity of its stride-2 5 x 5 window, with a
// window maximum of 2-5 km updraft helicity (map1.y) above 60 m2/s2 and of updraft (map1.x) above 12 m/s. Appends
// (i, j, x, y, zeta, uh, w) per candidate; the host restores the lattice order (j, then i).
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_tor_candidates(const float4* __restrict__ maps, int nx, int ny, float dx, float zmin, float* out, int cap,
                                 unsigned* count) {
  const int i = 6 + 2 * (blockIdx.x * blockDim.x + threadIdx.x), j = 6 + 2 * (blockIdx.y * blockDim.y + threadIdx.y);
  if (i >= nx - 6 || j >= ny - 6) return;
  const float4* m0 = maps;
  const float4* m1 = maps + size_t(nx) * ny;
  const float4 c = __ldg(m0 + j * nx + i);
  const float z1 = c.w;
  if (z1 < zmin || c.z < -4.5f) return;
  bool is_max = true;
  float uh = 0.f, w = 0.f;
  for (int dj = -4; dj <= 4; dj += 2)
    for (int di = -4; di <= 4; di += 2) {
      const int q = (i + di) + nx * (j + dj);
      if ((di || dj) && __ldg(m0 + q).w > z1) is_max = false;
      const float4 b = __ldg(m1 + q);
      uh = fmaxf(uh, b.y);
      w = fmaxf(w, b.x);
    }
  if (!(is_max && uh > 60.f && w > 12.f)) return;
  const unsigned slot = atomicAdd(count, 1u);
  if (slot >= unsigned(cap)) return;
  float* o = out + size_t(slot) * 7;
  o[0] = float(i); o[1] = float(j); o[2] = (float(i) + 0.5f) * dx; o[3] = (float(j) + 0.5f) * dx; o[4] = z1; o[5] = uh; o[6] = w;
}
// ---------------------------------------------------------------------------------------------------------------
// grouped launches (ensemble steps)
// ---------------------------------------------------------------------------------------------------------------
int group_kind(int pass) {
  switch (pass) {
    case kGroupLSF: case kGroupCI: case kGroupRAIN: return kGroup2D;
    case kGroupNUT: case kGroupADVQ1: case kGroupADVQ2: case kGroupDIV: return kGroupCell;
    default: return kGroupStag;
  }
}

dim3 group_default_block(int pass) { return group_kind(pass) == kGroup2D ? kB2 : kB3; }

bool group_block_fixed(int pass) {
  // the scalar advection and the physics pass share the 32 x 4 bricks of the clear-air flags; the 2-D passes are
  // not worth tuning
  return pass == kGroupADVQ1 || pass == kGroupADVQ2 || pass == kGroupPHYS || group_kind(pass) == kGroup2D;
}

int group_map(const Grid* grids, const int* pos, int n, int pass, dim3 block, std::vector<uint2>& map) {
  if (n < 1 || n > kMaxMembers) return -1;
  const int kind = group_kind(pass);
  map.clear();
  int Z = -1;
  for (int i = 0; i < n; i++) {
    const Grid& g = grids[i];
    int X = g.nx, Y = g.ny, z = g.nz;
    if (kind == kGroupStag) { X++; Y++; z++; }
    if (kind == kGroup2D) z = 1;
    if (Z >= 0 && z != Z) return -1;  // the members share nz
    Z = z;
    const int gx = (X + block.x - 1) / block.x, gy = (Y + block.y - 1) / block.y;
    if (gx > 65535 || gy > 65535) return -1;
    for (int by = 0; by < gy; by++)
      for (int bx = 0; bx < gx; bx++) map.push_back(make_uint2(unsigned(pos[i]), unsigned(bx) | (unsigned(by) << 16)));
  }
  return Z;
}

int group_upload_members(const MemberC* d_src, int n, cudaStream_t s) {
  if (n < 1 || n > kMaxMembers) return -1;
  return cudaMemcpyToSymbolAsync(c_members, d_src, sizeof(MemberC) * n, 0, cudaMemcpyDeviceToDevice, s) == cudaSuccess ? 0 : -1;
}

void launch_group(int pass, const uint2* map, int nxy, int Z, dim3 block, int par, cudaStream_t s, int micro_mode) {
  if (nxy < 1 || Z < 1) return;
  const dim3 grid(nxy, 1, Z);
  switch (pass) {
    case kGroupLSF: k_lsf_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupCI: k_ci_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupNUT: k_nut_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupADVV1: k_advv1_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupADVV2: k_advv2_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupADVQ1: k_advq1_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupADVQ2: k_advq2_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupPHYS:
      if (micro_mode == kMicroRecord) k_phys_grp<kMicroRecord><<<grid, block, 0, s>>>(map, par);
      else if (micro_mode == kMicroSurrogate) k_phys_grp<kMicroSurrogate><<<grid, block, 0, s>>>(map, par);
      else k_phys_grp<kMicroPlain><<<grid, block, 0, s>>>(map, par);
      break;
    case kGroupDIV: k_div_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupPROJ: k_proj_grp<<<grid, block, 0, s>>>(map, par); break;
    case kGroupRAIN: k_rain_grp<<<grid, block, 0, s>>>(map, par); break;
    default: break;
  }
}

void launch_tor_candidates(const Grid& g, float dx, const float4* maps, float zmin, float* out, int cap, unsigned* count, cudaStream_t s) {
  const int ni = (g.nx - 12 + 1) / 2, nj = (g.ny - 12 + 1) / 2;
  if (ni <= 0 || nj <= 0) return;
  k_tor_candidates<<<dim3((ni + 31) / 32, (nj + 7) / 8), dim3(32, 8), 0, s>>>(maps, g.nx, g.ny, dx, zmin, out, cap, count);
}
void launch_pack(const Grid& g, const Ptr8& src, int nch, int X, int Y, int Z, float* dst, cudaStream_t s) {
  k_pack<<<grid3(X, Y, Z, kB3), kB3, 0, s>>>(g, src, nch, X, Y, Z, dst);
}
void launch_unpack(const Grid& g, const Ptr8& dst, int nch, int X, int Y, int Z, const float* src, cudaStream_t s) {
  k_unpack<<<grid3(X, Y, Z, kB3), kB3, 0, s>>>(g, dst, nch, X, Y, Z, src);
}

}  // namespace ob
