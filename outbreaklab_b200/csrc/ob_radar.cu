// ob_radar.cu — virtual WSR-88D gate sampling for sm_100a (radar.js:41-268).
//
// k_radar_cut restates WGSL_R_CUT: one thread per gate (the reference packs 4 gates per thread), gates of one radial
// along x so that neighbouring lanes sample neighbouring points of the model (250 m apart) and share L1 lines. Each
// gate samples the model three times across the beam (beam filling), turns the hydrometeors into reflectivity,
// radial velocity, spectrum width, ZDR, rho_hv and KDP, and stores one 8-bit Level II code per moment. The codes go
// out as bytes: a warp stores 32 consecutive codes of a radial, which is the reference's little-endian packing of
// 4 codes per u32 word (radar.js:229-240) written as one 32-byte sector.
//
// k_radar_phi restates WGSL_R_PHI: PhiDP is a running fp32 sum of 2 * KDP * dr along each radial, in gate order, so
// each radial stays sequential (a parallel scan would round differently). One warp handles 32 radials: it stages a
// 32 x 32 tile of KDP through shared memory so the global reads and the code stores are coalesced, then every lane
// walks its own radial through the tile.
//
// The quantisation code() and the PhiDP accumulation use explicitly rounded fp32 operations (no FMA contraction),
// so identical moments give bit-identical codes to the CPU restatement; the geometry and microphysics use CUDA's
// IEEE-accurate math functions and may contract to FMA.
#include <cstdint>

#include "ob_common.cuh"
#include "ob_radar.cuh"

namespace ob {

namespace {

struct Smp {
  float zr, zs, zg, vt, u, v, w, T, rho, nu, lr;
  bool inside;
};

__device__ __forceinline__ float db2lin(float d) { return powf(10.f, 0.1f * d); }
__device__ __forceinline__ float sqf(float x) { return x * x; }

// WGSL code(): u32(clamp(round(v * sc + ofs), 2, 255)), round half-to-even
__device__ __forceinline__ uint32_t lcode(float v, float sc, float ofs) {
  const float t = rintf(__fadd_rn(__fmul_rn(v, sc), ofs));
  return uint32_t(fminf(fmaxf(t, 2.f), 255.f));
}

// great-circle destination (bearing a rad, ground distance s m) -> model metres (radar.js:51-64)
__device__ __forceinline__ float2 gatePos(const RadarU& R, float a, float s) {
  const float RE = 6371000.f;
  const float p1 = R.geo.z, l1 = R.geo.w, d = s / RE;
  const float sp2 = sinf(p1) * cosf(d) + cosf(p1) * sinf(d) * cosf(a);
  const float p2 = asinf(clampf(sp2, -1.f, 1.f));
  const float l2 = l1 + atan2f(sinf(a) * sinf(d) * cosf(p1), cosf(d) - sinf(p1) * sp2);
  const float p0 = R.geo.x, dl = l2 - R.geo.y;
  const float cc = clampf(sinf(p0) * sinf(p2) + cosf(p0) * cosf(p2) * cosf(dl), -1.f, 1.f);
  const float c = acosf(cc);
  const float k = c < 1e-6f ? 1.f : c / sinf(c);
  return make_float2(RE * k * cosf(p2) * sinf(dl) - R.mdl2.z, RE * k * (cosf(p0) * sinf(p2) - sinf(p0) * cosf(p2) * cosf(dl)) - R.mdl2.w);
}
// 4/3-earth beam: (height above the antenna, ground distance) at slant range r (radar.js:66-72)
__device__ __forceinline__ float2 beam(const RadarU& R, float r, float el) {
  const float a = R.site.w;
  const float q = r * r + 2.f * r * a * sinf(el);
  const float h = q / (sqrtf(q + a * a) + a);
  return make_float2(h, a * asinf(clampf(r * cosf(el) / (a + h), -1.f, 1.f)));
}

// radar.js:89-139; full = false skips what the outer samples of the beam never use (w, fall speed, nu)
template <bool FULL>
__device__ __forceinline__ Smp sample(const RadarU& R, const Grid& g, const Fields& F, int par, float px, float py, float z) {
  Smp o;
  const float n0 = R.mdl.x, n1 = R.mdl.y, n2 = R.mdl.z, dx = R.mdl.w, dz = R.mdl2.x;
  const float gx = px / dx, gy = py / dx, gz = z / dz;
  o.inside = gx >= 0.f && gy >= 0.f && gz >= 0.f && gx <= n0 && gy <= n1 && gz <= n2 && z >= 0.f;
  const float cx = clampf(gx, 0.f, n0), cy = clampf(gy, 0.f, n1), cz = clampf(gz, 0.f, n2);
  const float qx = cx - 0.5f, qy = cy - 0.5f, qz = cz - 0.5f;
  const bool thm = R.phys.z > 0.5f;
  const float qr = fmaxf(trilerp(F.Q[0][3], g, g.nx, g.ny, g.nz, qx, qy, qz), 0.f);
  const float qs = fmaxf(trilerp(F.Q[0][4], g, g.nx, g.ny, g.nz, qx, qy, qz), 0.f);
  const float qg = fmaxf(trilerp(F.Q[0][5], g, g.nx, g.ny, g.nz, qx, qy, qz), 0.f);
  const int X = g.nx + 1, Y = g.ny + 1, Z = g.nz + 1;
  o.u = trilerp(F.V[par][0], g, X, Y, Z, cx, cy - 0.5f, cz - 0.5f);
  o.v = trilerp(F.V[par][1], g, X, Y, Z, cx - 0.5f, cy, cz - 0.5f);
  o.w = FULL ? trilerp(F.V[par][2], g, X, Y, Z, cx - 0.5f, cy - 0.5f, cz) : 0.f;
  const float th = trilerp(F.V[par][3], g, X, Y, Z, qx, qy, qz);
  const int k = int(clampf(floorf(cz), 0.f, n2 - 1.f));
  const float4 A = bsA(F.B, g.nz, k), B = bsB(F.B, g.nz, k);
  const float rho = A.z, T = th * B.x;
  o.zr = 3.63e9f * powf(rho * qr, 1.75f);
  o.zs = 9.80e8f * powf(rho * qs, 1.75f) * 0.224f * 4.0f;
  o.zg = (T < 273.15f ? 1.2e10f : 4.33e10f) * powf(rho * qg, 1.75f);
  const float sq = sqrtf(R.phys.x / rho);
  float vr = 0.f, vs = 0.f, vg = 0.f;
  if (FULL) {
    vr = fminf(36.34f * powf(fmaxf(0.001f * rho * qr, 0.f), 0.1364f) * sq, 10.f * sq);
    vs = clampf(1.1f * powf(fmaxf(1000.f * rho * qs, 1e-6f), 0.11f), 0.3f, 2.2f) * sq;
    vg = clampf(9.f * powf(fmaxf(1000.f * rho * qg, 1e-6f), 0.42f), 1.f, 55.f) * sq;
    const float rr = qg / 0.009f;
    vg = fminf(vg * (1.f + rr * rr), 65.f);
  }
  // hurricane mode's maritime graupel (radar.js:113)
  if (R.phys2.x > 0.5f && !thm) {
    o.zg = (T < 273.15f ? 1.3e9f : 1.0e10f) * powf(rho * qg, 1.75f);
    if (FULL) vg = clampf(5.f * powf(fmaxf(1000.f * rho * qg, 1e-6f), 0.25f), 1.f, 9.f) * sq;
  }
  o.lr = FULL ? powf(float(3.14159 * 1000.0 * 8e6) / fmaxf(rho * qr, 1e-9f), 0.25f) : 0.f;
  if (thm) {
    const float nr = fmaxf(trilerp(F.Q[0][6], g, g.nx, g.ny, g.nz, qx, qy, qz), 0.f);
    if (qr > 1e-9f) {
      const float l = clampf(powf(float(3.14159 * 1000.0) * fmaxf(nr, 1e-3f) / qr, 0.33333f), 1000.f, 1.0e5f);
      const float nb = qr * l * l * l / 3141.59f;
      o.zr = 720e18f * rho * nb / powf(l, 6.f);
      if (FULL) {
        o.lr = l;
        vr = fminf(3949.f * powf(l, -0.8f), 10.f) * sq;
      }
    } else {
      o.zr = 0.f;
    }
    if (qg > 1e-9f) {
      const float n0g = clampf(200.f / (rho * qg), 1e4f, 3e6f);
      const float l = powf(float(3.14159 * 500.0) * n0g / (rho * qg), 0.25f);
      o.zg = 720e18f * n0g / powf(l, 7.f) * (T < 273.15f ? 0.0666f : 0.24f);
      if (FULL) vg = fminf(2483.f * powf(l, -0.89f), 30.f) * sq;
    } else {
      o.zg = 0.f;
    }
  }
  const float zt = o.zr + o.zs + o.zg;
  o.vt = (FULL && zt > 1e-6f) ? (o.zr * vr + o.zs * vs + o.zg * vg) / zt : 0.f;
  o.T = T;
  o.rho = rho;
  o.nu = FULL ? trilerp(F.aux[0], g, g.nx, g.ny, g.nz, qx, qy, qz) : 0.f;
  return o;
}

struct GateOut {
  uint32_t c[5];  // REF, VEL, SW, ZDR, RHO codes (0 = empty)
  float kdp;      // -1 = empty
  float m[6];     // moments (dBZ, Vr, SW, ZDR, rho_hv, KDP), NaN where empty
};

// radar.js:144-227
__device__ GateOut gate(const RadarU& R, const Grid& g, const Fields& F, int par, const float* __restrict__ tor, int ri, int gi) {
  GateOut G;
#pragma unroll
  for (int i = 0; i < 5; i++) G.c[i] = 0u;
  G.kdp = -1.f;
#pragma unroll
  for (int i = 0; i < 6; i++) G.m[i] = __int_as_float(0x7fc00000);
  const float r = R.gates.z + R.gates.w * float(gi);
  const float el = R.cut.x;
  const float az = (R.cut.y + R.cut.z * float(ri)) * 0.017453293f;
  const float bw = 0.0165f;
  const float2 hc = beam(R, r, el);
  const float2 p = gatePos(R, az, hc.y);
  const float2 p2 = gatePos(R, az, hc.y + 200.f);
  float ex = p2.x - p.x, ey = p2.y - p.y;
  const float en = sqrtf(ex * ex + ey * ey);
  ex /= en;
  ey /= en;
  const float zAnt = R.site.z - R.mdl2.y;
  const float zc = zAnt + hc.x;
  if (zc > R.mdl.z * R.mdl2.x - 200.f) return G;
  const float hl = beam(R, r, el - 0.4f * bw).x + zAnt, hu = beam(R, r, el + 0.4f * bw).x + zAnt;
  const Smp s0 = sample<true>(R, g, F, par, p.x, p.y, fmaxf(zc, 5.f));
  if (!s0.inside) return G;
  const Smp s1 = sample<false>(R, g, F, par, p.x, p.y, fmaxf(hl, 5.f));
  const Smp s2 = sample<false>(R, g, F, par, p.x, p.y, fmaxf(hu, 5.f));
  const float zr = 0.5f * s0.zr + 0.25f * (s1.zr + s2.zr), zs = 0.5f * s0.zs + 0.25f * (s1.zs + s2.zs);
  const float zg = 0.5f * s0.zg + 0.25f * (s1.zg + s2.zg);
  const float zmet = zr + zs + zg;
  // sub-grid tornadoes: beam-smeared Rankine vortex and lofted debris
  float zdeb = 0.f, dvx = 0.f, dvy = 0.f, swt = 0.f;
  const float bwm = 0.5f * r * bw;
  const int ntor = int(R.phys.w);
  for (int q = 0; q < ntor; q++) {
    const float4 A = __ldg(reinterpret_cast<const float4*>(tor) + 2 * q), B = __ldg(reinterpret_cast<const float4*>(tor) + 2 * q + 1);
    const float dxv = p.x - A.x, dyv = p.y - A.y;
    const float rt = sqrtf(dxv * dxv + dyv * dyv);
    const float Re = sqrtf(A.z * A.z + bwm * bwm + 125.f * 125.f);
    if (rt > 8.f * Re) continue;
    const float vmx = A.w * A.z / Re;
    const float vt = vmx * (rt < Re ? rt / Re : Re / fmaxf(rt, 1.f));
    const float ir = fmaxf(rt, 1.f);
    const float etx = -dyv / ir, ety = dxv / ir, erx = dxv / ir, ery = dyv / ir;
    const float fz = 1.f - sstep(1200.f, 3500.f, zc);
    dvx += (vt * etx - 0.25f * vt * erx) * fz;
    dvy += (vt * ety - 0.25f * vt * ery) * fz;
    swt = fmaxf(swt, vmx * 0.4f * expf(-rt * rt / (4.f * Re * Re)) * fz);
    if (B.z > 0.f && zc < B.x) {
      const float rd = fmaxf(1.4f * A.z, 150.f);
      zdeb += db2lin(B.y) * fminf(1.f, rd * rd / (Re * Re)) * expf(-rt * rt / (Re * Re)) * (1.f - sstep(0.55f * B.x, B.x, zc)) * B.z;
    }
  }
  const float ztot = zmet + zdeb;
  if (ztot <= 1e-6f) return G;
  const float dbz = 10.f * logf(ztot) / 2.302585f;
  if (dbz < R.phys.y) return G;
  G.m[0] = dbz;
  G.c[0] = lcode(dbz, 2.f, 66.f);
  if (gi >= int(R.gates.y)) return G;
  const float ce = cosf(el), se = sinf(el);
  const float vtf = s0.vt * zmet / ztot;
  float vr = ((s0.u + dvx) * ex + (s0.v + dvy) * ey) * ce + (s0.w - vtf) * se;
  const float nyq = R.nyq.x;
  vr = vr - 2.f * nyq * floorf((vr + nyq) / (2.f * nyq));
  G.m[1] = vr;
  G.c[1] = lcode(vr, 2.f, 129.f);
  const float vru = (s2.u * ex + s2.v * ey) * ce, vrl = (s1.u * ex + s1.v * ey) * ce;
  const float swv = sqrtf(1.f + sqf(clampf(2.5f * sqrtf(fmaxf(s0.nu, 0.f) / 1000.f), 0.f, 8.f)) + sqf((vru - vrl) / 2.5f) +
                          sqf(0.15f * s0.vt * se) + sqf(swt));
  G.m[2] = fminf(swv, 19.5f);
  G.c[2] = lcode(G.m[2], 2.f, 129.f);
  const float d0 = 3.67f / s0.lr * 1000.f;
  const bool melt = s0.T > 273.15f;
  const float zdrR = clampf(0.2f + 1.15f * (d0 - 0.5f), 0.1f, 4.8f);
  const float zdrS = melt ? 1.3f : 0.3f;
  const float zdrG = melt ? (zg > 3.2e5f ? 0.f : 0.7f) : 0.15f;
  const float zv = zr / db2lin(zdrR) + zs / db2lin(zdrS) + zg / db2lin(zdrG) + zdeb / db2lin(0.2f);
  const float zdr = 10.f * logf(fmaxf(ztot, 1e-9f) / fmaxf(zv, 1e-9f)) / 2.302585f;
  G.m[3] = clampf(zdr, -7.9f, 7.9f);
  G.c[3] = lcode(G.m[3], 16.f, 128.f);
  const float fr = zr / ztot, fs = zs / ztot, fg = zg / ztot, fd = zdeb / ztot;
  float cc = fr * (d0 > 2.5f ? 0.986f : 0.995f) + fs * (melt ? 0.93f : 0.985f) + fg * (melt ? (zg > 3.2e5f ? 0.90f : 0.94f) : 0.985f) +
             fd * 0.55f;
  cc -= 0.24f * fr * fg;
  G.m[4] = clampf(cc, 0.2f, 1.05f);
  G.c[4] = lcode(G.m[4], 300.f, -60.5f);
  G.kdp = powf(0.017f * powf(fmaxf(zr, 0.f), 0.714f) / 44.f, 1.2165f);
  G.m[5] = G.kdp;
  return G;
}

// one thread per gate: x = gate along the radial, y = radial
__global__ void __launch_bounds__(128) k_radar_cut(RadarU R, Grid g, Fields F, int par, const float* __restrict__ tor,
                                                   uint8_t* __restrict__ out, float* __restrict__ kdp, float* __restrict__ mom) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x, ri = blockIdx.y;
  const int ngR = int(R.gates.x), ngD = int(R.gates.y);
  if (gi >= ngR) return;
  const GateOut G = gate(R, g, F, par, tor, ri, gi);
  const uint32_t mask = uint32_t(R.offB.w);
  out[size_t(R.offA.x) * 4 + size_t(ri) * ngR + gi] = uint8_t(G.c[0]);
  if (gi < ngD) {
    const size_t o = size_t(ri) * ngD + gi;
    if (mask & 2u) out[size_t(R.offA.y) * 4 + o] = uint8_t(G.c[1]);
    if (mask & 4u) out[size_t(R.offA.z) * 4 + o] = uint8_t(G.c[2]);
    if (mask & 8u) out[size_t(R.offA.w) * 4 + o] = uint8_t(G.c[3]);
    if (mask & 32u) out[size_t(R.offB.y) * 4 + o] = uint8_t(G.c[4]);
    kdp[o] = G.kdp;
  }
  if (mom) {
    float* mp = mom + (size_t(ri) * ngR + gi) * 6;
#pragma unroll
    for (int c = 0; c < 6; c++) mp[c] = G.m[c];
  }
}

// PhiDP: one warp per 32 radials, 32 x 32 KDP tiles staged through shared memory (radar.js:243-268)
__global__ void __launch_bounds__(128) k_radar_phi(RadarU R, const float* __restrict__ kdp, uint8_t* __restrict__ out) {
  __shared__ float tile[4][32][33];
  __shared__ uint8_t codes[4][32][36];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int r0 = (blockIdx.x * 4 + wid) * 32;
  const int nrad = int(R.cut.w), ng = int(R.gates.y), ngq = (ng / 4) * 4;
  if (r0 >= nrad) return;
  const float gw = R.gates.w;
  float acc = R.nyq.w;
  uint8_t* dst = out + size_t(R.offB.x) * 4;
  for (int g0 = 0; g0 < ngq; g0 += 32) {
    for (int r = 0; r < 32; r++) {
      const int ri = r0 + r;
      tile[wid][r][lane] = (ri < nrad && g0 + lane < ngq) ? __ldg(kdp + size_t(ri) * ng + g0 + lane) : -1.f;
    }
    __syncwarp();
    const int n = min(32, ngq - g0);
    for (int t = 0; t < n; t++) {
      const float kd = tile[wid][lane][t];
      uint8_t c = 0;
      if (kd >= 0.f) {
        acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(__fmul_rn(2.f, kd), gw), 0.001f));
        const float ph = __fsub_rn(acc, __fmul_rn(360.f, floorf(__fdiv_rn(acc, 360.f))));
        c = uint8_t(fminf(fmaxf(rintf(__fadd_rn(__fdiv_rn(__fmul_rn(ph, 253.f), 360.f), 2.f)), 2.f), 255.f));
      }
      codes[wid][lane][t] = c;
    }
    __syncwarp();
    for (int r = 0; r < 32; r++) {
      const int ri = r0 + r;
      if (ri < nrad && lane < n) dst[size_t(ri) * ng + g0 + lane] = codes[wid][r][lane];
    }
    __syncwarp();
  }
}

}  // namespace

void launch_radar_cut(const RadarU& R, const Grid& g, const Fields& F, int par, const float* tor, uint8_t* out, float* kdp,
                      float* mom, cudaStream_t s) {
  const int ngR = int(R.gates.x), nrad = int(R.cut.w);
  k_radar_cut<<<dim3((ngR + 127) / 128, nrad), 128, 0, s>>>(R, g, F, par, tor, out, kdp, mom);
  if (uint32_t(R.offB.w) & 16u) k_radar_phi<<<(nrad + 127) / 128, 128, 0, s>>>(R, kdp, out);
}

}  // namespace ob
