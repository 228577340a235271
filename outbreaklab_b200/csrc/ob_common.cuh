// ob_common.cuh — device-side layout, uniforms and physics helpers of the B200 storm-model step.
//
// Layout in HBM (structure of arrays): every 3-D field is one fp32 array over the staggered texel box
// (nx+1) x (ny+1) x (nz+1), x fastest, rows padded to a pitch that is a multiple of 32 floats (128 B), so that a warp
// reading a row segment issues whole 128-byte lines and every field shares one index i + px*(j + py*k). Cell-centred
// fields (Q, aux, phT) use the same index and leave the i = nx, j = ny, k = nz planes unused. One channel per array
// means a semi-Lagrangian gather of u touches only u bytes (a float4 texel would drag v, w, theta through L1/L2).
//
// The physics formulas restate the reference's WGSL (model.js:41-134, 578-907) in fp32 with IEEE division and
// square root; the hurricane-mode branches (model.js:107-119 and the kernels' hurricane parts) are template flags or
// separate kernels, so the outbreak-mode kernels carry none of their code.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace ob {

// uniform block (model.js:23-37), packed on the host per step (model.js:1391-1425)
struct Uni {
  float4 dims, dzv, step, sponge, turb, micro, misc, cor, ci, pad, micro2, hur, hur2, hur3, hur4, hur5, vtx, vtx2, cn;
  float4 der;  // derived on the host per step: (dt/dx, dt/dz, 1/dx^2, 1/dz^2), so no thread divides uniforms
  float4 der2; // (1/dt, 0, 0, 0), derived on the host per step
  // step.y (the model time of the reference's block) stays 0 here: the kernels read the time from Fields::clock
};

struct Grid {
  int nx, ny, nz;
  int px;        // row pitch in floats (>= nx+1, multiple of 32)
  int py;        // rows per plane (= ny+1)
  int plane;     // px*py
  int pad, nxp, nyp;  // pressure-solve padding and padded extents (model.js:1220-1223)
  __host__ __device__ __forceinline__ int at(int i, int j, int k) const { return i + px * (j + py * k); }
  __host__ __device__ __forceinline__ int pidx(int i, int j, int k) const { return (i + pad) + nxp * ((j + pad) + nyp * k); }
};

// device pointers of one model's state
struct Fields {
  float* V[2][4];   // (u, v, w, theta) ping-pong
  float* Vt[4];     // advection scratch (ADVV1 output)
  float* Vlo[4];    // min and max of the 8 texels around each texel's departure point (ADVV1 output; the limiter
  float* Vhi[4];    // of ADVV2 reads them instead of tracing and gathering the same 8 texels again)
  float* Q[2][8];   // (qv, qc, qi, qr, qs, qg, Nr, spare): slot 0 = state, slot 1 = after advection
  float* Qt[8];     // advection scratch (ADVQ1 output)
  float* aux[2];    // nu_h, nu_v
  float* phT;       // target hydrostatic phi
  float4* lsfA;     // 2-D nx*ny
  float4* lsfB;
  float4* ciMap;
  float4* sfc;
  const float* B;   // base state (nz+1)*8
  float* rhs;       // padded solve grid nxp*nyp*nz
  __nv_bfloat16* rhs_hi;  // tensor-core solve: the right-hand side split into bf16 hi/lo, row pitch rhs_ld
  __nv_bfloat16* rhs_lo;
  int rhs_ld;
  float* phi;
  double* rain;     // nx*ny accumulated surface precipitation
  const float* bnd; // OB_MAX_BOUNDS x 148
  const float* ci;  // events x 12
  unsigned int* flags;  // [0] NaN/Inf counter
  // clear-air skip of the hydrometeor channels, per brick of 32 x 4 x 1 cells (nbx x nby x nz bricks)
  unsigned int* actQ0;   // Q slot 0 holds a hydrometeor or a nonzero spare channel in the brick
  unsigned int* actQt;   // the advection scratch Qt holds one (its block computed them)
  unsigned int* zeroQt;  // the scratch's hydrometeor and spare channels are known to be zero there
  unsigned int* zeroQ1;  // Q slot 1's hydrometeor and spare channels are known to be zero there
  int nbx, nby;
  float fallmax;         // bound on every hydrometeor fall speed of the base state (m/s)
  // sponge coefficients tabulated once per parameter set (k_tables): spz[2k] = top sponge at the cell centre height
  // (k + 1/2) dz, spz[2k+1] at the face height k dz; slx[2i] = lateral sponge of the x distance alone at the face
  // x = i dx, slx[2i+1] at the centre (i + 1/2) dx; sly likewise in y. The lateral sponge of a point is
  // max(slx, sly): it is a non-increasing function of min(x distance, y distance), so the maximum of the two
  // one-dimensional values is the same float as the formula applied to the minimum distance.
  const float* spz;
  const float* slx;
  const float* sly;
  // microphysics surrogate: in record mode mlp_buf holds sampled (state, tendency) pairs (24 floats each, cells
  // drawn with probability mlp_rate), in surrogate mode the queue of cell offsets; mlp_count is the append counter
  float* mlp_buf;
  unsigned* mlp_count;
  unsigned mlp_cap;
  float mlp_rate;
  // model time (s) on the device: read by the passes that move with time (LSF, CI, the record-mode draw) and
  // advanced by the last pass of each step, so a captured step replays unchanged
  double* clock;
  // hurricane mode: the winds the advection carries (WGSL_M_PREP; null outside hurricane mode) and the initial
  // vortex table (nz x nr of (tangential wind, theta', 0, 0); null when there is none)
  float* Vp[4];
  const float4* vx;
};

// ---- hurricane mode (model.js:107-119) ----
__device__ __forceinline__ bool hurOn(const Uni& U) { return U.hur.x > 0.5f; }
// cloud ice settles in hurricane mode (model.js:112)
__device__ __forceinline__ float vtI(const Uni& U, float q, float rho) {
  return (U.hur.x > 0.5f && q > 1e-9f) ? fminf(3.29f * powf(fmaxf(rho * q, 1e-12f), 0.16f), 1.5f) : 0.f;
}
// drag coefficient for the lowest-level wind u1 over sea and land (model.js:115-119)
__device__ __forceinline__ float cdSfc(const Uni& U, float u1, float land) {
  const float f = U.hur2.w;
  const float cs = fminf((0.75f + 0.067f * f * u1) * 1e-3f, U.hur5.x) * f * f;
  const float t = fminf(fmaxf(land, 0.f), 1.f);
  return cs * (1.f - t) + U.hur3.x * t;
}

// ---- grouped launches: one launch of a pass over every member of an ensemble ----
constexpr int kMaxMembers = 48;
constexpr int kMaxLanes = 2;  // concurrent groups of members within one ensemble step
// one member of a grouped launch (held in constant memory by the step kernels)
struct MemberC {
  Grid g;
  Uni U;
  Fields F;
  double* lsfT;  // model time of the member's last LSF pass (device copy of the host's bookkeeping)
  int micro;     // microphysics mode of the step (0 the scheme, 2 the surrogate)
};
constexpr float T0K = 273.15f;
constexpr double CPDd = 1005.7, RVCd = 461.5, LVCd = 2.501e6, LFCd = 3.337e5, LSCd = 2.834e6;

__device__ __forceinline__ int clampi(int x, int a, int b) { return min(max(x, a), b); }
__device__ __forceinline__ float clampf(float x, float a, float b) { return fminf(fmaxf(x, a), b); }
__device__ __forceinline__ float sstep(float a, float b, float x) {
  float t = clampf((x - a) / (b - a), 0.f, 1.f);
  return t * t * (3.f - 2.f * t);
}
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.f - t) + b * t; }

// base state per level: A = (theta0, qv0, rho_c, rho_w bottom), B = (pi0, p0, u0, v0)
__device__ __forceinline__ float4 bsA(const float* B, int nz, int k) {
  return __ldg(reinterpret_cast<const float4*>(B) + clampi(k, 0, nz - 1) * 2);
}
__device__ __forceinline__ float4 bsB(const float* B, int nz, int k) {
  return __ldg(reinterpret_cast<const float4*>(B) + clampi(k, 0, nz - 1) * 2 + 1);
}
__device__ __forceinline__ float rhoW(const float* B, int nz, int k) { return __ldg(B + clampi(k, 0, nz) * 8 + 3); }

// ---- noise.js:4-27 ----
__device__ __forceinline__ uint32_t pcg(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
__device__ __forceinline__ uint32_t hash2i(int x, int y) { return pcg(uint32_t(x) ^ pcg(uint32_t(y) + 0x9e3779b9u)); }
__device__ __forceinline__ uint32_t hash3i(int x, int y, int z) {
  return pcg(uint32_t(x) ^ pcg(uint32_t(y) ^ pcg(uint32_t(z) + 0x7f4a7c15u)));
}
__device__ __forceinline__ float rnd3(int x, int y, int z) { return float(hash3i(x, y, z) >> 8u) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float fadef(float t) { return t * t * t * (t * (t * 6.f - 15.f) + 10.f); }
__device__ __forceinline__ float gdot(int ix, int iy, float fx, float fy) {
  float a = float(hash2i(ix, iy) >> 8u) * (6.2831853f / 16777216.0f);
  return cosf(a) * fx + sinf(a) * fy;
}
__device__ __forceinline__ float gnoise2(float px, float py) {
  float fx0 = floorf(px), fy0 = floorf(py);
  int ix = int(fx0), iy = int(fy0);
  float fx = px - fx0, fy = py - fy0;
  float ux = fadef(fx), uy = fadef(fy);
  float a = gdot(ix, iy, fx, fy), b = gdot(ix + 1, iy, fx - 1.f, fy);
  float c = gdot(ix, iy + 1, fx, fy - 1.f), d = gdot(ix + 1, iy + 1, fx - 1.f, fy - 1.f);
  return mixf(mixf(a, b, ux), mixf(c, d, ux), uy) * 1.4142f;
}
__device__ __forceinline__ float fbm2(float px, float py, int oct) {
  float a = 0.5f, s = 0.f;
  for (int i = 0; i < oct; i++) {
    s += a * gnoise2(px, py);
    float nx = 1.6f * px - 1.2f * py + 17.1f, ny = 1.2f * px + 1.6f * py + 3.7f;
    px = nx;
    py = ny;
    a *= 0.5f;
  }
  return s;
}

// ---- saturation and fall speeds (model.js:59-101) ----
__device__ __forceinline__ float esl(float T) { return 611.2f * expf(17.67f * (T - T0K) / (T - 29.65f)); }
__device__ __forceinline__ float esi(float T) { return 611.2f * expf(21.8745584f * (T - 273.16f) / (T - 7.66f)); }
__device__ __forceinline__ float fIce(float T) { return clampf((T0K - T) / 40.f, 0.f, 1.f); }
__device__ __forceinline__ float qvsat(float T, float p, float f) {
  float e = mixf(esl(T), esi(T), f);
  return 0.622f * e / fmaxf(p - e, 100.f);
}
// qvsat with one exponential where the ice fraction is exactly 0 or 1: mix(a, b, 0) == a and mix(a, b, 1) == b for
// finite a, b, so the result is bit-identical to qvsat
__device__ __forceinline__ float qvsat1(float T, float p, float f) {
  float e;
  if (f == 0.f) e = esl(T);
  else if (f == 1.f) e = esi(T);
  else e = mixf(esl(T), esi(T), f);
  return 0.622f * e / fmaxf(p - e, 100.f);
}
struct Fall {
  float rsfc;   // surface density (step.z)
  bool thm;     // Thompson-style scheme
  bool mar = false;  // maritime graupel (hurricane mode, Lin scheme: model.js:87-92)
  __device__ __forceinline__ float vtR(float q, float rho) const {
    float f = sqrtf(rsfc / rho);
    return fminf(36.34f * powf(fmaxf(0.001f * rho * q, 0.f), 0.1364f) * f, 10.f * f);
  }
  __device__ __forceinline__ float vtS(float q, float rho) const {
    return clampf(1.1f * powf(fmaxf(1000.f * rho * q, 1e-6f), 0.11f), 0.3f, 2.2f) * sqrtf(rsfc / rho);
  }
  __device__ __forceinline__ float vtG(float q, float rho) const {
    float v = clampf(9.f * powf(fmaxf(1000.f * rho * q, 1e-6f), 0.42f), 1.f, 55.f) * sqrtf(rsfc / rho);
    float r = q / 0.009f;
    return fminf(v * (1.f + r * r), 65.f);
  }
  static __device__ __forceinline__ float lamR(float q, float n) {
    return clampf(powf(float(3.14159 * 1000.0) * fmaxf(n, 1e-3f) / fmaxf(q, 1e-12f), 0.33333f), 1000.f, 1.0e5f);
  }
  static __device__ __forceinline__ float n0G(float q, float rho) { return clampf(200.f / fmaxf(rho * q, 1e-9f), 1e4f, 3e6f); }
  static __device__ __forceinline__ float lamG(float q, float rho) {
    return powf(float(3.14159 * 500.0) * n0G(q, rho) / fmaxf(rho * q, 1e-12f), 0.25f);
  }
  __device__ __forceinline__ float vtGT(float q, float rho) const {
    return fminf(1503.f * powf(lamG(q, rho), -0.89f), 25.f) * sqrtf(rsfc / rho);
  }
  // rain fall speed (mass-weighted, number-weighted)
  __device__ __forceinline__ float2 vtRain(float qr, float nr, float rho) const {
    if (thm) {
      float l = powf(lamR(qr, nr), -0.8f), s = sqrtf(rsfc / rho);
      return make_float2(fminf(2503.f * l, 10.f) * s, fminf(784.f * l, 10.f) * s);
    }
    float v = vtR(qr, rho);
    return make_float2(v, v);
  }
  __device__ __forceinline__ float vtGM(float q, float rho) const {
    return clampf(5.f * powf(fmaxf(1000.f * rho * q, 1e-6f), 0.25f), 1.f, 9.f) * sqrtf(rsfc / rho);
  }
  __device__ __forceinline__ float vtGrau(float qg, float rho) const {
    if (mar) return vtGM(qg, rho);
    return thm ? vtGT(qg, rho) : vtG(qg, rho);
  }
  // equivalent reflectivity (mm^6/m^3), model.js:103-116
  __device__ __forceinline__ float zRain(float qr, float nr, float rho) const {
    if (!thm) return 3.63e9f * powf(fmaxf(rho * qr, 0.f), 1.75f);
    if (qr < 1e-9f) return 0.f;
    float l = lamR(qr, nr);
    float nb = qr * l * l * l / 3141.59f;
    return 720e18f * rho * nb / (l * l * l * l * l * l);
  }
  __device__ __forceinline__ float zGrau(float qg, float rho, float T) const {
    if (mar) return (T < T0K ? 1.3e9f : 1.0e10f) * powf(fmaxf(rho * qg, 0.f), 1.75f);
    if (!thm) return (T < T0K ? 1.2e10f : 4.33e10f) * powf(fmaxf(rho * qg, 0.f), 1.75f);
    if (qg < 1e-9f) return 0.f;
    float l = lamG(qg, rho), l2 = l * l;
    return 720e18f * n0G(qg, rho) / (l2 * l2 * l2 * l) * (T < T0K ? 0.0666f : 0.24f);
  }
};

// linear filter with clamp-to-edge on an (X, Y, Z) box stored at pitch (px, py); x, y, z in texel units
__device__ __forceinline__ float trilerp(const float* __restrict__ f, const Grid& g, int X, int Y, int Z, float x, float y, float z) {
  float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  int i0 = int(fx), j0 = int(fy), k0 = int(fz);
  float ax = x - fx, ay = y - fy, az = z - fz;
  int i1 = clampi(i0 + 1, 0, X - 1), j1 = clampi(j0 + 1, 0, Y - 1), k1 = clampi(k0 + 1, 0, Z - 1);
  i0 = clampi(i0, 0, X - 1);
  j0 = clampi(j0, 0, Y - 1);
  k0 = clampi(k0, 0, Z - 1);
  const int r00 = g.px * (j0 + g.py * k0), r10 = g.px * (j1 + g.py * k0), r01 = g.px * (j0 + g.py * k1), r11 = g.px * (j1 + g.py * k1);
  float c00 = __ldg(f + r00 + i0) * (1.f - ax) + __ldg(f + r00 + i1) * ax;
  float c10 = __ldg(f + r10 + i0) * (1.f - ax) + __ldg(f + r10 + i1) * ax;
  float c01 = __ldg(f + r01 + i0) * (1.f - ax) + __ldg(f + r01 + i1) * ax;
  float c11 = __ldg(f + r11 + i0) * (1.f - ax) + __ldg(f + r11 + i1) * ax;
  float c0 = c00 * (1.f - ay) + c10 * ay;
  float c1 = c01 * (1.f - ay) + c11 * ay;
  return c0 * (1.f - az) + c1 * az;
}

// the same filter where the trace is already clamped to the box, so that the floor index of every axis lies in
// [-1, extent - 1]: then max(i0, 0) and min(i0 + 1, extent - 1) are the clamped corners (same texels, fewer bounds)
// the same sample, and the min / max of its 8 texels (the MacCormack limiter's window at that point)
__device__ __forceinline__ float trilerpB_mm(const float* __restrict__ f, const Grid& g, int X, int Y, int Z, float x, float y, float z,
                                             float& lo, float& hi) {
  const int i0 = __float2int_rd(x), j0 = __float2int_rd(y), k0 = __float2int_rd(z);
  const float ax = x - float(i0), ay = y - float(j0), az = z - float(k0);
  const int ia = max(i0, 0), ib = min(i0 + 1, X - 1);
  const int ja = max(j0, 0), jb = min(j0 + 1, Y - 1);
  const int ka = max(k0, 0), kb = min(k0 + 1, Z - 1);
  const int r00 = g.px * (ja + g.py * ka), r10 = g.px * (jb + g.py * ka), r01 = g.px * (ja + g.py * kb), r11 = g.px * (jb + g.py * kb);
  const float a = __ldg(f + r00 + ia), b = __ldg(f + r00 + ib), c = __ldg(f + r10 + ia), d = __ldg(f + r10 + ib);
  const float e = __ldg(f + r01 + ia), h = __ldg(f + r01 + ib), k = __ldg(f + r11 + ia), l = __ldg(f + r11 + ib);
  lo = fminf(fminf(fminf(a, b), fminf(c, d)), fminf(fminf(e, h), fminf(k, l)));
  hi = fmaxf(fmaxf(fmaxf(a, b), fmaxf(c, d)), fmaxf(fmaxf(e, h), fmaxf(k, l)));
  const float c00 = a * (1.f - ax) + b * ax;
  const float c10 = c * (1.f - ax) + d * ax;
  const float c01 = e * (1.f - ax) + h * ax;
  const float c11 = k * (1.f - ax) + l * ax;
  const float c0 = c00 * (1.f - ay) + c10 * ay;
  const float c1 = c01 * (1.f - ay) + c11 * ay;
  return c0 * (1.f - az) + c1 * az;
}
__device__ __forceinline__ float trilerpB(const float* __restrict__ f, const Grid& g, int X, int Y, int Z, float x, float y, float z) {
  const int i0 = __float2int_rd(x), j0 = __float2int_rd(y), k0 = __float2int_rd(z);
  const float ax = x - float(i0), ay = y - float(j0), az = z - float(k0);
  const int ia = max(i0, 0), ib = min(i0 + 1, X - 1);
  const int ja = max(j0, 0), jb = min(j0 + 1, Y - 1);
  const int ka = max(k0, 0), kb = min(k0 + 1, Z - 1);
  const int r00 = g.px * (ja + g.py * ka), r10 = g.px * (jb + g.py * ka), r01 = g.px * (ja + g.py * kb), r11 = g.px * (jb + g.py * kb);
  float c00 = __ldg(f + r00 + ia) * (1.f - ax) + __ldg(f + r00 + ib) * ax;
  float c10 = __ldg(f + r10 + ia) * (1.f - ax) + __ldg(f + r10 + ib) * ax;
  float c01 = __ldg(f + r01 + ia) * (1.f - ax) + __ldg(f + r01 + ib) * ax;
  float c11 = __ldg(f + r11 + ia) * (1.f - ax) + __ldg(f + r11 + ib) * ax;
  float c0 = c00 * (1.f - ay) + c10 * ay;
  float c1 = c01 * (1.f - ay) + c11 * ay;
  return c0 * (1.f - az) + c1 * az;
}

}  // namespace ob
