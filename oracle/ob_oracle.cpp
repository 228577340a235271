// ob_oracle.cpp — TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// CPU restatement of OutbreakLab's storm-model time step (Julianfinnerty/outbreakLab), written from the reference's
// WGSL kernels and host classes. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
// Templated on the arithmetic type: the float instantiation is the parity oracle and the timed CPU baseline, the
// double instantiation is the FP64 error reference of every reported number.
//
// PARITY UNPINNED: the reference ships no tests, golden vectors or fixtures, and its WGSL runs only on a browser
// WebGPU device, which this machine does not have (no node, no graphics stack). The restatement is therefore pinned
// only by known-answer tests from the mathematics (DST orthonormality and eigen-identity, exact tridiagonal solves,
// pcg hash arithmetic, the Level II code table of l2writer.py, hydrostatic base state).
//
// Sampler convention (model.js:1167, 411-418, 485): WebGPU linear filtering, clamp-to-edge, texel centres at
// (i + 1/2)/N in normalised coordinates. This restatement works in texel units directly and uses exact linear
// weights; the hardware's low-precision fixed-point filter weights are not reproduced.
//
// Outbreak mode and hurricane mode (setSurface with a hurricane, model.js:1290-1365, 1402-1420): the hurricane branches
// (model.js:107-119, 308-336, 377-386, 424-433, 494-499, 640-690, 713-774, 893-896, 948-1026) are restated too
// are not restated.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../include/ob.h"

namespace oro {

static inline int clampi(int x, int a, int b) { return x < a ? a : (x > b ? b : x); }
template <class R> static inline R clampv(R x, R a, R b) { return std::min(std::max(x, a), b); }
template <class R> static inline R sstep(R a, R b, R x) {  // model.js:42
  R t = clampv((x - a) / (b - a), R(0), R(1));
  return t * t * (R(3) - R(2) * t);
}
template <class R> static inline R mixv(R a, R b, R t) { return a * (R(1) - t) + b * t; }
template <class R> static inline R fractv(R x) { return x - std::floor(x); }

// ---- noise.js:4-27 ----
static inline uint32_t pcg(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
static inline uint32_t hash2i(int x, int y) { return pcg(uint32_t(x) ^ pcg(uint32_t(y) + 0x9e3779b9u)); }
static inline uint32_t hash3i(int x, int y, int z) {
  return pcg(uint32_t(x) ^ pcg(uint32_t(y) ^ pcg(uint32_t(z) + 0x7f4a7c15u)));
}
template <class R> static inline R rnd3(int x, int y, int z) { return R(hash3i(x, y, z) >> 8u) * R(1.0 / 16777216.0); }
template <class R> static inline void grad2(int x, int y, R& gx, R& gy) {
  R a = R(hash2i(x, y) >> 8u) * R(6.2831853 / 16777216.0);
  gx = std::cos(a);
  gy = std::sin(a);
}
template <class R> static inline R fade(R t) { return t * t * t * (t * (t * R(6) - R(15)) + R(10)); }
template <class R> static R gnoise2(R px, R py) {  // noise.js:18-24
  R fx0 = std::floor(px), fy0 = std::floor(py);
  int ix = int(fx0), iy = int(fy0);
  R fx = px - fx0, fy = py - fy0;
  R ux = fade(fx), uy = fade(fy);
  R gx, gy;
  grad2<R>(ix, iy, gx, gy);
  R a = gx * fx + gy * fy;
  grad2<R>(ix + 1, iy, gx, gy);
  R b = gx * (fx - R(1)) + gy * fy;
  grad2<R>(ix, iy + 1, gx, gy);
  R c = gx * fx + gy * (fy - R(1));
  grad2<R>(ix + 1, iy + 1, gx, gy);
  R d = gx * (fx - R(1)) + gy * (fy - R(1));
  return mixv(mixv(a, b, ux), mixv(c, d, ux), uy) * R(1.4142);
}
template <class R> static R fbm2(R px, R py, int oct) {  // noise.js:25-29
  R a = R(0.5), s = R(0);
  for (int i = 0; i < oct; i++) {
    s += a * gnoise2(px, py);
    R nx = R(1.6) * px + R(-1.2) * py + R(17.1);
    R ny = R(1.2) * px + R(1.6) * py + R(3.7);
    px = nx;
    py = ny;
    a *= R(0.5);
  }
  return s;
}

template <class R> struct V4 {
  R x, y, z, w;
};
// uniform block MU (model.js:23-37, packed by writeUniforms model.js:1391-1425)
template <class R> struct MU {
  V4<R> dims, dzv, step, sponge, turb, micro, misc, cor, ci, pad, micro2, hur, hur2, hur3, hur4, hur5, vtx, vtx2, cn;
};

// constants of model.js:58
static const double T0K = 273.15, CPD = 1005.7, RVC = 461.5, LVC = 2.501e6, LFC = 3.337e5, LSC = 2.834e6;

// ---------------------------------------------------------------------------------------------------------------
// Pressure solver (solver.js:105-165)
// ---------------------------------------------------------------------------------------------------------------
template <class R> struct Poisson {
  int nx = 0, ny = 0, nz = 0;
  double dx = 0, dz = 0;
  std::vector<R> qix, qx, qiy, qy, lam;  // qi[l*N+i] = v_l(i); q[i*N+l] = v_l(i)  (solver.js:115-125)
  std::vector<R> zop;                      // (lo, up, diag, rhoC) per level (solver.js:139-146)
  std::vector<R> tmp, hat;

  void init(int nx_, int ny_, int nz_, double dx_, double dz_) {
    nx = nx_; ny = ny_; nz = nz_; dx = dx_; dz = dz_;
    auto dst = [](int N, std::vector<R>& q, std::vector<R>& qi) {
      q.assign(size_t(N) * N, R(0));
      qi.assign(size_t(N) * N, R(0));
      for (int i = 0; i < N; i++)
        for (int l = 0; l < N; l++) {
          double c = std::sqrt((l == N - 1 ? 1.0 : 2.0) / N);
          double v = c * std::sin(M_PI * (l + 1) * (i + 0.5) / N);
          q[size_t(i) * N + l] = R(v);
          qi[size_t(l) * N + i] = R(v);
        }
    };
    dst(nx, qx, qix);
    dst(ny, qy, qiy);
    lam.resize(nx + ny);
    for (int l = 0; l < nx; l++) lam[l] = R(-4.0 / (dx * dx) * std::pow(std::sin(M_PI * (l + 1) / (2.0 * nx)), 2));
    for (int m = 0; m < ny; m++) lam[nx + m] = R(-4.0 / (dx * dx) * std::pow(std::sin(M_PI * (m + 1) / (2.0 * ny)), 2));
    std::vector<double> rc(nz, 1.0), rw(nz + 1, 1.0);
    set_density(rc.data(), rw.data());
    tmp.assign(size_t(nx) * ny * nz, R(0));
    hat.assign(size_t(nx) * ny * nz, R(0));
  }
  void set_density(const double* rhoC, const double* rhoW) {  // solver.js:139-146
    zop.assign(size_t(nz) * 4, R(0));
    double a = 1.0 / (dz * dz);
    for (int k = 0; k < nz; k++) {
      double lo = k > 0 ? rhoW[k] * a : 0, up = k < nz - 1 ? rhoW[k + 1] * a : 0;
      zop[k * 4 + 0] = R(lo);
      zop[k * 4 + 1] = R(up);
      zop[k * 4 + 2] = R(-(lo + up));
      zop[k * 4 + 3] = R(rhoC[k]);
    }
  }
  // mode 0 (solver.js:13-22): dst(l, col) = sum_i M(l, i) src(i, col), col = j + ny k
  void gemm_x(const std::vector<R>& M, const R* src, R* dst) const {
    const long cols = long(ny) * nz;
#pragma omp parallel for schedule(static)
    for (long col = 0; col < cols; col++) {
      const R* s = src + col * nx;
      R* d = dst + col * nx;
      for (int l = 0; l < nx; l++) {
        const R* m = &M[size_t(l) * nx];
        R acc = R(0);
        for (int i = 0; i < nx; i++) acc += m[i] * s[i];
        d[l] = acc;
      }
    }
  }
  // mode 1: per z-plane dst(i, m, k) = sum_j src(i, j, k) M(m, j)
  void gemm_y(const std::vector<R>& M, const R* src, R* dst) const {
#pragma omp parallel for schedule(static)
    for (long km = 0; km < long(nz) * ny; km++) {
      int k = int(km / ny), m = int(km % ny);
      const R* mrow = &M[size_t(m) * ny];
      R* d = dst + (size_t(k) * ny + m) * nx;
      for (int i = 0; i < nx; i++) d[i] = R(0);
      for (int j = 0; j < ny; j++) {
        const R* s = src + (size_t(k) * ny + j) * nx;
        R w = mrow[j];
        for (int i = 0; i < nx; i++) d[i] += s[i] * w;
      }
    }
  }
  void tri(R* h) const {  // solver.js:70-103
    const long sxy = long(nx) * ny;
#pragma omp parallel for schedule(static)
    for (long base = 0; base < sxy; base++) {
      int l = int(base % nx), m = int(base / nx);
      R shift = lam[l] + lam[nx + m];
      std::vector<R> cp(nz);
      R cprev = R(0), dprev = R(0);
      for (int k = 0; k < nz; k++) {
        const R* o = &zop[k * 4];
        long idx = base + sxy * k;
        R den = o[2] + shift * o[3] - o[0] * cprev;
        cprev = o[1] / den;
        dprev = (h[idx] - o[0] * dprev) / den;
        cp[k] = cprev;
        h[idx] = dprev;
      }
      R above = h[base + sxy * (nz - 1)];
      for (int k = nz - 2; k >= 0; k--) {
        long idx = base + sxy * k;
        above = h[idx] - cp[k] * above;
        h[idx] = above;
      }
    }
  }
  void solve(const R* rhs, R* phi) {  // solver.js:155-163
    gemm_x(qix, rhs, tmp.data());
    gemm_y(qiy, tmp.data(), hat.data());
    tri(hat.data());
    gemm_y(qy, hat.data(), tmp.data());
    gemm_x(qx, tmp.data(), phi);
  }
};

// ---------------------------------------------------------------------------------------------------------------
// RegionalModel (model.js:1156-1496) with its WGSL kernels
// ---------------------------------------------------------------------------------------------------------------
template <class R> struct Model {
  int nx = 0, ny = 0, nz = 0, pad = 0, nxp = 0, nyp = 0;
  double dx = 0, dz = 0, Lx = 0, Ly = 0;
  ObParams P{};
  MU<R> S{};
  std::vector<R> B;  // base state, (nz+1)*8 (sounding.js:139-142)
  // textures: V* are (nx+1)(ny+1)(nz+1) x 4; Q* nx ny nz x 4; aux x 2; phT x 1; 2-D maps nx ny x 4
  std::vector<R> V[2], Vt, Q1[2], Q2[2], Q1t, Q2t, aux, phT, lsfA, lsfB, ciMap, sfc, phi, rhs;
  std::vector<float> bnd, ciev;
  int nb = 0, nci = 0;
  Poisson<R> solver;
  double time = 0, lsfT = 0;
  int steps = 0, parity = 0;
  double rhoSfc = 1.15;
  std::vector<double> rain;
  // hurricane mode (model.js:1290-1365, 1402-1420)
  bool hur_on = false;
  ObHurricane H{};
  std::vector<R> Vp;   // the winds the advection carries (WGSL_M_PREP)
  std::vector<R> vx;   // vortex table, nz x nr x (tangential wind, theta')
  int vx_nr = 0;
  double vx_x = 0, vx_y = 0, vx_dr = 1, vx_moistR = 1, vx_moistRH = 0;
  bool vortex = false;
  double phiScale = 1;
  bool cnNow = false, filtNow = false;
  const std::vector<R>* trajV = nullptr;  // the winds the midpoint trajectories sample

  int VX() const { return nx + 1; }
  int VY() const { return ny + 1; }
  int VZ() const { return nz + 1; }
  size_t vidx(int i, int j, int k) const { return (size_t(k) * VY() + j) * VX() + i; }
  size_t qidx(int i, int j, int k) const { return (size_t(k) * ny + j) * nx + i; }
  int pidx(int x, int y, int z) const { return (x + pad) + nyp_stride() * ((y + pad) + nyp * z); }
  int nyp_stride() const { return nxp; }

  void create(int nx_, int ny_, int nz_, double dx_) {  // model.js:1202-1237
    nx = nx_; ny = ny_; nz = nz_; dx = dx_; dz = 20000.0 / nz;
    Lx = nx * dx; Ly = ny * dx;
    ob_params_default(&P);
    P.spongeW = float(std::min(std::max(0.08 * std::min(Lx, Ly), 5000.0), 40000.0));
    size_t nv = size_t(VX()) * VY() * VZ() * 4, nq = size_t(nx) * ny * nz * 4, n2 = size_t(nx) * ny * 4;
    for (int p = 0; p < 2; p++) {
      V[p].assign(nv, R(0));
      Q1[p].assign(nq, R(0));
      Q2[p].assign(nq, R(0));
    }
    Vt.assign(nv, R(0));
    Q1t.assign(nq, R(0));
    Q2t.assign(nq, R(0));
    aux.assign(size_t(nx) * ny * nz * 2, R(0));
    phT.assign(size_t(nx) * ny * nz, R(0));
    lsfA.assign(n2, R(0));
    lsfB.assign(n2, R(0));
    ciMap.assign(n2, R(0));
    sfc.assign(n2, R(0));
    pad = ob_grid_pad(float(dx));
    nxp = nx + 2 * pad;
    nyp = ny + 2 * pad;
    phi.assign(size_t(nxp) * nyp * nz, R(0));
    rhs.assign(size_t(nxp) * nyp * nz, R(0));
    solver.init(nxp, nyp, nz, dx, dz);
    B.assign(size_t(nz + 1) * 8, R(0));
    for (int k = 0; k <= nz; k++) {  // a neutral placeholder until a base state is set
      B[k * 8 + 0] = R(300); B[k * 8 + 2] = R(1); B[k * 8 + 3] = R(1); B[k * 8 + 4] = R(1); B[k * 8 + 5] = R(1e5);
    }
    bnd.assign(size_t(OB_MAX_BOUNDS) * OB_BOUNDARY_FLOATS, 0.f);
    ciev.assign(OB_CI_FLOATS, 0.f);
    rain.assign(size_t(nx) * ny, 0.0);
  }
  void set_base_state(const float* Bf) {  // model.js:1276-1288
    for (size_t i = 0; i < B.size(); i++) B[i] = R(Bf[i]);
    rhoSfc = Bf[2];
    std::vector<double> rc(nz), rw(nz + 1);
    for (int k = 0; k < nz; k++) rc[k] = Bf[k * 8 + 2];
    for (int k = 0; k <= nz; k++) rw[k] = Bf[k * 8 + 3];
    solver.set_density(rc.data(), rw.data());
  }

  // ---- uniforms (model.js:1391-1425), outbreak mode ----
  void write_uniforms(double dt) {
    const double DEG = M_PI / 180.0;
    auto v4 = [](double a, double b, double c, double d) { return V4<R>{R(float(a)), R(float(b)), R(float(c)), R(float(d))}; };
    S.dims = v4(nx, ny, nz, dx);
    S.step = v4(dt, time, rhoSfc, 9.81);
    S.sponge = v4(P.spongeW, P.spongeTau, P.dampZ, P.dampTau);
    S.turb = v4(P.cs, P.nu0, P.evap, P.drag != 0 ? 1 : 0);
    double cd = std::pow(0.41 / std::log(0.5 * dz / P.z0 + 1), 2);
    S.micro = v4(P.autoc, P.qc0, P.freeze, cd);
    S.misc = v4(P.vcap, P.mc, P.noise, P.ciRate);
    S.cor = v4(2 * 7.292e-5 * std::sin(P.lat * DEG), P.nudgeTau, nb, P.moistMix);
    S.ci = v4(nci, 0, 0, 0);
    S.micro2 = v4(0, P.sortQ, P.scheme > 0.5f ? 1 : 0, P.evapT);
    if (hur_on) {
      S.hur = v4(1, H.ck, H.landMoist, H.sfcP);
      S.hur2 = v4(H.tauRad, H.radCap, H.blDepth, H.u10f);
      S.hur3 = v4(std::pow(0.41 / std::log(0.5 * dz / 0.3 + 1), 2), H.gust, double(H.thermals) * double(H.thermalScale), H.maritime > 0.5f ? 1 : 0);
      filtNow = steps % 4 == 3 && H.filter4 > 0;
      S.hur5 = v4(H.cdCap, H.dissHeat > 0.5f ? 1 : 0, 4 * double(H.filter4), 0);
      S.hur4 = v4(H.centreX, H.centreY, H.thermalR, H.envR);
    } else {
      S.hur = v4(0, 0, 0, 0);
      S.hur2 = v4(1, 0, 1, 0.8);
      S.hur3 = v4(0, 1, 0, 0);
      S.hur4 = v4(0, 0, 1, 1e9);
      S.hur5 = v4(2.4e-3, 0, 0, 0);
      filtNow = false;
    }
    // off-centred trajectory-averaged pressure force, not on the first step after a reset (model.js:1413-1417)
    const bool cn = hur_on && steps > 0 && H.cnOld > 0;
    cnNow = cn;
    S.cn = v4(cn ? H.cnOld : 0, phiScale, cn ? 1 / (1 - double(H.cnOld)) : 1, hur_on && H.traj2 > 0.5f ? 1 : 0);
    if (vortex) {
      S.vtx = v4(vx_x, vx_y, vx_dr, vx_nr);
      S.vtx2 = v4(vx_moistR, vx_moistRH, 1, 0);
    } else {
      S.vtx = v4(0, 0, 1, 0);
      S.vtx2 = v4(1, 0, 0, 0);
    }
    S.pad = v4(pad, nxp, nyp, 0);
    S.dzv = v4(dz, 1 / dx, 1 / dz, P.mcFloor);
    // the uniforms are f32 on the GPU; in the FP64 instantiation they are those same f32 values widened, except
    // the grid spacings, which are exact in both
  }

  // ---- shared WGSL helpers (model.js:41-134) ----
  R DXS() const { return S.dims.w; }
  R DZS() const { return S.dzv.x; }
  R DTS() const { return S.step.x; }
  const R* bsA(int k) const { return &B[size_t(clampi(k, 0, nz - 1)) * 8]; }
  const R* bsB(int k) const { return &B[size_t(clampi(k, 0, nz - 1)) * 8 + 4]; }
  R rhoW(int k) const { return B[size_t(clampi(k, 0, nz)) * 8 + 3]; }
  bool thompson() const { return S.micro2.z > R(0.5); }
  static R esl(R T) { return R(611.2) * std::exp(R(17.67) * (T - R(T0K)) / (T - R(29.65))); }
  static R esi(R T) { return R(611.2) * std::exp(R(21.8745584) * (T - R(273.16)) / (T - R(7.66))); }
  static R fIce(R T) { return clampv((R(T0K) - T) / R(40), R(0), R(1)); }
  static R qvsat(R T, R p, R f) {
    R e = mixv(esl(T), esi(T), f);
    return R(0.622) * e / std::max(p - e, R(100));
  }
  R vtR(R q, R rho) const {
    R f = std::sqrt(S.step.z / rho);
    return std::min(R(36.34) * std::pow(std::max(R(0.001) * rho * q, R(0)), R(0.1364)) * f, R(10) * f);
  }
  R vtS(R q, R rho) const {
    return clampv(R(1.1) * std::pow(std::max(R(1000) * rho * q, R(1e-6)), R(0.11)), R(0.3), R(2.2)) * std::sqrt(S.step.z / rho);
  }
  R vtG(R q, R rho) const {
    R v = clampv(R(9) * std::pow(std::max(R(1000) * rho * q, R(1e-6)), R(0.42)), R(1), R(55)) * std::sqrt(S.step.z / rho);
    R r = q / R(0.009);
    return std::min(v * (R(1) + r * r), R(65));
  }
  static R lamR(R q, R n) {
    return clampv(std::pow(R(3.14159 * 1000.0) * std::max(n, R(1e-3)) / std::max(q, R(1e-12)), R(0.33333)), R(1000), R(1.0e5));
  }
  void vtRT(R q, R n, R rho, R& vm, R& vn) const {
    R l = std::pow(lamR(q, n), R(-0.8));
    R s = std::sqrt(S.step.z / rho);
    vm = std::min(R(2503) * l, R(10)) * s;
    vn = std::min(R(784) * l, R(10)) * s;
  }
  static R n0G(R q, R rho) { return clampv(R(200) / std::max(rho * q, R(1e-9)), R(1e4), R(3e6)); }
  static R lamG(R q, R rho) { return std::pow(R(3.14159 * 500.0) * n0G(q, rho) / std::max(rho * q, R(1e-12)), R(0.25)); }
  R vtGT(R q, R rho) const { return std::min(R(1503) * std::pow(lamG(q, rho), R(-0.89)), R(25)) * std::sqrt(S.step.z / rho); }
  void vtRain(R qr, R nr, R rho, R& vm, R& vn) const {
    if (thompson()) { vtRT(qr, nr, rho, vm, vn); return; }
    vm = vn = vtR(qr, rho);
  }
  bool hurOn() const { return S.hur.x > R(0.5); }
  bool maritime() const { return S.hur3.w > R(0.5) && !thompson(); }  // model.js:90
  R vtGM(R q, R rho) const {  // model.js:91
    return clampv(R(5) * std::pow(std::max(R(1000) * rho * q, R(1e-6)), R(0.25)), R(1), R(9)) * std::sqrt(S.step.z / rho);
  }
  R vtGrau(R qg, R rho) const {
    if (maritime()) return vtGM(qg, rho);
    return thompson() ? vtGT(qg, rho) : vtG(qg, rho);
  }
  R vtI(R q, R rho) const {  // model.js:112: cloud ice settles in hurricane mode
    return (hurOn() && q > R(1e-9)) ? std::min(R(3.29) * std::pow(std::max(rho * q, R(1e-12)), R(0.16)), R(1.5)) : R(0);
  }
  R cdSfc(R u1, R land) const {  // model.js:115-119
    R f = S.hur2.w;
    R cs = std::min((R(0.75) + R(0.067) * f * u1) * R(1e-3), S.hur5.x) * f * f;
    return mixv(cs, S.hur3.x, clampv(land, R(0), R(1)));
  }
  R zRain(R qr, R nr, R rho) const {
    if (!thompson()) return R(3.63e9) * std::pow(std::max(rho * qr, R(0)), R(1.75));
    if (qr < R(1e-9)) return R(0);
    R l = lamR(qr, nr);
    R nb_ = qr * l * l * l / R(3141.59);
    return R(720e18) * rho * nb_ / (l * l * l * l * l * l);
  }
  R zGrau(R qg, R rho, R T) const {
    if (maritime()) return (T < R(T0K) ? R(1.3e9) : R(1.0e10)) * std::pow(std::max(rho * qg, R(0)), R(1.75));
    if (!thompson()) return (T < R(T0K) ? R(1.2e10) : R(4.33e10)) * std::pow(std::max(rho * qg, R(0)), R(1.75));
    if (qg < R(1e-9)) return R(0);
    R l = lamG(qg, rho), l2 = l * l;
    return R(720e18) * n0G(qg, rho) / (l2 * l2 * l2 * l) * (T < R(T0K) ? R(0.0666) : R(0.24));
  }

  // texel loads with the clamps of the kernels
  const R* ldV(const std::vector<R>& t, int i, int j, int k) const {
    return &t[vidx(clampi(i, 0, nx), clampi(j, 0, ny), clampi(k, 0, nz)) * 4];
  }
  const R* ldQ(const std::vector<R>& t, int i, int j, int k) const {
    return &t[qidx(clampi(i, 0, nx - 1), clampi(j, 0, ny - 1), clampi(k, 0, nz - 1)) * 4];
  }
  const R* l2(const std::vector<R>& t, int i, int j) const {
    return &t[(size_t(clampi(j, 0, ny - 1)) * nx + clampi(i, 0, nx - 1)) * 4];
  }
  // linear sampler, clamp-to-edge, coordinates in texel units (texel i centred at x = i)
  R sampleV(const std::vector<R>& t, R x, R y, R z, int ch) const { return sample(t, VX(), VY(), VZ(), x, y, z, ch); }
  R sampleQ(const std::vector<R>& t, R x, R y, R z, int ch) const { return sample(t, nx, ny, nz, x, y, z, ch); }
  R sample(const std::vector<R>& t, int X, int Y, int Z, R x, R y, R z, int ch, int nch = 4) const {
    R fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    int i0 = int(fx), j0 = int(fy), k0 = int(fz);
    R ax = x - fx, ay = y - fy, az = z - fz;
    int i1 = clampi(i0 + 1, 0, X - 1), j1 = clampi(j0 + 1, 0, Y - 1), k1 = clampi(k0 + 1, 0, Z - 1);
    i0 = clampi(i0, 0, X - 1); j0 = clampi(j0, 0, Y - 1); k0 = clampi(k0, 0, Z - 1);
    auto at = [&](int i, int j, int k) { return t[((size_t(k) * Y + j) * X + i) * nch + ch]; };
    R c00 = at(i0, j0, k0) * (R(1) - ax) + at(i1, j0, k0) * ax;
    R c10 = at(i0, j1, k0) * (R(1) - ax) + at(i1, j1, k0) * ax;
    R c01 = at(i0, j0, k1) * (R(1) - ax) + at(i1, j0, k1) * ax;
    R c11 = at(i0, j1, k1) * (R(1) - ax) + at(i1, j1, k1) * ax;
    R c0 = c00 * (R(1) - ay) + c10 * ay;
    R c1 = c01 * (R(1) - ay) + c11 * ay;
    return c0 * (R(1) - az) + c1 * az;
  }

  // ---- target state (model.js:121-134) ----
  static R tprof(R z, R H) { return R(1) - sstep(R(0.7) * H, R(1.15) * H, z); }
  R tgtTh(const R* A, int k) const {
    R z = (R(k) + R(0.5)) * DZS();
    return bsA(k)[0] + A[0] / bsB(k)[0] * tprof(z, A[1]);
  }
  R tgtQv(const R* A, int k) const {
    R z = (R(k) + R(0.5)) * DZS();
    return bsA(k)[1] * (R(1) - A[2] * tprof(z, A[3]));
  }
  R tgtU(int i, int j, int k) const {
    R z = (R(k) + R(0.5)) * DZS();
    const R* a = l2(lsfB, i - 1, j);
    const R* b = l2(lsfB, i, j);
    return bsB(k)[2] + R(0.5) * (a[0] * tprof(z, a[2]) + b[0] * tprof(z, b[2]));
  }
  R tgtV(int i, int j, int k) const {
    R z = (R(k) + R(0.5)) * DZS();
    const R* a = l2(lsfB, i, j - 1);
    const R* b = l2(lsfB, i, j);
    return bsB(k)[3] + R(0.5) * (a[1] * tprof(z, a[2]) + b[1] * tprof(z, b[2]));
  }

  // ---- WGSL_M_LSF (model.js:142-244) ----
  const float* bd(int b) const { return &bnd[size_t(b) * OB_BOUNDARY_FLOATS]; }
  void bpt(int b, int i, R& x, R& y) const {
    const float* q = bd(b) + 20 + 4 * i;
    x = R(q[0]) + R(q[2]) * S.step.y;
    y = R(q[1]) + R(q[3]) * S.step.y;
  }
  void sdist(int b, R x, R y, R& sd, R& over, R& along) const {
    int np = int(bd(b)[0]);
    R best = R(1e30), sg = R(1), s0 = R(0);
    over = R(0); along = R(0);
    for (int i = 0; i < np - 1; i++) {
      R ax, ay, ex, ey;
      bpt(b, i, ax, ay);
      bpt(b, i + 1, ex, ey);
      R abx = ex - ax, aby = ey - ay;
      R la = std::max(std::sqrt(abx * abx + aby * aby), R(1));
      R t0 = ((x - ax) * abx + (y - ay) * aby) / (la * la);
      R t = t0;
      if (i > 0) t = std::max(t, R(0));
      if (i < np - 2) t = std::min(t, R(1));
      R dxp = x - (ax + t * abx), dyp = y - (ay + t * aby);
      R d = std::sqrt(dxp * dxp + dyp * dyp);
      if (d < best) {
        best = d;
        sg = (abx * (y - ay) - aby * (x - ax) > R(0)) ? R(1) : R(-1);
        over = (i == 0 ? std::max(-t0, R(0)) * la : R(0)) + (i == np - 2 ? std::max(t0 - R(1), R(0)) * la : R(0));
        along = s0 + t * la;
      }
      s0 += la;
    }
    sd = best * sg * R(bd(b)[15]);
  }
  R alongVar(int b, R s) const {
    const float* P4 = bd(b) + 16;
    if (P4[0] <= 0.f) return R(0);
    return clampv(fbm2<R>(s / R(P4[2]), R(P4[1]) + S.step.y / R(5400), 2) * R(1.6), R(-1), R(1));
  }
  R hotSpots(int b, R s) const {
    const float* P4 = bd(b) + 16;
    R L = R(P4[2]);
    // the hash seed is an integer the reference derives in f32 (model.js:192); deriving it in double would pick
    // another integer (5632.69f * 1000 rounds to 5632690 in f32, 5632689.94 in double) and another noise pattern
    int sd = int(P4[1] * 1000.f);
    R ph = S.step.y / R(4800);
    int e = int(std::floor(ph));
    R fe = sstep(R(0), R(1), fractv(ph));
    int k0 = int(std::floor(s / L));
    R acc = R(0);
    for (int k = k0 - 1; k <= k0 + 1; k++)
      for (int q = 0; q < 2; q++) {
        uint32_t h = hash3i(k, e + q, sd);
        R r1 = R(h & 0xffffu) / R(65535), r2 = R((h >> 16u) & 0xffffu) / R(65535);
        R z = (s - (R(k) + R(0.5) + R(0.7) * (r1 - R(0.5))) * L) / (R(0.17) * L);
        acc += (q == 1 ? fe : R(1) - fe) * (R(0.35) + R(0.65) * r2) * std::exp(-z * z);
      }
    return clampv(acc, R(0), R(1));
  }
  void k_lsf() {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        R x = (R(i) + R(0.5)) * DXS(), y = (R(j) + R(0.5)) * DXS();
        R sT = 0, sH = 0, sQ = 0, sHq = 0, sU = 0, sV = 0, sHw = 0, sw = 0, nud = 0;
        int nbb = int(S.cor.z);
        for (int b = 0; b < nbb; b++) {
          R d, over, along;
          sdist(b, x, y, d, over, along);
          const float* p = bd(b);
          R P0w = R(p[3]);
          R P1x = R(p[4]), P1y = R(p[5]), P1z = R(p[6]), P1w = R(p[7]);
          R P2x = R(p[8]), P2y = R(p[9]), P2z = R(p[10]), P2w = R(p[11]);
          R P3x = R(p[12]), P3y = R(p[13]), P3z = R(p[14]);
          R w = sstep(-P0w, P0w, d) * (R(1) - sstep(R(0), R(60000), over));
          if (w <= R(0)) continue;
          R vr = R(p[16]);
          R fadev = R(1) - sstep(R(30000), R(90000), d);
          R av = vr * alongVar(b, along) * fadev;
          R lift = vr > R(0) ? mixv(R(1), mixv(R(1) - R(0.85) * vr, R(1) + R(1.3) * vr, hotSpots(b, along)), fadev) : R(1);
          R Hmin = P1w * clampv(lift, R(0.15), R(3));
          R H = std::min(std::max(P1z * std::max(d + P0w, R(0)) * (R(1) + R(0.4) * av), Hmin), P1y);
          sT += w * P1x * std::exp(R(0.5) * av);
          sQ += w * P2x;
          sU += w * P2z * lift;
          sV += w * P2w * lift;
          sH += w * H;
          sHq += w * H * P2y;
          sHw += w * H * P3x;
          sw += w;
          nud = std::max(nud, P3y * sstep(P3z, P3z + R(40000), d) * (R(1) - sstep(R(0), R(60000), over)));
        }
        R iw = R(1) / std::max(sw, R(1e-6));
        R A[4] = {clampv(sT, R(-20), R(10)), std::max(sH * iw, R(100)), clampv(sQ, R(0), R(0.92)), std::max(sHq * iw, R(100))};
        R Bv[4] = {sU, sV, std::max(sHw * iw, R(100)), nud};
        size_t o = (size_t(j) * nx + i) * 4;
        for (int c = 0; c < 4; c++) { lsfA[o + c] = A[c]; lsfB[o + c] = Bv[c]; }
        R dzz = DZS(), ph = 0, bprev = 0;
        for (int k = nz - 1; k >= 0; k--) {
          R z = (R(k) + R(0.5)) * dzz;
          const R* a = bsA(k);
          const R* bb = bsB(k);
          R dth = A[0] / bb[0] * tprof(z, A[1]);
          R dqv = -a[1] * A[2] * tprof(z, A[3]);
          R bt = R(9.81) * (dth / a[0] + R(0.608) * dqv);
          if (k == nz - 1) ph = -bt * R(0.5) * dzz;
          else ph -= R(0.5) * (bt + bprev) * dzz;
          bprev = bt;
          phT[qidx(i, j, k)] = ph;
        }
      }
  }

  // ---- WGSL_M_CI (model.js:249-281) ----
  void k_ci() {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        R x = (R(i) + R(0.5)) * DXS(), y = (R(j) + R(0.5)) * DXS();
        R t = S.step.y;
        R best[4] = {R(0), R(0), R(1500), R(1500)};
        int ne = int(S.ci.x);
        for (int e = 0; e < ne; e++) {
          const float* E = &ciev[size_t(e) * OB_CI_FLOATS];
          R a0 = E[0], a1 = E[1], a2 = E[2], a3 = E[3], b0 = E[4], b1 = E[5], b2 = E[6], b3 = E[7];
          R c0 = E[8], c1 = E[9], c2 = E[10], c3 = E[11];
          if (t < b2 || t > b3) continue;
          R dxv = x - (a0 + c0 * (t - b2)), dyv = y - (a1 + c1 * (t - b2));
          R ang = std::atan2(dyv, dxv);
          R wob = R(1) + R(0.25) * gnoise2(std::cos(ang) * R(1.6) + c2, std::sin(ang) * R(1.6) + R(3.7) * c2);
          R g = sstep(b2, b2 + std::max(c3, R(60)), t);
          R r = std::sqrt(dxv * dxv + dyv * dyv) / (a3 * wob * (R(0.35) + R(0.65) * g));
          if (r >= R(1)) continue;
          R Lxv = R(nx) * DXS(), Lyv = R(ny) * DXS();
          R edge = std::min(std::min(x, Lxv - x), std::min(y, Lyv - y));
          R h = sstep(b2, b2 + R(60), t) * (R(1) - sstep(b3 - R(180), b3, t)) * sstep(S.sponge.x, S.sponge.x + R(10000), edge);
          R wt = b1 * (R(0.4) + R(0.6) * g) * std::cos(R(1.5707963) * r);
          if (h * wt > best[0] * best[1]) { best[0] = h; best[1] = wt; best[2] = a2; best[3] = b0; }
        }
        size_t o = (size_t(j) * nx + i) * 4;
        for (int c = 0; c < 4; c++) ciMap[o + c] = best[c];
      }
  }

  // ---- WGSL_M_INIT (model.js:284-339) ----
  // the vortex table at radius r, level k (model.js:292-297)
  void vxAt(R r, int k, R& vt, R& th) const {
    int nr = int(S.vtx.w);
    R fr = r / S.vtx.z;
    int i0 = int(std::floor(fr));
    if (i0 >= nr - 1) { vt = R(0); th = R(0); return; }
    size_t o = (size_t(clampi(k, 0, nz - 1)) * nr + i0) * 4;
    R a = fr - R(i0);
    vt = mixv(vx[o], vx[o + 4], a);
    th = mixv(vx[o + 1], vx[o + 5], a);
  }
  void k_init() {
#pragma omp parallel for schedule(static)
    for (int ck = 0; ck <= nz; ck++)
      for (int cj = 0; cj <= ny; cj++)
        for (int ci = 0; ci <= nx; ci++) {
          int k = std::min(ck, nz - 1);
          const R* A = l2(lsfA, ci, cj);
          R z = (R(k) + R(0.5)) * DZS();
          R nz0 = sstep(R(800), R(1500), z);
          const R dxv = DXS();
          if (S.vtx2.z > R(0.5)) {
            R px = (R(ci) + R(0.5)) * dxv - S.vtx.x, py = (R(cj) + R(0.5)) * dxv - S.vtx.y;
            nz0 = std::sqrt(px * px + py * py) < S.vtx2.x ? sstep(R(6000), R(8000), z) : R(1);
          }
          R noise = S.misc.z * (rnd3<R>(ci + 17, cj + 3, ck + 5) - R(0.5)) * R(2) * (R(1) - nz0);
          R th = tgtTh(A, k) + noise;
          R u = (cj < ny && ck < nz) ? tgtU(ci, cj, k) : R(0);
          R v = (ci < nx && ck < nz) ? tgtV(ci, cj, k) : R(0);
          const bool vort = S.vtx2.z > R(0.5);
          if (vort) {  // a warm-core vortex in gradient-wind and hydrostatic balance (setVortex's table)
            R pux = R(ci) * dxv - S.vtx.x, puy = (R(cj) + R(0.5)) * dxv - S.vtx.y;
            R ru = std::max(std::sqrt(pux * pux + puy * puy), R(1));
            R pvx = (R(ci) + R(0.5)) * dxv - S.vtx.x, pvy = R(cj) * dxv - S.vtx.y;
            R rv = std::max(std::sqrt(pvx * pvx + pvy * pvy), R(1));
            R pcx = (R(ci) + R(0.5)) * dxv - S.vtx.x, pcy = (R(cj) + R(0.5)) * dxv - S.vtx.y;
            R rc = std::sqrt(pcx * pcx + pcy * pcy);
            R vt, tp;
            vxAt(ru, k, vt, tp);
            u -= vt * puy / ru;
            vxAt(rv, k, vt, tp);
            v += vt * pvx / rv;
            vxAt(rc, k, vt, tp);
            th += tp;
          }
          R T = th * bsB(k)[0];
          R qv = std::min(tgtQv(A, k), R(0.95) * qvsat(T, bsB(k)[1], fIce(T)));
          if (vort) {  // a nearly saturated core; the same density
            R pcx = (R(ci) + R(0.5)) * dxv - S.vtx.x, pcy = (R(cj) + R(0.5)) * dxv - S.vtx.y;
            R f = (R(1) - sstep(R(0.6), R(1), std::sqrt(pcx * pcx + pcy * pcy) / S.vtx2.x)) * sstep(R(500), R(1500), z) *
                  (R(1) - sstep(R(7000), R(10000), z));
            R q2 = std::max(qv, f * S.vtx2.y * qvsat(T, bsB(k)[1], fIce(T)));
            R dqv = q2 - qv;
            qv = q2;
            th -= R(0.608) * dqv * bsA(k)[0];
          }
          R* o = &V[0][vidx(ci, cj, ck) * 4];
          o[0] = u; o[1] = v; o[2] = R(0); o[3] = th;
          if (ci < nx && cj < ny && ck < nz) {
            R* q1 = &Q1[0][qidx(ci, cj, ck) * 4];
            R* q2 = &Q2[0][qidx(ci, cj, ck) * 4];
            q1[0] = qv; q1[1] = q1[2] = q1[3] = R(0);
            q2[0] = q2[1] = q2[2] = q2[3] = R(0);
          }
        }
  }

  // ---- WGSL_M_NUT (model.js:342-389) ----
  void k_nut(const std::vector<R>& Vin, const std::vector<R>& Q1in) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          R dxv = DXS(), dzv = DZS();
          auto L = [&](int a, int b, int c) { return ldV(Vin, a, b, c); };
          auto uc = [&](int a, int b, int c) { int kk = clampi(c, 0, nz - 1); return R(0.5) * (L(a, b, c)[0] + L(a + 1, b, c)[0]) - bsB(kk)[2]; };
          auto vc = [&](int a, int b, int c) { int kk = clampi(c, 0, nz - 1); return R(0.5) * (L(a, b, c)[1] + L(a, b + 1, c)[1]) - bsB(kk)[3]; };
          auto wc = [&](int a, int b, int c) { return R(0.5) * (L(a, b, c)[2] + L(a, b, c + 1)[2]); };
          const R* v0 = L(i, j, k);
          R dudx = (L(i + 1, j, k)[0] - v0[0]) / dxv, dvdy = (L(i, j + 1, k)[1] - v0[1]) / dxv, dwdz = (L(i, j, k + 1)[2] - v0[2]) / dzv;
          R dudy = (uc(i, j + 1, k) - uc(i, j - 1, k)) / (R(2) * dxv), dudz = (uc(i, j, k + 1) - uc(i, j, k - 1)) / (R(2) * dzv);
          R dvdx = (vc(i + 1, j, k) - vc(i - 1, j, k)) / (R(2) * dxv), dvdz = (vc(i, j, k + 1) - vc(i, j, k - 1)) / (R(2) * dzv);
          R dwdx = (wc(i + 1, j, k) - wc(i - 1, j, k)) / (R(2) * dxv), dwdy = (wc(i, j + 1, k) - wc(i, j - 1, k)) / (R(2) * dxv);
          R s12 = R(0.5) * (dudy + dvdx), s13 = R(0.5) * (dudz + dwdx), s23 = R(0.5) * (dvdz + dwdy);
          R S2 = R(2) * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + R(4) * (s12 * s12 + s13 * s13 + s23 * s23);
          int kz0 = std::max(k - 1, 0), kz1 = std::min(k + 1, nz - 1);
          R N2 = R(9.81) / bsA(k)[0] * (L(i, j, kz1)[3] - L(i, j, kz0)[3]) / (R(kz1 - kz0) * dzv);
          const R* q1 = &Q1in[qidx(i, j, k) * 4];
          if (S.cor.w > R(0.5) && q1[1] + q1[2] > R(1e-5)) N2 = std::min(N2, R(0));
          R Ri = N2 / std::max(S2, R(1e-10));
          R fst = std::sqrt(std::max(R(0), R(1) - Ri / R(0.33)));
          R sS = std::sqrt(std::max(S2, R(0)));
          R lh = S.turb.x * dxv, lv = R(0.18) * dzv;
          R nuh = std::min(lh * lh * sS * fst, R(0.08) * dxv * dxv / std::max(DTS(), R(0.1)));
          R nuv = std::min(lv * lv * sS * fst, R(0.15) * dzv * dzv / std::max(DTS(), R(0.1)));
          R zc = (R(k) + R(0.5)) * dzv, h = S.hur2.z;
          if (hurOn() && zc < h) {  // K-profile boundary layer (model.js:377-386)
            const R* s0 = L(i, j, 0);
            R ua = R(0.5) * (s0[0] + L(i + 1, j, 0)[0]), va = R(0.5) * (s0[1] + L(i, j + 1, 0)[1]);
            R u1 = std::sqrt(ua * ua + va * va);
            R ust = std::sqrt(cdSfc(u1, sfc[(size_t(j) * nx + i) * 4])) * std::max(u1, S.hur3.y);
            R q = R(1) - zc / h;
            nuv = std::max(nuv, std::min(R(0.4) * ust * zc * q * q, R(0.15) * dzv * dzv / std::max(DTS(), R(0.1))));
          }
          size_t o = qidx(i, j, k) * 2;
          aux[o] = nuh;
          aux[o + 1] = nuv;
        }
  }

  // ---- advection helpers (model.js:391-433, 482-499) ----
  struct Loc {
    R vu[3], vv[3], vw[3], vc[3];
  };
  Loc localVel(const std::vector<R>& Vin, int i, int j, int k) const {
    auto L = [&](int a, int b, int c) { return ldV(Vin, a, b, c); };
    const R *p = L(i, j, k), *xm = L(i - 1, j, k), *xp = L(i + 1, j, k), *ym = L(i, j - 1, k), *yp = L(i, j + 1, k);
    const R *zm = L(i, j, k - 1), *zp = L(i, j, k + 1);
    const R *xmyp = L(i - 1, j + 1, k), *xmzp = L(i - 1, j, k + 1), *xpym = L(i + 1, j - 1, k), *ymzp = L(i, j - 1, k + 1);
    const R *xpzm = L(i + 1, j, k - 1), *ypzm = L(i, j + 1, k - 1);
    Loc o;
    o.vu[0] = p[0]; o.vu[1] = R(0.25) * (xm[1] + p[1] + xmyp[1] + yp[1]); o.vu[2] = R(0.25) * (xm[2] + p[2] + xmzp[2] + zp[2]);
    o.vv[0] = R(0.25) * (ym[0] + p[0] + xpym[0] + xp[0]); o.vv[1] = p[1]; o.vv[2] = R(0.25) * (ym[2] + p[2] + ymzp[2] + zp[2]);
    o.vw[0] = R(0.25) * (zm[0] + p[0] + xpzm[0] + xp[0]); o.vw[1] = R(0.25) * (zm[1] + p[1] + ypzm[1] + yp[1]); o.vw[2] = p[2];
    o.vc[0] = R(0.5) * (p[0] + xp[0]); o.vc[1] = R(0.5) * (p[1] + yp[1]); o.vc[2] = R(0.5) * (p[2] + zp[2]);
    return o;
  }
  void kvec(R k[3]) const { k[0] = DTS() / DXS(); k[1] = DTS() / DXS(); k[2] = DTS() / DZS(); }
  // the wind at a point in grid units (model.js:420-423)
  void velAt(const R x[3], R v[3]) const {
    const std::vector<R>& W = *trajV;
    v[0] = sampleV(W, x[0], x[1] - R(0.5), x[2] - R(0.5), 0);
    v[1] = sampleV(W, x[0] - R(0.5), x[1], x[2] - R(0.5), 1);
    v[2] = sampleV(W, x[0] - R(0.5), x[1] - R(0.5), x[2], 2);
  }
  // trace (model.js:424-433): first order clampX(p - s k v0); midpoint with the wind at p - s k v0 / 2 (cn.w)
  void trace(const R p[3], const R v0[3], R s, R out[3]) const {
    R k[3];
    kvec(k);
    R N[3] = {R(nx), R(ny), R(nz)};
    if (S.cn.w < R(0.5)) {
      for (int a = 0; a < 3; a++) out[a] = clampv(p[a] - s * k[a] * v0[a], R(0), N[a]);
      return;
    }
    R m[3], vm[3];
    for (int a = 0; a < 3; a++) m[a] = clampv(p[a] - R(0.5) * s * k[a] * v0[a], R(0), N[a]);
    velAt(m, vm);
    for (int a = 0; a < 3; a++) out[a] = clampv(p[a] - s * k[a] * vm[a], R(0), N[a]);
  }
  // 8-texel min/max at the departure cell (model.js:455-459)
  void mmV(const std::vector<R>& Vv, const R x[3], const R off[3], int ch, R& lo, R& hi) const {
    int i0 = int(std::floor(x[0] - off[0])), j0 = int(std::floor(x[1] - off[1])), k0 = int(std::floor(x[2] - off[2]));
    lo = R(1e30); hi = R(-1e30);
    for (int q = 0; q < 8; q++) {
      R s = ldV(Vv, i0 + (q & 1), j0 + ((q >> 1) & 1), k0 + (q >> 2))[ch];
      lo = std::min(lo, s); hi = std::max(hi, s);
    }
  }

  // ---- WGSL_M_ADVV1 (model.js:434-450): trajectories from Vin, values carried from Vval (Vp in hurricane mode) ----
  void k_advv1(const std::vector<R>& Vin, const std::vector<R>& Vval) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= nz; k++)
      for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
          Loc L = localVel(Vin, i, j, k);
          R pu[3] = {R(i), R(j) + R(0.5), R(k) + R(0.5)}, pv[3] = {R(i) + R(0.5), R(j), R(k) + R(0.5)};
          R pw[3] = {R(i) + R(0.5), R(j) + R(0.5), R(k)}, pc[3] = {R(i) + R(0.5), R(j) + R(0.5), R(k) + R(0.5)};
          R x[3];
          R* o = &Vt[vidx(i, j, k) * 4];
          trace(pu, L.vu, R(1), x);
          o[0] = sampleV(Vval, x[0], x[1] - R(0.5), x[2] - R(0.5), 0);
          trace(pv, L.vv, R(1), x);
          o[1] = sampleV(Vval, x[0] - R(0.5), x[1], x[2] - R(0.5), 1);
          trace(pw, L.vw, R(1), x);
          o[2] = sampleV(Vval, x[0] - R(0.5), x[1] - R(0.5), x[2], 2);
          trace(pc, L.vc, R(1), x);
          o[3] = sampleV(Vval, x[0] - R(0.5), x[1] - R(0.5), x[2] - R(0.5), 3);
        }
  }
  // ---- WGSL_M_ADVV2 (model.js:451-481) ----
  void k_advv2(const std::vector<R>& Vin, const std::vector<R>& Vval, std::vector<R>& Vout) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= nz; k++)
      for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
          Loc L = localVel(Vin, i, j, k);
          R kk[3];
          kvec(kk);
          R pu[3] = {R(i), R(j) + R(0.5), R(k) + R(0.5)}, pv[3] = {R(i) + R(0.5), R(j), R(k) + R(0.5)};
          R pw[3] = {R(i) + R(0.5), R(j) + R(0.5), R(k)}, pc[3] = {R(i) + R(0.5), R(j) + R(0.5), R(k) + R(0.5)};
          const R* hat = &Vt[vidx(i, j, k) * 4];
          const R* old = ldV(Vval, i, j, k);
          R x[3], b[4];
          trace(pu, L.vu, R(-1), x);
          b[0] = sampleV(Vt, x[0], x[1] - R(0.5), x[2] - R(0.5), 0);
          trace(pv, L.vv, R(-1), x);
          b[1] = sampleV(Vt, x[0] - R(0.5), x[1], x[2] - R(0.5), 1);
          trace(pw, L.vw, R(-1), x);
          b[2] = sampleV(Vt, x[0] - R(0.5), x[1] - R(0.5), x[2], 2);
          trace(pc, L.vc, R(-1), x);
          b[3] = sampleV(Vt, x[0] - R(0.5), x[1] - R(0.5), x[2] - R(0.5), 3);
          R cx = L.vc[0] * kk[0], cy = L.vc[1] * kk[1], cz = L.vc[2] * kk[2];
          R cour = std::sqrt(cx * cx + cy * cy + cz * cz);
          R sm = R(0.5) * S.misc.y * clampv(cour / R(0.35), S.dzv.w, R(1));
          R r[4];
          for (int c = 0; c < 4; c++) r[c] = hat[c] + sm * (old[c] - b[c]);
          static const R offs[4][3] = {{R(0), R(0.5), R(0.5)}, {R(0.5), R(0), R(0.5)}, {R(0.5), R(0.5), R(0)}, {R(0.5), R(0.5), R(0.5)}};
          const R* vels[4] = {L.vu, L.vv, L.vw, L.vc};
          const R* pts[4] = {pu, pv, pw, pc};
          R* o = &Vout[vidx(i, j, k) * 4];
          for (int c = 0; c < 4; c++) {
            trace(pts[c], vels[c], R(1), x);
            R lo, hi;
            mmV(Vval, x, offs[c], c, lo, hi);
            o[c] = clampv(r[c], lo, hi);
          }
        }
  }

  // ---- scalar advection (model.js:482-576) ----
  void cellVel(const std::vector<R>& Vin, int i, int j, int k, R v[3]) const {
    const R* p = ldV(Vin, i, j, k);
    v[0] = R(0.5) * (p[0] + ldV(Vin, i + 1, j, k)[0]);
    v[1] = R(0.5) * (p[1] + ldV(Vin, i, j + 1, k)[1]);
    v[2] = R(0.5) * (p[2] + ldV(Vin, i, j, k + 1)[2]);
  }
  void traceQ(const R p[3], const R v0[3], R fall, R s, R out[3]) const {  // model.js:494-499
    R k[3];
    kvec(k);
    R N[3] = {R(nx), R(ny), R(nz)};
    R f[3] = {R(0), R(0), fall};
    if (S.cn.w < R(0.5)) {
      for (int a = 0; a < 3; a++) out[a] = clampv(p[a] - s * k[a] * (v0[a] - f[a]), R(0.5), N[a] - R(0.5));
      return;
    }
    R m[3], vm[3];
    for (int a = 0; a < 3; a++) m[a] = clampv(p[a] - R(0.5) * s * k[a] * (v0[a] - f[a]), R(0), N[a]);
    velAt(m, vm);
    for (int a = 0; a < 3; a++) out[a] = clampv(p[a] - s * k[a] * (vm[a] - f[a]), R(0.5), N[a] - R(0.5));
  }
  R sQ(const std::vector<R>& t, const R x[3], int ch) const { return sampleQ(t, x[0] - R(0.5), x[1] - R(0.5), x[2] - R(0.5), ch); }
  void mmQ(const std::vector<R>& t, const R x[3], R lo[4], R hi[4]) const {
    int i0 = int(std::floor(x[0] - R(0.5))), j0 = int(std::floor(x[1] - R(0.5))), k0 = int(std::floor(x[2] - R(0.5)));
    for (int c = 0; c < 4; c++) { lo[c] = R(1e30); hi[c] = R(-1e30); }
    for (int q = 0; q < 8; q++) {
      const R* s = ldQ(t, i0 + (q & 1), j0 + ((q >> 1) & 1), k0 + (q >> 2));
      for (int c = 0; c < 4; c++) { lo[c] = std::min(lo[c], s[c]); hi[c] = std::max(hi[c], s[c]); }
    }
  }
  void k_advq1(const std::vector<R>& Vin) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          R v[3], p[3] = {R(i) + R(0.5), R(j) + R(0.5), R(k) + R(0.5)}, x[3];
          cellVel(Vin, i, j, k, v);
          const R* q1 = &Q1[0][qidx(i, j, k) * 4];
          const R* q2 = &Q2[0][qidx(i, j, k) * 4];
          R rho = bsA(k)[2];
          R fr, fn;
          vtRain(q1[3], q2[2], rho, fr, fn);
          R fs = vtS(q2[0], rho), fg = vtGrau(q2[1], rho), fi = vtI(q1[2], rho);
          R a[4];
          traceQ(p, v, R(0), R(1), x);
          for (int c = 0; c < 4; c++) a[c] = sQ(Q1[0], x, c);
          R bq0[3] = {x[0], x[1], x[2]};
          if (fi > R(0)) {
            traceQ(p, v, fi, R(1), x);
            a[2] = sQ(Q1[0], x, 2);
          }
          x[0] = bq0[0]; x[1] = bq0[1]; x[2] = bq0[2];
          R bq[4];
          for (int c = 0; c < 4; c++) bq[c] = sQ(Q2[0], x, c);
          traceQ(p, v, fr, R(1), x);
          R r = sQ(Q1[0], x, 3);
          traceQ(p, v, fs, R(1), x);
          R s = sQ(Q2[0], x, 0);
          traceQ(p, v, fg, R(1), x);
          R g = sQ(Q2[0], x, 1);
          R nr = bq[2];
          if (thompson()) { traceQ(p, v, fn, R(1), x); nr = sQ(Q2[0], x, 2); }
          R* o1 = &Q1t[qidx(i, j, k) * 4];
          R* o2 = &Q2t[qidx(i, j, k) * 4];
          o1[0] = a[0]; o1[1] = a[1]; o1[2] = a[2]; o1[3] = r;
          o2[0] = s; o2[1] = g; o2[2] = nr; o2[3] = bq[3];
        }
  }
  void k_advq2(const std::vector<R>& Vin) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          R v[3], p[3] = {R(i) + R(0.5), R(j) + R(0.5), R(k) + R(0.5)}, x[3], kk[3];
          cellVel(Vin, i, j, k, v);
          kvec(kk);
          const R* q1 = ldQ(Q1[0], i, j, k);
          const R* q2 = ldQ(Q2[0], i, j, k);
          R rho = bsA(k)[2];
          R fr, fnv;
          vtRain(q1[3], q2[2], rho, fr, fnv);
          R fs = vtS(q2[0], rho), fg = vtGrau(q2[1], rho), fi = vtI(q1[2], rho);
          const R* h1 = &Q1t[qidx(i, j, k) * 4];
          const R* h2 = &Q2t[qidx(i, j, k) * 4];
          R cx = v[0] * kk[0], cy = v[1] * kk[1], cz = v[2] * kk[2];
          R cour = std::sqrt(cx * cx + cy * cy + cz * cz);
          R sm = R(0.5) * S.misc.y * clampv(cour / R(0.35), S.dzv.w, R(1));
          R b1[4], b2[4];
          traceQ(p, v, R(0), R(-1), x);
          for (int c = 0; c < 4; c++) { b1[c] = sQ(Q1t, x, c); b2[c] = sQ(Q2t, x, c); }
          traceQ(p, v, fr, R(-1), x);
          R br = sQ(Q1t, x, 3);
          traceQ(p, v, fs, R(-1), x);
          R bs = sQ(Q2t, x, 0);
          traceQ(p, v, fg, R(-1), x);
          R bg = sQ(Q2t, x, 1);
          R fn_ = thompson() ? fnv : R(0);
          traceQ(p, v, fn_, R(-1), x);
          R bn = sQ(Q2t, x, 2);
          R bi = b1[2];
          if (fi > R(0)) {
            traceQ(p, v, fi, R(-1), x);
            bi = sQ(Q1t, x, 2);
          }
          R r1[4] = {h1[0] + sm * (q1[0] - b1[0]), h1[1] + sm * (q1[1] - b1[1]), h1[2] + sm * (q1[2] - bi), h1[3] + sm * (q1[3] - br)};
          R r2[4] = {h2[0] + sm * (q2[0] - bs), h2[1] + sm * (q2[1] - bg), h2[2] + sm * (q2[2] - bn), h2[3] + sm * (q2[3] - b2[3])};
          R lo[4], hi[4], lo2[4], hi2[4];
          traceQ(p, v, R(0), R(1), x);
          mmQ(Q1[0], x, lo, hi);
          mmQ(Q2[0], x, lo2, hi2);
          r1[0] = clampv(r1[0], lo[0], hi[0]);
          r1[1] = clampv(r1[1], lo[1], hi[1]);
          r2[3] = clampv(r2[3], lo2[3], hi2[3]);
          {  // cloud ice at its own fall speed (the air's trace when it does not fall: mi = m1)
            R xi[3], loi[4], hii[4];
            traceQ(p, v, fi, R(1), xi);
            mmQ(Q1[0], xi, loi, hii);
            r1[2] = clampv(r1[2], loi[2], hii[2]);
          }
          traceQ(p, v, fr, R(1), x);
          mmQ(Q1[0], x, lo, hi);
          r1[3] = clampv(r1[3], lo[3], hi[3]);
          traceQ(p, v, fs, R(1), x);
          mmQ(Q2[0], x, lo, hi);
          r2[0] = clampv(r2[0], lo[0], hi[0]);
          traceQ(p, v, fg, R(1), x);
          mmQ(Q2[0], x, lo, hi);
          r2[1] = clampv(r2[1], lo[1], hi[1]);
          traceQ(p, v, fn_, R(1), x);
          mmQ(Q2[0], x, lo, hi);
          r2[2] = clampv(r2[2], lo[2], hi[2]);
          R* o1 = &Q1[1][qidx(i, j, k) * 4];
          R* o2 = &Q2[1][qidx(i, j, k) * 4];
          for (int c = 0; c < 4; c++) { o1[c] = std::max(r1[c], R(0)); o2[c] = std::max(r2[c], R(0)); }
        }
  }

  // ---- WGSL_M_PHYS (model.js:578-907), outbreak mode ----
  R spongeLat(R xmx, R xmy) const {
    R Lxv = R(nx) * DXS(), Lyv = R(ny) * DXS();
    R e = std::min(std::min(xmx, Lxv - xmx), std::min(xmy, Lyv - xmy));
    R d = clampv(R(1) - e / S.sponge.x, R(0), R(1));
    return d * (R(0.3) + R(0.7) * d) / S.sponge.y;
  }
  R spongeTop(R z) const {
    R ztop = R(nz) * DZS();
    if (z < S.sponge.z) return R(0);
    R s = std::sin(R(1.5707963) * (z - S.sponge.z) / (ztop - S.sponge.z));
    return s * s / S.sponge.w;
  }
  R bsV(int k, int ch) const {
    int kk = clampi(k, 0, nz - 1);
    if (ch == 0) return bsB(kk)[2];
    if (ch == 1) return bsB(kk)[3];
    if (ch == 3) return bsA(kk)[0];
    return R(0);
  }
  void k_phys(const std::vector<R>& Vin, std::vector<R>& Vout) {
    const std::vector<R>& Q1in = Q1[1];
    const std::vector<R>& Q2in = Q2[1];
#pragma omp parallel for schedule(static)
    for (int ck = 0; ck <= nz; ck++)
      for (int cj = 0; cj <= ny; cj++)
        for (int ci = 0; ci <= nx; ci++) {
          auto L = [&](int a, int b, int c) { return ldV(Vin, a, b, c); };
          auto ldA = [&](int a, int b, int c) { return &aux[qidx(clampi(a, 0, nx - 1), clampi(b, 0, ny - 1), clampi(c, 0, nz - 1)) * 2]; };
          auto ldP = [&](int a, int b, int c) { return phT[qidx(clampi(a, 0, nx - 1), clampi(b, 0, ny - 1), clampi(c, 0, nz - 1))]; };
          auto lapH = [&](int ch, R me) { return L(ci + 1, cj, ck)[ch] + L(ci - 1, cj, ck)[ch] + L(ci, cj + 1, ck)[ch] + L(ci, cj - 1, ck)[ch] - R(4) * me; };
          auto lapZ = [&](int ch, R me, bool lo, bool hi) {
            R a = lo ? me : L(ci, cj, ck - 1)[ch];
            R b = hi ? me : L(ci, cj, ck + 1)[ch];
            return a + b - R(2) * me;
          };
          auto lapZp = [&](int ch, R me, bool lo, bool hi) {
            R m0 = me - bsV(ck, ch);
            R a = lo ? m0 : L(ci, cj, ck - 1)[ch] - bsV(ck - 1, ch);
            R b = hi ? m0 : L(ci, cj, ck + 1)[ch] - bsV(ck + 1, ch);
            return a + b - R(2) * m0;
          };
          auto buoy = [&](int a, int b, int c) {
            const R* A = bsA(c);
            const R* v = L(a, b, c);
            const R* q1 = ldQ(Q1in, a, b, c);
            const R* q2 = ldQ(Q2in, a, b, c);
            return R(9.81) * ((v[3] - A[0]) / A[0] + R(0.608) * (q1[0] - A[1]) - (q1[1] + q1[2] + q1[3] + q2[0] + q2[1]));
          };
          const R dxv = DXS(), dzv = DZS(), dt = DTS();
          const R* V = L(ci, cj, ck);
          R o[4] = {V[0], V[1], V[2], V[3]};
          R ix2 = R(1) / (dxv * dxv), iz2 = R(1) / (dzv * dzv);
          R fc = S.cor.x, nudR = R(1) / S.cor.y;
          // u
          if (cj < ny && ck < nz) {
            R xmx = R(ci) * dxv, xmy = (R(cj) + R(0.5)) * dxv, z = (R(ck) + R(0.5)) * dzv;
            const R *a0 = ldA(ci - 1, cj, ck), *a1 = ldA(ci, cj, ck);
            R nux = R(0.5) * (a0[0] + a1[0]) + S.turb.y, nuy = R(0.5) * (a0[1] + a1[1]) + S.turb.y;
            R du = nux * lapH(0, V[0]) * ix2 + nuy * lapZp(0, V[0], ck == 0, ck == nz - 1) * iz2;
            R ut = tgtU(ci, cj, ck);
            R vbar = R(0.25) * (L(ci - 1, cj, ck)[1] + V[1] + L(ci - 1, cj + 1, ck)[1] + L(ci, cj + 1, ck)[1]);
            R vtb = R(0.5) * (tgtV(ci - 1, cj, ck) + tgtV(ci, cj + 1, ck));
            R nw = R(0.5) * (l2(lsfB, ci - 1, cj)[3] + l2(lsfB, ci, cj)[3]);
            du += (spongeLat(xmx, xmy) + spongeTop(z) + nw * nudR) * (ut - V[0]);
            du += fc * (vbar - vtb);
            if (ci > 0 && ci < nx) du -= (ldP(ci, cj, ck) - ldP(ci - 1, cj, ck)) / dxv;
            if (ck == 0 && S.turb.w > R(0.5)) {
              R g0 = V[0], g1 = vbar, h0 = ut, h1 = vtb;
              R cd = S.micro.w;
              if (hurOn()) {
                R land = R(0.5) * (sfc[(size_t(cj) * nx + std::max(ci - 1, 0)) * 4] + sfc[(size_t(std::min(cj, ny - 1)) * nx + std::min(ci, nx - 1)) * 4]);
                cd = cdSfc(std::sqrt(g0 * g0 + g1 * g1), land);
              }
              du += cd * (-std::sqrt(g0 * g0 + g1 * g1) * g0 + std::sqrt(h0 * h0 + h1 * h1) * h0) / dzv;
            }
            o[0] = V[0] + dt * du;
          } else o[0] = R(0);
          // v
          if (ci < nx && ck < nz) {
            R xmx = (R(ci) + R(0.5)) * dxv, xmy = R(cj) * dxv, z = (R(ck) + R(0.5)) * dzv;
            const R *a0 = ldA(ci, cj - 1, ck), *a1 = ldA(ci, cj, ck);
            R nux = R(0.5) * (a0[0] + a1[0]) + S.turb.y, nuy = R(0.5) * (a0[1] + a1[1]) + S.turb.y;
            R dv = nux * lapH(1, V[1]) * ix2 + nuy * lapZp(1, V[1], ck == 0, ck == nz - 1) * iz2;
            R vt = tgtV(ci, cj, ck);
            R ubar = R(0.25) * (L(ci, cj - 1, ck)[0] + V[0] + L(ci + 1, cj - 1, ck)[0] + L(ci + 1, cj, ck)[0]);
            R utb = R(0.5) * (tgtU(ci, cj - 1, ck) + tgtU(ci + 1, cj, ck));
            R nw = R(0.5) * (l2(lsfB, ci, cj - 1)[3] + l2(lsfB, ci, cj)[3]);
            dv += (spongeLat(xmx, xmy) + spongeTop(z) + nw * nudR) * (vt - V[1]);
            dv -= fc * (ubar - utb);
            if (cj > 0 && cj < ny) dv -= (ldP(ci, cj, ck) - ldP(ci, cj - 1, ck)) / dxv;
            if (ck == 0 && S.turb.w > R(0.5)) {
              R g0 = ubar, g1 = V[1], h0 = utb, h1 = vt;
              R cd = S.micro.w;
              if (hurOn()) {
                R land = R(0.5) * (sfc[(size_t(std::max(cj - 1, 0)) * nx + ci) * 4] + sfc[(size_t(std::min(cj, ny - 1)) * nx + std::min(ci, nx - 1)) * 4]);
                cd = cdSfc(std::sqrt(g0 * g0 + g1 * g1), land);
              }
              dv += cd * (-std::sqrt(g0 * g0 + g1 * g1) * g1 + std::sqrt(h0 * h0 + h1 * h1) * h1) / dzv;
            }
            o[1] = V[1] + dt * dv;
          } else o[1] = R(0);
          // w
          if (ci < nx && cj < ny && ck > 0 && ck < nz) {
            R xmx = (R(ci) + R(0.5)) * dxv, xmy = (R(cj) + R(0.5)) * dxv, z = R(ck) * dzv;
            const R *a0 = ldA(ci, cj, ck - 1), *a1 = ldA(ci, cj, ck);
            R nux = R(0.5) * (a0[0] + a1[0]) + S.turb.y, nuy = R(0.5) * (a0[1] + a1[1]) + S.turb.y;
            R dw = nux * lapH(2, V[2]) * ix2 + nuy * lapZ(2, V[2], false, false) * iz2;
            dw += R(0.5) * (buoy(ci, cj, ck - 1) + buoy(ci, cj, ck)) - (ldP(ci, cj, ck) - ldP(ci, cj, ck - 1)) / dzv;
            dw += (spongeLat(xmx, xmy) + spongeTop(z)) * (R(0) - V[2]);
            const R* civ = &ciMap[(size_t(cj) * nx + ci) * 4];
            if (civ[0] > R(0) && !hurOn()) {
              R zz = std::abs(z - civ[2]) / civ[3];
              if (zz < R(1)) {
                R cv = std::cos(R(1.5707963) * zz);
                dw += S.misc.w * civ[0] * cv * std::max(civ[1] * cv - V[2], R(0));
              }
            }
            o[2] = V[2] + dt * dw;
          } else o[2] = R(0);
          // theta + microphysics
          if (ci < nx && cj < ny && ck < nz) {
            R xmx = (R(ci) + R(0.5)) * dxv, xmy = (R(cj) + R(0.5)) * dxv, z = (R(ck) + R(0.5)) * dzv;
            const R* A = bsA(ck);
            const R* Bb = bsB(ck);
            const R* LA = l2(lsfA, ci, cj);
            R nw = l2(lsfB, ci, cj)[3];
            R tth = tgtTh(LA, ck), tqv = tgtQv(LA, ck);
            R relax = spongeLat(xmx, xmy) + nw * nudR;
            const R* ax = ldA(ci, cj, ck);
            R nux = ax[0] * R(3) + S.turb.y, nuy = ax[1] * R(3) + S.turb.y;
            R th = V[3] + dt * (nux * lapH(3, V[3]) * ix2 + nuy * lapZp(3, V[3], ck == 0, ck == nz - 1) * iz2 + (relax + spongeTop(z)) * (tth - V[3]));
            R q1[4], q2[4];
            for (int c = 0; c < 4; c++) { q1[c] = ldQ(Q1in, ci, cj, ck)[c]; q2[c] = ldQ(Q2in, ci, cj, ck)[c]; }
            R l1[3], l1z[3];
            for (int c = 0; c < 3; c++) {
              l1[c] = ldQ(Q1in, ci + 1, cj, ck)[c] + ldQ(Q1in, ci - 1, cj, ck)[c] + ldQ(Q1in, ci, cj + 1, ck)[c] + ldQ(Q1in, ci, cj - 1, ck)[c] - R(4) * q1[c];
              l1z[c] = (ck == 0 ? q1[c] : ldQ(Q1in, ci, cj, ck - 1)[c]) + (ck == nz - 1 ? q1[c] : ldQ(Q1in, ci, cj, ck + 1)[c]) - R(2) * q1[c];
            }
            R qvb = (ck == 0 ? A[1] : bsA(ck - 1)[1]) + (ck == nz - 1 ? A[1] : bsA(ck + 1)[1]) - R(2) * A[1];
            l1z[0] -= qvb;
            for (int c = 0; c < 3; c++) q1[c] = q1[c] + dt * (nux * l1[c] * ix2 + nuy * l1z[c] * iz2);
            q1[0] += dt * relax * (tqv - q1[0]);
            if (hurOn()) {  // model.js:713-774
              th += dt * clampv((tth - V[3]) / S.hur2.x, -S.hur2.y, S.hur2.y);
              const R* cs = &ciMap[(size_t(cj) * nx + ci) * 4];
              if (cs[0] > R(0)) {
                R zz = std::abs(z - cs[2]) / cs[3];
                if (zz < R(1)) {
                  R f = cs[0] * std::cos(R(1.5707963) * zz) * cs[1] / R(8);
                  th += dt * R(1.2e-3) * f;
                  q1[0] += dt * f / R(600) * std::max(R(0.97) * qvsat(V[3] * Bb[0], Bb[1], R(0)) - q1[0], R(0));
                }
              }
              R dxh = xmx - S.hur4.x, dyh = xmy - S.hur4.y;
              R rS = std::sqrt(dxh * dxh + dyh * dyh);
              R wEnv = sstep(S.hur4.w, R(1.5) * S.hur4.w, rS) / R(3600);
              th += dt * wEnv * (tth - V[3]);
              q1[0] += dt * wEnv * (tqv - q1[0]);
              if (z < S.hur2.z) {
                const R* s0 = L(ci, cj, 0);
                R ua = R(0.5) * (s0[0] + L(ci + 1, cj, 0)[0]), va = R(0.5) * (s0[1] + L(ci, cj + 1, 0)[1]);
                R u1 = std::sqrt(ua * ua + va * va);
                R e = S.step.y / R(900), e0 = std::floor(e);
                R qx = xmx / R(6000), qy = xmy / R(6000);
                R r = R(0.5) * mixv(gnoise2<R>(qx + R(37.1) * e0, qy + R(11.3) * e0), gnoise2<R>(qx + R(37.1) * (e0 + R(1)), qy + R(11.3) * (e0 + R(1))),
                                    sstep(R(0), R(1), fractv(e)));
                R fu = std::min(u1 * u1 / R(225), R(1)) * (R(1) - sstep(R(20), R(32), u1)) * (R(1) - sstep(S.hur4.z, R(1.5) * S.hur4.z, rS));
                th += dt * S.hur3.z * R(2) * r * fu * (R(1) - z / S.hur2.z);
              }
              if (ck == 0) {  // the sea's sensible and latent heat, dissipative heating
                const R* sf = &sfc[(size_t(cj) * nx + ci) * 4];
                R land = clampv(sf[0], R(0), R(1));
                R ua = R(0.5) * (V[0] + L(ci + 1, cj, ck)[0]), va = R(0.5) * (V[1] + L(ci, cj + 1, ck)[1]);
                R u1 = std::sqrt(ua * ua + va * va);
                R ch = S.hur.y * S.hur2.w * std::max(u1, S.hur3.y) / dzv;
                R ps = std::max(S.hur.w + A[2] * S.cn.y * phi[pidx(ci, cj, ck)], R(50000));
                R ths = sf[1] * std::pow(R(1e5) / ps, R(0.2854));
                th += dt * ch * (R(1) - land) * (ths - V[3]);
                if (S.hur5.y > R(0.5)) {
                  R cdh = cdSfc(u1, land);
                  th += dt * cdh * u1 * u1 * u1 / (R(CPD) * dzv) / Bb[0];
                }
                R qsS = qvsat(sf[1], ps, R(0));
                R qsL = qvsat(V[3] * Bb[0], ps, R(0));
                q1[0] += dt * ch * ((R(1) - land) * (qsS - q1[0]) + land * S.hur.z * std::max(qsL - q1[0], R(0)));
              }
            }
            for (int c = 0; c < 4; c++) { q1[c] = std::max(q1[c], R(0)); q2[c] = std::max(q2[c], R(0)); }
            R pi0 = Bb[0], p0 = Bb[1], rho = A[2];
            R T = th * pi0;
            R qv = q1[0], qc = q1[1], qi = q1[2], qr = q1[3], qs = q2[0], qg = q2[1];
            bool thm = thompson();
            R nr = std::max(q2[2], R(0));
            R rq = R(1000) * rho;
            R rs = std::sqrt(S.step.z / rho);
            R pauto = S.micro.x * std::max(qc - S.micro.y, R(0));
            R accr = R(2.2) * qc * std::pow(qr, R(0.875));
            if (thm && qr > R(1e-9)) {
              R l = lamR(qr, nr);
              accr = R(3100) * rho * nr * std::pow(l, R(-2.8)) * qc * rs;
            }
            R da = std::min(pauto * dt, qc);
            R dc = std::min(accr * dt, qc - da);
            qc -= da + dc;
            qr += da + dc;
            nr += da / R(2.68e-10);
            R dTc = T - R(T0K);
            if (dTc < R(0)) {
              R psaut = R(1e-3) * std::exp(R(0.025) * dTc) * std::max(qi - R(6e-4), R(0));
              R psacw = R(5.4e-3) * qc * std::pow(std::max(rq * qs, R(0)), R(0.81)) * rs;
              R psaci = R(5.4e-3) * qi * std::pow(std::max(rq * qs, R(0)), R(0.81)) * std::exp(R(0.025) * dTc) * rs;
              R ewet = R(1) / (R(1) + qg / R(0.008));
              R pgacw = R(3.1e-3) * qc * std::pow(std::max(rq * qg, R(0)), R(0.875)) * rs * ewet;
              R pgaci = R(3.0e-4) * qi * std::pow(std::max(rq * qg, R(0)), R(0.875)) * rs;
              R pgacr = R(3.1e-3) * qr * std::pow(std::max(rq * qg, R(0)), R(0.875)) * rs * ewet;
              R pgfr = std::min(R(2e-4) * S.micro.z * (std::exp(R(0.66) * std::min(-dTc, R(20))) - R(1)), R(0.08)) * qr;
              R pgaut = R(1e-3) * std::exp(R(0.09) * dTc) * std::max(qs - R(6e-4), R(0)) * (thm ? R(0.25) : R(1));
              R a1 = std::min((psaut + psaci + pgaci) * dt, qi);
              R fs1 = (psaut + psaci) / std::max(psaut + psaci + pgaci, R(1e-20));
              qi -= a1; qs += a1 * fs1; qg += a1 * (R(1) - fs1);
              R a2 = std::min((psacw + pgacw) * dt, qc);
              R fs2 = psacw / std::max(psacw + pgacw, R(1e-20));
              R rimeS = thm ? R(0.95) : R(0.7);
              qc -= a2; qs += a2 * fs2 * rimeS; qg += a2 * (R(1) - fs2 * rimeS);
              R a3 = std::min((pgacr + pgfr) * dt, qr);
              if (T < R(235)) a3 = qr;
              if (qr > R(1e-12)) nr *= (qr - a3) / qr;
              qr -= a3; qg += a3;
              R a4 = std::min(pgaut * dt, qs);
              qs -= a4; qg += a4;
              T += R(LFC / CPD) * (a2 + a3);
            } else {
              R m1 = std::min(R(0.012) * dTc * qs * dt, qs);
              R m2 = std::min(R(0.0022) * dTc * qg * dt, qg);
              if (thm) {
                if (qg > R(1e-9)) {
                  R l = lamG(qg, rho), n0 = n0G(qg, rho);
                  R vent = R(0.78) / (l * l) + R(0.31 * 0.843 * 1.89 * 5430.0) * std::pow(S.step.z / rho, R(0.25)) * std::pow(l, R(-2.945));
                  R heat = R(2.4e-2) * dTc - R(LVC * 2.26e-5) * rho * (qvsat(R(T0K), p0, R(0)) - qv);
                  m2 = clampv(R(6.2832) / (rho * R(LFC)) * heat * n0 * vent * dt, R(0), qg);
                  nr += m2 / qg * n0 / (rho * l);
                }
                if (qs > R(1e-9)) {
                  R ls = std::pow(R(3.14159 * 100.0 * 2e6) / (rho * qs), R(0.25));
                  nr += m1 / qs * R(2e6) / (rho * ls);
                }
              }
              qs -= m1; qg -= m2; qr += m1 + m2;
              T -= R(LFC / CPD) * (m1 + m2);
            }
            R qvsl = qvsat(T, p0, R(0));
            if (qr > R(0) && qv < qvsl) {
              R rc = R(0.001) * rho * qr;
              R ern = ((R(1.6) + R(124.9) * std::pow(rc, R(0.2046))) * std::pow(rc, R(0.525)) / (R(2.55e8) / (p0 * qvsl) + R(5.4e5))) *
                      ((qvsl - qv) / (R(0.001) * rho * qvsl));
              R srt = S.micro2.y > R(0) ? std::sqrt(rc / (rc + R(0.001) * rho * S.micro2.y)) : R(1);
              R e = ern * srt * dt * S.turb.z;
              if (thm) {
                R l = lamR(qr, nr), n0 = rho * nr * l;
                R Ap = R(LVC * LVC) / (R(2.4e-2 * RVC) * T * T);
                R Bp = R(1) / (rho * qvsl * R(2.26e-5));
                R vent = R(0.78) / (l * l) + R(0.31 * 0.843 * 1.827 * 7492.0) * std::pow(S.step.z / rho, R(0.25)) * std::pow(l, R(-2.9));
                e = R(6.2832) * (R(1) - qv / qvsl) * n0 * vent / (rho * (Ap + Bp)) * dt * S.micro2.w;
              }
              e = clampv(e, R(0), std::min(qr, qvsl - qv));
              if (thm && qr > R(1e-12)) nr *= (qr - e) / qr;
              qr -= e; qv += e; T -= R(LVC / CPD) * e;
            }
            if (thm) {
              if (qr > R(1e-9)) {
                R dm = R(1.817) / lamR(qr, nr);
                R fb = clampv(R(1) - std::exp(R(2300) * (dm - R(1.1e-3))), R(-2), R(1));
                nr *= std::exp(R(-7.12) * rho * qr * fb * dt);
                nr = clampv(nr, qr * R(3.183e5), qr * R(3.183e11));
              } else nr = R(0);
            }
            R qvsi = qvsat(T, p0, R(1));
            if (dTc < R(0) && qv < qvsi) {
              R sub = std::max(R(1) - qv / qvsi, R(0));
              R e = std::min((R(2e-3) * qs + R(5e-4) * qg) * sub * dt, (qvsi - qv) * R(0.5));
              R fsn = qs / std::max(qs + qg, R(1e-20));
              e = std::min(e, qs + qg);
              qs -= e * fsn; qg -= e * (R(1) - fsn); qv += e; T -= R(LSC / CPD) * e;
            }
            R qi0 = qi, qcl = qc + qi, dsum = R(0);
            for (int it = 0; it < 3; it++) {
              R f = fIce(T);
              R qs_ = qvsat(T, p0, f);
              R Lh = mixv(R(LVC), R(LSC), f);
              R d = (qv - qs_) / (R(1) + Lh * Lh * qs_ / (R(CPD * RVC) * T * T));
              d = std::max(d, -qcl);
              qv -= d; qcl += d; T += Lh / R(CPD) * d; dsum += d;
            }
            R f = fIce(T);
            qi = f * qcl; qc = qcl - qi;
            T += R(LFC / CPD) * (qi - qi0 - f * dsum);
            th = T / pi0;
            R envDecay = R(0);
            if (hurOn()) {
              R dxh = xmx - S.hur4.x, dyh = xmy - S.hur4.y;
              envDecay = sstep(S.hur4.w, R(1.5) * S.hur4.w, std::sqrt(dxh * dxh + dyh * dyh)) / R(1800);
            }
            R keep = R(1) / (R(1) + R(2) * dt * spongeLat(xmx, xmy) + dt * envDecay);
            qc *= keep; qi *= keep; qr *= keep; qs *= keep; qg *= keep; nr *= keep;
            R* o1 = &Q1[0][qidx(ci, cj, ck) * 4];
            R* o2 = &Q2[0][qidx(ci, cj, ck) * 4];
            o1[0] = std::max(qv, R(0)); o1[1] = std::max(qc, R(0)); o1[2] = std::max(qi, R(0)); o1[3] = std::max(qr, R(0));
            o2[0] = std::max(qs, R(0)); o2[1] = std::max(qg, R(0)); o2[2] = thm ? std::max(nr, R(0)) : q2[2]; o2[3] = q2[3];
            o[3] = th;
          }
          R sp = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
          if (sp > S.misc.x) { R s = S.misc.x / sp; o[0] *= s; o[1] *= s; o[2] *= s; }
          if (!(o[0] == o[0]) || !(o[1] == o[1]) || !(o[2] == o[2]) || !(o[3] == o[3])) {
            o[0] = bsB(ck)[2]; o[1] = bsB(ck)[3]; o[2] = R(0); o[3] = bsA(ck)[0];
          }
          R* out = &Vout[vidx(ci, cj, ck) * 4];
          for (int c = 0; c < 4; c++) out[c] = o[c];
        }
  }

  // ---- WGSL_M_DIV (model.js:909-925) ----
  void k_div(const std::vector<R>& Vin) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          const R* p = ldV(Vin, i, j, k);
          R rc = bsA(k)[2];
          R wt = k == nz - 1 ? R(0) : ldV(Vin, i, j, k + 1)[2];
          R wb = k == 0 ? R(0) : p[2];
          R d = rc * (ldV(Vin, i + 1, j, k)[0] - p[0] + ldV(Vin, i, j + 1, k)[1] - p[1]) / DXS() + (rhoW(k + 1) * wt - rhoW(k) * wb) / DZS();
          rhs[pidx(i, j, k)] = d / DTS();
        }
  }
  // ---- WGSL_M_PROJ (model.js:927-946) ----
  void k_proj(const std::vector<R>& Vin, std::vector<R>& Vout) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= nz; k++)
      for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
          auto Pf = [&](int a, int b, int c) {
            return phi[pidx(clampi(a, -pad, nx + pad - 1), clampi(b, -pad, ny + pad - 1), clampi(c, 0, nz - 1))];
          };
          const R* V = ldV(Vin, i, j, k);
          R o[4] = {V[0], V[1], V[2], V[3]};
          R kx = DTS() / DXS(), kz = DTS() / DZS();
          if (j < ny && k < nz) o[0] = V[0] - kx * (Pf(i, j, k) - Pf(i - 1, j, k));
          if (i < nx && k < nz) o[1] = V[1] - kx * (Pf(i, j, k) - Pf(i, j - 1, k));
          if (i < nx && j < ny && k > 0 && k < nz) o[2] = V[2] - kz * (Pf(i, j, k) - Pf(i, j, k - 1));
          else o[2] = R(0);
          R* out = &Vout[vidx(i, j, k) * 4];
          for (int c = 0; c < 4; c++) out[c] = o[c];
        }
  }

  // accumulated surface precipitation: rho(0) * sum_x q_x vt_x at the lowest level, x dt. No counterpart in the
  // reference; the fall speeds are those the scalar advection uses (model.js:487).
  void k_rain(double dt) {
    const R rho = bsA(0)[2];
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const R* q1 = &Q1[0][qidx(i, j, 0) * 4];
        const R* q2 = &Q2[0][qidx(i, j, 0) * 4];
        R fr, fn;
        vtRain(q1[3], q2[2], rho, fr, fn);
        double flux = double(rho) * (double(q1[3]) * double(fr) + double(q2[0]) * double(vtS(q2[0], rho)) + double(q2[1]) * double(vtGrau(q2[1], rho)));
        rain[size_t(j) * nx + i] += flux * dt;
      }
  }

  // ---- WGSL_M_FILT (model.js:948-994): the 2-dx filter of hurricane mode, into V[1-parity], Q1[1], Q2[1] ----
  void k_filt(const std::vector<R>& Vin, std::vector<R>& Vout) {
    const R a = S.hur5.z;
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= nz; k++)
      for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
          auto bih = [&](auto ld, int c) {
            return R(20) * ld(i, j, c) - R(8) * (ld(i + 1, j, c) + ld(i - 1, j, c) + ld(i, j + 1, c) + ld(i, j - 1, c)) +
                   R(2) * (ld(i + 1, j + 1, c) + ld(i + 1, j - 1, c) + ld(i - 1, j + 1, c) + ld(i - 1, j - 1, c)) + ld(i + 2, j, c) +
                   ld(i - 2, j, c) + ld(i, j + 2, c) + ld(i, j - 2, c);
          };
          R* o = &Vout[vidx(i, j, k) * 4];
          for (int c = 0; c < 4; c++) {
            auto ldv = [&](int a_, int b_, int c_) { return ldV(Vin, a_, b_, k)[c_]; };
            o[c] = ldV(Vin, i, j, k)[c] - a * bih(ldv, c);
          }
          if (k == 0 || k >= nz) o[2] = R(0);
          if (i < nx && j < ny && k < nz) {
            R* o1 = &Q1[1][qidx(i, j, k) * 4];
            R* o2 = &Q2[1][qidx(i, j, k) * 4];
            for (int c = 0; c < 4; c++) {
              auto ld1 = [&](int a_, int b_, int c_) { return ldQ(Q1[0], a_, b_, k)[c_]; };
              auto ld2 = [&](int a_, int b_, int c_) { return ldQ(Q2[0], a_, b_, k)[c_]; };
              o1[c] = std::max(ldQ(Q1[0], i, j, k)[c] - a * bih(ld1, c), R(0));
              o2[c] = std::max(ldQ(Q2[0], i, j, k)[c] - a * bih(ld2, c), R(0));
            }
          }
        }
  }
  // ---- WGSL_M_PREP (model.js:996-1026): the winds the advection carries, with cn.x of the last pressure force ----
  void k_prep(const std::vector<R>& Vin) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= nz; k++)
      for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
          auto Pf = [&](int a, int b, int c) {
            return phi[pidx(clampi(a, -pad, nx + pad - 1), clampi(b, -pad, ny + pad - 1), clampi(c, 0, nz - 1))];
          };
          const R* V = ldV(Vin, i, j, k);
          R o[4] = {V[0], V[1], V[2], V[3]};
          R f = S.cn.x * S.cn.y;
          R kx = f * DTS() / DXS(), kz = f * DTS() / DZS();
          if (j < ny && k < nz) o[0] = V[0] - kx * (Pf(i, j, k) - Pf(i - 1, j, k));
          if (i < nx && k < nz) o[1] = V[1] - kx * (Pf(i, j, k) - Pf(i, j - 1, k));
          if (i < nx && j < ny && k > 0 && k < nz) o[2] = V[2] - kz * (Pf(i, j, k) - Pf(i, j, k - 1));
          R* out = &Vp[vidx(i, j, k) * 4];
          for (int c = 0; c < 4; c++) out[c] = o[c];
        }
  }

  // ---- RegionalModel.reset / encStep (model.js:1427-1476) ----
  void reset() {
    time = 0; steps = 0; parity = 0; phiScale = 1;
    write_uniforms(1);
    k_lsf();
    k_init();
    std::fill(phi.begin(), phi.end(), R(0));
    std::fill(rhs.begin(), rhs.end(), R(0));
    V[1] = V[0];
    lsfT = 0;
    std::fill(rain.begin(), rain.end(), 0.0);
  }
  void step(double dt) {
    write_uniforms(dt);
    std::vector<R>& Vc = V[parity];
    std::vector<R>& Vn = V[1 - parity];
    if (hur_on && filtNow) {  // every 4th step: state -> scratch -> back (model.js:1448-1455)
      k_filt(Vc, Vn);
      Vc = Vn;
      Q1[0] = Q1[1];
      Q2[0] = Q2[1];
    }
    if (hur_on) k_prep(Vc);
    const std::vector<R>& Vval = hur_on ? Vp : Vc;
    trajV = &Vc;
    if (time - lsfT >= 60 || time == 0) { k_lsf(); lsfT = time; }
    k_ci();
    k_nut(Vc, Q1[0]);
    k_advv1(Vc, Vval);
    k_advv2(Vc, Vval, Vn);
    k_advq1(Vc);
    k_advq2(Vc);
    k_phys(Vn, Vc);
    k_div(Vc);
    solver.solve(rhs.data(), phi.data());
    k_proj(Vc, Vn);
    k_rain(dt);
    parity = 1 - parity;
    time += dt;
    steps++;
    phiScale = cnNow ? 1 / (1 - double(H.cnOld)) : 1;
  }
  // setSurface (model.js:1296-1303): surf nx*ny*4 (land fraction, SST K, 0, 0) or null; hur null = outbreak mode
  void set_surface(const float* surf, const ObHurricane* h) {
    for (size_t i = 0; i < sfc.size(); i++) sfc[i] = surf ? R(surf[i]) : R(0);
    hur_on = h != nullptr;
    if (h) H = *h;
    if (hur_on) Vp.assign(V[0].size(), R(0));
    else Vp.clear();
  }
  // setVortex's table (model.js:1318-1365, built on the host): nz x nr x 4; nr = 0 clears it
  void set_vortex(const float* tab, int nr, double x, double y, double dr, double moistR, double moistRH) {
    vortex = nr > 0 && tab;
    vx_nr = nr; vx_x = x; vx_y = y; vx_dr = dr; vx_moistR = moistR; vx_moistRH = moistRH;
    vx.assign(vortex ? size_t(nz) * nr * 4 : 0, R(0));
    for (size_t i = 0; i < vx.size(); i++) vx[i] = R(tab[i]);
  }

  // ---- WGSL_M_MAP (model.js:1028-1100) ----
  void maps(float* out) {
    // the uniforms of the last step; in hurricane mode they carry that step's pressure factors (cn), which a rewrite
    // after the step would change
    if (!hur_on) write_uniforms(S.step.x);
    const std::vector<R>& Vin = V[parity];
    const size_t n2 = size_t(nx) * ny;
    auto cvel = [&](int i, int j, int k, R v[3]) { cellVel(Vin, i, j, k, v); };
    auto dbz = [&](int i, int j, int k) {
      const R* q1 = &Q1[0][qidx(i, j, k) * 4];
      const R* q2 = &Q2[0][qidx(i, j, k) * 4];
      R rho = bsA(k)[2];
      R T = ldV(Vin, i, j, k)[3] * bsB(k)[0];
      R Zr = zRain(q1[3], q2[2], rho);
      R Zs = R(9.80e8) * std::pow(std::max(rho * q2[0], R(0)), R(1.75)) * R(0.224) * R(4);
      R Zg = zGrau(q2[1], rho, T);
      R Z = Zr + Zs + Zg;
      return Z > R(1e-3) ? R(10) * std::log(Z) / R(2.302585) : R(-30);
    };
    auto zeta = [&](int i, int j, int k) {
      R a[3], b[3], c[3], d[3];
      cvel(i + 1, j, k, a); cvel(i - 1, j, k, b); cvel(i, j + 1, k, c); cvel(i, j - 1, k, d);
      return (a[1] - b[1] - c[0] + d[0]) / (R(2) * DXS());
    };
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        R dzv = DZS();
        R comp = R(-30), wmx = R(0), uh = R(0);
        int k12 = std::min(int(R(12000) / dzv), nz - 1);
        for (int k = 0; k < k12; k++) {
          R v[3];
          cvel(i, j, k, v);
          R w = v[2];
          wmx = std::max(wmx, w);
          comp = std::max(comp, dbz(i, j, k));
          R z = (R(k) + R(0.5)) * dzv;
          if (z > R(2000) && z < R(5000) && w > R(0)) uh += w * std::max(zeta(i, j, k), R(0)) * dzv;
        }
        int k1 = clampi(int(R(1000) / dzv), 1, nz - 2);
        R v0[3], v1[3];
        cvel(i, j, 0, v0);
        R conv = -((ldV(Vin, i + 1, j, 0)[0] - ldV(Vin, i, j, 0)[0] + ldV(Vin, i, j + 1, 0)[1] - ldV(Vin, i, j, 0)[1]) / DXS()) * R(1000);
        size_t idx = size_t(j) * nx + i;
        float* m0 = out + idx * 4;
        m0[0] = float(comp); m0[1] = float(dbz(i, j, k1)); m0[2] = float(ldV(Vin, i, j, 0)[3] - bsA(0)[0]); m0[3] = float(zeta(i, j, k1));
        float* m1 = out + (idx + n2) * 4;
        m1[0] = float(wmx); m1[1] = float(uh); m1[2] = float(conv); m1[3] = float(std::sqrt(v0[0] * v0[0] + v0[1] * v0[1]));
        cvel(i, j, k1, v1);
        float* m2 = out + (idx + 2 * n2) * 4;
        m2[0] = float(v0[0]); m2[1] = float(v0[1]); m2[2] = float(v1[0]); m2[3] = float(v1[1]);
        R tr = R(1), bt = R(0);
        for (int k = nz - 1; k >= 0; k--) {
          const R* q1 = &Q1[0][qidx(i, j, k) * 4];
          const R* q2 = &Q2[0][qidx(i, j, k) * 4];
          R dtau = (R(80) * q1[1] + R(60) * q1[2] + R(25) * q2[0] + R(4) * q2[1] + R(1) * q1[3]) * bsA(k)[2] * dzv;
          R a = R(1) - std::exp(-dtau);
          bt += tr * a * ldV(Vin, i, j, k)[3] * bsB(k)[0];
          tr *= R(1) - a;
          if (tr < R(1e-3)) break;
        }
        R sst = sfc[idx * 4 + 1];
        bt += tr * (sst > R(200) ? sst : ldV(Vin, i, j, 0)[3] * bsB(0)[0]);
        R ps = bsA(0)[2] * S.cn.z * phi[(i + pad) + nxp * (j + pad)] / R(100);
        int k5 = clampi(int(R(5000) / dzv), 1, nz - 2);
        float* m3 = out + (idx + 3 * n2) * 4;
        m3[0] = float(ps); m3[1] = float(bt); m3[2] = float(S.hur2.w * std::sqrt(v0[0] * v0[0] + v0[1] * v0[1])); m3[3] = float(zeta(i, j, k5));
      }
  }

  // field access in the texel layouts of ob.h
  std::vector<R>* field_vec(int f, int& ch) {
    switch (f) {
      case OB_FIELD_V: ch = 4; return &V[parity];
      case OB_FIELD_Q1: ch = 4; return &Q1[0];
      case OB_FIELD_Q2: ch = 4; return &Q2[0];
      case OB_FIELD_AUX: ch = 2; return &aux;
      case OB_FIELD_PHI: ch = 1; return &phi;
      case OB_FIELD_LSF_A: ch = 4; return &lsfA;
      case OB_FIELD_LSF_B: ch = 4; return &lsfB;
      case OB_FIELD_CI_MAP: ch = 4; return &ciMap;
      case OB_FIELD_PHT: ch = 1; return &phT;
      default: return nullptr;
    }
  }
};


// ---------------------------------------------------------------------------------------------------------------
// Virtual radar (radar.js:41-268): WGSL_R_CUT's gate moments and Level II codes, WGSL_R_PHI's sequential PhiDP.
// U is the cut's uniform block (radar.js:36-39, 11 vec4 = 44 floats, the layout of ObRadarCut in ob.h):
//   site, geo, cut, gates, nyq, offA, offB, mdl, mdl2, phys, phys2.
// Sampling uses the model's current state V[parity], Q1/Q2 slot 0 and aux, as RadarSim.makeBind binds them
// (radar.js:331-336); textureSampleLevel with normalised coordinates becomes a texel-unit lerp (texel i at x = i).
// ---------------------------------------------------------------------------------------------------------------
template <class R> struct RadarCut {
  const Model<R>& M;
  R U[44];
  const float* tor;
  explicit RadarCut(const Model<R>& m, const float* u, const float* t) : M(m), tor(t) {
    for (int i = 0; i < 44; i++) U[i] = R(u[i]);
  }
  R u(int v, int c) const { return U[v * 4 + c]; }  // vec4 v, component c
  enum { SITE, GEO, CUT, GATES, NYQ, OFFA, OFFB, MDL, MDL2, PHYS, PHYS2 };
  static R sq(R x) { return x * x; }
  static R db2lin(R d) { return std::pow(R(10), R(0.1) * d); }
  // great-circle destination (bearing a, ground distance s) -> model metres (radar.js:51-64)
  void gatePos(R a, R s, R& x, R& y) const {
    const R RE = R(6371000.0);
    R p1 = u(GEO, 2), l1 = u(GEO, 3), d = s / RE;
    R sp2 = std::sin(p1) * std::cos(d) + std::cos(p1) * std::sin(d) * std::cos(a);
    R p2 = std::asin(clampv(sp2, R(-1), R(1)));
    R l2 = l1 + std::atan2(std::sin(a) * std::sin(d) * std::cos(p1), std::cos(d) - std::sin(p1) * sp2);
    R p0 = u(GEO, 0), dl = l2 - u(GEO, 1);
    R cc = clampv(std::sin(p0) * std::sin(p2) + std::cos(p0) * std::cos(p2) * std::cos(dl), R(-1), R(1));
    R c = std::acos(cc);
    R k = c < R(1e-6) ? R(1) : c / std::sin(c);
    x = RE * k * std::cos(p2) * std::sin(dl) - u(MDL2, 2);
    y = RE * k * (std::cos(p0) * std::sin(p2) - std::sin(p0) * std::cos(p2) * std::cos(dl)) - u(MDL2, 3);
  }
  // 4/3-earth beam: height above the antenna and ground distance at slant range r (radar.js:66-72)
  void beam(R r, R el, R& h, R& s) const {
    R a = u(SITE, 3);
    R q = r * r + R(2) * r * a * std::sin(el);
    h = q / (std::sqrt(q + a * a) + a);
    s = a * std::asin(clampv(r * std::cos(el) / (a + h), R(-1), R(1)));
  }
  struct Smp { R zr, zs, zg, vt, u[3], T, qr, rho, nu, inside, lr; };
  // radar.js:89-139
  Smp sample(R px, R py, R z) const {
    Smp o{};
    const R n[3] = {u(MDL, 0), u(MDL, 1), u(MDL, 2)};
    const R dx = u(MDL, 3), dz = u(MDL2, 0);
    const R g[3] = {px / dx, py / dx, z / dz};
    o.inside = (g[0] >= 0 && g[1] >= 0 && g[2] >= 0 && g[0] <= n[0] && g[1] <= n[1] && g[2] <= n[2] && z >= 0) ? R(1) : R(0);
    R gc[3];
    for (int c = 0; c < 3; c++) gc[c] = clampv(g[c], R(0), n[c]);
    const std::vector<R>& Vs = M.V[M.parity];
    auto q1 = [&](int ch) { return M.sampleQ(M.Q1[0], gc[0] - R(0.5), gc[1] - R(0.5), gc[2] - R(0.5), ch); };
    auto q2 = [&](int ch) { return M.sampleQ(M.Q2[0], gc[0] - R(0.5), gc[1] - R(0.5), gc[2] - R(0.5), ch); };
    const R uu = M.sampleV(Vs, gc[0], gc[1] - R(0.5), gc[2] - R(0.5), 0);
    const R vv = M.sampleV(Vs, gc[0] - R(0.5), gc[1], gc[2] - R(0.5), 1);
    const R ww = M.sampleV(Vs, gc[0] - R(0.5), gc[1] - R(0.5), gc[2], 2);
    const R th = M.sampleV(Vs, gc[0] - R(0.5), gc[1] - R(0.5), gc[2] - R(0.5), 3);
    const int k = int(clampv(std::floor(gc[2]), R(0), n[2] - R(1)));
    const R* A = M.bsA(k);
    const R* B = M.bsB(k);
    const R rho = A[2], T = th * B[0];
    const R qr = std::max(q1(3), R(0)), qs = std::max(q2(0), R(0)), qg = std::max(q2(1), R(0));
    o.zr = R(3.63e9) * std::pow(rho * qr, R(1.75));
    o.zs = R(9.80e8) * std::pow(rho * qs, R(1.75)) * R(0.224) * R(4.0);
    o.zg = (T < R(273.15) ? R(1.2e10) : R(4.33e10)) * std::pow(rho * qg, R(1.75));
    const R sqv = std::sqrt(u(PHYS, 0) / rho);
    R vr = std::min(R(36.34) * std::pow(std::max(R(0.001) * rho * qr, R(0)), R(0.1364)) * sqv, R(10) * sqv);
    const R vs = clampv(R(1.1) * std::pow(std::max(R(1000) * rho * qs, R(1e-6)), R(0.11)), R(0.3), R(2.2)) * sqv;
    R vg = clampv(R(9) * std::pow(std::max(R(1000) * rho * qg, R(1e-6)), R(0.42)), R(1), R(55)) * sqv;
    const R rr = qg / R(0.009);
    vg = std::min(vg * (R(1) + rr * rr), R(65));
    if (u(PHYS2, 0) > R(0.5) && u(PHYS, 2) < R(0.5)) {
      o.zg = (T < R(273.15) ? R(1.3e9) : R(1.0e10)) * std::pow(rho * qg, R(1.75));
      vg = clampv(R(5) * std::pow(std::max(R(1000) * rho * qg, R(1e-6)), R(0.25)), R(1), R(9)) * sqv;
    }
    o.lr = std::pow(R(3.14159 * 1000.0 * 8e6) / std::max(rho * qr, R(1e-9)), R(0.25));
    if (u(PHYS, 2) > R(0.5)) {
      const R nr = std::max(q2(2), R(0));
      if (qr > R(1e-9)) {
        const R l = clampv(std::pow(R(3.14159 * 1000.0) * std::max(nr, R(1e-3)) / qr, R(0.33333)), R(1000), R(1.0e5));
        const R nb = qr * l * l * l / R(3141.59);
        o.zr = R(720e18) * rho * nb / std::pow(l, R(6));
        o.lr = l;
        vr = std::min(R(3949) * std::pow(l, R(-0.8)), R(10)) * sqv;
      } else {
        o.zr = R(0);
      }
      if (qg > R(1e-9)) {
        const R n0 = clampv(R(200) / (rho * qg), R(1e4), R(3e6));
        const R l = std::pow(R(3.14159 * 500.0) * n0 / (rho * qg), R(0.25));
        o.zg = R(720e18) * n0 / std::pow(l, R(7)) * (T < R(273.15) ? R(0.0666) : R(0.24));
        vg = std::min(R(2483) * std::pow(l, R(-0.89)), R(30)) * sqv;
      } else {
        o.zg = R(0);
      }
    }
    const R zt = o.zr + o.zs + o.zg;
    o.vt = zt > R(1e-6) ? (o.zr * vr + o.zs * vs + o.zg * vg) / zt : R(0);
    o.u[0] = uu; o.u[1] = vv; o.u[2] = ww;
    o.T = T; o.qr = qr; o.rho = rho;
    o.nu = M.sample(M.aux, M.nx, M.ny, M.nz, gc[0] - R(0.5), gc[1] - R(0.5), gc[2] - R(0.5), 0, 2);
    return o;
  }
  // WGSL code(): u32(clamp(round(v*sc + ofs), 2, 255)); WGSL round is half-to-even
  static uint32_t code(R v, R sc, R ofs) {
    R t = std::nearbyint(v * sc + ofs);
    return uint32_t(clampv(t, R(2), R(255)));
  }
  // one gate (radar.js:144-227). mom = (dBZ, Vr, SW, ZDR, rho_hv, KDP), NaN where the gate or moment is empty.
  void gate(int ri, int gi, uint8_t cd[5], R& kdp, R mom[6]) const {
    for (int i = 0; i < 5; i++) cd[i] = 0;
    kdp = R(-1);
    for (int i = 0; i < 6; i++) mom[i] = std::numeric_limits<R>::quiet_NaN();
    const R r = u(GATES, 2) + u(GATES, 3) * R(gi);
    const R el = u(CUT, 0);
    const R az = (u(CUT, 1) + u(CUT, 2) * R(ri)) * R(0.017453293);
    const R bw = R(0.0165);
    R hch, hcs;
    beam(r, el, hch, hcs);
    R px, py, qx, qy;
    gatePos(az, hcs, px, py);
    gatePos(az, hcs + R(200), qx, qy);
    R ex = qx - px, ey = qy - py;
    const R el_ = std::sqrt(ex * ex + ey * ey);
    ex /= el_; ey /= el_;
    const R zAnt = u(SITE, 2) - u(MDL2, 1);
    const R zc = zAnt + hch;
    if (zc > u(MDL, 2) * u(MDL2, 0) - R(200)) return;
    R hl, hu, tmp;
    beam(r, el - R(0.4) * bw, hl, tmp);
    beam(r, el + R(0.4) * bw, hu, tmp);
    hl += zAnt; hu += zAnt;
    const Smp s0 = sample(px, py, std::max(zc, R(5))), s1 = sample(px, py, std::max(hl, R(5))), s2 = sample(px, py, std::max(hu, R(5)));
    if (s0.inside < R(0.5)) return;
    const R zr = R(0.5) * s0.zr + R(0.25) * (s1.zr + s2.zr), zs = R(0.5) * s0.zs + R(0.25) * (s1.zs + s2.zs);
    const R zg = R(0.5) * s0.zg + R(0.25) * (s1.zg + s2.zg);
    const R zmet = zr + zs + zg;
    R zdeb = 0, dvx = 0, dvy = 0, swt = 0;
    const R bwm = R(0.5) * r * bw;
    const int ntor = int(u(PHYS, 3));
    for (int q = 0; q < ntor; q++) {
      const float* A = tor + 8 * q;
      const float* B = A + 4;
      const R dxv = px - R(A[0]), dyv = py - R(A[1]);
      const R rt = std::sqrt(dxv * dxv + dyv * dyv);
      const R Re = std::sqrt(R(A[2]) * R(A[2]) + bwm * bwm + R(125.0 * 125.0));
      if (rt > R(8) * Re) continue;
      const R vmx = R(A[3]) * R(A[2]) / Re;
      const R vt = vmx * (rt < Re ? rt / Re : Re / std::max(rt, R(1)));
      const R etx = -dyv / std::max(rt, R(1)), ety = dxv / std::max(rt, R(1));
      const R erx = dxv / std::max(rt, R(1)), ery = dyv / std::max(rt, R(1));
      const R fz = R(1) - sstep(R(1200), R(3500), zc);
      dvx += (vt * etx - R(0.25) * vt * erx) * fz;
      dvy += (vt * ety - R(0.25) * vt * ery) * fz;
      swt = std::max(swt, vmx * R(0.4) * std::exp(-rt * rt / (R(4) * Re * Re)) * fz);
      if (B[2] > 0.f && zc < R(B[0])) {
        const R rd = std::max(R(1.4) * R(A[2]), R(150));
        zdeb += db2lin(R(B[1])) * std::min(R(1), rd * rd / (Re * Re)) * std::exp(-rt * rt / (Re * Re)) *
                (R(1) - sstep(R(0.55) * R(B[0]), R(B[0]), zc)) * R(B[2]);
      }
    }
    const R ztot = zmet + zdeb;
    if (ztot <= R(1e-6)) return;
    const R dbz = R(10) * std::log(ztot) / R(2.302585);
    if (dbz < u(PHYS, 1)) return;
    mom[0] = dbz;
    cd[0] = uint8_t(code(dbz, R(2), R(66)));
    if (gi >= int(u(GATES, 1))) return;
    const R ce = std::cos(el), se = std::sin(el);
    const R vtf = s0.vt * zmet / ztot;
    R vr = ((s0.u[0] + dvx) * ex + (s0.u[1] + dvy) * ey) * ce + (s0.u[2] - vtf) * se;
    const R nyq = u(NYQ, 0);
    vr = vr - R(2) * nyq * std::floor((vr + nyq) / (R(2) * nyq));
    mom[1] = vr;
    cd[1] = uint8_t(code(vr, R(2), R(129)));
    const R vru = (s2.u[0] * ex + s2.u[1] * ey) * ce, vrl = (s1.u[0] * ex + s1.u[1] * ey) * ce;
    const R swv = std::sqrt(R(1) + sq(clampv(R(2.5) * std::sqrt(std::max(s0.nu, R(0)) / R(1000)), R(0), R(8))) +
                            sq((vru - vrl) / R(2.5)) + sq(R(0.15) * s0.vt * se) + sq(swt));
    mom[2] = std::min(swv, R(19.5));
    cd[2] = uint8_t(code(mom[2], R(2), R(129)));
    const R d0 = R(3.67) / s0.lr * R(1000);
    const bool melt = s0.T > R(273.15);
    const R zdrR = clampv(R(0.2) + R(1.15) * (d0 - R(0.5)), R(0.1), R(4.8));
    const R zdrS = melt ? R(1.3) : R(0.3);
    const R zdrG = melt ? (zg > R(3.2e5) ? R(0) : R(0.7)) : R(0.15);
    const R zv = zr / db2lin(zdrR) + zs / db2lin(zdrS) + zg / db2lin(zdrG) + zdeb / db2lin(R(0.2));
    const R zdr = R(10) * std::log(std::max(ztot, R(1e-9)) / std::max(zv, R(1e-9))) / R(2.302585);
    mom[3] = clampv(zdr, R(-7.9), R(7.9));
    cd[3] = uint8_t(code(mom[3], R(16), R(128)));
    const R fr = zr / ztot, fs = zs / ztot, fg = zg / ztot, fd = zdeb / ztot;
    R cc = fr * (d0 > R(2.5) ? R(0.986) : R(0.995)) + fs * (melt ? R(0.93) : R(0.985)) +
           fg * (melt ? (zg > R(3.2e5) ? R(0.90) : R(0.94)) : R(0.985)) + fd * R(0.55);
    cc -= R(0.24) * fr * fg;
    mom[4] = clampv(cc, R(0.2), R(1.05));
    cd[4] = uint8_t(code(mom[4], R(300), R(-60.5)));
    kdp = std::pow(R(0.017) * std::pow(std::max(zr, R(0)), R(0.714)) / R(44), R(1.2165));
    mom[5] = kdp;
  }
  // WGSL_R_CUT main (radar.js:229-240) over every radial, then WGSL_R_PHI (radar.js:243-268). out = the volume's
  // bytes (codes stored little-endian, 4 per u32 word as the reference packs them); kdp = nrad*ngDop scratch;
  // mom (optional) = nrad*ngRef*6 moments.
  void run(uint8_t* out, R* kdp, R* mom) const {
    const int nrad = int(u(CUT, 3)), ngR = int(u(GATES, 0)), ngD = int(u(GATES, 1));
    const uint32_t mask = uint32_t(u(OFFB, 3));
    const size_t oR = size_t(u(OFFA, 0)) * 4, oV = size_t(u(OFFA, 1)) * 4, oS = size_t(u(OFFA, 2)) * 4,
                 oZ = size_t(u(OFFA, 3)) * 4, oP = size_t(u(OFFB, 0)) * 4, oH = size_t(u(OFFB, 1)) * 4;
#pragma omp parallel for schedule(dynamic, 4)
    for (int ri = 0; ri < nrad; ri++)
      for (int gi = 0; gi < ngR; gi++) {
        uint8_t cd[5];
        R kd, m6[6];
        gate(ri, gi, cd, kd, m6);
        out[oR + size_t(ri) * ngR + gi] = cd[0];
        if (gi < ngD) {
          const size_t o = size_t(ri) * ngD + gi;
          if (mask & 2u) out[oV + o] = cd[1];
          if (mask & 4u) out[oS + o] = cd[2];
          if (mask & 8u) out[oZ + o] = cd[3];
          if (mask & 32u) out[oH + o] = cd[4];
          kdp[o] = kd;
        }
        if (mom)
          for (int c = 0; c < 6; c++) mom[(size_t(ri) * ngR + gi) * 6 + c] = m6[c];
      }
    if (mask & 16u) phi(out + oP, kdp, nrad, ngD);
  }
  // WGSL_R_PHI: fp32 accumulation in gate order, 2 * KDP * dr (km), mod 360 (radar.js:251-264)
  void phi(uint8_t* out, const R* kdp, int nrad, int ng) const {
    for (int ri = 0; ri < nrad; ri++) {
      R acc = u(NYQ, 3);
      for (int gi = 0; gi < (ng / 4) * 4; gi++) {
        const R kd = kdp[size_t(ri) * ng + gi];
        uint8_t c = 0;
        if (kd >= R(0)) {
          acc += R(2) * kd * u(GATES, 3) * R(0.001);
          const R ph = acc - R(360) * std::floor(acc / R(360));
          c = uint8_t(clampv(std::nearbyint(ph * R(253) / R(360) + R(2)), R(2), R(255)));
        }
        out[size_t(ri) * ng + gi] = c;
      }
    }
  }
};

}  // namespace oro

// ---------------------------------------------------------------------------------------------------------------
// C entry points for the tests (ctypes). The ObParams defaults mirror the library's ob_params_default.
// ---------------------------------------------------------------------------------------------------------------
extern "C" {

void ob_params_default(ObParams* p) {
  // model.js:1176-1180, with the outbreak overrides of app.js:1613
  p->cs = 0.18f; p->nu0 = 1.0f; p->drag = 1.0f; p->z0 = 0.1f;
  p->spongeW = 36000.f; p->spongeTau = 100.f; p->dampZ = 15000.f; p->dampTau = 150.f;
  p->autoc = 1e-3f; p->qc0 = 2e-3f; p->freeze = 1.0f; p->noise = 0.25f;
  p->mc = 1.0f; p->vcap = 110.f; p->evap = 0.22f; p->sortQ = 5e-4f;
  p->ciRate = 0.5f; p->nudgeTau = 5400.f; p->lat = 35.f; p->moistMix = 0.f;
  p->mcFloor = 0.25f; p->scheme = 0.f; p->evapT = 0.3f; p->dtScale = 1.0f;
}
void ob_hurricane_default(ObHurricane* h) {
  // app.js:1631 and the writeUniforms defaults (model.js:1402-1420); centre at the origin, sfcP for 1000 hPa
  h->ck = 1.3e-3f; h->landMoist = 0.3f; h->sfcP = 100000.f; h->tauRad = 43200.f; h->radCap = 2.f / 86400.f;
  h->blDepth = 1000.f; h->u10f = 0.8f; h->gust = 1.5f; h->thermals = 0.4f / 300.f; h->thermalScale = 1.f;
  h->maritime = 1.f; h->filter4 = 0.003f; h->cdCap = 2.0e-3f; h->dissHeat = 1.f; h->centreX = 0.f; h->centreY = 0.f;
  h->thermalR = 200000.f; h->envR = 300000.f; h->cnOld = 0.4f; h->traj2 = 1.f;
}
int ob_grid_pad(float dx) {  // model.js:1122
  double v = std::round(10000.0 / dx / 8.0) * 8.0;
  return int(std::min(std::max(v, 8.0), 64.0));
}

struct OroModel {
  int prec;
  oro::Model<float>* f;
  oro::Model<double>* d;
};

OroModel* oro_create(int nx, int ny, int nz, double dx, int precision) {
  OroModel* m = new OroModel{precision, nullptr, nullptr};
  if (precision == 8) { m->d = new oro::Model<double>(); m->d->create(nx, ny, nz, dx); }
  else { m->f = new oro::Model<float>(); m->f->create(nx, ny, nz, dx); }
  return m;
}
void oro_destroy(OroModel* m) { delete m->f; delete m->d; delete m; }

#define ORO_BOTH(...) do { if (m->f) { auto& M = *m->f; __VA_ARGS__; } else { auto& M = *m->d; __VA_ARGS__; } } while (0)

void oro_set_base_state(OroModel* m, const float* B) { ORO_BOTH(M.set_base_state(B)); }
void oro_set_params(OroModel* m, const ObParams* p) {
  ORO_BOTH({ float sw = M.P.spongeW; M.P = *p; M.P.spongeW = sw; });
}
void oro_set_boundaries(OroModel* m, const float* packed, int n) {
  ORO_BOTH({
    M.nb = std::min(n, OB_MAX_BOUNDS);
    std::fill(M.bnd.begin(), M.bnd.end(), 0.f);
    if (M.nb > 0) std::memcpy(M.bnd.data(), packed, sizeof(float) * M.nb * OB_BOUNDARY_FLOATS);
  });
}
void oro_set_ci(OroModel* m, const float* ev, int n) {
  ORO_BOTH({
    M.nci = std::min(n, OB_MAX_CI);
    M.ciev.assign(size_t(std::max(1, M.nci)) * OB_CI_FLOATS, 0.f);
    if (M.nci > 0) std::memcpy(M.ciev.data(), ev, sizeof(float) * M.nci * OB_CI_FLOATS);
  });
}
void oro_reset(OroModel* m) { ORO_BOTH(M.reset()); }
void oro_set_surface(OroModel* m, const float* surf, const ObHurricane* h) { ORO_BOTH(M.set_surface(surf, h)); }
void oro_set_vortex(OroModel* m, const float* tab, int nr, double x, double y, double dr, double moistR, double moistRH) {
  ORO_BOTH(M.set_vortex(tab, nr, x, y, dr, moistR, moistRH));
}
void oro_step(OroModel* m, double dt, int nsteps) { ORO_BOTH(for (int s = 0; s < nsteps; s++) M.step(dt)); }
double oro_time(OroModel* m) { double t = 0; ORO_BOTH(t = M.time); return t; }
int oro_parity(OroModel* m) { int p = 0; ORO_BOTH(p = M.parity); return p; }
void oro_maps(OroModel* m, float* out) { ORO_BOTH(M.maps(out)); }
// float32 copy of a field (texel layout)
int oro_get_field(OroModel* m, int field, float* out, size_t count) {
  int rc = -1;
  ORO_BOTH({
    int ch = 0;
    auto* v = M.field_vec(field, ch);
    if (v && v->size() == count) { for (size_t i = 0; i < count; i++) out[i] = float((*v)[i]); rc = 0; }
  });
  return rc;
}
int oro_get_field_f64(OroModel* m, int field, double* out, size_t count) {
  int rc = -1;
  ORO_BOTH({
    int ch = 0;
    auto* v = M.field_vec(field, ch);
    if (v && v->size() == count) { for (size_t i = 0; i < count; i++) out[i] = double((*v)[i]); rc = 0; }
  });
  return rc;
}
int oro_set_field(OroModel* m, int field, const float* in, size_t count) {
  int rc = -1;
  ORO_BOTH({
    int ch = 0;
    auto* v = M.field_vec(field, ch);
    if (v && v->size() == count) { for (size_t i = 0; i < count; i++) (*v)[i] = in[i]; rc = 0; }
  });
  return rc;
}
void oro_rain(OroModel* m, double* out) { ORO_BOTH(std::memcpy(out, M.rain.data(), sizeof(double) * M.rain.size())); }
// state budgets: sum rho q_t dV, sum rho dV (FP64 sums)
void oro_budgets(OroModel* m, double* water, double* mass) {
  ORO_BOTH({
    double w = 0, ms = 0, dV = M.dx * M.dx * M.dz;
    for (int k = 0; k < M.nz; k++) {
      double rho = double(M.bsA(k)[2]);
      for (size_t c = 0; c < size_t(M.nx) * M.ny; c++) {
        size_t q = size_t(k) * M.nx * M.ny + c;
        const auto* q1 = &M.Q1[0][q * 4];
        const auto* q2 = &M.Q2[0][q * 4];
        w += rho * (double(q1[0]) + double(q1[1]) + double(q1[2]) + double(q1[3]) + double(q2[0]) + double(q2[1])) * dV;
        ms += rho * dV;
      }
    }
    *water = w; *mass = ms;
  });
}

// standalone pressure solve (solver.js): rhs, phi nx*ny*nz; rhoC[nz], rhoW[nz+1]
void oro_poisson_solve_f32(int nx, int ny, int nz, double dx, double dz, const float* rhoC, const float* rhoW, const float* rhs, float* phi) {
  oro::Poisson<float> P;
  P.init(nx, ny, nz, dx, dz);
  std::vector<double> rc(rhoC, rhoC + nz), rw(rhoW, rhoW + nz + 1);
  P.set_density(rc.data(), rw.data());
  P.solve(rhs, phi);
}
void oro_poisson_solve_f64(int nx, int ny, int nz, double dx, double dz, const double* rhoC, const double* rhoW, const double* rhs, double* phi) {
  oro::Poisson<double> P;
  P.init(nx, ny, nz, dx, dz);
  P.set_density(rhoC, rhoW);
  P.solve(rhs, phi);
}
// FP64 operator apply: out = rhoC(k) lap_h(phi) + d/dz(rhoW d phi/dz), phi = 0 outside x/y (antisymmetric ghosts),
// Neumann at the ground and the lid (the operator solver.js inverts, solver.js:1-9, 139-146)
void oro_poisson_apply_f64(int nx, int ny, int nz, double dx, double dz, const double* rhoC, const double* rhoW, const double* phi, double* out) {
  const double ix2 = 1.0 / (dx * dx), iz2 = 1.0 / (dz * dz);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        auto P = [&](int a, int b, int c) -> double {
          if (a < 0 || a >= nx || b < 0 || b >= ny) return -phi[(size_t(c) * ny + std::min(std::max(b, 0), ny - 1)) * nx + std::min(std::max(a, 0), nx - 1)];
          return phi[(size_t(c) * ny + b) * nx + a];
        };
        double p = phi[(size_t(k) * ny + j) * nx + i];
        double lh = (P(i + 1, j, k) + P(i - 1, j, k) + P(i, j + 1, k) + P(i, j - 1, k) - 4 * p) * ix2;
        double up = k < nz - 1 ? rhoW[k + 1] * (phi[(size_t(k + 1) * ny + j) * nx + i] - p) : 0.0;
        double lo = k > 0 ? rhoW[k] * (p - phi[(size_t(k - 1) * ny + j) * nx + i]) : 0.0;
        out[(size_t(k) * ny + j) * nx + i] = rhoC[k] * lh + (up - lo) * iz2;
      }
}

// one radar cut on the model's current state (radar.js:229-268); out = volume bytes, kdp = nrad*ngDop,
// mom = nrad*ngRef*6 (may be null); the FP64 model writes double moments into mom64 instead
void oro_radar_cut(OroModel* m, const float* U, const float* tor, uint8_t* out, float* kdp, float* mom) {
  oro::Model<float>& M = *m->f;
  oro::RadarCut<float> rc(M, U, tor);
  rc.run(out, kdp, mom);
}
void oro_radar_cut_f64(OroModel* m, const float* U, const float* tor, uint8_t* out, double* kdp, double* mom) {
  oro::Model<double>& M = *m->d;
  oro::RadarCut<double> rc(M, U, tor);
  rc.run(out, kdp, mom);
}
// WGSL code() and the PhiDP accumulation alone, for quantising given moments
uint32_t oro_radar_code(float v, float sc, float ofs) { return oro::RadarCut<float>::code(v, sc, ofs); }
void oro_radar_phi(const float* U, const float* kdp, int nrad, int ng, uint8_t* out) {
  oro::Model<float> dummy;
  oro::RadarCut<float> rc(dummy, U, nullptr);
  rc.phi(out, kdp, nrad, ng);
}

// helpers exposed for known-answer tests
uint32_t oro_pcg(uint32_t v) { return oro::pcg(v); }
uint32_t oro_hash3i(int x, int y, int z) { return oro::hash3i(x, y, z); }
float oro_gnoise2(float x, float y) { return oro::gnoise2<float>(x, y); }
void oro_dst_matrix(int N, double* q) {  // q[i*N + l] = v_l(i), solver.js:115-121
  for (int i = 0; i < N; i++)
    for (int l = 0; l < N; l++) q[size_t(i) * N + l] = std::sqrt((l == N - 1 ? 1.0 : 2.0) / N) * std::sin(M_PI * (l + 1) * (i + 0.5) / N);
}
}
