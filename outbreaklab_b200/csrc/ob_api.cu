// ob_api.cu — the C ABI of include/ob.h: model and solver handles, device memory, the per-step dispatch sequence.
//
// RegionalModel (model.js:1156-1496) restated as a C++ handle that owns one CUDA stream (the WebGPU queue) and all
// device memory of one domain. encStep's dispatch order (model.js:1457-1472) is kept; the ping-pong of V and the
// two Q slots follows model.js:1248-1266.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ob.h"
#include "ob_common.cuh"
#include "ob_mlp.cuh"
#include "ob_poisson.cuh"
#include "ob_radar.cuh"
#include "ob_step.cuh"

namespace ob {

static thread_local char g_err[1024] = "";
void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
static int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return OB_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? OB_ERR_OOM : OB_ERR_DEVICE;
}
#define OB_TRY(expr)              \
  do {                            \
    int rc__ = (expr);            \
    if (rc__ != OB_OK) return rc__; \
  } while (0)

// two timing events, destroyed on every return path of the function that holds them
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  int create() {
    OB_TRY(cuda_status(cudaEventCreate(&a), "event"));
    return cuda_status(cudaEventCreate(&b), "event");
  }
  // device time from a to b (waits for b)
  int elapsed(float* ms, const char* what) const {
    OB_TRY(cuda_status(cudaEventSynchronize(b), what));
    return cuda_status(cudaEventElapsedTime(ms, a, b), what);
  }
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// sum rho q_total dV and sum rho dV over the interior cells, and the accumulated surface rain, in FP64 and in a
// fixed order, so that the same state gives the same bits. Block b of k_budget takes rows (y, z) [R b / nb, R (b+1) /
// nb) and reads them four cells at a time (rows start 16-byte aligned: the pitch is a multiple of 32 floats); the
// block's sums go to part[2 b], part[2 b + 1]. Cells of a 32 x 4 brick whose hydrometeor flag (act, from the last
// physics pass or the flags rebuilt after a field write) is clear hold exactly zero condensate, so they add qv alone:
// q0 + 0 + 0 + 0 + 0 + 0 is q0, the same bits, from one array instead of six. k_sum_rain writes one partial per
// block the same way, and k_budget_final adds the partials in block order.
constexpr int kBudgetBlocks = 592;   // 4 blocks of 256 threads per SM of a 148-SM B200
constexpr int kRainBlocks = 296;  // 2 blocks of 256 threads per SM
constexpr int kRedDoubles = 8 + 2 * kBudgetBlocks + kRainBlocks;   // results, then the partials
__device__ __forceinline__ double block_sum(double v, double* sh) {   // fixed order: shuffle tree, then warps 0..7
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < int(blockDim.x >> 5); w++) t += sh[w];
  return t;
}
__global__ void __launch_bounds__(256) k_budget(Grid g, const float* __restrict__ B, float* const* q, const unsigned int* __restrict__ act,
                                                int nbx, int nby, double dV, double* __restrict__ part) {
  __shared__ double sh[8];
  const float* __restrict__ qc[6] = {q[0], q[1], q[2], q[3], q[4], q[5]};
  const int nrows = g.ny * g.nz, nc = (g.nx + 3) >> 2;
  const int r0 = int(long(nrows) * blockIdx.x / gridDim.x), r1 = int(long(nrows) * (blockIdx.x + 1) / gridDim.x);
  double w = 0.0;
  for (long t = threadIdx.x; t < long(r1 - r0) * nc; t += blockDim.x) {
    const int r = r0 + int(t / nc), i0 = int(t % nc) << 2;
    const int j = r % g.ny, k = r / g.ny;
    const int o = g.at(i0, j, k);
    const int nch = __ldg(act + (i0 >> 5) + nbx * ((j >> 2) + nby * k)) != 0u ? 6 : 1;
    double s = 0.0;
    if (i0 + 4 <= g.nx) {
      for (int c = 0; c < nch; c++) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(qc[c] + o));
        s += double(v.x) + double(v.y) + double(v.z) + double(v.w);
      }
    } else {
      for (int c = 0; c < nch; c++)
        for (int i = i0; i < g.nx; i++) s += double(__ldg(qc[c] + o + (i - i0)));
    }
    w += s * double(__ldg(B + k * 8 + 2));
  }
  double mass = 0.0;
  if (threadIdx.x == 0)
    for (int r = r0; r < r1; r++) mass += double(__ldg(B + (r / g.ny) * 8 + 2)) * g.nx;
  w = block_sum(w, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = w * dV;
    part[2 * blockIdx.x + 1] = mass * dV;
  }
}
__global__ void __launch_bounds__(256) k_sum_rain(const double* __restrict__ rain, int n, double cell_area, double* __restrict__ part) {
  __shared__ double sh[8];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += rain[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s * cell_area;
}
// out[0..2] = (water, mass, rain) from the partials, in a fixed order: thread t adds partials t, t + 256, ... in
// turn, then block_sum adds the threads' sums in its fixed tree
__global__ void __launch_bounds__(256) k_budget_final(const double* __restrict__ part, int nb, const double* __restrict__ rpart, int nr,
                                                      double* __restrict__ out) {
  __shared__ double sh[8];
  double w = 0.0, m = 0.0, r = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    w += part[2 * b];
    m += part[2 * b + 1];
  }
  for (int b = threadIdx.x; b < nr; b += blockDim.x) r += rpart[b];
  w = block_sum(w, sh);
  m = block_sum(m, sh);
  r = block_sum(r, sh);
  if (threadIdx.x == 0) {
    out[0] = w;
    out[1] = m;
    out[2] = r;
  }
}

}  // namespace ob

using namespace ob;

struct ObModel {
  Grid g{};
  ObParams P{};
  Uni U{};
  cudaStream_t stream = nullptr;
  // NUT and ADVQ read only the previous state, as ADVV does: they run on two side streams between a fork event
  // after CI and a join before PHYS, so the three issue-bound passes share the SMs
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
  float* pool = nullptr;
  float* stage = nullptr;      // texel-layout staging for field transfers
  size_t stage_bytes = 0;
  Fields F{};
  float* d_B = nullptr;
  float* d_bnd = nullptr;
  float* d_ci = nullptr;
  double* d_rain = nullptr;
  unsigned* d_flags = nullptr;
  float4* d_maps = nullptr;
  float4* d_2d = nullptr;
  double* d_red = nullptr;
  float* d_qptr = nullptr;
  // asynchronous host hand-offs (made on first use): pinned slots for requested budgets, each with the event of its
  // device-to-host copy and the ticket it holds; a pinned staging ring for the storm-start list, each slot with the
  // event of its upload
  static constexpr int kSlots = 4;
  double* h_req = nullptr;         // [kSlots][8]
  cudaEvent_t ev_req[kSlots] = {};
  long long req_ticket[kSlots] = {-1, -1, -1, -1};
  long long next_ticket = 0;
  float* h_ci = nullptr;           // [kSlots][OB_MAX_CI * OB_CI_FLOATS]
  cudaEvent_t ev_ci[kSlots] = {};
  int ci_slot = 0;
  float* rhs32 = nullptr;  // the fp32 right-hand side buffer (F.rhs points here when a solver reads it)
  unsigned int* d_act = nullptr;  // 4 brick-flag arrays (clear-air skip of the scalar advection)
  float* d_tab = nullptr;          // sponge tables of the physics pass (Fields::spz/slx/sly)
  float tab_key[8] = {};           // the uniforms the tables were made from; NaN = never made
  unsigned tab_gen = ~0u, base_gen = 0;  // base-state version the tables saw / current
  // microphysics surrogate: queue of cells for it, its counters (queued, fallbacks), its inference copy
  unsigned* d_queue = nullptr;
  unsigned* d_mlpc = nullptr;
  unsigned queue_cap = 0;
  void* d_surr = nullptr;
  const ObMlp* surr_net = nullptr;  // the network the inference copy was made from
  mlp::Norm surr_norm{};
  bool surrogate = false;
  ObMlp* rec = nullptr;  // recording (state, tendency) pairs into this network's buffer, at rate rec_rate
  float rec_rate = 0.f;
  double* d_clock = nullptr;  // model time on the device (Fields::clock)
  // captured steps, one per (parity, LSF this step, microphysics mode); replayed while the uniforms and field
  // pointers they were captured with are unchanged (model time is on the device)
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    Uni U{};
    Fields F{};
    int seen = 0;
  } graphs[2][2][3][2];  // [parity][LSF][microphysics mode][2-dx filter this step]
  bool use_graphs = true;
  PoissonPlan solver;
  std::vector<float> Bh;
  double rhoSfc = 1.15, dx = 0, dz = 0, Lx = 0, Ly = 0;
  int nb = 0, nci = 0;
  double time = 0, lsfT = 0;
  int steps = 0, parity = 0;
  // hurricane mode (setSurface / setVortex, model.js:1290-1365; uniforms model.js:1402-1420)
  bool hur_on = false;
  ObHurricane H{};
  size_t fs = 0;             // floats per field array
  float* d_vp = nullptr;     // the winds the advection carries (4 arrays), hurricane mode only
  float4* d_vx = nullptr;    // vortex table
  int vx_nr = 0;
  double vx_x = 0, vx_y = 0, vx_dr = 1, vx_moistR = 1, vx_moistRH = 0;
  bool vortex = false;
  double phiScale = 1;       // stored phi -> p'/rho factor of the next step (cn.y)
  bool cnNow = false, filtNow = false;
  // member of an ensemble: its work goes to the ensemble's stream meanwhile (own_stream is the model's own)
  void* ens = nullptr;
  cudaStream_t own_stream = nullptr;
};

// where the divergence pass writes the solve's right-hand side for the current solver precision
static void model_bind_solver(ObModel* m) {
  m->F.rhs_hi = m->F.rhs_lo = nullptr;
  m->F.rhs_ld = 0;
  m->F.rhs = m->rhs32;
  if (m->solver.precision >= 1) {
    m->solver.tc_rhs_split(&m->F.rhs_hi, &m->F.rhs_lo, &m->F.rhs_ld);
    m->solver.presplit = true;
    if (m->solver.precision == 1) m->F.rhs = nullptr;  // no fp32 copy needed
    // precision 5's first pass is plain bf16 (the hi plane alone) and its refinement starts from the fp32 residual:
    // the lo plane of the right-hand side is never read
    if (m->solver.precision == 5) m->F.rhs_lo = nullptr;
  }
}

static void drop_graphs(ObModel* m) {
  for (auto& a : m->graphs)
    for (auto& b : a)
      for (auto& c : b)
        for (auto& G : c) {
          if (G.exec) cudaGraphExecDestroy(G.exec);
          G = ObModel::StepGraph{};
        }
}

static void model_free(ObModel* m) {
  if (!m) return;
  drop_graphs(m);
  m->solver.destroy();
  for (void* p : {(void*)m->d_vp, (void*)m->d_vx, (void*)m->pool, (void*)m->stage, (void*)m->rhs32, (void*)m->d_act, (void*)m->d_tab, (void*)m->d_queue, (void*)m->d_mlpc, m->d_surr, (void*)m->d_clock, (void*)m->d_B, (void*)m->d_bnd, (void*)m->d_ci, (void*)m->d_rain,
                  (void*)m->d_flags, (void*)m->d_maps, (void*)m->d_2d, (void*)m->d_red, (void*)m->d_qptr})
    if (p) cudaFree(p);
  for (int i = 0; i < 2; i++) {
    if (m->side[i]) cudaStreamDestroy(m->side[i]);
    if (m->ev_join[i]) cudaEventDestroy(m->ev_join[i]);
  }
  if (m->ev_fork) cudaEventDestroy(m->ev_fork);
  for (int i = 0; i < ObModel::kSlots; i++) {
    if (m->ev_req[i]) cudaEventDestroy(m->ev_req[i]);
    if (m->ev_ci[i]) cudaEventDestroy(m->ev_ci[i]);
  }
  if (m->h_req) cudaFreeHost(m->h_req);
  if (m->h_ci) cudaFreeHost(m->h_ci);
  if (m->ens) m->stream = m->own_stream;  // the ensemble's stream is not the model's to destroy
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

// RegionalModel.writeUniforms (model.js:1391-1425), outbreak mode
static void write_uniforms(ObModel* m, double dt, cudaStream_t ts = nullptr) {
  const ObParams& P = m->P;
  const double DEG = M_PI / 180.0;
  auto v4 = [](double a, double b, double c, double d) { return make_float4(float(a), float(b), float(c), float(d)); };
  Uni& U = m->U;
  U.dims = v4(m->g.nx, m->g.ny, m->g.nz, m->dx);
  U.step = v4(dt, 0.0, m->rhoSfc, 9.81);  // model time: Fields::clock on the device
  U.sponge = v4(P.spongeW, P.spongeTau, P.dampZ, P.dampTau);
  U.turb = v4(P.cs, P.nu0, P.evap, P.drag != 0.f ? 1 : 0);
  const double cd = std::pow(0.41 / std::log(0.5 * m->dz / P.z0 + 1), 2);
  U.micro = v4(P.autoc, P.qc0, P.freeze, cd);
  U.misc = v4(P.vcap, P.mc, P.noise, P.ciRate);
  U.cor = v4(2 * 7.292e-5 * std::sin(P.lat * DEG), P.nudgeTau, m->nb, P.moistMix);
  U.ci = v4(m->nci, 0, 0, 0);
  U.micro2 = v4(0, P.sortQ, P.scheme > 0.5f ? 1 : 0, P.evapT);
  if (m->hur_on) {
    const ObHurricane& H = m->H;
    U.hur = v4(1, H.ck, H.landMoist, H.sfcP);
    U.hur2 = v4(H.tauRad, H.radCap, H.blDepth, H.u10f);
    U.hur3 = v4(std::pow(0.41 / std::log(0.5 * m->dz / 0.3 + 1), 2), H.gust, double(H.thermals) * double(H.thermalScale), H.maritime > 0.5f ? 1 : 0);
    m->filtNow = m->steps % 4 == 3 && H.filter4 > 0;  // the 2-dx filter: every 4th step at 4x strength
    U.hur5 = v4(H.cdCap, H.dissHeat > 0.5f ? 1 : 0, 4 * double(H.filter4), 0);
    U.hur4 = v4(H.centreX, H.centreY, H.thermalR, H.envR);
  } else {
    U.hur = v4(0, 0, 0, 0);
    U.hur2 = v4(1, 0, 1, 0.8);
    U.hur3 = v4(0, 1, 0, 0);
    U.hur4 = v4(0, 0, 1, 1e9);
    U.hur5 = v4(2.4e-3, 0, 0, 0);
    m->filtNow = false;
  }
  // the trajectory-averaged pressure force: off-centred, not on the first step after a reset (model.js:1413-1417)
  const bool cn = m->hur_on && m->steps > 0 && m->H.cnOld > 0;
  m->cnNow = cn;
  U.cn = v4(cn ? m->H.cnOld : 0, m->phiScale, cn ? 1 / (1 - double(m->H.cnOld)) : 1, m->hur_on && m->H.traj2 > 0.5f ? 1 : 0);
  if (m->vortex) {
    U.vtx = v4(m->vx_x, m->vx_y, m->vx_dr, m->vx_nr);
    U.vtx2 = v4(m->vx_moistR, m->vx_moistRH, 1, 0);
  } else {
    U.vtx = v4(0, 0, 1, 0);
    U.vtx2 = v4(1, 0, 0, 0);
  }
  U.pad = v4(m->g.pad, m->g.nxp, m->g.nyp, 0);
  U.dzv = v4(m->dz, 1 / m->dx, 1 / m->dz, P.mcFloor);
  // the same float expressions the kernels would evaluate per thread, once on the host (IEEE float arithmetic)
  const float fdt = U.step.x, fdx = U.dims.w, fdz = U.dzv.x;
  U.der = make_float4(fdt / fdx, fdt / fdz, 1.f / (fdx * fdx), 1.f / (fdz * fdz));
  U.der2 = make_float4(1.f / fdt, 0.f, 0.f, 0.f);
  // sponge tables, remade when a uniform they read or the base state changed
  const float key[8] = {U.sponge.x, U.sponge.y, U.sponge.z, U.sponge.w, U.step.z, fdx, fdz, 0.f};
  if (m->tab_gen != m->base_gen || std::memcmp(key, m->tab_key, sizeof(key)) != 0) {
    launch_tables(m->g, U, m->F, ts ? ts : m->stream);
    std::memcpy(m->tab_key, key, sizeof(key));
    m->tab_gen = m->base_gen;
  }
}

extern "C" {

const char* ob_last_error(void) { return g_err; }
const char* ob_version(void) { return "outbreaklab-b200 0.1 (sm_100a)"; }

void ob_params_default(ObParams* p) {
  // model.js:1176-1180 with the outbreak-mode overrides of app.js:1613
  p->cs = 0.18f; p->nu0 = 1.0f; p->drag = 1.0f; p->z0 = 0.1f;
  p->spongeW = 36000.f; p->spongeTau = 100.f; p->dampZ = 15000.f; p->dampTau = 150.f;
  p->autoc = 1e-3f; p->qc0 = 2e-3f; p->freeze = 1.0f; p->noise = 0.25f;
  p->mc = 1.0f; p->vcap = 110.f; p->evap = 0.22f; p->sortQ = 5e-4f;
  p->ciRate = 0.5f; p->nudgeTau = 5400.f; p->lat = 35.f; p->moistMix = 0.f;
  p->mcFloor = 0.25f; p->scheme = 0.f; p->evapT = 0.3f; p->dtScale = 1.0f;
}

int ob_grid_pad(float dx) {  // gridPad, model.js:1122
  const double v = std::round(10000.0 / dx / 8.0) * 8.0;
  return int(std::fmin(std::fmax(v, 8.0), 64.0));
}

int ob_model_create(const ObGrid* grid, ObModel** out) {
  if (!grid || !out) { set_error("ob_model_create: null argument"); return OB_ERR_INVALID; }
  *out = nullptr;
  const int nx = grid->nx, ny = grid->ny, nz = grid->nz;
  if (nx < 4 || ny < 4 || nz < 4 || nz > 512 || !(grid->dx > 0.f)) {
    set_error("ob_model_create: bad grid %d x %d x %d, dx %g", nx, ny, nz, double(grid->dx));
    return OB_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("ob_model_create: no CUDA device"); return OB_ERR_DEVICE; }
  ObModel* m = new ObModel();
  Grid& g = m->g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.px = ((nx + 1) + 31) / 32 * 32;
  g.py = ny + 1;
  g.plane = g.px * g.py;
  g.pad = ob_grid_pad(grid->dx);
  g.nxp = nx + 2 * g.pad;
  g.nyp = ny + 2 * g.pad;
  m->dx = grid->dx;
  m->dz = 20000.0 / nz;
  m->Lx = nx * m->dx;
  m->Ly = ny * m->dx;
  ob_params_default(&m->P);
  m->P.spongeW = float(std::fmin(std::fmax(0.08 * std::fmin(m->Lx, m->Ly), 5000.0), 40000.0));  // model.js:1207
  const double fieldsz = double(g.plane) * (nz + 1);
  if (fieldsz * 39 * 4 > 170e9) { delete m; set_error("ob_model_create: grid too large for one GPU"); return OB_ERR_INVALID; }
  const size_t fs = (size_t(g.plane) * (nz + 1) + 63) / 64 * 64;
  m->fs = fs;
  const size_t n2 = size_t(nx) * ny, np = size_t(g.nxp) * g.nyp * nz;
  int rc = OB_OK;
  auto alloc = [&](void** p, size_t bytes, const char* what) {
    if (rc != OB_OK) return;
    rc = cuda_status(cudaMalloc(p, bytes), what);
    if (rc == OB_OK) rc = cuda_status(cudaMemset(*p, 0, bytes), what);
  };
  rc = cuda_status(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "stream");
  for (int i = 0; i < 2 && rc == OB_OK; i++) {
    rc = cuda_status(cudaStreamCreateWithFlags(&m->side[i], cudaStreamNonBlocking), "side stream");
    if (rc == OB_OK) rc = cuda_status(cudaEventCreateWithFlags(&m->ev_join[i], cudaEventDisableTiming), "event");
  }
  if (rc == OB_OK) rc = cuda_status(cudaEventCreateWithFlags(&m->ev_fork, cudaEventDisableTiming), "event");
  alloc((void**)&m->pool, fs * 47 * sizeof(float), "model fields");
  alloc((void**)&m->d_B, size_t(nz + 1) * 8 * sizeof(float), "base state");
  alloc((void**)&m->d_bnd, size_t(OB_MAX_BOUNDS) * OB_BOUNDARY_FLOATS * sizeof(float), "boundaries");
  alloc((void**)&m->d_ci, size_t(OB_MAX_CI) * OB_CI_FLOATS * sizeof(float), "CI events");
  alloc((void**)&m->d_rain, n2 * sizeof(double), "rain");
  alloc((void**)&m->d_flags, 64 * sizeof(unsigned), "flags");
  alloc((void**)&m->d_maps, n2 * 4 * sizeof(float4), "maps");
  alloc((void**)&m->d_2d, n2 * 4 * sizeof(float4), "2-D fields");
  alloc((void**)&m->d_red, kRedDoubles * sizeof(double), "reductions");
  alloc((void**)&m->d_clock, sizeof(double), "model clock");
  alloc((void**)&m->rhs32, np * sizeof(float), "rhs");
  alloc((void**)&m->F.phi, np * sizeof(float), "phi");
  m->stage_bytes = std::max(size_t(nx + 1) * (ny + 1) * (nz + 1) * 4, np) * sizeof(float);
  alloc((void**)&m->stage, m->stage_bytes, "staging");
  alloc((void**)&m->d_qptr, 8 * sizeof(float*), "pointer table");
  const int nbx = (nx + 31) / 32, nby = (ny + 3) / 4;
  const size_t nbr = size_t(nbx) * nby * nz;
  alloc((void**)&m->d_act, 4 * nbr * sizeof(unsigned int), "activity flags");
  const size_t ntab = size_t(4) * (nz + 1) + 2 * size_t(nx + 1) + 2 * size_t(ny + 1);
  alloc((void**)&m->d_tab, ntab * sizeof(float), "sponge tables");
  // the refined tensor-core solve (a plain-bf16 pass refined by a bf16x3 sweep) where its tridiagonal kernel is
  // specialised, else fp32
  const int prec = (nz == 16 || nz == 40 || nz == 80) ? 5 : 0;
  if (rc == OB_OK) rc = m->solver.create(g.nxp, g.nyp, nz, m->dx, m->dz, prec);
  if (rc != OB_OK) {
    if (rc == OB_ERR_OOM) {
      const double gb = (fs * 47.0 * 4 + np * 4.0 * 5 + n2 * 200.0) / 1e9;
      set_error("not enough GPU memory for this grid (it needs about %.1f GB)", gb);
    }
    model_free(m);
    return rc;
  }
  float* p = m->pool;
  auto take = [&]() { float* r = p; p += fs; return r; };
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 4; c++) m->F.V[s][c] = take();
  for (int c = 0; c < 4; c++) m->F.Vt[c] = take();
  for (int c = 0; c < 4; c++) m->F.Vlo[c] = take();
  for (int c = 0; c < 4; c++) m->F.Vhi[c] = take();
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 8; c++) m->F.Q[s][c] = take();
  for (int c = 0; c < 8; c++) m->F.Qt[c] = take();
  m->F.aux[0] = take();
  m->F.aux[1] = take();
  m->F.phT = take();
  m->F.lsfA = m->d_2d;
  m->F.lsfB = m->d_2d + n2;
  m->F.ciMap = m->d_2d + 2 * n2;
  m->F.sfc = m->d_2d + 3 * n2;
  m->F.B = m->d_B;
  m->F.rain = m->d_rain;
  model_bind_solver(m);
  m->F.bnd = m->d_bnd;
  m->F.ci = m->d_ci;
  m->F.flags = m->d_flags;
  m->F.clock = m->d_clock;
  m->F.nbx = nbx;
  m->F.nby = nby;
  m->F.actQ0 = m->d_act;
  m->F.actQt = m->d_act + nbr;
  m->F.zeroQt = m->d_act + 2 * nbr;
  m->F.zeroQ1 = m->d_act + 3 * nbr;
  m->F.fallmax = 100.f;
  m->F.spz = m->d_tab;                      // 4 floats per level: 16-byte aligned
  m->F.slx = m->d_tab + 4 * (nz + 1);       // 2 floats per column: 8-byte aligned
  m->F.sly = m->F.slx + 2 * (nx + 1);
  rc = cuda_status(cudaMemcpy(m->d_qptr, m->F.Q[0], 8 * sizeof(float*), cudaMemcpyHostToDevice), "pointer table");
  // a neutral base state until one is set
  m->Bh.assign(size_t(nz + 1) * 8, 0.f);
  for (int k = 0; k <= nz; k++) {
    m->Bh[k * 8 + 0] = 300.f; m->Bh[k * 8 + 2] = 1.f; m->Bh[k * 8 + 3] = 1.f; m->Bh[k * 8 + 4] = 1.f; m->Bh[k * 8 + 5] = 1e5f;
  }
  if (rc == OB_OK) rc = cuda_status(cudaMemcpy(m->d_B, m->Bh.data(), m->Bh.size() * sizeof(float), cudaMemcpyHostToDevice), "base state");
  if (rc != OB_OK) {
    model_free(m);
    return rc;
  }
  *out = m;
  return OB_OK;
}

int ob_model_destroy(ObModel* m) {
  if (m) {
    cudaStreamSynchronize(m->stream);
    model_free(m);
  }
  return OB_OK;
}

int ob_model_set_base_state(ObModel* m, const float* B, int nz) {
  if (!m || !B || nz != m->g.nz) { set_error("ob_model_set_base_state: expected nz = %d", m ? m->g.nz : -1); return OB_ERR_INVALID; }
  // captured steps hold the solve's z-operator by value (the tridiagonal's kernel parameters): recapture after it
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "base state"));
  drop_graphs(m);
  m->Bh.assign(B, B + size_t(nz + 1) * 8);
  m->rhoSfc = B[2];
  m->base_gen++;
  {
    // the largest fall speed any hydrometeor can reach (model.js:63-99): rain <= 10, snow <= 2.2, Thompson graupel
    // <= 25 m/s, each times sqrt(rho_sfc / rho), Lin graupel <= 65 m/s; bounds the vertical reach of a fall trace
    double rmin = 1e30;
    for (int k = 0; k < nz; k++) rmin = std::min(rmin, double(B[k * 8 + 2]));
    const double s = std::sqrt(std::max(double(m->rhoSfc), 1e-6) / std::max(rmin, 1e-6));
    m->F.fallmax = float(std::max(65.0, 25.0 * s) * 1.01 + 1.0);
  }
  OB_TRY(cuda_status(cudaMemcpyAsync(m->d_B, m->Bh.data(), m->Bh.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream), "base state"));
  std::vector<float> rc(nz), rw(nz + 1);
  for (int k = 0; k < nz; k++) rc[k] = B[k * 8 + 2];
  for (int k = 0; k <= nz; k++) rw[k] = B[k * 8 + 3];
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "base state"));
  return m->solver.set_density(rc.data(), rw.data());
}

int ob_model_set_params(ObModel* m, const ObParams* p) {
  if (!m || !p) { set_error("ob_model_set_params: null argument"); return OB_ERR_INVALID; }
  const float sw = m->P.spongeW;  // the sponge width follows the domain (model.js:1207)
  m->P = *p;
  m->P.spongeW = sw;
  return OB_OK;
}

int ob_model_set_boundaries(ObModel* m, const float* packed, int n) {
  if (!m || n < 0 || (n > 0 && !packed)) { set_error("ob_model_set_boundaries: bad arguments"); return OB_ERR_INVALID; }
  m->nb = n < OB_MAX_BOUNDS ? n : OB_MAX_BOUNDS;
  std::vector<float> f(size_t(OB_MAX_BOUNDS) * OB_BOUNDARY_FLOATS, 0.f);
  if (m->nb) std::memcpy(f.data(), packed, sizeof(float) * m->nb * OB_BOUNDARY_FLOATS);
  OB_TRY(cuda_status(cudaMemcpyAsync(m->d_bnd, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream), "boundaries"));
  return cuda_status(cudaStreamSynchronize(m->stream), "boundaries");
}

// the pinned slots and events of the asynchronous hand-offs, made on first use
static int async_slots(ObModel* m) {
  if (m->h_req) return OB_OK;
  OB_TRY(cuda_status(cudaHostAlloc(&m->h_ci, sizeof(float) * ObModel::kSlots * OB_MAX_CI * OB_CI_FLOATS, cudaHostAllocDefault), "host slots"));
  for (int i = 0; i < ObModel::kSlots; i++) {
    OB_TRY(cuda_status(cudaEventCreateWithFlags(&m->ev_req[i], cudaEventDisableTiming), "host slots"));
    OB_TRY(cuda_status(cudaEventCreateWithFlags(&m->ev_ci[i], cudaEventDisableTiming), "host slots"));
  }
  return cuda_status(cudaHostAlloc(&m->h_req, sizeof(double) * ObModel::kSlots * 8, cudaHostAllocDefault), "host slots");
}

int ob_model_set_ci(ObModel* m, const float* ev, int n) {
  if (!m || n < 0 || (n > 0 && !ev)) { set_error("ob_model_set_ci: bad arguments"); return OB_ERR_INVALID; }
  m->nci = n < OB_MAX_CI ? n : OB_MAX_CI;
  if (m->nci) {
    // the list is copied at the call, as queue.writeBuffer does: into a pinned staging slot, whose upload is queued
    // on the model's stream without waiting for it (the slot is reused once its previous upload has been done)
    OB_TRY(async_slots(m));
    const int sl = m->ci_slot;
    m->ci_slot = (sl + 1) % ObModel::kSlots;
    OB_TRY(cuda_status(cudaEventSynchronize(m->ev_ci[sl]), "CI"));
    float* stage = m->h_ci + size_t(sl) * OB_MAX_CI * OB_CI_FLOATS;
    const float* src = ev + size_t(n - m->nci) * OB_CI_FLOATS;  // the most recent MAX_CI (model.js:1384)
    std::memcpy(stage, src, sizeof(float) * m->nci * OB_CI_FLOATS);
    OB_TRY(cuda_status(cudaMemcpyAsync(m->d_ci, stage, sizeof(float) * m->nci * OB_CI_FLOATS, cudaMemcpyHostToDevice, m->stream), "CI"));
    OB_TRY(cuda_status(cudaEventRecord(m->ev_ci[sl], m->stream), "CI"));
  }
  return OB_OK;
}

int ob_model_reset(ObModel* m) {
  if (!m) { set_error("ob_model_reset: null model"); return OB_ERR_INVALID; }
  m->time = 0; m->steps = 0; m->parity = 0; m->phiScale = 1;
  OB_TRY(cuda_status(cudaMemsetAsync(m->d_clock, 0, sizeof(double), m->stream), "reset"));
  write_uniforms(m, 1.0);
  const Grid& g = m->g;
  launch_lsf(g, m->U, m->F, m->stream);
  launch_init(g, m->U, m->F, m->stream);
  const size_t np = size_t(g.nxp) * g.nyp * g.nz;
  OB_TRY(cuda_status(cudaMemsetAsync(m->F.phi, 0, np * sizeof(float), m->stream), "reset"));
  OB_TRY(cuda_status(cudaMemsetAsync(m->rhs32, 0, np * sizeof(float), m->stream), "reset"));
  OB_TRY(cuda_status(cudaMemsetAsync(m->d_rain, 0, size_t(g.nx) * g.ny * sizeof(double), m->stream), "reset"));
  OB_TRY(cuda_status(cudaMemsetAsync(m->d_flags, 0, 64 * sizeof(unsigned), m->stream), "reset"));
  launch_activity(g, m->F, m->stream);
  m->lsfT = 0;
  return cuda_status(cudaGetLastError(), "reset");
}

extern "C++" {
namespace ob {
int surrogate_prepare(const ObMlp* net, void** d_image, mlp::Norm* norm);
void launch_surrogate(const Grid& g, const Uni& U, const Fields& F, int par, const void* d_image, const mlp::Norm& nm,
                      unsigned int* err, cudaStream_t s);
void launch_surrogate_grp(const MemberC* d_members, int n, int par, const void* d_image, const mlp::Norm& nm, unsigned int* err,
                          cudaStream_t s);
void mlp_record_target(ObMlp* n, float** buf, unsigned** count, unsigned* cap);
void launch_level2(const uint8_t* vol, size_t vol_bytes, const ObL2Sweep* d_sweeps, int nsweeps, int max_nrad, const uint8_t* d_tpl,
                   uint8_t* d_out, cudaStream_t s);
}  // namespace ob
}

// the physics pass with the model's microphysics mode: the scheme, the scheme while recording pairs, or the surrogate
static int micro_mode(const ObModel* m) { return m->surrogate ? kMicroSurrogate : (m->rec && m->rec_rate > 0.f) ? kMicroRecord : kMicroPlain; }

// the microphysics fields of the kernel parameters for the model's mode (before a step is launched or captured)
static int prepare_micro(ObModel* m) {
  const int mode = micro_mode(m);
  if (m->hur_on && mode != kMicroPlain) { set_error("hurricane mode runs the plain microphysics (no surrogate, no pair recording)"); return OB_ERR_INVALID; }
  if (mode == kMicroSurrogate) {
    if (m->P.scheme < 0.5f) { set_error("the microphysics surrogate emulates the Thompson-style scheme (params.scheme = 1)"); return OB_ERR_INVALID; }
    m->F.mlp_buf = reinterpret_cast<float*>(m->d_queue);
    m->F.mlp_count = m->d_mlpc;
    m->F.mlp_cap = m->queue_cap;
    m->F.mlp_rate = 0.f;
  } else if (mode == kMicroRecord) {
    mlp_record_target(m->rec, &m->F.mlp_buf, &m->F.mlp_count, &m->F.mlp_cap);
    m->F.mlp_rate = m->rec_rate;
  } else {
    m->F.mlp_buf = nullptr;
    m->F.mlp_count = nullptr;
    m->F.mlp_cap = 0;
    m->F.mlp_rate = 0.f;
  }
  return OB_OK;
}

// the physics pass with the model's microphysics mode: the scheme, the scheme while recording pairs, or the surrogate
static int physics_pass(ObModel* m, int par, cudaStream_t s) {
  const Grid& g = m->g;
  OB_TRY(prepare_micro(m));
  const int mode = micro_mode(m);
  if (mode == kMicroSurrogate) {
    OB_TRY(cuda_status(cudaMemsetAsync(m->d_mlpc, 0, 2 * sizeof(unsigned), s), "surrogate counters"));
    launch_phys(g, m->U, m->F, par, s, kMicroSurrogate);
    launch_surrogate(g, m->U, m->F, par, m->d_surr, m->surr_norm, m->d_flags + 1, s);
  } else {
    launch_phys(g, m->U, m->F, par, s, m->F.mlp_buf ? mode : kMicroPlain);
  }
  return OB_OK;
}

// every pass of one step, queued on the model's stream (NUT and ADVQ on the side streams)
static int enqueue_step(ObModel* m, bool lsf, cudaStream_t s) {
  const Grid& g = m->g;
  const int par = m->parity;
  if (m->hur_on && m->filtNow) {  // state -> scratch -> back (model.js:1448-1455)
    launch_filt(g, m->U, m->F, par, s);
    const size_t bytes = m->fs * sizeof(float);
    for (int c = 0; c < 4; c++) OB_TRY(cuda_status(cudaMemcpyAsync(m->F.V[par][c], m->F.V[1 - par][c], bytes, cudaMemcpyDeviceToDevice, s), "filter"));
    for (int c = 0; c < 8; c++) OB_TRY(cuda_status(cudaMemcpyAsync(m->F.Q[0][c], m->F.Q[1][c], bytes, cudaMemcpyDeviceToDevice, s), "filter"));
  }
  if (m->hur_on) launch_prep(g, m->U, m->F, par, s);
  if (lsf) launch_lsf(g, m->U, m->F, s);
  launch_ci(g, m->U, m->F, s);
  cudaEventRecord(m->ev_fork, s);
  for (int i = 0; i < 2; i++) cudaStreamWaitEvent(m->side[i], m->ev_fork, 0);
  launch_nut(g, m->U, m->F, par, m->side[0]);
  cudaEventRecord(m->ev_join[0], m->side[0]);
  launch_advq(g, m->U, m->F, par, m->side[1]);
  cudaEventRecord(m->ev_join[1], m->side[1]);
  launch_advv(g, m->U, m->F, par, s);
  for (int i = 0; i < 2; i++) cudaStreamWaitEvent(s, m->ev_join[i], 0);
  OB_TRY(physics_pass(m, par, s));
  launch_div(g, m->U, m->F, par, s);
  OB_TRY(m->solver.solve(m->F.rhs, m->F.phi, s));
  launch_proj(g, m->U, m->F, par, s);
  launch_rain(g, m->U, m->F, s);
  return OB_OK;
}

// One step. With graphs on, the second occurrence of a (parity, LSF, microphysics mode) variant is captured and
// later occurrences replay it as long as the uniforms and the kernels' field pointers are the ones it was captured
// with (the model time lives on the device); the first occurrence runs uncaptured, so every lazy set-up (function
// attributes, device queries) has happened before any capture.
static int model_step_once(ObModel* m, double dt) {
  write_uniforms(m, dt);
  cudaStream_t s = m->stream;
  const bool lsf = m->time - m->lsfT >= 60 || m->time == 0;
  if (lsf) m->lsfT = m->time;
  OB_TRY(prepare_micro(m));
  if (!m->use_graphs) {
    OB_TRY(enqueue_step(m, lsf, s));
  } else {
    ObModel::StepGraph& G = m->graphs[m->parity][lsf ? 1 : 0][micro_mode(m)][m->filtNow ? 1 : 0];
    const bool match = G.exec && std::memcmp(&G.U, &m->U, sizeof(Uni)) == 0 && std::memcmp(&G.F, &m->F, sizeof(Fields)) == 0;
    if (match) {
      OB_TRY(cuda_status(cudaGraphLaunch(G.exec, s), "step graph launch"));
    } else if (G.seen == 0) {
      G.seen = 1;
      OB_TRY(enqueue_step(m, lsf, s));
    } else {
      if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
      OB_TRY(cuda_status(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "step capture"));
      const int rc = enqueue_step(m, lsf, s);
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(s, &graph);
      if (rc != OB_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
      OB_TRY(cuda_status(ec, "step capture"));
      const cudaError_t ei = cudaGraphInstantiate(&G.exec, graph, 0);
      cudaGraphDestroy(graph);
      OB_TRY(cuda_status(ei, "step graph instantiate"));
      G.U = m->U;
      G.F = m->F;
      OB_TRY(cuda_status(cudaGraphLaunch(G.exec, s), "step graph launch"));
    }
  }
  m->parity = 1 - m->parity;
  m->time += dt;
  m->steps++;
  m->phiScale = m->cnNow ? 1 / (1 - double(m->H.cnOld)) : 1;
  return cuda_status(cudaGetLastError(), "step launch");
}

int ob_model_step(ObModel* m, float dt, int nsteps) {
  if (!m || !(dt > 0.f) || nsteps < 0) { set_error("ob_model_step: bad arguments"); return OB_ERR_INVALID; }
  for (int s = 0; s < nsteps; s++) OB_TRY(model_step_once(m, dt));
  return OB_OK;
}

int ob_model_sync(ObModel* m) {
  if (!m) { set_error("ob_model_sync: null model"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "step"));
  return m->solver.tc_check();
}

int ob_model_maps(ObModel* m, float* out) {
  if (!m || !out) { set_error("ob_model_maps: null argument"); return OB_ERR_INVALID; }
  launch_maps(m->g, m->U, m->F, m->parity, m->d_maps, m->stream);
  const size_t bytes = size_t(m->g.nx) * m->g.ny * 4 * sizeof(float4);
  OB_TRY(cuda_status(cudaMemcpyAsync(out, m->d_maps, bytes, cudaMemcpyDeviceToHost, m->stream), "maps"));
  return cuda_status(cudaStreamSynchronize(m->stream), "maps");
}

int ob_model_tornado_candidates(ObModel* m, float zeta_min, float* out, int cap, int* count) {
  if (!m || !out || cap < 1 || !count) { set_error("ob_model_tornado_candidates: bad arguments"); return OB_ERR_INVALID; }
  float* d_out = nullptr;
  unsigned* d_n = nullptr;
  int rc = cuda_status(cudaMalloc(&d_out, size_t(cap) * 7 * sizeof(float)), "tornado candidates");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&d_n, sizeof(unsigned)), "tornado candidates");
  if (rc == OB_OK) rc = cuda_status(cudaMemsetAsync(d_n, 0, sizeof(unsigned), m->stream), "tornado candidates");
  unsigned n = 0;
  if (rc == OB_OK) {
    launch_tor_candidates(m->g, float(m->dx), m->d_maps, zeta_min, d_out, cap, d_n, m->stream);
    rc = cuda_status(cudaMemcpyAsync(&n, d_n, sizeof(unsigned), cudaMemcpyDeviceToHost, m->stream), "tornado candidates");
  }
  if (rc == OB_OK) rc = cuda_status(cudaStreamSynchronize(m->stream), "tornado candidates");
  if (rc == OB_OK && n > 0)
    rc = cuda_status(cudaMemcpy(out, d_out, size_t(std::min<unsigned>(n, unsigned(cap))) * 7 * sizeof(float), cudaMemcpyDeviceToHost), "tornado candidates");
  *count = int(n);
  if (d_out) cudaFree(d_out);
  if (d_n) cudaFree(d_n);
  return rc;
}

static int field_layout(ObModel* m, int field, Ptr8& p, int& nch, int& X, int& Y, int& Z) {
  const Grid& g = m->g;
  switch (field) {
    case OB_FIELD_V:
      for (int c = 0; c < 4; c++) p.p[c] = m->F.V[m->parity][c];
      nch = 4; X = g.nx + 1; Y = g.ny + 1; Z = g.nz + 1; return OB_OK;
    case OB_FIELD_Q1:
    case OB_FIELD_Q2:
      for (int c = 0; c < 4; c++) p.p[c] = m->F.Q[0][c + (field == OB_FIELD_Q2 ? 4 : 0)];
      nch = 4; X = g.nx; Y = g.ny; Z = g.nz; return OB_OK;
    case OB_FIELD_AUX:
      p.p[0] = m->F.aux[0]; p.p[1] = m->F.aux[1];
      nch = 2; X = g.nx; Y = g.ny; Z = g.nz; return OB_OK;
    case OB_FIELD_PHT:
      p.p[0] = m->F.phT;
      nch = 1; X = g.nx; Y = g.ny; Z = g.nz; return OB_OK;
    default:
      set_error("unknown field %d", field);
      return OB_ERR_INVALID;
  }
}

int ob_model_get_field(ObModel* m, int field, void* host, size_t bytes) {
  if (!m || !host) { set_error("ob_model_get_field: null argument"); return OB_ERR_INVALID; }
  const Grid& g = m->g;
  if (field == OB_FIELD_LSF_A || field == OB_FIELD_LSF_B || field == OB_FIELD_CI_MAP) {
    const size_t need = size_t(g.nx) * g.ny * sizeof(float4);
    if (bytes != need) { set_error("ob_model_get_field: %zu bytes, expected %zu", bytes, need); return OB_ERR_INVALID; }
    const void* src = field == OB_FIELD_LSF_A ? (const void*)m->F.lsfA : field == OB_FIELD_LSF_B ? (const void*)m->F.lsfB
                                                                                                 : (const void*)m->F.ciMap;
    OB_TRY(cuda_status(cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, m->stream), "get field"));
    return cuda_status(cudaStreamSynchronize(m->stream), "get field");
  }
  if (field == OB_FIELD_PHI || field == OB_FIELD_RAIN) {
    const size_t need = field == OB_FIELD_PHI ? size_t(g.nxp) * g.nyp * g.nz * sizeof(float) : size_t(g.nx) * g.ny * sizeof(double);
    if (bytes != need) { set_error("ob_model_get_field: %zu bytes, expected %zu", bytes, need); return OB_ERR_INVALID; }
    const void* src = field == OB_FIELD_PHI ? (const void*)m->F.phi : (const void*)m->d_rain;
    OB_TRY(cuda_status(cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, m->stream), "get field"));
    return cuda_status(cudaStreamSynchronize(m->stream), "get field");
  }
  Ptr8 p{};
  int nch, X, Y, Z;
  OB_TRY(field_layout(m, field, p, nch, X, Y, Z));
  const size_t need = size_t(X) * Y * Z * nch * sizeof(float);
  if (bytes != need) { set_error("ob_model_get_field: %zu bytes, expected %zu", bytes, need); return OB_ERR_INVALID; }
  launch_pack(g, p, nch, X, Y, Z, m->stage, m->stream);
  OB_TRY(cuda_status(cudaMemcpyAsync(host, m->stage, bytes, cudaMemcpyDeviceToHost, m->stream), "get field"));
  return cuda_status(cudaStreamSynchronize(m->stream), "get field");
}

int ob_model_set_field(ObModel* m, int field, const void* host, size_t bytes) {
  if (!m || !host) { set_error("ob_model_set_field: null argument"); return OB_ERR_INVALID; }
  const Grid& g = m->g;
  if (field >= OB_FIELD_LSF_A && field <= OB_FIELD_PHT) {
    set_error("ob_model_set_field: field %d is a read-only diagnostic (the LSF and CI passes write it)", field);
    return OB_ERR_INVALID;
  }
  if (field == OB_FIELD_PHI || field == OB_FIELD_RAIN) {
    const size_t need = field == OB_FIELD_PHI ? size_t(g.nxp) * g.nyp * g.nz * sizeof(float) : size_t(g.nx) * g.ny * sizeof(double);
    if (bytes != need) { set_error("ob_model_set_field: %zu bytes, expected %zu", bytes, need); return OB_ERR_INVALID; }
    void* dst = field == OB_FIELD_PHI ? (void*)m->F.phi : (void*)m->d_rain;
    OB_TRY(cuda_status(cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, m->stream), "set field"));
    return cuda_status(cudaStreamSynchronize(m->stream), "set field");
  }
  Ptr8 p{};
  int nch, X, Y, Z;
  OB_TRY(field_layout(m, field, p, nch, X, Y, Z));
  const size_t need = size_t(X) * Y * Z * nch * sizeof(float);
  if (bytes != need) { set_error("ob_model_set_field: %zu bytes, expected %zu", bytes, need); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaMemcpyAsync(m->stage, host, bytes, cudaMemcpyHostToDevice, m->stream), "set field"));
  launch_unpack(g, p, nch, X, Y, Z, m->stage, m->stream);
  if (field == OB_FIELD_Q1 || field == OB_FIELD_Q2) launch_activity(g, m->F, m->stream);
  return cuda_status(cudaStreamSynchronize(m->stream), "set field");
}

int ob_model_time(ObModel* m, double* time, int* steps, int* parity) {
  if (!m) { set_error("ob_model_time: null model"); return OB_ERR_INVALID; }
  if (time) *time = m->time;
  if (steps) *steps = m->steps;
  if (parity) *parity = m->parity;
  return OB_OK;
}

// the budget reductions into d_red, queued on the model's stream
static int queue_budgets(ObModel* m) {
  const Grid& g = m->g;
  OB_TRY(cuda_status(cudaMemsetAsync(m->d_red, 0, 8 * sizeof(double), m->stream), "budgets"));
  const int nb = std::min(g.ny * g.nz, kBudgetBlocks);
  double* part = m->d_red + 8;
  double* rpart = part + 2 * kBudgetBlocks;
  k_budget<<<nb, 256, 0, m->stream>>>(g, m->d_B, reinterpret_cast<float* const*>(m->d_qptr), m->F.actQ0, m->F.nbx, m->F.nby,
                                      m->dx * m->dx * m->dz, part);
  k_sum_rain<<<kRainBlocks, 256, 0, m->stream>>>(m->d_rain, g.nx * g.ny, m->dx * m->dx, rpart);
  k_budget_final<<<1, 256, 0, m->stream>>>(part, nb, rpart, kRainBlocks, m->d_red);
  return cuda_status(cudaGetLastError(), "budgets");
}

int ob_model_request_budgets(ObModel* m, long long* ticket) {
  if (!m || !ticket) { set_error("ob_model_request_budgets: null argument"); return OB_ERR_INVALID; }
  OB_TRY(async_slots(m));
  const long long t = m->next_ticket;
  const int sl = int(t % ObModel::kSlots);
  OB_TRY(cuda_status(cudaEventSynchronize(m->ev_req[sl]), "request budgets"));   // the slot's previous copy is done
  OB_TRY(queue_budgets(m));
  OB_TRY(cuda_status(cudaMemcpyAsync(m->h_req + size_t(sl) * 8, m->d_red, 8 * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "request budgets"));
  OB_TRY(cuda_status(cudaEventRecord(m->ev_req[sl], m->stream), "request budgets"));
  m->req_ticket[sl] = t;
  m->next_ticket = t + 1;
  *ticket = t;
  return OB_OK;
}

int ob_model_read_budgets(ObModel* m, long long ticket, double* water, double* mass, double* rain) {
  if (!m) { set_error("ob_model_read_budgets: null model"); return OB_ERR_INVALID; }
  const int sl = ticket >= 0 ? int(ticket % ObModel::kSlots) : 0;
  if (ticket < 0 || !m->h_req || m->req_ticket[sl] != ticket) {
    set_error("ob_model_read_budgets: ticket %lld was not requested or its slot has been reused (%d slots)", ticket, ObModel::kSlots);
    return OB_ERR_INVALID;
  }
  OB_TRY(cuda_status(cudaEventSynchronize(m->ev_req[sl]), "read budgets"));
  const double* h = m->h_req + size_t(sl) * 8;
  if (water) *water = h[0];
  if (mass) *mass = h[1];
  if (rain) *rain = h[2];
  return OB_OK;
}

int ob_model_budgets(ObModel* m, double* water, double* mass, double* rain) {
  if (!m) { set_error("ob_model_budgets: null model"); return OB_ERR_INVALID; }
  OB_TRY(queue_budgets(m));
  double h[8];
  OB_TRY(cuda_status(cudaMemcpyAsync(h, m->d_red, sizeof(h), cudaMemcpyDeviceToHost, m->stream), "budgets"));
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "budgets"));
  if (water) *water = h[0];
  if (mass) *mass = h[1];
  if (rain) *rain = h[2];
  return OB_OK;
}

// K steps bracketed by CUDA events on the model's stream; *ms = device time of the K steps
int ob_model_timed_steps(ObModel* m, float dt, int nsteps, float* ms) {
  if (!m || !ms || !(dt > 0.f) || nsteps < 0) { set_error("ob_model_timed_steps: bad arguments"); return OB_ERR_INVALID; }
  EventPair ev;
  OB_TRY(ev.create());
  OB_TRY(cuda_status(cudaEventRecord(ev.a, m->stream), "timed steps"));
  int rc = OB_OK;
  for (int s = 0; s < nsteps && rc == OB_OK; s++) rc = model_step_once(m, dt);
  if (rc == OB_OK) rc = cuda_status(cudaEventRecord(ev.b, m->stream), "timed steps");
  if (rc == OB_OK) rc = ev.elapsed(ms, "timed steps");
  return rc;
}

// one step with an event between passes: ms[i] = device time of pass i (OB_PASS_* order), returns the pass count
int ob_model_profile_step(ObModel* m, float dt, float* ms, int max_passes) {
  if (!m || !ms || max_passes < OB_NPASS) { set_error("ob_model_profile_step: need %d slots", OB_NPASS); return -OB_ERR_INVALID; }
  // the pass boundaries: OB_NPASS + 1 events, destroyed on every return path
  struct Events {
    cudaEvent_t e[OB_NPASS + 1] = {};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } evs;
  cudaEvent_t* ev = evs.e;
  for (int i = 0; i <= OB_NPASS; i++)
    if (cuda_status(cudaEventCreate(&ev[i]), "profile step") != OB_OK) return -OB_ERR_DEVICE;
  write_uniforms(m, dt);
  const Grid& g = m->g;
  const int par = m->parity;
  cudaStream_t s = m->stream;
  int e = 0;
  cudaEventRecord(ev[e++], s);
  if (m->time - m->lsfT >= 60 || m->time == 0) { launch_lsf(g, m->U, m->F, s); m->lsfT = m->time; }
  launch_ci(g, m->U, m->F, s);
  cudaEventRecord(ev[e++], s);
  launch_nut(g, m->U, m->F, par, s);
  cudaEventRecord(ev[e++], s);
  launch_advv(g, m->U, m->F, par, s);
  cudaEventRecord(ev[e++], s);
  launch_advq(g, m->U, m->F, par, s);
  cudaEventRecord(ev[e++], s);
  const int prc = physics_pass(m, par, s);
  cudaEventRecord(ev[e++], s);
  launch_div(g, m->U, m->F, par, s);
  cudaEventRecord(ev[e++], s);
  int rc = m->solver.solve(m->F.rhs, m->F.phi, s);
  if (rc == OB_OK) rc = prc;
  cudaEventRecord(ev[e++], s);
  launch_proj(g, m->U, m->F, par, s);
  launch_rain(g, m->U, m->F, s);
  cudaEventRecord(ev[e++], s);
  m->parity = 1 - m->parity;
  m->time += dt;
  m->steps++;
  if (rc == OB_OK) rc = cuda_status(cudaGetLastError(), "profile step");
  if (rc == OB_OK) rc = cuda_status(cudaEventSynchronize(ev[e - 1]), "profile step");
  for (int i = 0; i + 1 < e && rc == OB_OK; i++) rc = cuda_status(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]), "profile step");
  return rc == OB_OK ? e - 1 : -rc;
}

int ob_model_set_graphs(ObModel* m, int on) {
  if (!m) { set_error("ob_model_set_graphs: null model"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "set graphs"));
  drop_graphs(m);
  m->use_graphs = on != 0;
  return OB_OK;
}

int ob_model_record_micro(ObModel* m, ObMlp* net, float rate) {
  if (!m || rate < 0.f || rate > 1.f) { set_error("ob_model_record_micro: bad arguments"); return OB_ERR_INVALID; }
  m->rec = rate > 0.f ? net : nullptr;
  m->rec_rate = rate;
  return OB_OK;
}

int ob_model_set_surrogate(ObModel* m, const ObMlp* net) {
  if (!m) { set_error("ob_model_set_surrogate: null model"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "set surrogate"));
  if (!net) { m->surrogate = false; return OB_OK; }
  if (!m->d_queue) {
    const size_t cells = size_t(m->g.nx) * m->g.ny * m->g.nz;
    OB_TRY(cuda_status(cudaMalloc(&m->d_queue, cells * sizeof(unsigned)), "surrogate queue"));
    OB_TRY(cuda_status(cudaMalloc(&m->d_mlpc, 2 * sizeof(unsigned)), "surrogate counters"));
    OB_TRY(cuda_status(cudaMemset(m->d_mlpc, 0, 2 * sizeof(unsigned)), "surrogate counters"));
    m->queue_cap = unsigned(cells);
  }
  OB_TRY(surrogate_prepare(net, &m->d_surr, &m->surr_norm));
  m->surrogate = true;
  m->surr_net = net;
  return OB_OK;
}

int ob_model_surrogate_stats(ObModel* m, unsigned* queued, unsigned* fallbacks) {
  if (!m || !queued || !fallbacks) { set_error("ob_model_surrogate_stats: null argument"); return OB_ERR_INVALID; }
  unsigned h[2] = {0, 0}, e = 0;
  if (m->d_mlpc) {
    OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "surrogate stats"));
    OB_TRY(cuda_status(cudaMemcpy(h, m->d_mlpc, sizeof(h), cudaMemcpyDeviceToHost), "surrogate stats"));
    OB_TRY(cuda_status(cudaMemcpy(&e, m->d_flags + 1, sizeof(e), cudaMemcpyDeviceToHost), "surrogate stats"));
  }
  *queued = h[0];
  *fallbacks = h[1];
  if (e) {
    cudaMemset(m->d_flags + 1, 0, sizeof(unsigned));
    set_error("surrogate: a tensor-core pipeline wait timed out (code %u)", e);
    return OB_ERR_TIMEOUT;
  }
  return OB_OK;
}

int ob_model_set_solver(ObModel* m, int precision) {
  if (!m || precision < 0 || precision > 5) { set_error("ob_model_set_solver: precision must be 0 to 5"); return OB_ERR_INVALID; }
  const Grid& g = m->g;
  if (precision >= 1 && g.nz != 16 && g.nz != 40 && g.nz != 80) {
    set_error("ob_model_set_solver: the tensor-core solve supports nz in {16, 40, 80}");
    return OB_ERR_INVALID;
  }
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "set solver"));
  drop_graphs(m);
  m->solver.destroy();
  OB_TRY(m->solver.create(g.nxp, g.nyp, g.nz, m->dx, m->dz, precision));
  std::vector<float> rc(g.nz), rw(g.nz + 1);
  for (int k = 0; k < g.nz; k++) rc[k] = m->Bh[k * 8 + 2];
  for (int k = 0; k <= g.nz; k++) rw[k] = m->Bh[k * 8 + 3];
  OB_TRY(m->solver.set_density(rc.data(), rw.data()));
  model_bind_solver(m);
  return OB_OK;
}

int ob_model_solver(ObModel* m) { return m ? m->solver.precision : -1; }

int ob_model_set_pair_tiles(ObModel* m, int on) {
  if (!m) { set_error("ob_model_set_pair_tiles: null model"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "set pair tiles"));
  drop_graphs(m);
  return m->solver.tc_set_pairs(on != 0);
}

int ob_model_set_tile_widths(ObModel* m, int bn_x, int bn_y) {
  if (!m) { set_error("ob_model_set_tile_widths: null model"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "set tile widths"));
  drop_graphs(m);
  return m->solver.tc_set_tile_widths(bn_x, bn_y);
}

unsigned ob_model_nan_count(ObModel* m) {
  unsigned h = 0;
  if (m && cudaMemcpy(&h, m->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) h = 0;
  return h;
}

void* ob_model_stream(ObModel* m) { return m ? (void*)m->stream : nullptr; }

void ob_hurricane_default(ObHurricane* h) {
  // app.js:1631 and the writeUniforms defaults (model.js:1402-1420); centre at the origin, sfcP for 1000 hPa
  h->ck = 1.3e-3f; h->landMoist = 0.3f; h->sfcP = 100000.f; h->tauRad = 43200.f; h->radCap = 2.f / 86400.f;
  h->blDepth = 1000.f; h->u10f = 0.8f; h->gust = 1.5f; h->thermals = 0.4f / 300.f; h->thermalScale = 1.f;
  h->maritime = 1.f; h->filter4 = 0.003f; h->cdCap = 2.0e-3f; h->dissHeat = 1.f; h->centreX = 0.f; h->centreY = 0.f;
  h->thermalR = 200000.f; h->envR = 300000.f; h->cnOld = 0.4f; h->traj2 = 1.f;
}

// setSurface (model.js:1296-1303): surf nx*ny*4 (land fraction, SST K, 0, 0) or null (no sea); hur null = outbreak
int ob_model_set_surface(ObModel* m, const float* surf, const ObHurricane* hur) {
  if (!m) { set_error("ob_model_set_surface: null model"); return OB_ERR_INVALID; }
  if (m->ens) { set_error("ob_model_set_surface: the model belongs to an ensemble (hurricane mode runs alone)"); return OB_ERR_INVALID; }
  const size_t n2 = size_t(m->g.nx) * m->g.ny;
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "set surface"));
  if (surf) OB_TRY(cuda_status(cudaMemcpy(const_cast<float4*>(m->F.sfc), surf, n2 * sizeof(float4), cudaMemcpyHostToDevice), "surface"));
  else OB_TRY(cuda_status(cudaMemset(const_cast<float4*>(m->F.sfc), 0, n2 * sizeof(float4)), "surface"));
  m->hur_on = hur != nullptr;
  if (hur) m->H = *hur;
  if (m->hur_on && !m->d_vp) {  // the prep field (model.js:1290-1295)
    OB_TRY(cuda_status(cudaMalloc(&m->d_vp, 4 * m->fs * sizeof(float)), "prep field"));
    OB_TRY(cuda_status(cudaMemset(m->d_vp, 0, 4 * m->fs * sizeof(float)), "prep field"));
  } else if (!m->hur_on && m->d_vp) {
    cudaFree(m->d_vp);
    m->d_vp = nullptr;
  }
  for (int c = 0; c < 4; c++) m->F.Vp[c] = m->d_vp ? m->d_vp + c * m->fs : nullptr;
  drop_graphs(m);
  return OB_OK;
}

// the hurricane's parameters alone (its centre follows the storm, app.js hurricaneUpdate)
int ob_model_set_hurricane(ObModel* m, const ObHurricane* hur) {
  if (!m || !hur) { set_error("ob_model_set_hurricane: bad arguments"); return OB_ERR_INVALID; }
  if (!m->hur_on) { set_error("ob_model_set_hurricane: not in hurricane mode (ob_model_set_surface first)"); return OB_ERR_INVALID; }
  m->H = *hur;
  return OB_OK;
}

// setVortex's table (built on the host, model.js:1318-1365): nz x nr of (tangential wind, theta', 0, 0), the centre,
// the table spacing, the moist core's radius and relative humidity; nr = 0 clears it
int ob_model_set_vortex(ObModel* m, const float* tab, int nr, float x, float y, float dr, float moistR, float moistRH) {
  if (!m || nr < 0 || (nr > 0 && (!tab || !(dr > 0.f)))) { set_error("ob_model_set_vortex: bad arguments"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(m->stream), "set vortex"));
  if (m->d_vx) { cudaFree(m->d_vx); m->d_vx = nullptr; }
  m->vortex = nr > 0;
  m->F.vx = nullptr;
  if (m->vortex) {
    const size_t n = size_t(m->g.nz) * nr;
    OB_TRY(cuda_status(cudaMalloc(&m->d_vx, n * sizeof(float4)), "vortex table"));
    OB_TRY(cuda_status(cudaMemcpy(m->d_vx, tab, n * sizeof(float4), cudaMemcpyHostToDevice), "vortex table"));
    m->F.vx = m->d_vx;
    m->vx_nr = nr; m->vx_x = x; m->vx_y = y; m->vx_dr = dr; m->vx_moistR = moistR; m->vx_moistRH = moistRH;
  }
  return OB_OK;
}

// ---- ensembles: every member's pass in one launch per lane ----
// Members are split into lanes (1 or 2) balanced by cell count; each lane runs the step's passes as grouped launches
// on its own streams, so that with two lanes one lane's solve (tensor cores) runs beside the other's stencils.
struct ObEnsemble {
  std::vector<ObModel*> mem;
  std::vector<float> dt;
  cudaStream_t stream = nullptr;  // lane 0's main stream; the ensemble's work is ordered on it
  cudaEvent_t ev_start = nullptr, ev_done = nullptr;
  struct Lane {
    std::vector<int> idx;  // members (indices into mem) at table positions base .. base + idx.size() - 1
    int base = 0;
    cudaStream_t s = nullptr;  // lane 0: the ensemble's stream
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    TcGroup* solve = nullptr;
    uint2* d_map[kGroupPasses] = {};  // block maps of the lane's grouped launches
    int nxy[kGroupPasses] = {}, Z[kGroupPasses] = {};
  } lane[kMaxLanes];
  int nlanes = 1;
  MemberC* d_members = nullptr;  // device copy of the member table, in lane order (the constant upload's source)
  std::vector<MemberC> h_members;
  bool members_valid = false;
  double* d_lsfT = nullptr;      // per member (mem order)
  dim3 shape[kGroupPasses];
  int bn_cap = 256;
  unsigned gen = 0;  // bumped when the tables or the member table change: captured steps are then stale
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    unsigned gen = ~0u;
    int seen = 0;
  } graphs[2];
  bool use_graphs = true;
  int parity = 0;
  std::vector<double> lsfT;  // what the device copy holds (the device updates it as the host does)
  int micro = kMicroPlain;   // every member's microphysics mode (the scheme, or one shared surrogate)
  unsigned* d_err = nullptr; // the grouped surrogate's timeout word
};

// the grouped kernels read their members from one constant-memory table per device: one ensemble at a time
static ObEnsemble* g_ensemble = nullptr;

static void ens_drop_graphs(ObEnsemble* e) {
  for (auto& G : e->graphs) {
    if (G.exec) cudaGraphExecDestroy(G.exec);
    G = ObEnsemble::StepGraph{};
  }
}

static void lane_free(ObEnsemble::Lane& L, bool own_stream) {
  if (L.solve) tc_group_destroy(L.solve);
  for (uint2* p : L.d_map)
    if (p) cudaFree(p);
  for (int i = 0; i < 2; i++) {
    if (L.side[i]) cudaStreamDestroy(L.side[i]);
    if (L.ev_join[i]) cudaEventDestroy(L.ev_join[i]);
  }
  if (L.ev_fork) cudaEventDestroy(L.ev_fork);
  if (own_stream && L.s) cudaStreamDestroy(L.s);
  L = ObEnsemble::Lane{};
}

static void ens_free(ObEnsemble* e) {
  if (!e) return;
  ens_drop_graphs(e);
  for (ObModel* m : e->mem)
    if (m && m->ens == e) {
      m->stream = m->own_stream;
      m->ens = nullptr;
    }
  for (int l = 0; l < kMaxLanes; l++) lane_free(e->lane[l], l > 0);
  for (void* p : {(void*)e->d_members, (void*)e->d_lsfT, (void*)e->d_err})
    if (p) cudaFree(p);
  if (e->ev_start) cudaEventDestroy(e->ev_start);
  if (e->ev_done) cudaEventDestroy(e->ev_done);
  if (e->stream) cudaStreamDestroy(e->stream);
  if (g_ensemble == e) g_ensemble = nullptr;
  delete e;
}

static int ens_build_tables(ObEnsemble* e) {
  for (int l = 0; l < e->nlanes; l++) {
    ObEnsemble::Lane& L = e->lane[l];
    std::vector<Grid> grids;
    std::vector<int> pos;
    for (size_t q = 0; q < L.idx.size(); q++) {
      grids.push_back(e->mem[L.idx[q]]->g);
      pos.push_back(L.base + int(q));
    }
    std::vector<uint2> map;
    for (int p = 0; p < kGroupPasses; p++) {
      const int Z = group_map(grids.data(), pos.data(), int(grids.size()), p, e->shape[p], map);
      if (Z < 1) { set_error("ensemble: members must share nz"); return OB_ERR_INVALID; }
      if (L.d_map[p]) { cudaFree(L.d_map[p]); L.d_map[p] = nullptr; }
      OB_TRY(cuda_status(cudaMalloc(&L.d_map[p], map.size() * sizeof(uint2)), "ensemble block maps"));
      OB_TRY(cuda_status(cudaMemcpy(L.d_map[p], map.data(), map.size() * sizeof(uint2), cudaMemcpyHostToDevice), "ensemble block maps"));
      L.nxy[p] = int(map.size());
      L.Z[p] = Z;
    }
  }
  e->gen++;
  return OB_OK;
}

// splits the members into k lanes (largest first onto the lane with fewer cells), with a grouped solve per lane
static int ens_set_lanes(ObEnsemble* e, int k) {
  const int n = int(e->mem.size());
  if (k < 1 || k > kMaxLanes || k > n) { set_error("ensemble: %d lanes for %d members (1..%d)", k, n, kMaxLanes); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(e->stream), "ensemble lanes"));
  for (int l = 1; l < kMaxLanes; l++)
    if (e->lane[l].s) OB_TRY(cuda_status(cudaStreamSynchronize(e->lane[l].s), "ensemble lanes"));
  ens_drop_graphs(e);
  for (int l = 0; l < kMaxLanes; l++) {
    ObEnsemble::Lane& L = e->lane[l];
    if (L.solve) { tc_group_destroy(L.solve); L.solve = nullptr; }
    L.idx.clear();
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const Grid &ga = e->mem[a]->g, &gb = e->mem[b]->g;
    return long(ga.nx) * ga.ny * ga.nz > long(gb.nx) * gb.ny * gb.nz;
  });
  std::vector<long> load(k, 0);
  for (int i : order) {
    int best = 0;
    for (int l = 1; l < k; l++)
      if (load[l] < load[best]) best = l;
    e->lane[best].idx.push_back(i);
    const Grid& g = e->mem[i]->g;
    load[best] += long(g.nx) * g.ny * g.nz;
  }
  int base = 0;
  for (int l = 0; l < k; l++) {
    ObEnsemble::Lane& L = e->lane[l];
    std::sort(L.idx.begin(), L.idx.end());
    L.base = base;
    base += int(L.idx.size());
    if (!L.s) {
      if (l == 0) L.s = e->stream;
      else OB_TRY(cuda_status(cudaStreamCreateWithFlags(&L.s, cudaStreamNonBlocking), "ensemble stream"));
    }
    for (int i = 0; i < 2; i++) {
      if (!L.side[i]) OB_TRY(cuda_status(cudaStreamCreateWithFlags(&L.side[i], cudaStreamNonBlocking), "ensemble stream"));
      if (!L.ev_join[i]) OB_TRY(cuda_status(cudaEventCreateWithFlags(&L.ev_join[i], cudaEventDisableTiming), "ensemble event"));
    }
    if (!L.ev_fork) OB_TRY(cuda_status(cudaEventCreateWithFlags(&L.ev_fork, cudaEventDisableTiming), "ensemble event"));
    std::vector<PoissonPlan*> plans;
    std::vector<float*> phi;
    std::vector<const float*> rhs;
    for (int i : L.idx) {
      plans.push_back(&e->mem[i]->solver);
      phi.push_back(e->mem[i]->F.phi);
      rhs.push_back(e->mem[i]->F.rhs);
    }
    OB_TRY(tc_group_create(plans.data(), phi.data(), rhs.data(), int(plans.size()), &L.solve));
    OB_TRY(tc_group_set_cap(L.solve, e->bn_cap));
    int nsm = 148, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) nsm = 148;
    tc_group_set_ctas(L.solve, k > 1 ? (nsm + k - 1) / k : 0);
  }
  e->nlanes = k;
  e->members_valid = false;  // table order follows the lanes
  return ens_build_tables(e);
}

// member table for this step (uniforms for each member's dt), in lane order; re-uploaded when it changed
static int ens_prepare(ObEnsemble* e) {
  const int n = int(e->mem.size());
  bool changed = !e->members_valid, lsf_changed = false;
  for (int l = 0; l < e->nlanes; l++) {
    const ObEnsemble::Lane& L = e->lane[l];
    for (size_t q = 0; q < L.idx.size(); q++) {
      const int i = L.idx[q];
      ObModel* m = e->mem[i];
      if (m->parity != e->parity) {
        set_error("ensemble: member %d was stepped alone an odd number of times (its step parity differs)", i);
        return OB_ERR_INVALID;
      }
      if (m->lsfT != e->lsfT[i]) {  // stepped alone since the last ensemble step
        e->lsfT[i] = m->lsfT;
        lsf_changed = true;
      }
      if (m->hur_on) { set_error("ensemble: member %d is in hurricane mode (it runs alone)", i); return OB_ERR_INVALID; }
      write_uniforms(m, e->dt[i], e->stream);
      const int mode = micro_mode(m);
      if (mode == kMicroRecord) { set_error("ensemble: member %d records microphysics pairs (record on the model alone)", i); return OB_ERR_INVALID; }
      if (l == 0 && q == 0) e->micro = mode;
      if (mode != e->micro) { set_error("ensemble: the members must all use the scheme or all the surrogate (member %d differs)", i); return OB_ERR_INVALID; }
      if (mode == kMicroSurrogate && m->surr_net != e->mem[e->lane[0].idx[0]]->surr_net) {
        set_error("ensemble: the members' surrogates must be one network (member %d differs)", i);
        return OB_ERR_INVALID;
      }
      OB_TRY(prepare_micro(m));
      MemberC c;
      std::memset(&c, 0, sizeof(c));
      c.g = m->g;
      c.U = m->U;
      c.F = m->F;
      c.lsfT = e->d_lsfT + i;
      c.micro = mode;
      MemberC& slot = e->h_members[L.base + q];
      if (std::memcmp(&c, &slot, sizeof(MemberC)) != 0) {
        slot = c;
        changed = true;
      }
    }
  }
  if (lsf_changed) {
    OB_TRY(cuda_status(cudaMemcpyAsync(e->d_lsfT, e->lsfT.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->stream), "ensemble members"));
    OB_TRY(cuda_status(cudaStreamSynchronize(e->stream), "ensemble members"));
  }
  if (changed) {
    OB_TRY(cuda_status(cudaMemcpyAsync(e->d_members, e->h_members.data(), sizeof(MemberC) * n, cudaMemcpyHostToDevice, e->stream), "ensemble members"));
    OB_TRY(cuda_status(cudaStreamSynchronize(e->stream), "ensemble members"));
    e->members_valid = true;
    e->gen++;
  }
  return OB_OK;
}

static int lane_enqueue(ObEnsemble* e, int l) {
  ObEnsemble::Lane& L = e->lane[l];
  const int par = e->parity;
  cudaStream_t s = L.s;
  auto G = [&](int p, cudaStream_t st) { launch_group(p, L.d_map[p], L.nxy[p], L.Z[p], e->shape[p], par, st, e->micro); };
  G(kGroupLSF, s);
  G(kGroupCI, s);
  cudaEventRecord(L.ev_fork, s);
  for (int i = 0; i < 2; i++) cudaStreamWaitEvent(L.side[i], L.ev_fork, 0);
  G(kGroupNUT, L.side[0]);
  cudaEventRecord(L.ev_join[0], L.side[0]);
  G(kGroupADVQ1, L.side[1]);
  G(kGroupADVQ2, L.side[1]);
  cudaEventRecord(L.ev_join[1], L.side[1]);
  G(kGroupADVV1, s);
  G(kGroupADVV2, s);
  for (int i = 0; i < 2; i++) cudaStreamWaitEvent(s, L.ev_join[i], 0);
  G(kGroupPHYS, s);
  if (e->micro == kMicroSurrogate) {
    const ObModel* m0 = e->mem[L.idx[0]];
    launch_surrogate_grp(e->d_members + L.base, int(L.idx.size()), par, m0->d_surr, m0->surr_norm, e->d_err, s);
  }
  G(kGroupDIV, s);
  OB_TRY(tc_group_solve(L.solve, s));
  G(kGroupPROJ, s);
  G(kGroupRAIN, s);
  return OB_OK;
}

static int ens_enqueue(ObEnsemble* e, cudaStream_t s) {
  const int n = int(e->mem.size());
  if (group_upload_members(e->d_members, n, s) != 0) { set_error("ensemble: member table upload failed"); return OB_ERR_DEVICE; }
  if (e->nlanes > 1) {
    cudaEventRecord(e->ev_start, s);
    for (int l = 1; l < e->nlanes; l++) cudaStreamWaitEvent(e->lane[l].s, e->ev_start, 0);
  }
  for (int l = 0; l < e->nlanes; l++) OB_TRY(lane_enqueue(e, l));
  for (int l = 1; l < e->nlanes; l++) {
    cudaEventRecord(e->ev_done, e->lane[l].s);
    cudaStreamWaitEvent(s, e->ev_done, 0);
  }
  return cuda_status(cudaGetLastError(), "ensemble step launch");
}

// one step of every member; captured per parity on its second occurrence and replayed while nothing changed
static int ens_step_once(ObEnsemble* e) {
  OB_TRY(ens_prepare(e));
  cudaStream_t s = e->stream;
  if (!e->use_graphs) {
    OB_TRY(ens_enqueue(e, s));
  } else {
    ObEnsemble::StepGraph& G = e->graphs[e->parity];
    if (G.exec && G.gen == e->gen) {
      OB_TRY(cuda_status(cudaGraphLaunch(G.exec, s), "ensemble graph launch"));
    } else if (G.seen == 0) {
      G.seen = 1;
      OB_TRY(ens_enqueue(e, s));
    } else {
      if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
      OB_TRY(cuda_status(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "ensemble capture"));
      const int rc = ens_enqueue(e, s);
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(s, &graph);
      if (rc != OB_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
      OB_TRY(cuda_status(ec, "ensemble capture"));
      const cudaError_t ei = cudaGraphInstantiate(&G.exec, graph, 0);
      cudaGraphDestroy(graph);
      OB_TRY(cuda_status(ei, "ensemble graph instantiate"));
      G.gen = e->gen;
      OB_TRY(cuda_status(cudaGraphLaunch(G.exec, s), "ensemble graph launch"));
    }
  }
  // the members' host bookkeeping, as model_step_once keeps it
  for (size_t i = 0; i < e->mem.size(); i++) {
    ObModel* m = e->mem[i];
    if (m->time - m->lsfT >= 60 || m->time == 0) m->lsfT = m->time;
    e->lsfT[i] = m->lsfT;
    m->parity = 1 - m->parity;
    m->time += e->dt[i];
    m->steps++;
  }
  e->parity = 1 - e->parity;
  return OB_OK;
}

int ob_ensemble_create(ObModel* const* members, const float* dts, int n, ObEnsemble** out) {
  if (!members || !dts || !out || n < 1) { set_error("ob_ensemble_create: bad arguments"); return OB_ERR_INVALID; }
  *out = nullptr;
  if (n > kMaxMembers) { set_error("ob_ensemble_create: at most %d members", kMaxMembers); return OB_ERR_INVALID; }
  for (int i = 0; i < n; i++) {
    if (!members[i] || !(dts[i] > 0.f)) { set_error("ob_ensemble_create: member %d is null or has dt <= 0", i); return OB_ERR_INVALID; }
    if (members[i]->parity != members[0]->parity) { set_error("ob_ensemble_create: members must be at the same step parity"); return OB_ERR_INVALID; }
    for (int j = 0; j < i; j++)
      if (members[j] == members[i]) { set_error("ob_ensemble_create: member %d appears twice", i); return OB_ERR_INVALID; }
    if (members[i]->ens) { set_error("ob_ensemble_create: member %d already belongs to an ensemble", i); return OB_ERR_INVALID; }
  }
  if (g_ensemble) { set_error("ob_ensemble_create: another ensemble exists (one at a time: its members sit in one constant-memory table)"); return OB_ERR_INVALID; }
  ObEnsemble* e = new ObEnsemble();
  g_ensemble = e;
  e->mem.assign(members, members + n);
  e->dt.assign(dts, dts + n);
  e->h_members.assign(n, MemberC{});
  for (auto& c : e->h_members) std::memset(&c, 0, sizeof(c));
  e->parity = members[0]->parity;
  for (int p = 0; p < kGroupPasses; p++) e->shape[p] = group_default_block(p);
  int rc = cuda_status(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "ensemble stream");
  if (rc == OB_OK) rc = cuda_status(cudaEventCreateWithFlags(&e->ev_start, cudaEventDisableTiming), "ensemble event");
  if (rc == OB_OK) rc = cuda_status(cudaEventCreateWithFlags(&e->ev_done, cudaEventDisableTiming), "ensemble event");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&e->d_members, sizeof(MemberC) * n), "ensemble members");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&e->d_lsfT, sizeof(double) * n), "ensemble members");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&e->d_err, sizeof(unsigned)), "ensemble error word");
  if (rc == OB_OK) rc = cuda_status(cudaMemset(e->d_err, 0, sizeof(unsigned)), "ensemble error word");
  // every member's queued work (reset, uploads) completes before the ensemble's streams take over
  for (int i = 0; i < n && rc == OB_OK; i++) rc = cuda_status(cudaStreamSynchronize(members[i]->stream), "ensemble members");
  if (rc == OB_OK) {
    e->lsfT.resize(n);
    for (int i = 0; i < n; i++) e->lsfT[i] = members[i]->lsfT;
    rc = cuda_status(cudaMemcpy(e->d_lsfT, e->lsfT.data(), sizeof(double) * n, cudaMemcpyHostToDevice), "ensemble members");
  }
  if (rc == OB_OK) rc = ens_set_lanes(e, 1);
  if (rc != OB_OK) { ens_free(e); return rc; }
  // while in the ensemble, each member's own work (field access, maps, radar cuts, a step alone) queues behind and
  // ahead of the ensemble's steps on one stream
  for (ObModel* m : e->mem) {
    m->own_stream = m->stream;
    m->stream = e->stream;
    m->ens = e;
  }
  *out = e;
  return OB_OK;
}

int ob_ensemble_set_lanes(ObEnsemble* e, int lanes) {
  if (!e) { set_error("ob_ensemble_set_lanes: null ensemble"); return OB_ERR_INVALID; }
  return ens_set_lanes(e, lanes);
}

int ob_ensemble_lanes(ObEnsemble* e) { return e ? e->nlanes : 0; }

int ob_ensemble_step(ObEnsemble* e, int nsteps) {
  if (!e || nsteps < 0) { set_error("ob_ensemble_step: bad arguments"); return OB_ERR_INVALID; }
  for (int s = 0; s < nsteps; s++) OB_TRY(ens_step_once(e));
  return OB_OK;
}

int ob_ensemble_timed_steps(ObEnsemble* e, int nsteps, float* ms) {
  if (!e || !ms || nsteps < 0) { set_error("ob_ensemble_timed_steps: bad arguments"); return OB_ERR_INVALID; }
  EventPair ev;
  OB_TRY(ev.create());
  OB_TRY(cuda_status(cudaEventRecord(ev.a, e->stream), "ensemble timed steps"));
  int rc = OB_OK;
  for (int s = 0; s < nsteps && rc == OB_OK; s++) rc = ens_step_once(e);
  if (rc == OB_OK) rc = cuda_status(cudaEventRecord(ev.b, e->stream), "ensemble timed steps");
  if (rc == OB_OK) rc = ev.elapsed(ms, "ensemble timed steps");
  return rc;
}

static int ens_check(ObEnsemble* e) {
  for (int l = 0; l < e->nlanes; l++) OB_TRY(tc_group_check(e->lane[l].solve));
  unsigned h = 0;
  OB_TRY(cuda_status(cudaMemcpy(&h, e->d_err, sizeof(h), cudaMemcpyDeviceToHost), "ensemble error word"));
  if (h) {
    OB_TRY(cuda_status(cudaMemset(e->d_err, 0, sizeof(unsigned)), "ensemble error word"));
    set_error("ensemble surrogate: a tensor-core pipeline wait timed out (code %u)", h);
    return OB_ERR_TIMEOUT;
  }
  return OB_OK;
}

int ob_ensemble_sync(ObEnsemble* e) {
  if (!e) { set_error("ob_ensemble_sync: null ensemble"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(e->stream), "ensemble step"));
  return ens_check(e);
}

int ob_ensemble_set_graphs(ObEnsemble* e, int on) {
  if (!e) { set_error("ob_ensemble_set_graphs: null ensemble"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(e->stream), "ensemble set graphs"));
  ens_drop_graphs(e);
  e->use_graphs = on != 0;
  return OB_OK;
}

// tiles[0 .. OB_ENS_NTILES-1]: block width in x (threads; 128 / width rows) of NUT, ADVV1, ADVV2, DIV, PROJ, then the
// widest transform tile of the solve
static const int kTunedPasses[OB_ENS_NTILES - 1] = {kGroupNUT, kGroupADVV1, kGroupADVV2, kGroupDIV, kGroupPROJ};

int ob_ensemble_set_tiles(ObEnsemble* e, const int* tiles) {
  if (!e || !tiles) { set_error("ob_ensemble_set_tiles: bad arguments"); return OB_ERR_INVALID; }
  for (int t = 0; t < OB_ENS_NTILES - 1; t++)
    if (tiles[t] != 16 && tiles[t] != 32 && tiles[t] != 64 && tiles[t] != 128) {
      set_error("ob_ensemble_set_tiles: block width %d not in {16, 32, 64, 128}", tiles[t]);
      return OB_ERR_INVALID;
    }
  const int cap = tiles[OB_ENS_NTILES - 1];
  if (cap < 16 || cap > 256 || cap % 16) { set_error("ob_ensemble_set_tiles: solve tile width %d not in 16..256 (multiple of 16)", cap); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaDeviceSynchronize(), "ensemble set tiles"));
  for (int t = 0; t < OB_ENS_NTILES - 1; t++) e->shape[kTunedPasses[t]] = dim3(tiles[t], 128 / tiles[t], 1);
  e->bn_cap = cap;
  for (int l = 0; l < e->nlanes; l++) OB_TRY(tc_group_set_cap(e->lane[l].solve, cap));
  return ens_build_tables(e);
}

int ob_ensemble_get_tiles(ObEnsemble* e, int* tiles) {
  if (!e || !tiles) { set_error("ob_ensemble_get_tiles: bad arguments"); return OB_ERR_INVALID; }
  for (int t = 0; t < OB_ENS_NTILES - 1; t++) tiles[t] = int(e->shape[kTunedPasses[t]].x);
  tiles[OB_ENS_NTILES - 1] = e->bn_cap;
  return OB_OK;
}

// device time of one grouped pass (tile slot t) with the ensemble's current state, averaged over reps launches (every
// lane's launch of it, one after another). Each timed pass only rewrites what the step recomputes from the state
// (viscosities, advection scratch and next-state slot, the right-hand side, the solve from it, the projected next
// state), so timing leaves the model state as it was.
int ob_ensemble_time_pass(ObEnsemble* e, int t, int reps, float* ms) {
  if (!e || !ms || t < 0 || t >= OB_ENS_NTILES || reps < 1) { set_error("ob_ensemble_time_pass: bad arguments"); return OB_ERR_INVALID; }
  OB_TRY(ens_prepare(e));
  cudaStream_t s = e->stream;
  if (group_upload_members(e->d_members, int(e->mem.size()), s) != 0) { set_error("ensemble: member table upload failed"); return OB_ERR_DEVICE; }
  EventPair ev;
  OB_TRY(ev.create());
  auto run = [&]() -> int {
    for (int l = 0; l < e->nlanes; l++) {
      if (t < OB_ENS_NTILES - 1) {
        const int p = kTunedPasses[t];
        const ObEnsemble::Lane& L = e->lane[l];
        launch_group(p, L.d_map[p], L.nxy[p], L.Z[p], e->shape[p], e->parity, s, kMicroPlain);
      } else {
        OB_TRY(tc_group_solve(e->lane[l].solve, s));
      }
    }
    return OB_OK;
  };
  int rc = run();  // warm
  if (rc == OB_OK) rc = cuda_status(cudaEventRecord(ev.a, s), "ensemble pass timing");
  for (int r = 0; r < reps && rc == OB_OK; r++) rc = run();
  if (rc == OB_OK) rc = cuda_status(cudaEventRecord(ev.b, s), "ensemble pass timing");
  float el = 0.f;
  if (rc == OB_OK) rc = ev.elapsed(&el, "ensemble pass timing");
  *ms = el / float(reps);
  return rc == OB_OK ? ens_check(e) : rc;
}

// the project's tile autotuner: each tunable slot is set to each of its candidates in turn and its pass timed (the
// passes are independent, so one slot at a time); the fastest candidate of every slot is kept
int ob_ensemble_tune(ObEnsemble* e, int reps, int* tiles, float* ms) {
  if (!e || !tiles || !ms || reps < 1) { set_error("ob_ensemble_tune: bad arguments"); return OB_ERR_INVALID; }
  int cur[OB_ENS_NTILES];
  OB_TRY(ob_ensemble_get_tiles(e, cur));
  static const int kBlockWidths[] = {32, 64, 128, 16};
  static const int kCaps[] = {256, 128, 64};
  for (int t = 0; t < OB_ENS_NTILES; t++) {
    const bool solve = t == OB_ENS_NTILES - 1;
    const int* cand = solve ? kCaps : kBlockWidths;
    const int nc = solve ? 3 : 4;
    int best = cur[t];
    float best_ms = 1e30f;
    for (int c = 0; c < nc; c++) {
      cur[t] = cand[c];
      OB_TRY(ob_ensemble_set_tiles(e, cur));
      float v = 0.f;
      OB_TRY(ob_ensemble_time_pass(e, t, reps, &v));
      if (v < best_ms) { best_ms = v; best = cand[c]; }
    }
    cur[t] = best;
    ms[t] = best_ms;
  }
  OB_TRY(ob_ensemble_set_tiles(e, cur));
  for (int t = 0; t < OB_ENS_NTILES; t++) tiles[t] = cur[t];
  return OB_OK;
}

int ob_ensemble_lsf_times(ObEnsemble* e, double* out) {
  if (!e || !out) { set_error("ob_ensemble_lsf_times: bad arguments"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaMemcpyAsync(out, e->d_lsfT, sizeof(double) * e->mem.size(), cudaMemcpyDeviceToHost, e->stream), "ensemble LSF times"));
  return cuda_status(cudaStreamSynchronize(e->stream), "ensemble LSF times");
}

void* ob_ensemble_stream(ObEnsemble* e) { return e ? (void*)e->stream : nullptr; }

void ob_ensemble_destroy(ObEnsemble* e) {
  if (!e) return;
  cudaDeviceSynchronize();
  ens_free(e);
}

// ---- PoissonDirect ----
struct ObPoisson {
  PoissonPlan plan;
  float* d_rhs = nullptr;
  float* d_phi = nullptr;
  double* d_norm = nullptr;  // residual-norm scratch (ob_poisson_residual)
  cudaStream_t stream = nullptr;
};

int ob_poisson_create(int nx, int ny, int nz, float dx, float dz, int precision, ObPoisson** out) {
  if (!out || precision < 0 || precision > 5) { set_error("ob_poisson_create: bad arguments"); return OB_ERR_INVALID; }
  *out = nullptr;
  ObPoisson* p = new ObPoisson();
  int rc = p->plan.create(nx, ny, nz, dx, dz, precision);
  const size_t n = size_t(nx) * ny * nz * sizeof(float);
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&p->d_rhs, n), "poisson rhs");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&p->d_phi, n), "poisson phi");
  if (rc == OB_OK) rc = cuda_status(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "poisson stream");
  if (rc != OB_OK) {
    ob_poisson_destroy(p);
    return rc;
  }
  *out = p;
  return OB_OK;
}
int ob_poisson_destroy(ObPoisson* p) {
  if (!p) return OB_OK;
  if (p->stream) cudaStreamSynchronize(p->stream);
  p->plan.destroy();
  if (p->d_rhs) cudaFree(p->d_rhs);
  if (p->d_phi) cudaFree(p->d_phi);
  if (p->d_norm) cudaFree(p->d_norm);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return OB_OK;
}
int ob_poisson_set_pair_tiles(ObPoisson* p, int on) {
  if (!p) { set_error("ob_poisson_set_pair_tiles: null handle"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(p->stream), "set pair tiles"));
  return p->plan.tc_set_pairs(on != 0);
}
int ob_poisson_set_tile_widths(ObPoisson* p, int bn_x, int bn_y) {
  if (!p) { set_error("ob_poisson_set_tile_widths: null handle"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaStreamSynchronize(p->stream), "set tile widths"));
  return p->plan.tc_set_tile_widths(bn_x, bn_y);
}
int ob_poisson_residual(ObPoisson* p, double* max_rel, double* l2_rel) {
  if (!p || !max_rel || !l2_rel) { set_error("ob_poisson_residual: null argument"); return OB_ERR_INVALID; }
  if (!p->d_norm) OB_TRY(cuda_status(cudaMalloc(&p->d_norm, (4 * 1024 + 4) * sizeof(double)), "poisson residual"));
  double rel[2];
  OB_TRY(poisson_residual(p->plan, p->d_rhs, p->d_phi, p->d_norm, rel, p->stream));
  *max_rel = rel[0];
  *l2_rel = rel[1];
  return OB_OK;
}
int ob_poisson_set_density(ObPoisson* p, const float* rhoC, const float* rhoW) {
  if (!p || !rhoC || !rhoW) { set_error("ob_poisson_set_density: null argument"); return OB_ERR_INVALID; }
  return p->plan.set_density(rhoC, rhoW);
}
int ob_poisson_solve(ObPoisson* p, const float* rhs, float* phi) {
  if (!p || !rhs || !phi) { set_error("ob_poisson_solve: null argument"); return OB_ERR_INVALID; }
  const size_t n = size_t(p->plan.nx) * p->plan.ny * p->plan.nz * sizeof(float);
  OB_TRY(cuda_status(cudaMemcpyAsync(p->d_rhs, rhs, n, cudaMemcpyHostToDevice, p->stream), "poisson upload"));
  OB_TRY(p->plan.solve(p->d_rhs, p->d_phi, p->stream));
  OB_TRY(cuda_status(cudaMemcpyAsync(phi, p->d_phi, n, cudaMemcpyDeviceToHost, p->stream), "poisson download"));
  OB_TRY(cuda_status(cudaStreamSynchronize(p->stream), "poisson solve"));
  return p->plan.tc_check();
}
int ob_poisson_time(ObPoisson* p, int reps, float* ms) {
  if (!p || reps < 1 || !ms) { set_error("ob_poisson_time: bad arguments"); return OB_ERR_INVALID; }
  EventPair ev;
  OB_TRY(ev.create());
  int rc = p->plan.solve(p->d_rhs, p->d_phi, p->stream);  // warm-up
  if (rc == OB_OK) rc = cuda_status(cudaEventRecord(ev.a, p->stream), "poisson timing");
  for (int r = 0; r < reps && rc == OB_OK; r++) rc = p->plan.solve(p->d_rhs, p->d_phi, p->stream);
  if (rc == OB_OK) rc = cuda_status(cudaEventRecord(ev.b, p->stream), "poisson timing");
  float t = 0.f;
  if (rc == OB_OK) rc = ev.elapsed(&t, "poisson timing");
  *ms = t / reps;
  if (rc == OB_OK) rc = p->plan.tc_check();
  return rc;
}

int ob_poisson_solve_device(ObPoisson* p, const float* d_rhs, float* d_phi, void* stream) {
  if (!p || !d_rhs || !d_phi) { set_error("ob_poisson_solve_device: null argument"); return OB_ERR_INVALID; }
  return p->plan.solve(d_rhs, d_phi, stream ? (cudaStream_t)stream : p->stream);
}

// ---- RadarSim (radar.js:271-413): the device side of one radar ----
struct ObRadar {
  ObModel* m = nullptr;
  uint8_t* d_out = nullptr;  // the volume: every cut's moments, radial-major, one byte per gate (radar.js:298-310)
  size_t bytes = 0;
  float* d_kdp = nullptr;    // OB_RADAR_MAX_RADIALS x ng_dop KDP of the cut being sampled (radar.js:316)
  int ng_dop = 0;
  float* d_tor = nullptr;    // OB_RADAR_MAX_TORNADOES x 8
  int ntor = 0;
  float* d_mom = nullptr;    // moments of the last cut (diagnostic path only)
  size_t mom_count = 0;
};

int ob_radar_create(ObModel* m, size_t volume_bytes, int ng_dop, ObRadar** out) {
  if (!m || !out || volume_bytes == 0 || volume_bytes % 4 != 0 || ng_dop <= 0 || ng_dop % 4 != 0) {
    set_error("ob_radar_create: bad arguments (volume bytes must be a positive multiple of 4, Doppler gates of 4)");
    return OB_ERR_INVALID;
  }
  *out = nullptr;
  ObRadar* r = new ObRadar();
  r->m = m;
  r->bytes = volume_bytes;
  r->ng_dop = ng_dop;
  int rc = cuda_status(cudaMalloc(&r->d_out, volume_bytes), "radar volume");
  if (rc == OB_OK) rc = cuda_status(cudaMemsetAsync(r->d_out, 0, volume_bytes, m->stream), "radar volume");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&r->d_kdp, size_t(OB_RADAR_MAX_RADIALS) * ng_dop * sizeof(float)), "radar KDP");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&r->d_tor, size_t(OB_RADAR_MAX_TORNADOES) * OB_RADAR_TORNADO_FLOATS * sizeof(float)), "radar tornadoes");
  if (rc == OB_OK) rc = cuda_status(cudaMemsetAsync(r->d_tor, 0, size_t(OB_RADAR_MAX_TORNADOES) * OB_RADAR_TORNADO_FLOATS * sizeof(float), m->stream), "radar tornadoes");
  if (rc == OB_OK) rc = cuda_status(cudaStreamSynchronize(m->stream), "radar create");
  if (rc != OB_OK) {
    ob_radar_destroy(r);
    return rc;
  }
  *out = r;
  return OB_OK;
}

int ob_radar_destroy(ObRadar* r) {
  if (!r) return OB_OK;
  if (r->m) cudaStreamSynchronize(r->m->stream);
  for (void* p : {(void*)r->d_out, (void*)r->d_kdp, (void*)r->d_tor, (void*)r->d_mom})
    if (p) cudaFree(p);
  delete r;
  return OB_OK;
}

int ob_radar_set_tornadoes(ObRadar* r, const float* tor, int n) {
  if (!r || n < 0 || (n > 0 && !tor)) { set_error("ob_radar_set_tornadoes: bad arguments"); return OB_ERR_INVALID; }
  r->ntor = n < OB_RADAR_MAX_TORNADOES ? n : OB_RADAR_MAX_TORNADOES;  // the first 64 (radar.js:282)
  if (r->ntor) {
    OB_TRY(cuda_status(cudaMemcpyAsync(r->d_tor, tor, sizeof(float) * OB_RADAR_TORNADO_FLOATS * r->ntor, cudaMemcpyHostToDevice, r->m->stream), "tornadoes"));
    OB_TRY(cuda_status(cudaStreamSynchronize(r->m->stream), "tornadoes"));
  }
  return OB_OK;
}

// every region the cut writes lies inside the volume, the KDP scratch holds the cut, and the tornado count is set
static int radar_check(const ObRadar* r, const ObRadarCut* c) {
  auto whole = [](float v) { return v >= 0.f && v < 16777216.f && float(int(v)) == v; };
  const float nradf = c->cut[3], ngRf = c->gates[0], ngDf = c->gates[1];
  if (!whole(nradf) || !whole(ngRf) || !whole(ngDf) || !whole(c->offB[3])) { set_error("ob_radar_cut: radials, gates and mask must be whole numbers"); return OB_ERR_INVALID; }
  const int nrad = int(nradf), ngR = int(ngRf), ngD = int(ngDf), mask = int(c->offB[3]);
  if (nrad < 1 || nrad > OB_RADAR_MAX_RADIALS || ngR < 4 || ngR % 4 || ngD < 0 || ngD % 4 || ngD > ngR || ngD > r->ng_dop) {
    set_error("ob_radar_cut: %d radials x %d REF / %d Doppler gates do not fit this radar (<= %d radials, <= %d Doppler gates, multiples of 4)",
              nrad, ngR, ngD, OB_RADAR_MAX_RADIALS, r->ng_dop);
    return OB_ERR_INVALID;
  }
  const float offs[6] = {c->offA[0], c->offA[1], c->offA[2], c->offA[3], c->offB[0], c->offB[1]};
  const int bit[6] = {1, 2, 4, 8, 16, 32};
  for (int i = 0; i < 6; i++) {
    if (i > 0 && !(mask & bit[i])) continue;
    if (!whole(offs[i])) { set_error("ob_radar_cut: moment offsets must be whole word counts"); return OB_ERR_INVALID; }
    const size_t end = size_t(offs[i]) * 4 + size_t(nrad) * (i == 0 ? ngR : ngD);
    if (end > r->bytes) { set_error("ob_radar_cut: moment %d ends at byte %zu, past the %zu-byte volume", i, end, r->bytes); return OB_ERR_INVALID; }
  }
  if (!whole(c->phys[3]) || int(c->phys[3]) > r->ntor) { set_error("ob_radar_cut: %g tornadoes requested, %d set", double(c->phys[3]), r->ntor); return OB_ERR_INVALID; }
  if (!(c->gates[3] > 0.f) || !(c->site[3] > 0.f) || !(c->mdl[3] > 0.f) || !(c->mdl2[0] > 0.f) || !(c->nyq[0] > 0.f)) {
    set_error("ob_radar_cut: gate spacing, earth radius, dx, dz and Nyquist must be positive");
    return OB_ERR_INVALID;
  }
  return OB_OK;
}

static int radar_launch(ObRadar* r, const ObRadarCut* c, float* d_mom) {
  RadarU U;
  static_assert(sizeof(ObRadarCut) == sizeof(RadarU), "ObRadarCut layout");
  std::memcpy(&U, c, sizeof(U));
  ObModel* m = r->m;
  launch_radar_cut(U, m->g, m->F, m->parity, r->d_tor, r->d_out, r->d_kdp, d_mom, m->stream);
  return cuda_status(cudaGetLastError(), "radar cut launch");
}

int ob_radar_cut(ObRadar* r, const ObRadarCut* c) {
  if (!r || !c) { set_error("ob_radar_cut: null argument"); return OB_ERR_INVALID; }
  OB_TRY(radar_check(r, c));
  return radar_launch(r, c, nullptr);
}

int ob_radar_cut_moments(ObRadar* r, const ObRadarCut* c, float* host, size_t count) {
  if (!r || !c || !host) { set_error("ob_radar_cut_moments: null argument"); return OB_ERR_INVALID; }
  OB_TRY(radar_check(r, c));
  const size_t need = size_t(c->cut[3]) * size_t(c->gates[0]) * 6;
  if (count != need) { set_error("ob_radar_cut_moments: %zu floats, expected %zu", count, need); return OB_ERR_INVALID; }
  if (r->mom_count < need) {
    if (r->d_mom) cudaFree(r->d_mom);
    r->d_mom = nullptr;
    r->mom_count = 0;
    OB_TRY(cuda_status(cudaMalloc(&r->d_mom, need * sizeof(float)), "radar moments"));
    r->mom_count = need;
  }
  OB_TRY(radar_launch(r, c, r->d_mom));
  OB_TRY(cuda_status(cudaMemcpyAsync(host, r->d_mom, need * sizeof(float), cudaMemcpyDeviceToHost, r->m->stream), "radar moments"));
  return cuda_status(cudaStreamSynchronize(r->m->stream), "radar moments");
}

int ob_radar_write(ObRadar* r, const void* host, size_t bytes) {
  if (!r || !host || bytes > r->bytes) { set_error("ob_radar_write: bad arguments"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaMemcpyAsync(r->d_out, host, bytes, cudaMemcpyHostToDevice, r->m->stream), "radar write"));
  return cuda_status(cudaStreamSynchronize(r->m->stream), "radar write");
}

int ob_radar_level2(ObRadar* r, const ObL2Sweep* sweeps, int nsweeps, const uint8_t* templates, size_t template_bytes,
                    uint8_t* host_out, size_t out_bytes) {
  if (!r || !sweeps || nsweeps < 1 || !templates || !host_out) { set_error("ob_radar_level2: null argument"); return OB_ERR_INVALID; }
  int max_nrad = 0;
  for (int i = 0; i < nsweeps; i++) {
    const ObL2Sweep& s = sweeps[i];
    if (s.nrad < 1 || s.nrad > OB_RADAR_MAX_RADIALS || s.nmom > 6 || s.rec_len < 64 || s.tpl_off + s.rec_len > template_bytes ||
        s.out_off + uint64_t(s.nrad) * s.rec_len > out_bytes) {
      set_error("ob_radar_level2: sweep %d does not fit its template or the output", i);
      return OB_ERR_INVALID;
    }
    for (uint32_t m = 0; m < s.nmom; m++)
      if (s.data_at[m] + s.ngates[m] > s.rec_len || s.src_off[m] + uint64_t(s.nrad) * s.ngates[m] > r->bytes) {
        set_error("ob_radar_level2: sweep %d moment %u lies outside its record or the volume", i, m);
        return OB_ERR_INVALID;
      }
    max_nrad = std::max(max_nrad, int(s.nrad));
  }
  cudaStream_t st = r->m->stream;
  void *d_sw = nullptr, *d_tpl = nullptr, *d_o = nullptr;
  int rc = cuda_status(cudaMalloc(&d_sw, sizeof(ObL2Sweep) * nsweeps), "level2 sweeps");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&d_tpl, template_bytes), "level2 templates");
  if (rc == OB_OK) rc = cuda_status(cudaMalloc(&d_o, out_bytes), "level2 records");
  if (rc == OB_OK) rc = cuda_status(cudaMemcpyAsync(d_sw, sweeps, sizeof(ObL2Sweep) * nsweeps, cudaMemcpyHostToDevice, st), "level2");
  if (rc == OB_OK) rc = cuda_status(cudaMemcpyAsync(d_tpl, templates, template_bytes, cudaMemcpyHostToDevice, st), "level2");
  if (rc == OB_OK) rc = cuda_status(cudaMemsetAsync(d_o, 0, out_bytes, st), "level2");
  if (rc == OB_OK) {
    launch_level2(r->d_out, r->bytes, static_cast<const ObL2Sweep*>(d_sw), nsweeps, max_nrad, static_cast<const uint8_t*>(d_tpl),
                  static_cast<uint8_t*>(d_o), st);
    rc = cuda_status(cudaMemcpyAsync(host_out, d_o, out_bytes, cudaMemcpyDeviceToHost, st), "level2 readback");
  }
  if (rc == OB_OK) rc = cuda_status(cudaStreamSynchronize(st), "level2");
  for (void* p : {d_sw, d_tpl, d_o})
    if (p) cudaFree(p);
  return rc;
}

int ob_radar_read(ObRadar* r, void* host, size_t bytes) {
  if (!r || !host || bytes > r->bytes) { set_error("ob_radar_read: bad arguments"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaMemcpyAsync(host, r->d_out, bytes, cudaMemcpyDeviceToHost, r->m->stream), "radar read"));
  return cuda_status(cudaStreamSynchronize(r->m->stream), "radar read");
}

int ob_radar_kdp(ObRadar* r, float* host, size_t count) {
  if (!r || !host || count > size_t(OB_RADAR_MAX_RADIALS) * r->ng_dop) { set_error("ob_radar_kdp: bad arguments"); return OB_ERR_INVALID; }
  OB_TRY(cuda_status(cudaMemcpyAsync(host, r->d_kdp, count * sizeof(float), cudaMemcpyDeviceToHost, r->m->stream), "radar KDP"));
  return cuda_status(cudaStreamSynchronize(r->m->stream), "radar KDP");
}

}  // extern "C"
