/*
 * ob.h — C ABI of the B200-native OutbreakLab storm-model time step.
 *
 * Every entry point is plain C: opaque handles, pointers and sizes, int status codes. A JavaScript (Node) host binds
 * it through N-API / node-ffi; Python binds it through ctypes (outbreaklab_b200/model.py).
 *
 * Each declaration names the reference interface it replaces (file:line in Julianfinnerty/outbreakLab). The
 * reference has no FFI: its boundary is the JS class API of RegionalModel (model.js), PoissonDirect (solver.js)
 * and RadarSim (radar.js).
 *
 * Ownership: the library owns all device memory. Host arrays passed in are copied (the semantics of WebGPU's
 * queue.writeBuffer, util.js:190). Readbacks go into caller-owned buffers.
 * Threading: one host thread per handle. Work runs on the handle's in-order CUDA stream (the WebGPU queue).
 * Errors: every call returns OB_OK or an OB_ERR_* code; ob_last_error() returns the message of the last failure on
 * the calling thread (model.js:1194-1200 turns such failures into a thrown JS Error).
 */
#ifndef OB_H_
#define OB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define OB_OK 0
#define OB_ERR_OOM 1        /* device allocation failed (model.js:1172-1174 "not enough GPU memory") */
#define OB_ERR_INVALID 2    /* bad argument, unsupported mode or size */
#define OB_ERR_DEVICE 3     /* a CUDA call failed, or no CUDA device */
#define OB_ERR_TIMEOUT 4    /* a bounded device-side wait gave up */
#define OB_ERR_NAN 5        /* the state holds NaN/Inf after a step (the reference resets such cells, model.js:904) */

/* ---- fields, in the texel layouts of model.js:1208-1233 ---- */
#define OB_FIELD_V 0    /* (nx+1)(ny+1)(nz+1) x float4 (u at x-face, v at y-face, w at z-face, theta), x fastest */
#define OB_FIELD_Q1 1   /* nx*ny*nz x float4 (qv, qc, qi, qr) */
#define OB_FIELD_Q2 2   /* nx*ny*nz x float4 (qs, qg, Nr per kg, spare) */
#define OB_FIELD_AUX 3  /* nx*ny*nz x float2 (nu_h, nu_v) */
#define OB_FIELD_PHI 4  /* (nx+2p)(ny+2p)nz float: the pressure solve's phi on the padded grid */
#define OB_FIELD_RAIN 5 /* nx*ny double: accumulated surface precipitation (kg/m^2); no counterpart in the reference */
/* Read-only diagnostics of the large-scale forcing and storm-start passes (ob_model_set_field rejects them):
 * the per-column textures lsfA, lsfB (model.js:122-124), ciMap (model.js:277-279) and the target's hydrostatic phi
 * phT (model.js:241), as the last LSF / CI pass left them. */
#define OB_FIELD_LSF_A 6  /* nx*ny x float4 (dT at the ground K, air-mass depth m, qv deficit, moisture depth m) */
#define OB_FIELD_LSF_B 7  /* nx*ny x float4 (du, dv at the ground m/s, wind-anomaly depth m, nudging weight) */
#define OB_FIELD_CI_MAP 8 /* nx*ny x float4 (push strength 0-1, target w m/s, centre height m, half-depth m) */
#define OB_FIELD_PHT 9    /* nx*ny*nz float: target hydrostatic phi (m^2/s^2), x fastest */

/* Physics and numerics knobs: RegionalModel.params (model.js:1176-1180) with the outbreak-mode overrides of
 * app.js:1613. ob_params_default() fills the outbreak defaults. */
typedef struct ObParams {
  float cs, nu0, drag, z0;               /* Smagorinsky cs, background viscosity, semi-slip drag on/off, z0 (m) */
  float spongeW, spongeTau, dampZ, dampTau;
  float autoc, qc0, freeze, noise;       /* Kessler rate, threshold, freezing factor, INIT noise amplitude (K) */
  float mc, vcap, evap, sortQ;           /* MacCormack strength, speed cap, rain evaporation factor, size sorting */
  float ciRate, nudgeTau, lat, moistMix;
  float mcFloor, scheme, evapT, dtScale; /* scheme: 0 Lin-type, 1 Thompson-style; dtScale (app.js:1666) */
} ObParams;

/* Hurricane mode (RegionalModel.setSurface's hur argument, model.js:1296-1303, with the values app.js:1631 passes
 * and the defaults writeUniforms applies, model.js:1402-1420): a warm sea under the domain. */
typedef struct ObHurricane {
  float ck;            /* bulk exchange coefficient of heat and moisture at 10 m */
  float landMoist;     /* moisture availability of land (0..1) */
  float sfcP;          /* base surface pressure (Pa) */
  float tauRad;        /* radiative relaxation time (s) */
  float radCap;        /* cap of the radiative relaxation (K/s) */
  float blDepth;       /* boundary-layer depth (m) */
  float u10f;          /* U10 / lowest-level wind */
  float gust;          /* gustiness (m/s) */
  float thermals;      /* boundary-layer thermal forcing (K/s, 0 = none) */
  float thermalScale;  /* its scale factor */
  float maritime;      /* 1: maritime graupel in the Lin scheme */
  float filter4;       /* 2-dx filter strength per pass (every 4th step, 4x); 0 = off */
  float cdCap;         /* sea drag cap at 10 m */
  float dissHeat;      /* 1: dissipative heating */
  float centreX, centreY;  /* storm centre (model m) for the environment hold and the thermals */
  float thermalR;      /* radius of the thermal forcing (m) */
  float envR;          /* environment-hold radius (m) */
  float cnOld;         /* share of the last step's pressure force applied before advection (0 = none) */
  float traj2;         /* 1: midpoint trajectories */
} ObHurricane;
void ob_hurricane_default(ObHurricane* h);  /* app.js:1631 and model.js:1402-1420 defaults, centre at the origin */

/* Grid: dx (m), nx, ny, nz. dz = 20000/nz and the solver padding gridPad(dx) follow model.js:1122, 1203. */
typedef struct ObGrid {
  int nx, ny, nz;
  float dx;
} ObGrid;

/* one moving boundary (air mass), 148 floats, the packing of RegionalModel.setBoundaries (model.js:1371-1380) */
#define OB_BOUNDARY_FLOATS 148
#define OB_MAX_BOUNDS 8
/* one updraft-nudging event, 12 floats (model.js:1383-1389) */
#define OB_CI_FLOATS 12
#define OB_MAX_CI 256

typedef struct ObModel ObModel;
typedef struct ObPoisson ObPoisson;

/* message of the last failed call on this thread ("" if none) */
const char* ob_last_error(void);
/* library version string */
const char* ob_version(void);
/* fills the outbreak-mode defaults of model.js:1176-1180 + app.js:1613 */
void ob_params_default(ObParams* p);
/* padding of the pressure solve, gridPad (model.js:1122) */
int ob_grid_pad(float dx);

/* ---- RegionalModel (model.js:1156-1496) ---- */
/* replaces RegionalModel.allocate / allocTextures (model.js:1186-1238); scheme is chosen by params */
int ob_model_create(const ObGrid* grid, ObModel** out);
/* replaces RegionalModel.destroy (model.js:1239-1247) */
int ob_model_destroy(ObModel* m);
/* replaces the base-state upload of setSounding (model.js:1276-1288): B = (nz+1)*8 floats, sounding.js:139-142 */
int ob_model_set_base_state(ObModel* m, const float* B, int nz);
/* replaces RegionalModel.params assignment (model.js:1176, app.js:1613) */
int ob_model_set_params(ObModel* m, const ObParams* p);
/* replaces setBoundaries (model.js:1371); n boundaries x OB_BOUNDARY_FLOATS */
int ob_model_set_boundaries(ObModel* m, const float* packed, int n);
/* replaces setCI (model.js:1383); n events x OB_CI_FLOATS, already filtered to the active ones. As writeBuffer, the
 * list is copied at the call (the caller may reuse its array at once); the upload is queued on the model's stream,
 * ordered before the steps queued after it, without waiting for the stream */
int ob_model_set_ci(ObModel* m, const float* events, int n);
/* replaces RegionalModel.reset (model.js:1427-1440): LSF + INIT, phi/rhs cleared, time = steps = parity = 0 */
int ob_model_reset(ObModel* m);
/* replaces encStep (model.js:1442-1476) nsteps times with the same dt; runs on the model's stream */
int ob_model_step(ObModel* m, float dt, int nsteps);
/* waits for the model's stream and reports any device error of the queued work */
int ob_model_sync(ObModel* m);
/* how many times the NaN/Inf guard of the physics pass reset a texel to the base state since the last reset
 * (model.js:904 does the reset silently; the count is this library's addition) */
unsigned ob_model_nan_count(ObModel* m);
/* replaces requestMaps (model.js:1478-1494): 16 floats per column, 4 maps of nx*ny float4 */
int ob_model_maps(ObModel* m, float* out16xN2);
/* ---- ensembles (no counterpart in the reference, which runs one domain per tab) ----
 * An ensemble steps its members together: each pass of the step (LSF, CI, NUT, ADVV1/2, ADVQ1/2, PHYS, DIV, the
 * solve's transforms, tridiagonals and residual, PROJ, rain) is one launch over every member, the members' sizes,
 * spacings, soundings and dt free to differ (they must share nz and the solver precision, use the tensor-core solve,
 * all the scheme or all one surrogate network (ob_model_set_surrogate on each member first: one grouped inference
 * launch serves every member's queue), and sit at the same step parity). The step is captured as a CUDA graph and replayed.
 * Members keep their handles: fields, maps, budgets and radars work on them as usual, queued on the ensemble's stream
 * while they belong to it (so they are ordered with its steps); stepping a member alone in between is allowed (an
 * even number of steps, to keep the parity). At most 48 members; one ensemble at a time (the members sit in one
 * constant-memory table); destroy the ensemble before its members. */
typedef struct ObEnsemble ObEnsemble;
#define OB_ENS_MAX_LANES 2
#define OB_ENS_NTILES 6   /* tunable tiles: block width of NUT, ADVV1, ADVV2, DIV, PROJ; widest solve transform tile */
int ob_ensemble_create(ObModel* const* members, const float* dts, int n, ObEnsemble** out);
/* members split into 1 or 2 lanes balanced by cells (default 1): each lane runs the passes as grouped launches on
 * its own streams, so that one lane's solve overlaps the other's stencils (2 x the launches) */
int ob_ensemble_set_lanes(ObEnsemble* e, int lanes);
int ob_ensemble_lanes(ObEnsemble* e);
int ob_ensemble_step(ObEnsemble* e, int nsteps);                     /* queued on the ensemble's stream */
int ob_ensemble_timed_steps(ObEnsemble* e, int nsteps, float* ms);  /* device time of nsteps steps */
int ob_ensemble_sync(ObEnsemble* e);
int ob_ensemble_set_graphs(ObEnsemble* e, int on);
int ob_ensemble_set_tiles(ObEnsemble* e, const int* tiles);        /* OB_ENS_NTILES values */
int ob_ensemble_get_tiles(ObEnsemble* e, int* tiles);
int ob_ensemble_time_pass(ObEnsemble* e, int tile_slot, int reps, float* ms);
/* the autotuner: times every candidate of every tile slot on the current state, keeps the fastest (tiles, ms:
 * OB_ENS_NTILES each) */
int ob_ensemble_tune(ObEnsemble* e, int reps, int* tiles, float* ms);
/* model time of each member's last LSF pass as the device keeps it (the grouped LSF launch decides on the device) */
int ob_ensemble_lsf_times(ObEnsemble* e, double* out);
void* ob_ensemble_stream(ObEnsemble* e);
void ob_ensemble_destroy(ObEnsemble* e);

/* hurricane mode (RegionalModel.setSurface / setVortex, model.js:1290-1365): surf nx*ny*4 floats (land fraction, SST K,
 * 0, 0) per column or NULL (no sea); hur NULL = outbreak mode. The kernels then run the hurricane branches: sea
 * fluxes, drag and dissipative heating, radiative relaxation, the far-field hold, boundary-layer thermals and the
 * K-profile boundary layer, warm-bubble storm starts, settling cloud ice, maritime graupel, midpoint trajectories,
 * 40 % of the last pressure force carried along the trajectories (WGSL_M_PREP) and the 2-dx filter every 4th step
 * (WGSL_M_FILT). The plain microphysics only; not inside an ensemble. */
int ob_model_set_surface(ObModel* m, const float* surf, const ObHurricane* hur);
int ob_model_set_hurricane(ObModel* m, const ObHurricane* hur);  /* parameters only (e.g. the tracked centre) */
/* setVortex's table, built on the host: nz x nr x 4 floats (tangential wind m/s, theta' K, 0, 0) at radii i*dr; the
 * centre (model m), the moist core's radius (m) and relative humidity; nr = 0 clears it. Read by ob_model_reset. */
int ob_model_set_vortex(ObModel* m, const float* tab, int nr, float x, float y, float dr, float moist_r, float moist_rh);

/* the sub-grid tornado scheme's candidates (tornadoCandidates, app.js:1457-1472), found on the GPU in the maps of the
 * last ob_model_maps call: 7 floats each (i, j, x, y, 1-km vorticity, 2-5 km updraft helicity, max updraft), in no
 * particular order; *count = all candidates found (only the first cap are written) */
int ob_model_tornado_candidates(ObModel* m, float zeta_min, float* out, int cap, int* count);
/* field up/download in the texel layouts above (bytes must match exactly) */
int ob_model_get_field(ObModel* m, int field, void* host, size_t bytes);
int ob_model_set_field(ObModel* m, int field, const void* host, size_t bytes);
/* model time (s), steps and parity (model.js:1156-1158, 1448-1450) */
int ob_model_time(ObModel* m, double* time, int* steps, int* parity);
/* domain budgets in FP64 on the device: sum rho*q_total*dV (kg), sum rho*dV (kg), accumulated surface rain (kg);
 * no counterpart in the reference (it keeps no budgets) */
int ob_model_budgets(ObModel* m, double* water, double* mass, double* rain);
/* the same budgets without waiting, in the manner of requestMaps (model.js:1478-1494): the reductions and their copy
 * to pinned host memory are queued on the model's stream after the work queued so far, and *ticket names the result;
 * ob_model_read_budgets waits for that copy alone (not for work queued after the request) and returns the sums. The
 * results of the last 4 requests can be read; an older ticket fails with OB_ERR_INVALID. No counterpart in the
 * reference. */
int ob_model_request_budgets(ObModel* m, long long* ticket);
int ob_model_read_budgets(ObModel* m, long long ticket, double* water, double* mass, double* rain);
/* nsteps steps bracketed by CUDA events on the model's stream; *ms = their device time (no counterpart in the
 * reference, whose GPUProfiler (util.js:194-230) is never instantiated) */
int ob_model_timed_steps(ObModel* m, float dt, int nsteps, float* ms);
/* one step with CUDA events between its passes; ms[i] = device time of pass i in the order
 * (LSF+CI, NUT, ADVV, ADVQ, PHYS, DIV, SOLVE, PROJ+RAIN). The passes run one after another on the model's stream
 * here (ob_model_step overlaps NUT, ADVV and ADVQ on side streams). Returns the number of passes, or -status. */
#define OB_NPASS 8
int ob_model_profile_step(ObModel* m, float dt, float* ms, int max_passes);
/* replay of captured steps (on by default; no counterpart in the reference): from the second step of each variant
 * (parity, LSF due, microphysics mode) on, ob_model_step replays a CUDA graph of the step instead of launching its
 * ~21 kernels one by one, as long as the step's uniforms and buffers are the ones it was captured with; on = 0
 * launches every kernel directly. Results are identical either way. */
int ob_model_set_graphs(ObModel* m, int on);
/* pressure-solve precision of the model: 0 = fp32 SIMT transforms (the reference's arithmetic), 1 = bf16x3
 * tensor-core transforms, 2 = bf16x3 + one bf16x3 refinement sweep,
 * 3 = bf16x3 + one plain-bf16 refinement sweep, 4 = bf16x3 + two bf16x3 refinement sweeps (the residual at the
 * floor that storing phi in fp32 sets), 5 = a plain-bf16 pass + one bf16x3 refinement sweep (the default where nz is
 * 16, 40 or 80: within 1.5 x the floor, as precision 2 is, for 4 products per transform element instead of 6).
 * No counterpart in the reference. */
int ob_model_set_solver(ObModel* m, int precision);
/* tile shape of the tensor-core solve's transforms: 1 (the default) = tiles of 256 field rows computed by pairs of SMs
 * (a cluster of two CTAs, tcgen05.mma.cta_group::2: each SM loads half of the DST-matrix tile and reads a third less
 * operand data per product), 0 = tiles of 128 rows on single SMs. The results are bit-identical. Precisions 1 to 5
 * only (ob_model_set_solver resets it to the default). No counterpart in the reference. */
int ob_model_set_pair_tiles(ObModel* m, int on);
/* outputs per tile of the x and y transforms (multiples of 16 in 32..256; 0 = automatic), for tuning; the results do
 * not depend on them. Precisions 1 to 5 only (ob_model_set_solver resets them). No counterpart in the reference. */
int ob_model_set_tile_widths(ObModel* m, int bn_x, int bn_y);
int ob_model_solver(ObModel* m);
/* CUDA stream of the model (cudaStream_t) for zero-copy hand-off */
void* ob_model_stream(ObModel* m);

/* ---- PoissonDirect (solver.js:105-165) ---- */
/* replaces new PoissonDirect(nx, ny, nz, dx, dz) (solver.js:106-137); precision 0 = FP32 SIMT transforms,
 * 1 = bf16x3 tensor-core transforms (FP32 accumulate), 2 = the same plus one iterative-refinement sweep on the
 * FP64-accumulated residual, 3 = that sweep in plain bf16, 4 = two bf16x3 refinement sweeps, 5 = a plain-bf16 pass
 * refined by one bf16x3 sweep (precisions 1 to 5 need
 * nz in {16, 40, 80}) */
int ob_poisson_create(int nx, int ny, int nz, float dx, float dz, int precision, ObPoisson** out);
int ob_poisson_destroy(ObPoisson* p);
/* replaces setDensity (solver.js:139-146): rhoC[nz] at centres, rhoW[nz+1] at bottom faces */
int ob_poisson_set_density(ObPoisson* p, const float* rhoC, const float* rhoW);
/* replaces bind + enc (solver.js:147-163): solves on host arrays of nx*ny*nz floats (x fastest) */
int ob_poisson_solve(ObPoisson* p, const float* rhs, float* phi);
/* the same on device pointers, on the given stream (cudaStream_t, may be NULL) */
int ob_poisson_solve_device(ObPoisson* p, const float* d_rhs, float* d_phi, void* stream);
/* device time of one solve on the handle's buffers (the last uploaded right-hand side), averaged over reps solves
 * bracketed by CUDA events; no counterpart in the reference */
int ob_poisson_time(ObPoisson* p, int reps, float* ms);
/* the residual r = rhs - A phi of the handle's last solve (the last uploaded right-hand side and its solution),
 * accumulated in FP64 on the device, A the operator the solve inverts (solver.js:139-146: the horizontal Laplacian
 * with phi = 0 beyond the grid, the z-operator with Neumann ends): *max_rel = max|r| / max|rhs|,
 * *l2_rel = ||r||_2 / ||rhs||_2. A diagnostic of the solve's precision; no counterpart in the reference. */
int ob_poisson_residual(ObPoisson* p, double* max_rel, double* l2_rel);
/* the transforms' tile shape, as ob_model_set_pair_tiles; no counterpart in the reference */
int ob_poisson_set_pair_tiles(ObPoisson* p, int on);
/* the transforms' tile widths, as ob_model_set_tile_widths; no counterpart in the reference */
int ob_poisson_set_tile_widths(ObPoisson* p, int bn_x, int bn_y);

/* ---- RadarSim (radar.js:271-413): virtual WSR-88D gate sampling ----
 * The host keeps RadarSim's VCP tables, volume layout and scan scheduling (radar.js:289-392); the library owns each
 * radar's device buffers and runs the cut (WGSL_R_CUT, radar.js:80-241) and PhiDP (WGSL_R_PHI, radar.js:243-268)
 * kernels on the model's stream, sampling the model's current state. */
#define OB_RADAR_MAX_RADIALS 720      /* super-resolution cuts (radar.js:300) */
#define OB_RADAR_MAX_TORNADOES 64     /* radar.js:282 */
#define OB_RADAR_TORNADO_FLOATS 8     /* x, y, core radius, Vmax, debris top, debris dBZ, debris 0-1, 0 (radar.js:283) */
/* one cut's uniform block RU (radar.js:36-39, filled by encCut radar.js:369-384); angles in radians unless noted */
typedef struct ObRadarCut {
  float site[4];   /* model x, model y, antenna height MSL (m), ke * earth radius (m) */
  float geo[4];    /* lat0, lon0 of the projection, site lat, site lon */
  float cut[4];    /* elevation, first azimuth (deg), azimuth step (deg), radials */
  float gates[4];  /* REF gates, Doppler gates, first gate (m), gate spacing (m) */
  float nyq[4];    /* Nyquist (m/s), time (s), noise seed, system PhiDP (deg) */
  float offA[4];   /* u32 word offsets in the volume of REF, VEL, SW, ZDR */
  float offB[4];   /* word offsets of PHI, RHO; unused; moment mask (REF 1, VEL 2, SW 4, ZDR 8, PHI 16, RHO 32) */
  float mdl[4];    /* nx, ny, nz, dx */
  float mdl2[4];   /* dz, ground MSL, domain x0, domain y0 (projected metres of the model's (0, 0) corner) */
  float phys[4];   /* rho at the ground, echo floor (dBZ), microphysics (0 Lin, 1 Thompson), tornadoes in use */
  float phys2[4];  /* maritime graupel (hurricane mode) 0/1, unused x3 */
} ObRadarCut;
typedef struct ObRadar ObRadar;
/* replaces the buffers addRadar creates (radar.js:313-316): a volume of volume_bytes (every cut's moments, one
 * byte per gate, radial-major) and the KDP scratch for up to OB_RADAR_MAX_RADIALS x ng_dop gates */
int ob_radar_create(ObModel* m, size_t volume_bytes, int ng_dop, ObRadar** out);
/* replaces RadarSim.destroy (radar.js:336-340) for one radar */
int ob_radar_destroy(ObRadar* r);
/* replaces setTornadoes (radar.js:280-286): n x OB_RADAR_TORNADO_FLOATS, the first 64 are kept */
int ob_radar_set_tornadoes(ObRadar* r, const float* tor, int n);
/* replaces encCut's dispatches (radar.js:385-390): samples one cut of the model's current state into the volume,
 * on the model's stream. Rejects (OB_ERR_INVALID) cuts whose moments would fall outside the volume. */
int ob_radar_cut(ObRadar* r, const ObRadarCut* cut);
/* replaces the volume's copyBufferToBuffer + mapAsync readback (radar.js:360-363, 394-401): the first bytes of the
 * volume into a caller buffer, after the queued cuts finish */
int ob_radar_read(ObRadar* r, void* host, size_t bytes);
/* Level II (Archive II message 31) radial records of one volume, assembled on the GPU from the radar volume: replaces
 * the per-sweep radial loop of the server's writer (_sweep_block, l2writer.py:91-158; encode_volume's records,
 * l2writer.py:161-182). The host builds each sweep's radial template (everything that is equal for all radials of
 * the sweep) and describes it below; each radial = the template with the sweep's gate codes dropped in at data_at
 * and its sequence number, collection time, radial number, azimuth and status patched (big-endian). host_out gets
 * every sweep's nrad x rec_len bytes at out_off; compressing the 120-radial records and framing the file stay on
 * the host. */
typedef struct ObL2Sweep {
  uint64_t tpl_off;      /* byte offset of the sweep's radial template in `templates` */
  uint64_t out_off;      /* byte offset of its radial 0 in host_out */
  uint32_t rec_len;      /* bytes per radial record (28-byte message header + message 31) */
  uint32_t nrad;         /* radials */
  uint32_t nmom;         /* moments present (<= 6) */
  uint32_t seq0;         /* message sequence number of radial 0 */
  uint32_t ei, nsw;      /* elevation index, sweeps in the volume */
  double t0_ms, dur_ms;  /* sweep start (epoch ms) and duration (ms) */
  double az0;            /* azimuth of radial 0 (deg); radials step 360 / nrad clockwise */
  uint32_t data_at[6];   /* byte offset of each moment's codes in the record */
  uint32_t ngates[6];
  uint64_t src_off[6];   /* byte offset of each moment's codes (nrad x ngates, radial-major) in the radar volume */
} ObL2Sweep;
int ob_radar_level2(ObRadar* r, const ObL2Sweep* sweeps, int nsweeps, const uint8_t* templates, size_t template_bytes,
                    uint8_t* host_out, size_t out_bytes);
/* upload bytes into the start of the radar volume (no counterpart in the reference: lets a host re-encode a volume
 * it holds, and tests feed known codes) */
int ob_radar_write(ObRadar* r, const void* host, size_t bytes);
/* diagnostics, no counterpart in the reference: the same cut, also returning per gate the moments it quantised
 * (dBZ, Vr, SW, ZDR, rho_hv, KDP; NaN where the gate or moment is empty), radials x REF gates x 6 floats; and the
 * KDP scratch of the last cut (radials x Doppler gates, -1 for empty gates) */
int ob_radar_cut_moments(ObRadar* r, const ObRadarCut* cut, float* host, size_t count);
int ob_radar_kdp(ObRadar* r, float* host, size_t count);

/* ---- diagnostics ----
 * One bf16x3 tensor-core transform as used by the precision-1 solve: C[p] = A * B[p]^T for p < planes, with
 * A[M][K], B[planes][N][K], C[planes][M][N] fp32 host arrays (K a multiple of 8). No counterpart in the reference
 * (its transforms are fp32 SIMT GEMMs, solver.js:12-68); it exists to test the tensor-core kernel in isolation. */
int ob_dst_tc_selftest(int M, int N, int K, int planes, const float* A, const float* B, float* C);

/* ---- microphysics surrogate (no counterpart in the reference) ----
 * A per-cell MLP (12 inputs -> 3 x 128 GELU -> 10 tendencies) that emulates the Thompson-style microphysics block
 * of the physics pass (model.js:775-905, micro2.z = 1). Inputs: (T, p, rho, qv, qc, qr, qi, qs, qg, Nr, Ni, w) of a
 * cell before the block; outputs: its change over one step of (T, qv, qc, qi, qr, qs, qg, Nr, Ni, w). The reference
 * has no ice number (the fourth Q2 channel is a spare) and the block leaves w alone, so those two outputs are never
 * applied. Training pairs come from the model's own plain-scheme steps (ob_model_record_micro); training runs on
 * the GPU (fp32 forward/backward kernels, Adam); inference runs inside the step on the tensor cores (BF16 weights,
 * FP32 accumulation) for the cells the scheme can change, with positivity and total-water conservation enforced
 * and the scheme itself as the fallback for inputs outside the training range. */
#define OB_MLP_NIN 12
#define OB_MLP_NOUT 10
#define OB_MLP_NPARAM 35978  /* W1[128][12] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] W4[10][128] b4[10] */
#define OB_MLP_PAIR 24       /* floats per recorded pair: 12 inputs, 10 tendencies, texel offset (uint32 bits), the
                              * model time of the recorded step */
#define OB_MLP_NNORM 59      /* in_mean[12] in_scale[12] out_scale[10] in_lo[12] in_hi[12] dt */
typedef struct ObMlp ObMlp;
int ob_mlp_create(unsigned seed, ObMlp** out);  /* He-initialised weights from the seed */
int ob_mlp_destroy(ObMlp* n);
int ob_mlp_set_params(ObMlp* n, const float* host, int count);  /* count = OB_MLP_NPARAM; resets Adam */
int ob_mlp_get_params(ObMlp* n, float* host, int count);
/* normalisation: inputs x' = (f(x) - in_mean) * in_scale with f = log(q + 1e-9) for the mixing ratios,
 * log(Nr + 1) for Nr, identity otherwise; outputs y = y' * out_scale; [in_lo, in_hi] is the raw input range the
 * surrogate is trusted on; dt the step of the training pairs */
int ob_mlp_set_norm(ObMlp* n, const float* host, int count);
int ob_mlp_get_norm(ObMlp* n, float* host, int count);
int ob_mlp_reserve_pairs(ObMlp* n, long long capacity);  /* device buffer for recorded pairs; clears the count */
int ob_mlp_pair_count(ObMlp* n, long long* count);
int ob_mlp_read_pairs(ObMlp* n, long long first, long long count, float* host);
int ob_mlp_write_pairs(ObMlp* n, const float* host, long long count);  /* replaces the buffer's pairs */
/* orders the recorded pairs by (model time of their step, texel offset), so that training on them does not depend on
 * the order in which the physics pass appended them (an atomic counter); the pair's last two floats carry the two
 * keys. A recording that passed the buffer's capacity holds a race-dependent subset of its last step's pairs: the sort
 * drops that step (the count becomes the index of its first pair). Allocates scratch for the call (about 1.3 x the
 * pairs' bytes). No counterpart in the reference. */
int ob_mlp_sort_pairs(ObMlp* n);
/* forward + backward on `count` host pairs (in order): the loss (mean squared error of the 8 scheme tendencies in
 * normalised units) and its gradient with respect to every parameter (OB_MLP_NPARAM floats) */
int ob_mlp_grad(ObMlp* n, const float* pairs, int count, double* loss, float* grad);
int ob_mlp_eval(ObMlp* n, const float* pairs, int count, float* out);  /* count x OB_MLP_NOUT tendencies */
/* `steps` Adam steps on batches of `batch` pairs drawn from the recorded pairs; mean loss over the steps. A seed and
 * the recorded pairs fix the result: every batch reduction adds its partial sums in a fixed order. */
int ob_mlp_train(ObMlp* n, int batch, int steps, float lr, unsigned seed, double* mean_loss);
/* the arithmetic of ob_mlp_train and ob_mlp_grad: 1 (the default) = BF16 operands with FP32 accumulation on the
 * tensor cores (tcgen05), the bias, GELU and its derivative, the loss and dY fused into the GEMM epilogues, for
 * batches that are a multiple of 128 (others use mode 0); 0 = FP32 SIMT kernels */
int ob_mlp_set_training(ObMlp* n, int mode);
/* record pairs of the plain scheme into net's buffer on every following step, each candidate cell (one the scheme
 * can change) with probability rate; rate 0 stops */
int ob_model_record_micro(ObModel* m, ObMlp* net, float rate);
/* run the microphysics through a copy of net's current weights from the next step on (NULL: the plain scheme) */
int ob_model_set_surrogate(ObModel* m, const ObMlp* net);
/* cells the last step queued for the surrogate and how many of them fell back to the scheme */
int ob_model_surrogate_stats(ObModel* m, unsigned* queued, unsigned* fallbacks);

/* ---- the pressure solve for callers that cannot allocate device memory ----
 * No counterpart in the reference. For a host that may not call cudaMalloc: a plugin that lives inside another
 * runtime which owns the GPU's memory and hands out only its own fixed budget, or a host whose rules forbid device
 * allocation after start-up. One fp32 solve of
 * rhoC lap_h(phi) + d/dz(rhoW dphi/dz) = rhs on nx*ny*nz with every working buffer in a fixed file-scope device array
 * (about 14 MB, held by each GPU that loads the library until the process exits). All pointers are device pointers
 * owned by the caller: rhoC[nz], rhoW[nz+1], rhs and phi (nx*ny*nz, x fastest); the work is queued on `stream`
 * (cudaStream_t, NULL = default stream). Sizes beyond the limits below return OB_ERR_INVALID. The first call on a
 * device looks up the array's address (cudaGetSymbolAddress), so make that first call before any stream capture.
 * Calls share the one array: two calls whose work overlaps on the GPU (different streams, or different host threads)
 * race and corrupt each other's results; serialise them on one stream. */
#define OB_STATIC_POISSON_MAX_SIDE 256
#define OB_STATIC_POISSON_MAX_NZ 512
#define OB_STATIC_POISSON_MAX_CELLS (1 << 20)
int ob_poisson_solve_static(int nx, int ny, int nz, float dx, float dz, const float* d_rhoC, const float* d_rhoW,
                            const float* d_rhs, float* d_phi, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OB_H_ */
