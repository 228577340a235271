// ob_radar.cuh — the virtual radar's uniform block and kernel launcher (ob_radar.cu).
#pragma once
#include <cstdint>

#include "ob_common.cuh"

namespace ob {

// RadarSim's uniform block RU (radar.js:36-39): 11 vec4, the layout of ObRadarCut in ob.h
struct RadarU {
  float4 site;   // model x, model y, antenna height MSL, ke * earth radius
  float4 geo;    // lat0, lon0, site lat, site lon (rad)
  float4 cut;    // elevation (rad), first azimuth (deg), azimuth step (deg), radials
  float4 gates;  // REF gates, Doppler gates, first gate (m), gate spacing (m)
  float4 nyq;    // Nyquist (m/s), time (s), noise seed, system PhiDP (deg)
  float4 offA;   // u32 word offsets of REF, VEL, SW, ZDR in the volume
  float4 offB;   // word offsets of PHI, RHO, -, moment mask (REF 1, VEL 2, SW 4, ZDR 8, PHI 16, RHO 32)
  float4 mdl;    // nx, ny, nz, dx
  float4 mdl2;   // dz, ground MSL, domain x0, domain y0 (projected metres of the model's (0, 0) corner)
  float4 phys;   // rho at the ground, echo floor (dBZ), microphysics (0 Lin, 1 Thompson), sub-grid tornadoes
  float4 phys2;  // maritime graupel (hurricane mode), -, -, -
};
static_assert(sizeof(RadarU) == 44 * sizeof(float), "RadarU must match ObRadarCut");

// R_CUT over every gate of the cut, then R_PHI when the cut carries PhiDP; out = the volume's bytes, kdp = radials x
// Doppler gates scratch, tor = 2 float4 per tornado, mom = optional radials x REF gates x 6 moments
void launch_radar_cut(const RadarU& R, const Grid& g, const Fields& F, int par, const float* tor, uint8_t* out, float* kdp,
                      float* mom, cudaStream_t s);

}  // namespace ob
