// ob_mlp.cuh — the per-cell MLP surrogate of the Thompson-style microphysics: layout shared by the training kernels,
// the tcgen05 inference kernel and the host.
//
// Network: 12 inputs -> 128 -> 128 -> 128 -> 10 outputs, GELU (tanh form) after each hidden layer.
//   inputs  (T, p, rho, qv, qc, qr, qi, qs, qg, Nr, Ni, w) of a cell before the microphysics block; the mixing ratios
//           enter as log(q + 1e-9), Nr as log(Nr + 1), then every input is standardised (x - mean) * scale
//   outputs tendencies over one step of (T, qv, qc, qi, qr, qs, qg, Nr, Ni, w), each scaled by its own spread; the
//           reference's scheme has no ice number (its fourth Q2 channel is a spare) and does not change w, so the
//           last two outputs have scale 0 and are never applied
#pragma once
#include <cstdint>

namespace ob {
namespace mlp {

constexpr int NIN = 12, NH = 128, NOUT = 10, NLOSS = 8;  // NLOSS: outputs that carry a tendency of the scheme
// fp32 master parameters, packed: W1[NH][NIN] b1[NH] W2[NH][NH] b2[NH] W3[NH][NH] b3[NH] W4[NOUT][NH] b4[NOUT]
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NH * NH,
              OW4 = OB3 + NH, OB4 = OW4 + NOUT * NH, NPARAM = OB4 + NOUT;
constexpr int PAIR = 24;  // floats per recorded pair: 12 inputs, 10 tendencies, texel offset (uint bits), pad
constexpr float QEPS = 1e-9f;

// normalisation, the raw input range seen in training (inputs outside it fall back to the scheme) and the time step
// of the training pairs (tendencies are per step; a model stepping with another dt scales them by dt / dt_train)
struct Norm {
  float in_mean[NIN], in_scale[NIN], out_scale[NOUT], in_lo[NIN], in_hi[NIN], dt;
};

#ifdef __CUDACC__
// GELU, tanh form (Hendrycks and Gimpel): g(z) = z/2 (1 + tanh(c (z + a z^3))), c = sqrt(2/pi), a = 0.044715
constexpr float GC = 0.7978845608f, GA = 0.044715f;
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + tanhf(GC * (z + GA * z * z * z))); }
__device__ __forceinline__ float gelu_grad(float z) {
  const float t = tanhf(GC * (z + GA * z * z * z));
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * GC * (1.f + 3.f * GA * z * z);
}
#endif

__host__ __device__ inline float feature(int i, float x) {
  if (i >= 3 && i <= 8) return logf(fmaxf(x, 0.f) + QEPS);
  if (i == 9) return logf(fmaxf(x, 0.f) + 1.f);
  return x;
}

}  // namespace mlp
}  // namespace ob
