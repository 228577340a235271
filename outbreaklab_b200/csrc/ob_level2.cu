// ob_level2.cu — message-31 radial assembly of a NEXRAD Archive II volume on the GPU (sm_100a).
//
// The reference writes Archive II on its server from the gate codes the browser uploads (l2writer.py:91-182): each
// radial is one message 31 of fixed layout per sweep, a template (message header, volume/elevation/radial blocks,
// moment headers) in which only the sequence number, collection time, radial number, azimuth and radial status
// change, followed by the radial's codes of every moment. Here the codes are already in the radar volume in device
// memory (radial-major per moment), so one block per radial copies the sweep's template, drops the codes in and
// patches the per-radial fields (big-endian); the host compresses the records (bzip2) and frames the file.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ob.h"

namespace ob {

__device__ __forceinline__ void be16(uint8_t* p, uint32_t v) { p[0] = uint8_t(v >> 8); p[1] = uint8_t(v); }
__device__ __forceinline__ void be32(uint8_t* p, uint32_t v) {
  p[0] = uint8_t(v >> 24); p[1] = uint8_t(v >> 16); p[2] = uint8_t(v >> 8); p[3] = uint8_t(v);
}

__global__ void __launch_bounds__(256) k_level2(const uint8_t* __restrict__ vol, size_t vol_bytes, const ObL2Sweep* __restrict__ sweeps,
                                                const uint8_t* __restrict__ tpl, uint8_t* __restrict__ out) {
  const ObL2Sweep s = sweeps[blockIdx.y];
  const int ri = blockIdx.x;
  if (ri >= int(s.nrad)) return;
  uint8_t* rec = out + s.out_off + size_t(ri) * s.rec_len;
  const uint8_t* t = tpl + s.tpl_off;
  for (uint32_t b = threadIdx.x; b < s.rec_len; b += blockDim.x) rec[b] = t[b];
  __syncthreads();
  for (uint32_t m = 0; m < s.nmom && m < 6; m++) {
    const size_t src = s.src_off[m] + size_t(ri) * s.ngates[m];
    for (uint32_t g = threadIdx.x; g < s.ngates[m]; g += blockDim.x)
      rec[s.data_at[m] + g] = src + g < vol_bytes ? vol[src + g] : uint8_t(0);
  }
  if (threadIdx.x == 0) {
    // collection time of radial ri: t0 + round-half-even(dur * ri / nrad) ms; Julian day from 1970-01-01 = day 1
    const double tms = s.t0_ms + rint(s.dur_ms * double(ri) / double(s.nrad));
    const long long tm = (long long)tms;
    const long long days = tm / 86400000LL;
    const uint32_t jd = uint32_t(days + 1) & 0xFFFFu, jms = uint32_t(tm - days * 86400000LL);
    const uint32_t seq = (s.seq0 + uint32_t(ri)) & 0xFFFFu;
    double az = fmod(s.az0 + double(ri) * (360.0 / double(s.nrad)), 360.0);
    if (az < 0.0) az += 360.0;
    const float azf = float(az);
    uint8_t status = 1;
    if (ri == 0) status = s.ei == 0 ? 3 : 0;
    if (ri == int(s.nrad) - 1) status = s.ei == s.nsw - 1 ? 4 : 2;
    be16(rec + 16, seq);   // message header: sequence, Julian date, milliseconds
    be16(rec + 18, jd);
    be32(rec + 20, jms);
    uint8_t* d = rec + 28;  // message 31 data header
    be32(d + 4, jms);
    be16(d + 8, jd);
    be16(d + 10, uint32_t(ri + 1));
    be32(d + 12, __float_as_uint(azf));
    d[21] = status;
  }
}

void launch_level2(const uint8_t* vol, size_t vol_bytes, const ObL2Sweep* d_sweeps, int nsweeps, int max_nrad, const uint8_t* d_tpl,
                   uint8_t* d_out, cudaStream_t s) {
  k_level2<<<dim3(max_nrad, nsweeps), 256, 0, s>>>(vol, vol_bytes, d_sweeps, d_tpl, d_out);
}

}  // namespace ob
