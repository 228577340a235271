// ob_micro.cuh — the microphysics block of the physics pass (model.js:775-905), shared by the step kernel and the
// surrogate kernel (which falls back to it for inputs outside its training range).
#pragma once
#include "ob_common.cuh"

namespace ob {

// the state the microphysics block reads and changes
struct MCell {
  float T, qv, qc, qi, qr, qs, qg, nr;
};

// The process rates of the Lin-type (micro2.z = 0) or Thompson-style (micro2.z = 1) microphysics on one cell: warm
// rain, ice-phase conversions, melting, rain evaporation, Thompson self-collection and sublimation (model.js:791-892).
// p0 and rho are the level's base-state pressure and density, rs = sqrt(rho_sfc / rho).
__device__ __forceinline__ void micro_processes(const Uni& U, float dt, float p0, float rho, float rs, MCell& m) {
  const bool thm = U.micro2.z > 0.5f;
  float T = m.T, qv = m.qv, qc = m.qc, qi = m.qi, qr = m.qr, qs = m.qs, qg = m.qg, nr = m.nr;
  const float rq = 1000.f * rho;
  // warm rain (model.js:791-799)
  // Clear-air shortcuts below skip only work whose result is exactly zero or a no-op in the reference's
  // arithmetic (every product with a zero mixing ratio is +0), so they change no bit of the output.
  const float pauto = U.micro.x * fmaxf(qc - U.micro.y, 0.f);
  float accr = 0.f;
  if (qc > 0.f) {
    accr = 2.2f * qc * powf(qr, 0.875f);
    if (thm && qr > 1e-9f) {
      const float l = Fall::lamR(qr, nr);
      accr = 3100.f * rho * nr * powf(l, -2.8f) * qc * rs;
    }
  }
  const float da = fminf(pauto * dt, qc);
  const float dc = fminf(accr * dt, qc - da);
  qc -= da + dc;
  qr += da + dc;
  nr += da / 2.68e-10f;
  const float dTc = T - T0K;
  if (dTc < 0.f && qc + qi + qr + qs + qg > 0.f) {  // ice-phase conversions (model.js:801-829)
    const float psaut = 1e-3f * expf(0.025f * dTc) * fmaxf(qi - 6e-4f, 0.f);
    const float psacw = 5.4e-3f * qc * powf(fmaxf(rq * qs, 0.f), 0.81f) * rs;
    const float psaci = 5.4e-3f * qi * powf(fmaxf(rq * qs, 0.f), 0.81f) * expf(0.025f * dTc) * rs;
    const float ewet = 1.f / (1.f + qg / 0.008f);
    const float pgq = powf(fmaxf(rq * qg, 0.f), 0.875f);
    const float pgacw = 3.1e-3f * qc * pgq * rs * ewet;
    const float pgaci = 3.0e-4f * qi * pgq * rs;
    const float pgacr = 3.1e-3f * qr * pgq * rs * ewet;
    const float pgfr = fminf(2e-4f * U.micro.z * (expf(0.66f * fminf(-dTc, 20.f)) - 1.f), 0.08f) * qr;
    const float pgaut = 1e-3f * expf(0.09f * dTc) * fmaxf(qs - 6e-4f, 0.f) * (thm ? 0.25f : 1.f);
    const float a1 = fminf((psaut + psaci + pgaci) * dt, qi);
    const float fs1 = (psaut + psaci) / fmaxf(psaut + psaci + pgaci, 1e-20f);
    qi -= a1;
    qs += a1 * fs1;
    qg += a1 * (1.f - fs1);
    const float a2 = fminf((psacw + pgacw) * dt, qc);
    const float fs2 = psacw / fmaxf(psacw + pgacw, 1e-20f);
    const float rimeS = thm ? 0.95f : 0.7f;
    qc -= a2;
    qs += a2 * fs2 * rimeS;
    qg += a2 * (1.f - fs2 * rimeS);
    float a3 = fminf((pgacr + pgfr) * dt, qr);
    if (T < 235.f) a3 = qr;
    if (qr > 1e-12f) nr *= (qr - a3) / qr;
    qr -= a3;
    qg += a3;
    const float a4 = fminf(pgaut * dt, qs);
    qs -= a4;
    qg += a4;
    T += float(LFCd / CPDd) * (a2 + a3);
  } else if (dTc >= 0.f && (qs > 0.f || qg > 0.f)) {  // melting (model.js:830-848)
    const float m1 = fminf(0.012f * dTc * qs * dt, qs);
    float m2 = fminf(0.0022f * dTc * qg * dt, qg);
    if (thm) {
      if (qg > 1e-9f) {
        const float l = Fall::lamG(qg, rho), n0 = Fall::n0G(qg, rho);
        const float vent = 0.78f / (l * l) + float(0.31 * 0.843 * 1.89 * 5430.0) * powf(U.step.z / rho, 0.25f) * powf(l, -2.945f);
        const float heat = 2.4e-2f * dTc - float(LVCd * 2.26e-5) * rho * (qvsat(T0K, p0, 0.f) - qv);
        m2 = clampf(6.2832f / (rho * float(LFCd)) * heat * n0 * vent * dt, 0.f, qg);
        nr += m2 / qg * n0 / (rho * l);
      }
      if (qs > 1e-9f) {
        const float ls = powf(float(3.14159 * 100.0 * 2e6) / (rho * qs), 0.25f);
        nr += m1 / qs * 2e6f / (rho * ls);
      }
    }
    qs -= m1;
    qg -= m2;
    qr += m1 + m2;
    T -= float(LFCd / CPDd) * (m1 + m2);
  }
  // rain evaporation (model.js:850-872)
  const float qvsl = qr > 0.f ? qvsat1(T, p0, 0.f) : 0.f;
  if (qr > 0.f && qv < qvsl) {
    const float rc = 0.001f * rho * qr;
    const float ern = ((1.6f + 124.9f * powf(rc, 0.2046f)) * powf(rc, 0.525f) / (2.55e8f / (p0 * qvsl) + 5.4e5f)) *
                      ((qvsl - qv) / (0.001f * rho * qvsl));
    const float srt = U.micro2.y > 0.f ? sqrtf(rc / (rc + 0.001f * rho * U.micro2.y)) : 1.f;
    float e = ern * srt * dt * U.turb.z;
    if (thm) {
      const float l = Fall::lamR(qr, nr), n0 = rho * nr * l;
      const float Ap = float(LVCd * LVCd) / (float(2.4e-2 * RVCd) * T * T);
      const float Bp = 1.f / (rho * qvsl * 2.26e-5f);
      const float vent = 0.78f / (l * l) + float(0.31 * 0.843 * 1.827 * 7492.0) * powf(U.step.z / rho, 0.25f) * powf(l, -2.9f);
      e = 6.2832f * (1.f - qv / qvsl) * n0 * vent / (rho * (Ap + Bp)) * dt * U.micro2.w;
    }
    e = clampf(e, 0.f, fminf(qr, qvsl - qv));
    if (thm && qr > 1e-12f) nr *= (qr - e) / qr;
    qr -= e;
    qv += e;
    T -= float(LVCd / CPDd) * e;
  }
  // Thompson: self-collection / breakup (model.js:874-884)
  if (thm) {
    if (qr > 1e-9f) {
      const float dm = 1.817f / Fall::lamR(qr, nr);
      const float fb = clampf(1.f - expf(2300.f * (dm - 1.1e-3f)), -2.f, 1.f);
      nr *= expf(-7.12f * rho * qr * fb * dt);
      nr = clampf(nr, qr * 3.183e5f, qr * 3.183e11f);
    } else nr = 0.f;
  }
  // sublimation (model.js:885-892)
  const bool sub_on = dTc < 0.f && (qs > 0.f || qg > 0.f);
  const float qvsi = sub_on ? qvsat1(T, p0, 1.f) : 0.f;
  if (sub_on && qv < qvsi) {
    const float sub = fmaxf(1.f - qv / qvsi, 0.f);
    float e = fminf((2e-3f * qs + 5e-4f * qg) * sub * dt, (qvsi - qv) * 0.5f);
    const float fsn = qs / fmaxf(qs + qg, 1e-20f);
    e = fminf(e, qs + qg);
    qs -= e * fsn;
    qg -= e * (1.f - fsn);
    qv += e;
    T -= float(LSCd / CPDd) * e;
  }
  m.T = T; m.qv = qv; m.qc = qc; m.qi = qi; m.qr = qr; m.qs = qs; m.qg = qg; m.nr = nr;
}

// the 3-iteration mixed-phase saturation adjustment that closes the block (model.js:893-905)
__device__ __forceinline__ void sat_adjust(float p0, MCell& m) {
  float T = m.T, qv = m.qv, qc = m.qc, qi = m.qi;
  // mixed-phase saturation adjustment, 3 iterations (model.js:893-905)
  const float qi0 = qi;
  float qcl = qc + qi, dsum = 0.f;
  for (int it = 0; it < 3; it++) {
    const float f = fIce(T);
    const float qs_ = qvsat1(T, p0, f);
    const float Lh = mixf(float(LVCd), float(LSCd), f);
    float d = (qv - qs_) / (1.f + Lh * Lh * qs_ / (float(CPDd * RVCd) * T * T));
    d = fmaxf(d, -qcl);
    if (d == 0.f) break;  // nothing changes: the remaining iterations would repeat this one exactly
    qv -= d;
    qcl += d;
    T += Lh / float(CPDd) * d;
    dsum += d;
  }
  const float f = fIce(T);
  qi = f * qcl;
  qc = qcl - qi;
  T += float(LFCd / CPDd) * (qi - qi0 - f * dsum);
  m.T = T; m.qv = qv; m.qc = qc; m.qi = qi;
}

// the whole block (model.js:775-905)
__device__ __forceinline__ void micro_plain(const Uni& U, float dt, float p0, float rho, float rs, MCell& m) {
  micro_processes(U, dt, p0, rho, rs, m);
  sat_adjust(p0, m);
}

// a cell the process rates can change: it holds a hydrometeor (without one, every rate is exactly zero)
__device__ __forceinline__ bool micro_has_hydrometeor(const MCell& m) { return m.qc + m.qi + m.qr + m.qs + m.qg > 0.f; }

// The surrogate's domain: cells holding at least this much condensate (kg/kg). Cells with only traces run the scheme,
// which removes traces exactly (complete evaporation or sublimation, the rain-number reset); a network's small
// errors on them would otherwise leave traces everywhere that never vanish.
constexpr float kSurrogateMinCondensate = 1e-5f;
__device__ __forceinline__ bool surrogate_cell(const MCell& m) {
  return m.qc + m.qi + m.qr + m.qs + m.qg >= kSurrogateMinCondensate;
}

// a cell the microphysics can change: it holds a hydrometeor or is supersaturated. Elsewhere micro_plain only sets
// the Thompson rain number to zero (no rain) and leaves everything else exactly as it is.
__device__ __forceinline__ bool micro_active(const MCell& m, float p0) {
  if (m.qc + m.qi + m.qr + m.qs + m.qg > 0.f) return true;
  return m.qv > qvsat1(m.T, p0, fIce(m.T));
}

}  // namespace ob
