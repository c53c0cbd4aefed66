// mi_fitcore.cuh -- device helpers shared by the peak fitters (mi_fit.cu, mi_fitjob.cu).
#pragma once

#include <math.h>

namespace mi {

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// TCH FWHM and mixing from (sig [centi-x^2], gam [centi-x]); also d/dsig, d/dgam
__device__ inline void tch(float sig, float gam, float *fw, float *eta, float *dfw_ds, float *dfw_dg,
                           float *deta_ds, float *deta_dg) {
  const float ln2x8 = 5.545177444479562f;
  const float s = fmaxf(sig, 1e-12f);
  const float fg = sqrtf(fmaxf(ln2x8 * s, 0.0f)) / 100.0f;
  const float fl = fmaxf(gam, 1e-6f) / 100.0f;
  const float dfg_ds = (sig > 1e-12f) ? fg / (2.0f * s) : 0.0f;
  const float dfl_dg = (gam > 1e-6f) ? 0.01f : 0.0f;
  const float g2 = fg * fg, g3 = g2 * fg, g4 = g3 * fg, g5 = g4 * fg;
  const float l2 = fl * fl, l3 = l2 * fl, l4 = l3 * fl, l5 = l4 * fl;
  const float P = g5 + 2.69269f * g4 * fl + 2.42843f * g3 * l2 + 4.47163f * g2 * l3 + 0.07842f * fg * l4 + l5;
  float F = powf(fmaxf(P, 1e-30f), 0.2f);
  const float dP_dg = 5.f * g4 + 4.f * 2.69269f * g3 * fl + 3.f * 2.42843f * g2 * l2 + 2.f * 4.47163f * fg * l3 +
                      0.07842f * l4;
  const float dP_dl = 2.69269f * g4 + 2.f * 2.42843f * g3 * fl + 3.f * 4.47163f * g2 * l2 + 4.f * 0.07842f * fg * l3 +
                      5.f * l4;
  const float dF_dP = (F > 1e-15f) ? 0.2f * F / fmaxf(P, 1e-30f) : 0.0f;
  if (F < 1e-15f) F = 1e-15f;
  const float dF_dg = dF_dP * dP_dg, dF_dl = dF_dP * dP_dl;
  const float r = fl / F;
  float e = 1.36603f * r - 0.47719f * r * r + 0.11116f * r * r * r;
  float de_dr = 1.36603f - 2.f * 0.47719f * r + 3.f * 0.11116f * r * r;
  if (e < 0.f || e > 1.f) de_dr = 0.f;
  e = fminf(fmaxf(e, 0.f), 1.f);
  const float dr_dl = 1.0f / F - fl * dF_dl / (F * F);
  const float dr_dg = -fl * dF_dg / (F * F);
  *fw = F;
  *eta = e;
  *dfw_ds = dF_dg * dfg_ds;
  *dfw_dg = dF_dl * dfl_dg;
  *deta_ds = de_dr * dr_dg * dfg_ds;
  *deta_dg = de_dr * dr_dl * dfl_dg;
}

}  // namespace mi
