// mi_fit.cu -- kernel (d): batched Levenberg-Marquardt pseudo-Voigt peak fits.
//
// One warp per (frame, peak) window of the eta-averaged lineout.  Window
// selection and initial guesses follow fitPeaks / pf_estimate_initial_params
// (FF_HEDM/src/PeakFit.c:218-250, 275-470): nearest bin to the requested peak
// position (rejected unless closer than 2 bins), ROI of +-half_window bins,
// background guess from the ROI ends, amplitude above background, FWHM from a
// half-maximum walk.  The reference minimises the same least-squares objective
// with NLopt L-BFGS; here it is minimised with Levenberg-Marquardt: residuals,
// Jacobian and model in FP32 on lane-strided samples, the normal equations
// J^T J and J^T r reduced across the warp in FP64 and solved by an FP64
// Cholesky factorisation (every lane solves the same 6x6 system).  The centre
// is carried relative to the window centre so FP32 keeps sub-1e-5 px
// resolution; the final centre and 2-theta are formed in FP64.
//
// Models
//   MI_FIT_PV : b0 + b1*xn + h*(eta*L + (1-eta)*G), L = 1/(1+u^2),
//               G = exp(-ln2*u^2), u = (x-c)/(w/2)           params c,h,w,eta,b0,b1
//   MI_FIT_TCH: area-normalised Thompson-Cox-Hastings pseudo-Voigt + 2-term
//               Chebyshev background (pf_calculate_model, PeakFit.c:50-92;
//               FWHM/eta from sig, gam per pf_tch_eta_fwhm, PeakFit.c:17-42)
//                                                             params A,c,sig,gam,b0,b1
#include <math.h>
#include <stdint.h>

#include "mi_fitcore.cuh"
#include "mi_internal.h"

namespace mi {

constexpr int kNP = 6;
constexpr int kMaxWin = 1024;  // samples per window (lane-strided)

struct FitArgs {
  const double *x, *lo, *peaks;
  int F, n_x, n_peaks, half, model, max_iter;
  double x_bin, px, lsd;
  double *out;
  int32_t *iters;
};

// model value and gradient at local x (relative to the window centre), xn in [-1, 1]
__device__ inline float model(int kind, const float *p, float xl, float xn, float *g) {
  if (kind == MI_FIT_PV) {
    const float c = p[0], h = p[1], w = fmaxf(p[2], 1e-6f), et = p[3];
    const float hw = 0.5f * w;
    const float u = (xl - c) / hw, u2 = u * u;
    const float L = 1.0f / (1.0f + u2);
    const float G = expf(-0.69314718f * u2);
    const float P = et * L + (1.0f - et) * G;
    const float dP_du2 = -et * L * L - (1.0f - et) * 0.69314718f * G;
    g[0] = h * dP_du2 * (-2.0f * u / hw);
    g[1] = P;
    g[2] = h * dP_du2 * (-u2 / hw);
    g[3] = h * (L - G);
    g[4] = 1.0f;
    g[5] = xn;
    return p[4] + p[5] * xn + h * P;
  }
  // TCH, area normalised
  const float A = p[0], c = p[1];
  float F, et, dF_ds, dF_dg, de_ds, de_dg;
  tch(p[2], p[3], &F, &et, &dF_ds, &dF_dg, &de_ds, &de_dg);
  const float sg = F * 0.42466090014400953f;  // FWHM / (2 sqrt(2 ln 2))
  const float Gn = 0.3989422804014327f / sg;  // 1 / (sg sqrt(2 pi))
  const float hw = 0.5f * F;
  const float dx = xl - c, dx2 = dx * dx;
  const float eg = expf(-0.5f * dx2 / (sg * sg));
  const float G = Gn * eg;
  const float den = dx2 + hw * hw;
  const float L = 0.3183098861837907f * hw / den;  // (hw/pi) / (dx^2 + hw^2)
  const float P = et * L + (1.0f - et) * G;
  // derivatives w.r.t. centre and FWHM
  const float dG_dc = G * dx / (sg * sg);
  const float dL_dc = L * 2.0f * dx / den;
  const float dsg_dF = 0.42466090014400953f;
  const float dG_dsg = G * (-1.0f / sg + dx2 / (sg * sg * sg));
  const float dL_dhw = 0.3183098861837907f * (den - 2.0f * hw * hw) / (den * den);
  const float dP_dF = et * dL_dhw * 0.5f + (1.0f - et) * dG_dsg * dsg_dF;
  const float dP_de = L - G;
  g[0] = P;
  g[1] = A * (et * dL_dc + (1.0f - et) * dG_dc);
  g[2] = A * (dP_dF * dF_ds + dP_de * de_ds);
  g[3] = A * (dP_dF * dF_dg + dP_de * de_dg);
  g[4] = 1.0f;
  g[5] = xn;
  return p[4] + p[5] * xn + A * P;
}

__device__ inline bool chol_solve(double A[kNP][kNP], const double *b, double *x) {
  double L[kNP][kNP];
  for (int i = 0; i < kNP; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = A[i][j];
      for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
      if (i == j) {
        if (!(s > 0.0)) return false;
        L[i][i] = sqrt(s);
      } else {
        L[i][j] = s / L[j][j];
      }
    }
  double y[kNP];
  for (int i = 0; i < kNP; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= L[i][k] * y[k];
    y[i] = s / L[i][i];
  }
  for (int i = kNP - 1; i >= 0; --i) {
    double s = y[i];
    for (int k = i + 1; k < kNP; ++k) s -= L[k][i] * x[k];
    x[i] = s / L[i][i];
  }
  return true;
}

__device__ inline void clamp_params(int kind, float *p, float half_span, float x_bin) {
  if (kind == MI_FIT_PV) {
    p[0] = fminf(fmaxf(p[0], -half_span), half_span);
    p[1] = fmaxf(p[1], 0.0f);
    p[2] = fminf(fmaxf(p[2], 0.05f * x_bin), 4.0f * half_span);
    p[3] = fminf(fmaxf(p[3], 0.0f), 1.0f);
  } else {
    p[0] = fmaxf(p[0], 0.0f);
    p[1] = fminf(fmaxf(p[1], -half_span), half_span);
    p[2] = fmaxf(p[2], 1e-6f);
    p[3] = fmaxf(p[3], 0.01f);
  }
}

__global__ void k_fit(FitArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wid >= (int64_t)a.F * a.n_peaks) return;
  const int f = (int)(wid / a.n_peaks), pk = (int)(wid % a.n_peaks);
  const double *x = a.x;
  const double *y = a.lo + (int64_t)f * a.n_x;
  double *out = a.out + wid * MI_FIT_NOUT;
  // ---- window (every lane computes the same thing)
  const double loc = a.peaks[pk];
  int best = -1;
  double bd = 1e300;
  for (int i = lane; i < a.n_x; i += 32) {
    const double d = fabs(x[i] - loc);
    if (d < bd || (d == bd && i < best)) { bd = d; best = i; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double od = __shfl_xor_sync(0xffffffffu, bd, o);
    const int ob = __shfl_xor_sync(0xffffffffu, best, o);
    if (od < bd || (od == bd && ob < best)) { bd = od; best = ob; }
  }
  if (best < 0 || !(bd < 2.0 * a.x_bin)) {
    if (lane < MI_FIT_NOUT) out[lane] = 0.0;
    if (lane == 0) a.iters[wid] = -1;
    return;
  }
  const int s0 = max(0, best - a.half), s1 = min(a.n_x - 1, best + a.half);
  const int n = s1 - s0 + 1;
  if (n < kNP + 1 || n > kMaxWin) {
    if (lane < MI_FIT_NOUT) out[lane] = 0.0;
    if (lane == 0) a.iters[wid] = -2;
    return;
  }
  const double xref = x[best];
  const double xlo = x[s0], xhi = x[s1];
  const double xr = fmax(xhi - xlo, 1e-12);
  const float half_span = (float)fmax(xhi - xref, xref - xlo);
  // ---- initial guess (pf_estimate_initial_params)
  const int bgw = max(1, min(5, n / 4));
  double bgs = 0.0;
  for (int i = 0; i < bgw; ++i) bgs += y[s0 + i] + y[s1 - i];
  const double bg = bgs / (2.0 * bgw);
  double amp = y[best] - bg;
  if (amp <= 0) amp = y[best];
  const double hm = bg + 0.5 * amp;
  int li = best - s0, ri = best - s0;
  while (li > 0 && y[s0 + li] > hm) --li;
  while (ri < n - 1 && y[s0 + ri] > hm) ++ri;
  double fwb = (double)(ri - li);
  if (!(fwb > 1.0)) fwb = 2.0;
  const double fwx = fwb * a.x_bin;
  float p[kNP];
  if (a.model == MI_FIT_PV) {
    p[0] = 0.0f; p[1] = (float)amp; p[2] = (float)fwx; p[3] = 0.5f; p[4] = (float)bg; p[5] = 0.0f;
  } else {
    const double fg0 = 0.5 * fwx;
    double sg = (fg0 * 100.0) * (fg0 * 100.0) / 5.545177444479562;
    if (sg < 1e-6) sg = 1.0;
    double gm = fwx * 0.5 * 100.0;
    if (gm < 0.01) gm = 1.0;
    double ar = amp * fwx * 1.5;
    if (ar <= 0) ar = 1.0;
    p[0] = (float)ar; p[1] = 0.0f; p[2] = (float)sg; p[3] = (float)gm; p[4] = (float)bg; p[5] = 0.0f;
  }
  clamp_params(a.model, p, half_span, (float)a.x_bin);
  // ---- LM
  auto eval = [&](const float *pp, double JtJ[kNP][kNP], double *Jtr, double *chi2) {
    double acc[kNP * (kNP + 1) / 2 + kNP + 1];
#pragma unroll
    for (int k = 0; k < kNP * (kNP + 1) / 2 + kNP + 1; ++k) acc[k] = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double xi = x[s0 + i];
      const float xl = (float)(xi - xref);
      const float xn = (float)(2.0 * (xi - xlo) / xr - 1.0);
      float g[kNP];
      const float m = model(a.model, pp, xl, xn, g);
      const float r = (float)(y[s0 + i] - (double)m);
      int q = 0;
#pragma unroll
      for (int u = 0; u < kNP; ++u)
#pragma unroll
        for (int v = 0; v <= u; ++v) acc[q++] += (double)g[u] * (double)g[v];
#pragma unroll
      for (int u = 0; u < kNP; ++u) acc[q++] += (double)g[u] * (double)r;
      acc[q] += (double)r * (double)r;
    }
    int q = 0;
#pragma unroll
    for (int u = 0; u < kNP; ++u)
#pragma unroll
      for (int v = 0; v <= u; ++v) {
        const double s = warp_sum(acc[q++]);
        if (JtJ) { JtJ[u][v] = s; JtJ[v][u] = s; }
      }
#pragma unroll
    for (int u = 0; u < kNP; ++u) {
      const double s = warp_sum(acc[q++]);
      if (Jtr) Jtr[u] = s;
    }
    *chi2 = warp_sum(acc[q]);
  };
  double JtJ[kNP][kNP], Jtr[kNP], chi2;
  eval(p, JtJ, Jtr, &chi2);
  double lam = 1e-3;
  int it = 0, stall = 0;
  for (; it < a.max_iter; ++it) {
    double A[kNP][kNP], d[kNP];
    for (int u = 0; u < kNP; ++u)
      for (int v = 0; v < kNP; ++v) A[u][v] = JtJ[u][v] + (u == v ? lam * fmax(JtJ[u][u], 1e-30) : 0.0);
    bool ok = chol_solve(A, Jtr, d);
    float pn[kNP];
    for (int u = 0; u < kNP; ++u) pn[u] = ok ? (float)((double)p[u] + d[u]) : p[u];
    clamp_params(a.model, pn, half_span, (float)a.x_bin);
    double c2n;
    eval(pn, nullptr, nullptr, &c2n);
    if (ok && c2n <= chi2) {
      double rel = 0.0;
      for (int u = 0; u < kNP; ++u)
        rel = fmax(rel, fabs((double)pn[u] - (double)p[u]) / fmax(fabs((double)p[u]), 1e-3));
      const double dec = chi2 - c2n;
      for (int u = 0; u < kNP; ++u) p[u] = pn[u];
      eval(p, JtJ, Jtr, &chi2);
      lam = fmax(lam * 0.1, 1e-12);
      if (rel < 1e-6 || dec <= 1e-9 * chi2) {
        if (++stall >= 2) { ++it; break; }
      } else {
        stall = 0;
      }
    } else {
      lam *= 10.0;
      if (lam > 1e12) { ++it; break; }
    }
  }
  // ---- outputs (FP64): [area, center, sig, gam, fwhm, eta, chi2_dof, height, bg0, bg1, 2theta]
  if (lane == 0) {
    double area, center, sig, gam, fw, et, height;
    if (a.model == MI_FIT_PV) {
      center = xref + (double)p[0];
      height = p[1];
      fw = p[2];
      et = p[3];
      area = height * fw * (et * 1.5707963267948966 + (1.0 - et) * 1.0644670194312262);
      sig = 0.0;
      gam = 0.0;
    } else {
      float F, e2, t0, t1, t2, t3;
      tch(p[2], p[3], &F, &e2, &t0, &t1, &t2, &t3);
      area = p[0];
      center = xref + (double)p[1];
      sig = p[2];
      gam = p[3];
      fw = F;
      et = e2;
      const double sgm = fw * 0.42466090014400953;
      height = area * (et * (2.0 / (3.141592653589793 * fw)) + (1.0 - et) * 0.3989422804014327 / sgm);
    }
    out[0] = area;
    out[1] = center;
    out[2] = sig;
    out[3] = gam;
    out[4] = fw;
    out[5] = et;
    out[6] = chi2 / fmax((double)(n - kNP), 1.0);
    out[7] = height;
    out[8] = p[4];
    out[9] = p[5];
    out[10] = (a.px > 0 && a.lsd > 0) ? atan(center * a.px / a.lsd) * 57.29577951308232 : 0.0;
    a.iters[wid] = it;
  }
}

}  // namespace mi

using namespace mi;

extern "C" int mi_fit_batch(const double *x, const double *lineouts, int n_frames, int n_x, const double *peaks,
                            int n_peaks, const mi_fit_opts *opts, double *out, int32_t *iters, void *stream) {
  if (!x || !lineouts || !peaks || !opts || !out || !iters) return set_error(MI_E_ARG, "mi_fit_batch: null argument");
  if (n_frames < 0 || n_x < 0 || n_peaks < 0) return set_error(MI_E_ARG, "mi_fit_batch: negative size");
  if (opts->model != MI_FIT_PV && opts->model != MI_FIT_TCH)
    return set_error(MI_E_ARG, "mi_fit_batch: unknown model %d", opts->model);
  if (opts->half_window < 3 || 2 * opts->half_window + 1 > kMaxWin)
    return set_error(MI_E_RANGE, "mi_fit_batch: half_window must be in [3, %d]", (kMaxWin - 1) / 2);
  if (!(opts->x_bin > 0)) return set_error(MI_E_ARG, "mi_fit_batch: x_bin must be > 0");
  if (n_frames == 0 || n_peaks == 0 || n_x == 0) return MI_OK;
  FitArgs a;
  a.x = x;
  a.lo = lineouts;
  a.peaks = peaks;
  a.F = n_frames;
  a.n_x = n_x;
  a.n_peaks = n_peaks;
  a.half = opts->half_window;
  a.model = opts->model;
  a.max_iter = opts->max_iter > 0 ? opts->max_iter : 100;
  a.x_bin = opts->x_bin;
  a.px = opts->px_um;
  a.lsd = opts->lsd_um;
  a.out = out;
  a.iters = iters;
  const int64_t warps = (int64_t)n_frames * n_peaks;
  const int64_t blocks = (warps * 32 + 127) / 128;
  if (blocks > INT32_MAX) return set_error(MI_E_RANGE, "mi_fit_batch: too many windows");
  k_fit<<<(unsigned)blocks, 128, 0, (cudaStream_t)stream>>>(a);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}
