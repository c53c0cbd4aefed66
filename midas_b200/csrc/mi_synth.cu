// mi_synth.cu -- seeded synthetic detector frames (benchmark and test input).
//
// Model per pixel of frame f (the powder/omega-sweep workloads of the caking
// benchmarks): flat background + sum over Debye-Scherrer rings of a radial
// pseudo-Voigt (peak-height normalised, shared FWHM, mixing eta) whose height
// carries a cos(2 eta) texture and a per-(frame, ring) uniform drift, plus
// Gaussian single-crystal spots at seeded positions; counts are Poisson
// distributed and the per-pixel dark (dark_mean + N(0, dark_sigma)) is added.
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), counter = (pixel, frame, purpose,
// attempt), key = seed.  Poisson variates: inversion by sequential search for
// mean < 12, otherwise the transformed rejection method with squeeze, PTRS
// (W. Hoermann, "The transformed rejection method for generating Poisson
// random variables", Insurance: Mathematics and Economics 12, 1993).
#include <math.h>
#include <stdint.h>

#include "mi_internal.h"

namespace mi {

struct P4 {
  uint32_t x, y, z, w;
};

__host__ __device__ inline P4 philox4x32_10(P4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)M0 * c.x, p1 = (uint64_t)M1 * c.z;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c = P4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// uniform in (0, 1]
__host__ __device__ inline float u01(uint32_t v) { return ((float)(v >> 8) + 1.0f) * (1.0f / 16777216.0f); }

struct SynthArgs {
  int ny, nz, n_rings, n_spots, poisson;
  float bcy, bcz;
  double px, lsd;
  double T[3][3];
  float rr[32], ra[32];
  float fwhm, mix, texture, bg, drift, spot_sigma, spot_amp, dark_mean, dark_sigma;
  uint32_t k0, k1;
};

enum : uint32_t { kPurposeDark = 1, kPurposeDrift = 2, kPurposeSpot = 3, kPurposeCount = 4 };

__device__ inline void pix_r_eta(const SynthArgs &a, int y, int z, float *R, float *ce2) {
  // untilted-detector projection with the same tilt matrix as the mapper
  const double yc = (-(double)y + a.bcy) * a.px, zc = ((double)z - a.bcz) * a.px;
  const double x0 = a.T[0][1] * yc + a.T[0][2] * zc;
  const double x1 = a.T[1][1] * yc + a.T[1][2] * zc;
  const double x2 = a.T[2][1] * yc + a.T[2][2] * zc;
  const double X = a.lsd + x0;
  const double rad = (a.lsd / X) * sqrt(x1 * x1 + x2 * x2);
  *R = (float)(rad / a.px);
  const double r2 = x1 * x1 + x2 * x2;
  // cos(2 eta) with eta = atan2(-x1, x2): (z^2 - y^2) / r^2
  *ce2 = r2 > 0 ? (float)((x2 * x2 - x1 * x1) / r2) : 1.0f;
}

__device__ inline float dark_value(const SynthArgs &a, int64_t p) {
  const P4 r = philox4x32_10(P4{(uint32_t)p, (uint32_t)(p >> 32), kPurposeDark, 0}, a.k0, a.k1);
  const float u1 = u01(r.x), u2 = u01(r.y);
  const float g = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);  // Box-Muller
  return a.dark_mean + a.dark_sigma * g;
}

__device__ inline float frame_uniform(const SynthArgs &a, int64_t f, uint32_t purpose, uint32_t idx) {
  const P4 r = philox4x32_10(P4{idx, (uint32_t)f, purpose, (uint32_t)(f >> 32)}, a.k0, a.k1);
  return u01(r.x);
}

__device__ inline uint32_t poisson(const SynthArgs &a, float mu, int64_t p, int64_t f) {
  if (!(mu > 0.0f)) return 0;
  uint32_t ctr = 0;
  P4 r = philox4x32_10(P4{(uint32_t)p, (uint32_t)f, kPurposeCount | ((uint32_t)(p >> 32) << 8), ctr}, a.k0, a.k1);
  int used = 0;
  auto next = [&]() -> float {
    if (used == 4) {
      ++ctr;
      r = philox4x32_10(P4{(uint32_t)p, (uint32_t)f, kPurposeCount | ((uint32_t)(p >> 32) << 8), ctr}, a.k0, a.k1);
      used = 0;
    }
    const uint32_t v = used == 0 ? r.x : (used == 1 ? r.y : (used == 2 ? r.z : r.w));
    ++used;
    return u01(v);
  };
  if (mu < 12.0f) {
    // inversion: walk the CDF
    const float u = next();
    float pk = expf(-mu), cdf = pk;
    uint32_t k = 0;
    while (u > cdf && k < 200) {
      ++k;
      pk *= mu / (float)k;
      cdf += pk;
    }
    return k;
  }
  const float smu = sqrtf(mu);
  const float b = 0.931f + 2.53f * smu;
  const float aa = -0.059f + 0.02483f * b;
  const float inv_alpha = 1.1239f + 1.1328f / (b - 3.4f);
  const float vr = 0.9277f - 3.6224f / (b - 2.0f);
  const float lmu = logf(mu);
  for (int it = 0; it < 64; ++it) {
    const float U = next() - 0.5f;
    const float V = next();
    const float us = 0.5f - fabsf(U);
    const float kf = floorf((2.0f * aa / us + b) * U + mu + 0.43f);
    if (us >= 0.07f && V <= vr) return kf < 0 ? 0u : (uint32_t)kf;
    if (kf < 0.0f || (us < 0.013f && V > us)) continue;
    if (logf(V) + logf(inv_alpha) - logf(aa / (us * us) + b) <= -mu + kf * lmu - lgammaf(kf + 1.0f))
      return (uint32_t)kf;
  }
  return (uint32_t)rintf(mu);  // bounded loop: never reached in practice
}

constexpr int kMaxSpots = 256;

// grid: (blocks per frame, n_frames); per-frame parameters are drawn once per block
template <typename T>
__global__ void k_synth(SynthArgs a, int64_t first, T *out, int64_t stride) {
  __shared__ float s_drift[32];
  __shared__ float s_spot[2 * kMaxSpots];
  const int64_t f = first + blockIdx.y;
  for (int k = threadIdx.x; k < a.n_rings; k += blockDim.x)
    s_drift[k] = 1.0f + a.drift * (2.0f * frame_uniform(a, f, kPurposeDrift, k) - 1.0f);
  for (int s = threadIdx.x; s < 2 * a.n_spots; s += blockDim.x)
    s_spot[s] = frame_uniform(a, f, kPurposeSpot, s) * ((s & 1) ? a.nz : a.ny);
  __syncthreads();
  const int64_t n_pix = (int64_t)a.ny * a.nz;
  const float hw = 0.5f * a.fwhm;
  const float lim2 = 36.0f * a.spot_sigma * a.spot_sigma;
  const float inv2s2 = 0.5f / (a.spot_sigma * a.spot_sigma);
  const float hi = sizeof(T) == 2 ? 65535.0f : 2147483647.0f;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pix; p += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(p % a.ny), z = (int)(p / a.ny);
    float R, ce2;
    pix_r_eta(a, y, z, &R, &ce2);
    const float tex = 1.0f + a.texture * ce2;
    float mu = a.bg;
    for (int k = 0; k < a.n_rings; ++k) {
      const float d = R - a.rr[k];
      const float x2 = (d * d) / (hw * hw);
      const float L = 1.0f / (1.0f + x2);
      const float G = expf(-0.69314718f * x2);
      mu += a.ra[k] * s_drift[k] * tex * (a.mix * L + (1.0f - a.mix) * G);
    }
    for (int s = 0; s < a.n_spots; ++s) {
      const float dy = (float)y - s_spot[2 * s], dz = (float)z - s_spot[2 * s + 1];
      const float r2 = dy * dy + dz * dz;
      if (r2 < lim2) mu += a.spot_amp * expf(-r2 * inv2s2);
    }
    const float dk = dark_value(a, p);
    const float cnt = a.poisson ? (float)poisson(a, mu, p, f) : rintf(mu);
    float v = cnt + rintf(dk);
    v = fminf(fmaxf(v, 0.0f), hi);
    out[(int64_t)blockIdx.y * stride + p] = (T)v;
  }
}

__global__ void k_synth_dark(SynthArgs a, float *out) {
  const int64_t n_pix = (int64_t)a.ny * a.nz;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pix; p += (int64_t)gridDim.x * blockDim.x)
    out[p] = dark_value(a, p);
}

static int make_args(const mi_synth_desc *d, SynthArgs *a) {
  if (!d || d->ny < 2 || d->nz < 2 || d->n_rings < 0 || d->n_rings > 32 || d->n_spots < 0 ||
      d->n_spots > kMaxSpots || d->px_um <= 0 ||
      d->lsd_um <= 0)
    return set_error(MI_E_ARG, "mi_synth: bad descriptor");
  a->ny = d->ny;
  a->nz = d->nz;
  a->n_rings = d->n_rings;
  a->n_spots = d->n_spots;
  a->poisson = d->poisson;
  a->bcy = (float)d->bc_y;
  a->bcz = (float)d->bc_z;
  a->px = d->px_um;
  a->lsd = d->lsd_um;
  const double b = d->ty * 0.017453292519943295, c = d->tz * 0.017453292519943295;
  // Ry(ty) * Rz(tz) (tx = 0)
  const double Ry[3][3] = {{cos(b), 0, sin(b)}, {0, 1, 0}, {-sin(b), 0, cos(b)}};
  const double Rz[3][3] = {{cos(c), -sin(c), 0}, {sin(c), cos(c), 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a->T[i][j] = Ry[i][0] * Rz[0][j] + Ry[i][1] * Rz[1][j] + Ry[i][2] * Rz[2][j];
  for (int k = 0; k < 32; ++k) {
    a->rr[k] = k < d->n_rings ? (float)d->ring_r_px[k] : 0.f;
    a->ra[k] = k < d->n_rings ? (float)d->ring_amp[k] : 0.f;
  }
  a->fwhm = (float)d->fwhm_px;
  a->mix = (float)d->mix_eta;
  a->texture = (float)d->texture;
  a->bg = (float)d->background;
  a->drift = (float)d->amp_drift;
  a->spot_sigma = (float)(d->spot_sigma > 0 ? d->spot_sigma : 1.0);
  a->spot_amp = (float)d->spot_amp;
  a->dark_mean = (float)d->dark_mean;
  a->dark_sigma = (float)d->dark_sigma;
  a->k0 = (uint32_t)d->seed;
  a->k1 = (uint32_t)(d->seed >> 32);
  return MI_OK;
}

}  // namespace mi

using namespace mi;

extern "C" {

int mi_synth_frames(const mi_synth_desc *d, int64_t first_frame, int n_frames, int dtype, void *out,
                    int64_t frame_stride, void *stream) {
  SynthArgs a;
  int rc = make_args(d, &a);
  if (rc) return rc;
  if (!out || n_frames < 0 || first_frame < 0) return set_error(MI_E_ARG, "mi_synth_frames: bad output");
  if (frame_stride < (int64_t)d->ny * d->nz) return set_error(MI_E_ARG, "mi_synth_frames: stride < ny*nz");
  if (n_frames == 0) return MI_OK;
  if (n_frames > 65535) return set_error(MI_E_RANGE, "mi_synth_frames: more than 65535 frames per call");
  const int64_t n_pix = (int64_t)d->ny * d->nz;
  int64_t gx = (n_pix + 255) / 256;
  if (gx > 1024) gx = 1024;
  const dim3 grid((unsigned)gx, (unsigned)n_frames);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == MI_DT_U16)
    k_synth<uint16_t><<<grid, 256, 0, s>>>(a, first_frame, (uint16_t *)out, frame_stride);
  else if (dtype == MI_DT_I32)
    k_synth<int32_t><<<grid, 256, 0, s>>>(a, first_frame, (int32_t *)out, frame_stride);
  else
    return set_error(MI_E_UNSUPPORTED, "mi_synth_frames: dtype %d (u16 or i32 only)", dtype);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

int mi_synth_dark(const mi_synth_desc *d, float *out, void *stream) {
  SynthArgs a;
  int rc = make_args(d, &a);
  if (rc) return rc;
  if (!out) return set_error(MI_E_ARG, "mi_synth_dark: null output");
  const int64_t n = (int64_t)d->ny * d->nz;
  int64_t grid = (n + 255) / 256;
  if (grid > 148 * 32) grid = 148 * 32;
  k_synth_dark<<<(unsigned)grid, 256, 0, (cudaStream_t)stream>>>(a, out);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

}  // extern "C"
