// mi_plain.cu -- kernel (a) (cast + dark, 128-bit vector loads) and the plain
// one-frame-per-launch path that runs the reference's own GPU algorithm:
//   process_direct_kernel<T>             FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:1148-1160
//   integrate_noMapMask                  IntegratorFitPeaksGPUStream.cu:975-1050
//     (one thread per bin, heaviest-first bin order, FP32 accumulation,
//      on-the-fly bilinear resampling in gradient mode, FP64 cake)
//   calculate_1D_profile_kernel          IntegratorFitPeaksGPUStream.cu:1162-1254
//   calculate_1D_profile_simple_mean_kernel  IntegratorFitPeaksGPUStream.cu:1256-1334
// The plain path is the baseline the batched kernel is measured against; it is
// written here from the algorithm, not copied.
#include <stdint.h>

#include <algorithm>

#include "mi_internal.h"

namespace mi {

// ---------------------------------------------------------------------------
// kernel (a): out[f][p] = (float)in[f][p] - dark[p], 16-byte loads of the input
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ float cvt(T v) {
  return (float)v;
}

template <typename T>
__global__ void k_cast_vec(const T *__restrict__ in, int64_t n_pixels, int n_frames,
                           const float *__restrict__ dark, float *__restrict__ out) {
  constexpr int V = 16 / sizeof(T);  // elements per 128-bit load
  const int64_t nvec = n_pixels / V;
  const int64_t total = nvec * n_frames;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = i / nvec, v = i - f * nvec;
    const int64_t p0 = v * V;
    union {
      uint4 u;
      T e[V];
    } x;
    x.u = __ldg((const uint4 *)(in + f * n_pixels) + v);
    float r[V];
#pragma unroll
    for (int k = 0; k < V; ++k) r[k] = cvt(x.e[k]);
    if (dark) {
      if (V >= 4) {
#pragma unroll
        for (int k = 0; k < V; k += 4) {
          const float4 d = __ldg((const float4 *)(dark + p0 + k));
          r[k] -= d.x; r[k + 1] -= d.y; r[k + 2] -= d.z; r[k + 3] -= d.w;
        }
      } else {
#pragma unroll
        for (int k = 0; k < V; ++k) r[k] -= __ldg(dark + p0 + k);
      }
    }
    float *o = out + f * n_pixels + p0;
    if (V >= 4 && (n_pixels % 4) == 0) {
#pragma unroll
      for (int k = 0; k < V; k += 4) *(float4 *)(o + k) = make_float4(r[k], r[k + 1], r[k + 2], r[k + 3]);
    } else {
#pragma unroll
      for (int k = 0; k < V; ++k) o[k] = r[k];
    }
  }
}

template <typename T>
__global__ void k_cast_scalar(const T *__restrict__ in, int64_t n_pixels, int n_frames, int64_t start,
                              const float *__restrict__ dark, float *__restrict__ out) {
  const int64_t per = n_pixels - start;
  const int64_t total = per * n_frames;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = i / per, p = start + (i - f * per);
    float r = cvt(in[f * n_pixels + p]);
    if (dark) r -= dark[p];
    out[f * n_pixels + p] = r;
  }
}

static int grid_for(int64_t work, int threads) {
  int64_t g = (work + threads - 1) / threads;
  const int64_t cap = 148 * 16;  // persistent-style cap: 16 CTAs per SM on 148 SMs
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

template <typename T>
static int cast_t(const void *frames, int64_t n_pixels, int n_frames, const float *dark, float *out,
                  cudaStream_t s) {
  constexpr int V = 16 / sizeof(T);
  const T *in = (const T *)frames;
  const bool aligned = ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0) &&
                       (!dark || (uintptr_t)dark % 16 == 0) && (n_pixels % V == 0);
  int64_t start = 0;
  if (aligned) {
    const int64_t work = (n_pixels / V) * n_frames;
    k_cast_vec<T><<<grid_for(work, 256), 256, 0, s>>>(in, n_pixels, n_frames, dark, out);
    MI_CUDA(cudaGetLastError());
    start = n_pixels;
  }
  if (start < n_pixels) {
    k_cast_scalar<T><<<grid_for((n_pixels - start) * n_frames, 256), 256, 0, s>>>(in, n_pixels, n_frames,
                                                                                start, dark, out);
    MI_CUDA(cudaGetLastError());
  }
  return MI_OK;
}

int launch_cast(const void *frames, int dtype, int64_t n_pixels, int n_frames, const float *dark, float *out,
                cudaStream_t s) {
  switch (dtype) {
    case MI_DT_U8: return cast_t<uint8_t>(frames, n_pixels, n_frames, dark, out, s);
    case MI_DT_U16: return cast_t<uint16_t>(frames, n_pixels, n_frames, dark, out, s);
    case MI_DT_U32: return cast_t<uint32_t>(frames, n_pixels, n_frames, dark, out, s);
    case MI_DT_I64: return cast_t<int64_t>(frames, n_pixels, n_frames, dark, out, s);
    case MI_DT_F32: return cast_t<float>(frames, n_pixels, n_frames, dark, out, s);
    case MI_DT_F64: return cast_t<double>(frames, n_pixels, n_frames, dark, out, s);
    case MI_DT_I32: return cast_t<int32_t>(frames, n_pixels, n_frames, dark, out, s);
  }
  return set_error(MI_E_ARG, "unknown dtype %d", dtype);
}

// ---------------------------------------------------------------------------
// plain integration: one thread per bin (bins visited heaviest first)
// ---------------------------------------------------------------------------
struct PlainArgs {
  const int32_t *nmap, *sorted, *off;
  const float *w, *aw, *dr, *py, *pz;
  const double *area_in;
  const float *img;
  double *cake;
  int64_t n_bins;
  int ny, nz, mode, sem, normalize;
  float bc_y, bc_z;
};

__global__ void k_plain_integrate(PlainArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_bins) return;
  const int b = a.sorted[t];
  const int cnt = a.nmap[2 * b], base = a.nmap[2 * b + 1];
  float I = 0.0f, A = 0.0f;
  for (int k = 0; k < cnt; ++k) {
    const int64_t j = (int64_t)base + k;
    const float w = a.w[j];
    float v = 0.0f;
    if (a.mode == MI_MODE_FLOOR) {
      const int o = a.off[j];
      v = (o >= 0) ? __ldg(a.img + o) : 0.0f;
    } else {
      float ry = a.py[j], rz = a.pz[j];
      if (a.mode == MI_MODE_GRADIENT) {
        const float dy = ry - a.bc_y, dz = rz - a.bc_z;
        const float R = sqrtf(dy * dy + dz * dz);
        if (R > 1.0f) {
          const float d = a.dr[j];
          ry -= d * dy / R;
          rz -= d * dz / R;
        }
      }
      int iy = (int)floorf(ry), iz = (int)floorf(rz);
      float fy = ry - (float)iy, fz = rz - (float)iz;
      if (iy < 0) { iy = 0; fy = 0.0f; }
      if (iy >= a.ny - 1) { iy = a.ny - 2; fy = 1.0f; }
      if (iz < 0) { iz = 0; fz = 0.0f; }
      if (iz >= a.nz - 1) { iz = a.nz - 2; fz = 1.0f; }
      const float *p = a.img + (int64_t)iz * a.ny + iy;
      v = __ldg(p) * (1.0f - fy) * (1.0f - fz) + __ldg(p + 1) * fy * (1.0f - fz) +
          __ldg(p + a.ny) * (1.0f - fy) * fz + __ldg(p + a.ny + 1) * fy * fz;
    }
    I += v * w;
    A += a.aw[j];
  }
  double out;
  if (a.sem == MI_SEM_GPUSTREAM) {
    out = (A > (float)kAreaThreshold) ? (a.normalize ? (double)(I / A) : (double)I) : 0.0;
  } else {
    const double ai = a.area_in[b];
    out = a.normalize ? (ai > kAreaThreshold ? (double)I / ai : 0.0) : (double)I;
  }
  a.cake[b] = out;
}

// one block per (R row, frame); both profiles in one pass.  variance != 0: the cake holds
// bin variances and the profiles are propagated variances (profile_1d_with_variance,
// packages/midas_integrate/midas_integrate/kernels.py:604-645): sum(A^2 V) / (sum A)^2 and
// sum(V) / N^2
template <typename T>
__global__ void k_profile(const T *cake, const double *area_in, int n_r, int n_eta, double *lo_aw,
                          double *lo_sm, int variance, int omp) {
  const int r = blockIdx.x;
  const int64_t f = blockIdx.y;
  if (r >= n_r) return;
  const T *ck = cake + f * (int64_t)n_r * n_eta;
  double s_ia = 0.0, s_a = 0.0, s_i = 0.0;
  int n = 0;
  for (int e = threadIdx.x; e < n_eta; e += blockDim.x) {
    const int64_t b = (int64_t)r * n_eta + e;
    const double A = area_in[b];
    const double I = (double)ck[b];
    if (omp) {
      // IntegratorZarrOMP.c:1829-1843: the mean of the row's nonzero, non-NaN bins; the
      // area-weighted mean over its valid, non-NaN bins
      if (!isnan(I)) {
        if (A > kAreaThreshold) {
          s_ia += I * A;
          s_a += A;
        }
        if (I != 0.0) {
          s_i += I;
          ++n;
        }
      }
    } else if (A > kAreaThreshold) {
      s_ia += variance ? I * A * A : I * A;
      s_a += A;
      s_i += I;
      ++n;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s_ia += __shfl_down_sync(0xffffffffu, s_ia, o);
    s_a += __shfl_down_sync(0xffffffffu, s_a, o);
    s_i += __shfl_down_sync(0xffffffffu, s_i, o);
    n += __shfl_down_sync(0xffffffffu, n, o);
  }
  __shared__ double sh[4][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[0][wid] = s_ia; sh[1][wid] = s_a; sh[2][wid] = s_i; sh[3][wid] = (double)n;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t_ia = 0, t_a = 0, t_i = 0, t_n = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      t_ia += sh[0][k]; t_a += sh[1][k]; t_i += sh[2][k]; t_n += sh[3][k];
    }
    const double d_a = variance ? t_a * t_a : t_a, d_n = variance ? t_n * t_n : t_n;
    if (lo_aw) lo_aw[f * n_r + r] = t_a > kAreaThreshold ? t_ia / d_a : 0.0;
    if (lo_sm) lo_sm[f * n_r + r] = t_n > 0 ? t_i / d_n : 0.0;
  }
}

int launch_profile(Plan *p, const void *cake, int cake_dtype, int n_frames, double *lo_aw, double *lo_sm,
                   cudaStream_t s) {
  if (n_frames <= 0 || (!lo_aw && !lo_sm)) return MI_OK;
  if (n_frames > 65535) return set_error(MI_E_RANGE, "mi_profile_batch: more than 65535 frames per call");
  const dim3 grid((unsigned)p->n_r, (unsigned)n_frames);
  if (cake_dtype == MI_DT_F32)
    k_profile<float><<<grid, 256, 0, s>>>((const float *)cake, p->d_area_in, p->n_r, p->n_eta, lo_aw, lo_sm,
                                          p->variance, p->semantics == MI_SEM_OMP);
  else if (cake_dtype == MI_DT_F64)
    k_profile<double><<<grid, 256, 0, s>>>((const double *)cake, p->d_area_in, p->n_r, p->n_eta, lo_aw, lo_sm,
                                           p->variance, p->semantics == MI_SEM_OMP);
  else
    return set_error(MI_E_ARG, "mi_profile_batch: cake dtype must be MI_DT_F32 or MI_DT_F64");
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

__global__ void k_nan_bins(float *cake, int64_t n_bins, const int32_t *bins, int n, int F) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n * F) return;
  const int64_t f = i / n;
  cake[f * n_bins + bins[i % n]] = __int_as_float(0x7fc00000);
}

int launch_nan_bins(Plan *p, float *cake, int n_frames, cudaStream_t s) {
  if (!cake || p->n_nan_bins == 0 || n_frames <= 0) return MI_OK;
  const int64_t n = (int64_t)p->n_nan_bins * n_frames;
  k_nan_bins<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cake, p->n_bins, p->d_nan_bins, p->n_nan_bins, n_frames);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

// SumImages (IntegratorFitPeaksGPUStream.cu:1043-1046 into dSumMatrix, allocated at
// :2141-2144): sum[b] += cake[f][b] over the batch's frames, in FP64, frames in order (the
// reference adds per frame with atomics in any order); NaN bins (masked bins of the OpenMP
// semantics) add nothing.  Thread per bin; eight frames' loads in flight before the adds.
__global__ void k_sum_cake(const float *__restrict__ cake, int F, int64_t n_bins, double *__restrict__ sum) {
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < n_bins; b += step) {
    double s = sum[b];
    int f = 0;
    for (; f + 8 <= F; f += 8) {
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = __ldcs(cake + (int64_t)(f + u) * n_bins + b);
#pragma unroll
      for (int u = 0; u < 8; ++u) s += isnan(v[u]) ? 0.0 : (double)v[u];
    }
    for (; f < F; ++f) {
      const float v = __ldcs(cake + (int64_t)f * n_bins + b);
      s += isnan(v) ? 0.0 : (double)v;
    }
    sum[b] = s;
  }
}

int launch_sum_cake(Plan *p, const float *cake, int n_frames, double *sum, cudaStream_t s) {
  if (n_frames <= 0 || p->n_bins == 0) return MI_OK;
  const int64_t blocks = std::min<int64_t>((p->n_bins + 255) / 256, (int64_t)std::max(p->n_sms, 1) * 8);
  k_sum_cake<<<(unsigned)blocks, 256, 0, s>>>(cake, n_frames, p->n_bins, sum);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

int launch_plain(Plan *p, const void *frame, int dtype, double *cake, double *lo_aw, double *lo_sm,
                 cudaStream_t s) {
  if (!cake) return set_error(MI_E_ARG, "mi_integrate_plain: cake output is required");
  const int64_t n_pix = (int64_t)p->ny * p->nz;
  int rc = launch_cast(frame, dtype, n_pix, 1, p->has_dark ? p->d_dark : nullptr, p->d_plain_img, s);
  if (rc) return rc;
  PlainArgs a;
  a.nmap = p->d_nmap;
  a.sorted = p->d_sorted;
  a.off = p->d_off;
  a.w = p->d_w;
  a.aw = p->d_aw;
  a.dr = p->d_dr;
  a.py = p->d_py;
  a.pz = p->d_pz;
  a.area_in = p->d_area_in;
  a.img = p->d_plain_img;
  a.cake = cake;
  a.n_bins = p->n_bins;
  a.ny = p->ny;
  a.nz = p->nz;
  a.mode = p->mode;
  a.sem = p->semantics;
  a.normalize = p->normalize;
  a.bc_y = (float)p->bc_y;
  a.bc_z = (float)p->bc_z;
  k_plain_integrate<<<(unsigned)((p->n_bins + 511) / 512), 512, 0, s>>>(a);
  MI_CUDA(cudaGetLastError());
  return launch_profile(p, cake, MI_DT_F64, 1, lo_aw, lo_sm, s);
}

}  // namespace mi
