// mi_cake.cu -- kernel (b): F-frame batched caking; kernel (c): lineout finalize.
//
// The map is a bin-major sparse matrix W (bins x pixels).  For a batch of F
// frames X (pixels x F) the cake is C = diag(scale) * W * (X - dark): a sparse
// x dense product whose dense dimension is the frame batch, so every map byte
// read from HBM is used F times.  Semantics per bin and frame are those of
// integrate() in packages/midas_integrate/midas_integrate/kernels.py:416-473
// (and integrate_noMapMask, FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:975-1050).
//
// One CTA runs one work item (a band of R rows x a range of eta columns).  Per
// staging tile it bulk-copies the tile blob into shared memory, stages the
// tile's referenced pixels of FG frames as (float)raw - dark into shared memory
// (pixel-major, frames innermost, padded rows so both the staging writes and
// the per-term reads are bank-conflict free), then one warp per bin walks the
// bin's terms with lane = frame.  Bin results go through shared memory so the
// cake stores are coalesced along eta, and the eta partial sums of the two
// lineouts are reduced inside the CTA: no global atomics anywhere.
#include <stdint.h>

#include "mi_internal.h"

namespace mi {

struct CakeArgs {
  const WorkItem *items;
  const TileRef *tiles;
  const uint8_t *blobs;
  const void *frames;
  int64_t stride;
  int F;
  const float *dark;
  float *cake;
  double *partial;  // [F][n_r][n_slots][2]
  int n_slots, n_r, n_eta;
  int64_t n_bins;
  int want_cake, want_lo;
  int rows_max;
  uint32_t off_val, off_out, off_lo;  // shared-memory section offsets (16-B aligned)
  int u_cap, nbp;
  int *err;
};

template <int FPL>
__host__ __device__ inline void cake_smem(uint32_t blob_cap, int u_cap, int nbp, int rows,
                                          uint32_t *off_val, uint32_t *off_out, uint32_t *off_lo,
                                          uint32_t *total) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  *off_val = a16(blob_cap);
  *off_out = a16(*off_val + (uint32_t)u_cap * 33u * FPL * 4u);
  *off_lo = a16(*off_out + 32u * FPL * (uint32_t)nbp * 4u);
  *total = *off_lo + 32u * FPL * (uint32_t)rows * 2u * 8u;
}

template <typename T>
__device__ __forceinline__ float to_f(T v) {
  return (float)v;
}

template <int N>
struct FVec;
template <>
struct FVec<1> {
  __device__ static __forceinline__ void ld(const float *p, float *v) { v[0] = *p; }
  __device__ static __forceinline__ void st(float *p, const float *v) { *p = v[0]; }
};
template <>
struct FVec<2> {
  __device__ static __forceinline__ void ld(const float *p, float *v) {
    float2 t = *(const float2 *)p;
    v[0] = t.x; v[1] = t.y;
  }
  __device__ static __forceinline__ void st(float *p, const float *v) {
    *(float2 *)p = make_float2(v[0], v[1]);
  }
};
template <>
struct FVec<4> {
  __device__ static __forceinline__ void ld(const float *p, float *v) {
    float4 t = *(const float4 *)p;
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  }
  __device__ static __forceinline__ void st(float *p, const float *v) {
    *(float4 *)p = make_float4(v[0], v[1], v[2], v[3]);
  }
};

constexpr int kCakeThreads = 256;

template <typename T, int FPL>
__global__ void __launch_bounds__(kCakeThreads) k_cake(CakeArgs a) {
  constexpr int FG = 32 * FPL;    // frames per group
  constexpr int SROW = 33 * FPL;  // staged row pitch (floats): conflict-free writes & reads
  constexpr int NW = kCakeThreads / 32;
  extern __shared__ __align__(16) uint8_t smem[];
  uint8_t *s_blob = smem;
  float *s_val = (float *)(smem + a.off_val);
  float *s_out = (float *)(smem + a.off_out);
  double *s_lo = (double *)(smem + a.off_lo);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const WorkItem it = a.items[blockIdx.x];
  const T *frames = (const T *)a.frames;
  const int nbp = a.nbp;

  for (int g0 = 0; g0 < a.F; g0 += FG) {
    const int fg_n = min(FG, a.F - g0);
    for (int i = tid; i < FG * a.rows_max * 2; i += kCakeThreads) s_lo[i] = 0.0;
    for (int t = it.tile_begin; t < it.tile_end; ++t) {
      __syncthreads();
      const TileRef ref = a.tiles[t];
      {
        const uint4 *src = (const uint4 *)(a.blobs + ref.off);
        uint4 *dst = (uint4 *)s_blob;
        const int n16 = (int)(ref.bytes >> 4);
        for (int i = tid; i < n16; i += kCakeThreads) dst[i] = __ldg(src + i);
      }
      __syncthreads();
      const TileHdr h = *(const TileHdr *)s_blob;
      uint32_t o_rp, o_sc, o_lw, o_up, o_lc, o_w, bytes;
      blob_layout(h.nb, h.nnz, h.n_u, &o_rp, &o_sc, &o_lw, &o_up, &o_lc, &o_w, &bytes);
      const uint32_t *rowp = (const uint32_t *)(s_blob + o_rp);
      const float *scale = (const float *)(s_blob + o_sc);
      const float *lw = (const float *)(s_blob + o_lw);
      const uint32_t *upix = (const uint32_t *)(s_blob + o_up);
      const uint16_t *lcol = (const uint16_t *)(s_blob + o_lc);
      const float *wt = (const float *)(s_blob + o_w);

      // ---- stage: s_val[u][q*FPL + k] = (float)frame[g0 + q*FPL + k][pix_u] - dark[pix_u]
      const int n_u = h.n_u;
      for (int i = tid; i < n_u * 32; i += kCakeThreads) {
        const int u = i % n_u, q = i / n_u;
        const uint32_t pix = upix[u];
        const float d = __ldg(a.dark + pix);
        float v[FPL];
#pragma unroll
        for (int k = 0; k < FPL; ++k) {
          const int f = q * FPL + k;
          v[k] = (f < fg_n) ? to_f(__ldg(frames + (int64_t)(g0 + f) * a.stride + pix)) - d : 0.0f;
        }
        FVec<FPL>::st(s_val + u * SROW + q * FPL, v);
      }
      __syncthreads();

      // ---- compute: warp per bin, lane = frame(s)
      for (int b = warp; b < h.nb; b += NW) {
        const uint32_t j0 = rowp[b], j1 = rowp[b + 1];
        float acc[FPL];
#pragma unroll
        for (int k = 0; k < FPL; ++k) acc[k] = 0.0f;
        uint32_t j = j0;
        for (; j + 4 <= j1; j += 4) {
          uint32_t c[4];
          float w[4], v[4][FPL];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            c[q] = lcol[j + q];
            w[q] = wt[j + q];
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) FVec<FPL>::ld(s_val + c[q] * SROW + lane * FPL, v[q]);
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int k = 0; k < FPL; ++k) acc[k] = fmaf(w[q], v[q][k], acc[k]);
        }
        for (; j < j1; ++j) {
          float v[FPL];
          FVec<FPL>::ld(s_val + (uint32_t)lcol[j] * SROW + lane * FPL, v);
          const float w = wt[j];
#pragma unroll
          for (int k = 0; k < FPL; ++k) acc[k] = fmaf(w, v[k], acc[k]);
        }
        const float sc = scale[b];
#pragma unroll
        for (int k = 0; k < FPL; ++k) s_out[(lane * FPL + k) * nbp + b] = acc[k] * sc;
      }
      __syncthreads();

      // ---- cake store: runs of n_cols contiguous floats per (frame, row)
      if (a.want_cake) {
        for (int i = tid; i < fg_n * h.nb; i += kCakeThreads) {
          const int f = i / h.nb, b = i - f * h.nb;
          const int r = b / h.n_cols, e = b - r * h.n_cols;
          a.cake[(int64_t)(g0 + f) * a.n_bins + (int64_t)(h.r0 + r) * a.n_eta + h.e0 + e] =
              s_out[f * nbp + b];
        }
      }
      // ---- lineout partials of this tile, accumulated per (frame, row of band)
      if (a.want_lo) {
        for (int i = tid; i < fg_n * h.n_rows; i += kCakeThreads) {
          const int f = i / h.n_rows, r = i - f * h.n_rows;
          double saw = 0.0, ssm = 0.0;
          for (int e = 0; e < h.n_cols; ++e) {
            const float v = s_out[f * nbp + r * h.n_cols + e];
            const float l = lw[r * h.n_cols + e];
            saw += (double)v * (double)l;
            ssm += (l > 0.0f) ? (double)v : 0.0;
          }
          double *dst = s_lo + ((size_t)f * a.rows_max + h.row_in_band + r) * 2;
          dst[0] += saw;
          dst[1] += ssm;
        }
      }
    }
    __syncthreads();
    if (a.want_lo) {
      for (int i = tid; i < fg_n * it.n_rows; i += kCakeThreads) {
        const int f = i / it.n_rows, r = i - f * it.n_rows;
        const double *src = s_lo + ((size_t)f * a.rows_max + r) * 2;
        double *dst = a.partial + (((int64_t)(g0 + f) * a.n_r + it.r0 + r) * a.n_slots + it.slot) * 2;
        dst[0] = src[0];
        dst[1] = src[1];
      }
    }
    __syncthreads();
  }
}

// kernel (c): lineout = sum over the band's work-item partials / denominator,
// matching profile_1d() (kernels.py:567-601) and calculate_1D_profile_kernel /
// calculate_1D_profile_simple_mean_kernel (…Stream.cu:1162-1334).
__global__ void k_lineout(const double *partial, int F, int n_r, int n_slots, const double *den_aw,
                          const double *cnt, double *lo_aw, double *lo_sm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)F * n_r) return;
  const int r = (int)(i % n_r);
  const double *p = partial + i * n_slots * 2;
  double saw = 0.0, ssm = 0.0;
  for (int s = 0; s < n_slots; ++s) {
    saw += p[2 * s];
    ssm += p[2 * s + 1];
  }
  const double d = den_aw[r], c = cnt[r];
  if (lo_aw) lo_aw[i] = d > kAreaThreshold ? saw / d : 0.0;
  if (lo_sm) lo_sm[i] = c > 0.0 ? ssm / c : 0.0;
}

template <typename T, int FPL>
static int launch_t(Plan *p, CakeArgs &a, cudaStream_t s) {
  uint32_t total = 0;
  cake_smem<FPL>((p->max_blob + 15u) & ~15u, a.u_cap, a.nbp, a.rows_max, &a.off_val, &a.off_out,
                 &a.off_lo, &total);
  const size_t smem = total;
  int dev_smem = 0;
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
  if (smem > (size_t)dev_smem)
    return set_error(MI_E_RANGE, "batched kernel needs %zu B shared memory (> %d); lower tile_pixels", smem,
                     dev_smem);
  MI_CUDA(cudaFuncSetAttribute(k_cake<T, FPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_cake<T, FPL><<<p->n_items, kCakeThreads, smem, s>>>(a);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

template <typename T>
static int launch_fpl(Plan *p, CakeArgs &a, cudaStream_t s) {
  switch (p->frames_per_lane) {
    case 1: return launch_t<T, 1>(p, a, s);
    case 2: return launch_t<T, 2>(p, a, s);
    case 4: return launch_t<T, 4>(p, a, s);
  }
  return set_error(MI_E_ARG, "bad frames_per_lane");
}

int launch_cake(Plan *p, const void *frames, int dtype, int n_frames, int64_t stride, float *cake,
                double *lo_aw, double *lo_sm, cudaStream_t s) {
  CakeArgs a;
  a.items = p->d_items;
  a.tiles = p->d_tiles;
  a.blobs = p->d_blobs;
  a.frames = frames;
  a.stride = stride;
  a.F = n_frames;
  a.dark = p->d_dark;
  a.cake = cake;
  a.partial = (double *)p->d_partial;
  a.n_slots = p->n_slots;
  a.n_r = p->n_r;
  a.n_eta = p->n_eta;
  a.n_bins = p->n_bins;
  a.want_cake = cake != nullptr;
  a.want_lo = (lo_aw != nullptr) || (lo_sm != nullptr);
  a.rows_max = p->lim.rows;
  a.u_cap = std::max(p->max_u, 1);
  a.nbp = (p->max_nb | 1);  // odd pitch: conflict-free column writes
  a.err = p->d_err;
  if (!a.want_cake && !a.want_lo) return MI_OK;
  int rc = MI_OK;
  switch (dtype) {
    case MI_DT_U8: rc = launch_fpl<uint8_t>(p, a, s); break;
    case MI_DT_U16: rc = launch_fpl<uint16_t>(p, a, s); break;
    case MI_DT_U32: rc = launch_fpl<uint32_t>(p, a, s); break;
    case MI_DT_I64: rc = launch_fpl<int64_t>(p, a, s); break;
    case MI_DT_F32: rc = launch_fpl<float>(p, a, s); break;
    case MI_DT_F64: rc = launch_fpl<double>(p, a, s); break;
    case MI_DT_I32: rc = launch_fpl<int32_t>(p, a, s); break;
    default: return set_error(MI_E_ARG, "unknown dtype %d", dtype);
  }
  if (rc) return rc;
  if (a.want_lo) {
    const int64_t n = (int64_t)n_frames * p->n_r;
    k_lineout<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a.partial, n_frames, p->n_r, p->n_slots,
                                                          p->d_den_aw, p->d_cnt, lo_aw, lo_sm);
    MI_CUDA(cudaGetLastError());
  }
  return MI_OK;
}

}  // namespace mi
