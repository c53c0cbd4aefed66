// mi_cake.cu -- kernel (b): F-frame batched caking; kernel (c): lineout finalize.
//
// The map is a bin-major sparse matrix W (bins x pixels).  For a batch of F
// frames X (pixels x F) the cake is C = diag(scale) * W * (X - dark): a sparse
// x dense product whose dense dimension is the frame batch, so every map byte
// read from HBM is used F times.  Semantics per bin and frame are those of
// integrate() in packages/midas_integrate/midas_integrate/kernels.py:416-473
// (and integrate_noMapMask, FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:975-1050).
//
// One CTA runs one work item (a band of R rows x a range of eta columns).  The
// item's staging tiles are streamed through shared memory: each tile blob is
// brought in by one bulk (TMA) copy, double-buffered so tile k+1 is in flight
// while tile k is computed; completion is tracked by an mbarrier whose waits
// are bounded (a wait that runs out sets the plan's error word and the CTA
// leaves).  Per tile and frame group the referenced pixels of FG frames are
// gathered as (float)raw - dark into shared memory (pixel-major, frames
// innermost, padded rows: bank-conflict-free writes and per-term reads), with
// 32 independent loads in flight per thread; then one warp per bin walks the
// bin's terms with lane = frame.  Bin results pass through shared memory so the
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
  uint32_t blob_cap;                          // bytes per blob buffer (16-B multiple)
  uint32_t off_val, off_out, off_lo, off_bar; // shared-memory section offsets
  int u_cap, nbp;
  int *err;
};

constexpr int kCakeThreads = 256;
constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before a wait is declared lost

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
  __device__ static __forceinline__ void st(float *p, const float *v) { *(float2 *)p = make_float2(v[0], v[1]); }
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

// ---- mbarrier + bulk copy (sm_90+ PTX) -------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait for phase `parity` of the barrier; false when the poll budget ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <typename T, int FPL>
__global__ void __launch_bounds__(kCakeThreads) k_cake(CakeArgs a) {
  constexpr int FG = 32 * FPL;    // frames per group
  constexpr int SROW = 33 * FPL;  // staged row pitch (floats)
  constexpr int NW = kCakeThreads / 32;
  extern __shared__ __align__(16) uint8_t smem[];
  float *s_val = (float *)(smem + a.off_val);
  float *s_out = (float *)(smem + a.off_out);
  double *s_lo = (double *)(smem + a.off_lo);
  uint64_t *bar = (uint64_t *)(smem + a.off_bar);
  __shared__ int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const WorkItem it = a.items[blockIdx.x];
  const T *frames = (const T *)a.frames;
  const int nbp = a.nbp;
  const int nt = it.tile_end - it.tile_begin;
  const int n_groups = (a.F + FG - 1) / FG;
  const int n_steps = nt * n_groups;  // (group, tile) pairs, group-major

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
    s_abort = 0;
  }
  __syncthreads();
  if (n_steps == 0) return;
  if (tid == 0) {
    const TileRef r0 = a.tiles[it.tile_begin];
    bulk_load(smem, a.blobs + r0.off, r0.bytes, &bar[0]);
  }

  for (int k = 0; k < n_steps; ++k) {
    const int g = k / nt, t = k - g * nt;
    const int g0 = g * FG;
    const int fg_n = min(FG, a.F - g0);
    const int buf = k & 1;
    uint8_t *s_blob = smem + buf * a.blob_cap;
    if (t == 0)
      for (int i = tid; i < FG * a.rows_max * 2; i += kCakeThreads) s_lo[i] = 0.0;
    // prefetch the next (group, tile) blob into the other buffer (its readers finished
    // at the barrier that ended step k-1)
    if (tid == 0 && k + 1 < n_steps) {
      const int t1 = (k + 1) % nt;
      const TileRef r1 = a.tiles[it.tile_begin + t1];
      fence_proxy_async();
      bulk_load(smem + (buf ^ 1) * a.blob_cap, a.blobs + r1.off, r1.bytes, &bar[buf ^ 1]);
    }
    if (!mbar_wait(&bar[buf], (uint32_t)((k >> 1) & 1))) {
      atomicExch(a.err, MI_E_TIMEOUT);
      s_abort = 1;
    }
    __syncthreads();
    if (s_abort) return;
    const TileHdr h = *(const TileHdr *)s_blob;
    uint32_t o_rp, o_sc, o_lw, o_up, o_lc, o_w, bytes;
    blob_layout(h.nb, h.nnz, h.n_u, &o_rp, &o_sc, &o_lw, &o_up, &o_lc, &o_w, &bytes);
    const uint32_t *rowp = (const uint32_t *)(s_blob + o_rp);
    const double *scale = (const double *)(s_blob + o_sc);
    const float *lw = (const float *)(s_blob + o_lw);
    const uint32_t *upix = (const uint32_t *)(s_blob + o_up);
    const uint16_t *lcol = (const uint16_t *)(s_blob + o_lc);
    const float *wt = (const float *)(s_blob + o_w);

    // ---- stage: thread owns pixel u, gathers 32 frames at a time (32 loads in flight)
    const int n_u = h.n_u;
    for (int u = tid; u < n_u; u += kCakeThreads) {
      const uint32_t pix = upix[u];
      const float d = __ldg(a.dark + pix);
      const T *src = frames + (int64_t)g0 * a.stride + pix;
      float *dst = s_val + u * SROW;
#pragma unroll
      for (int c = 0; c < FG; c += 32) {
        float v[32];
#pragma unroll
        for (int f = 0; f < 32; ++f)
          v[f] = (c + f < fg_n) ? to_f(__ldg(src + (int64_t)(c + f) * a.stride)) : d;
#pragma unroll
        for (int f = 0; f < 32; ++f) v[f] -= d;
#pragma unroll
        for (int f = 0; f < 32; f += FPL) FVec<FPL>::st(dst + c + f, v + f);
      }
    }
    __syncthreads();

    // ---- compute: warp per bin, lane = frame(s)
    for (int b = warp; b < h.nb; b += NW) {
      const uint32_t j0 = rowp[b], j1 = rowp[b + 1];
      // FP64 sums of the exact FP64 products (no error growth with the bin's term count)
      double acc[FPL];
#pragma unroll
      for (int q = 0; q < FPL; ++q) acc[q] = 0.0;
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
          for (int r = 0; r < FPL; ++r) acc[r] = fma((double)w[q], (double)v[q][r], acc[r]);
      }
      for (; j < j1; ++j) {
        float v[FPL];
        FVec<FPL>::ld(s_val + (uint32_t)lcol[j] * SROW + lane * FPL, v);
        const float w = wt[j];
#pragma unroll
        for (int r = 0; r < FPL; ++r) acc[r] = fma((double)w, (double)v[r], acc[r]);
      }
      const double sc = scale[b];
#pragma unroll
      for (int r = 0; r < FPL; ++r) s_out[(lane * FPL + r) * nbp + b] = (float)(acc[r] * sc);
    }
    __syncthreads();

    // ---- cake store: runs of n_cols contiguous floats per (frame, row)
    if (a.want_cake) {
      for (int i = tid; i < fg_n * h.nb; i += kCakeThreads) {
        const int f = i / h.nb, b = i - f * h.nb;
        const int r = b / h.n_cols, e = b - r * h.n_cols;
        a.cake[(int64_t)(g0 + f) * a.n_bins + (int64_t)(h.r0 + r) * a.n_eta + h.e0 + e] = s_out[f * nbp + b];
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
    if (t == nt - 1 && a.want_lo) {
      __syncthreads();
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
  if (lo_aw) lo_aw[i] = d > 0.0 ? saw / d : 0.0;   // d is 0 or a sum of areas > 1e-9
  if (lo_sm) lo_sm[i] = c > 0.0 ? ssm / c : 0.0;
}

template <typename T, int FPL>
static int launch_t(Plan *p, CakeArgs &a, cudaStream_t s) {
  const size_t smem =
      cake_smem_layout(FPL, a.blob_cap, a.u_cap, a.nbp, a.rows_max, &a.off_val, &a.off_out, &a.off_lo, &a.off_bar);
  int dev_smem = 0;
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
  if (smem + 64 > (size_t)dev_smem)
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

int launch_lineout(Plan *p, const double *partial, int n_frames, double *lo_aw, double *lo_sm, cudaStream_t s) {
  const int64_t n = (int64_t)n_frames * p->n_r;
  if (n == 0) return MI_OK;
  k_lineout<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(partial, n_frames, p->n_r, p->n_slots, p->d_den_aw,
                                                        p->d_cnt, lo_aw, lo_sm);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

int launch_cake(Plan *p, const void *frames, int dtype, int n_frames, int64_t stride, float *cake,
                double *lo_aw, double *lo_sm, double *partial, cudaStream_t s) {
  if (p->panels.size() > 1)
    return set_error(MI_E_ARG, "a panel plan takes its frames per panel: use mi_integrate_panels");
  CakeArgs a;
  a.items = p->d_items;
  a.tiles = p->d_tiles;
  a.blobs = p->d_blobs;
  a.frames = frames;
  a.stride = stride;
  a.F = n_frames;
  a.dark = p->d_dark;
  a.cake = cake;
  a.partial = partial;
  a.n_slots = p->n_slots;
  a.n_r = p->n_r;
  a.n_eta = p->n_eta;
  a.n_bins = p->n_bins;
  a.want_cake = cake != nullptr;
  a.want_lo = (lo_aw != nullptr) || (lo_sm != nullptr);
  // MI_SEM_OMP: masked bins are NaN and the lineouts come from the cake (mean of nonzero,
  // non-NaN bins), not from the kernels' partial sums
  const bool omp = p->semantics == MI_SEM_OMP;
  const bool want_lo_omp = omp && a.want_lo;
  if (want_lo_omp && !cake)
    return set_error(MI_E_ARG, "OpenMP-integrator semantics computes the lineouts from the cake: pass a cake");
  if (omp) a.want_lo = false;
  a.rows_max = p->lim.rows;
  a.blob_cap = (p->max_blob + 15u) & ~15u;
  a.u_cap = std::max(p->max_u, 1);
  a.nbp = (p->max_nb | 1);  // odd pitch: conflict-free column writes
  a.err = p->d_err;
  if (!a.want_cake && !a.want_lo) return MI_OK;
  int rc = MI_OK;
  if (p->encoding == MI_ENC_MMA) {
    // kernel (a) splits a chunk of frames into byte planes, then kernel (b) on the tensor cores
    if (!(dtype == MI_DT_U16 || dtype == MI_DT_U8))
      return set_error(MI_E_UNSUPPORTED, "MMA plans cake 8/16-bit frames only (dtype %d)", dtype);
    const size_t es = dtype_size(dtype);
    for (int f0 = 0; f0 < n_frames && rc == MI_OK; f0 += kMmaFrames) {
      const int nf = std::min(kMmaFrames, n_frames - f0);
      rc = launch_xc(p, 0, (const uint8_t *)frames + (size_t)f0 * stride * es, dtype, nf, stride, false, s);
      if (rc == MI_OK)
        rc = launch_mma(p, nf, cake ? cake + (size_t)f0 * p->n_bins : nullptr,
                        partial + (size_t)f0 * p->n_r * p->n_slots * 2, a.want_lo, s);
    }
  } else if (p->encoding == MI_ENC_MMAD) {
    // kernel (b) on the tensor cores, reading the frames in place: no staging pass
    if (!(dtype == MI_DT_U16 || dtype == MI_DT_U8))
      return set_error(MI_E_UNSUPPORTED, "direct MMA plans cake 8/16-bit frames only (dtype %d)", dtype);
    const size_t es = dtype_size(dtype);
    for (int f0 = 0; f0 < n_frames && rc == MI_OK; f0 += kMmaFrames) {
      const int nf = std::min(kMmaFrames, n_frames - f0);
      rc = launch_mmad(p, (const uint8_t *)frames + (size_t)f0 * stride * es, dtype, nf, stride,
                       cake ? cake + (size_t)f0 * p->n_bins : nullptr, partial + (size_t)f0 * p->n_r * p->n_slots * 2,
                       a.want_lo, s);
    }
  } else if (p->encoding == MI_ENC_RUNS) {
    rc = launch_runs(p, frames, dtype, n_frames, stride, cake, partial, a.want_lo, s);
  } else switch (dtype) {
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
  if (omp) {
    rc = launch_nan_bins(p, cake, n_frames, s);
    if (rc == MI_OK && want_lo_omp) rc = launch_profile(p, cake, MI_DT_F32, n_frames, lo_aw, lo_sm, s);
    return rc;
  }
  return a.want_lo ? launch_lineout(p, partial, n_frames, lo_aw, lo_sm, s) : MI_OK;
}

}  // namespace mi
