// mi_runs.cu -- kernel (b), run encoding: batched caking with register-blocked bins.
//
// Same contract and semantics as the CSR kernel of mi_cake.cu (integrate() of
// packages/midas_integrate/midas_integrate/kernels.py:416-473): cake =
// diag(scale) * W * (frames - dark) for a batch of frames, plus the eta
// partial sums of both lineouts, with no global atomics.
//
// What changes is the inner loop.  A tile's bins are grouped into strips (one
// eta column, G consecutive R rows).  A warp owns a strip (or a slice of its rs
// range when the tile has fewer strips than warps) and keeps the strip's G bin
// accumulators in registers for its frames.  The map arrives as records
// {staged pixel, first row rs, weights for rows rs..rs+L-1}; records are sorted
// by rs and the loop over rs is unrolled at compile time, so each record does
// one shared-memory read of the pixel's frame values and L FMAs per frame into
// statically indexed registers: a pixel's radial run (the R bins its
// pixel-split or bilinear footprint reaches) costs one staged read, not one per
// bin.
//
// Frames of 8/16-bit types are staged as u16 and, with G <= 16, each lane reads
// one 32-bit word = two frames (64 frames per group); the dark is subtracted at
// use, (float)raw - dark, the reference's arithmetic.  Wider types are staged as
// (float)raw - dark, one frame per lane (32 per group).  After the record loop
// the partial sums of the units of a strip are combined in a fixed order (the
// result of a frame never depends on the batch), scaled, and eta-reduced for
// the lineouts in the same warp-per-row pass.
#include <stdint.h>

#include "mi_internal.h"

namespace mi {

struct RunArgs {
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
  uint32_t blob_cap;
  uint32_t off_val, off_dark, slot_bytes, off_out, off_lo, off_bar;
  int nbp;
  int *err;
};

constexpr int kRunThreads = (kRunWarps + kRunProducerWarps) * 32;
constexpr uint32_t kRunWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t r_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void r_bulk(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(r_smem(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(r_smem(dst)),
      "l"(src), "r"(bytes), "r"(r_smem(bar))
      : "memory");
}

// Bounded wait for phase `parity`; false when the poll budget ran out.
__device__ __forceinline__ bool r_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = r_smem(bar);
  for (uint32_t it = 0; it < kRunWaitLimit; ++it) {
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

template <typename T>
__device__ __forceinline__ float r_cvt(T v) {
  return (float)v;
}

template <int L>
__device__ __forceinline__ void load_weights(const float *wr, float *w) {
  if constexpr (L % 4 == 0) {
#pragma unroll
    for (int q = 0; q < L; q += 4) {
      const float4 t4 = *(const float4 *)(wr + q);
      w[q] = t4.x; w[q + 1] = t4.y; w[q + 2] = t4.z; w[q + 3] = t4.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < L; q += 2) {
      const float2 t2 = *(const float2 *)(wr + q);
      w[q] = t2.x; w[q + 1] = t2.y;
    }
  }
}

// Named barriers (bar.sync / bar.arrive with an id and a thread count) hand the two
// pipeline slots back and forth between the producer warps (gather) and the consumer
// warps (compute).  Id 1: consumers only.  Ids 2+b: slot b staged.  Ids 4+b: slot b free.
__device__ __forceinline__ void nb_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void nb_arrive(int id, int n) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

template <typename T, int G, int L>
__global__ void __launch_bounds__(kRunThreads, 1) k_runs(RunArgs a) {
  constexpr bool kU16 = sizeof(T) <= 2;              // staged as u16
  constexpr int FG = runs_frames_per_group(sizeof(T), G);
  constexpr int FPL = FG / 32;                       // frames per lane
  constexpr int NRS = G - L + 2;
  constexpr int NC = kRunWarps;                      // consumer warps
  constexpr int NCT = NC * 32;
  constexpr int NPT = kRunProducerWarps * 32;        // producer threads
  constexpr int NALL = NCT + NPT;
  extern __shared__ __align__(16) uint8_t smem[];
  float *s_out = (float *)(smem + a.off_out);        // [FG][nbp]
  double *s_lo = (double *)(smem + a.off_lo);        // [rows][FG][2]
  uint64_t *bar = (uint64_t *)(smem + a.off_bar);
  __shared__ int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const WorkItem it = a.items[blockIdx.x];
  const int nbp = a.nbp;
  const int nt = it.tile_end - it.tile_begin;
  const int n_groups = (a.F + FG - 1) / FG;
  const int n_steps = nt * n_groups;

  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(r_smem(&bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(r_smem(&bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();
  if (n_steps == 0) return;

  if (warp >= NC) {
    // ================= producers: bring tile blob k in (TMA), gather its pixels
    const int ptid = tid - NCT;
    const T *frames = (const T *)a.frames;
    for (int k = 0; k < n_steps; ++k) {
      const int b = k & 1;
      const int g0 = (k / nt) * FG;
      const int fg_n = min(FG, a.F - g0);
      uint8_t *slot = smem + b * a.slot_bytes;
      if (k >= 2) nb_sync(4 + b, NALL);              // consumers are done with slot b (step k-2)
      if (ptid == 0) {
        const TileRef r = a.tiles[it.tile_begin + k % nt];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        r_bulk(slot, a.blobs + r.off, r.bytes, &bar[b]);
      }
      if (!r_wait(&bar[b], (uint32_t)((k >> 1) & 1))) {
        atomicExch(a.err, MI_E_TIMEOUT);
        s_abort = 1;
      }
      asm volatile("bar.sync 6, %0;" ::"r"(NPT) : "memory");   // producers agree on the abort flag
      if (s_abort) {
        nb_arrive(2 + b, NALL);
        return;
      }
      const TileHdr h = *(const TileHdr *)slot;
      uint32_t o_rsp, o_sc, o_lw, o_up, o_lc, o_w;
      runs_blob_layout(h.nb, h.n_cols, h.nnz, h.n_u, G, L, &o_rsp, &o_sc, &o_lw, &o_up, &o_lc, &o_w);
      const uint32_t *upix = (const uint32_t *)(slot + o_up);
      uint8_t *s_val = slot + a.off_val;
      float *s_dark = (float *)(slot + a.off_dark);
      for (int u = ptid; u < h.n_u; u += NPT) {
        const uint32_t pix = upix[u];
        const float d = __ldg(a.dark + pix);
        const T *src = frames + (int64_t)g0 * a.stride + pix;
        uint8_t *row = s_val + (size_t)u * kRunPitch;
        if (kU16) {
          // all FG frames of the pixel in flight at once, packed two per word
          uint32_t v[FG / 2];
#pragma unroll
          for (int f = 0; f < FG; f += 2) {
            const uint32_t lo = (f < fg_n) ? (uint32_t)__ldg(src + (int64_t)f * a.stride) : 0u;
            const uint32_t hi = (f + 1 < fg_n) ? (uint32_t)__ldg(src + (int64_t)(f + 1) * a.stride) : 0u;
            v[f / 2] = lo | (hi << 16);
          }
          uint4 *dst = (uint4 *)row;
#pragma unroll
          for (int q = 0; q < FG / 8; ++q) dst[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
#pragma unroll
        for (int c = 0; c < FG; c += 32) {
          if (kU16) {
          } else {
            float v[32];
#pragma unroll
            for (int f = 0; f < 32; ++f)
              v[f] = (c + f < fg_n) ? r_cvt(__ldg(src + (int64_t)(c + f) * a.stride)) - d : 0.0f;
            float4 *dst = (float4 *)(row + 4 * c);
#pragma unroll
            for (int q = 0; q < 8; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
          }
        }
        s_dark[u] = d;
      }
      nb_arrive(2 + b, NALL);                         // slot b staged
    }
    // take the consumers' last two slot releases so no barrier generation is left open
    for (int k = n_steps; k < n_steps + 2; ++k)
      if (k >= 2) nb_sync(4 + (k & 1), NALL);
    return;
  }

  // ================= consumers: records -> registers -> combine -> cake + lineouts
  for (int k = 0; k < n_steps; ++k) {
    const int b = k & 1;
    const int g = k / nt, t = k - g * nt;
    const int g0 = g * FG;
    const int fg_n = min(FG, a.F - g0);
    const uint8_t *blob = smem + b * a.slot_bytes;
    const uint8_t *s_val = blob + a.off_val;
    const float *s_dark = (const float *)(blob + a.off_dark);
    float *s_part = (float *)(smem + b * a.slot_bytes + a.off_val);   // reuses slot b's staging
    if (t == 0)
      for (int i = tid; i < FG * a.rows_max * 2; i += NCT) s_lo[i] = 0.0;
    nb_sync(2 + b, NALL);                             // slot b staged
    if (s_abort) return;
    // the blob was written by the bulk copy (async proxy): observe its completed phase too
    if (!r_wait(&bar[b], (uint32_t)((k >> 1) & 1))) atomicExch(a.err, MI_E_TIMEOUT);
    const TileHdr h = *(const TileHdr *)blob;
    uint32_t o_rsp, o_sc, o_lw, o_up, o_lc, o_w;
    runs_blob_layout(h.nb, h.n_cols, h.nnz, h.n_u, G, L, &o_rsp, &o_sc, &o_lw, &o_up, &o_lc, &o_w);
    const uint16_t *rsp = (const uint16_t *)(blob + o_rsp);
    const float *scale = (const float *)(blob + o_sc);
    const float *lw = (const float *)(blob + o_lw);
    const uint16_t *lcol = (const uint16_t *)(blob + o_lc);
    const float *wts = (const float *)(blob + o_w);

    const int ns = h.n_cols;
    const int K = NC / ns;               // units per strip (>= 1: tiles hold <= NC strips)
    const int n_units = ns * K;
    float acc[G][FPL];
#pragma unroll
    for (int i = 0; i < G; ++i)
#pragma unroll
      for (int p = 0; p < FPL; ++p) acc[i][p] = 0.0f;
    if (warp < n_units) {
      const int s = warp / K, kk = warp - s * K;
      const int rs_lo = ((NRS - 1) * kk) / K, rs_hi = ((NRS - 1) * (kk + 1)) / K;
      const uint16_t *rp = rsp + s * NRS;
#pragma unroll
      for (int rs = 0; rs <= G - L; ++rs) {
        if (rs < rs_lo || rs >= rs_hi) continue;
        const int jb = rp[rs], je = rp[rs + 1];
        for (int j = jb; j < je; ++j) {
          const uint32_t u = lcol[j];
          const uint8_t *row = s_val + (size_t)u * kRunPitch;
          float v[FPL];
          if constexpr (kU16 && FPL == 2) {
            const uint32_t w2 = ((const uint32_t *)row)[lane];
            const float d = s_dark[u];
            v[0] = (float)(w2 & 0xFFFFu) - d;
            v[1] = (float)(w2 >> 16) - d;
          } else if constexpr (kU16) {
            v[0] = (float)((const uint16_t *)row)[lane] - s_dark[u];
          } else {
            v[0] = ((const float *)row)[lane];
          }
          float w[L];
          load_weights<L>(wts + (size_t)j * L, w);
#pragma unroll
          for (int q = 0; q < L; ++q)
#pragma unroll
            for (int p = 0; p < FPL; ++p) acc[rs + q][p] = fmaf(w[q], v[p], acc[rs + q][p]);
        }
      }
    }
    nb_sync(1, NCT);                     // staging of slot b consumed: holds the partials now
    if (warp < n_units) {
#pragma unroll
      for (int i = 0; i < G; ++i) {
        float *d = s_part + ((size_t)warp * G + i) * FG + lane * FPL;
        if constexpr (FPL == 2) *(float2 *)d = make_float2(acc[i][0], acc[i][1]);
        else d[0] = acc[i][0];
      }
    }
    nb_sync(1, NCT);

    // ---- combine (fixed unit order), scale, lineout partials: warp per row, lanes = frames
    for (int i = warp; i < h.n_rows; i += NC) {
      double saw[FPL], ssm[FPL];
#pragma unroll
      for (int p = 0; p < FPL; ++p) saw[p] = ssm[p] = 0.0;
      for (int s = 0; s < ns; ++s) {
        float v[FPL];
#pragma unroll
        for (int p = 0; p < FPL; ++p) v[p] = 0.0f;
        for (int kk = 0; kk < K; ++kk) {
          const float *src = s_part + ((size_t)(s * K + kk) * G + i) * FG + lane * FPL;
#pragma unroll
          for (int p = 0; p < FPL; ++p) v[p] += src[p];
        }
        const int bb = i * ns + s;
        const float sc = scale[bb], l = lw[bb];
#pragma unroll
        for (int p = 0; p < FPL; ++p) {
          const float o = v[p] * sc;
          s_out[(lane * FPL + p) * nbp + bb] = o;
          saw[p] += (double)o * (double)l;
          ssm[p] += (l > 0.0f) ? (double)o : 0.0;
        }
      }
      if (a.want_lo) {
        double *dst = s_lo + ((size_t)(h.row_in_band + i) * FG + lane * FPL) * 2;
#pragma unroll
        for (int p = 0; p < FPL; ++p) {
          dst[2 * p] += saw[p];
          dst[2 * p + 1] += ssm[p];
        }
      }
    }
    nb_sync(1, NCT);
    // slot b (blob + staging/partials) is no longer read: hand it back to the producers
    nb_arrive(4 + b, NALL);

    // ---- cake store: warp per frame, lanes over the tile's bins (runs of n_cols contiguous
    // floats per row); row/col from a float reciprocal (exact for b < 2^12)
    if (a.want_cake) {
      const float inv_ns = 1.0f / (float)ns;
      for (int f = warp; f < fg_n; f += NC) {
        float *dst = a.cake + (int64_t)(g0 + f) * a.n_bins + (int64_t)h.r0 * a.n_eta + h.e0;
        const float *src = s_out + f * nbp;
        for (int bb = lane; bb < h.nb; bb += 32) {
          const int r = (int)(((float)bb + 0.5f) * inv_ns);
          dst[(int64_t)r * a.n_eta + (bb - r * ns)] = src[bb];
        }
      }
    }
    if (t == nt - 1 && a.want_lo) {
      for (int f = warp; f < fg_n; f += NC)
        for (int r = lane; r < it.n_rows; r += 32) {
          const double *src = s_lo + ((size_t)r * FG + f) * 2;
          double *dst = a.partial + (((int64_t)(g0 + f) * a.n_r + it.r0 + r) * a.n_slots + it.slot) * 2;
          dst[0] = src[0];
          dst[1] = src[1];
        }
    }
    nb_sync(1, NCT);                     // s_out / s_lo free for the next step
  }
}

template <typename T, int G, int L>
static int launch_runs_t(Plan *p, RunArgs &a, cudaStream_t s) {
  const size_t smem = runs_smem_layout(a.blob_cap, std::max(p->max_u, 1), a.nbp, a.rows_max, G,
                                       runs_frames_per_group(sizeof(T), G), &a.off_val, &a.off_dark, &a.slot_bytes,
                                       &a.off_out, &a.off_lo, &a.off_bar);
  int dev_smem = 0;
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
  if (smem + 64 > (size_t)dev_smem)
    return set_error(MI_E_RANGE, "run kernel needs %zu B shared memory (> %d)", smem, dev_smem);
  MI_CUDA(cudaFuncSetAttribute(k_runs<T, G, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  MI_CUDA(cudaFuncSetAttribute(k_runs<T, G, L>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared));
  k_runs<T, G, L><<<p->n_items, kRunThreads, smem, s>>>(a);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

template <typename T>
static int launch_runs_gl(Plan *p, RunArgs &a, cudaStream_t s) {
  const int G = p->run_g, L = p->run_l;
  if (G == 8 && L == 2) return launch_runs_t<T, 8, 2>(p, a, s);
  if (G == 8 && L == 4) return launch_runs_t<T, 8, 4>(p, a, s);
  if (G == 16 && L == 4) return launch_runs_t<T, 16, 4>(p, a, s);
  if (G == 16 && L == 8) return launch_runs_t<T, 16, 8>(p, a, s);
  if (G == 32 && L == 4) return launch_runs_t<T, 32, 4>(p, a, s);
  if (G == 32 && L == 8) return launch_runs_t<T, 32, 8>(p, a, s);
  return set_error(MI_E_UNSUPPORTED, "run encoding with G=%d L=%d", G, L);
}

int launch_runs(Plan *p, const void *frames, int dtype, int n_frames, int64_t stride, float *cake, bool want_lo,
                cudaStream_t s) {
  RunArgs a;
  a.items = p->d_items;
  a.tiles = p->d_tiles;
  a.blobs = p->d_blobs;
  a.frames = frames;
  a.stride = stride;
  a.F = n_frames;
  a.dark = p->d_dark;
  a.cake = cake;
  a.partial = p->d_partial;
  a.n_slots = p->n_slots;
  a.n_r = p->n_r;
  a.n_eta = p->n_eta;
  a.n_bins = p->n_bins;
  a.want_cake = cake != nullptr;
  a.want_lo = want_lo;
  a.rows_max = p->lim.rows;
  a.blob_cap = (p->max_blob + 15u) & ~15u;
  a.nbp = (p->max_nb | 1);
  a.err = p->d_err;
  switch (dtype) {
    case MI_DT_U8: return launch_runs_gl<uint8_t>(p, a, s);
    case MI_DT_U16: return launch_runs_gl<uint16_t>(p, a, s);
    case MI_DT_U32: return launch_runs_gl<uint32_t>(p, a, s);
    case MI_DT_I64: return launch_runs_gl<int64_t>(p, a, s);
    case MI_DT_F32: return launch_runs_gl<float>(p, a, s);
    case MI_DT_F64: return launch_runs_gl<double>(p, a, s);
    case MI_DT_I32: return launch_runs_gl<int32_t>(p, a, s);
  }
  return set_error(MI_E_ARG, "unknown dtype %d", dtype);
}

}  // namespace mi
