// mi_runs.cu -- kernel (b), run encoding: batched caking with register-blocked bins.
//
// Same contract and semantics as the CSR kernel of mi_cake.cu (integrate() of
// packages/midas_integrate/midas_integrate/kernels.py:416-473): cake =
// diag(scale) * W * (frames - dark) for a batch of frames, plus the eta
// partial sums of both lineouts, with no global atomics on the data.
//
// A tile's bins are grouped into strips (one eta column, G consecutive R rows).  The
// map arrives as records {staged pixel, first row rs, weights for rows rs..rs+L-1};
// records of a strip are sorted by rs, the loop over rs is unrolled at compile time,
// and each record does one shared-memory read of the pixel's frame values and L FMAs
// per frame into statically indexed registers: a pixel's radial run (the R bins its
// pixel-split or bilinear footprint reaches) costs one staged read, not one per bin.
// Each of the 8 consumer warps owns a unit: a contiguous record range of one strip,
// chosen on the host so that the units of a tile carry equal numbers of records.
//
// The kernel is persistent (one CTA per SM) and warp-specialized: producer warps
// claim work items from a counter (heaviest first), bring each tile's blob in with
// one bulk copy (TMA) and stage its pixels into one of two slots; consumer warps run
// the record loop, combine the unit partials in a fixed order (a frame's result never
// depends on the rest of its batch), scale, reduce the lineouts, store the cake and
// hand the slot back.  Staging comes from the pixel-major buffer written by kernel (a)
// (mi_stage.cu): one 128-byte bulk copy per pixel and frame group (64 u16 frames with the
// dark subtracted at use as (float)raw - dark, the reference's arithmetic; or 32 fp32
// frames already dark-subtracted).  Plans without row spans (strips of 32 rows) gather
// from frame-major memory.
#include <stdint.h>

#include <algorithm>

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
  uint32_t off_val, slot_bytes, off_part, off_lo, off_bar;
  int nbp;
  int *err;
  int n_items;
  int *counter;     // work-item claims of this launch (zero at launch)
  // pixel-major staging: row of compact pixel c at xc + c * xc_pitch bytes, frame group g at
  // byte 128 g of the row; c = row_off[z] + y - span_lo[z]
  const uint8_t *xc;
  int64_t xc_pitch;
  const int32_t *span_lo, *row_off;
  int ny;
};

constexpr uint32_t kRunWaitLimit = 1u << 26;
constexpr int kRecBatch = 4;   // records whose loads are issued together in the record loop
constexpr int kStoreSlots = 8; // bins per lane in the cake store: tiles hold <= 256 bins

__device__ __forceinline__ uint32_t r_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void r_bulk(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(r_smem(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(r_smem(dst)),
      "l"(src), "r"(bytes), "r"(r_smem(bar))
      : "memory");
}

// Bulk copy whose bytes count against an expect_tx made earlier on the same barrier.
__device__ __forceinline__ void r_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
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
// pipeline slots back and forth between the producer warps and the consumer warps.
// Id 1: consumers only.  Ids 2+b: slot b staged.  Ids 4+b: slot b free.  Id 6: producers.
__device__ __forceinline__ void nb_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void nb_arrive(int id, int n) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// u16 -> float exactly, on the FMA/ALU pipes: 2^23 + x has x in its low mantissa bits
__device__ __forceinline__ float u16lo_to_f(uint32_t w) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7610)) - 8388608.0f;
}
__device__ __forceinline__ float u16hi_to_f(uint32_t w) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7632)) - 8388608.0f;
}

// The FPL frame values of one staged pixel for this lane, dark subtracted.
#ifdef MI_RUNS_ACC32
using Acc = float;
#else
using Acc = double;
#endif

template <bool kU16, int FPL, int FG>
__device__ __forceinline__ void staged_values(const uint8_t *s_val, uint32_t u, int lane, float *v) {
  const uint8_t *row = s_val + u * (uint32_t)kRunPitch;
  if constexpr (kU16 && FPL == 2) {
    const uint32_t w2 = *(const uint32_t *)(row + 4 * lane);
    const float d = *(const float *)(row + FG * 2);
    v[0] = u16lo_to_f(w2) - d;
    v[1] = u16hi_to_f(w2) - d;
  } else if constexpr (kU16) {
    v[0] = (float)*(const uint16_t *)(row + 2 * lane) - *(const float *)(row + FG * 2);
  } else {
    v[0] = *(const float *)(row + 4 * lane);
  }
}

// Per-slot schedule record written by the producers: which item, frame group and
// tile the slot holds (item < 0: no more work for this CTA).
struct SlotTag {
  int32_t item, g, t, nt;          // item, frame group, tile of the item, tiles of the item
  int32_t r0, n_rows, slot, pad;   // the item's rows and lineout slot
};

template <typename T, int G, int L, bool XC, int NP>
__global__ void __launch_bounds__((kRunWarps + NP) * 32, kRunCtasPerSm) k_runs(RunArgs a) {
  constexpr bool kU16 = sizeof(T) <= 2;              // staged as u16
  constexpr int FG = runs_frames_per_group(sizeof(T), G);
  constexpr int FPL = FG / 32;                       // frames per lane
  constexpr int NRS = G - L + 2;
  constexpr int NC = kRunWarps;                      // consumer warps
  constexpr int NCT = NC * 32;
  constexpr int NPT = NP * 32;                       // producer threads
  constexpr int NALL = NCT + NPT;
  static_assert(!XC || (kU16 && FG == kXcFrames) || (!kU16 && FG == kXcFramesF),
                "pixel-major staging holds 128-byte frame groups");
  extern __shared__ __align__(16) uint8_t smem[];
  float *s_part = (float *)(smem + a.off_part);      // [NC units][G][FG]
  double *s_lo = (double *)(smem + a.off_lo);        // [rows][FG][2]
  uint64_t *bar = (uint64_t *)(smem + a.off_bar);    // [0,1]: blob of slot b; [2,3]: staging of slot b
  __shared__ SlotTag s_tag[2];
  __shared__ int s_abort, s_next;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nbp = a.nbp;
  const int n_groups = (a.F + FG - 1) / FG;

  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(r_smem(&bar[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();

  if (warp >= NC) {
    // ================= producers: claim work items, bring tile blobs in (TMA), stage pixels
    const int ptid = tid - NCT;
    const T *frames = (const T *)a.frames;
    int k = 0, item = -1, nt = 0, g = 0, t = 0;
    WorkItem it{};
    // the claim of the next item is issued when the current one starts, so its latency
    // overlaps the current item's tiles
    int next_claim = (ptid == 0) ? atomicAdd(a.counter, 1) : 0;
    for (;; ++k) {
      const int b = k & 1;
      // next (item, group, tile); items are claimed from the launch's counter
      if (item >= 0 && ++t == nt) {
        t = 0;
        if (++g == n_groups) item = -1;
      }
      while (item < 0) {
        if (ptid == 0) s_next = next_claim;
        asm volatile("bar.sync 6, %0;" ::"r"(NPT) : "memory");
        const int claimed = s_next;
        asm volatile("bar.sync 6, %0;" ::"r"(NPT) : "memory");
        if (claimed >= a.n_items) break;
        if (ptid == 0) next_claim = atomicAdd(a.counter, 1);
        it = a.items[claimed];
        nt = it.tile_end - it.tile_begin;
        g = 0;
        t = 0;
        if (nt > 0) item = claimed;
      }
      TileRef tref{};
      if (ptid == 0 && item >= 0) tref = a.tiles[it.tile_begin + t];   // in flight during the wait
      if (k >= 2) nb_sync(4 + b, NALL);              // consumers are done with slot b (step k-2)
      if (item < 0) {
        if (ptid == 0) s_tag[b] = SlotTag{-1, 0, 0, 0, 0, 0, 0, 0};
        nb_arrive(2 + b, NALL);
        break;
      }
      const int g0 = g * FG;
      const int fg_n = min(FG, a.F - g0);
      uint8_t *slot = smem + b * a.slot_bytes;
      if (ptid == 0) {
        s_tag[b] = SlotTag{item, g, t, nt, it.r0, it.n_rows, it.slot, 0};
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        r_bulk(slot, a.blobs + tref.off, tref.bytes, &bar[b]);
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
      if constexpr (XC) {
        // one 128-byte bulk copy per staged pixel from the pixel-major buffer (frame group g);
        // the staging barrier of slot b expects all of them before any is issued
        constexpr uint32_t kRow = 128;
        if (ptid == 0)
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(r_smem(&bar[2 + b])),
                       "r"((uint32_t)h.n_u * kRow)
                       : "memory");
        asm volatile("bar.sync 6, %0;" ::"r"(NPT) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint8_t *xg = a.xc + (size_t)g * kRow;
        for (int u = ptid; u < h.n_u; u += NPT) {
          const uint32_t pix = upix[u];
          const uint32_t z = pix / (uint32_t)a.ny;
          const uint32_t c = (uint32_t)__ldg(a.row_off + z) + (pix - z * (uint32_t)a.ny) - (uint32_t)__ldg(a.span_lo + z);
          uint8_t *row = s_val + (size_t)u * kRunPitch;
          r_copy(row, xg + (size_t)c * a.xc_pitch, kRow, &bar[2 + b]);
          if constexpr (kU16) *(float *)(row + kRow) = __ldg(a.dark + pix);   // beside the copied bytes
        }
        nb_arrive(2 + b, NALL);                       // copies issued, darks written
        continue;
      }
      for (int u = ptid; u < h.n_u; u += NPT) {
        const uint32_t pix = upix[u];
        const float d = __ldg(a.dark + pix);
        const T *src = frames + (int64_t)g0 * a.stride + pix;
        uint8_t *row = s_val + (size_t)u * kRunPitch;
        if constexpr (kU16) {
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
          *(float *)(row + FG * 2) = d;
        } else {
          float v[32];
#pragma unroll
          for (int f = 0; f < 32; ++f) v[f] = (f < fg_n) ? r_cvt(__ldg(src + (int64_t)f * a.stride)) - d : 0.0f;
          float4 *dst = (float4 *)row;
#pragma unroll
          for (int q = 0; q < 8; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
      }
      nb_arrive(2 + b, NALL);                         // slot b staged
    }
    // take the consumers' last two slot releases so no barrier generation is left open
    for (int kk = k + 1; kk < k + 3; ++kk)
      if (kk >= 2) nb_sync(4 + (kk & 1), NALL);
    return;
  }

  // ================= consumers: records -> registers -> combine -> cake + lineouts
  for (int k = 0;; ++k) {
    const int b = k & 1;
    const uint8_t *blob = smem + b * a.slot_bytes;
    const uint8_t *s_val = blob + a.off_val;
    nb_sync(2 + b, NALL);                             // slot b staged (or the end marker)
    if (s_abort) return;
    const SlotTag tag = s_tag[b];
    if (tag.item < 0) {
      nb_arrive(4 + b, NALL);
      return;
    }
    const int nt = tag.nt;
    const int t = tag.t, g0 = tag.g * FG;
    const int fg_n = min(FG, a.F - g0);
    if (t == 0)
      for (int i = tid; i < FG * a.rows_max * 2; i += NCT) s_lo[i] = 0.0;
    // the blob and the staging were written by bulk copies (async proxy): observe their phases
    if (!r_wait(&bar[b], (uint32_t)((k >> 1) & 1))) atomicExch(a.err, MI_E_TIMEOUT);
    if constexpr (XC) {
      if (!r_wait(&bar[2 + b], (uint32_t)((k >> 1) & 1))) atomicExch(a.err, MI_E_TIMEOUT);
    }
    const TileHdr h = *(const TileHdr *)blob;
    uint32_t o_rsp, o_sc, o_lw, o_up, o_lc, o_w;
    runs_blob_layout(h.nb, h.n_cols, h.nnz, h.n_u, G, L, &o_rsp, &o_sc, &o_lw, &o_up, &o_lc, &o_w);
    const uint16_t *rsp = (const uint16_t *)(blob + o_rsp);
    const double *scale = (const double *)(blob + o_sc);
    const float *lw = (const float *)(blob + o_lw);
    const uint16_t *lcol = (const uint16_t *)(blob + o_lc);
    const float *wts = (const float *)(blob + o_w);
    const uint16_t *units = (const uint16_t *)(blob + kRunUnitsOff);
    const uint32_t *strips = (const uint32_t *)(units + 4 * kRunWarps);   // {first unit | count << 16}

    const int ns = h.n_cols;
    // FP64 accumulation of the exact FP64 products of the FP32 weights and staged values
    // (compensates the FP32 rounding of long sums); built with MI_RUNS_ACC32: FP32
    Acc acc[G][FPL];
#pragma unroll
    for (int i = 0; i < G; ++i)
#pragma unroll
      for (int p = 0; p < FPL; ++p) acc[i][p] = (Acc)0;
    {
      // this warp's unit: records [j0, j1) of strip s, walked rs by rs
      const uint2 ud = *(const uint2 *)(units + 4 * warp);
      const int s = ud.x & 0xFFFF, j0 = ud.x >> 16, j1 = ud.y & 0xFFFF;
      const uint16_t *rp = rsp + s * NRS;
#pragma unroll
      for (int rs = 0; rs <= G - L; ++rs) {
        const int jb = max((int)rp[rs], j0), je = min((int)rp[rs + 1], j1);
        int j = jb;
        // kRecBatch records per iteration: all their loads in flight before the
        // conversions and FMAs
        for (; j + kRecBatch - 1 < je; j += kRecBatch) {
          uint32_t uu[kRecBatch];
#pragma unroll
          for (int r = 0; r < kRecBatch; ++r) uu[r] = lcol[j + r];
          float vv[kRecBatch][FPL], ww[kRecBatch][L];
#pragma unroll
          for (int r = 0; r < kRecBatch; ++r) {
            staged_values<kU16, FPL, FG>(s_val, uu[r], lane, vv[r]);
            load_weights<L>(wts + (size_t)(j + r) * L, ww[r]);
          }
#pragma unroll
          for (int r = 0; r < kRecBatch; ++r)
#pragma unroll
            for (int q = 0; q < L; ++q)
#pragma unroll
              for (int p = 0; p < FPL; ++p) acc[rs + q][p] = fma((Acc)ww[r][q], (Acc)vv[r][p], acc[rs + q][p]);
        }
        for (; j < je; ++j) {
          float v0[FPL], w0[L];
          staged_values<kU16, FPL, FG>(s_val, lcol[j], lane, v0);
          load_weights<L>(wts + (size_t)j * L, w0);
#pragma unroll
          for (int q = 0; q < L; ++q)
#pragma unroll
            for (int p = 0; p < FPL; ++p) acc[rs + q][p] = fma((Acc)w0[q], (Acc)v0[p], acc[rs + q][p]);
        }
      }
      // unit partials
#pragma unroll
      for (int i = 0; i < G; ++i) {
        float *d = s_part + ((size_t)warp * G + i) * FG + lane * FPL;
        if constexpr (FPL == 2) *(float2 *)d = make_float2((float)acc[i][0], (float)acc[i][1]);
        else d[0] = (float)acc[i][0];
      }
    }
    nb_sync(1, NCT);                     // unit partials written; staging of slot b consumed

    // ---- combine (fixed unit order), scale, lineout partials: warp per row, lanes = frames;
    // the bin results go to slot b's staging area, which the record loop no longer reads
    float *s_out = (float *)(smem + b * a.slot_bytes + a.off_val);   // [FG][nbp]
    for (int i = warp; i < h.n_rows; i += NC) {
      double saw[FPL], ssm[FPL];
#pragma unroll
      for (int p = 0; p < FPL; ++p) saw[p] = ssm[p] = 0.0;
      for (int s = 0; s < ns; ++s) {
        const uint32_t st = strips[s];
        const int u0 = st & 0xFFFF, nu = st >> 16;
        double v[FPL];
#pragma unroll
        for (int p = 0; p < FPL; ++p) v[p] = 0.0;
        for (int kk = 0; kk < nu; ++kk) {
          const float *src = s_part + ((size_t)(u0 + kk) * G + i) * FG + lane * FPL;
          if constexpr (FPL == 2) {
            const float2 t2 = *(const float2 *)src;
            v[0] += (double)t2.x;
            v[1] += (double)t2.y;
          } else {
            v[0] += (double)src[0];
          }
        }
        const int bb = i * ns + s;
        const double sc = scale[bb];
        const float l = lw[bb];
#pragma unroll
        for (int p = 0; p < FPL; ++p) {
          const double o = v[p] * sc;
          s_out[(lane * FPL + p) * nbp + bb] = (float)o;
          saw[p] += o * (double)l;
          ssm[p] += (l > 0.0f) ? o : 0.0;
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

    // ---- cake store: warp per frame, lanes over the tile's bins (runs of n_cols contiguous
    // floats per row); row/col from a float reciprocal (exact for b < 2^12)
    if (a.want_cake) {
      // the bins this lane stores (bb = lane + 32 k) and their offsets in a frame's cake,
      // computed once per tile; tiles hold at most kStoreSlots * 32 bins
      const float inv_ns = 1.0f / (float)ns;
      int off[kStoreSlots];
#pragma unroll
      for (int k = 0; k < kStoreSlots; ++k) {
        const int bb = lane + 32 * k;
        const int r = (int)(((float)bb + 0.5f) * inv_ns);
        off[k] = bb < h.nb ? r * a.n_eta + (bb - r * ns) : -1;
      }
      const int64_t tile0 = (int64_t)h.r0 * a.n_eta + h.e0;
      for (int f = warp; f < fg_n; f += NC) {
        float *dst = a.cake + (int64_t)(g0 + f) * a.n_bins + tile0;
        const float *src = s_out + f * nbp + lane;
#pragma unroll
        for (int k = 0; k < kStoreSlots; ++k)
          if (off[k] >= 0) dst[off[k]] = src[32 * k];
      }
    }
    if (t == nt - 1 && a.want_lo) {
      for (int f = warp; f < fg_n; f += NC)
        for (int r = lane; r < tag.n_rows; r += 32) {
          const double *src = s_lo + ((size_t)r * FG + f) * 2;
          double *dst = a.partial + (((int64_t)(g0 + f) * a.n_r + tag.r0 + r) * a.n_slots + tag.slot) * 2;
          dst[0] = src[0];
          dst[1] = src[1];
        }
    }
    // this warp is done with slot b (blob, bin results): hand it back to the producers, whose
    // bulk copies (async proxy) will overwrite the bin results written here
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    nb_arrive(4 + b, NALL);
    nb_sync(1, NCT);                     // s_lo / s_part free for the next step
  }
}

template <typename T, int G, int L, bool XC, int NP>
static int launch_runs_t(Plan *p, RunArgs &a, cudaStream_t s) {
  const size_t smem = runs_smem_layout(a.blob_cap, std::max(p->max_u, 1), a.nbp, a.rows_max, G,
                                       runs_frames_per_group(sizeof(T), G), &a.off_val, &a.slot_bytes, &a.off_part,
                                       &a.off_lo, &a.off_bar);
  int dev_smem = 0;
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
  if (smem + 64 > (size_t)dev_smem)
    return set_error(MI_E_RANGE, "run kernel needs %zu B shared memory (> %d)", smem, dev_smem);
  auto kern = k_runs<T, G, L, XC, NP>;
  MI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  MI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  // persistent: one CTA per SM claims work items (heaviest first) from a counter
  MI_CUDA(cudaMemsetAsync(p->d_ctr, 0, sizeof(int), s));
  const int grid = std::max(1, std::min(p->n_items, p->n_sms * kRunCtasPerSm));
  kern<<<grid, (kRunWarps + NP) * 32, smem, s>>>(a);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

template <typename T>
static int launch_runs_gl(Plan *p, RunArgs &a, cudaStream_t s) {
  const int G = p->run_g, L = p->run_l;
  if (G == 8 && L == 2) return launch_runs_t<T, 8, 2, false, kRunProducerWarps>(p, a, s);
  if (G == 8 && L == 4) return launch_runs_t<T, 8, 4, false, kRunProducerWarps>(p, a, s);
  if (G == 16 && L == 4) return launch_runs_t<T, 16, 4, false, kRunProducerWarps>(p, a, s);
  if (G == 16 && L == 8) return launch_runs_t<T, 16, 8, false, kRunProducerWarps>(p, a, s);
  if (G == 32 && L == 4) return launch_runs_t<T, 32, 4, false, kRunProducerWarps>(p, a, s);
  if (G == 32 && L == 8) return launch_runs_t<T, 32, 8, false, kRunProducerWarps>(p, a, s);
  return set_error(MI_E_UNSUPPORTED, "run encoding with G=%d L=%d", G, L);
}

// pixel-major staging (spans exist for G <= 16): u16 rows (8/16-bit frames) or fp32 rows
template <typename T>
static int launch_runs_xc(Plan *p, RunArgs &a, cudaStream_t s) {
  const int G = p->run_g, L = p->run_l;
  if (G == 8 && L == 2) return launch_runs_t<T, 8, 2, true, kRunProducersXc>(p, a, s);
  if (G == 8 && L == 4) return launch_runs_t<T, 8, 4, true, kRunProducersXc>(p, a, s);
  if (G == 16 && L == 4) return launch_runs_t<T, 16, 4, true, kRunProducersXc>(p, a, s);
  if (G == 16 && L == 8) return launch_runs_t<T, 16, 8, true, kRunProducersXc>(p, a, s);
  return set_error(MI_E_UNSUPPORTED, "pixel-major staging with G=%d L=%d", G, L);
}

static RunArgs run_args(Plan *p, float *cake, bool want_lo) {
  RunArgs a;
  a.items = p->d_items;
  a.tiles = p->d_tiles;
  a.blobs = p->d_blobs;
  a.frames = nullptr;
  a.stride = 0;
  a.F = 0;
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
  a.n_items = p->n_items;
  a.counter = p->d_ctr;
  a.xc = p->d_xc;
  a.xc_pitch = kXcRowBytes;
  a.span_lo = p->d_span_lo;
  a.row_off = p->d_row_off;
  a.ny = p->ny;
  return a;
}

int launch_runs_staged(Plan *p, bool as_f32, int F, float *cake, double *partial, bool want_lo, cudaStream_t s) {
  RunArgs a = run_args(p, cake, want_lo);
  a.F = F;
  a.partial = partial;
  return as_f32 ? launch_runs_xc<float>(p, a, s) : launch_runs_xc<uint16_t>(p, a, s);
}

int launch_runs(Plan *p, const void *frames, int dtype, int n_frames, int64_t stride, float *cake, double *partial,
                bool want_lo, cudaStream_t s) {
  RunArgs a = run_args(p, cake, want_lo);
  a.partial = partial;
  a.frames = frames;
  a.stride = stride;
  a.F = n_frames;
  if (runs_uses_xc(p, dtype)) {
    // kernel (a) transposes a chunk of frames into the pixel-major buffer, kernel (b) stages
    // from it; the partial sums of frame f live at row f of the scratch
    const bool as_f32 = !(dtype == MI_DT_U16 || dtype == MI_DT_U8);
    const size_t es = dtype_size(dtype);
    const int chunk = as_f32 ? kXcFramesF * kXcGroupsF : kXcFrames * kXcGroups;
    for (int f0 = 0; f0 < n_frames; f0 += chunk) {
      const int nf = std::min(chunk, n_frames - f0);
      int rc = launch_xc(p, 0, (const uint8_t *)frames + (size_t)f0 * stride * es, dtype, nf, stride, as_f32, s);
      if (rc) return rc;
      rc = launch_runs_staged(p, as_f32, nf, cake ? cake + (size_t)f0 * p->n_bins : nullptr,
                              partial + (size_t)f0 * p->n_r * p->n_slots * 2, want_lo, s);
      if (rc) return rc;
    }
    return MI_OK;
  }
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
