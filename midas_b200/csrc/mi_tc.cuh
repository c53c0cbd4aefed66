// mi_tc.cuh -- PTX helpers of the tensor-core caking kernels (mi_mma.cu, mi_mmad.cu):
// mbarriers with bounded waits, bulk copies, shared-memory matrix descriptors, tcgen05
// commit / fences / TMEM loads, and the driver's tensor-map encoder.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mi_internal.h"

namespace mi {

constexpr uint32_t kMmaWaitLimit = 1u << 26;   // mbarrier polls before a wait is declared lost

__device__ __forceinline__ uint32_t m_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool m_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = m_smem(bar);
  for (uint32_t it = 0; it < kMmaWaitLimit; ++it) {
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

__device__ __forceinline__ void m_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(m_smem(bar)) : "memory");
}
__device__ __forceinline__ void m_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(m_smem(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void m_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(m_smem(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void m_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(m_smem(dst)),
      "l"(src), "r"(bytes), "r"(m_smem(bar))
      : "memory");
}

// shared-memory matrix descriptors (version 1): start address, leading / stride byte
// offsets in 16-byte units, layout type in bits 61-63 (0 = no swizzle, 2 = 128B swizzle)
__device__ __forceinline__ uint64_t m_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}

__device__ __forceinline__ void m_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(m_smem(bar))
               : "memory");
}
__device__ __forceinline__ void m_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void m_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void m_ld16(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void m_ld8(uint32_t taddr, uint32_t *r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void m_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// The five int32 accumulators of a bin (byte shifts 0..4) as one value: sum_k 2^(8k) acc_k
// summed exactly in int64 on the integer pipe, then rounded once to FP64.  |acc_k| < 2^31,
// so |sum| < 2^31 (1 + 2^8 + 2^16 + 2^24 + 2^32) < 2^63.
__device__ __forceinline__ double m_acc5(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t a4) {
  const long long s = (long long)(int)a0 + (long long)(int)a1 * 256LL + (long long)(int)a2 * 65536LL +
                      (long long)(int)a3 * 16777216LL + (long long)(int)a4 * 4294967296LL;
  return __ll2double_rn(s);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda)
inline EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)f;
  }
  return fn;
}

// ---- cake store boxes of the tensor-core kernels.  An item's tiles leave in pairs: tiles 2i
// and 2i+1 (8 adjacent columns) share one shared-memory image and one TMA tensor store; an
// item's odd last tile goes alone (4 columns).  The tensor map views the [F][n_r][n_eta]
// cake as (n_eta, F, n_r), so a box's image is [rows][128 frames][columns]: the epilogue
// lane of frame m writes float4s 32 (pair) or 16 bytes apart from its neighbours'.  Pair
// images use the 32-byte swizzle (the 16-byte half of a row flipped when bit 7 of its
// address, here bit 2 of the frame, is set), so every 8 lanes of a warp cover the 32 banks
// once: 4 wavefronts per warp store, the minimum for 512 bytes.
constexpr int kCakeBoxes = 8;   // 4 and 8 columns x 12, 6, 3, 1 rows
__device__ __forceinline__ int cake_box_off(int row, int m, int pitch, int coff) {
  return (row * kMmaFrames + m) * pitch + (pitch == 2 * kMmaCols ? (coff ^ ((m & 4) ? kMmaCols : 0)) : coff);
}
__device__ __forceinline__ int cake_box_index(int box_rows, bool pair) {
  return (box_rows == kMmaRows ? 0 : (box_rows == 6 ? 1 : (box_rows == 3 ? 2 : 3))) + (pair ? 4 : 0);
}
// the eight maps of a call's cake (F frames); the caller has checked n_eta % 4 == 0 and a
// 16-byte aligned cake
inline int encode_cake_boxes(CUtensorMap *maps, float *cake, int n_eta, int n_r, int64_t n_bins, int F,
                             const char *who) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return set_error(MI_E_CUDA, "%s: cuTensorMapEncodeTiled is not available", who);
  const cuuint64_t dims[3] = {(cuuint64_t)n_eta, (cuuint64_t)F, (cuuint64_t)n_r};
  const cuuint64_t strides[2] = {(cuuint64_t)n_bins * 4u, (cuuint64_t)n_eta * 4u};
  const cuuint32_t estr[3] = {1, 1, 1};
  const int rows[4] = {kMmaRows, 6, 3, 1};
  for (int i = 0; i < kCakeBoxes; ++i) {
    const bool pair = i >= 4;
    const cuuint32_t box[3] = {(cuuint32_t)(pair ? 2 * kMmaCols : kMmaCols), (cuuint32_t)kMmaFrames,
                               (cuuint32_t)rows[i % 4]};
    const CUresult r = enc(&maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, cake, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, pair ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(MI_E_CUDA, "%s: cuTensorMapEncodeTiled failed (%d)", who, (int)r);
  }
  return MI_OK;
}

}  // namespace mi
