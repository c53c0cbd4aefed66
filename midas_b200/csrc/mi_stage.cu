// mi_stage.cu -- kernel (a) of the batched path for 8/16-bit frames: pixel-major staging.
//
// The reference casts each frame to float and subtracts the dark per pixel before the
// per-bin sums (process_direct_kernel<T>, FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:
// 1148-1160).  Here the cast and the dark stay in the caking kernel (the dark is
// subtracted per staged value, (float)raw - dark, as the reference does); this kernel
// only changes the layout: the up to 128 frames of a launch are transposed from
// frame-major [f][z][y] to pixel-major xc[c][f] over the compact pixel index c of the
// plan's row spans, so a tile stages each of its pixels (64 frames of one group) with one
// 128-byte bulk copy instead of 64 scattered 2-byte loads.
//
// One CTA per chunk (<= 256 pixels of one span): 16-byte loads of the chunk's frame
// rows into shared memory (16-byte groups XOR-swizzled by frame octet so the
// transposed reads are conflict-free), then 16-byte stores of 8 frames of one pixel,
// eight consecutive threads writing one pixel's 128-byte row of a frame group.
#include <stdint.h>

#include "mi_internal.h"

namespace mi {

template <typename T, bool VEC>
__global__ void __launch_bounds__(256) k_xc(const T *__restrict__ frames, int64_t stride, int F, int ny,
                                            const XcChunk *__restrict__ chunks, uint16_t *__restrict__ xc) {
  constexpr int kPitch = kXcFrames * kXcGroups;
  __shared__ __align__(16) uint16_t S[kXcFrames][kXcChunk + 8];
  const XcChunk ch = chunks[blockIdx.x];
  const int nv = (ch.n + 7) >> 3;  // groups of 8 pixels
  const int64_t base = (int64_t)ch.z * ny + ch.y0;
  for (int h = 0; h * kXcFrames < F; ++h) {
    const int fh = min(kXcFrames, F - h * kXcFrames);
    if (h) __syncthreads();
    for (int i = threadIdx.x; i < kXcFrames * nv; i += blockDim.x) {
      const int f = i / nv, v = i - f * nv;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (f < fh) {
        const T *src = frames + (int64_t)(h * kXcFrames + f) * stride + base + 8 * v;
        if constexpr (VEC) {
          val = __ldg((const uint4 *)src);
        } else {
          uint32_t t[4];
#pragma unroll
          for (int j = 0; j < 8; j += 2) {
            const uint32_t lo = (8 * v + j < ch.n) ? (uint32_t)(uint16_t)__ldg(src + j) : 0u;
            const uint32_t hi = (8 * v + j + 1 < ch.n) ? (uint32_t)(uint16_t)__ldg(src + j + 1) : 0u;
            t[j / 2] = lo | (hi << 16);
          }
          val = make_uint4(t[0], t[1], t[2], t[3]);
        }
      }
      *(uint4 *)&S[f][8 * (v ^ ((f >> 3) & 7))] = val;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ch.n * 8; i += blockDim.x) {
      const int p = i >> 3, q = i & 7;
      const int col = 8 * ((p >> 3) ^ q) + (p & 7);
      uint32_t w[4];
#pragma unroll
      for (int j = 0; j < 8; j += 2)
        w[j / 2] = (uint32_t)S[8 * q + j][col] | ((uint32_t)S[8 * q + j + 1][col] << 16);
      *(uint4 *)(xc + (int64_t)(ch.c0 + p) * kPitch + h * kXcFrames + 8 * q) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

bool runs_uses_xc(const Plan *p, int dtype) {
  return p->n_xc > 0 && (dtype == MI_DT_U16 || dtype == MI_DT_U8);
}

// Transpose frames [0, F) (F <= kXcFrames * kXcGroups) of a launch into the plan's
// pixel-major buffer.
int launch_xc(Plan *p, const void *frames, int dtype, int F, int64_t stride, cudaStream_t s) {
  if (F <= 0 || F > kXcFrames * kXcGroups)
    return set_error(MI_E_ARG, "launch_xc: %d frames (1..%d)", F, kXcFrames * kXcGroups);
  if (p->n_xchunks == 0) return MI_OK;
  const unsigned grid = (unsigned)p->n_xchunks;
  if (dtype == MI_DT_U16) {
    const bool vec = ((uintptr_t)frames % 16 == 0) && ((stride * 2) % 16 == 0) && ((p->ny * 2) % 16 == 0);
    if (vec)
      k_xc<uint16_t, true><<<grid, 256, 0, s>>>((const uint16_t *)frames, stride, F, p->ny, p->d_xchunks, p->d_xc);
    else
      k_xc<uint16_t, false><<<grid, 256, 0, s>>>((const uint16_t *)frames, stride, F, p->ny, p->d_xchunks, p->d_xc);
  } else if (dtype == MI_DT_U8) {
    k_xc<uint8_t, false><<<grid, 256, 0, s>>>((const uint8_t *)frames, stride, F, p->ny, p->d_xchunks, p->d_xc);
  } else {
    return set_error(MI_E_ARG, "launch_xc: dtype %d is not staged pixel-major", dtype);
  }
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

}  // namespace mi
