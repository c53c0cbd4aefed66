// mi_static.cu -- mi_integrate_batch_static: batched caking that allocates nothing.
//
// Some callers cannot have device memory allocated on their behalf once they are
// running: a detector front-end that reserves the device's whole memory budget at
// start-up and hands the library only its own buffers.  This entry point runs the same kernels as mi_integrate_batch
// (batched caking + lineout reduction) but keeps their only scratch -- the per-row
// lineout partial sums -- in a fixed array compiled into the library, so a call
// touches nothing but the plan, the caller's frames and outputs, and that array.
//
// The array holds kStaticScratchDoubles doubles (8 MiB) on every GPU that loads the
// library, until the process exits.  A batch needs n_r x 12 x 2 doubles per frame;
// batches are processed in chunks that fit, and a plan whose single frame does not
// fit is rejected with MI_E_RANGE.  The first call on a device looks up the array's
// device address (cudaGetSymbolAddress) -- make that first call before any stream
// capture.  The address is kept for the life of the process, so a device reset
// (cudaDeviceReset, or a reset of the primary context) while the library is loaded is not
// supported: the module reloads and the kept address goes stale.  All calls share the
// array: calls that overlap on the GPU (other streams, other threads) race on it.  Nothing
// in it must start at zero: every launch writes every partial it later reads.  A call
// copies nothing of the plan; it passes the array to the same launchers as
// mi_integrate_batch.  On a tensor-core (MMA) plan the chunk is at most what the array
// holds (a 3960 x 360 bin plan with 12 partial slots per row: 11 frames per launch), and
// that encoding's cost is per pass over the map, so such a plan runs slower per frame here
// than through mi_integrate_batch.
#include <mutex>

#include "mi_internal.h"

namespace mi {

constexpr size_t kStaticScratchDoubles = (size_t)1 << 20;  // 8 MiB
static __device__ __align__(256) double g_static_partial[kStaticScratchDoubles];

constexpr int kStaticMaxDevices = 64;
static std::mutex g_static_mu;
static double *g_static_ptr[kStaticMaxDevices] = {};

// Device address of the fixed array on `device` (looked up once, with that device current).
static int static_scratch(int device, double **out) {
  if (device < 0 || device >= kStaticMaxDevices)
    return set_error(MI_E_RANGE, "mi_integrate_batch_static: device %d beyond %d", device, kStaticMaxDevices);
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[device]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_partial);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_static_partial)", __FILE__, __LINE__);
    g_static_ptr[device] = (double *)ptr;
  }
  *out = g_static_ptr[device];
  return MI_OK;
}

}  // namespace mi

using namespace mi;

struct mi_plan : public mi::Plan {};

extern "C" int mi_integrate_batch_static(mi_plan *p, const void *frames, int dtype, int n_frames, int64_t stride,
                                         float *cake, double *lo_aw, double *lo_sm, void *stream) {
  if (!p || !frames) return set_error(MI_E_ARG, "mi_integrate_batch_static: null argument");
  if (n_frames < 0) return set_error(MI_E_ARG, "mi_integrate_batch_static: n_frames < 0");
  if (dtype_size(dtype) == 0)
    return set_error(MI_E_ARG, "mi_integrate_batch_static: unknown dtype code %d", dtype);
  if (stride < (int64_t)p->ny * p->nz)
    return set_error(MI_E_ARG, "mi_integrate_batch_static: frame_stride %lld < ny*nz", (long long)stride);
  const size_t per_frame = (size_t)p->n_r * (size_t)p->n_slots * 2;
  if (per_frame > kStaticScratchDoubles)
    return set_error(MI_E_RANGE,
                     "mi_integrate_batch_static: the plan needs %zu doubles of lineout scratch per frame; "
                     "the fixed array holds %zu (use mi_integrate_batch)",
                     per_frame, kStaticScratchDoubles);
  if (n_frames == 0) return MI_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != p->device) MI_CUDA(cudaSetDevice(p->device));
  double *scratch = nullptr;
  int rc = static_scratch(p->device, &scratch);
  if (rc == MI_OK) {
    // the same launches as mi_integrate_batch, with the lineout partials in the fixed array
    const int chunk = (int)std::min<size_t>((size_t)kMaxFramesPerLaunch, kStaticScratchDoubles / per_frame);
    const size_t es = dtype_size(dtype);
    for (int f0 = 0; f0 < n_frames && rc == MI_OK; f0 += chunk) {
      const int nf = std::min(chunk, n_frames - f0);
      rc = launch_cake(p, (const uint8_t *)frames + (size_t)f0 * stride * es, dtype, nf, stride,
                       cake ? cake + (size_t)f0 * p->n_bins : nullptr, lo_aw ? lo_aw + (size_t)f0 * p->n_r : nullptr,
                       lo_sm ? lo_sm + (size_t)f0 * p->n_r : nullptr, scratch, (cudaStream_t)stream);
    }
  }
  if (prev != p->device) cudaSetDevice(prev);
  return rc;
}
