// noalloc.cu - left-right check that allocates nothing (csgm_lr_check_noalloc).
//
// Some callers cannot let the library allocate device memory: a JVM host that carves every
// device buffer out of one region it manages through its foreign-memory API, or a real-time
// capture loop in which cudaMalloc / cudaFree would synchronise the whole device and stall the
// other streams.  This entry point takes device pointers for all inputs and outputs and keeps the
// only scratch it needs in a fixed-size array in the module's static device memory.
//
// Check semantics: CensusSgm.java:181-201, identical to lr_check_kernel (stereo_kernels.cu).
// The rejected-pixel count is reduced through per-row partial counts in the scratch instead of a
// session-owned counter:
//   scratch[0 .. kLrMaxRows)  partial count of row y, written by the block of row y before it is
//                             read (needs no initial value);
//   scratch[kLrMaxRows]       number of finished rows; MUST be zero when a launch starts.  The
//                             entry point clears it on the caller's stream before every launch and
//                             the last block leaves it at zero.
// Two calls whose kernels overlap in time on one device (different streams, or different host
// threads without ordering) share the scratch and corrupt each other's count; serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "collinea_sgm.h"
#include "pipeline.h"
#include "sgm_device.cuh"

namespace csgm {
namespace {

constexpr int kLrMaxRows = 16384;  // rows supported by the static scratch (64 KiB of counts)
constexpr int kLrThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned int g_lr_scratch[kLrMaxRows + 64];

struct LrNoAllocArgs {
  const float* dl;
  const float* dr;
  float* out;
  uint8_t* reasons;
  unsigned long long* rejected;  // optional device output
  unsigned int* scratch;         // g_lr_scratch of the current device
  int w, h, wx, wy;
  double threshold;
};

// One block per row.
__global__ void __launch_bounds__(kLrThreads) lr_check_rows_kernel(LrNoAllocArgs a) {
  __shared__ unsigned int warp_counts[kLrThreads / 32];
  __shared__ bool last;
  const int y = blockIdx.x;
  const int rx = a.wx / 2, ry = a.wy / 2;
  unsigned int rejected = 0;
  for (int x = threadIdx.x; x < a.w; x += blockDim.x) {
    const int64_t p = (int64_t)y * a.w + x;
    float result = __int_as_float(0x7fc00000);
    if (x >= rx && x < a.w - rx && y >= ry && y < a.h - ry) {
      const float d = a.dl[p];
      if (isfinite(d)) {
        const int xr = java_round_float(__fsub_rn((float)x, d));
        if (xr < rx || xr >= a.w - rx) {
          if (a.reasons) a.reasons[p] = 4;
        } else {
          const float other = a.dr[(int64_t)y * a.w + xr];
          if (isfinite(other) && (double)fabsf(__fsub_rn(d, other)) <= a.threshold) {
            result = d;
          } else {
            rejected++;
            if (a.reasons) a.reasons[p] = 4;
          }
        }
      }
    }
    a.out[p] = result;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  rejected = __reduce_add_sync(0xffffffffu, rejected);
  if (lane == 0) warp_counts[warp] = rejected;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int row = 0;
    for (int i = 0; i < kLrThreads / 32; i++) row += warp_counts[i];
    a.scratch[y] = row;
    __threadfence();  // the row count is visible before this block is counted as finished
    last = atomicAdd(&a.scratch[kLrMaxRows], 1u) == (unsigned)a.h - 1;
  }
  __syncthreads();
  if (!last) return;
  // The last block to finish adds the row counts and leaves the finished-row counter at zero.
  __threadfence();
  unsigned long long total = 0;
  for (int r = threadIdx.x; r < a.h; r += blockDim.x)
    total += *(volatile unsigned int*)&a.scratch[r];
  total = __reduce_add_sync(0xffffffffu, (unsigned)total);  // per-warp sums fit 32 bits
  __shared__ unsigned long long block_total;
  if (threadIdx.x == 0) block_total = 0;
  __syncthreads();
  if (lane == 0) atomicAdd(&block_total, total);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (a.rejected) *a.rejected = block_total;
    a.scratch[kLrMaxRows] = 0;
  }
}

std::mutex g_setup_mutex;

// The scratch address per device, with the id of the context it was looked up in.
struct ScratchAddress {
  unsigned long long context = 0;  // cuCtxGetId of that context (0 = not looked up)
  unsigned int* ptr = nullptr;
};
ScratchAddress g_scratch[kMaxDevices];

// Unique id of the calling thread's current context (cuCtxGetCurrent + cuCtxGetId, reached
// through the runtime's driver entry points, so the library links no driver library).  Ids are
// never reused in a process, so a context recreated after cudaDeviceReset has a new one.
// Returns false while no context is current.
bool current_context_id(unsigned long long* id) {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return false;
    }
    get_current = (GetCurrent)a;
    get_id = (GetId)b;
  }
  void* ctx = nullptr;
  if (get_current(&ctx) != 0 || !ctx) return false;
  return get_id(ctx, id) == 0 && *id != 0;
}

// Address of the scratch array in the current device's copy of this module.  It is looked up on
// the first call made with the device current, and again whenever the device's context has been
// replaced since (after cudaDeviceReset, the old address would point into a context that is
// gone).  Checking the context costs two driver queries and allocates nothing.
int scratch_for_current_device(unsigned int** out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (device < 0 || device >= kMaxDevices)
    return fail(CSGM_E_UNSUPPORTED, "csgm_lr_check_noalloc: device ordinal %d >= %d", device,
                kMaxDevices);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  ScratchAddress& slot = g_scratch[device];
  unsigned long long id = 0;
  if (!current_context_id(&id) || id != slot.context || !slot.ptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lr_scratch);  // makes the device's primary context current
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(lr scratch)");
    if (!current_context_id(&id)) id = 0;  // no id: looked up again on the next call
    slot.context = id;
    slot.ptr = (unsigned int*)p;
  }
  *out = slot.ptr;
  return CSGM_OK;
}

}  // namespace
}  // namespace csgm

extern "C" int csgm_lr_check_noalloc(const float* disp_l, const float* disp_r, int32_t w,
                                     int32_t h, int32_t window_x, int32_t window_y,
                                     double lr_threshold, float* lr_checked, uint8_t* reasons,
                                     unsigned long long* lr_rejected, void* stream) {
  using namespace csgm;
  if (!disp_l || !disp_r || !lr_checked)
    return fail(CSGM_E_INVALID, "csgm_lr_check_noalloc: disp_l, disp_r and lr_checked are required");
  if (w < 1 || h < 1 || (int64_t)w * h > (int64_t)INT32_MAX)
    return fail(CSGM_E_INVALID, "csgm_lr_check_noalloc: invalid image size %dx%d", w, h);
  if (h > kLrMaxRows)
    return fail(CSGM_E_INVALID,
                "csgm_lr_check_noalloc: height %d exceeds the %d rows its static scratch holds", h,
                kLrMaxRows);
  for (int size : {window_x, window_y})
    if (size < 3 || size > 11 || size % 2 == 0)
      return fail(CSGM_E_INVALID, "Census window must be odd, 3..11");
  if (!(lr_threshold > 0)) return fail(CSGM_E_INVALID, "lr_threshold must be positive");
  unsigned int* scratch = nullptr;
  int status = scratch_for_current_device(&scratch);
  if (status) return status;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(scratch + kLrMaxRows, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return cuda_fail(e, "csgm_lr_check_noalloc: counter clear");
  LrNoAllocArgs a{disp_l, disp_r, lr_checked, reasons, lr_rejected, scratch,
                  w, h, window_x, window_y, lr_threshold};
  lr_check_rows_kernel<<<h, kLrThreads, 0, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "csgm_lr_check_noalloc: launch");
  return CSGM_OK;
}
