// capi.cu - the C ABI of include/collinea_sgm.h: sessions, budgeted device workspace, profiling
// and the per-pair / per-view pipelines.  No CPU fallback: every failure is returned as a status
// with a thread-local message (the reference's exceptions, GpuSgm.java:56-58,260-265).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "collinea_sgm.h"
#include "pipeline.h"
#include "stereo_kernels.h"

namespace csgm {

static thread_local std::string g_error;

int fail(int status, const char* fmt, ...) {
  char buffer[512];
  va_list args;
  va_start(args, fmt);
  vsnprintf(buffer, sizeof buffer, fmt, args);
  va_end(args);
  g_error = buffer;
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a non-sticky error so the session stays usable
  int status = e == cudaErrorMemoryAllocation ? CSGM_E_NOMEM : CSGM_E_CUDA;
  return fail(status, "%s failed (CUDA %d: %s)", what, (int)e, cudaGetErrorString(e));
}

static int64_t java_round_host(double v) {
  double f = std::floor(v);
  return (int64_t)(v - f >= 0.5 ? f + 1.0 : f);
}

// ---------------------------------------------------------------------------------------------
// Session workspace.

void* Workspace::get(int slot, size_t bytes, int* status) {
  Buffer& b = buffers[slot];
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return b.ptr;
  if (b.ptr) {
    if (async_stream)
      cudaFreeAsync(b.ptr, async_stream);
    else
      cudaFree(b.ptr);
    allocated -= b.bytes;
    b.ptr = nullptr;
    b.bytes = 0;
  }
  if (allocated + bytes > budget) {
    *status = fail(CSGM_E_NOMEM, "GPU SGM workspace exceeds the device budget (%.1f MiB > %.1f MiB)",
                   (allocated + bytes) / 1048576.0, budget / 1048576.0);
    return nullptr;
  }
  generation++;
  cudaError_t e = async_stream ? cudaMallocAsync(&b.ptr, bytes, async_stream) : cudaMalloc(&b.ptr, bytes);
  if (e != cudaSuccess) {
    *status = cuda_fail(e, "GPU buffer allocation");
    b.ptr = nullptr;
    return nullptr;
  }
  b.bytes = bytes;
  allocated += bytes;
  return b.ptr;
}

void Workspace::release(int slot) {
  Buffer& b = buffers[slot];
  if (!b.ptr) return;
  generation++;
  if (async_stream)
    cudaFreeAsync(b.ptr, async_stream);
  else
    cudaFree(b.ptr);
  allocated -= b.bytes;
  b.ptr = nullptr;
  b.bytes = 0;
}

void Workspace::release_all() {
  generation++;
  for (auto& b : buffers)
    if (b.ptr) {
      if (async_stream)
        cudaFreeAsync(b.ptr, async_stream);
      else
        cudaFree(b.ptr);
      b.ptr = nullptr;
      b.bytes = 0;
    }
  allocated = 0;
}

// ---------------------------------------------------------------------------------------------
// Profiling: events bracket every launch at level 2; the sums are collected after the call's
// stream synchronisation.

void Profiler::begin_call(cudaStream_t s) {
  stream = s;
  if (pending.empty()) used = 0;  // events of uncollected asynchronous calls stay reserved
}

cudaEvent_t Profiler::event() {
  if (used == events.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    events.push_back(e);
  }
  return events[used++];
}

void Profiler::kernel_begin() {
  if (level < 2) return;
  current_start = event();
  cudaEventRecord(current_start, stream);
}

void Profiler::kernel_end(const char* name) {
  launches++;
  if (level < 2) return;
  cudaEvent_t stop = event();
  cudaEventRecord(stop, stream);
  pending.push_back({name, current_start, stop});
}

void Profiler::collect() {
  for (auto& p : pending) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p.start, p.stop) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    KernelTotal* slot = nullptr;
    for (auto& k : kernels)
      if (k.name == p.name) slot = &k;
    if (!slot) {
      kernels.push_back({p.name, 0, 0});
      slot = &kernels.back();
    }
    slot->launches++;
    slot->total_ns += (int64_t)((double)ms * 1e6);
  }
  pending.clear();
}

Profiler::~Profiler() {
  for (auto e : events) cudaEventDestroy(e);
}

}  // namespace csgm

using namespace csgm;

namespace csgm {

void session_settings(Context& ctx, csgm_session* s, const csgm_params& p, int w, int h) {
  ctx.wait_limit = s->wait_limit;
  ctx.sgm_mode = s->sgm_mode;
  ctx.strip_rows = s->strip_rows;
  ctx.candidates = s->candidates;
  ctx.host_budget = s->host_budget;
  ctx.compact_report = s->compact_report;
  ctx.host_partial = &s->host_partial;
  if (s->tuning_forced)
    ctx.tuning = s->forced_tuning;
  else if (const TuningTable::Entry* e = s->tuning.find(p, w, h))
    ctx.tuning = e->t;
}

int validate_params(const csgm_params* p, int w, int h) {
  if (!p) return fail(CSGM_E_INVALID, "params is NULL");
  if (p->disparities < 3 || p->disparities > 4096)
    return fail(CSGM_E_INVALID, "--disparities must be 3..4096 (got %d)", p->disparities);
  if ((int64_t)p->min_disparity + p->disparities > INT32_MAX ||
      (int64_t)p->min_disparity < -(int64_t)INT32_MAX)
    return fail(CSGM_E_INVALID, "disparity range must fit an integer");
  for (int size : {p->window_x, p->window_y})
    if (size < 3 || size > 11 || size % 2 == 0)
      return fail(CSGM_E_INVALID, "Census window must be odd, 3..11");
  if (p->cost_mode < 0 || p->cost_mode > 3) return fail(CSGM_E_INVALID, "Unknown matching cost");
  if (p->census_weight_milli < 0 || p->census_weight_milli > 1000 || p->ad_truncation < 1 ||
      p->ad_truncation > 255 || p->gradient_truncation < 1 || p->gradient_truncation > 1020)
    return fail(CSGM_E_INVALID, "Invalid matching-cost weight/truncation");
  if (p->p1 < 0 || p->p2 <= p->p1 || p->p2 > 100000000)
    return fail(CSGM_E_INVALID, "Require 0 <= P1 < P2 (effective penalties)");
  if (p->edge_scale < 0 || p->edge_scale > 255)
    return fail(CSGM_E_INVALID, "--sgm-edge-scale must be 0..255");
  if (p->directions != 4 && p->directions != 8 && p->directions != 16)
    return fail(CSGM_E_INVALID, "Directions must be 4, 8 or 16");
  if (p->aggregate_bytes != 2 && p->aggregate_bytes != 4)
    return fail(CSGM_E_INVALID, "aggregate_bytes must be 2 or 4");
  int64_t bound = (int64_t)p->directions * (512 + (int64_t)p->p2);
  if (p->aggregate_bytes == 2 && bound > 65535)
    return fail(CSGM_E_INVALID, "16-bit SGM aggregate cannot hold proved bound %lld",
                (long long)bound);
  if (bound > INT32_MAX) return fail(CSGM_E_INVALID, "aggregate bound exceeds int32");
  if (!(p->uniqueness >= 0 && p->uniqueness < 1))
    return fail(CSGM_E_INVALID, "Require 0 <= uniqueness < 1");
  if (!(p->lr_threshold > 0)) return fail(CSGM_E_INVALID, "lr_threshold must be positive");
  if (p->flags & ~CSGM_FLAG_GENERAL) return fail(CSGM_E_INVALID, "unknown params.flags bits");
  if (w < p->window_x + 2 || h < p->window_y + 2)
    return fail(CSGM_E_INVALID, "Invalid stereo image dimensions");
  if ((int64_t)w * h > (int64_t)INT32_MAX)
    return fail(CSGM_E_INVALID, "image exceeds 2^31 pixels");
  return CSGM_OK;
}

}  // namespace csgm

extern "C" {

int csgm_version(void) { return CSGM_ABI_VERSION; }

const char* csgm_last_error(void) { return g_error.c_str(); }

int csgm_effective_penalties(double p1, double p2, int32_t wx, int32_t wy, int32_t* p1_eff,
                             int32_t* p2_eff) {
  if (!p1_eff || !p2_eff) return fail(CSGM_E_INVALID, "NULL output");
  if (wx < 3 || wy < 3) return fail(CSGM_E_INVALID, "Census window must be odd, 3..11");
  int bits = wx * wy - 1;
  int64_t a = java_round_host(p1 * bits / 24.0), b = java_round_host(p2 * bits / 24.0);
  *p1_eff = (int32_t)a;
  *p2_eff = (int32_t)std::max<int64_t>(a + 1, b);
  return CSGM_OK;
}

int csgm_aggregate_bytes(int32_t directions, int32_t p2_eff, int32_t mode, int32_t* bytes,
                         int64_t* bound) {
  if (!bytes) return fail(CSGM_E_INVALID, "NULL output");
  int64_t b = (int64_t)directions * (512 + (int64_t)p2_eff);
  if (bound) *bound = b;
  bool fits = b <= 65535;
  if (mode == 16 && !fits)
    return fail(CSGM_E_INVALID, "16-bit SGM aggregate cannot hold proved bound %lld", (long long)b);
  if (mode != 0 && mode != 16 && mode != 32) return fail(CSGM_E_INVALID, "mode must be 0, 16 or 32");
  *bytes = mode != 32 && fits ? 2 : 4;
  return CSGM_OK;
}

int csgm_device_count(int32_t* count) {
  if (!count) return fail(CSGM_E_INVALID, "NULL output");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
    cudaGetLastError();
    *count = 0;
    return CSGM_OK;
  }
  if (e != cudaSuccess) return cuda_fail(e, "Device enumeration");
  *count = n;
  return CSGM_OK;
}

int csgm_device_info_get(int32_t device, csgm_device_info* info) {
  if (!info) return fail(CSGM_E_INVALID, "NULL output");
  int32_t count = 0;
  int rc = csgm_device_count(&count);
  if (rc) return rc;
  if (device < 0 || device >= count)
    return fail(CSGM_E_NODEVICE, "No CUDA GPU at index %d", device);
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return cuda_fail(e, "Device information");
  memset(info, 0, sizeof *info);
  snprintf(info->name, sizeof info->name, "%s", prop.name);
  info->memory_bytes = (int64_t)prop.totalGlobalMem;
  info->sm_count = prop.multiProcessorCount;
  info->cc_major = prop.major;
  info->cc_minor = prop.minor;
  return CSGM_OK;
}

int csgm_session_open(int32_t device, csgm_session** out) {
  if (!out) return fail(CSGM_E_INVALID, "NULL output");
  *out = nullptr;
  csgm_device_info info;
  int rc = csgm_device_info_get(device, &info);
  if (rc) return rc;
  if (info.cc_major < 10)
    return fail(CSGM_E_UNSUPPORTED, "device %d (%s, sm_%d%d) is not an sm_100a GPU", device,
                info.name, info.cc_major, info.cc_minor);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  csgm_session* s = new csgm_session();
  s->device = device;
  s->sm_count = info.sm_count;
  s->memory = (size_t)info.memory_bytes;
  s->workspace.budget = s->memory / 10 * 7;  // GpuSgm.budget with --gpu-memory-mb 0
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete s;
    return cuda_fail(e, "Queue creation");
  }
  *out = s;
  return CSGM_OK;
}

void csgm_session_close(csgm_session* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  release_batch_slots(s);
  s->graph_cache.clear();
  s->workspace.release_all();
  s->host_partial.release();
  cudaStreamDestroy(s->stream);
  delete s;  // destroys the profiler's events on the current device
}

int csgm_session_set_budget(csgm_session* s, int64_t bytes) {
  if (!s || bytes < 0) return fail(CSGM_E_INVALID, "invalid session or budget");
  std::lock_guard<std::mutex> guard(s->lock);
  s->workspace.budget = bytes == 0 ? s->memory / 10 * 7
                                   : std::min<size_t>(s->memory / 100 * 95, (size_t)bytes);
  return CSGM_OK;
}

int csgm_session_set_wait_limit(csgm_session* s, int64_t cycles) {
  if (!s || cycles < 0) return fail(CSGM_E_INVALID, "invalid session or wait limit");
  std::lock_guard<std::mutex> guard(s->lock);
  s->wait_limit = cycles;
  return CSGM_OK;
}

int csgm_session_set_streaming(csgm_session* s, int32_t mode, int32_t strip_rows) {
  if (!s || mode < CSGM_SGM_AUTO || mode > CSGM_SGM_COMPACT || strip_rows < 0)
    return fail(CSGM_E_INVALID, "invalid session, streaming mode or strip height");
  std::lock_guard<std::mutex> guard(s->lock);
  s->sgm_mode = mode;
  s->strip_rows = strip_rows ? strip_rows : 64;  // Options.gpuStripRows default
  return CSGM_OK;
}

int csgm_session_set_candidates(csgm_session* s, int32_t per_path) {
  // Options.java:781-782.
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  if (per_path < 1 || per_path > 4) return fail(CSGM_E_INVALID, "--esgm-candidates must be 1..4");
  std::lock_guard<std::mutex> guard(s->lock);
  s->candidates = per_path;
  return CSGM_OK;
}

int csgm_session_set_host_budget(csgm_session* s, int64_t bytes) {
  if (!s || bytes < 0) return fail(CSGM_E_INVALID, "invalid session or host budget");
  std::lock_guard<std::mutex> guard(s->lock);
  s->host_budget = (size_t)bytes;
  return CSGM_OK;
}

int csgm_session_compact_report(csgm_session* s, int32_t reverse, int64_t* certified,
                                int64_t* verified) {
  if (!s || (reverse != 0 && reverse != 1)) return fail(CSGM_E_INVALID, "invalid session or view");
  std::lock_guard<std::mutex> guard(s->lock);
  if (certified) *certified = s->compact_report[2 * reverse];
  if (verified) *verified = s->compact_report[2 * reverse + 1];
  return CSGM_OK;
}

int csgm_session_set_graphs(csgm_session* s, int32_t enabled) {
  if (!s || (enabled != 0 && enabled != 1)) return fail(CSGM_E_INVALID, "invalid session or flag");
  std::lock_guard<std::mutex> guard(s->lock);
  cudaSetDevice(s->device);
  s->graphs = enabled != 0;
  if (!s->graphs) s->graph_cache.clear();
  return CSGM_OK;
}

int csgm_graph_stats(csgm_session* s, int64_t* captured, int64_t* replayed) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  std::lock_guard<std::mutex> guard(s->lock);
  if (captured) *captured = s->graph_cache.captured;
  if (replayed) *replayed = s->graph_cache.replayed;
  return CSGM_OK;
}

int csgm_session_set_profiling(csgm_session* s, int32_t level) {
  if (!s || level < 0 || level > 2) return fail(CSGM_E_INVALID, "invalid session or level");
  std::lock_guard<std::mutex> guard(s->lock);
  s->profiler.level = level;
  return CSGM_OK;
}

int csgm_session_synchronize(csgm_session* s) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  cudaSetDevice(s->device);
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "Stream synchronisation");
  std::lock_guard<std::mutex> guard(s->lock);
  s->profiler.collect();
  return CSGM_OK;
}

int csgm_profile_get(csgm_session* s, csgm_profile* out, int32_t reset) {
  if (!s || !out) return fail(CSGM_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> guard(s->lock);
  *out = s->profile;
  out->launches = s->profiler.launches;
  if (reset) {
    s->profile = csgm_profile{};
    s->profiler.launches = 0;
  }
  return CSGM_OK;
}

int csgm_kernel_times(csgm_session* s, csgm_kernel_time* out, int32_t capacity, int32_t* count,
                      int32_t reset) {
  if (!s || !count || (capacity > 0 && !out)) return fail(CSGM_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> guard(s->lock);
  *count = (int32_t)s->profiler.kernels.size();
  for (int i = 0; i < capacity && i < (int)s->profiler.kernels.size(); i++) {
    memset(&out[i], 0, sizeof out[i]);
    snprintf(out[i].name, sizeof out[i].name, "%s", s->profiler.kernels[i].name.c_str());
    out[i].launches = s->profiler.kernels[i].launches;
    out[i].total_ns = s->profiler.kernels[i].total_ns;
  }
  if (reset) s->profiler.kernels.clear();
  return CSGM_OK;
}

// A context with the session's budget, streaming and tuning settings, for planning only.
static Context planning_context(csgm_session* s, const csgm_params& p, int w, int h) {
  Context ctx{s->stream, s->sm_count, &s->workspace, &s->profiler, &s->profile};
  session_settings(ctx, s, p, w, h);
  return ctx;
}

int csgm_plan_detail(csgm_session* s, const csgm_params* p, int32_t w, int32_t h,
                     int32_t* strip_rows, int64_t* device_bytes, int64_t* host_bytes) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  ViewPlan plan;
  rc = plan_pair(planning_context(s, *p, w, h), *p, w, h, true, &plan);
  if (rc) return rc;
  if (strip_rows) *strip_rows = plan.rows;
  if (device_bytes) *device_bytes = (int64_t)plan.device_bytes;
  if (host_bytes) *host_bytes = (int64_t)plan.host_bytes;
  return CSGM_OK;
}

int csgm_plan(csgm_session* s, const csgm_params* p, int32_t w, int32_t h, int64_t* bytes) {
  if (!s || !bytes) return fail(CSGM_E_INVALID, "NULL argument");
  return csgm_plan_detail(s, p, w, h, nullptr, bytes, nullptr);
}

int csgm_disparity_limit(csgm_session* s, const csgm_params* p, int32_t w, int32_t h,
                         int32_t* limit) {
  // GpuStereo.limit (GpuStereo.java:86-94): binary search over the plan.
  if (!s || !p || !limit) return fail(CSGM_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> guard(s->lock);
  int low = 2, high = 4096;
  while (low < high) {
    int mid = (low + high + 1) / 2;
    csgm_params q = *p;
    q.disparities = mid;
    ViewPlan plan;
    bool fits = validate_params(&q, w, h) == CSGM_OK &&
                plan_pair(planning_context(s, q, w, h), q, w, h, true, &plan) == 0;
    if (fits)
      low = mid;
    else
      high = mid - 1;
  }
  *limit = low == 2 ? 0 : low;
  g_error.clear();
  return CSGM_OK;
}

int csgm_match(csgm_session* s, const csgm_params* p, const uint64_t* desc_a,
               const uint64_t* desc_b, const uint8_t* gray_a, const uint8_t* gray_b,
               const uint8_t* tex_a, const uint8_t* tex_b, int32_t w, int32_t h, int32_t reverse,
               float* out_disp, int32_t* out_summary, uint8_t* reasons, uint8_t* boundary,
               csgm_stats* stats) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  if (!desc_a || !desc_b || !gray_a || !gray_b || !tex_a || !tex_b || !out_disp)
    return fail(CSGM_E_INVALID, "NULL input or output buffer");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  Context ctx{s->stream, s->sm_count, &s->workspace, &s->profiler, &s->profile};
  session_settings(ctx, s, *p, w, h);
  ctx.twin = &s->twin;
  return run_match_host(ctx, *p, desc_a, desc_b, gray_a, gray_b, tex_a, tex_b, w, h, reverse,
                        out_disp, out_summary, reasons, boundary, stats);
}

int csgm_pair(csgm_session* s, const csgm_params* p, const uint8_t* left, const uint8_t* right,
              const uint8_t* valid_l, const uint8_t* valid_r, int32_t w, int32_t h,
              float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
              uint8_t* boundary, csgm_stats* stats) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  if (!left || !right || !lr_checked) return fail(CSGM_E_INVALID, "NULL image or output buffer");
  if ((valid_l == nullptr) != (valid_r == nullptr))
    return fail(CSGM_E_INVALID, "Invalid stereo mask dimensions");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  Context ctx{s->stream, s->sm_count, &s->workspace, &s->profiler, &s->profile};
  session_settings(ctx, s, *p, w, h);
  return run_pair_host(ctx, *p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l, disp_r,
                       reasons, boundary, stats);
}

int csgm_pair_color(csgm_session* s, const csgm_params* p, const uint8_t* left,
                    const uint8_t* right, const uint8_t* left_bgr, const uint8_t* right_bgr,
                    const uint8_t* valid_l, const uint8_t* valid_r, int32_t w, int32_t h,
                    float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                    uint8_t* boundary, csgm_stats* stats) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  if (!left || !right || !lr_checked) return fail(CSGM_E_INVALID, "NULL image or output buffer");
  if (!left_bgr || !right_bgr)
    return fail(CSGM_E_INVALID, "Color-distance census requires interleaved BGR inputs");
  if ((valid_l == nullptr) != (valid_r == nullptr))
    return fail(CSGM_E_INVALID, "Invalid stereo mask dimensions");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  Context ctx{s->stream, s->sm_count, &s->workspace, &s->profiler, &s->profile};
  session_settings(ctx, s, *p, w, h);
  return run_pair_host(ctx, *p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l, disp_r,
                       reasons, boundary, stats, left_bgr, right_bgr);
}

int csgm_pair_device(csgm_session* s, const csgm_params* p, const uint8_t* left,
                     const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r,
                     int32_t w, int32_t h, float* lr_checked, float* disp_l, float* disp_r,
                     uint8_t* reasons, uint8_t* boundary, csgm_stats* stats, int32_t sync) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  if (!left || !right || !lr_checked) return fail(CSGM_E_INVALID, "NULL image or output buffer");
  if ((valid_l == nullptr) != (valid_r == nullptr))
    return fail(CSGM_E_INVALID, "Invalid stereo mask dimensions");
  if (!sync && stats) return fail(CSGM_E_INVALID, "stats need sync != 0");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  Context ctx{s->stream, s->sm_count, &s->workspace, &s->profiler, &s->profile};
  session_settings(ctx, s, *p, w, h);
  if (s->graphs && s->profiler.level < 2)
    return run_pair_device_graph(ctx, s->graph_cache, *p, left, right, valid_l, valid_r, w, h,
                                 lr_checked, disp_l, disp_r, reasons, boundary, stats, sync != 0);
  return run_pair_device(ctx, *p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l, disp_r,
                         reasons, boundary, stats, sync != 0);
}

}  // extern "C"
