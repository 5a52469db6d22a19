// batch.cu - batched and served pairs.  A session's slots each hold one pair in flight with its own
// CUDA stream and a resident device workspace (stream-ordered allocations from a pool that keeps
// freed memory).  All slots' sweeps share one high-priority stream, so sweeps run back to back
// (two chains of row blocks at once slow each other more than they gain), while the other pairs'
// uploads, census, cost volumes, line passes, selections and downloads overlap them in the shared
// memory and issue slots a sweep leaves free.  Admission checks each pair's device
// memory (W*H*D bytes of cost volumes and aggregates, plus images and outputs) against the batch
// budget; a pair that does not fit right now is refused with CSGM_E_BUSY and can be submitted
// again once a slot or memory frees up (continuous batching).
//
// There is no batch interface in the reference: GpuSgm serves one pair per call and one session
// per Java thread (GpuSgm.java:22,163-303).  The per-pair semantics, and so every result, are
// those of csgm_pair.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "collinea_sgm.h"
#include "pipeline.h"

using namespace csgm;

namespace {

// Releases every slot: waits for its work, frees its workspace, stream, event and pinned stats.
void release_slots(csgm_session* s) {
  for (auto& slot : s->slots) {
    if (slot.stream) cudaStreamSynchronize(slot.stream);
    slot.ws.release_all();
    if (slot.stream) {
      cudaStreamSynchronize(slot.stream);  // stream-ordered frees complete
      cudaStreamDestroy(slot.stream);
    }
    if (slot.sweep_stream) cudaStreamDestroy(slot.sweep_stream);
    if (slot.sweep_ready) cudaEventDestroy(slot.sweep_ready);
    if (slot.sweep_done) cudaEventDestroy(slot.sweep_done);
    if (slot.done) cudaEventDestroy(slot.done);
    if (slot.host_stats) cudaFreeHost(slot.host_stats);
  }
  s->slots.clear();
}

size_t reserved_total(const csgm_session* s) {
  size_t total = 0;
  for (const auto& slot : s->slots) total += slot.id ? slot.reserved : 0;
  return total;
}

size_t allocated_total(const csgm_session* s) {
  size_t total = 0;
  for (const auto& slot : s->slots) total += slot.ws.allocated;
  return total;
}

}  // namespace

extern "C" {

int csgm_batch_configure(csgm_session* s, int32_t slots, int64_t budget_bytes) {
  if (!s || slots < 1 || slots > 64 || budget_bytes < 0)
    return fail(CSGM_E_INVALID, "invalid session, slot count (1..64) or budget");
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  for (const auto& slot : s->slots)
    if (slot.id) return fail(CSGM_E_BUSY, "batch requests are still in flight");
  release_slots(s);
  s->batch_budget = budget_bytes == 0 ? s->memory / 10 * 7
                                      : std::min<size_t>(s->memory / 100 * 95, (size_t)budget_bytes);
  // Slot workspaces grow and shrink stream-ordered: memory they give back stays in the device's
  // pool for the next pair instead of returning to the driver.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  s->slots.resize((size_t)slots);
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  for (auto& slot : s->slots) {
    e = cudaStreamCreateWithPriority(&slot.stream, cudaStreamNonBlocking, least);
    // One high-priority stream carries every slot's sweep: sweeps run back to back at the speed
    // of a lone pair (each sweep fills the GPU with its chain of row blocks; two at once slow each
    // other down more than they gain), while the other slots' uploads, cost volumes, selections
    // and downloads use the SMs a sweep leaves idle.
    if (e == cudaSuccess && &slot != &s->slots[0]) {
      slot.sweep_stream = nullptr;  // borrows slot 0's stream below
    } else if (e == cudaSuccess) {
      e = cudaStreamCreateWithPriority(&slot.sweep_stream, cudaStreamNonBlocking, greatest);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.sweep_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.sweep_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&slot.host_stats, sizeof(DeviceStats));
    if (e != cudaSuccess) {
      release_slots(s);
      return cuda_fail(e, "batch slot creation");
    }
    slot.ws.async_stream = slot.stream;
    slot.ws.budget = s->batch_budget;
  }
  for (auto& slot : s->slots)
    if (!slot.sweep_stream) slot.shared_sweep = s->slots[0].sweep_stream;
  return CSGM_OK;
}

int csgm_batch_submit(csgm_session* s, const csgm_params* p, const uint8_t* left,
                      const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r,
                      int32_t w, int32_t h, float* lr_checked, float* disp_l, float* disp_r,
                      uint8_t* reasons, uint8_t* boundary, int64_t* request) {
  if (!s || !request) return fail(CSGM_E_INVALID, "NULL session or request");
  if (!left || !right || !lr_checked) return fail(CSGM_E_INVALID, "NULL image or output buffer");
  if ((valid_l == nullptr) != (valid_r == nullptr))
    return fail(CSGM_E_INVALID, "Invalid stereo mask dimensions");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  if (s->slots.empty()) return fail(CSGM_E_INVALID, "csgm_batch_configure was not called");
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  const size_t need = pair_workspace_bytes(*p, w, h, true);
  if (need > s->batch_budget)
    return fail(CSGM_E_NOMEM, "pair needs %.1f MiB, batch budget %.1f MiB", need / 1048576.0,
                s->batch_budget / 1048576.0);
  // Admission: the bytes of the pairs in flight plus this one stay inside the budget.
  if (reserved_total(s) + need > s->batch_budget)
    return fail(CSGM_E_BUSY, "batch memory budget in use");
  // The free slot with the smallest resident workspace that already fits the pair, else the free
  // slot with the largest one (the least to grow).
  BatchSlot* fits = nullptr;
  BatchSlot* largest = nullptr;
  for (auto& c : s->slots) {
    if (c.id) continue;
    if (c.ws.allocated >= need && (!fits || c.ws.allocated < fits->ws.allocated)) fits = &c;
    if (!largest || c.ws.allocated > largest->ws.allocated) largest = &c;
  }
  BatchSlot* slot = fits ? fits : largest;
  if (!slot) return fail(CSGM_E_BUSY, "every batch slot is in flight");
  // Resident workspaces of idle slots give their memory back when the physical total would
  // otherwise exceed the budget.
  if (slot->ws.allocated < need && allocated_total(s) - slot->ws.allocated + need > s->batch_budget)
    for (auto& c : s->slots)
      if (!c.id && &c != slot && c.ws.allocated) c.ws.release_all();
  if (allocated_total(s) - slot->ws.allocated + need > s->batch_budget) slot->ws.release_all();
  const size_t held = allocated_total(s) - slot->ws.allocated;  // resident in other slots
  if (held + need > s->batch_budget)
    return fail(CSGM_E_BUSY, "batch memory held by pairs in flight");
  slot->ws.budget = s->batch_budget - held;
  Context ctx{slot->stream, s->sm_count, &slot->ws, &slot->prof, &slot->profile};
  ctx.wait_limit = s->wait_limit;
  // Batch slots keep their pairs resident (admission counts whole volumes).
  ctx.sgm_mode = CSGM_SGM_RESIDENT;
  ctx.sweep_stream = slot->sweep_stream ? slot->sweep_stream : slot->shared_sweep;
  ctx.sweep_ready = slot->sweep_ready;
  ctx.sweep_done = slot->sweep_done;
  // Batched sweeps take no SM alone: the other slots' census, cost, line and selection kernels fill
  // the shared memory and issue slots a sweep CTA leaves free (48 mixed pairs, 3 slots: 1.41x the
  // per-pair path's pairs/s, against 1.25x with SM-exclusive sweeps).
  ctx.exclusive_sweep = false;
  // The line kernel on the slot's stream overlaps other pairs' sweeps (48 mixed pairs, 4 slots:
  // 130.9 pairs/s, against 123.0 with the lines inside the serialised sweeps).
  ctx.lines_in_sweep = false;
  rc = enqueue_pair_host(ctx, *p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l, disp_r,
                         reasons, boundary, slot->host_stats);
  if (rc == CSGM_OK) {
    e = cudaEventRecord(slot->done, slot->stream);
    if (e != cudaSuccess) rc = cuda_fail(e, "batch completion event");
  }
  if (rc != CSGM_OK) {
    cudaStreamSynchronize(slot->stream);  // nothing half-queued is left behind
    cudaGetLastError();
    return rc;
  }
  slot->id = s->next_request++;
  slot->reserved = need;
  *request = slot->id;
  return CSGM_OK;
}

int csgm_batch_poll(csgm_session* s, int64_t request, int32_t wait, csgm_stats* stats) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  cudaEvent_t done = nullptr;
  {
    std::lock_guard<std::mutex> guard(s->lock);
    for (auto& c : s->slots)
      if (c.id == request && request != 0) done = c.done;
    if (!done) return fail(CSGM_E_INVALID, "unknown batch request %lld", (long long)request);
  }
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  // Waiting happens outside the session lock, so other threads keep submitting meanwhile.
  e = wait ? cudaEventSynchronize(done) : cudaEventQuery(done);
  if (e == cudaErrorNotReady) {
    cudaGetLastError();
    return fail(CSGM_E_BUSY, "batch request %lld not finished", (long long)request);
  }
  std::lock_guard<std::mutex> guard(s->lock);
  BatchSlot* slot = nullptr;
  for (auto& c : s->slots)
    if (c.id == request) slot = &c;
  if (!slot) return fail(CSGM_E_INVALID, "batch request %lld already collected", (long long)request);
  slot->id = 0;
  slot->reserved = 0;
  if (e != cudaSuccess) return cuda_fail(e, "GPU SGM execution");
  slot->prof.collect();
  const DeviceStats host = *slot->host_stats;
  if (host.pad)
    return fail(CSGM_E_TIMEOUT, "a bounded device wait expired (code %llu)", host.pad);
  if (stats) copy_stats(host, stats, false);
  return CSGM_OK;
}

int csgm_batch_status(csgm_session* s, int32_t* in_flight, int64_t* reserved_bytes,
                      int64_t* resident_bytes) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  std::lock_guard<std::mutex> guard(s->lock);
  int n = 0;
  for (const auto& c : s->slots) n += c.id != 0;
  if (in_flight) *in_flight = n;
  if (reserved_bytes) *reserved_bytes = (int64_t)reserved_total(s);
  if (resident_bytes) *resident_bytes = (int64_t)allocated_total(s);
  return CSGM_OK;
}

int csgm_host_alloc(int64_t bytes, void** ptr) {
  if (!ptr || bytes <= 0) return fail(CSGM_E_INVALID, "invalid size or NULL output");
  *ptr = nullptr;
  cudaError_t e = cudaMallocHost(ptr, (size_t)bytes);
  if (e != cudaSuccess) return cuda_fail(e, "pinned host allocation");
  return CSGM_OK;
}

void csgm_host_free(void* ptr) {
  if (ptr) cudaFreeHost(ptr);
}

}  // extern "C"

namespace csgm {
// Session teardown of the batch slots (called by csgm_session_close).
void release_batch_slots(csgm_session* s) { release_slots(s); }
}  // namespace csgm
