// pipeline.h - session workspace, profiler and the stage sequences behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <mutex>
#include <vector>

#include "collinea_sgm.h"
#include "sgm_device.cuh"

namespace csgm {

struct Context;
int fail(int status, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
int validate_params(const csgm_params* p, int w, int h);

enum Slot {
  kImgL, kImgR, kValidL, kValidR, kDescL, kDescR, kTexL, kTexR,
  kCostL, kCostR, kSum, kSumUp, kSumLines, kPen, kDispL, kDispR, kChecked, kReasons, kBoundary, kSummary, kStats,
  kCarry, kFlags, kPixelInfo, kStripCarry, kBgrL, kBgrR,
  // csgm_match on the fused kernels: two sets of view inputs (descriptors l/r, grays l/r, masks
  // l/r in the pair's order), per-view outputs, the comparison flag.
  kMatchIn0, kMatchIn1 = kMatchIn0 + 6, kMatchDisp = kMatchIn1 + 6, kMatchReasons = kMatchDisp + 2,
  kMatchBoundary = kMatchReasons + 2, kMatchSummary = kMatchBoundary + 2,
  kMatchStats = kMatchSummary + 2, kMatchEqual,
  // Compact SGM: proposals, compact aggregates, lower bounds, the unresolved pixels and their
  // exact aggregates and cost rows.
  kEsgmCand, kEsgmCompact, kEsgmOutside, kEsgmSlots, kEsgmPixels, kEsgmCount, kEsgmSum, kEsgmCost,
  kSlotCount
};

// Pinned host memory that a session grows on demand (the streamed down pass parks its partial
// aggregate there, GpuStereo.java:339-437 keeps the reference's in host RAM).
struct HostBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  void* get(size_t want, int* status);
  void release();
};

// Captured device pipelines of csgm_pair_device, replayed when a call repeats one (same
// parameters, size, buffers and launch shape) and the workspace has not been reallocated since.
struct GraphCache {
  struct Entry {
    std::vector<uint8_t> key;
    cudaGraphExec_t exec = nullptr;  // null: the work could not be captured; run it plainly
    uint64_t generation = 0;
    uint64_t used = 0;
    int64_t launches = 0;  // kernels in the graph
  };
  static constexpr size_t kCapacity = 8;
  std::vector<Entry> entries;
  uint64_t clock = 0;
  int64_t captured = 0, replayed = 0;
  void clear();
  ~GraphCache() { clear(); }
};

// Launch shape of the fused sweep (the autotuner's knobs).  0 / -1 fields: the default.
struct SweepTuning {
  int rows = 0;         // rows per sweep CTA (row warps)
  int line_warps = -1;  // line warps per sweep CTA walking the anti-diagonal lines
  int line_slack = 0;   // percent of a block's remaining pixels a line may take
};

// Autotuned launch shapes per shape bucket (padded D, paths, half-octave width and height),
// filled by csgm_autotune and loaded from its cache file.
struct TuningTable {
  struct Entry {
    int dp, paths, wb, hb;
    SweepTuning t;
    double ms;
  };
  std::vector<Entry> entries;
  static int bucket(int v);
  const Entry* find(const csgm_params& p, int w, int h) const;
  void put(const csgm_params& p, int w, int h, const SweepTuning& t, double ms);
};

// How a pair's views run: resident (the whole volume in device memory: the fused kernels where
// they apply, else the general ones) or streamed through strips of `rows` rows (general kernels).
struct ViewPlan {
  bool streamed = false;
  bool compact = false;       // compact SGM (CSGM_SGM_COMPACT)
  int pool = 0;               // its proposals per path
  int views = 1;              // its views at once (2: a pair's views share the path launches)
  int rows = 0;               // strip height (the image height when resident)
  size_t device_bytes = 0;    // device memory of the plan
  size_t host_bytes = 0;      // pinned host memory of the plan
};

// csgm_match runs both views of a pair whenever it runs the fused kernels: the reference always
// follows the left view's match(a, b, ..., reverse=false) with match(b, a, ..., reverse=true)
// (CensusSgm.java:135-162), whose result is the pair's other view.  That view's results stay on
// the device, with the inputs they came from, until a call whose inputs are identical asks for it.
struct MatchTwin {
  bool valid = false;
  int set = 0;   // input set (kMatchIn0 / kMatchIn1) the pair was computed from
  int view = 0;  // the view held: 0 = reverse false, 1 = reverse true
  csgm_params params{};
  int w = 0, h = 0;
  bool summary = false;  // winners records were computed (reason codes and flags always are)
  DeviceStats stats{};   // the held view's selection counters
};

// Device buffers owned by a session, grown on demand inside the memory budget.
struct Workspace {
  struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
  };
  Buffer buffers[kSlotCount];
  size_t allocated = 0;
  size_t budget = 0;
  // Advances whenever a buffer is allocated again or released: a captured graph that refers to
  // the buffers is valid only for the generation it was captured in.
  uint64_t generation = 0;
  // When set, buffers are allocated and freed stream-ordered on this stream (no device-wide
  // synchronisation while other streams' kernels run).
  cudaStream_t async_stream = nullptr;
  void* get(int slot, size_t bytes, int* status);
  void release_all();
  // Frees one buffer (nothing when it holds none).
  void release(int slot);
};

struct Profiler {
  struct Pending {
    std::string name;
    cudaEvent_t start, stop;
  };
  struct KernelTotal {
    std::string name;
    int64_t launches;
    int64_t total_ns;
  };
  int level = 0;
  cudaStream_t stream = nullptr;
  std::vector<cudaEvent_t> events;
  size_t used = 0;
  cudaEvent_t current_start = nullptr;
  std::vector<Pending> pending;
  std::vector<KernelTotal> kernels;
  int64_t launches = 0;
  void begin_call(cudaStream_t s);
  cudaEvent_t event();
  void kernel_begin();
  void kernel_end(const char* name);
  void collect();
  ~Profiler();
};

struct Context {
  cudaStream_t stream;
  int sm_count;
  Workspace* ws;
  Profiler* prof;
  csgm_profile* profile;
  // One sweep CTA per SM (a lone pair runs fastest so); batched pairs share SMs instead.
  bool exclusive_sweep = true;
  // 8 paths: the sweep's CTAs also walk the anti-diagonal lines (line warps on the issue slots
  // the row warps leave idle).  Batched pairs run them as a kernel of their own on the pair's
  // stream instead, beside the other pairs' sweeps.
  bool lines_in_sweep = true;
  // Optional separate stream for the sweep (ordered after and before ctx.stream by the events).
  cudaStream_t sweep_stream = nullptr;
  cudaEvent_t sweep_ready = nullptr, sweep_done = nullptr;
  // SM clock cycles a bounded device-side wait may go without progress (0 = the default).
  long long wait_limit = 0;
  // The session's held view of csgm_match (null: csgm_match is not the caller).
  MatchTwin* twin = nullptr;
  // Options.gpuSgm (CSGM_SGM_*) and Options.gpuStripRows: resident or streamed views.
  int sgm_mode = CSGM_SGM_AUTO;
  int strip_rows = 64;
  int candidates = 2;  // Options.esgmCandidates
  // Host memory a streamed plan may park its aggregate in (0: no limit; csgm_session_set_host_budget).
  size_t host_budget = 0;
  // Compact SGM's last outcome per view (reverse 0/1): certified pixels, pixels verified exactly.
  int64_t* compact_report = nullptr;
  HostBuffer* host_partial = nullptr;  // null: streaming unavailable (batch slots)
  // Launch shape of the fused sweep for this call (from the session's tuning table).
  SweepTuning tuning;
};

// One batch slot: a pair in flight with its own stream and resident workspace.
struct BatchSlot {
  cudaStream_t stream = nullptr;
  cudaStream_t sweep_stream = nullptr;  // high priority, owned by this slot
  cudaStream_t shared_sweep = nullptr;  // or another slot's (not owned)
  cudaEvent_t sweep_ready = nullptr, sweep_done = nullptr;
  cudaEvent_t done = nullptr;
  Workspace ws;
  Profiler prof;
  csgm_profile profile{};
  DeviceStats* host_stats = nullptr;  // pinned
  int64_t id = 0;                     // request in flight, 0 = free
  size_t reserved = 0;                // bytes admitted for it
};

// Bytes of device workspace a pair needs (host_inputs: include the upload/download staging;
// color: the two interleaved BGR images of --census-mode color-distance).
size_t pair_workspace_bytes(const csgm_params& p, int w, int h, bool host_inputs,
                            bool color = false, const SweepTuning& tuning = SweepTuning{});

// The plan of a pair (GpuStereo.plan, GpuStereo.java:33-84) under the context's budget, mode and
// strip height; CSGM_E_NOMEM when no plan fits.
int plan_pair(const Context& ctx, const csgm_params& p, int w, int h, bool host_inputs,
              ViewPlan* plan, bool color = false);

int run_pair_device(Context& ctx, const csgm_params& p, const uint8_t* left, const uint8_t* right,
                    const uint8_t* valid_l, const uint8_t* valid_r, int w, int h,
                    float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                    uint8_t* boundary, csgm_stats* stats, bool sync);

// bgr_l / bgr_r (optional, both or neither): the interleaved BGR images whose colour-distance
// census gives the descriptors and texture (--census-mode color-distance).
// run_pair_device through the graph cache (device buffers; replays a captured pipeline).
int run_pair_device_graph(Context& ctx, GraphCache& cache, const csgm_params& p,
                          const uint8_t* left, const uint8_t* right, const uint8_t* valid_l,
                          const uint8_t* valid_r, int w, int h, float* lr_checked, float* disp_l,
                          float* disp_r, uint8_t* reasons, uint8_t* boundary, csgm_stats* stats,
                          bool sync);

int run_pair_host(Context& ctx, const csgm_params& p, const uint8_t* left, const uint8_t* right,
                  const uint8_t* valid_l, const uint8_t* valid_r, int w, int h,
                  float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                  uint8_t* boundary, csgm_stats* stats, const uint8_t* bgr_l = nullptr,
                  const uint8_t* bgr_r = nullptr);

int run_match_host(Context& ctx, const csgm_params& p, const uint64_t* desc_a,
                   const uint64_t* desc_b, const uint8_t* gray_a, const uint8_t* gray_b,
                   const uint8_t* tex_a, const uint8_t* tex_b, int w, int h, int reverse,
                   float* out_disp, int32_t* out_summary, uint8_t* reasons, uint8_t* boundary,
                   csgm_stats* stats);

// Adds (add) or copies device selection counters into the ABI's stats record.
void copy_stats(const DeviceStats& d, csgm_stats* out, bool add);

// Queues a pair with host buffers on ctx.stream without waiting: uploads, the device pipeline,
// downloads, and the selection counters into *host_stats (pinned).  The caller synchronises.
int enqueue_pair_host(Context& ctx, const csgm_params& p, const uint8_t* left,
                      const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r, int w,
                      int h, float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                      uint8_t* boundary, DeviceStats* host_stats);

}  // namespace csgm

namespace csgm {
struct BatchSlot;
void release_batch_slots(csgm_session* s);
}  // namespace csgm

struct csgm_session {
  int device = 0;
  int sm_count = 0;
  size_t memory = 0;
  cudaStream_t stream = nullptr;
  std::mutex lock;
  csgm::Workspace workspace;
  csgm::Profiler profiler;
  csgm_profile profile{};
  int64_t wait_limit = 0;  // csgm_session_set_wait_limit (0 = default)
  csgm::MatchTwin twin;    // csgm_match's held view
  int sgm_mode = CSGM_SGM_AUTO;  // csgm_session_set_streaming
  int strip_rows = 64;
  int candidates = 2;             // csgm_session_set_candidates
  size_t host_budget = 0;         // csgm_session_set_host_budget
  int64_t compact_report[4] = {0, 0, 0, 0};
  csgm::HostBuffer host_partial;
  csgm::TuningTable tuning;  // csgm_autotune / csgm_session_load_tuning
  bool graphs = false;       // csgm_session_set_graphs
  csgm::GraphCache graph_cache;
  bool tuning_forced = false;  // csgm_session_set_tuning
  csgm::SweepTuning forced_tuning;
  // Batched / served pairs (batch.cu).
  std::vector<csgm::BatchSlot> slots;
  size_t batch_budget = 0;
  int64_t next_request = 1;
};

namespace csgm {
// Copies the session's wait limit, streaming mode and (for these parameters and size) sweep
// tuning into a call's context.
void session_settings(Context& ctx, csgm_session* s, const csgm_params& p, int w, int h);
}  // namespace csgm
