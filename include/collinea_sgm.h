/*
 * collinea_sgm.h - C ABI of the B200 semi-global stereo matcher.
 *
 * This is the drop-in boundary for Collinea's GPU stereo backend.  In the reference the Java host
 * calls OpenCL through Panama FFM downcalls (src/main/java/sgm/GpuSgm.java:30-54); a maintainer
 * replaces those downcalls with downcalls into this library (libcollinea_sgm.so).  Every entry
 * point below names the reference interface it replaces.
 *
 * Conventions
 *   - Plain C types only: pointers, sizes, int32/int64/double.  No CUDA or torch types.
 *   - Every function returns CSGM_OK (0) or a negative CSGM_E_* code.  The message of the last
 *     failure on the calling thread is returned by csgm_last_error().
 *   - All host buffers are owned by the caller.  They may be pageable or pinned.  The library owns
 *     every device allocation it makes, inside the session's memory budget.
 *   - There is no CPU fallback: when the GPU path cannot run, the call fails.
 *   - A session is bound to one CUDA device and one stream.  Calls on one session are serialised
 *     by the session's own lock; different sessions may be used from different threads.
 *
 * Image and volume layouts
 *   - Images are row-major uint8, index p = y * w + x.
 *   - Census descriptors are word-major: desc[word * w * h + p], the layout the reference uploads
 *     (src/main/java/sgm/GpuStereo.java:243-250).  Bit order follows CensusSgm.census
 *     (src/main/java/sgm/CensusSgm.java:540-555): row-major over the window, centre skipped.
 *   - Masks are uint8, non-zero = true.
 */
#ifndef COLLINEA_SGM_H
#define COLLINEA_SGM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CSGM_ABI_VERSION 1

/* Status codes. */
#define CSGM_OK 0
#define CSGM_E_INVALID (-1)     /* bad argument: IllegalArgumentException in the reference */
#define CSGM_E_CUDA (-2)        /* CUDA runtime failure: IllegalStateException("... failed") */
#define CSGM_E_NOMEM (-3)       /* device allocation failed or the memory plan exceeds the budget */
#define CSGM_E_NODEVICE (-4)    /* no CUDA device at the requested index */
#define CSGM_E_TIMEOUT (-5)     /* a bounded device-side wait expired; the context stays usable */
#define CSGM_E_BUSY (-6)        /* batch queue full or request not finished */
#define CSGM_E_UNSUPPORTED (-7) /* parameter combination outside what the kernels implement */

/* params.flags: run the general kernels (one warp per path line, any D) even where the fused
 * sweep would apply.  Same results; used to compare the two paths and as the plain per-pair path. */
#define CSGM_FLAG_GENERAL 1

/* Matching-cost codes: StereoCost.code (src/main/java/sgm/StereoCost.java:7-15). */
#define CSGM_COST_CENSUS 0
#define CSGM_COST_AD_CENSUS 1
#define CSGM_COST_CENSUS_GRADIENT 2
#define CSGM_COST_ZNCC 3

/*
 * Matcher parameters.  Mirrors the scalar arguments of the reference `costs`/`paths` kernels
 * (src/main/java/sgm/GpuStereo.java:384-403,600-614) plus the selection and LR settings.
 * Penalties are the EFFECTIVE integer penalties, i.e. StereoCost.penalty(o.p1, o) and
 * StereoCost.p2(o) (src/main/java/sgm/StereoCost.java:17-23); csgm_effective_penalties()
 * computes them from Options-style values.
 */
typedef struct csgm_params {
  int32_t disparities;         /* D = Options.disparities, 3..4096 */
  int32_t min_disparity;       /* Options.minDisparity */
  int32_t window_x;            /* census/texture/ZNCC window width  (Options.census) */
  int32_t window_y;            /* census/texture/ZNCC window height (== window_x in the reference) */
  int32_t cost_mode;           /* CSGM_COST_* */
  int32_t census_weight_milli; /* (int) Math.round(Options.censusWeight * 1000) */
  int32_t ad_truncation;       /* Options.adTruncation */
  int32_t gradient_truncation; /* Options.gradientTruncation */
  int32_t p1;                  /* effective P1 */
  int32_t p2;                  /* effective P2 */
  int32_t edge_scale;          /* Options.sgmEdgeScale, 0..255 (0 = constant P2) */
  int32_t directions;          /* 4 or 8 (reference); 16 adds the (+-1,+-2),(+-2,+-1) paths */
  int32_t aggregate_bytes;     /* 2 (uint16) or 4 (uint32): StereoCost.aggregateBytes */
  int32_t flags;               /* 0, or CSGM_FLAG_GENERAL */
  double uniqueness;           /* Options.uniqueness */
  double lr_threshold;         /* Options.lrThreshold */
} csgm_params;

/* Rejection counters: CensusSgm.Stats (src/main/java/sgm/CensusSgm.java:683-737). */
typedef struct csgm_stats {
  int64_t lower_boundary_rejected;
  int64_t full_interval_pixels;
  int64_t boundary_rejected;
  int64_t upper_boundary_rejected;
  int64_t ambiguity_rejected;
  int64_t selected;
  int64_t lr_rejected;
  int64_t post_median_lr_rejected;
  int64_t photometric_rejected;
  int64_t speckle_rejected;
  int64_t valid;
} csgm_stats;

/* Device description: GpuSgm.Device (src/main/java/sgm/GpuSgm.java:11-18). */
typedef struct csgm_device_info {
  char name[256];
  int64_t memory_bytes;
  int32_t sm_count;
  int32_t cc_major;
  int32_t cc_minor;
} csgm_device_info;

/* Per-session device timing: GpuSgm.Compute.profile (src/main/java/sgm/GpuSgm.java:592-604). */
typedef struct csgm_profile {
  int64_t kernel_ns;   /* summed device time of the library's kernels (CUDA events) */
  int64_t upload_ns;   /* host->device copy time */
  int64_t download_ns; /* device->host copy time */
  int64_t uploaded_bytes;
  int64_t downloaded_bytes;
  int64_t launches;    /* kernels launched by the library */
  int64_t calls;       /* csgm_match/csgm_pair calls profiled */
} csgm_profile;

typedef struct csgm_session csgm_session;

/* ---- library ---------------------------------------------------------------------------- */

/* ABI version (CSGM_ABI_VERSION). */
int csgm_version(void);

/* Message of the last failure on this thread ("" if none).  Thread-local, like the exception
 * text the reference attaches in GpuSgm.check (src/main/java/sgm/GpuSgm.java:56-58). */
const char* csgm_last_error(void);

/* Effective penalties from Options values: StereoCost.penalty / StereoCost.p2
 * (src/main/java/sgm/StereoCost.java:17-23), with bits = window_x * window_y - 1. */
int csgm_effective_penalties(double p1, double p2, int32_t window_x, int32_t window_y,
                             int32_t* p1_eff, int32_t* p2_eff);

/* Aggregate width: StereoCost.aggregateBound / aggregateBytes (src/main/java/sgm/StereoCost.java:31-41).
 * mode: 0 auto, 16 force uint16 (fails with CSGM_E_INVALID if the bound does not fit), 32 force uint32. */
int csgm_aggregate_bytes(int32_t directions, int32_t p2_eff, int32_t mode, int32_t* bytes,
                         int64_t* bound);

/* ---- devices and sessions ----------------------------------------------------------------- */

/* Number of CUDA devices: GpuSgm.devices (src/main/java/sgm/GpuSgm.java:79-141). */
int csgm_device_count(int32_t* count);

/* Device description: GpuSgm.enumerateDevices (src/main/java/sgm/GpuSgm.java:120-136). */
int csgm_device_info_get(int32_t device, csgm_device_info* info);

/* Open a session on a device: GpuSgm.session + constructor (src/main/java/sgm/GpuSgm.java:163-221).
 * CSGM_E_NODEVICE when the index does not exist (the reference's "No OpenCL GPU at index"). */
int csgm_session_open(int32_t device, csgm_session** session);

/* Close a session and free its device memory: GpuSgm.closeSession (src/main/java/sgm/GpuSgm.java:392-397). */
void csgm_session_close(csgm_session* session);

/* Device memory budget in bytes (0 = 70% of device memory): GpuSgm.budget
 * (src/main/java/sgm/GpuSgm.java:629-633). */
int csgm_session_set_budget(csgm_session* session, int64_t bytes);

/* How the views run: Options.gpuSgm (src/main/java/sgm/Options.java:32,780).  AUTO keeps the
 * whole cost volume and aggregate in device memory when they fit the budget and streams otherwise;
 * RESIDENT fails with CSGM_E_NOMEM when they do not fit; STREAMED always streams.  Streamed views
 * run on the general kernels through strips of rows (GpuStereo.java:339-437): a down pass over
 * the strips from the top aggregates the directions with dy >= 0, carrying path states across
 * strip edges and parking the strip's partial aggregate in pinned host memory, and an up pass from
 * the bottom adds the directions with dy < 0 to it and selects the strip's disparities.  Results
 * are bit-identical to the resident views. */
#define CSGM_SGM_AUTO 0
#define CSGM_SGM_RESIDENT 1
#define CSGM_SGM_STREAMED 2
/* Compact SGM, the reference's --gpu-sgm esgm (src/main/java/sgm/GpuCandidateStereo.java:53-167):
 * grayscale Census with 16-bit aggregates, no cost volume and no aggregate volume.  Every path
 * proposes a few separated disparities per pixel (csgm_session_set_candidates); the exact
 * aggregate at each proposal and its two neighbours and a lower bound of it elsewhere certify most
 * pixels' outcomes, and the others are aggregated exactly over every disparity.  Results are
 * bit-identical to the resident views; the winners records of certified pixels hold the best
 * known second value instead of the exact one. */
#define CSGM_SGM_COMPACT 3

/* mode: CSGM_SGM_*; strip_rows: the largest strip height (Options.gpuStripRows, 0 = 64), halved
 * until a strip fits the budget (GpuStereo.plan, src/main/java/sgm/GpuStereo.java:59-62). */
int csgm_session_set_streaming(csgm_session* session, int32_t mode, int32_t strip_rows);

/* Options.esgmCandidates (src/main/java/sgm/Options.java:35,244,781): the separated proposals each
 * path keeps per pixel in compact SGM, 1..4 (default 2); the plan lowers it until it fits. */
int csgm_session_set_candidates(csgm_session* session, int32_t per_path);

/* Host memory a streamed plan may use for its parked aggregate, GpuCandidateStereo.hostBudget
 * (src/main/java/sgm/GpuCandidateStereo.java:15-16: --memory-mb); 0 = no limit (the default).
 * Over it, AUTO runs compact SGM where it applies (grayscale Census, 16-bit aggregates;
 * GpuStereo.execute, src/main/java/sgm/GpuStereo.java:184-193) and otherwise, like STREAMED,
 * fails with CSGM_E_NOMEM. */
int csgm_session_set_host_budget(csgm_session* session, int64_t bytes);

/* Compact SGM's outcome for the session's last view of each side (reverse 0 = left, 1 = right):
 * the pixels its proposals certified and those it aggregated exactly (the reference's
 * esgm_left/right report, GpuCandidateStereo.java:106-131). */
int csgm_session_compact_report(csgm_session* session, int32_t reverse, int64_t* certified,
                                int64_t* verified);

/* Device bytes csgm_pair needs for a w x h pair under the session's budget and streaming mode;
 * CSGM_E_NOMEM if no plan fits.  Replaces GpuStereo.plan (src/main/java/sgm/GpuStereo.java:33-84). */
int csgm_plan(csgm_session* session, const csgm_params* params, int32_t w, int32_t h,
              int64_t* device_bytes);

/* The same plan in detail, the reference's Plan record (GpuStereo.java:33-84): strip_rows = h for
 * a resident plan, else the strip height; host_bytes = the pinned host memory a streamed plan
 * parks its partial aggregate in (0 when resident).  Any output may be NULL. */
int csgm_plan_detail(csgm_session* session, const csgm_params* params, int32_t w, int32_t h,
                     int32_t* strip_rows, int64_t* device_bytes, int64_t* host_bytes);

/* Largest disparity count whose plan fits the budget (0 if none):
 * GpuSgm.disparityLimit / GpuStereo.limit (src/main/java/sgm/GpuSgm.java:237-245,
 * src/main/java/sgm/GpuStereo.java:86-94). */
int csgm_disparity_limit(csgm_session* session, const csgm_params* params, int32_t w, int32_t h,
                         int32_t* limit);

/*
 * Launch shape of the fused sweep, picked per shape bucket by an autotuner (no counterpart in the
 * reference, whose OpenCL work-group size is a device property, src/main/java/sgm/GpuSgm.java:163-221).
 * Buckets: disparities rounded up to 64, paths, width and height in half-octaves.  Tuning never
 * changes results.
 */
typedef struct csgm_tuning {
  int32_t rows_per_block;  /* row warps per sweep CTA: 4, 8 (12 at 65..128 disparities) */
  int32_t line_warps;      /* warps per sweep CTA walking the anti-diagonal lines: 0, 4, 8 */
  int32_t line_slack;      /* percent of a block's remaining pixels a line may take: 10..1000 */
  int32_t disparity_lanes; /* disparities per lane and register half (fixed: padded D / 32) */
  double milliseconds;     /* measured pair time of this shape (0 when not measured) */
} csgm_tuning;

/* Times the candidate shapes on a synthetic w x h pair with these parameters, keeps the fastest
 * for the bucket in the session and, when cache_path is not NULL, stores it in that cache file
 * (text, one entry per line; other entries are kept).  CSGM_E_UNSUPPORTED when the fused kernels
 * do not run the parameters.  best (optional) receives the chosen shape and its time. */
int csgm_autotune(csgm_session* session, const csgm_params* params, int32_t w, int32_t h,
                  const char* cache_path, csgm_tuning* best);

/* Adds the entries of a tuning cache file to the session (a missing file adds nothing). */
int csgm_session_load_tuning(csgm_session* session, const char* cache_path);

/* Forces one shape for every call of the session (NULL: back to the tuned / default shapes). */
int csgm_session_set_tuning(csgm_session* session, const csgm_tuning* tuning);

/* The shape a call with these parameters and size would use now. */
int csgm_tuning_get(csgm_session* session, const csgm_params* params, int32_t w, int32_t h,
                    csgm_tuning* out);

/* The cache file's entry for these parameters and size, without a session or device;
 * out->rows_per_block is 0 when the file has none. */
int csgm_tuning_cache_lookup(const char* cache_path, const csgm_params* params, int32_t w,
                             int32_t h, csgm_tuning* out);

/* Accumulated device timing since the last reset (reset != 0 clears it afterwards). */
int csgm_profile_get(csgm_session* session, csgm_profile* out, int32_t reset);

/* Per-kernel device time, measured with CUDA events on the session's stream when profiling
 * level 2 is on.  The reference collects the same per-kernel sums from OpenCL profiling events
 * (src/main/java/sgm/GpuSgm.java:558-590). */
typedef struct csgm_kernel_time {
  char name[32];
  int64_t launches;
  int64_t total_ns;
} csgm_kernel_time;

/* 0 = off, 1 = per-call timing (csgm_profile), 2 = per-call and per-kernel timing. */
int csgm_session_set_profiling(csgm_session* session, int32_t level);

/* Copies up to `capacity` per-kernel records; *count receives the number of kernels seen. */
int csgm_kernel_times(csgm_session* session, csgm_kernel_time* out, int32_t capacity,
                      int32_t* count, int32_t reset);

/* CUDA graphs for csgm_pair_device (0 off, the default; 1 on): the first call with given
 * parameters, size, device buffers and launch shape runs normally and captures its device work
 * into a graph; calls that repeat it replay the graph (one launch instead of about a dozen).  A
 * graph is dropped when the session's workspace is reallocated.  Streamed pairs and per-kernel
 * profiling (level 2) run without graphs.  No counterpart in the reference. */
int csgm_session_set_graphs(csgm_session* session, int32_t enabled);

/* Graphs captured and replayed by the session so far. */
int csgm_graph_stats(csgm_session* session, int64_t* captured, int64_t* replayed);

/* Waits for all work queued on the session's stream. */
int csgm_session_synchronize(csgm_session* session);

/* Watchdog of the aggregation sweep's device-side waits (a CTA waiting for a bulk copy, for the
 * previous row block's carry row or for its own row warps): a wait that sees no progress for
 * `cycles` SM clock cycles gives up, the kernel winds down with no copy left in flight, and the
 * call returns CSGM_E_TIMEOUT with the wait's site code (1 cost chunk, 3 carry chunk, 5 copy drain,
 * 6 carry-in or publisher warp) in the message.  The context and the session stay usable.
 * 0 restores the default, 4e9 cycles (about two seconds).  The reference has no device-side wait
 * to bound: its OpenCL host blocks in clFinish (src/main/java/sgm/GpuSgm.java:606-609). */
int csgm_session_set_wait_limit(csgm_session* session, int64_t cycles);

/* ---- the hot path ------------------------------------------------------------------------ */

/*
 * One view of the matcher: cost volume, path aggregation, WTA, uniqueness and parabolic subpixel.
 * Exact drop-in for GpuSgm.match -> GpuStereo.execute (src/main/java/sgm/GpuSgm.java:267-303,
 * src/main/java/sgm/GpuStereo.java:170-210), i.e. for the CPU loops CensusSgm.match
 * (src/main/java/sgm/CensusSgm.java:375-516).
 *   desc_a/desc_b : [words][w*h] census words of the matching/target view (words = ceil(bits/64))
 *   gray_a/gray_b : matching/target images (edge-aware P2 and the AD/gradient/ZNCC costs)
 *   tex_a/tex_b   : textured & valid masks
 *   reverse       : 0 = left view (target x - d), 1 = right view (target x + d)
 *   out_disp      : float[w*h], NaN where no disparity is selected
 *   out_summary   : optional int32[6*w*h] winners record (best, value, second, before, after,
 *                   full-interval flags), src/main/java/sgm/GpuStereo.java:758-769
 *   reasons       : optional uint8[w*h]; pixels decided here get 0 (selected), 2 (boundary) or
 *                   3 (ambiguous); others are left as the caller set them
 *   boundary      : optional uint8[w*h] searchBoundary flags (4 full interval, |1 lower, |2 upper)
 *   stats         : optional; the six selection counters are ADDED to it, as GpuSgm.match merges
 *                   them (src/main/java/sgm/GpuSgm.java:289-294)
 */
int csgm_match(csgm_session* session, const csgm_params* params, const uint64_t* desc_a,
               const uint64_t* desc_b, const uint8_t* gray_a, const uint8_t* gray_b,
               const uint8_t* tex_a, const uint8_t* tex_b, int32_t w, int32_t h, int32_t reverse,
               float* out_disp, int32_t* out_summary, uint8_t* reasons, uint8_t* boundary,
               csgm_stats* stats);

/*
 * A whole rectified pair on the GPU: census + texture masks of both images (masks ANDed with the
 * optional validity masks), left and right views, and the left-right check.  Replaces
 * CensusSgm.computeRecorded up to the LR check (src/main/java/sgm/CensusSgm.java:56-201).
 *   left/right      : uint8[w*h] rectified images
 *   valid_l/valid_r : optional uint8[w*h] validity masks (both or neither)
 *   lr_checked      : float[w*h] left disparities that pass the LR check, NaN elsewhere
 *   disp_l/disp_r   : optional float[w*h] raw left/right view disparities (dl, dr)
 *   reasons         : optional uint8[w*h]; set to 1 everywhere, then 0/2/3 by the left view and 4
 *                     by the LR check (src/main/java/sgm/CensusSgm.java:104-106,190,198)
 *   boundary        : optional uint8[w*h] searchBoundary flags of the left view
 *   stats           : optional; overwritten with the left view's counters plus lr_rejected
 */
int csgm_pair(csgm_session* session, const csgm_params* params, const uint8_t* left,
              const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r, int32_t w,
              int32_t h, float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
              uint8_t* boundary, csgm_stats* stats);

/*
 * csgm_pair for --census-mode color-distance: the descriptors and texture masks come from the
 * colour-distance census of the interleaved BGR images (CensusSgm.colorCensus,
 * src/main/java/sgm/CensusSgm.java:108-120,302-332), the costs and penalties from the gray images,
 * as CensusSgm.computeRecorded runs it up to the LR check (:56-201).
 *   left_bgr/right_bgr : uint8[3*w*h] interleaved B, G, R; both required
 * Other arguments and outputs as csgm_pair.  HOST pointers.
 */
int csgm_pair_color(csgm_session* session, const csgm_params* params, const uint8_t* left,
                    const uint8_t* right, const uint8_t* left_bgr, const uint8_t* right_bgr,
                    const uint8_t* valid_l, const uint8_t* valid_r, int32_t w, int32_t h,
                    float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                    uint8_t* boundary, csgm_stats* stats);

/*
 * csgm_pair on device-resident buffers: every image/mask/output pointer is a device pointer on the
 * session's device (outputs may be NULL except lr_checked).  For callers whose rectified images
 * are already in HBM (a GPU rectifier upstream, or a batch driver).  With sync == 0 the call only
 * queues work on the session's stream and `stats` must be NULL; csgm_session_synchronize waits.
 * Same semantics as csgm_pair otherwise.
 */
int csgm_pair_device(csgm_session* session, const csgm_params* params, const uint8_t* left,
                     const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r,
                     int32_t w, int32_t h, float* lr_checked, float* disp_l, float* disp_r,
                     uint8_t* reasons, uint8_t* boundary, csgm_stats* stats, int32_t sync);

/*
 * Batched and served pairs.  No counterpart in the reference, which matches one pair per call and
 * keeps one session per Java thread (src/main/java/sgm/GpuSgm.java:22,163-303); every result is
 * bit-identical to csgm_pair on the same inputs.
 *
 * csgm_batch_configure: gives the session `slots` pair slots (1..64), each with its own CUDA stream
 * and a device workspace that stays resident between pairs, and a device-memory budget for all
 * of them (0 = 70% of device memory).  Fails with CSGM_E_BUSY while requests are in flight.
 */
int csgm_batch_configure(csgm_session* session, int32_t slots, int64_t budget_bytes);

/*
 * Queues one pair (arguments as csgm_pair) on a free slot and returns at once with *request set.
 * Host buffers must stay valid until csgm_batch_poll reports the request finished; pinned host
 * memory lets uploads and downloads overlap other pairs' kernels.  Admission: the workspace bytes
 * of the pairs in flight (cost volumes and aggregates, W*H*D based, plus images and outputs) and
 * this pair's must fit the budget, and a slot must be free; otherwise CSGM_E_BUSY and nothing is
 * queued (submit again after a poll).  CSGM_E_NOMEM: the pair alone exceeds the budget.
 */
int csgm_batch_submit(csgm_session* session, const csgm_params* params, const uint8_t* left,
                      const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r,
                      int32_t w, int32_t h, float* lr_checked, float* disp_l, float* disp_r,
                      uint8_t* reasons, uint8_t* boundary, int64_t* request);

/*
 * Collects a request: CSGM_OK once its outputs are in the caller's buffers (stats as csgm_pair),
 * CSGM_E_BUSY while it is still running (wait == 0), or the pair's own error status.  Waiting does
 * not hold the session lock: other threads may submit meanwhile.
 */
int csgm_batch_poll(csgm_session* session, int64_t request, int32_t wait, csgm_stats* stats);

/* Requests in flight, bytes admitted for them, bytes of resident slot workspaces. */
int csgm_batch_status(csgm_session* session, int32_t* in_flight, int64_t* reserved_bytes,
                      int64_t* resident_bytes);

/*
 * CensusSgm.colorCensus on the GPU (src/main/java/sgm/CensusSgm.java:302-332), the descriptor
 * step of --census-mode color-distance that the reference runs on the CPU before GpuSgm.match:
 * descriptors [words][w*h] (words = ceil((wx*wy-1)/64)) and the texture mask of an interleaved
 * BGR image, for csgm_match.  Windows are odd, wx*wy - 1 <= 128 bits.  HOST pointers; returns when
 * the outputs are written.
 */
int csgm_color_census(csgm_session* s, const uint8_t* bgr, int32_t w, int32_t h,
                      int32_t window_x, int32_t window_y, uint64_t* descriptors,
                      uint8_t* textured);

/* Post-filter settings: the Options fields that computeRecorded reads after the LR check
 * (src/main/java/sgm/CensusSgm.java:203-272; option checks src/main/java/sgm/Options.java). */
typedef struct csgm_post {
  int32_t median;                /* Options.median: odd window side 1..11 (1 = off) */
  int32_t median_classic;        /* 1 = Options.medianMode "classic", 0 = "edge-preserving" */
  int32_t median_edge_threshold; /* Options.medianEdgeThreshold, 0..255 (0 = no gray gate) */
  int32_t correlation_window;    /* Options.correlationWindow, odd 3..15 */
  int32_t speckle_size;          /* Options.speckleSize, >= 0 (<= 1 = off) */
  int32_t speckle_connectivity;  /* Options.speckleConnectivity, 4 or 8 */
  int32_t border;                /* reciprocity radius: Options.census / 2 */
  int32_t reserved;              /* 0 */
  double median_max_change;      /* Options.medianMaxChange, >= 0 */
  double correlation;            /* Options.correlation, -1..1 */
  double lr_threshold;           /* Options.lrThreshold, > 0 */
  double speckle_range;          /* Options.speckleRange, >= 0 */
} csgm_post;

/*
 * The post-filters of CensusSgm.computeRecorded on the GPU (src/main/java/sgm/CensusSgm.java:
 * 203-272): the classic (:557-573) or edge-preserving (:576-601) median of the LR-checked map,
 * the post-median reciprocity check against the right view (:226-239, :604-612), the ZNCC
 * photometric gate on the gray images (:240-257, :615-644, FP64) and the speckle removal
 * (:264-271, :647-681).  checked is updated in place; reasons (optional) receives 5 / 6 / 7 where
 * a pixel is rejected by the reciprocity check / the gate / the speckle removal.  stats (optional):
 * post_median_lr_rejected, photometric_rejected and valid are added to, speckle_rejected is set.
 *   left, right : gray images uint8 [h][w] (the matcher's inputs)
 *   disp_r      : the right view's disparities (csgm_pair's disp_r)
 * All pointers are HOST pointers; the call returns when the outputs are written.
 */
int csgm_postfilter(csgm_session* s, const csgm_post* post, const uint8_t* left,
                    const uint8_t* right, const float* disp_r, int32_t w, int32_t h,
                    float* checked, uint8_t* reasons, csgm_stats* stats);

/* csgm_postfilter for --census-mode color-distance: the photometric gate correlates the three
 * channels of the interleaved BGR images (CensusSgm.java:222-224,240-250, zncc :615-644 with
 * channels = 3); the edge-preserving median still reads the gray left image (:208-214).
 *   left_bgr/right_bgr : uint8[3*w*h]; other arguments as csgm_postfilter.  HOST pointers. */
int csgm_postfilter_color(csgm_session* s, const csgm_post* post, const uint8_t* left,
                          const uint8_t* right, const uint8_t* left_bgr, const uint8_t* right_bgr,
                          const float* disp_r, int32_t w, int32_t h, float* checked,
                          uint8_t* reasons, csgm_stats* stats);

/* Page-locked host memory (cudaMallocHost) for batch inputs and outputs; csgm_host_free releases
 * it.  No counterpart in the reference (its FFM arenas are pageable). */
int csgm_host_alloc(int64_t bytes, void** ptr);
void csgm_host_free(void* ptr);

/*
 * Left-right check that allocates nothing; no counterpart in the reference, whose check
 * (src/main/java/sgm/CensusSgm.java:181-201) always runs inside the matcher.  Same results as the
 * check inside csgm_pair: lr_checked[p] keeps disp_l[p] where the right view agrees within
 * lr_threshold, else NaN; reasons[p] (optional) becomes 4 where a pixel is rejected or its match
 * leaves the window interior; *lr_rejected (optional) receives the rejected count.
 *   disp_l, disp_r, lr_checked, reasons, lr_rejected : DEVICE pointers on the current device
 *   stream : cudaStream_t to queue on (NULL = default stream); the call returns after queueing
 * For callers that cannot let the library allocate device memory: the only scratch is a fixed
 * array in the library's static device memory, sized for h <= 16384 rows (larger heights are
 * rejected with CSGM_E_INVALID).  The first call on a device looks the array up, and so does the
 * first call after that device's context has been replaced (cudaDeviceReset); make those calls
 * before any stream capture.  Calls whose work overlaps in time on one device share the scratch
 * and must be serialised by the caller.
 */
int csgm_lr_check_noalloc(const float* disp_l, const float* disp_r, int32_t w, int32_t h,
                          int32_t window_x, int32_t window_y, double lr_threshold,
                          float* lr_checked, uint8_t* reasons, unsigned long long* lr_rejected,
                          void* stream);

#ifdef __cplusplus
}
#endif

#endif /* COLLINEA_SGM_H */
