// pipeline.cu - stage sequences of the matcher on one CUDA stream.
//
// A pair (CensusSgm.computeRecorded :56-201): census + texture of both images, the left view
// (CensusSgm.match with reverse=false), the right view (reverse=true), the left-right check.
// A view: cost volume, path aggregation, winner selection.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pipeline.h"
#include "stereo_fused.h"
#include "stereo_kernels.h"

namespace csgm {

#define CK(expr, what)                                 \
  do {                                                 \
    cudaError_t e_ = (expr);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

#define WS(var, type, slot, bytes)                            \
  type* var = (type*)ctx.ws->get((slot), (bytes), &status);   \
  if (!var) return status;

static int words_of(const csgm_params& p) { return (p.window_x * p.window_y - 1 + 63) / 64; }

// The fused kernels run the pair when its parameters allow them and it is at most 65535 rows
// tall (the sweep's row-block indices); otherwise the general kernels do.
static bool use_fused(const csgm_params& p, int h) {
  return !(p.flags & CSGM_FLAG_GENERAL) && fused_supported(p) && h <= 65535;
}

// Device bytes of a pair besides its cost volumes and aggregates: descriptors, masks, the views'
// disparities, counters and (host_inputs) the upload / download buffers.
static size_t pair_fixed_bytes(const csgm_params& p, int w, int h, bool host_inputs,
                               bool color) {
  size_t n = (size_t)w * h, words = (size_t)words_of(p);
  size_t bytes = color ? 6 * n : 0;  // BGR images
  bytes += 2 * n * words * 8;  // descriptors
  bytes += 2 * n;              // texture masks
  bytes += 2 * n * 4;          // raw view disparities
  bytes += sizeof(DeviceStats);
  if (host_inputs) bytes += 4 * n + n * 4 + 2 * n;  // images, masks, checked, reasons, boundary
  return bytes;
}

size_t pair_workspace_bytes(const csgm_params& p, int w, int h, bool host_inputs, bool color,
                            const SweepTuning& tuning) {
  size_t n = (size_t)w * h, D = (size_t)p.disparities;
  size_t bytes = pair_fixed_bytes(p, w, h, host_inputs, color);
  if (use_fused(p, h))
    bytes += fused_workspace_bytes(p, w, h, tuning);
  else
    bytes += n * D * 2 + n * D * p.aggregate_bytes;  // one cost volume + one aggregate
  return bytes;
}

// Device bytes of one streamed strip of `rows` rows: its cost volume and partial aggregate, and
// the path-state carries (two buffers of |dy| rows per direction that crosses strip edges).
static size_t strip_bytes(const csgm_params& p, int w, int rows) {
  const size_t D = (size_t)p.disparities, cells = (size_t)w * rows * D;
  size_t carry = 0;
  for (int d = 0; d < p.directions; d++) {
    int dx, dy;
    direction(d, dx, dy);
    carry += 2 * (size_t)(dy < 0 ? -dy : dy) * w * D * 4;
  }
  return cells * (2 + p.aggregate_bytes) + carry + 4 * 256;
}

// Device bytes of compact SGM besides `fixed`: proposals and compact aggregates (8 bytes per
// proposal and pixel), the lower bounds, the unresolved slots and list, and one image row of exact
// aggregates and cost rows (the least chunk of the exact pass).
static size_t compact_bytes(const csgm_params& p, int w, int h, int pool, int views) {
  const size_t n = (size_t)w * h, C = (size_t)p.directions * pool;
  return views * n * (C * 8 + 4 + 8) + 16 + (size_t)w * p.disparities * 4;
}

// GpuCandidateStereo.plan (GpuCandidateStereo.java:20-47): grayscale Census with 16-bit
// aggregates only; the proposals per path start at the session's count and drop until the
// compact buffers fit the budget.  A pair first tries both views at once (`views` = 2: twice the
// arrays, the path launches shared), then one view after the other.
static int compact_plan(const Context& ctx, const csgm_params& p, int w, int h, size_t fixed,
                        ViewPlan* plan, int views) {
  if (p.cost_mode != CSGM_COST_CENSUS || p.aggregate_bytes != 2)
    return fail(CSGM_E_INVALID, "compact SGM needs grayscale Census with 16-bit aggregates");
  if ((int64_t)w * h > INT32_MAX)  // the unresolved pixels' slots and list are int32
    return fail(CSGM_E_UNSUPPORTED, "compact SGM supports at most %d pixels", INT32_MAX);
  for (int at_once = views; at_once >= 1; at_once--) {
    for (int pool = ctx.candidates; pool >= 1; pool--) {
      const size_t bytes = fixed + compact_bytes(p, w, h, pool, at_once);
      if (bytes <= ctx.ws->budget) {
        plan->streamed = false;
        plan->compact = true;
        plan->views = at_once;
        plan->pool = pool;
        plan->rows = h;
        plan->device_bytes = bytes;
        plan->host_bytes = 0;
        return CSGM_OK;
      }
    }
  }
  return fail(CSGM_E_NOMEM,
              "No compact Census/16-bit GPU plan fits: needs %.1f MiB, budget %.1f MiB",
              (fixed + compact_bytes(p, w, h, 1, 1)) / 1048576.0, ctx.ws->budget / 1048576.0);
}

// GpuStereo.plan (GpuStereo.java:33-84): resident when the whole volume fits the budget (unless
// streaming is forced), else strips whose height starts at the session's strip height and halves
// until one fits.  Strips are at least two rows high with 16 paths, so that a (+-1,+-2) path's
// predecessor always lies in the previous strip.
static int choose_plan(const Context& ctx, const csgm_params& p, int w, int h, size_t fixed,
                       size_t resident, ViewPlan* plan, bool gray = true, int views = 2) {
  if (ctx.sgm_mode == CSGM_SGM_COMPACT) return compact_plan(ctx, p, w, h, fixed, plan, views);
  const size_t budget = ctx.ws->budget;
  if (ctx.sgm_mode != CSGM_SGM_STREAMED && resident <= budget) {
    plan->streamed = false;
    plan->rows = h;
    plan->device_bytes = resident;
    plan->host_bytes = 0;
    return CSGM_OK;
  }
  if (ctx.sgm_mode == CSGM_SGM_RESIDENT || !ctx.host_partial)
    return fail(CSGM_E_NOMEM,
                "GPU SGM search exceeds the device budget: needs %.1f MiB, budget %.1f MiB",
                resident / 1048576.0, budget / 1048576.0);
  const int min_rows = p.directions == 16 ? 2 : 1;
  for (int rows = std::min(h, std::max(ctx.strip_rows, min_rows)); rows >= min_rows; rows /= 2) {
    const size_t bytes = fixed + strip_bytes(p, w, rows);
    if (bytes <= budget) {
      const size_t host = (size_t)w * h * p.disparities * p.aggregate_bytes;
      if (ctx.host_budget && host > ctx.host_budget) {
        // GpuStereo.execute (GpuStereo.java:184-193): under auto, a view whose aggregate does
        // not fit host memory runs compact SGM where it applies.
        if (ctx.sgm_mode == CSGM_SGM_AUTO && gray && p.cost_mode == CSGM_COST_CENSUS &&
            p.aggregate_bytes == 2)
          return compact_plan(ctx, p, w, h, fixed, plan, views);
        return fail(CSGM_E_NOMEM,
                    "streamed SGM parks a %.1f MiB aggregate in host memory, over the host "
                    "budget of %.1f MiB",
                    host / 1048576.0, ctx.host_budget / 1048576.0);
      }
      plan->streamed = true;
      plan->rows = rows;
      plan->device_bytes = bytes;
      plan->host_bytes = (size_t)w * h * p.disparities * p.aggregate_bytes;
      return CSGM_OK;
    }
  }
  return fail(CSGM_E_NOMEM,
              "GPU SGM search exceeds the device budget even in strips of %d rows: needs %.1f "
              "MiB, budget %.1f MiB",
              min_rows, (fixed + strip_bytes(p, w, min_rows)) / 1048576.0, budget / 1048576.0);
}

int plan_pair(const Context& ctx, const csgm_params& p, int w, int h, bool host_inputs,
              ViewPlan* plan, bool color) {
  if (color && ctx.sgm_mode == CSGM_SGM_COMPACT)
    return fail(CSGM_E_INVALID, "compact SGM needs grayscale Census with 16-bit aggregates");
  return choose_plan(ctx, p, w, h, pair_fixed_bytes(p, w, h, host_inputs, color),
                     pair_workspace_bytes(p, w, h, host_inputs, color, ctx.tuning), plan, !color);
}

void* HostBuffer::get(size_t want, int* status) {
  if (bytes >= want && ptr) return ptr;
  release();
  cudaError_t e = cudaMallocHost(&ptr, want);
  if (e != cudaSuccess) {
    ptr = nullptr;
    *status = cuda_fail(e, "pinned host buffer of the streamed aggregate");
    return nullptr;
  }
  bytes = want;
  return ptr;
}

void HostBuffer::release() {
  if (ptr) cudaFreeHost(ptr);
  ptr = nullptr;
  bytes = 0;
}

// One view through the general kernels: cost volume, every path, selection.
static int run_view_general(Context& ctx, const csgm_params& p, const uint64_t* desc_a,
                            const uint64_t* desc_b, const uint8_t* tex_a, const uint8_t* tex_b,
                            const uint8_t* gray_a, const uint8_t* gray_b, int w, int h,
                            int reverse, float* out, int32_t* summary, uint8_t* reasons,
                            uint8_t* boundary, DeviceStats* dstats) {
  int status = CSGM_OK;
  size_t n = (size_t)w * h, D = (size_t)p.disparities;
  WS(cost, uint16_t, kCostL, n * D * 2);
  WS(sum, void, kSum, n * D * p.aggregate_bytes);
  CostArgs c{desc_a, desc_b, tex_a, tex_b, gray_a, gray_b, cost, w, h, p.disparities,
             p.min_disparity, reverse, p.window_x, p.window_y, words_of(p), p.cost_mode,
             p.census_weight_milli, p.ad_truncation, p.gradient_truncation,
             p.window_x * p.window_y - 1};
  ctx.prof->kernel_begin();
  CK(launch_cost_volume(c, ctx.sm_count, ctx.stream), "cost kernel launch");
  ctx.prof->kernel_end("cost_volume");
  CK(cudaMemsetAsync(sum, 0, n * D * p.aggregate_bytes, ctx.stream), "aggregate clear");
  for (int d = 0; d < p.directions; d++) {
    PathArgs a{cost, tex_a, gray_a, w, h, p.disparities, 0, 0, p.p1, p.p2, p.edge_scale};
    direction(d, a.dx, a.dy);
    ctx.prof->kernel_begin();
    CK(launch_paths_line(a, sum, p.aggregate_bytes, ctx.sm_count, ctx.stream),
       "paths kernel launch");
    ctx.prof->kernel_end("paths_line");
  }
  SelectArgs s{cost, out, summary, reasons, boundary, dstats, w, h, p.disparities,
               p.window_x, p.window_y, p.min_disparity, p.uniqueness};
  ctx.prof->kernel_begin();
  CK(launch_winners(s, sum, p.aggregate_bytes, ctx.sm_count, ctx.stream), "winners kernel launch");
  ctx.prof->kernel_end("winners");
  return CSGM_OK;
}

// The outputs of one compact SGM view.
struct CompactOut {
  float* out;
  int32_t* summary;
  uint8_t* reasons;
  uint8_t* boundary;
  DeviceStats* dstats;
};

// One view, or both views of a pair, through compact SGM (GpuCandidateStereo.execute,
// GpuCandidateStereo.java:53-167): every direction's proposals, then every direction's compact
// aggregates and lower bounds (both views in the same launches), then each view's selection of
// the certified pixels and list of the others.  The listed pixels of each view are then
// aggregated exactly, every path walked again with only their rows kept, in chunks that fit the
// budget, and selected from their full aggregates.  With two views, the second is the mirrored
// view of the first (a and b swapped, reverse flipped).
static int run_views_compact(Context& ctx, const csgm_params& p, int pool, int views,
                             const uint64_t* desc_a, const uint64_t* desc_b,
                             const uint8_t* tex_a, const uint8_t* tex_b, const uint8_t* gray_a,
                             const uint8_t* gray_b, int w, int h, int reverse,
                             const CompactOut* outs) {
  int status = CSGM_OK;
  const size_t n = (size_t)w * h, D = (size_t)p.disparities;
  const int C = p.directions * pool;
  WS(cand, uint16_t, kEsgmCand, views * n * C * 2);
  WS(compact, uint16_t, kEsgmCompact, views * n * C * 6);
  WS(outside, uint32_t, kEsgmOutside, views * n * 4);
  WS(slots, int32_t, kEsgmSlots, views * n * 4);
  WS(pixels, int32_t, kEsgmPixels, views * n * 4);
  WS(count, int32_t, kEsgmCount, 16);
  CostArgs c{desc_a, desc_b, tex_a, tex_b, gray_a, gray_b, nullptr, w, h, p.disparities,
             p.min_disparity, reverse, p.window_x, p.window_y, words_of(p), p.cost_mode,
             p.census_weight_milli, p.ad_truncation, p.gradient_truncation,
             p.window_x * p.window_y - 1};
  CK(cudaMemsetAsync(compact, 0, views * n * C * 6, ctx.stream), "compact clear");
  CK(cudaMemsetAsync(outside, 0, views * n * 4, ctx.stream), "bound clear");
  CK(cudaMemsetAsync(count, 0, 16, ctx.stream), "count clear");
  EsgmArgs e{c, p.directions, p.p1, p.p2, p.edge_scale, cand, compact, outside, C, pool, slots,
             nullptr};
  e.views = views;
  for (int phase = 0; phase < 2; phase++) {
    ctx.prof->kernel_begin();
    CK(launch_esgm_paths(e, phase, ctx.sm_count, ctx.stream), "compact path kernel launch");
    ctx.prof->kernel_end(phase == 0 ? "esgm_proposals" : "esgm_compact");
  }
  // View v's inputs and arrays.
  auto view_args = [&](int v) {
    EsgmArgs x = e;
    x.views = 1;
    if (v) {
      std::swap(x.cost.desc_a, x.cost.desc_b);
      std::swap(x.cost.tex_a, x.cost.tex_b);
      std::swap(x.cost.gray_a, x.cost.gray_b);
      x.cost.reverse = !x.cost.reverse;
    }
    x.cand = cand + v * n * C;
    x.compact = compact + v * 3 * n * C;
    x.outside = outside + v * n;
    x.slots = slots + v * n;
    return x;
  };
  for (int v = 0; v < views; v++) {
    const EsgmArgs x = view_args(v);
    const CompactOut& o = outs[v];
    SelectArgs s{nullptr, o.out, o.summary, o.reasons, o.boundary, o.dstats, w, h,
                 p.disparities, p.window_x, p.window_y, p.min_disparity, p.uniqueness};
    EsgmSelectArgs sel{x.cost, x.cand, x.compact, x.outside, s, C, slots + v * n,
                       pixels + v * n, count + v};
    ctx.prof->kernel_begin();
    CK(launch_esgm_select(sel, ctx.sm_count, ctx.stream), "compact select kernel launch");
    ctx.prof->kernel_end("esgm_select");
  }
  int32_t unresolved[2] = {0, 0};
  CK(cudaMemcpyAsync(unresolved, count, 8, cudaMemcpyDeviceToHost, ctx.stream),
     "unresolved count readback");
  CK(cudaStreamSynchronize(ctx.stream), "compact SGM proposals");
  for (int v = 0; v < views; v++) {
    const int side = views == 2 ? v : reverse;
    if (ctx.compact_report) {
      ctx.compact_report[2 * side] = (int64_t)n - unresolved[v];
      ctx.compact_report[2 * side + 1] = unresolved[v];
    }
  }
  // Both views' listed pixels in one exact pass when their rows fit the budget together.
  if (views == 2 && unresolved[0] > 0 && unresolved[1] > 0) {
    const Workspace& ws = *ctx.ws;
    const size_t held = ws.buffers[kEsgmSum].bytes + ws.buffers[kEsgmCost].bytes;
    const size_t room = ws.budget > ws.allocated - held ? ws.budget - (ws.allocated - held) : 0;
    const int64_t rows = (int64_t)unresolved[0] + unresolved[1];
    if ((size_t)rows * 4 * D <= room) {
      WS(sum, uint16_t, kEsgmSum, (size_t)rows * D * 2);
      WS(cost, uint16_t, kEsgmCost, (size_t)rows * D * 2);
      CK(cudaMemsetAsync(sum, 0, (size_t)rows * D * 2, ctx.stream), "exact aggregate clear");
      EsgmArgs x = e;  // view 0's arrays; the kernel finds view 1's after them
      x.sum = sum;
      x.slot_lo = 0;
      x.slot_hi = unresolved[0];
      x.sum2 = sum + (size_t)unresolved[0] * D;
      x.slot_lo2 = 0;
      x.slot_hi2 = unresolved[1];
      ctx.prof->kernel_begin();
      CK(launch_esgm_paths(x, 2, ctx.sm_count, ctx.stream), "exact path kernel launch");
      ctx.prof->kernel_end("esgm_exact");
      for (int v = 0; v < 2; v++) {
        const CompactOut& o = outs[v];
        const size_t first = v ? (size_t)unresolved[0] : 0;
        CostArgs cr = view_args(v).cost;
        cr.out = cost + first * D;
        cr.pixels = pixels + v * n;
        cr.npixels = unresolved[v];
        ctx.prof->kernel_begin();
        CK(launch_cost_volume(cr, ctx.sm_count, ctx.stream), "cost kernel launch");
        ctx.prof->kernel_end("cost_volume");
        SelectArgs sw{cost + first * D, o.out, o.summary, o.reasons, o.boundary, o.dstats, w, h,
                      p.disparities, p.window_x, p.window_y, p.min_disparity, p.uniqueness};
        sw.pixels = pixels + v * n;
        sw.npixels = unresolved[v];
        ctx.prof->kernel_begin();
        CK(launch_winners(sw, sum + first * D, 2, ctx.sm_count, ctx.stream),
           "winners kernel launch");
        ctx.prof->kernel_end("winners");
      }
      return CSGM_OK;
    }
  }
  for (int v = 0; v < views; v++) {
    if (unresolved[v] == 0) continue;
    const EsgmArgs x0 = view_args(v);
    const CompactOut& o = outs[v];
    // Exact pass in chunks of listed pixels: each chunk's aggregates and cost rows (4 bytes per
    // disparity and pixel) within what the budget leaves.
    const Workspace& ws = *ctx.ws;
    const size_t held = ws.buffers[kEsgmSum].bytes + ws.buffers[kEsgmCost].bytes;
    const size_t room = ws.budget > ws.allocated - held ? ws.budget - (ws.allocated - held) : 0;
    const int64_t chunk = std::min<int64_t>(unresolved[v], (int64_t)(room / (4 * D)));
    if (chunk < 1)
      return fail(CSGM_E_NOMEM, "compact SGM's exact pass exceeds the device budget");
    WS(sum, uint16_t, kEsgmSum, (size_t)chunk * D * 2);
    WS(cost, uint16_t, kEsgmCost, (size_t)chunk * D * 2);
    const int32_t* list = pixels + v * n;
    SelectArgs s{nullptr, o.out, o.summary, o.reasons, o.boundary, o.dstats, w, h,
                 p.disparities, p.window_x, p.window_y, p.min_disparity, p.uniqueness};
    for (int64_t lo = 0; lo < unresolved[v]; lo += chunk) {
      const int64_t rows = std::min<int64_t>(chunk, unresolved[v] - lo);
      CK(cudaMemsetAsync(sum, 0, (size_t)rows * D * 2, ctx.stream), "exact aggregate clear");
      EsgmArgs x = x0;
      x.sum = sum;
      x.slot_lo = (int32_t)lo;
      x.slot_hi = (int32_t)(lo + rows);
      ctx.prof->kernel_begin();
      CK(launch_esgm_paths(x, 2, ctx.sm_count, ctx.stream), "exact path kernel launch");
      ctx.prof->kernel_end("esgm_exact");
      CostArgs cr = x0.cost;
      cr.out = cost;
      cr.pixels = list + lo;
      cr.npixels = (int)rows;
      ctx.prof->kernel_begin();
      CK(launch_cost_volume(cr, ctx.sm_count, ctx.stream), "cost kernel launch");
      ctx.prof->kernel_end("cost_volume");
      SelectArgs sw = s;
      sw.cost = cost;
      sw.pixels = list + lo;
      sw.npixels = (int)rows;
      ctx.prof->kernel_begin();
      CK(launch_winners(sw, sum, 2, ctx.sm_count, ctx.stream), "winners kernel launch");
      ctx.prof->kernel_end("winners");
    }
  }
  return CSGM_OK;
}

// One view through strips of `rows` rows (GpuStereo.java:339-437, in two passes instead of one
// per direction).  The down pass visits the strips from the top and aggregates every direction
// with dy >= 0, each strip's lines starting from the path states its predecessor strip left in
// the carries; the strip's partial aggregate goes to pinned host memory.  The up pass visits the
// strips from the bottom, brings the partial back, adds the directions with dy < 0 and selects the
// strip's disparities.  Cost volumes are recomputed per pass.  A pixel's aggregate is the same
// sum of the same path costs as in the resident view (modular uint16 / exact int32 addition does
// not depend on the order), so the results are identical.
static int run_view_streamed(Context& ctx, const csgm_params& p, const uint64_t* desc_a,
                             const uint64_t* desc_b, const uint8_t* tex_a, const uint8_t* tex_b,
                             const uint8_t* gray_a, const uint8_t* gray_b, int w, int h,
                             int reverse, float* out, int32_t* summary, uint8_t* reasons,
                             uint8_t* boundary, DeviceStats* dstats, int rows) {
  int status = CSGM_OK;
  const size_t D = (size_t)p.disparities, Sb = (size_t)p.aggregate_bytes;
  const size_t strip_cells = (size_t)w * rows * D, row_cells = (size_t)w * D;
  WS(cost, uint16_t, kCostL, strip_cells * 2);
  WS(sum, uint8_t, kSum, strip_cells * Sb);
  size_t carry_offset[kMaxDirections] = {}, carry_words = 0;
  for (int d = 0; d < p.directions; d++) {
    int dx, dy;
    direction(d, dx, dy);
    carry_offset[d] = carry_words;
    carry_words += 2 * (size_t)(dy < 0 ? -dy : dy) * row_cells;
  }
  WS(carry, int32_t, kStripCarry, carry_words * 4);
  uint8_t* host = (uint8_t*)ctx.host_partial->get((size_t)w * h * D * Sb, &status);
  if (!host) return status;
  const int strips = (h + rows - 1) / rows;
  for (int pass = 0; pass < 2; pass++) {
    for (int ord = 0; ord < strips; ord++) {
      const int strip = pass == 0 ? ord : strips - 1 - ord;
      const int y0 = strip * rows, actual = std::min(rows, h - y0);
      const size_t cells = (size_t)w * actual * D;
      CostArgs c{desc_a, desc_b, tex_a, tex_b, gray_a, gray_b, cost, w, h, p.disparities,
                 p.min_disparity, reverse, p.window_x, p.window_y, words_of(p), p.cost_mode,
                 p.census_weight_milli, p.ad_truncation, p.gradient_truncation,
                 p.window_x * p.window_y - 1};
      c.y0 = y0;
      c.rows = actual;
      ctx.prof->kernel_begin();
      CK(launch_cost_volume(c, ctx.sm_count, ctx.stream), "cost kernel launch");
      ctx.prof->kernel_end("cost_volume");
      if (pass == 0)
        CK(cudaMemsetAsync(sum, 0, cells * Sb, ctx.stream), "aggregate clear");
      else
        CK(cudaMemcpyAsync(sum, host + (size_t)y0 * row_cells * Sb, cells * Sb,
                           cudaMemcpyHostToDevice, ctx.stream),
           "partial aggregate upload");
      for (int d = 0; d < p.directions; d++) {
        int dx, dy;
        direction(d, dx, dy);
        if ((pass == 0) != (dy >= 0)) continue;
        PathArgs a{cost, tex_a, gray_a, w, h, p.disparities, dx, dy, p.p1, p.p2, p.edge_scale};
        a.y0 = y0;
        a.rows = actual;
        if (dy != 0) {
          // Two carry buffers per direction, alternating: strip `ord` reads the one its
          // predecessor in path order wrote and writes the other.
          const size_t half = (size_t)(dy < 0 ? -dy : dy) * row_cells;
          int32_t* base = carry + carry_offset[d];
          a.carry_in = ord > 0 ? base + ((ord + 1) % 2) * half : nullptr;
          a.carry_out = base + (ord % 2) * half;
        }
        ctx.prof->kernel_begin();
        CK(launch_paths_line(a, sum, p.aggregate_bytes, ctx.sm_count, ctx.stream),
           "paths kernel launch");
        ctx.prof->kernel_end("paths_line");
      }
      if (pass == 0) {
        CK(cudaMemcpyAsync(host + (size_t)y0 * row_cells * Sb, sum, cells * Sb,
                           cudaMemcpyDeviceToHost, ctx.stream),
           "partial aggregate download");
      } else {
        SelectArgs sa{cost, out, summary, reasons, boundary, dstats, w, h, p.disparities,
                      p.window_x, p.window_y, p.min_disparity, p.uniqueness};
        sa.y0 = y0;
        sa.rows = actual;
        ctx.prof->kernel_begin();
        CK(launch_winners(sa, sum, p.aggregate_bytes, ctx.sm_count, ctx.stream),
           "winners kernel launch");
        ctx.prof->kernel_end("winners");
      }
    }
  }
  return CSGM_OK;
}

void copy_stats(const DeviceStats& d, csgm_stats* out, bool add) {
  if (!add) memset(out, 0, sizeof *out);
  out->lower_boundary_rejected += (int64_t)d.lower_boundary_rejected;
  out->full_interval_pixels += (int64_t)d.full_interval_pixels;
  out->boundary_rejected += (int64_t)d.boundary_rejected;
  out->upper_boundary_rejected += (int64_t)d.upper_boundary_rejected;
  out->ambiguity_rejected += (int64_t)d.ambiguity_rejected;
  out->selected += (int64_t)d.selected;
  out->lr_rejected += (int64_t)d.lr_rejected;
}

static float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return ms;
}

// A session's workspace keeps its buffers from call to call.  A call on a compact plan frees the
// volumes of the other plans first, and any other call frees compact SGM's arrays, so that the
// buffers the call's own plan counts fit the budget (nothing is freed when the plan repeats).
static void release_other_plans(Workspace& ws, bool compact) {
  static const int volumes[] = {kCostL, kCostR,    kSum,       kSumUp,     kSumLines,
                                kPen,   kCarry,    kFlags,     kPixelInfo, kStripCarry};
  static const int arrays[] = {kEsgmCand,   kEsgmCompact, kEsgmOutside, kEsgmSlots,
                               kEsgmPixels, kEsgmCount,   kEsgmSum,     kEsgmCost};
  if (compact)
    for (int slot : volumes) ws.release(slot);
  else
    for (int slot : arrays) ws.release(slot);
}

// The device part of a pair.  `own_call` = this is the whole call (csgm_pair_device), so it owns
// the call-level timing; csgm_pair times its own copies around it.
static int pair_on_device(Context& ctx, const csgm_params& p, const ViewPlan& plan,
                          const uint8_t* left, const uint8_t* right, const uint8_t* valid_l,
                          const uint8_t* valid_r, int w, int h, float* lr_checked, float* disp_l,
                          float* disp_r, uint8_t* reasons, uint8_t* boundary, csgm_stats* stats,
                          bool sync, bool own_call, const uint8_t* bgr_l = nullptr,
                          const uint8_t* bgr_r = nullptr) {
  int status = CSGM_OK;
  size_t n = (size_t)w * h;
  int words = words_of(p);
  release_other_plans(*ctx.ws, plan.compact);
  if (own_call) ctx.prof->begin_call(ctx.stream);
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (own_call && ctx.prof->level >= 1) {
    t0 = ctx.prof->event();
    t1 = ctx.prof->event();
    CK(cudaEventRecord(t0, ctx.stream), "event record");
  }
  WS(desc_l, uint64_t, kDescL, n * words * 8);
  WS(desc_r, uint64_t, kDescR, n * words * 8);
  WS(tex_l, uint8_t, kTexL, n);
  WS(tex_r, uint8_t, kTexR, n);
  WS(dstats, DeviceStats, kStats, sizeof(DeviceStats));
  if (!disp_l) {
    WS(buf, float, kDispL, n * 4);
    disp_l = buf;
  }
  if (!disp_r) {
    WS(buf, float, kDispR, n * 4);
    disp_r = buf;
  }
  CK(cudaMemsetAsync(dstats, 0, sizeof(DeviceStats), ctx.stream), "stats clear");
  if (reasons) CK(cudaMemsetAsync(reasons, 1, n, ctx.stream), "reasons init");
  if (boundary) CK(cudaMemsetAsync(boundary, 0, n, ctx.stream), "boundary init");
  if (bgr_l) {
    // CensusSgm.java:108-120,127-134: colour-distance descriptors and texture of the BGR images,
    // AND with the validity masks.
    ctx.prof->kernel_begin();
    CK(launch_color_census(bgr_l, valid_l, w, h, p.window_x, p.window_y, desc_l, tex_l,
                           ctx.sm_count, ctx.stream),
       "colour census launch");
    CK(launch_color_census(bgr_r, valid_r, w, h, p.window_x, p.window_y, desc_r, tex_r,
                           ctx.sm_count, ctx.stream),
       "colour census launch");
    ctx.prof->kernel_end("color_census");
  } else {
    // CensusSgm.java:122-134: descriptors, texture masks, AND with the validity masks.
    CensusArgs ca{};
    ca.image[0] = {left, valid_l, desc_l, tex_l};
    ca.image[1] = {right, valid_r, desc_r, tex_r};
    ca.w = w;
    ca.h = h;
    ca.wx = p.window_x;
    ca.wy = p.window_y;
    ca.words = words;
    ctx.prof->kernel_begin();
    CK(launch_census_texture(ca, 2, ctx.stream), "census kernel launch");
    ctx.prof->kernel_end("census_texture");
  }
  if (plan.streamed) {
    // Both views through strips (general kernels); the right view's counters are discarded.
    status = run_view_streamed(ctx, p, desc_l, desc_r, tex_l, tex_r, left, right, w, h, 0, disp_l,
                               nullptr, reasons, boundary, dstats, plan.rows);
    if (status) return status;
    status = run_view_streamed(ctx, p, desc_r, desc_l, tex_r, tex_l, right, left, w, h, 1, disp_r,
                               nullptr, nullptr, nullptr, nullptr, plan.rows);
    if (status) return status;
  } else if (plan.compact) {
    // Both views; the right view's counters are discarded.
    const CompactOut outs[2] = {{disp_l, nullptr, reasons, boundary, dstats},
                                {disp_r, nullptr, nullptr, nullptr, nullptr}};
    if (plan.views == 2) {
      status = run_views_compact(ctx, p, plan.pool, 2, desc_l, desc_r, tex_l, tex_r, left, right,
                                 w, h, 0, outs);
    } else {
      status = run_views_compact(ctx, p, plan.pool, 1, desc_l, desc_r, tex_l, tex_r, left, right,
                                 w, h, 0, &outs[0]);
      if (status) return status;
      status = run_views_compact(ctx, p, plan.pool, 1, desc_r, desc_l, tex_r, tex_l, right, left,
                                 w, h, 1, &outs[1]);
    }
    if (status) return status;
  } else if (use_fused(p, h)) {
    // Both views in one pass structure (stereo_fused.cu).
    FusedViews v{desc_l,           desc_r,           tex_l,          tex_r,
                 left,             right,            disp_l,         disp_r,
                 {reasons, nullptr}, {boundary, nullptr}, {dstats, nullptr}, {nullptr, nullptr}};
    int* error_flag = nullptr;
    status = run_views_fused(ctx, p, v, w, h, &error_flag);
    if (status) return status;
    CK(cudaMemcpyAsync(&dstats->pad, error_flag, sizeof(int), cudaMemcpyDeviceToDevice,
                       ctx.stream),
       "error flag copy");
  } else {
    status = run_view_general(ctx, p, desc_l, desc_r, tex_l, tex_r, left, right, w, h, 0, disp_l,
                              nullptr, reasons, boundary, dstats);
    if (status) return status;
    // Right view: a/b, masks and grays swapped, reverse=true; its counters are discarded
    // (CensusSgm.java:149-162 passes a fresh Stats and no reasons).
    status = run_view_general(ctx, p, desc_r, desc_l, tex_r, tex_l, right, left, w, h, 1, disp_r,
                              nullptr, nullptr, nullptr, nullptr);
    if (status) return status;
  }
  LrArgs lr{disp_l, disp_r, lr_checked, reasons, dstats, w, h, p.window_x, p.window_y,
            p.lr_threshold};
  ctx.prof->kernel_begin();
  CK(launch_lr_check(lr, ctx.sm_count, ctx.stream), "LR kernel launch");
  ctx.prof->kernel_end("lr_check");
  if (t1) CK(cudaEventRecord(t1, ctx.stream), "event record");
  if (!sync) return CSGM_OK;
  DeviceStats host{};
  CK(cudaMemcpyAsync(&host, dstats, sizeof host, cudaMemcpyDeviceToHost, ctx.stream),
     "stats readback");
  CK(cudaStreamSynchronize(ctx.stream), "GPU SGM execution");
  if (host.pad) return fail(CSGM_E_TIMEOUT, "a bounded device wait expired (code %llu)", host.pad);
  if (stats) copy_stats(host, stats, false);
  if (t1) {
    ctx.profile->kernel_ns += (int64_t)(elapsed_ms(t0, t1) * 1e6);
    ctx.profile->calls++;
  }
  ctx.prof->collect();
  return CSGM_OK;
}

int run_pair_device(Context& ctx, const csgm_params& p, const uint8_t* left, const uint8_t* right,
                    const uint8_t* valid_l, const uint8_t* valid_r, int w, int h,
                    float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                    uint8_t* boundary, csgm_stats* stats, bool sync) {
  ViewPlan plan;
  int status = plan_pair(ctx, p, w, h, false, &plan);
  if (status) return status;
  if (plan.streamed && !sync)
    return fail(CSGM_E_INVALID, "a streamed pair needs sync != 0 (its strips use host memory)");
  if (plan.compact && !sync)
    return fail(CSGM_E_INVALID, "a compact SGM pair needs sync != 0 (it reads back its count)");
  return pair_on_device(ctx, p, plan, left, right, valid_l, valid_r, w, h, lr_checked, disp_l,
                        disp_r, reasons, boundary, stats, sync, true);
}

void GraphCache::clear() {
  for (auto& e : entries)
    if (e.exec) cudaGraphExecDestroy(e.exec);
  entries.clear();
}

int run_pair_device_graph(Context& ctx, GraphCache& cache, const csgm_params& p,
                          const uint8_t* left, const uint8_t* right, const uint8_t* valid_l,
                          const uint8_t* valid_r, int w, int h, float* lr_checked, float* disp_l,
                          float* disp_r, uint8_t* reasons, uint8_t* boundary, csgm_stats* stats,
                          bool sync) {
  ViewPlan plan;
  int status = plan_pair(ctx, p, w, h, false, &plan);
  if (status) return status;
  if (plan.streamed || plan.compact)  // host copies and a count readback: not captured
    return run_pair_device(ctx, p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l,
                           disp_r, reasons, boundary, stats, sync);
  // The key: everything the captured work depends on.
  struct Key {
    csgm_params p;
    int w, h;
    const void* ptr[9];
    SweepTuning tuning;
    long long wait_limit;
  } key{};
  key.p = p;
  key.w = w;
  key.h = h;
  const void* ptrs[9] = {left, right, valid_l, valid_r, lr_checked, disp_l, disp_r, reasons,
                         boundary};
  memcpy(key.ptr, ptrs, sizeof ptrs);
  key.tuning = ctx.tuning;
  key.wait_limit = ctx.wait_limit;
  std::vector<uint8_t> bytes((const uint8_t*)&key, (const uint8_t*)&key + sizeof key);
  GraphCache::Entry* hit = nullptr;
  for (auto& e : cache.entries)
    if (e.key == bytes && e.generation == ctx.ws->generation) hit = &e;
  if (!hit) {
    // The plain run allocates what the pipeline needs and gives this call's results; the same
    // work is then captured for the calls that repeat it.
    status = run_pair_device(ctx, p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l,
                             disp_r, reasons, boundary, stats, sync);
    if (status) return status;
    const uint64_t generation = ctx.ws->generation;
    CK(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    const int level = ctx.prof->level;
    ctx.prof->level = 0;
    const int64_t launches = ctx.prof->launches;
    const int captured = pair_on_device(ctx, p, plan, left, right, valid_l, valid_r, w, h,
                                        lr_checked, disp_l, disp_r, reasons, boundary, nullptr,
                                        false, false);
    ctx.prof->level = level;
    const int64_t in_graph = ctx.prof->launches - launches;
    ctx.prof->launches = launches;
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(ctx.stream, &graph);
    cudaGraphExec_t exec = nullptr;
    const bool ok = captured == CSGM_OK && end == cudaSuccess && graph &&
                    ctx.ws->generation == generation &&
                    cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();  // a capture that did not work leaves the plain run's results
    if (cache.entries.size() >= GraphCache::kCapacity) {
      auto oldest = std::min_element(cache.entries.begin(), cache.entries.end(),
                                     [](const GraphCache::Entry& a, const GraphCache::Entry& b) {
                                       return a.used < b.used;
                                     });
      if (oldest->exec) cudaGraphExecDestroy(oldest->exec);
      cache.entries.erase(oldest);
    }
    // A key whose work could not be captured is remembered too, so it runs plainly from now on.
    cache.entries.push_back({bytes, ok ? exec : nullptr, generation, ++cache.clock, in_graph});
    if (ok) cache.captured++;
    return CSGM_OK;
  }
  if (!hit->exec)
    return run_pair_device(ctx, p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l,
                           disp_r, reasons, boundary, stats, sync);
  // Replay.
  hit->used = ++cache.clock;
  cache.replayed++;
  ctx.prof->begin_call(ctx.stream);
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (ctx.prof->level >= 1) {
    t0 = ctx.prof->event();
    t1 = ctx.prof->event();
    CK(cudaEventRecord(t0, ctx.stream), "event record");
  }
  CK(cudaGraphLaunch(hit->exec, ctx.stream), "graph launch");
  if (t1) CK(cudaEventRecord(t1, ctx.stream), "event record");
  ctx.prof->launches += hit->launches;
  if (!sync) return CSGM_OK;
  DeviceStats host{};
  CK(cudaMemcpyAsync(&host, ctx.ws->buffers[kStats].ptr, sizeof host, cudaMemcpyDeviceToHost,
                     ctx.stream),
     "stats readback");
  CK(cudaStreamSynchronize(ctx.stream), "GPU SGM execution");
  if (host.pad) return fail(CSGM_E_TIMEOUT, "a bounded device wait expired (code %llu)", host.pad);
  if (stats) copy_stats(host, stats, false);
  if (t1) {
    ctx.profile->kernel_ns += (int64_t)(elapsed_ms(t0, t1) * 1e6);
    ctx.profile->calls++;
  }
  return CSGM_OK;
}

// Uploads, device pipeline and downloads of a pair with host buffers, queued on ctx.stream.
// pinned_stats (may be null) receives the selection counters; *host_d2h_stats says whether it was
// queued.  Returns before the GPU has finished.
static int queue_pair_host(Context& ctx, const csgm_params& p, const uint8_t* left,
                           const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r,
                           int w, int h, float* lr_checked, float* disp_l, float* disp_r,
                           uint8_t* reasons, uint8_t* boundary, DeviceStats* stats_dst,
                           cudaEvent_t* timing /* [4] or null */,
                           const uint8_t* bgr_l = nullptr, const uint8_t* bgr_r = nullptr) {
  int status = CSGM_OK;
  size_t n = (size_t)w * h;
  // The plan is settled before the upload, so a budget failure costs no copies.
  ViewPlan plan;
  status = plan_pair(ctx, p, w, h, true, &plan, bgr_l != nullptr);
  if (status) return status;
  uint8_t *d_bgr_l = nullptr, *d_bgr_r = nullptr;
  if (bgr_l) {
    WS(a, uint8_t, kBgrL, 3 * n);
    WS(b, uint8_t, kBgrR, 3 * n);
    d_bgr_l = a;
    d_bgr_r = b;
  }
  WS(d_left, uint8_t, kImgL, n);
  WS(d_right, uint8_t, kImgR, n);
  uint8_t *d_vl = nullptr, *d_vr = nullptr;
  if (valid_l) {
    WS(a, uint8_t, kValidL, n);
    WS(b, uint8_t, kValidR, n);
    d_vl = a;
    d_vr = b;
  }
  WS(d_checked, float, kChecked, n * 4);
  WS(d_dl, float, kDispL, n * 4);
  WS(d_dr, float, kDispR, n * 4);
  uint8_t* d_reasons = nullptr;
  uint8_t* d_boundary = nullptr;
  if (reasons) {
    WS(r, uint8_t, kReasons, n);
    d_reasons = r;
  }
  if (boundary) {
    WS(b, uint8_t, kBoundary, n);
    d_boundary = b;
  }
  if (timing) CK(cudaEventRecord(timing[0], ctx.stream), "event record");
  CK(cudaMemcpyAsync(d_left, left, n, cudaMemcpyHostToDevice, ctx.stream), "image upload");
  CK(cudaMemcpyAsync(d_right, right, n, cudaMemcpyHostToDevice, ctx.stream), "image upload");
  if (valid_l) {
    CK(cudaMemcpyAsync(d_vl, valid_l, n, cudaMemcpyHostToDevice, ctx.stream), "mask upload");
    CK(cudaMemcpyAsync(d_vr, valid_r, n, cudaMemcpyHostToDevice, ctx.stream), "mask upload");
  }
  if (bgr_l) {
    CK(cudaMemcpyAsync(d_bgr_l, bgr_l, 3 * n, cudaMemcpyHostToDevice, ctx.stream), "BGR upload");
    CK(cudaMemcpyAsync(d_bgr_r, bgr_r, 3 * n, cudaMemcpyHostToDevice, ctx.stream), "BGR upload");
  }
  if (timing) CK(cudaEventRecord(timing[1], ctx.stream), "event record");
  status = pair_on_device(ctx, p, plan, d_left, d_right, d_vl, d_vr, w, h, d_checked, d_dl, d_dr,
                          d_reasons, d_boundary, nullptr, false, false, d_bgr_l, d_bgr_r);
  if (status) return status;
  if (timing) CK(cudaEventRecord(timing[2], ctx.stream), "event record");
  CK(cudaMemcpyAsync(lr_checked, d_checked, n * 4, cudaMemcpyDeviceToHost, ctx.stream),
     "disparity readback");
  if (disp_l)
    CK(cudaMemcpyAsync(disp_l, d_dl, n * 4, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  if (disp_r)
    CK(cudaMemcpyAsync(disp_r, d_dr, n * 4, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  if (reasons)
    CK(cudaMemcpyAsync(reasons, d_reasons, n, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  if (boundary)
    CK(cudaMemcpyAsync(boundary, d_boundary, n, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  WS(dstats, DeviceStats, kStats, sizeof(DeviceStats));
  CK(cudaMemcpyAsync(stats_dst, dstats, sizeof(DeviceStats), cudaMemcpyDeviceToHost, ctx.stream),
     "stats readback");
  if (timing) CK(cudaEventRecord(timing[3], ctx.stream), "event record");
  return CSGM_OK;
}

int enqueue_pair_host(Context& ctx, const csgm_params& p, const uint8_t* left,
                      const uint8_t* right, const uint8_t* valid_l, const uint8_t* valid_r, int w,
                      int h, float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                      uint8_t* boundary, DeviceStats* host_stats) {
  ctx.prof->begin_call(ctx.stream);
  return queue_pair_host(ctx, p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l, disp_r,
                         reasons, boundary, host_stats, nullptr);
}

int run_pair_host(Context& ctx, const csgm_params& p, const uint8_t* left, const uint8_t* right,
                  const uint8_t* valid_l, const uint8_t* valid_r, int w, int h,
                  float* lr_checked, float* disp_l, float* disp_r, uint8_t* reasons,
                  uint8_t* boundary, csgm_stats* stats, const uint8_t* bgr_l,
                  const uint8_t* bgr_r) {
  size_t n = (size_t)w * h;
  bool timed = ctx.prof->level >= 1;
  ctx.prof->begin_call(ctx.stream);
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (timed)
    for (auto& e : ev) e = ctx.prof->event();
  DeviceStats host{};
  int status = queue_pair_host(ctx, p, left, right, valid_l, valid_r, w, h, lr_checked, disp_l,
                               disp_r, reasons, boundary, &host, timed ? ev : nullptr, bgr_l,
                               bgr_r);
  if (status) return status;
  CK(cudaStreamSynchronize(ctx.stream), "GPU SGM execution");
  if (host.pad) return fail(CSGM_E_TIMEOUT, "a bounded device wait expired (code %llu)", host.pad);
  if (stats) copy_stats(host, stats, false);
  if (timed) {
    ctx.profile->upload_ns += (int64_t)(elapsed_ms(ev[0], ev[1]) * 1e6);
    ctx.profile->kernel_ns += (int64_t)(elapsed_ms(ev[1], ev[2]) * 1e6);
    ctx.profile->download_ns += (int64_t)(elapsed_ms(ev[2], ev[3]) * 1e6);
    ctx.profile->uploaded_bytes += (int64_t)((valid_l ? 4 * n : 2 * n) + (bgr_l ? 6 * n : 0));
    ctx.profile->downloaded_bytes += (int64_t)(n * 4 * (1 + (disp_l != 0) + (disp_r != 0)) +
                                               (reasons ? n : 0) + (boundary ? n : 0));
    ctx.profile->calls++;
  }
  ctx.prof->collect();
  return CSGM_OK;
}

// Device bytes of csgm_match on the fused kernels (summary: winners records requested).
static size_t match_fused_bytes(const csgm_params& p, int w, int h, bool summary,
                                const SweepTuning& tuning) {
  const size_t n = (size_t)w * h, words = (size_t)words_of(p);
  const size_t inputs = 2 * n * words * 8 + 4 * n;  // one set: descriptors, grays, masks
  return fused_workspace_bytes(p, w, h, tuning) + 2 * inputs +
         2 * (4 * n + 2 * n + (summary ? 24 * n : 0) + sizeof(DeviceStats)) + 16 * 256;
}

// Caller's reason codes / boundary flags updated from the device's per-view codes, 0xff = the
// selection did not decide this pixel (the caller's value stays), as GpuSgm.match copies back
// only what the selection wrote (GpuSgm.java:289-296).
static void merge_codes(const std::vector<uint8_t>& codes, uint8_t* dst) {
  const size_t n = codes.size();
  const uint8_t* c = codes.data();
  for (size_t i = 0; i < n; i++) dst[i] = c[i] != 0xff ? c[i] : dst[i];
}

// csgm_match on the fused kernels.  Both views of the pair are computed; the requested one is
// returned and the other is held on the device (MatchTwin) for the mirrored call that follows.
// A call whose inputs, after upload, are byte-identical to the held pair's (and whose parameters
// and size are equal) returns the held view without computing.
static int run_match_fused(Context& ctx, const csgm_params& p, const uint64_t* desc_a,
                           const uint64_t* desc_b, const uint8_t* gray_a, const uint8_t* gray_b,
                           const uint8_t* tex_a, const uint8_t* tex_b, int w, int h, int reverse,
                           float* out_disp, int32_t* out_summary, uint8_t* reasons,
                           uint8_t* boundary, csgm_stats* stats) {
  int status = CSGM_OK;
  MatchTwin& twin = *ctx.twin;
  const size_t n = (size_t)w * h;
  const size_t desc_bytes = n * words_of(p) * 8;
  const int view = reverse ? 1 : 0;
  // Inputs in the pair's order: view 0 matches l against r.
  const void* host_in[6] = {reverse ? desc_b : desc_a, reverse ? desc_a : desc_b,
                            reverse ? gray_b : gray_a, reverse ? gray_a : gray_b,
                            reverse ? tex_b : tex_a,   reverse ? tex_a : tex_b};
  const size_t in_bytes[6] = {desc_bytes, desc_bytes, n, n, n, n};
  const int set = twin.valid ? 1 - twin.set : 0;  // keep the held pair's inputs
  const int base = set ? kMatchIn1 : kMatchIn0;
  void* in[6];
  for (int i = 0; i < 6; i++) {
    in[i] = ctx.ws->get(base + i, in_bytes[i], &status);
    if (!in[i]) return status;
  }
  WS(equal_flag, int, kMatchEqual, sizeof(int));
  const bool timed = ctx.prof->level >= 1;
  ctx.prof->begin_call(ctx.stream);
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (timed)
    for (auto& e : ev) e = ctx.prof->event();
  if (timed) CK(cudaEventRecord(ev[0], ctx.stream), "event record");
  for (int i = 0; i < 6; i++)
    CK(cudaMemcpyAsync(in[i], host_in[i], in_bytes[i], cudaMemcpyHostToDevice, ctx.stream),
       "input upload");
  if (timed) CK(cudaEventRecord(ev[1], ctx.stream), "event record");
  uint8_t* codes_r[2];
  uint8_t* codes_b[2];
  float* disp[2];
  for (int v = 0; v < 2; v++) {
    WS(d, float, kMatchDisp + v, n * 4);
    WS(r, uint8_t, kMatchReasons + v, n);
    WS(b, uint8_t, kMatchBoundary + v, n);
    disp[v] = d;
    codes_r[v] = r;
    codes_b[v] = b;
  }
  WS(dstats, DeviceStats, kMatchStats, 2 * sizeof(DeviceStats));
  int32_t* summary[2] = {nullptr, nullptr};
  const bool held = twin.valid && twin.view == view && twin.w == w && twin.h == h &&
                    memcmp(&twin.params, &p, sizeof p) == 0 && (!out_summary || twin.summary);
  bool served = false;
  if (held) {
    // The mirrored call: compare its inputs with the held pair's.
    const int held_base = twin.set ? kMatchIn1 : kMatchIn0;
    CK(cudaMemsetAsync(equal_flag, 0, sizeof(int), ctx.stream), "flag clear");
    for (int i = 0; i < 6; i++) {
      ctx.prof->kernel_begin();
      CK(launch_bytes_differ(in[i], ctx.ws->buffers[held_base + i].ptr, in_bytes[i], equal_flag,
                             ctx.sm_count, ctx.stream),
         "input comparison");
      ctx.prof->kernel_end("bytes_differ");
    }
    int differ = 1;
    CK(cudaMemcpyAsync(&differ, equal_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream),
       "flag readback");
    CK(cudaStreamSynchronize(ctx.stream), "input comparison");
    served = differ == 0;
  }
  twin.valid = false;
  DeviceStats host_stats[2] = {};
  if (served) {
    host_stats[view] = twin.stats;
    if (out_summary) {
      WS(sm, int32_t, kMatchSummary + view, n * 24);
      summary[view] = sm;
    }
  } else {
    if (out_summary)
      for (int v = 0; v < 2; v++) {
        WS(sm, int32_t, kMatchSummary + v, n * 24);
        summary[v] = sm;
      }
    for (int v = 0; v < 2; v++) {
      CK(cudaMemsetAsync(codes_r[v], 0xff, n, ctx.stream), "reason codes init");
      CK(cudaMemsetAsync(codes_b[v], 0xff, n, ctx.stream), "boundary codes init");
    }
    CK(cudaMemsetAsync(dstats, 0, 2 * sizeof(DeviceStats), ctx.stream), "stats clear");
    FusedViews fv{(const uint64_t*)in[0], (const uint64_t*)in[1], (const uint8_t*)in[4],
                  (const uint8_t*)in[5],  (const uint8_t*)in[2],  (const uint8_t*)in[3],
                  disp[0],                disp[1],                {codes_r[0], codes_r[1]},
                  {codes_b[0], codes_b[1]}, {dstats, dstats + 1}, {summary[0], summary[1]}};
    int* error_flag = nullptr;
    status = run_views_fused(ctx, p, fv, w, h, &error_flag);
    if (status) return status;
    CK(cudaMemcpyAsync(&dstats->pad, error_flag, sizeof(int), cudaMemcpyDeviceToDevice,
                       ctx.stream),
       "error flag copy");
    CK(cudaMemcpyAsync(host_stats, dstats, 2 * sizeof(DeviceStats), cudaMemcpyDeviceToHost,
                       ctx.stream),
       "stats readback");
  }
  if (timed) CK(cudaEventRecord(ev[2], ctx.stream), "event record");
  CK(cudaMemcpyAsync(out_disp, disp[view], n * 4, cudaMemcpyDeviceToHost, ctx.stream),
     "readback");
  if (out_summary)
    CK(cudaMemcpyAsync(out_summary, summary[view], n * 24, cudaMemcpyDeviceToHost, ctx.stream),
       "readback");
  std::vector<uint8_t> rcodes(reasons ? n : 0), bcodes(boundary ? n : 0);
  if (reasons)
    CK(cudaMemcpyAsync(rcodes.data(), codes_r[view], n, cudaMemcpyDeviceToHost, ctx.stream),
       "readback");
  if (boundary)
    CK(cudaMemcpyAsync(bcodes.data(), codes_b[view], n, cudaMemcpyDeviceToHost, ctx.stream),
       "readback");
  if (timed) CK(cudaEventRecord(ev[3], ctx.stream), "event record");
  CK(cudaStreamSynchronize(ctx.stream), "GPU SGM execution");
  if (!served && host_stats[0].pad)
    return fail(CSGM_E_TIMEOUT, "a bounded device wait expired (code %llu)", host_stats[0].pad);
  if (reasons) merge_codes(rcodes, reasons);
  if (boundary) merge_codes(bcodes, boundary);
  if (stats) copy_stats(host_stats[view], stats, true);
  if (!served) {
    twin.valid = true;
    twin.set = set;
    twin.view = 1 - view;
    twin.params = p;
    twin.w = w;
    twin.h = h;
    twin.summary = out_summary != nullptr;
    twin.stats = host_stats[1 - view];
  }
  if (timed) {
    ctx.profile->upload_ns += (int64_t)(elapsed_ms(ev[0], ev[1]) * 1e6);
    ctx.profile->kernel_ns += (int64_t)(elapsed_ms(ev[1], ev[2]) * 1e6);
    ctx.profile->download_ns += (int64_t)(elapsed_ms(ev[2], ev[3]) * 1e6);
    ctx.profile->uploaded_bytes += (int64_t)(2 * desc_bytes + 4 * n);
    ctx.profile->downloaded_bytes += (int64_t)(n * 4 + (out_summary ? 24 * n : 0) +
                                               (reasons ? n : 0) + (boundary ? n : 0));
    ctx.profile->calls++;
  }
  ctx.prof->collect();
  return CSGM_OK;
}

// csgm_match through the general kernels: one view, any D, uint32 aggregates, 16 paths.
// Device bytes of csgm_match on the general kernels besides its cost volume and aggregate.
static size_t match_fixed_bytes(const csgm_params& p, int w, int h, bool summary) {
  const size_t n = (size_t)w * h;
  return 2 * n * words_of(p) * 8 + 6 * n + n * 4 + (summary ? 24 * n : 0) + sizeof(DeviceStats);
}

static int run_match_general(Context& ctx, const csgm_params& p, const ViewPlan& plan,
                             const uint64_t* desc_a, const uint64_t* desc_b, const uint8_t* gray_a,
                             const uint8_t* gray_b, const uint8_t* tex_a, const uint8_t* tex_b,
                             int w, int h, int reverse, float* out_disp, int32_t* out_summary,
                             uint8_t* reasons, uint8_t* boundary, csgm_stats* stats) {
  int status = CSGM_OK;
  size_t n = (size_t)w * h;
  int words = words_of(p);
  release_other_plans(*ctx.ws, plan.compact);
  WS(d_a, uint64_t, kDescL, n * words * 8);
  WS(d_b, uint64_t, kDescR, n * words * 8);
  WS(d_ga, uint8_t, kImgL, n);
  WS(d_gb, uint8_t, kImgR, n);
  WS(d_ta, uint8_t, kTexL, n);
  WS(d_tb, uint8_t, kTexR, n);
  WS(d_out, float, kDispL, n * 4);
  WS(dstats, DeviceStats, kStats, sizeof(DeviceStats));
  int32_t* d_summary = nullptr;
  uint8_t *d_reasons = nullptr, *d_boundary = nullptr;
  if (out_summary) {
    WS(s, int32_t, kSummary, n * 24);
    d_summary = s;
  }
  if (reasons) {
    WS(r, uint8_t, kReasons, n);
    d_reasons = r;
  }
  if (boundary) {
    WS(b, uint8_t, kBoundary, n);
    d_boundary = b;
  }
  ctx.prof->begin_call(ctx.stream);
  CK(cudaMemcpyAsync(d_a, desc_a, n * words * 8, cudaMemcpyHostToDevice, ctx.stream), "upload");
  CK(cudaMemcpyAsync(d_b, desc_b, n * words * 8, cudaMemcpyHostToDevice, ctx.stream), "upload");
  CK(cudaMemcpyAsync(d_ga, gray_a, n, cudaMemcpyHostToDevice, ctx.stream), "upload");
  CK(cudaMemcpyAsync(d_gb, gray_b, n, cudaMemcpyHostToDevice, ctx.stream), "upload");
  CK(cudaMemcpyAsync(d_ta, tex_a, n, cudaMemcpyHostToDevice, ctx.stream), "upload");
  CK(cudaMemcpyAsync(d_tb, tex_b, n, cudaMemcpyHostToDevice, ctx.stream), "upload");
  // Untouched pixels keep the caller's codes, as GpuSgm.match clones and copies them back.
  if (reasons) CK(cudaMemcpyAsync(d_reasons, reasons, n, cudaMemcpyHostToDevice, ctx.stream), "upload");
  if (boundary)
    CK(cudaMemcpyAsync(d_boundary, boundary, n, cudaMemcpyHostToDevice, ctx.stream), "upload");
  CK(cudaMemsetAsync(dstats, 0, sizeof(DeviceStats), ctx.stream), "stats clear");
  if (plan.streamed)
    status = run_view_streamed(ctx, p, d_a, d_b, d_ta, d_tb, d_ga, d_gb, w, h, reverse, d_out,
                               d_summary, d_reasons, d_boundary, dstats, plan.rows);
  else if (plan.compact) {
    const CompactOut out{d_out, d_summary, d_reasons, d_boundary, dstats};
    status = run_views_compact(ctx, p, plan.pool, 1, d_a, d_b, d_ta, d_tb, d_ga, d_gb, w, h,
                               reverse, &out);
  } else
    status = run_view_general(ctx, p, d_a, d_b, d_ta, d_tb, d_ga, d_gb, w, h, reverse, d_out,
                              d_summary, d_reasons, d_boundary, dstats);
  if (status) return status;
  CK(cudaMemcpyAsync(out_disp, d_out, n * 4, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  if (out_summary)
    CK(cudaMemcpyAsync(out_summary, d_summary, n * 24, cudaMemcpyDeviceToHost, ctx.stream),
       "readback");
  if (reasons) CK(cudaMemcpyAsync(reasons, d_reasons, n, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  if (boundary)
    CK(cudaMemcpyAsync(boundary, d_boundary, n, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  DeviceStats host{};
  CK(cudaMemcpyAsync(&host, dstats, sizeof host, cudaMemcpyDeviceToHost, ctx.stream), "readback");
  CK(cudaStreamSynchronize(ctx.stream), "GPU SGM execution");
  if (stats) copy_stats(host, stats, true);
  ctx.prof->collect();
  return CSGM_OK;
}

int run_match_host(Context& ctx, const csgm_params& p, const uint64_t* desc_a,
                   const uint64_t* desc_b, const uint8_t* gray_a, const uint8_t* gray_b,
                   const uint8_t* tex_a, const uint8_t* tex_b, int w, int h, int reverse,
                   float* out_disp, int32_t* out_summary, uint8_t* reasons, uint8_t* boundary,
                   csgm_stats* stats) {
  // Resident on the fused kernels when they apply and their workspace fits the budget, else
  // resident on the general ones, else streamed (as the session's mode allows).
  const bool summary = out_summary != nullptr;
  if (ctx.twin && ctx.sgm_mode != CSGM_SGM_STREAMED && ctx.sgm_mode != CSGM_SGM_COMPACT &&
      use_fused(p, h) &&
      match_fused_bytes(p, w, h, summary, ctx.tuning) <= ctx.ws->budget) {
    release_other_plans(*ctx.ws, false);
    return run_match_fused(ctx, p, desc_a, desc_b, gray_a, gray_b, tex_a, tex_b, w, h, reverse,
                           out_disp, out_summary, reasons, boundary, stats);
  }
  if (ctx.twin) ctx.twin->valid = false;
  const size_t fixed = match_fixed_bytes(p, w, h, summary);
  const size_t cells = (size_t)w * h * p.disparities;
  ViewPlan plan;
  int status = choose_plan(ctx, p, w, h, fixed, fixed + cells * (2 + p.aggregate_bytes), &plan,
                           true, 1);
  if (status) return status;
  return run_match_general(ctx, p, plan, desc_a, desc_b, gray_a, gray_b, tex_a, tex_b, w, h,
                           reverse, out_disp, out_summary, reasons, boundary, stats);
}

}  // namespace csgm
