// autotune.cu - launch shapes of the fused sweep per shape bucket, measured and cached on disk.
//
// The fused sweep has three launch knobs: rows per CTA (row warps; the chain of row blocks and how
// many of them wait for an SM), line warps per CTA (the anti-diagonal lines walked on the issue
// slots the row warps leave idle) and the line slack (how long a line a line warp may take for
// the pixels its block has left).  Disparity lanes per thread are fixed by the disparity count
// (D rounded up to 64, over 32 lanes).  csgm_autotune times the candidate shapes on a synthetic
// pair of the requested size and keeps the fastest per bucket: padded disparity count, paths, and
// width and height in half-octaves.  A session uses the entry of a call's bucket; calls without an
// entry use the built-in defaults.  Tuning never changes results, only the time.
//
// The reference has no counterpart: its OpenCL work-group size is a device property
// (src/main/java/sgm/GpuSgm.java:163-221).
//
// Cache file: one entry per line,
//   csgm-tuning v1 dp=128 paths=8 wb=21 hb=20 rows=12 line_warps=8 line_slack=100 ms=3.712
// rewritten whole (through a temporary file and a rename) when an entry is added.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "collinea_sgm.h"
#include "pipeline.h"
#include "stereo_fused.h"

namespace csgm {

int TuningTable::bucket(int v) { return (int)std::lround(2.0 * std::log2((double)std::max(v, 1))); }

static int padded(int D) { return (D + 63) / 64 * 64; }

const TuningTable::Entry* TuningTable::find(const csgm_params& p, int w, int h) const {
  const int dp = padded(p.disparities), wb = bucket(w), hb = bucket(h);
  for (const auto& e : entries)
    if (e.dp == dp && e.paths == p.directions && e.wb == wb && e.hb == hb) return &e;
  return nullptr;
}

void TuningTable::put(const csgm_params& p, int w, int h, const SweepTuning& t, double ms) {
  const int dp = padded(p.disparities), wb = bucket(w), hb = bucket(h);
  for (auto& e : entries)
    if (e.dp == dp && e.paths == p.directions && e.wb == wb && e.hb == hb) {
      e.t = t;
      e.ms = ms;
      return;
    }
  entries.push_back({dp, p.directions, wb, hb, t, ms});
}

namespace {

bool parse_line(const char* line, TuningTable::Entry* e) {
  int dp, paths, wb, hb, rows, lw, slack;
  double ms;
  if (sscanf(line,
             "csgm-tuning v1 dp=%d paths=%d wb=%d hb=%d rows=%d line_warps=%d line_slack=%d "
             "ms=%lf",
             &dp, &paths, &wb, &hb, &rows, &lw, &slack, &ms) != 8)
    return false;
  e->dp = dp;
  e->paths = paths;
  e->wb = wb;
  e->hb = hb;
  e->t.rows = rows;
  e->t.line_warps = lw;
  e->t.line_slack = slack;
  e->ms = ms;
  return true;
}

// Entries of a cache file (a missing file is an empty table); malformed lines are skipped.
std::vector<TuningTable::Entry> read_cache(const char* path) {
  std::vector<TuningTable::Entry> out;
  FILE* f = fopen(path, "r");
  if (!f) return out;
  char line[512];
  while (fgets(line, sizeof line, f)) {
    TuningTable::Entry e;
    if (parse_line(line, &e)) out.push_back(e);
  }
  fclose(f);
  return out;
}

int write_cache(const char* path, const std::vector<TuningTable::Entry>& entries) {
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = fopen(tmp.c_str(), "w");
  if (!f) return fail(CSGM_E_INVALID, "cannot write the tuning cache %s", tmp.c_str());
  for (const auto& e : entries)
    fprintf(f,
            "csgm-tuning v1 dp=%d paths=%d wb=%d hb=%d rows=%d line_warps=%d line_slack=%d "
            "ms=%.6f\n",
            e.dp, e.paths, e.wb, e.hb, e.t.rows, e.t.line_warps, e.t.line_slack, e.ms);
  const bool ok = fclose(f) == 0;
  if (!ok || rename(tmp.c_str(), path) != 0)
    return fail(CSGM_E_INVALID, "cannot replace the tuning cache %s", path);
  return CSGM_OK;
}

void to_abi(const SweepTuning& t, const csgm_params& p, double ms, csgm_tuning* out) {
  memset(out, 0, sizeof *out);
  out->rows_per_block = t.rows;
  out->line_warps = t.line_warps;
  out->line_slack = t.line_slack;
  out->disparity_lanes = padded(p.disparities) / 32;
  out->milliseconds = ms;
}

// A textured synthetic pair: uniform noise, the right image the left shifted by `shift` pixels
// with fresh noise where it enters.  The sweep's time does not depend on the content beyond the
// share of textured pixels, which noise keeps near one as real imagery does.
__device__ __forceinline__ uint32_t mix(uint32_t v) {
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}

__global__ void synthetic_pair_kernel(uint8_t* left, uint8_t* right, int w, int h, int shift) {
  const int64_t n = (int64_t)w * h;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % w);
    left[p] = (uint8_t)(mix((uint32_t)p) >> 24);
    right[p] = (uint8_t)(x + shift < w ? mix((uint32_t)(p + shift)) >> 24
                                       : mix((uint32_t)p ^ 0x9e3779b9u) >> 24);
  }
}

}  // namespace
}  // namespace csgm

using namespace csgm;

extern "C" {

int csgm_tuning_cache_lookup(const char* cache_path, const csgm_params* p, int32_t w, int32_t h,
                             csgm_tuning* out) {
  if (!cache_path || !p || !out) return fail(CSGM_E_INVALID, "NULL argument");
  TuningTable table;
  table.entries = read_cache(cache_path);
  memset(out, 0, sizeof *out);
  if (const TuningTable::Entry* e = table.find(*p, w, h)) to_abi(e->t, *p, e->ms, out);
  return CSGM_OK;
}

int csgm_session_load_tuning(csgm_session* s, const char* cache_path) {
  if (!s || !cache_path) return fail(CSGM_E_INVALID, "NULL argument");
  std::vector<TuningTable::Entry> entries = read_cache(cache_path);
  std::lock_guard<std::mutex> guard(s->lock);
  for (const auto& e : entries) {
    bool replaced = false;
    for (auto& mine : s->tuning.entries)
      if (mine.dp == e.dp && mine.paths == e.paths && mine.wb == e.wb && mine.hb == e.hb) {
        mine = e;
        replaced = true;
      }
    if (!replaced) s->tuning.entries.push_back(e);
  }
  return CSGM_OK;
}

int csgm_session_set_tuning(csgm_session* s, const csgm_tuning* t) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  std::lock_guard<std::mutex> guard(s->lock);
  s->tuning_forced = t != nullptr;
  if (t) {
    s->forced_tuning.rows = t->rows_per_block;
    s->forced_tuning.line_warps = t->line_warps;
    s->forced_tuning.line_slack = t->line_slack;
  }
  return CSGM_OK;
}

int csgm_tuning_get(csgm_session* s, const csgm_params* p, int32_t w, int32_t h,
                    csgm_tuning* out) {
  if (!s || !out) return fail(CSGM_E_INVALID, "NULL argument");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  Context ctx{s->stream, s->sm_count, &s->workspace, &s->profiler, &s->profile};
  session_settings(ctx, s, *p, w, h);
  const TuningTable::Entry* e = s->tuning_forced ? nullptr : s->tuning.find(*p, w, h);
  to_abi(resolve_tuning(*p, ctx.tuning), *p, e ? e->ms : 0.0, out);
  return CSGM_OK;
}

int csgm_autotune(csgm_session* s, const csgm_params* p, int32_t w, int32_t h,
                  const char* cache_path, csgm_tuning* best) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  int rc = validate_params(p, w, h);
  if (rc) return rc;
  csgm_params q = *p;
  q.flags = 0;
  if (!fused_supported(q) || h > 65535)
    return fail(CSGM_E_UNSUPPORTED, "the fused kernels do not run these parameters: no tuning");
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  const size_t n = (size_t)w * h;
  int status = CSGM_OK;
  uint8_t* left = (uint8_t*)s->workspace.get(kImgL, n, &status);
  uint8_t* right = left ? (uint8_t*)s->workspace.get(kImgR, n, &status) : nullptr;
  float* checked = right ? (float*)s->workspace.get(kChecked, n * 4, &status) : nullptr;
  if (!checked) return status;
  const int64_t blocks = std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)s->sm_count * 16);
  synthetic_pair_kernel<<<(int)blocks, 256, 0, s->stream>>>(left, right, w, h,
                                                            std::max(1, q.disparities / 3));
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "synthetic pair");

  // Candidate shapes, each as the resolver would run it (duplicates dropped).
  const int regs = padded(q.disparities) / 32;
  std::vector<SweepTuning> candidates;
  for (int rows : {4, 8, 12}) {
    if (rows == 12 && regs != 4) continue;
    for (int lw : {0, 4, 8}) {
      if (q.directions < 8 && lw) continue;
      SweepTuning want;
      want.rows = rows;
      want.line_warps = lw;
      want.line_slack = 100;
      const SweepTuning t = resolve_tuning(q, want);
      bool seen = false;
      for (const auto& c : candidates)
        seen |= c.rows == t.rows && c.line_warps == t.line_warps && c.line_slack == t.line_slack;
      if (!seen) candidates.push_back(t);
    }
  }
  cudaEvent_t start, stop;
  if (cudaEventCreate(&start) != cudaSuccess || cudaEventCreate(&stop) != cudaSuccess)
    return cuda_fail(cudaGetLastError(), "event creation");
  SweepTuning chosen;
  double chosen_ms = 1e30;
  for (const auto& t : candidates) {
    double fastest = 1e30;
    for (int run = 0; run < 3 && status == CSGM_OK; run++) {  // the first run warms up
      Context ctx{s->stream, s->sm_count, &s->workspace, &s->profiler, &s->profile};
      session_settings(ctx, s, q, w, h);
      ctx.tuning = t;
      cudaEventRecord(start, s->stream);
      status = run_pair_device(ctx, q, left, right, nullptr, nullptr, w, h, checked, nullptr,
                               nullptr, nullptr, nullptr, nullptr, true);
      cudaEventRecord(stop, s->stream);
      cudaEventSynchronize(stop);
      float ms = 0;
      cudaEventElapsedTime(&ms, start, stop);
      if (run > 0) fastest = std::min(fastest, (double)ms);
    }
    if (status != CSGM_OK) break;
    if (fastest < chosen_ms) {
      chosen_ms = fastest;
      chosen = t;
    }
  }
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  if (status != CSGM_OK) return status;
  s->tuning.put(q, w, h, chosen, chosen_ms);
  if (best) to_abi(chosen, q, chosen_ms, best);
  if (cache_path) {
    TuningTable file;
    file.entries = read_cache(cache_path);
    file.put(q, w, h, chosen, chosen_ms);
    return write_cache(cache_path, file.entries);
  }
  return CSGM_OK;
}

}  // extern "C"
