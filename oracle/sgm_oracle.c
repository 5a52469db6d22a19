/*
 * sgm_oracle.c - CPU restatement of Collinea's stereo matcher.  TEST INFRASTRUCTURE ONLY: the
 * parity checker and the timed CPU baseline, never part of the product library.  Every function
 * cites the reference lines it follows (paths relative to the reference project root).
 *
 * Parity is pinned by the reference's known-answer tests and by an independent restatement of its
 * GPU kernels; no bit-exact output of the reference itself exists (see sgm_oracle.h).
 *
 * Build with -ffp-contract=off: Java never fuses a*b+c.
 */
#include "sgm_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define INVALID_COST 512 /* CensusSgm.java:11 */

static int g_threads = 1;

void oracle_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }
int oracle_get_threads(void) { return g_threads; }

int64_t oracle_java_round(double v) {
  /* Math.round(double) (Java 7+): floor(v + 1/2) evaluated exactly, i.e. ties toward +inf. */
  double f = floor(v);
  return (int64_t)(v - f >= 0.5 ? f + 1.0 : f);
}

static int java_round_float(float v) {
  /* Math.round(float): floor(v + 1/2) exactly; the double sum of a float and 0.5 is exact. */
  return (int)floor((double)v + 0.5);
}

int oracle_words(int wx, int wy) { return (wx * wy - 1 + 63) / 64; } /* CensusSgm.java:519-521 */

void oracle_census(const uint8_t* img, int w, int h, int wx, int wy, uint64_t* desc) {
  /* CensusSgm.java:540-555 with rx = wx/2, ry = wy/2 (the reference: rx = ry = window/2). */
  int rx = wx / 2, ry = wy / 2, words = oracle_words(wx, wy);
  long n = (long)w * h;
  memset(desc, 0, sizeof(uint64_t) * (size_t)words * (size_t)n);
  for (int y = ry; y < h - ry; y++)
    for (int x = rx; x < w - rx; x++) {
      long p = (long)y * w + x;
      int bit = 0, center = img[p];
      for (int yy = -ry; yy <= ry; yy++)
        for (int xx = -rx; xx <= rx; xx++) {
          if (xx == 0 && yy == 0) continue;
          if (img[(long)(y + yy) * w + x + xx] < center)
            desc[(long)(bit / 64) * n + p] |= 1ULL << (bit % 64);
          bit++;
        }
    }
}

void oracle_texture(const uint8_t* img, int w, int h, int wx, int wy, uint8_t* tex) {
  /* CensusSgm.java:523-538. */
  int rx = wx / 2, ry = wy / 2;
  memset(tex, 0, (size_t)w * h);
  for (int y = ry; y < h - ry; y++)
    for (int x = rx; x < w - rx; x++) {
      int low = 255, high = 0;
      for (int yy = -ry; yy <= ry; yy++)
        for (int xx = -rx; xx <= rx; xx++) {
          int v = img[(long)(y + yy) * w + x + xx];
          if (v < low) low = v;
          if (v > high) high = v;
        }
      tex[(long)y * w + x] = high - low >= 4;
    }
}

void oracle_color_census(const uint8_t* bgr, int w, int h, int wx, int wy, uint64_t* desc,
                         uint8_t* tex) {
  /* CensusSgm.java:302-332: Euclidean BGR distances, mean over the window including the centre. */
  int rx = wx / 2, ry = wy / 2, words = oracle_words(wx, wy), count = wx * wy - 1;
  long n = (long)w * h;
  double* distances = (double*)malloc(sizeof(double) * (size_t)count);
  memset(desc, 0, sizeof(uint64_t) * (size_t)words * (size_t)n);
  memset(tex, 0, (size_t)n);
  for (int y = ry; y < h - ry; y++)
    for (int x = rx; x < w - rx; x++) {
      long p = (long)y * w + x, center = 3 * p;
      int bit = 0;
      double total = 0, maximum = 0;
      for (int dy = -ry; dy <= ry; dy++)
        for (int dx = -rx; dx <= rx; dx++) {
          if (dx == 0 && dy == 0) continue;
          long q = 3 * ((long)(y + dy) * w + x + dx);
          double squared = 0;
          for (int c = 0; c < 3; c++) {
            int difference = (int)bgr[q + c] - (int)bgr[center + c];
            squared += (double)(difference * difference);
          }
          double distance = sqrt(squared);
          distances[bit++] = distance;
          total += distance;
          maximum = maximum > distance ? maximum : distance;
        }
      double mean = total / (double)(wx * wy);
      tex[p] = maximum >= 4;
      for (int k = 0; k < count; k++)
        if (distances[k] >= mean) desc[(long)(k / 64) * n + p] |= 1ULL << (k % 64);
    }
  free(distances);
}

int oracle_path_p2(int p1, int p2, int scale, const uint8_t* gray, int current, int previous) {
  /* StereoCost.java:44-48. */
  if (scale == 0) return p2;
  int difference = abs((int)gray[current] - (int)gray[previous]);
  int v = (int)((int64_t)p2 * scale / (scale + difference));
  return p1 + 1 > v ? p1 + 1 : v;
}

int oracle_cost(const csgm_params* prm, const uint64_t* a, const uint64_t* b, int words, int n,
                const uint8_t* ga, const uint8_t* gb, int p, int q, int w) {
  /* StereoCost.java:50-90. */
  int hamming = 0;
  for (int word = 0; word < words; word++)
    hamming += __builtin_popcountll(a[(long)word * n + p] ^ b[(long)word * n + q]);
  int mode = prm->cost_mode, bits = prm->window_x * prm->window_y - 1;
  if (mode == CSGM_COST_CENSUS) return hamming;
  if (mode == CSGM_COST_AD_CENSUS || mode == CSGM_COST_CENSUS_GRADIENT) {
    int difference, cap;
    if (mode == CSGM_COST_AD_CENSUS) {
      difference = abs((int)ga[p] - (int)gb[q]);
      cap = prm->ad_truncation;
    } else {
      int ax = (int)ga[p + 1] - (int)ga[p - 1], ay = (int)ga[p + w] - (int)ga[p - w];
      int bx = (int)gb[q + 1] - (int)gb[q - 1], by = (int)gb[q + w] - (int)gb[q - w];
      difference = abs(ax - bx) + abs(ay - by);
      cap = prm->gradient_truncation;
    }
    int weight = prm->census_weight_milli, denominator = 1000 * cap;
    int clipped = difference < cap ? difference : cap;
    return (weight * hamming * cap + (1000 - weight) * clipped * bits + denominator / 2) /
           denominator;
  }
  /* ZNCC: int64 window sums, FP64 correlation. */
  int rx = prm->window_x / 2, ry = prm->window_y / 2, count = prm->window_x * prm->window_y;
  int64_t sa = 0, sb = 0, saa = 0, sbb = 0, sab = 0;
  for (int dy = -ry; dy <= ry; dy++)
    for (int dx = -rx; dx <= rx; dx++) {
      int x = ga[p + dy * w + dx], y = gb[q + dy * w + dx];
      sa += x;
      sb += y;
      saa += x * x;
      sbb += y * y;
      sab += x * y;
    }
  int64_t va = count * saa - sa * sa, vb = count * sbb - sb * sb;
  if (va <= 0 || vb <= 0) return INVALID_COST;
  double correlation = (double)(count * sab - sa * sb) / sqrt((double)va * (double)vb);
  double clamped = correlation < 1 ? correlation : 1;
  clamped = clamped > -1 ? clamped : -1;
  return (int)oracle_java_round((1 - clamped) * .5 * bits);
}

/* Direction table: CensusSgm.java:421.  Entries 8..15 are the 16-path extension. */
static const int kPaths[16][2] = {{1, 0},  {-1, 0}, {0, 1},   {0, -1},  {1, 1},  {-1, 1},
                                  {1, -1}, {-1, -1}, {1, 2},  {2, 1},   {-1, 2}, {-2, 1},
                                  {1, -2}, {2, -1},  {-1, -2}, {-2, -1}};

typedef struct {
  uint16_t* u16;
  int32_t* i32;
} agg_store;

static inline int agg_get(const agg_store* s, long i) {
  /* PagedVolume.get (PagedVolume.java:160-166): shorts are read unsigned. */
  return s->u16 ? (int)s->u16[i] : s->i32[i];
}

static inline void agg_set(agg_store* s, long i, int v) {
  /* PagedVolume.set (PagedVolume.java:200-214): (short) truncation for 2-byte storage. */
  if (s->u16)
    s->u16[i] = (uint16_t)v;
  else
    s->i32[i] = v;
}

/* One path step for pixel (x, y): the body of CensusSgm.java:430-453. */
static void path_pixel(const csgm_params* prm, const uint16_t* costs, agg_store* agg,
                       const uint8_t* ta, const uint8_t* ga, int w, int h, int x, int y, int dx,
                       int dy, const int* prev_row, int* row, int p1, int p2) {
  int nd = prm->disparities;
  int px = x - dx, py = y - dy, dest = x * nd;
  long base = ((long)y * w + x) * nd;
  int has = px >= 0 && px < w && py >= 0 && py < h && ta[(long)py * w + px];
  int prev_base = has ? px * nd : 0, min_prev = INT_MAX;
  if (has)
    for (int k = 0; k < nd; k++)
      if (prev_row[prev_base + k] < min_prev) min_prev = prev_row[prev_base + k];
  int local_p2 = has ? oracle_path_p2(p1, p2, prm->edge_scale, ga, y * w + x, py * w + px) : p2;
  for (int k = 0; k < nd; k++) {
    int value = costs[base + k];
    if (has) {
      int t = prev_row[prev_base + k], c = min_prev + local_p2;
      if (c < t) t = c;
      if (k > 0 && prev_row[prev_base + k - 1] + p1 < t) t = prev_row[prev_base + k - 1] + p1;
      if (k + 1 < nd && prev_row[prev_base + k + 1] + p1 < t)
        t = prev_row[prev_base + k + 1] + p1;
      value += t - min_prev;
    }
    row[dest + k] = value;
    agg_set(agg, base + k, agg_get(agg, base + k) + value);
  }
}

int oracle_match(const csgm_params* prm, const uint64_t* a, const uint64_t* b, const uint8_t* ga,
                 const uint8_t* gb, const uint8_t* ta, const uint8_t* tb, int w, int h,
                 int reverse, float* out, csgm_stats* stats, uint8_t* reasons, uint8_t* boundary,
                 uint16_t* cost_out, uint32_t* agg_out, int32_t* summary_out) {
  int nd = prm->disparities, rx = prm->window_x / 2, ry = prm->window_y / 2;
  int words = oracle_words(prm->window_x, prm->window_y);
  long count = (long)w * h, cells = count * nd;
  if (nd < 1 || w < 1 || h < 1 || (prm->aggregate_bytes != 2 && prm->aggregate_bytes != 4) ||
      prm->directions < 1 || prm->directions > 16)
    return -1;
  uint16_t* costs = cost_out ? cost_out : (uint16_t*)malloc(sizeof(uint16_t) * (size_t)cells);
  agg_store agg = {0, 0};
  if (prm->aggregate_bytes == 2)
    agg.u16 = (uint16_t*)calloc((size_t)cells, sizeof(uint16_t));
  else
    agg.i32 = (int32_t*)calloc((size_t)cells, sizeof(int32_t));
  if (!costs || (!agg.u16 && !agg.i32)) {
    if (!cost_out) free(costs);
    free(agg.u16);
    free(agg.i32);
    return -1;
  }
  /* PagedVolume(..., 2, INVALID_COST, ...): every cost cell starts at 512 (CensusSgm.java:394-396). */
  for (long i = 0; i < cells; i++) costs[i] = INVALID_COST;
  /* Cost fill, CensusSgm.java:405-420. */
#pragma omp parallel for schedule(dynamic, 4) num_threads(g_threads)
  for (int y = ry; y < h - ry; y++) {
    for (int x = rx; x < w - rx; x++) {
      int p = y * w + x;
      long base = (long)p * nd;
      if (!ta[p]) continue;
      for (int k = 0; k < nd; k++) {
        int disparity = prm->min_disparity + k;
        long target = (long)x + (reverse ? (long)disparity : -(long)disparity);
        if (target < rx || target >= w - rx) continue;
        int q = y * w + (int)target;
        if (!tb[q]) continue;
        costs[base + k] = (uint16_t)oracle_cost(prm, a, b, words, (int)count, ga, gb, p, q, w);
      }
    }
  }
  /* Path aggregation, CensusSgm.java:421-459 (reference order; lines of one direction in
   * parallel only when the reference's order makes them independent). */
  int p1 = prm->p1, p2 = prm->p2;
  for (int path = 0; path < prm->directions; path++) {
    int dx = kPaths[path][0], dy = kPaths[path][1];
    int xStart = dx < 0 ? w - 1 : 0, xStep = dx < 0 ? -1 : 1;
    if (dy == 0) {
      /* Rows are independent for horizontal paths. */
#pragma omp parallel num_threads(g_threads)
      {
        int* row = (int*)malloc(sizeof(int) * (size_t)w * nd);
#pragma omp for schedule(dynamic, 8)
        for (int y = 0; y < h; y++)
          for (int xi = 0, x = xStart; xi < w; xi++, x += xStep)
            path_pixel(prm, costs, &agg, ta, ga, w, h, x, y, dx, dy, row, row, p1, p2);
        free(row);
      }
    } else {
      int ady = dy < 0 ? -dy : dy, ring = ady + 1;
      int yStart = dy < 0 ? h - 1 : 0, yStep = dy < 0 ? -1 : 1;
      int* rows = (int*)calloc((size_t)ring * w * nd, sizeof(int));
      for (int yi = 0, y = yStart; yi < h; yi++, y += yStep) {
        int* row = rows + (long)(yi % ring) * w * nd;
        const int* prev = rows + (long)((yi - ady + ring) % ring) * w * nd;
        /* Pixels of one row only read earlier rows: independent. */
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
        for (int xi = 0; xi < w; xi++) {
          int x = xStart + xi * xStep;
          path_pixel(prm, costs, &agg, ta, ga, w, h, x, y, dx, dy, prev, row, p1, p2);
        }
      }
      free(rows);
    }
  }
  /* Winner selection, CensusSgm.java:460-515. */
  for (long i = 0; i < count; i++) out[i] = NAN;
  if (summary_out)
    for (long p = 0; p < count; p++) {
      int32_t* s = summary_out + 6 * p;
      s[0] = -1;
      s[1] = INT_MAX;
      s[2] = INT_MAX;
      s[3] = -1;
      s[4] = -1;
      s[5] = (costs[p * nd] != INVALID_COST ? 1 : 0) | (costs[p * nd + nd - 1] != INVALID_COST ? 2 : 0);
    }
  int64_t full_n = 0, boundary_n = 0, lower_n = 0, upper_n = 0, ambiguous_n = 0, selected_n = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(g_threads) \
    reduction(+ : full_n, boundary_n, lower_n, upper_n, ambiguous_n, selected_n)
  for (int y = ry; y < h - ry; y++)
    for (int x = rx; x < w - rx; x++) {
      int pixel = y * w + x, best = -1, best_cost = INT_MAX;
      long base = (long)pixel * nd;
      for (int k = 0; k < nd; k++)
        if (costs[base + k] != INVALID_COST && agg_get(&agg, base + k) < best_cost) {
          best = k;
          best_cost = agg_get(&agg, base + k);
        }
      if (summary_out && best >= 0) {
        /* Winners record, GpuStereo.java:760-768. */
        int32_t* s = summary_out + 6 * (long)pixel;
        int second = INT_MAX;
        for (int k = 0; k < nd; k++)
          if (abs(k - best) > 1 && costs[base + k] != INVALID_COST) {
            int v = agg_get(&agg, base + k);
            if (v < second) second = v;
          }
        s[0] = best;
        s[1] = best_cost;
        s[2] = second;
        s[3] = best > 0 && costs[base + best - 1] != INVALID_COST ? agg_get(&agg, base + best - 1) : -1;
        s[4] = best + 1 < nd && costs[base + best + 1] != INVALID_COST ? agg_get(&agg, base + best + 1) : -1;
      }
      if (best < 0) continue;
      int full = costs[base] != INVALID_COST && costs[base + nd - 1] != INVALID_COST;
      if (full) {
        full_n++;
        if (boundary) boundary[pixel] = 4;
      }
      if (best == 0 || best == nd - 1) {
        boundary_n++;
        if (reasons) reasons[pixel] = 2;
        if (full && best == 0) {
          lower_n++;
          if (boundary) boundary[pixel] |= 1;
        }
        if (full && best == nd - 1) {
          upper_n++;
          if (boundary) boundary[pixel] |= 2;
        }
        continue;
      }
      int second = INT_MAX;
      for (int k = 0; k < nd; k++)
        if (abs(k - best) > 1 && costs[base + k] != INVALID_COST) {
          int v = agg_get(&agg, base + k);
          if (v < second) second = v;
        }
      /* second - bestCost <= Math.max(1, bestCost * uniqueness): int vs double comparison. */
      double slack = (double)best_cost * prm->uniqueness;
      if (slack < 1.0) slack = 1.0;
      if (second != INT_MAX && (double)(second - best_cost) <= slack) {
        ambiguous_n++;
        if (reasons) reasons[pixel] = 3;
        continue;
      }
      double offset = 0;
      if (best > 0 && best + 1 < nd && costs[base + best - 1] != INVALID_COST &&
          costs[base + best + 1] != INVALID_COST) {
        double before = agg_get(&agg, base + best - 1), after = agg_get(&agg, base + best + 1);
        double curvature = before + after - 2.0 * (double)best_cost;
        if (curvature > 0) {
          double o = .5 * (before - after) / curvature;
          o = o < .5 ? o : .5;
          offset = o > -.5 ? o : -.5;
        }
      }
      out[pixel] = (float)((double)(prm->min_disparity + best) + offset);
      selected_n++;
      if (reasons) reasons[pixel] = 0;
    }
  if (stats) {
    stats->full_interval_pixels += full_n;
    stats->boundary_rejected += boundary_n;
    stats->lower_boundary_rejected += lower_n;
    stats->upper_boundary_rejected += upper_n;
    stats->ambiguity_rejected += ambiguous_n;
    stats->selected += selected_n;
  }
  if (agg_out)
    for (long i = 0; i < cells; i++) agg_out[i] = (uint32_t)agg_get(&agg, i);
  if (!cost_out) free(costs);
  free(agg.u16);
  free(agg.i32);
  return 0;
}

void oracle_lr_check(const float* dl, const float* dr, int w, int h, int rx, int ry,
                     double threshold, float* checked, csgm_stats* stats, uint8_t* reasons) {
  /* CensusSgm.java:181-201. */
  long n = (long)w * h;
  for (long i = 0; i < n; i++) checked[i] = NAN;
  for (int y = ry; y < h - ry; y++)
    for (int x = rx; x < w - rx; x++) {
      long p = (long)y * w + x;
      if (!isfinite(dl[p])) continue;
      int xr = java_round_float((float)x - dl[p]);
      if (xr < rx || xr >= w - rx) {
        if (reasons) reasons[p] = 4;
        continue;
      }
      float other = dr[(long)y * w + xr];
      if (isfinite(other) && (double)fabsf(dl[p] - other) <= threshold)
        checked[p] = dl[p];
      else {
        if (stats) stats->lr_rejected++;
        if (reasons) reasons[p] = 4;
      }
    }
}

static int pair_impl(const csgm_params* prm, const uint8_t* left, const uint8_t* right,
                     const uint8_t* left_bgr, const uint8_t* right_bgr, const uint8_t* valid_l,
                     const uint8_t* valid_r, int w, int h, float* checked, float* dl, float* dr,
                     csgm_stats* stats, uint8_t* reasons, uint8_t* boundary);

int oracle_pair(const csgm_params* prm, const uint8_t* left, const uint8_t* right,
                const uint8_t* valid_l, const uint8_t* valid_r, int w, int h, float* checked,
                float* dl, float* dr, csgm_stats* stats, uint8_t* reasons, uint8_t* boundary) {
  return pair_impl(prm, left, right, 0, 0, valid_l, valid_r, w, h, checked, dl, dr, stats,
                   reasons, boundary);
}

int oracle_pair_color(const csgm_params* prm, const uint8_t* left, const uint8_t* right,
                      const uint8_t* left_bgr, const uint8_t* right_bgr, const uint8_t* valid_l,
                      const uint8_t* valid_r, int w, int h, float* checked, float* dl, float* dr,
                      csgm_stats* stats, uint8_t* reasons, uint8_t* boundary) {
  if (!left_bgr || !right_bgr) return -1; /* :110-115 */
  return pair_impl(prm, left, right, left_bgr, right_bgr, valid_l, valid_r, w, h, checked, dl, dr,
                   stats, reasons, boundary);
}

static int pair_impl(const csgm_params* prm, const uint8_t* left, const uint8_t* right,
                     const uint8_t* left_bgr, const uint8_t* right_bgr, const uint8_t* valid_l,
                     const uint8_t* valid_r, int w, int h, float* checked, float* dl, float* dr,
                     csgm_stats* stats, uint8_t* reasons, uint8_t* boundary) {
  /* CensusSgm.computeRecorded, CensusSgm.java:56-201; colour-distance descriptors and texture
   * (:108-120) when the BGR images are given, gray census otherwise (:121-126). */
  if (w < prm->window_x + 2 || h < prm->window_y + 2) return -1; /* :56-60 */
  long n = (long)w * h;
  int words = oracle_words(prm->window_x, prm->window_y);
  uint64_t* a = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)words * (size_t)n);
  uint64_t* b = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)words * (size_t)n);
  uint8_t* ta = (uint8_t*)malloc((size_t)n);
  uint8_t* tb = (uint8_t*)malloc((size_t)n);
  float* own_l = dl ? dl : (float*)malloc(sizeof(float) * (size_t)n);
  float* own_r = dr ? dr : (float*)malloc(sizeof(float) * (size_t)n);
  csgm_stats local;
  memset(&local, 0, sizeof local);
  if (reasons) memset(reasons, 1, (size_t)n); /* :104-106 */
  if (boundary) memset(boundary, 0, (size_t)n);
  if (left_bgr) {
    oracle_color_census(left_bgr, w, h, prm->window_x, prm->window_y, a, ta);  /* :116 */
    oracle_color_census(right_bgr, w, h, prm->window_x, prm->window_y, b, tb); /* :117 */
  } else {
    oracle_census(left, w, h, prm->window_x, prm->window_y, a);   /* :122 */
    oracle_census(right, w, h, prm->window_x, prm->window_y, b);  /* :123 */
    oracle_texture(left, w, h, prm->window_x, prm->window_y, ta);  /* :124 */
    oracle_texture(right, w, h, prm->window_x, prm->window_y, tb); /* :125 */
  }
  if (valid_l && valid_r) /* :127-134 */
    for (long i = 0; i < n; i++) {
      ta[i] = ta[i] && valid_l[i];
      tb[i] = tb[i] && valid_r[i];
    }
  int rc = oracle_match(prm, a, b, left, right, ta, tb, w, h, 0, own_l, &local, reasons, boundary,
                        0, 0, 0); /* :135-148 */
  csgm_stats discarded;
  memset(&discarded, 0, sizeof discarded);
  if (rc == 0)
    rc = oracle_match(prm, b, a, right, left, tb, ta, w, h, 1, own_r, &discarded, 0, 0, 0, 0,
                      0); /* :149-162 */
  if (rc == 0)
    oracle_lr_check(own_l, own_r, w, h, prm->window_x / 2, prm->window_y / 2, prm->lr_threshold,
                    checked, &local, reasons);
  if (stats) *stats = local;
  free(a);
  free(b);
  free(ta);
  free(tb);
  if (!dl) free(own_l);
  if (!dr) free(own_r);
  return rc;
}

/* ---- post-filters ---- */

static int cmp_float(const void* x, const void* y) {
  /* Arrays.sort(float[]) order for finite values. */
  float a = *(const float*)x, b = *(const float*)y;
  return a < b ? -1 : a > b ? 1 : 0;
}

void oracle_median_valid(const float* a, int w, int h, int window, float* out) {
  /* CensusSgm.java:557-573. */
  int r = window / 2;
  float* values = (float*)malloc(sizeof(float) * (size_t)window * window);
  memcpy(out, a, sizeof(float) * (size_t)w * h);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      if (!isfinite(a[(long)y * w + x])) continue;
      int n = 0;
      for (int yy = y - r < 0 ? 0 : y - r; yy <= (y + r < h - 1 ? y + r : h - 1); yy++)
        for (int xx = x - r < 0 ? 0 : x - r; xx <= (x + r < w - 1 ? x + r : w - 1); xx++) {
          float v = a[(long)yy * w + xx];
          if (isfinite(v)) values[n++] = v;
        }
      qsort(values, (size_t)n, sizeof(float), cmp_float);
      out[(long)y * w + x] = values[n / 2];
    }
  free(values);
}

void oracle_median_edge_preserving(const float* a, int w, int h, int window, double max_change,
                                   const uint8_t* gray, int edge_threshold, float* out) {
  /* CensusSgm.java:576-601. */
  int r = window / 2;
  float* values = (float*)malloc(sizeof(float) * (size_t)window * window);
  oracle_median_valid(a, w, h, window, out);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      float center = a[(long)y * w + x];
      if (!isfinite(center)) continue;
      if ((double)fabsf(out[(long)y * w + x] - center) < max_change) continue;
      int n = 0;
      for (int yy = y - r < 0 ? 0 : y - r; yy <= (y + r < h - 1 ? y + r : h - 1); yy++)
        for (int xx = x - r < 0 ? 0 : x - r; xx <= (x + r < w - 1 ? x + r : w - 1); xx++) {
          float value = a[(long)yy * w + xx];
          if (isfinite(value) && (double)fabsf(value - center) <= max_change &&
              (edge_threshold == 0 ||
               abs((int)gray[(long)yy * w + xx] - (int)gray[(long)y * w + x]) <= edge_threshold))
            values[n++] = value;
        }
      if (n > 0) {
        qsort(values, (size_t)n, sizeof(float), cmp_float);
        out[(long)y * w + x] = values[n / 2];
      }
    }
  free(values);
}

int oracle_reciprocal(const float* right, int w, int h, int x, int y, float disparity,
                      double tolerance, int border) {
  /* CensusSgm.java:604-612. */
  if (!isfinite(disparity) || y < border || y >= h - border) return 0;
  int xr = java_round_float((float)x - disparity);
  return xr >= border && xr < w - border && isfinite(right[(long)y * w + xr]) &&
         (double)fabsf(disparity - right[(long)y * w + xr]) <= tolerance;
}

double oracle_zncc(const uint8_t* a, const uint8_t* b, int w, int h, int x, int y,
                   double disparity, int r, int channels) {
  /* CensusSgm.java:615-644. */
  double target = x - disparity;
  int bx = (int)floor(target);
  double fraction = target - bx;
  if (x - r < 0 || x + r >= w || y - r < 0 || y + r >= h || bx - r < 0 || bx + r + 1 >= w)
    return -1;
  double covariance = 0, var_a = 0, var_b = 0;
  int n = (2 * r + 1) * (2 * r + 1);
  for (int channel = 0; channel < channels; channel++) {
    double sa = 0, sb = 0, saa = 0, sbb = 0, sab = 0;
    for (int dy = -r; dy <= r; dy++)
      for (int dx = -r; dx <= r; dx++) {
        long ai = ((long)(y + dy) * w + x + dx) * channels + channel;
        long bi = ((long)(y + dy) * w + bx + dx) * channels + channel;
        double av = a[ai], bv = (1 - fraction) * b[bi] + fraction * b[bi + channels];
        sa += av;
        sb += bv;
        saa += av * av;
        sbb += bv * bv;
        sab += av * bv;
      }
    covariance += sab - sa * sb / n;
    var_a += saa - sa * sa / n;
    var_b += sbb - sb * sb / n;
  }
  if (var_a < channels * n * 4 || var_b < channels * n * 4) return -1;
  double product = var_a * var_b;
  return covariance / sqrt(product > 1e-12 ? product : 1e-12);
}

int64_t oracle_remove_speckles(float* a, int w, int h, int minimum, double range,
                               int connectivity) {
  /* CensusSgm.java:651-681. */
  if (minimum <= 1) return 0;
  long n = (long)w * h;
  uint8_t* seen = (uint8_t*)calloc((size_t)n, 1);
  int* queue = (int*)malloc(sizeof(int) * (size_t)n);
  int64_t rejected = 0;
  for (long start = 0; start < n; start++) {
    if (seen[start] || !isfinite(a[start])) continue;
    long head = 0, tail = 0;
    queue[tail++] = (int)start;
    seen[start] = 1;
    while (head < tail) {
      int p = queue[head++], x = p % w, y = p / w;
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          if ((dx == 0 && dy == 0) || (connectivity == 4 && dx != 0 && dy != 0)) continue;
          int xx = x + dx, yy = y + dy;
          if (xx < 0 || xx >= w || yy < 0 || yy >= h) continue;
          int q = yy * w + xx;
          if (seen[q] || !isfinite(a[q]) || (double)fabsf(a[q] - a[p]) > range) continue;
          seen[q] = 1;
          queue[tail++] = q;
        }
    }
    if (tail < minimum)
      for (long i = 0; i < tail; i++) {
        a[queue[i]] = NAN;
        rejected++;
      }
  }
  free(seen);
  free(queue);
  return rejected;
}

static void postfilter_impl(const oracle_post* post, const uint8_t* left, const uint8_t* right,
                            const uint8_t* photo_left, const uint8_t* photo_right, int channels,
                            const float* dr, int w, int h, float* checked, csgm_stats* stats,
                            uint8_t* reasons);

void oracle_postfilter(const oracle_post* post, const uint8_t* left, const uint8_t* right,
                       const float* dr, int w, int h, float* checked, csgm_stats* stats,
                       uint8_t* reasons) {
  /* Gray census mode: the photometric gate on the gray images, one channel (:222-224). */
  postfilter_impl(post, left, right, left, right, 1, dr, w, h, checked, stats, reasons);
}

void oracle_postfilter_color(const oracle_post* post, const uint8_t* left, const uint8_t* right,
                             const uint8_t* left_bgr, const uint8_t* right_bgr, const float* dr,
                             int w, int h, float* checked, csgm_stats* stats, uint8_t* reasons) {
  /* --census-mode color-distance: the gate on the interleaved BGR images, three channels
   * (:222-224); the edge-preserving median still reads the gray left image (:208-214). */
  postfilter_impl(post, left, right, left_bgr, right_bgr, 3, dr, w, h, checked, stats, reasons);
}

static void postfilter_impl(const oracle_post* post, const uint8_t* left, const uint8_t* right,
                            const uint8_t* photo_left, const uint8_t* photo_right, int channels,
                            const float* dr, int w, int h, float* checked, csgm_stats* stats,
                            uint8_t* reasons) {
  /* CensusSgm.java:203-272. */
  (void)right;
  long n = (long)w * h;
  if (post->median > 1) { /* :203-214 */
    float* filtered = (float*)malloc(sizeof(float) * (size_t)n);
    if (post->median_classic)
      oracle_median_valid(checked, w, h, post->median, filtered);
    else
      oracle_median_edge_preserving(checked, w, h, post->median, post->median_max_change, left,
                                    post->median_edge_threshold, filtered);
    memcpy(checked, filtered, sizeof(float) * (size_t)n);
    free(filtered);
  }
  for (int y = 0; y < h; y++) /* :226-257 */
    for (int x = 0; x < w; x++) {
      long p = (long)y * w + x;
      float disparity = checked[p];
      if (!isfinite(disparity)) continue;
      if (!oracle_reciprocal(dr, w, h, x, y, disparity, post->lr_threshold, post->border)) {
        checked[p] = NAN;
        stats->post_median_lr_rejected++;
        if (reasons) reasons[p] = 5;
        continue;
      }
      double score = oracle_zncc(photo_left, photo_right, w, h, x, y, disparity,
                                 post->correlation_window / 2, channels);
      if (score < post->correlation) {
        checked[p] = NAN;
        stats->photometric_rejected++;
        if (reasons) reasons[p] = 6;
      }
    }
  float* before = reasons ? (float*)malloc(sizeof(float) * (size_t)n) : 0;
  if (before) memcpy(before, checked, sizeof(float) * (size_t)n);
  stats->speckle_rejected = oracle_remove_speckles(checked, w, h, post->speckle_size,
                                                   post->speckle_range,
                                                   post->speckle_connectivity); /* :264-271 */
  for (long i = 0; i < n; i++)
    if (isfinite(checked[i])) stats->valid++; /* :272 */
  if (before) {
    for (long i = 0; i < n; i++)
      if (isfinite(before[i]) && !isfinite(checked[i])) reasons[i] = 7; /* :274-275 */
    free(before);
  }
}
