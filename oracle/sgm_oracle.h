/*
 * sgm_oracle.h - CPU restatement of Collinea's stereo matcher.  TEST INFRASTRUCTURE ONLY.
 *
 * This library is the parity oracle for the CUDA matcher and the timed CPU baseline.  Only the
 * test suite, the smoke check and the benchmark's CPU-baseline leg load it; the product library
 * (libcollinea_sgm.so) never links or calls it.
 *
 * It restates, loop for loop, the reference's single-threaded CPU code:
 *   src/main/java/sgm/CensusSgm.java:45-280, 302-332, 344-555, 557-681
 *   src/main/java/sgm/StereoCost.java:7-90
 *   src/main/java/sgm/PagedVolume.java:160-214 (uint16 aggregate storage, unsigned reads)
 *   src/main/java/sgm/GpuStereo.java:631-687,758-769 (summary record and select arithmetic)
 * with Java's integer and IEEE-754 semantics (Math.round ties toward +inf, no FMA contraction).
 *
 * Parity pinning: the reference ships no golden disparity files and cannot run here (it needs a
 * JDK).  This restatement is pinned by the reference's own known-answer tests (the accuracy,
 * signed-range, constant-texture and penalty-unit checks of SelfTest, UpgradeStereoRegression and
 * MatchingCostBenchmark) on fixtures regenerated bit-exactly from java.util.Random, and by a
 * second, independent restatement of the reference's GPU kernels (tests/kernel_restatement.py)
 * that must agree with it bit for bit.  No bit-exact output of the reference itself is available.
 *
 * Extensions not in the reference (rectangular windows such as 9x7 and 16 paths) are pinned only
 * by reduction: with window_x == window_y and directions 4/8 the code is the reference's.
 */
#ifndef SGM_ORACLE_H
#define SGM_ORACLE_H

#include <stdint.h>

#include "../include/collinea_sgm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* java.lang.Math.round(double): closest long, ties toward positive infinity. */
int64_t oracle_java_round(double v);

/* Number of 64-bit census words: CensusSgm.words (CensusSgm.java:519-521), bits = wx*wy-1. */
int oracle_words(int wx, int wy);

/* CensusSgm.census (CensusSgm.java:540-555).  desc is [words][w*h], zero-filled here. */
void oracle_census(const uint8_t* img, int w, int h, int wx, int wy, uint64_t* desc);

/* CensusSgm.textureMask (CensusSgm.java:523-538).  tex[p] = 1 iff max-min over the window >= 4. */
void oracle_texture(const uint8_t* img, int w, int h, int wx, int wy, uint8_t* tex);

/* CensusSgm.colorCensus (CensusSgm.java:302-332): RGB-distance census from interleaved BGR. */
void oracle_color_census(const uint8_t* bgr, int w, int h, int wx, int wy, uint64_t* desc,
                         uint8_t* tex);

/* StereoCost.value (StereoCost.java:50-90) for matching pixel p and target pixel q. */
int oracle_cost(const csgm_params* prm, const uint64_t* a, const uint64_t* b, int words, int n,
                const uint8_t* ga, const uint8_t* gb, int p, int q, int w);

/* StereoCost.pathP2 (StereoCost.java:44-48). */
int oracle_path_p2(int p1, int p2, int scale, const uint8_t* gray, int current, int previous);

/*
 * CensusSgm.match CPU branch (CensusSgm.java:375-516) for one view.
 * Optional outputs (NULL to skip): cost_out uint16[n*D], agg_out uint32[n*D] (the aggregate as
 * stored: uint16 values widened, or int32), summary_out int32[6n] in the layout of the `winners`
 * kernel (GpuStereo.java:758-769).  reasons/boundary/stats follow the reference.  Returns 0, or
 * -1 for invalid arguments / allocation failure.
 */
int oracle_match(const csgm_params* prm, const uint64_t* a, const uint64_t* b, const uint8_t* ga,
                 const uint8_t* gb, const uint8_t* ta, const uint8_t* tb, int w, int h,
                 int reverse, float* out, csgm_stats* stats, uint8_t* reasons, uint8_t* boundary,
                 uint16_t* cost_out, uint32_t* agg_out, int32_t* summary_out);

/* Left-right check (CensusSgm.java:181-201).  checked must not alias dl. */
void oracle_lr_check(const float* dl, const float* dr, int w, int h, int rx, int ry,
                     double threshold, float* checked, csgm_stats* stats, uint8_t* reasons);

/*
 * CensusSgm.computeRecorded up to the LR check (CensusSgm.java:56-201): census and texture of
 * both images, AND with the optional validity masks, left and right views, LR check.
 * Stats are reset first.  dl/dr/reasons/boundary are optional.  Returns 0 or -1.
 */
int oracle_pair(const csgm_params* prm, const uint8_t* left, const uint8_t* right,
                const uint8_t* valid_l, const uint8_t* valid_r, int w, int h, float* checked,
                float* dl, float* dr, csgm_stats* stats, uint8_t* reasons, uint8_t* boundary);

/* ---- post-filters (CensusSgm.java:203-279, 557-681) ---- */

void oracle_median_valid(const float* a, int w, int h, int window, float* out);
void oracle_median_edge_preserving(const float* a, int w, int h, int window, double max_change,
                                   const uint8_t* gray, int edge_threshold, float* out);
int oracle_reciprocal(const float* right, int w, int h, int x, int y, float disparity,
                      double tolerance, int border);
double oracle_zncc(const uint8_t* a, const uint8_t* b, int w, int h, int x, int y,
                   double disparity, int r, int channels);
int64_t oracle_remove_speckles(float* a, int w, int h, int minimum, double range,
                               int connectivity);

/* Post-filter settings of computeRecorded (Options fields). */
typedef struct oracle_post {
  int32_t median;               /* Options.median (1 = off) */
  int32_t median_classic;       /* 1 = Options.medianMode "classic" */
  int32_t median_edge_threshold;
  int32_t correlation_window;   /* Options.correlationWindow */
  int32_t speckle_size;
  int32_t speckle_connectivity;
  int32_t border;               /* LR radius (census/2) */
  int32_t reserved;
  double median_max_change;
  double correlation;           /* Options.correlation */
  double lr_threshold;
  double speckle_range;
} oracle_post;

/* computeRecorded from the median to the final count (CensusSgm.java:203-272).  checked is
 * updated in place; reasons optional (5 post-median LR, 6 photometric, 7 speckle). */
void oracle_postfilter(const oracle_post* post, const uint8_t* left, const uint8_t* right,
                       const float* dr, int w, int h, float* checked, csgm_stats* stats,
                       uint8_t* reasons);

/* --census-mode color-distance: the pair from colour-distance descriptors and texture of the
 * interleaved BGR images (CensusSgm.java:108-120), the gray images for the costs and penalties. */
int oracle_pair_color(const csgm_params* prm, const uint8_t* left, const uint8_t* right,
                      const uint8_t* left_bgr, const uint8_t* right_bgr, const uint8_t* valid_l,
                      const uint8_t* valid_r, int w, int h, float* checked, float* dl, float* dr,
                      csgm_stats* stats, uint8_t* reasons, uint8_t* boundary);

/* The post-filters in colour-distance mode: the photometric gate over three channels of the BGR
 * images (CensusSgm.java:222-224,240-250). */
void oracle_postfilter_color(const oracle_post* post, const uint8_t* left, const uint8_t* right,
                             const uint8_t* left_bgr, const uint8_t* right_bgr, const float* dr,
                             int w, int h, float* checked, csgm_stats* stats, uint8_t* reasons);

/* Worker threads used by oracle_match/oracle_pair (1 = the reference's single thread). */
void oracle_set_threads(int threads);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
