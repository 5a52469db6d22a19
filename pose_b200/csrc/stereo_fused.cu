// stereo_fused.cu - fast path of the matcher for D <= 256, 4/8 paths, uint16 aggregate.
//
// Reference semantics: cost CensusSgm.java:405-420 + StereoCost.java:50-90; aggregation
// CensusSgm.java:421-459; selection CensusSgm.java:460-515.  Results are bit-identical to the
// general kernels (stereo_kernels.cu) and to the CPU reference.
//
// Design (B200):
//  * cost_pair_kernel writes both views' cost volumes once, as uint8 [H][W][Dp] with
//    Dp = D rounded up to 64 and 0x80 marking the reference's invalid cost 512.
//  * sweep_kernel runs FOUR wavefront streams in one launch: left-down, left-up, right-down,
//    right-up.  A "down" stream processes rows top to bottom, pixels left to right, and owns the
//    paths whose predecessor lies above or to the left: (1,0), (0,1), (1,1), (-1,1).  An "up"
//    stream is the same code on the image mirrored in x and y and owns the four opposite paths.
//  * One CTA = R consecutive rows, one warp per row; warp w processes pixel x at step x + 2w.
//    The (0,1), (1,1), (-1,1) path states of a row reach the next row through a 4-slot ring in
//    shared memory; the (1,0) state stays in registers.  The last row of a CTA also writes a
//    global carry row that the next CTA of the stream reads (release/acquire progress counter).
//  * Meet in the middle: for rows above `split` the down stream runs first and stores its partial
//    aggregate (uint16); the up stream adds its four paths and selects the winner in registers.
//    Below `split` the roles swap.  The partial aggregate crosses HBM once each way.
//  * Disparities live in registers as packed uint16 pairs (REGS registers per lane per path);
//    the min-plus step uses the DPX instructions __vimin3_u16x2 / __viaddmin_u16x2 and the
//    warp-wide minimum __reduce_min_sync.
//  * Cost, partial-aggregate and carry slices are staged in shared memory by cp.async.bulk with
//    mbarrier completion (no multicast).  Every wait is bounded; a wait that runs out sets an
//    error flag that the host turns into CSGM_E_TIMEOUT.
//  * CTAs take tickets in launch order; a CTA only waits on lower tickets, so the schedule cannot
//    deadlock even when not every CTA is resident.
#include <climits>

#include "stereo_fused.h"
#include "stereo_kernels.h"

namespace csgm {

namespace {

constexpr int kRows = 8;      // rows (warps) per CTA
constexpr int kRing = 4;      // ring slots per row
constexpr int kRecords = 32;  // selections buffered per warp before the scalar select

__host__ __device__ inline int padded_d(int D) { return (D + 63) / 64 * 64; }

// ---------------------------------------------------------------------------------------------
// PTX helpers: shared-memory mbarriers and bulk copies (single CTA, no multicast).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// PRMT in the generic mode: selector nibbles with bit 3 set replicate the selected byte's sign.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

// Bounded waits.  The whole warp waits; `error` short-circuits every later wait.
__device__ __forceinline__ void wait_bar(uint64_t* bar, uint32_t parity, int* error,
                                         long long limit) {
  long long start = clock64();
  while (!mbar_test(bar, parity)) {
    if (*(volatile int*)error) return;
    if (clock64() - start > limit) {
      atomicExch(error, 1);
      return;
    }
  }
}

__device__ __forceinline__ void wait_flag(const int* flag, int target, int* error,
                                          long long limit) {
  long long start = clock64();
  while (*(volatile const int*)flag < target) {
    if (*(volatile int*)error) return;
    if (clock64() - start > limit) {
      atomicExch(error, 2);
      return;
    }
    __nanosleep(64);
  }
  __threadfence();  // acquire: later reads see what the producer wrote before its release
}

// ---------------------------------------------------------------------------------------------
// Cost volumes of both views (uint8, 0x80 = invalid).  One warp per pixel of one view; lanes own
// contiguous groups of Dp/32 disparities.
struct CostPairArgs {
  CostArgs view[2];  // per view: a = matching image, b = target image, reverse 0/1
  uint8_t* out[2];
  int Dp;
};

__global__ void cost_pair_kernel(CostPairArgs a) {
  const CostArgs& c = a.view[blockIdx.y];
  uint8_t* out = a.out[blockIdx.y];
  int w = c.w, h = c.h, D = c.D, Dp = a.Dp;
  int64_t n = (int64_t)w * h;
  int rx = c.wx / 2, ry = c.wy / 2;
  int lane = threadIdx.x & 31;
  int per = Dp / 32;  // 2..8 cells per lane
  int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = warp; p < n; p += warps) {
    int x = (int)(p % w), y = (int)(p / w);
    bool inside = x >= rx && x < w - rx && y >= ry && y < h - ry && c.tex_a[p];
    uint64_t packed = 0;
    for (int j = 0; j < per; j++) {
      int k = lane * per + j;
      int value = 0x80;
      if (inside && k < D) {
        long long disparity = (long long)c.min_disparity + k;
        long long target = (long long)x + (c.reverse ? disparity : -disparity);
        if (target >= rx && target < w - rx) {
          int64_t q = (int64_t)y * w + target;
          if (c.tex_b[q]) {
            int v = cell_cost(c, p, q, n);
            value = v == kInvalidCost ? 0x80 : v;
          }
        }
      }
      packed |= (uint64_t)value << (8 * j);
    }
    uint8_t* dst = out + p * Dp + lane * per;
    if (per == 8)
      *(uint64_t*)dst = packed;
    else if (per == 4)
      *(uint32_t*)dst = (uint32_t)packed;
    else if (per == 2)
      *(uint16_t*)dst = (uint16_t)packed;
    else
      for (int j = 0; j < per; j++) dst[j] = (uint8_t)(packed >> (8 * j));
  }
}

// ---------------------------------------------------------------------------------------------
struct SweepArgs {
  const uint8_t* cost[2];  // [H][W][Dp] per view
  const uint8_t* gray[2];  // matching-view image per view
  const uint8_t* tex[2];   // matching-view texture per view
  uint16_t* sum[2];        // partial aggregate [H][W][Dp] per view
  float* disp[2];
  uint8_t* carry;     // [4][nb][W][slot] bytes
  int* progress;      // [4][nb]
  int* row_done;      // [2][H]
  int* ticket;
  int* error;
  uint8_t* reasons;   // left view only
  uint8_t* boundary;  // left view only
  DeviceStats* stats; // left view only
  int W, H, D, Dp, nb, Hp, split, p1, p2, edge_scale, min_disparity, rx, ry, chunk;
  double uniqueness;
  long long timeout;
};

// Shared-memory layout (byte offsets), identical on host and device.
struct SweepLayout {
  int slot;       // one ring slot: 3 paths x Dp uint16 + 4 uint32 minima
  int lut, bars, cost, sum, ring, carry, rec, total;
  __host__ __device__ SweepLayout(int Dp, int K) {
    slot = 3 * Dp * 2 + 16;
    lut = 0;                                     // 256 x uint32
    bars = lut + 256 * 4;                        // kRows x 4 + 3 mbarriers
    cost = bars + (kRows * 4 + 3) * 8;
    cost = (cost + 127) / 128 * 128;
    sum = cost + kRows * 2 * K * Dp;             // cost chunks, double-buffered per warp
    ring = sum + kRows * 2 * K * Dp * 2;         // partial-aggregate chunks
    carry = ring + kRows * kRing * slot;         // row-to-row ring
    rec = carry + 3 * K * slot;                  // carry chunks of the row above the CTA
    total = rec + kRows * kRecords * 6 * 4;      // winners records
  }
};

// The (P2' - P1) table of StereoCost.pathP2 for every |gray difference|, replicated to u16x2.
__device__ __forceinline__ uint32_t lut_value(int p1, int p2, int scale, int diff) {
  int v = scale == 0 ? p2 : max(p1 + 1, (int)(((long long)p2 * scale) / (scale + diff)));
  uint32_t d = (uint32_t)(v - p1);
  return d | (d << 16);
}

template <int REGS>
struct PathState {
  uint32_t v[REGS];
  uint32_t m;  // replicated minimum
};

// One min-plus step of one path for the lane's 2*REGS disparities.
//   prev  predecessor path costs (zeros = no predecessor: the result is then the cost itself)
//   q     min(prev) + P2' - P1 (replicated), c the pixel's costs, p1 = P1 replicated.
template <int REGS>
__device__ __forceinline__ void path_step(const PathState<REGS>& prev, uint32_t q, uint32_t p1x2,
                                          const uint32_t (&c)[REGS], const uint32_t (&pad)[REGS],
                                          int lane, PathState<REGS>& out) {
  uint32_t below = __shfl_up_sync(0xffffffffu, prev.v[REGS - 1], 1);
  uint32_t above = __shfl_down_sync(0xffffffffu, prev.v[0], 1);
  if (lane == 0) below = 0xffffffffu;
  if (lane == 31) above = 0xffffffffu;
  uint32_t e[REGS];
#pragma unroll
  for (int j = 0; j < REGS; j++) e[j] = __byte_perm(prev.v[j], j + 1 < REGS ? prev.v[j + 1] : above, 0x5432);
  uint32_t dn0 = __byte_perm(below, prev.v[0], 0x5432);
  uint32_t mm = 0xffffffffu;
#pragma unroll
  for (int j = 0; j < REGS; j++) {
    uint32_t dn = j == 0 ? dn0 : e[j - 1];
    uint32_t m3 = __vimin3_u16x2(dn, e[j], q);
    uint32_t t = __viaddmin_u16x2(m3, p1x2, prev.v[j]);
    uint32_t L = (t + c[j] - prev.m) | pad[j];
    out.v[j] = L;
    mm = __vminu2(mm, L);
  }
  mm = __vminu2(mm, __byte_perm(mm, 0, 0x1032));
  out.m = __reduce_min_sync(0xffffffffu, mm);
}

template <int REGS>
__device__ __forceinline__ void load_state(const uint8_t* slot, int path, int Dp, int lane,
                                           PathState<REGS>& s) {
  const uint32_t* src = (const uint32_t*)(slot + 2 * (path * Dp + lane * 2 * REGS));
  if (REGS == 4) {
    uint4 v = *(const uint4*)src;
    s.v[0] = v.x; s.v[REGS > 1 ? 1 : 0] = v.y; s.v[REGS > 2 ? 2 : 0] = v.z; s.v[REGS > 3 ? 3 : 0] = v.w;
  } else if (REGS == 2) {
    uint2 v = *(const uint2*)src;
    s.v[0] = v.x; s.v[REGS > 1 ? 1 : 0] = v.y;
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j++) s.v[j] = src[j];
  }
  s.m = ((const uint32_t*)(slot + 6 * Dp))[path];
}

template <int REGS>
__device__ __forceinline__ void store_state(uint8_t* slot, int path, int Dp, int lane,
                                            const PathState<REGS>& s) {
  uint32_t* dst = (uint32_t*)(slot + 2 * (path * Dp + lane * 2 * REGS));
  if (REGS == 4) {
    *(uint4*)dst = make_uint4(s.v[0], s.v[REGS > 1 ? 1 : 0], s.v[REGS > 2 ? 2 : 0], s.v[REGS > 3 ? 3 : 0]);
  } else if (REGS == 2) {
    *(uint2*)dst = make_uint2(s.v[0], s.v[REGS > 1 ? 1 : 0]);
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j++) dst[j] = s.v[j];
  }
  if (lane == 0) ((uint32_t*)(slot + 6 * Dp))[path] = s.m;
}

template <int REGS>
__device__ __forceinline__ void zero_state(PathState<REGS>& s) {
#pragma unroll
  for (int j = 0; j < REGS; j++) s.v[j] = 0;
  s.m = 0;
}

// Scalar selection of one buffered winners record (CensusSgm.java:471-513 semantics).
__device__ void select_record(const SweepArgs& a, int view, const int32_t* r, int64_t p,
                              unsigned (&counts)[6]) {
  int best = r[0], value = r[1], second = r[2], before = r[3], after = r[4], flags = r[5];
  float out = __int_as_float(0x7fc00000);
  uint8_t* reasons = view == 0 ? a.reasons : nullptr;
  uint8_t* boundary = view == 0 ? a.boundary : nullptr;
  if (best >= 0) {
    bool full = flags == 3;
    bool done = false;
    if (full) {
      counts[1]++;
      if (boundary) boundary[p] = 4;
    }
    if (best == 0 || best == a.D - 1) {
      counts[2]++;
      if (reasons) reasons[p] = 2;
      if (full && best == 0) {
        counts[0]++;
        if (boundary) boundary[p] |= 1;
      }
      if (full && best == a.D - 1) {
        counts[3]++;
        if (boundary) boundary[p] |= 2;
      }
      done = true;
    }
    if (!done && second != INT_MAX) {
      double slack = fmax(1.0, __dmul_rn((double)value, a.uniqueness));
      if ((double)(second - value) <= slack) {
        counts[4]++;
        if (reasons) reasons[p] = 3;
        done = true;
      }
    }
    if (!done) {
      double offset = 0;
      if (before >= 0 && after >= 0) {
        double curvature =
            __dsub_rn(__dadd_rn((double)before, (double)after), __dmul_rn(2.0, (double)value));
        if (curvature > 0) {
          double o =
              __ddiv_rn(__dmul_rn(0.5, __dsub_rn((double)before, (double)after)), curvature);
          offset = fmax(-0.5, fmin(0.5, o));
        }
      }
      out = __double2float_rn(__dadd_rn((double)(a.min_disparity + best), offset));
      counts[5]++;
      if (reasons) reasons[p] = 0;
    }
  }
  a.disp[view][p] = out;
}

template <int REGS, int NPATH>
__global__ void __launch_bounds__(kRows * 32) sweep_kernel(const SweepArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  const int K = a.chunk;
  const SweepLayout L(a.Dp, K);
  uint32_t* lut = (uint32_t*)(smem + L.lut);
  uint64_t* bars = (uint64_t*)(smem + L.bars);
  __shared__ int s_ticket;

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int W = a.W, H = a.H, Dp = a.Dp;
  if (threadIdx.x == 0) s_ticket = atomicAdd(a.ticket, 1);
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = lut_value(a.p1, a.p2, a.edge_scale, i);
  if (lane == 0) {
    for (int i = 0; i < 4; i++) mbar_init(&bars[w * 4 + i], 1);
    if (w == 0)
      for (int i = 0; i < 3; i++) mbar_init(&bars[kRows * 4 + i], 1);
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();

  const int ticket = s_ticket;
  const int stream = ticket & 3, b = ticket >> 2;
  const int view = stream >> 1;
  const bool mirror = (stream & 1) != 0;
  const int yp = b * kRows + w;                 // row in stream coordinates
  const int y = mirror ? a.Hp - 1 - yp : yp;    // image row
  const bool exists = y >= 0 && y < H;
  const bool first = exists && ((y < a.split) != mirror);
  const bool finalize = exists && !first;
  const bool has_next = b + 1 < a.nb;
  const int ya = mirror ? y + 1 : y - 1;        // image row of the row above (stream order)
  const bool above_exists = yp >= 1 && ya >= 0 && ya < H;

  const uint8_t* cost = a.cost[view];
  const uint8_t* gray = a.gray[view];
  const uint8_t* tex = a.tex[view];
  uint16_t* sum = a.sum[view];
  const int nchunks = (W + K - 1) / K;
  uint8_t* cost_buf = smem + L.cost + w * 2 * K * Dp;
  uint16_t* sum_buf = (uint16_t*)(smem + L.sum + w * 2 * K * Dp * 2);
  uint8_t* ring = smem + L.ring + w * kRing * L.slot;
  const uint8_t* ring_above = smem + L.ring + (w - 1) * kRing * L.slot;
  uint8_t* carry_buf = smem + L.carry;
  int32_t* rec = (int32_t*)(smem + L.rec) + w * kRecords * 6;
  uint64_t* cost_bar = &bars[w * 4];
  uint64_t* sum_bar = &bars[w * 4 + 2];
  uint64_t* carry_bar = &bars[kRows * 4];
  const long long limit = a.timeout;

  // Stream x' -> image column, and the contiguous memory range of a chunk.
  auto col = [&](int xs) { return mirror ? W - 1 - xs : xs; };
  auto chunk_first_col = [&](int c) {
    int lo = c * K, hi = min(W, lo + K);
    return mirror ? W - hi : lo;
  };
  auto chunk_pixels = [&](int c) { return min(W, c * K + K) - c * K; };
  auto chunk_slot = [&](int xs) {  // position of stream pixel xs inside its chunk buffer
    int c = xs / K;
    return mirror ? (min(W, c * K + K) - 1 - xs) : xs - c * K;
  };
  int issued_cost = 0, issued_sum = 0, issued_carry = 0;  // chunks issued (uniform per warp)
  auto issue_cost = [&](int c) {
    issued_cost = c + 1;
    if (lane == 0) {
      fence_proxy_async_shared();
      bulk_load(cost_buf + (c & 1) * K * Dp, cost + ((int64_t)y * W + chunk_first_col(c)) * Dp,
                (uint32_t)(chunk_pixels(c) * Dp), &cost_bar[c & 1]);
    }
  };
  auto issue_sum = [&](int c) {
    issued_sum = c + 1;
    if (lane == 0) {
      fence_proxy_async_shared();
      bulk_load(sum_buf + (c & 1) * K * Dp, sum + ((int64_t)y * W + chunk_first_col(c)) * Dp,
                (uint32_t)(chunk_pixels(c) * Dp * 2), &sum_bar[c & 1]);
    }
  };
  const int up_index = (stream * a.nb + b - 1);  // carry row written by the previous CTA
  auto issue_carry = [&](int c) {
    issued_carry = c + 1;
    if (lane == 0) {
      int need = min(W, c * K + K);
      wait_flag(&a.progress[up_index], need, a.error, limit);
      fence_proxy_async_global();
      fence_proxy_async_shared();
      bulk_load(carry_buf + (c % 3) * K * L.slot,
                a.carry + ((int64_t)up_index * W + c * K) * L.slot,
                (uint32_t)(chunk_pixels(c) * L.slot), &carry_bar[c % 3]);
    }
  };

  // Per-lane padding mask: disparities >= D stay at 0xffff so they never win a minimum.
  uint32_t pad[REGS];
#pragma unroll
  for (int j = 0; j < REGS; j++) {
    int k = lane * 2 * REGS + 2 * j;
    pad[j] = (k >= a.D ? 0xffffu : 0u) | (k + 1 >= a.D ? 0xffff0000u : 0u);
  }
  const uint32_t p1x2 = (uint32_t)a.p1 | ((uint32_t)a.p1 << 16);
  const bool use_carry = w == 0 && b > 0;

  // Prologue.
  if (exists) {
    issue_cost(0);
    if (finalize) {
      if (lane == 0) {
        wait_flag(&a.row_done[view * H + y], 1, a.error, limit);
        fence_proxy_async_global();
      }
      __syncwarp();
      issue_sum(0);
    }
  }
  if (use_carry) issue_carry(0);

  PathState<REGS> horiz;  // (1,0) path in stream coordinates
  zero_state(horiz);
  int g_left = 0, ga_l = 0, ga_c = 0, ga_r = 0;
  if (above_exists) ga_r = __ldg(&gray[(int64_t)ya * W + col(0)]);
  unsigned counts[6] = {0, 0, 0, 0, 0, 0};
  const bool region_row = y >= a.ry && y < H - a.ry;

  const int steps = W + 2 * (kRows - 1);
  for (int step = 0; step < steps; step++) {
    const int xs = step - 2 * w;
    if (xs >= 0 && xs < W) {
      uint8_t* out_slot = ring + (xs & (kRing - 1)) * L.slot;
      // Carry chunks of the row above this CTA.
      if (use_carry) {
        int c = xs / K;
        if (xs % K == 0) {
          if (xs == 0) wait_bar(&carry_bar[0], 0, a.error, limit);
          if (c + 1 < nchunks) issue_carry(c + 1);
        }
        if (xs % K == K - 1 && c + 1 < nchunks)
          wait_bar(&carry_bar[(c + 1) % 3], ((c + 1) / 3) & 1, a.error, limit);
      }
      if (exists) {
        const int c = xs / K;
        if (xs % K == 0) {
          wait_bar(&cost_bar[c & 1], (c >> 1) & 1, a.error, limit);
          if (finalize) wait_bar(&sum_bar[c & 1], (c >> 1) & 1, a.error, limit);
          __syncwarp();
          if (c + 1 < nchunks) {
            issue_cost(c + 1);
            if (finalize) issue_sum(c + 1);
          }
        }
        const int slot = chunk_slot(xs);
        const int x = col(xs);
        const int64_t p = (int64_t)y * W + x;
        // Costs: 2*REGS bytes per lane -> REGS packed uint16 pairs, 0x80 -> 512.
        const uint8_t* cb = cost_buf + (c & 1) * K * Dp + slot * Dp + lane * 2 * REGS;
        uint32_t cst[REGS];
        if (REGS % 2 == 0) {
#pragma unroll
          for (int j = 0; j < REGS; j++) {
            uint32_t word = ((const uint32_t*)cb)[j / 2];
            uint32_t sel = (j & 1) ? 0xb3a2u : 0x9180u;  // bytes 2j,2j+1, sign-replicated high bytes
            cst[j] = prmt(word, 0, sel) & 0x027f027fu;
          }
        } else {
#pragma unroll
          for (int j = 0; j < REGS; j++)
            cst[j] = prmt(((const uint16_t*)cb)[j], 0, 0x9180u) & 0x027f027fu;
        }
        // Gray values for the edge-aware penalties (stream coordinates).
        const int g_cur = __ldg(&gray[p]);
        ga_l = ga_c;
        ga_c = ga_r;
        ga_r = (above_exists && xs + 1 < W) ? __ldg(&gray[(int64_t)ya * W + col(xs + 1)]) : 0;
        const bool textured = __ldg(&tex[p]) != 0;

        PathState<REGS> out[NPATH];
        // (1,0): predecessor xs-1 in this row.
        {
          uint32_t q = horiz.m + lut[abs(g_cur - g_left)];
          path_step<REGS>(horiz, q, p1x2, cst, pad, lane, out[0]);
        }
        // Paths from the row above: (0,1) at xs, (1,1) at xs-1, (-1,1) at xs+1.
        const uint8_t* above_slot[3] = {nullptr, nullptr, nullptr};
        if (above_exists) {
          if (w > 0) {
            above_slot[0] = ring_above + (xs & 3) * L.slot;
            if (xs >= 1) above_slot[1] = ring_above + ((xs - 1) & 3) * L.slot;
            if (xs + 1 < W) above_slot[2] = ring_above + ((xs + 1) & 3) * L.slot;
          } else if (use_carry) {
            auto cslot = [&](int xx) {
              return carry_buf + ((xx / K) % 3) * K * L.slot + (xx % K) * L.slot;
            };
            above_slot[0] = cslot(xs);
            if (xs >= 1) above_slot[1] = cslot(xs - 1);
            if (xs + 1 < W) above_slot[2] = cslot(xs + 1);
          }
        }
        const int g_above[3] = {ga_c, ga_l, ga_r};
#pragma unroll
        for (int i = 0; i < NPATH - 1; i++) {
          PathState<REGS> prev;
          if (above_slot[i])
            load_state<REGS>(above_slot[i], i, Dp, lane, prev);
          else
            zero_state(prev);
          uint32_t q = prev.m + lut[abs(g_cur - g_above[i])];
          path_step<REGS>(prev, q, p1x2, cst, pad, lane, out[i + 1]);
        }
        // Partial aggregate of this stream's paths.
        uint32_t s[REGS];
#pragma unroll
        for (int j = 0; j < REGS; j++) {
          uint32_t acc = out[0].v[j];
#pragma unroll
          for (int i = 1; i < NPATH; i++) acc += out[i].v[j];
          s[j] = acc;
        }
        // Outputs for the row below: the three vertical paths, zeros if this pixel is untextured.
        if (NPATH > 1) {
#pragma unroll
          for (int i = 0; i < NPATH - 1; i++) {
            PathState<REGS> o = out[i + 1];
            if (!textured) zero_state(o);
            store_state<REGS>(out_slot, i, Dp, lane, o);
            if (w == kRows - 1 && has_next)
              store_state<REGS>(a.carry + ((int64_t)(stream * a.nb + b) * W + xs) * L.slot, i, Dp,
                                lane, o);
          }
        }
        horiz = out[0];
        if (!textured) zero_state(horiz);
        g_left = g_cur;

        if (first) {
          uint32_t* dst = (uint32_t*)(sum + p * Dp + lane * 2 * REGS);
#pragma unroll
          for (int j = 0; j < REGS; j++) dst[j] = s[j];
        } else {
          const uint32_t* other =
              (const uint32_t*)(sum_buf + (c & 1) * K * Dp + slot * Dp + lane * 2 * REGS);
#pragma unroll
          for (int j = 0; j < REGS; j++) s[j] += other[j];
          // Winners record (GpuStereo.java:758-769) for pixels inside the census border.
          int r0 = -1, r1 = INT_MAX, r2 = INT_MAX, r3 = -1, r4 = -1, r5;
          const int k0 = lane * 2 * REGS;
          bool valid[2 * REGS];
#pragma unroll
          for (int j = 0; j < 2 * REGS; j++) valid[j] = cb[j] != 0x80;
          bool f0 = __any_sync(0xffffffffu, lane == 0 && valid[0]);
          int last = a.D - 1 - k0;
          bool fl = false;
#pragma unroll
          for (int j = 0; j < 2 * REGS; j++) fl |= (j == last) && valid[j];
          fl = __any_sync(0xffffffffu, fl);
          r5 = (f0 ? 1 : 0) | (fl ? 2 : 0);
          if (region_row && x >= a.rx && x < W - a.rx) {
            uint32_t key = 0xffffffffu;
#pragma unroll
            for (int j = 0; j < 2 * REGS; j++) {
              uint32_t sv = (s[j / 2] >> (16 * (j & 1))) & 0xffffu;
              uint32_t kk = (sv << 12) | (uint32_t)(k0 + j);
              if (valid[j]) key = min(key, kk);
            }
            key = __reduce_min_sync(0xffffffffu, key);
            if (key != 0xffffffffu) {
              int best = (int)(key & 0xfffu);
              uint32_t sec = 0x7fffffffu, bef = 0xffffffffu, aft = 0xffffffffu;
#pragma unroll
              for (int j = 0; j < 2 * REGS; j++) {
                int k = k0 + j;
                uint32_t sv = (s[j / 2] >> (16 * (j & 1))) & 0xffffu;
                if (valid[j] && abs(k - best) > 1) sec = min(sec, sv);
                if (valid[j] && k == best - 1) bef = sv;
                if (valid[j] && k == best + 1) aft = sv;
              }
              r0 = best;
              r1 = (int)(key >> 12);
              r2 = (int)__reduce_min_sync(0xffffffffu, sec);
              bef = __reduce_min_sync(0xffffffffu, bef);
              aft = __reduce_min_sync(0xffffffffu, aft);
              r3 = bef == 0xffffffffu ? -1 : (int)bef;
              r4 = aft == 0xffffffffu ? -1 : (int)aft;
            }
          }
          const int ri = xs % kRecords;
          if (lane < 6) {
            int v = lane == 0 ? r0 : lane == 1 ? r1 : lane == 2 ? r2 : lane == 3 ? r3 : lane == 4 ? r4 : r5;
            rec[ri * 6 + lane] = v;
          }
          if (ri == kRecords - 1 || xs == W - 1) {
            __syncwarp();
            const int base = xs - ri;
            if (lane <= ri) {
              int xx = col(base + lane);
              select_record(a, view, rec + lane * 6, (int64_t)y * W + xx, counts);
            }
            __syncwarp();
          }
        }
        if (first && xs == W - 1) {  // whole row of partial aggregate stored: publish it
          __syncwarp();
          if (lane == 0) {
            __threadfence();
            atomicExch(&a.row_done[view * H + y], 1);
          }
        }
      } else {
        // Rows beyond the image: the row below sees no predecessor.
        PathState<REGS> z;
        zero_state(z);
        for (int i = 0; i < NPATH - 1; i++) {
          store_state<REGS>(out_slot, i, Dp, lane, z);
          if (w == kRows - 1 && has_next)
            store_state<REGS>(a.carry + ((int64_t)(stream * a.nb + b) * W + xs) * L.slot, i, Dp,
                              lane, z);
        }
      }
      // Publish carry progress every chunk (and at the end of the row).
      if (w == kRows - 1 && has_next && ((xs + 1) % K == 0 || xs == W - 1)) {
        __syncwarp();
        if (lane == 0) {
          __threadfence();
          atomicExch(&a.progress[stream * a.nb + b], xs + 1);
        }
      }
    }
    __syncthreads();
  }
  // Drain: every bulk copy this warp issued has landed before the CTA's shared memory is released
  // (normally already true; after a timed-out wait this bounds the exit on the copies in flight).
  {
    int dummy = 0;
    const long long drain = a.timeout / 4;
    for (int c = max(0, issued_cost - 2); c < issued_cost; c++)
      wait_bar(&cost_bar[c & 1], (c >> 1) & 1, &dummy, drain);
    for (int c = max(0, issued_sum - 2); c < issued_sum; c++)
      wait_bar(&sum_bar[c & 1], (c >> 1) & 1, &dummy, drain);
    for (int c = max(0, issued_carry - 3); c < issued_carry; c++)
      wait_bar(&carry_bar[c % 3], (c / 3) & 1, &dummy, drain);
  }
  // Selection counters of the left view.
  if (view == 0 && a.stats) {
    unsigned long long* dst[6] = {&a.stats->lower_boundary_rejected,
                                  &a.stats->full_interval_pixels, &a.stats->boundary_rejected,
                                  &a.stats->upper_boundary_rejected,
                                  &a.stats->ambiguity_rejected, &a.stats->selected};
#pragma unroll
    for (int i = 0; i < 6; i++) {
      unsigned total = __reduce_add_sync(0xffffffffu, counts[i]);
      if (lane == 0 && total) atomicAdd(dst[i], (unsigned long long)total);
    }
  }
}

template <int REGS, int NPATH>
cudaError_t launch_sweep(const SweepArgs& a, int shared, cudaStream_t stream) {
  auto kernel = sweep_kernel<REGS, NPATH>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, shared);
  if (e != cudaSuccess) return e;
  kernel<<<4 * a.nb, kRows * 32, shared, stream>>>(a);
  return cudaGetLastError();
}

struct FusedLayout {
  size_t cost, sum, carry, flags, total;
  int Dp, nb, K, slot;
  FusedLayout(const csgm_params& p, int w, int h) {
    Dp = padded_d(p.disparities);
    nb = (h + kRows - 1) / kRows;
    K = Dp <= 128 ? 8 : 4;
    slot = 3 * Dp * 2 + 16;
    size_t n = (size_t)w * h;
    cost = n * Dp;
    sum = n * Dp * 2;
    carry = (size_t)4 * nb * w * slot;
    flags = ((size_t)4 * nb + 2 * (size_t)h + 8) * sizeof(int);
    total = 2 * cost + 2 * sum + carry + flags + 4 * 256;
  }
};

}  // namespace

bool fused_supported(const csgm_params& p) {
  if (p.disparities > 256 || p.aggregate_bytes != 2) return false;
  if (p.directions != 4 && p.directions != 8) return false;
  if (512 + 2 * (int64_t)p.p2 + p.p1 > 65535) return false;
  return true;
}

size_t fused_workspace_bytes(const csgm_params& p, int w, int h) {
  return FusedLayout(p, w, h).total;
}

int run_views_fused(Context& ctx, const csgm_params& p, const FusedViews& v, int w, int h,
                    int** error_flag) {
  int status = CSGM_OK;
  FusedLayout F(p, w, h);
  uint8_t* cost_l = (uint8_t*)ctx.ws->get(kCostL, F.cost, &status);
  if (!cost_l) return status;
  uint8_t* cost_r = (uint8_t*)ctx.ws->get(kCostR, F.cost, &status);
  if (!cost_r) return status;
  uint16_t* sum_l = (uint16_t*)ctx.ws->get(kSum, F.sum, &status);
  if (!sum_l) return status;
  uint16_t* sum_r = (uint16_t*)ctx.ws->get(kSumR, F.sum, &status);
  if (!sum_r) return status;
  uint8_t* carry = (uint8_t*)ctx.ws->get(kCarry, F.carry, &status);
  if (!carry) return status;
  int* flags = (int*)ctx.ws->get(kFlags, F.flags, &status);
  if (!flags) return status;

  int words = (p.window_x * p.window_y - 1 + 63) / 64;
  CostPairArgs ca{};
  ca.view[0] = CostArgs{v.desc_l, v.desc_r, v.tex_l, v.tex_r, v.gray_l, v.gray_r, nullptr, w, h,
                        p.disparities, p.min_disparity, 0, p.window_x, p.window_y, words,
                        p.cost_mode, p.census_weight_milli, p.ad_truncation,
                        p.gradient_truncation, p.window_x * p.window_y - 1};
  ca.view[1] = ca.view[0];
  ca.view[1].desc_a = v.desc_r;
  ca.view[1].desc_b = v.desc_l;
  ca.view[1].tex_a = v.tex_r;
  ca.view[1].tex_b = v.tex_l;
  ca.view[1].gray_a = v.gray_r;
  ca.view[1].gray_b = v.gray_l;
  ca.view[1].reverse = 1;
  ca.out[0] = cost_l;
  ca.out[1] = cost_r;
  ca.Dp = F.Dp;
  {
    int64_t n = (int64_t)w * h;
    int64_t blocks = (n * 32 + 255) / 256;
    int grid = (int)std::min<int64_t>(blocks, (int64_t)ctx.sm_count * 32);
    ctx.prof->kernel_begin();
    cost_pair_kernel<<<dim3(grid, 2), 256, 0, ctx.stream>>>(ca);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "cost kernel launch");
    ctx.prof->kernel_end("cost_pair");
  }
  cudaError_t e = cudaMemsetAsync(flags, 0, F.flags, ctx.stream);
  if (e != cudaSuccess) return cuda_fail(e, "flag clear");

  SweepArgs a{};
  a.cost[0] = cost_l;
  a.cost[1] = cost_r;
  a.gray[0] = v.gray_l;
  a.gray[1] = v.gray_r;
  a.tex[0] = v.tex_l;
  a.tex[1] = v.tex_r;
  a.sum[0] = sum_l;
  a.sum[1] = sum_r;
  a.disp[0] = v.disp_l;
  a.disp[1] = v.disp_r;
  a.carry = carry;
  a.progress = flags;
  a.row_done = flags + 4 * F.nb;
  a.ticket = flags + 4 * F.nb + 2 * h;
  a.error = a.ticket + 1;
  *error_flag = a.error;
  a.reasons = v.reasons;
  a.boundary = v.boundary;
  a.stats = v.stats;
  a.W = w;
  a.H = h;
  a.D = p.disparities;
  a.Dp = F.Dp;
  a.nb = F.nb;
  a.Hp = F.nb * kRows;
  a.split = kRows * ((F.nb + 1) / 2);
  a.p1 = p.p1;
  a.p2 = p.p2;
  a.edge_scale = p.edge_scale;
  a.min_disparity = p.min_disparity;
  a.rx = p.window_x / 2;
  a.ry = p.window_y / 2;
  a.chunk = F.K;
  a.uniqueness = p.uniqueness;
  a.timeout = 4000000000LL;  // ~2 s at 2 GHz
  int shared = SweepLayout(F.Dp, F.K).total;
  int regs = F.Dp / 64;
  bool eight = p.directions == 8;
  ctx.prof->kernel_begin();
  switch (regs * 2 + (eight ? 1 : 0)) {
    case 2: e = launch_sweep<1, 2>(a, shared, ctx.stream); break;
    case 3: e = launch_sweep<1, 4>(a, shared, ctx.stream); break;
    case 4: e = launch_sweep<2, 2>(a, shared, ctx.stream); break;
    case 5: e = launch_sweep<2, 4>(a, shared, ctx.stream); break;
    case 6: e = launch_sweep<3, 2>(a, shared, ctx.stream); break;
    case 7: e = launch_sweep<3, 4>(a, shared, ctx.stream); break;
    case 8: e = launch_sweep<4, 2>(a, shared, ctx.stream); break;
    case 9: e = launch_sweep<4, 4>(a, shared, ctx.stream); break;
    default: return fail(CSGM_E_UNSUPPORTED, "fused path: unsupported D");
  }
  if (e != cudaSuccess) return cuda_fail(e, "sweep kernel launch");
  ctx.prof->kernel_end("sweep");
  return CSGM_OK;
}

}  // namespace csgm
