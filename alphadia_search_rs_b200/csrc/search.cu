// PeakGroupSelection.search on the device (src/peak_group_selection/mod.rs:87-195).
//
// Stages, all on one stream:
//   1. prep_kernel      one warp per precursor: RT cycle limits, quadrupole
//                       windows, fragment filter / top-k / m/z sort, m/z bin
//                       range of every kept fragment.
//   2. classify_kernel  precursors into RT-window length classes.
//   3. search_kernel    one instance per class, one warp per precursor
//                       (persistent warps pulling from an atomic counter): XIC
//                       gather into shared memory, Gaussian convolution,
//                       log-dot score, 5-point local maxima, top-K.  Arithmetic
//                       follows the reference's operation order with explicitly
//                       rounded f32 ops, so the only difference to the reference
//                       is its logf (see ln_rn).
//   4. compaction       order-preserving concatenation of the per-precursor
//                       candidates into the nine to_arrays() columns.
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <memory>
#include <thread>

#include <cuda_bf16.h>

#include "common.cuh"

namespace ads {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxHalf = 31;       // taps passed as kernel parameters up to this half width
// widest Gaussian kernel accepted: a run has at most 65,536 cycles (u16 cycle indices)
// and a kernel wider than the run yields no output anywhere
constexpr int64_t kMaxKernelSize = 65536;
constexpr int kPrepThreads = 256;  // 8 precursors per prep block
constexpr int kScanBlock = 1024;

// Rust 1.88 slice::binary_search (Ok: the LAST equal element; Err: insertion
// point) on a sorted array, for the u16 cycle lists of fill_xic_slice
// (src/quadrupole_observation/mod.rs:91-94).
__device__ __forceinline__ int64_t rust_bsearch_u16(const uint16_t* a, int64_t n, int x) {
  if (n == 0) return 0;
  int64_t size = n, base = 0;
  while (size > 1) {
    const int64_t half = size / 2, mid = base + half;
    base = ((int)a[mid] > x) ? base : mid;
    size -= half;
  }
  const int v = a[base];
  if (v == x) return base;
  return base + (v < x ? 1 : 0);
}

// First index with a[i] >= x.
__device__ __forceinline__ int64_t lower_bound_u16(const uint16_t* a, int64_t n, int x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int)a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Same Rust search on the RT index (binary_search_by with partial_cmp,
// src/rt_index/mod.rs:123-135).
// `a` may be in shared or global memory (plain loads).
__device__ __forceinline__ int rust_bsearch_f32(const float* a, int n, float x) {
  int size = n, base = 0;
  while (size > 1) {
    const int half = size / 2, mid = base + half;
    base = (a[mid] > x) ? base : mid;
    size -= half;
  }
  const float v = a[base];
  if (v == x) return base;
  return base + (v < x ? 1 : 0);
}

// RTIndex::get_cycle_idx_limits (src/rt_index/mod.rs:89-138).  `rt` may be in shared or
// global memory.
__device__ __forceinline__ void rt_limits(const float* rt, int n, float dt, float prt, float tol,
                                          float pad, int* lo, int* hi) {
  if (n == 0) {
    *lo = 0;
    *hi = 0;
    return;
  }
  const float min_tol = __fmul_rn(__fadd_rn(10.0f, pad), dt);
  const float eff = fmaxf(tol, min_tol);
  const float lower = __fsub_rn(prt, eff), upper = __fadd_rn(prt, eff);
  const float r0 = rt[0], rn = rt[n - 1];
  if (upper < r0) {
    *lo = 0;
    *hi = 0;
    return;
  }
  if (lower > rn) {
    *lo = n;
    *hi = n;
    return;
  }
  *lo = (lower <= r0) ? 0 : rust_bsearch_f32(rt, n, lower);
  *hi = (upper >= rn) ? n : rust_bsearch_f32(rt, n, upper);
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ------------------------------------------------------------------ prep

struct PrepArgs {
  int64_t n_prec;
  const float* pmz;
  const float* prt;
  const float* ptol;  // nullable
  float rt_tol;
  const uint64_t* fstart;
  const uint64_t* fstop;
  const float* fmz;
  const float* fint;
  const uint8_t* fnum;
  const uint8_t* ftype;
  const float* rt;
  int n_rt;
  float delta_t;
  float pad;  // kernel_size as f32 (num_cycles_padding)
  const WinInfo* win;
  int n_obs;
  GridView g;
  float mass_tol;
  int top_k;
  int kf;     // per-precursor fragment stride
  int maxw;   // per-precursor window stride
  int min_c;  // cycle ranges shorter than this cannot hold a local maximum
  uint8_t* keep;  // scratch, keep_stride bytes per prep warp
  int64_t keep_stride;
  int* nf;
  int* cs;
  int* ce;
  int* nwin;
  int* wins;
  float* fw;
  uint32_t* blo;
  uint32_t* bhi;
  int* err;
  int win_in_smem;  // stage the isolation windows / the RT index in shared memory
  int rt_in_smem;
};

// Shared memory of a prep block: the isolation windows, then the MS1 retention times,
// each when it fits the 48 KB a block gets without opting in.
constexpr size_t kPrepSmemBytes = 48 * 1024;

__host__ __device__ inline size_t prep_win_bytes(int n_obs) { return ((size_t)n_obs * sizeof(WinInfo) + 15) / 16 * 16; }

size_t plan_prep_smem(PrepArgs* a) {
  const size_t wb = prep_win_bytes(a->n_obs), rb = (size_t)a->n_rt * sizeof(float);
  a->win_in_smem = wb <= kPrepSmemBytes;
  a->rt_in_smem = (a->win_in_smem ? wb : 0) + rb <= kPrepSmemBytes;
  return (a->win_in_smem ? wb : 0) + (a->rt_in_smem ? rb : 0);
}

// Fragment m/z ordering key: NaN sorts after every number (ties by library
// position), so the output positions always form a permutation.
__device__ __forceinline__ float mz_key(float m) { return m != m ? INFINITY : m; }

// The ppm bin range of one kept fragment (src/quadrupole_observation/mod.rs:79-83,
// src/mz_index/mod.rs:95-127), stored at its position in m/z order.
__device__ __forceinline__ void write_fragment(const PrepArgs& a, int64_t p, int pos, float mz,
                                               float w) {
  const float delta = __fmul_rn(__fmul_rn(mz, a.mass_tol), 1e-6f);
  const float lo = __fsub_rn(mz, delta), hi = __fadd_rn(mz, delta);
  const uint32_t b0 = grid_lower_bound(a.g, lo);
  const uint32_t b1 = max(b0, grid_upper_bound(a.g, hi));
  const int64_t o = p * a.kf + pos;
  a.fw[o] = w;
  a.blo[o] = b0;
  a.bhi[o] = b1;
}

// get_precursor_filtered / filter_sort_fragments (src/speclib_flat/mod.rs:240-345,
// 388-456): non_zero and y1 filters, top-k by intensity, sort by fragment m/z;
// ties go to the lower library position.
__device__ int select_fragments(const PrepArgs& a, int64_t p, int lane, uint8_t* keep) {
  const int64_t s = (int64_t)a.fstart[p];
  const int64_t n = (int64_t)a.fstop[p] - s;
  if (n <= 32) {
    // one fragment per lane; rankings through shuffles
    const bool have = lane < n;
    const float I = have ? __ldg(a.fint + s + lane) : 0.0f;
    bool k = have && (I > 0.0f) && !(__ldg(a.ftype + s + lane) == 121 && __ldg(a.fnum + s + lane) == 1);
    unsigned km = __ballot_sync(kFull, k);
    if (__popc(km) > a.top_k) {
      const float ik = k ? I : -1.0f;
      int rank = 0;
      for (int j = 0; j < (int)n; ++j) {
        const float J = __shfl_sync(kFull, ik, j);
        rank += (J > ik) || (J == ik && j < lane);
      }
      k = k && rank < a.top_k;
      km = __ballot_sync(kFull, k);
    }
    const float mz = have ? __ldg(a.fmz + s + lane) : 0.0f;
    const float key = mz_key(mz);
    int pos = 0;
    for (int j = 0; j < (int)n; ++j) {
      const float m = __shfl_sync(kFull, key, j);
      if ((km >> j) & 1u) pos += (m < key) || (m == key && j < lane);
    }
    if (k) write_fragment(a, p, pos, mz, I);
    __syncwarp();
    return __popc(km);
  }
  int nk = 0;
  for (int64_t i0 = 0; i0 < n; i0 += 32) {
    const int64_t i = i0 + lane;
    bool k = false;
    if (i < n) {
      const float I = __ldg(a.fint + s + i);
      k = (I > 0.0f) && !(__ldg(a.ftype + s + i) == 121 && __ldg(a.fnum + s + i) == 1);
      keep[i] = k ? 1 : 0;
    }
    nk += __popc(__ballot_sync(kFull, k));
  }
  __syncwarp();
  const bool topk = nk > a.top_k;
  if (topk) {
    for (int64_t i0 = 0; i0 < n; i0 += 32) {
      const int64_t i = i0 + lane;
      if (i < n && keep[i]) {
        const float I = __ldg(a.fint + s + i);
        int rank = 0;
        for (int64_t j = 0; j < n; ++j) {
          if (!keep[j]) continue;
          const float J = __ldg(a.fint + s + j);
          rank += (J > I) || (J == I && j < i);
        }
        if (rank < a.top_k) keep[i] = 2;
      }
    }
    __syncwarp();
  }
  const int need = topk ? 2 : 1;
  const int F = topk ? a.top_k : nk;
  for (int64_t i0 = 0; i0 < n; i0 += 32) {
    const int64_t i = i0 + lane;
    if (i < n && keep[i] >= need) {
      const float mz = __ldg(a.fmz + s + i);
      const float key = mz_key(mz);
      int pos = 0;
      for (int64_t j = 0; j < n; ++j) {
        if (keep[j] < need) continue;
        const float m = mz_key(__ldg(a.fmz + s + j));
        pos += (m < key) || (m == key && j < i);
      }
      write_fragment(a, p, pos, mz, __ldg(a.fint + s + i));
    }
  }
  __syncwarp();
  return F;
}

// Statistics pass: sum over searched precursors of (kept fragments x cycles), the
// XIC cells the convolution and the score visit.
__global__ void cells_kernel(int64_t n, const int* nf, const int* cs, const int* ce,
                             unsigned long long* out) {
  unsigned long long v = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int C = ce[p] - cs[p];
    if (nf[p] > 0 && C > 0) v += (unsigned long long)nf[p] * (unsigned long long)C;
  }
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(out, v);
}

// 8 blocks of 256 threads per SM (32 registers): the kernel waits on its global loads,
// so occupancy pays (0.33 -> 0.27 ms per search of 200,000 precursors on 3000 x 300 data,
// against 4 blocks at 62 registers)
__global__ void __launch_bounds__(kPrepThreads, 8) prep_kernel(PrepArgs a) {
  extern __shared__ __align__(16) unsigned char prep_smem[];
  const int lane = threadIdx.x & 31;
  const WinInfo* win = a.win;
  const float* rt = a.rt;
  {
    size_t o = 0;
    if (a.win_in_smem) {
      WinInfo* ws = reinterpret_cast<WinInfo*>(prep_smem);
      for (int i = threadIdx.x; i < a.n_obs; i += blockDim.x) ws[i] = a.win[i];
      win = ws;
      o = prep_win_bytes(a.n_obs);
    }
    if (a.rt_in_smem) {
      float* rs = reinterpret_cast<float*>(prep_smem + o);
      for (int i = threadIdx.x; i < a.n_rt; i += blockDim.x) rs[i] = __ldg(a.rt + i);
      rt = rs;
    }
    __syncthreads();
  }
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = warp0; p < a.n_prec; p += n_warps) {
    const float tol = a.ptol ? __ldg(a.ptol + p) : a.rt_tol;
    int cs, ce;
    rt_limits(rt, a.n_rt, a.delta_t, __ldg(a.prt + p), tol, a.pad, &cs, &ce);
    bool skip = (ce - cs) < a.min_c;
    int nw = 0;
    if (!skip) {
      const float pmz = __ldg(a.pmz + p);
      for (int base = 0; base < a.n_obs; base += 32) {
        const int w = base + lane;
        bool hit = false;
        if (w < a.n_obs) {
          const WinInfo wi = win[w];
          hit = wi.ss_off >= 0 && wi.lo <= pmz && wi.hi >= pmz;
        }
        const unsigned m = __ballot_sync(kFull, hit);
        if (hit) {
          const int pos = nw + __popc(m & lanemask_lt());
          if (pos < a.maxw) a.wins[p * a.maxw + pos] = w;
        }
        nw += __popc(m);
      }
      if (nw > a.maxw) {
        if (lane == 0) atomicOr(a.err, 1);
        nw = a.maxw;
      }
      skip = nw == 0;
    }
    int F = 0;
    if (!skip) {
      F = select_fragments(a, p, lane, a.keep + warp0 * a.keep_stride);
      skip = F == 0;
    }
    if (lane == 0) {
      a.cs[p] = cs;
      a.ce[p] = skip ? cs : ce;
      a.nf[p] = skip ? 0 : F;
      a.nwin[p] = skip ? 0 : nw;
    }
  }
}

#include "search_kernel.cuh"

// Cycles per lane the search kernel is compiled for, and its instances: fully
// unrolled stencils for the half widths of kernel_size 20, 21-22 and 31-32, any
// other half width through the generic path.
constexpr int kLaneCycles[] = {4, 8, 10, 12, 16};
constexpr int kGrowLaneCycles = 16;  // cycles per lane of long-window (GROW) launches
// Global working sets of one long-window launch: at most this many bytes (the grid
// is trimmed to fit; a warp's set is about 15 bytes per cycle of the longest window).
constexpr int64_t kGrowBudgetBytes = int64_t(1) << 30;
constexpr int kDefaultWarpsPerBlock = 4;
constexpr int kMaxClasses = 10;
constexpr int kStats = 7;  // statistics-pass counters (ads_selection_last_stats)

// Length classes of one search: class b covers C <= bound[b] with S[b] cycles per
// lane (bound[last] = the longest window, searched in one or more passes).
struct LenClasses {
  int bound[kMaxClasses];
  int S[kMaxClasses];
};

// Relative cost of searching a c-cycle window with S cycles per lane: passes times
// (S outputs + about 6 outputs' worth of per-pass loads and control per lane).
int lane_cost(int64_t c, int S) { return (int)((c + 32 * S - 1) / (32 * S)) * (S + 6); }

// The cheapest lane width for a c-cycle window, ties to the larger S.
int best_lane_cycles(int64_t c) {
  int S = kLaneCycles[0];
  int best = -1;
  for (int cand : kLaneCycles) {
    const int cost = lane_cost(c, cand);
    if (best < 0 || cost <= best) {
      best = cost;
      S = cand;
    }
  }
  return S;
}

// Length classes: every bound 32 * S * k (k <= 4 passes) below the longest window, at
// least 20 % apart, each with its cheapest lane width, then one class for the rest.
// A fixed cycles_per_lane gives a single class.  Windows longer than kSmemMaxCycles
// get a class of their own, searched with the warps' working sets in global memory
// (GROW, kGrowLaneCycles cycles per lane); everything up to kSmemMaxCycles then stays
// in shared-memory classes.
int plan_classes(int64_t c_max, int fixed_S, LenClasses* out) {
  int n = 0;
  const bool grow = c_max > kSmemMaxCycles;
  const int64_t c_sm = std::min<int64_t>(c_max, kSmemMaxCycles);
  if (fixed_S == 0) {
    std::vector<int> bounds;
    for (int S : kLaneCycles)
      for (int k = 1; k <= 4; ++k)
        if ((int64_t)32 * S * k < c_sm) bounds.push_back(32 * S * k);
    std::sort(bounds.begin(), bounds.end());
    int last = 0;
    for (int b : bounds) {
      if (n == kMaxClasses - 1 - (grow ? 1 : 0)) break;
      if (last > 0 && (int64_t)b * 5 < (int64_t)last * 6) continue;
      out->bound[n] = b;
      out->S[n] = best_lane_cycles(b);
      last = b;
      ++n;
    }
  }
  if (grow) {
    out->bound[n] = kSmemMaxCycles;
    out->S[n] = fixed_S ? fixed_S : best_lane_cycles(kSmemMaxCycles);
    ++n;
    out->bound[n] = (int)c_max;
    out->S[n] = kGrowLaneCycles;
    return n + 1;
  }
  out->bound[n] = (int)c_max;
  out->S[n] = fixed_S ? fixed_S : best_lane_cycles(c_max);
  return n + 1;
}

template <int H, bool FAST, bool STATS>
void (*pick_for_h(int S, bool grow))(SearchArgs) {
  if (grow) return search_kernel<H, kGrowLaneCycles, FAST, true, STATS>;
  switch (S) {
    case 4: return search_kernel<H, 4, FAST, false, STATS>;
    case 8: return search_kernel<H, 8, FAST, false, STATS>;
    case 10: return search_kernel<H, 10, FAST, false, STATS>;
    case 12: return search_kernel<H, 12, FAST, false, STATS>;
    default: return search_kernel<H, 16, FAST, false, STATS>;
  }
}

// The statistics pass counts gather work, which the half width does not change: it
// runs the generic-h instances with the counters compiled in.
template <bool FAST>
void (*pick_for_precision(int h, int S, bool grow, bool stats))(SearchArgs) {
  if (stats) return pick_for_h<0, FAST, true>(S, grow);
  switch (h) {
    case 10: return pick_for_h<10, FAST, false>(S, grow);
    case 11: return pick_for_h<11, FAST, false>(S, grow);
    case 16: return pick_for_h<16, FAST, false>(S, grow);
    default: return pick_for_h<0, FAST, false>(S, grow);
  }
}

// fast: BF16 intensity storage with the fast f32 arithmetic (ADS_PRECISION_BF16);
// grow: working sets in global memory (long windows; S must be kGrowLaneCycles);
// stats: the statistics pass's instances (work counters compiled in)
void (*pick_search_kernel(int h, int S, bool fast, bool grow, bool stats))(SearchArgs) {
  return fast ? pick_for_precision<true>(h, S, grow, stats)
              : pick_for_precision<false>(h, S, grow, stats);
}

// Largest block (in warps) an instance may launch: its launch bounds (LaunchShape); the
// statistics pass runs the generic-h instances (256 threads).
int max_warps_per_block(bool fast, int h, bool grow, bool stats) {
  return (stats ? 256 : launch_threads(h, fast, grow)) / 32;
}

// Long-window launches: blocks whose working sets fit kGrowBudgetBytes (at least one).
int64_t grow_blocks(int64_t blocks, int nw, size_t warp_bytes, size_t budget) {
  const int64_t fit = (int64_t)(budget / std::max<size_t>(warp_bytes, 1)) / nw;
  return std::max<int64_t>(1, std::min(blocks, fit));
}

// Kernel taps w[0..h] of a launch, also each twice as one packed f32x2 operand,
// and the packed zeros of the exact stencil.  Taps past kMaxHalf are read from
// `kw_dev` (device memory holding w[0..h]).
void set_taps(SearchArgs* sa, const float* kernel, int h, const float* kw_dev) {
  sa->kw_dev = h > kMaxHalf ? kw_dev : nullptr;
  for (int k = 0; k <= std::min(h, kMaxHalf); ++k) {
    sa->kw[k] = kernel[k];
    uint32_t b;
    std::memcpy(&b, &kernel[k], 4);
    sa->kw2[k] = ((unsigned long long)b << 32) | b;
  }
  sa->zero2 = 0ull;
  sa->nzero2 = 0x8000000080000000ull;
}

// ------------------------------------------------------------ compaction

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* sh, int64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) sh[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int64_t w = lane < nw ? sh[lane] : 0;
    int64_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t t = __shfl_up_sync(kFull, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < nw) sh[lane] = wi - w;
    if (lane == 31) sh[32] = wi;
  }
  __syncthreads();
  const int64_t r = sh[warp] + incl - v;
  *total = sh[32];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanBlock) block_sum_kernel(const int* cand_n, int64_t n,
                                                               int64_t* block_sums) {
  __shared__ int64_t sh[33];
  const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  int64_t total;
  block_exclusive_scan(i < n ? cand_n[i] : 0, sh, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) scan_block_sums_kernel(int64_t* sums, int64_t nb,
                                                                     int64_t* total_out) {
  __shared__ int64_t sh[33];
  int64_t carry = 0;
  for (int64_t b0 = 0; b0 < nb; b0 += kScanBlock) {
    const int64_t i = b0 + threadIdx.x;
    const int64_t v = i < nb ? sums[i] : 0;
    int64_t tot;
    const int64_t ex = block_exclusive_scan(v, sh, &tot);
    if (i < nb) sums[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total_out = carry;
}

struct ScatterArgs {
  int64_t n_prec;
  int k_out;
  uint64_t peak_length;
  uint64_t rt_len;
  const int* cand_n;
  const float* cand_score;
  const int* cand_center;
  const uint64_t* pidx;
  const int64_t* block_off;
  uint64_t* o_pidx;
  uint64_t* o_rank;
  float* o_score;
  uint64_t* o_center;
  uint64_t* o_start;
  uint64_t* o_stop;
};

// Candidate::new (src/candidate/entry.rs:19-38) as assembled in
// src/peak_group_selection/mod.rs:172-192, written in precursor then rank order.
__global__ void __launch_bounds__(kScanBlock) scatter_kernel(ScatterArgs a) {
  __shared__ int64_t sh[33];
  const int64_t p = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  const int n = p < a.n_prec ? a.cand_n[p] : 0;
  int64_t total;
  const int64_t off = a.block_off[blockIdx.x] + block_exclusive_scan(n, sh, &total);
  for (int r = 0; r < n; ++r) {
    const int64_t o = off + r;
    const uint64_t center = (uint64_t)a.cand_center[p * a.k_out + r];
    a.o_pidx[o] = a.pidx[p];
    a.o_rank[o] = (uint64_t)r;
    a.o_score[o] = a.cand_score[p * a.k_out + r];
    a.o_center[o] = center;
    a.o_start[o] = center - a.peak_length;  // usize arithmetic of a release build (wraps)
    const uint64_t stop = center + a.peak_length + 1;
    a.o_stop[o] = stop < a.rt_len ? stop : a.rt_len;
  }
}

}  // namespace
}  // namespace ads

// ================================================================ handles

struct AdsSelection {
  int device = 0;
  AdsSelectionParams p{};
  AdsEngineOptions o{};
  std::vector<float> kernel;
  int h = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  int64_t last_launches = 0;
  bool stats_on = false;
  ads::DevBuf<unsigned long long> stats;
  int64_t last_stats[ads::kStats] = {0, 0, 0, 0, 0, 0, 0};
  // workspace
  ads::DevBuf<int> nf, cs, ce, nwin, wins, cand_n, cand_center;
  ads::DevBuf<float> fw, cand_score;
  ads::DevBuf<uint32_t> blo, bhi;
  ads::DevBuf<uint8_t> keep;
  ads::DevBuf<unsigned long long> work;
  ads::DevBuf<int> class_lists;
  ads::DevBuf<unsigned int> class_hist;  // (class, fragment count) histogram, then cursors
  ads::DevBuf<int64_t> block_sums;
  ads::DevBuf<float> grow;  // warps' working sets of long-window launches
  ads::DevBuf<float> taps;  // kernel taps on the device, for half widths past kMaxHalf
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // one set of four events per timed search since the last read-out
  std::vector<std::array<cudaEvent_t, 4>> stage_pool;
  size_t stage_used = 0;
  cudaEvent_t* stage_ev = nullptr;  // set of the search being enqueued
  // use_graph: the pipeline captured for one (run, library, collection) and the
  // buffers it was captured with
  cudaGraphExec_t graph = nullptr;
  std::vector<const void*> graph_key;
  int64_t graph_launches = 0;
};

// A candidate collection does not depend on the selection that filled it: the
// search records `done` on the selection's stream, and every later read waits on
// that event from the calling thread's per-thread stream.

namespace ads {
namespace {

int check_params(const AdsSelectionParams& p, std::vector<float>* kernel, int* h) {
  if (p.kernel_size < 1)
    return fail(ADS_ERR_INVALID_ARGUMENT, "kernel_size must be >= 1 (the reference panics on 0)");
  if (p.kernel_size > kMaxKernelSize)
    return fail(ADS_ERR_INVALID_ARGUMENT,
                "kernel_size above 65536 (wider than any run's 65,536 cycles) is not supported");
  if (p.peak_length < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "peak_length < 0");
  if (p.candidate_count < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "candidate_count < 0");
  if (p.top_k_fragments < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "top_k_fragments < 0");
  *kernel = gaussian_kernel(p.fwhm_rt, 1.0f, p.kernel_size, 1.0f);
  *h = (int)kernel->size() / 2;
  return ADS_OK;
}

// Upper bound on stop - start over all precursors for RT half-windows up to
// `tol` (src/rt_index/mod.rs:99-137): the index span of any closed RT interval
// of width 2 * max(tol, min_tol), plus margin for the float rounding.
int64_t max_cycle_span(const std::vector<float>& rt, float delta_t, float tol, int64_t ks) {
  const int64_t n = (int64_t)rt.size();
  if (n == 0) return 0;
  const float min_tol = (10.0f + (float)ks) * delta_t;
  const double eff = std::max((double)tol, (double)min_tol);
  if (!std::isfinite(eff)) return n;
  const double width = 2.0 * eff * (1.0 + 1e-6) + 1e-3;
  int64_t best = 0, j = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (j < i) j = i;
    while (j < n && (double)rt[j] - (double)rt[i] <= width) ++j;
    best = std::max(best, j - i);
  }
  return std::min<int64_t>(n, best + 4);
}

// Sorts the precursors into length classes: class b holds those with
// bound[b-1] < C <= bound[b] (C = stop - start cycles), searched by a kernel
// instance whose lanes cover the class's longest window.  Precursors with nothing
// to search get no candidates here.  Order inside a class is arbitrary; results do
// not depend on it.
__global__ void classify_kernel(int64_t P, const int* nf, const int* cs, const int* ce, int n_cls,
                                LenClasses cls, int* lists, unsigned int* counts, int* cand_n) {
  const int lane = threadIdx.x & 31;
  for (int64_t p0 = blockIdx.x * (int64_t)blockDim.x; p0 < P; p0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = p0 + threadIdx.x;
    int b = -1;
    if (p < P) {
      const int C = ce[p] - cs[p];
      if (nf[p] == 0 || C <= 0) {
        cand_n[p] = 0;
      } else {
        b = n_cls - 1;
        for (int i = 0; i < n_cls - 1; ++i)
          if (C <= cls.bound[i]) {
            b = i;
            break;
          }
      }
    }
    // one atomic per class present in the warp
    const unsigned grp = __match_any_sync(kFull, b);
    const int leader = __ffs(grp) - 1;
    unsigned base = 0;
    if (b >= 0 && lane == leader) base = atomicAdd(counts + b, (unsigned)__popc(grp));
    base = __shfl_sync(kFull, base, leader);
    if (b >= 0) lists[(int64_t)b * P + base + __popc(grp & ((1u << lane) - 1u))] = (int)p;
  }
}

// Class lists in order of decreasing fragment count (longest-processing-time first:
// the warps that pull the last precursors of a launch get light ones, so the launch
// ends on a short tail).  A counting sort over (class, fragment count): a histogram,
// its exclusive scan in descending key order, then a scatter.  Keys above
// kOrderKeys - 1 share the top bucket.
constexpr int kOrderKeys = 256;

__device__ __forceinline__ int precursor_class(const int* nf, const int* cs, const int* ce, int64_t p,
                                               int n_cls, const LenClasses& cls, int* key) {
  const int C = ce[p] - cs[p];
  const int F = nf[p];
  if (F == 0 || C <= 0) return -1;
  int b = n_cls - 1;
  for (int i = 0; i < n_cls - 1; ++i)
    if (C <= cls.bound[i]) {
      b = i;
      break;
    }
  *key = min(F, kOrderKeys - 1);
  return b;
}

__global__ void class_hist_kernel(int64_t P, const int* nf, const int* cs, const int* ce, int n_cls,
                                  LenClasses cls, unsigned int* hist, int* cand_n) {
  const int lane = threadIdx.x & 31;
  for (int64_t p0 = blockIdx.x * (int64_t)blockDim.x; p0 < P; p0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = p0 + threadIdx.x;
    int b = -1, key = 0;
    if (p < P) {
      b = precursor_class(nf, cs, ce, p, n_cls, cls, &key);
      if (b < 0) cand_n[p] = 0;
    }
    const int slot = b < 0 ? -1 : b * kOrderKeys + key;
    const unsigned grp = __match_any_sync(kFull, slot);
    if (slot >= 0 && lane == __ffs(grp) - 1) atomicAdd(hist + slot, (unsigned)__popc(grp));
  }
}

// One block of kOrderKeys threads: per class, cursor[b][k] = precursors of class b with
// a larger key; class_len[b] = the class's size.
__global__ void __launch_bounds__(kOrderKeys) class_offsets_kernel(int n_cls, const unsigned int* hist,
                                                                   unsigned int* cursor,
                                                                   unsigned int* class_len) {
  __shared__ unsigned int sh[kOrderKeys];
  const int t = threadIdx.x;  // position in descending key order
  const int k = kOrderKeys - 1 - t;
  for (int b = 0; b < n_cls; ++b) {
    const unsigned int v = hist[b * kOrderKeys + k];
    sh[t] = v;
    __syncthreads();
    for (int o = 1; o < kOrderKeys; o <<= 1) {  // inclusive scan (Hillis-Steele)
      const unsigned int add = t >= o ? sh[t - o] : 0u;
      __syncthreads();
      sh[t] += add;
      __syncthreads();
    }
    cursor[b * kOrderKeys + k] = sh[t] - v;
    if (t == kOrderKeys - 1) class_len[b] = sh[t];
    __syncthreads();
  }
}

__global__ void class_scatter_kernel(int64_t P, const int* nf, const int* cs, const int* ce, int n_cls,
                                     LenClasses cls, unsigned int* cursor, int* lists) {
  const int lane = threadIdx.x & 31;
  for (int64_t p0 = blockIdx.x * (int64_t)blockDim.x; p0 < P; p0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = p0 + threadIdx.x;
    int b = -1, key = 0;
    if (p < P) b = precursor_class(nf, cs, ce, p, n_cls, cls, &key);
    const int slot = b < 0 ? -1 : b * kOrderKeys + key;
    const unsigned grp = __match_any_sync(kFull, slot);
    const int leader = __ffs(grp) - 1;
    unsigned base = 0;
    if (slot >= 0 && lane == leader) base = atomicAdd(cursor + slot, (unsigned)__popc(grp));
    base = __shfl_sync(kFull, base, leader);
    if (slot >= 0) lists[(int64_t)b * P + base + __popc(grp & ((1u << lane) - 1u))] = (int)p;
  }
}

__global__ void to_bf16_kernel(int64_t n, const float* __restrict__ in, uint16_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __bfloat16_as_ushort(__float2bfloat16_rn(in[i]));
}

// The bfloat16 copy of a run's intensities (round to nearest even), made on the
// first BF16-storage search of that run and kept with it.
int ensure_bf16_intensities(AdsDia* d, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(d->mu);
  if (d->intens_bf16.p || d->n_entries == 0) return ADS_OK;
  ADS_TRY(d->intens_bf16.alloc((size_t)d->n_entries));
  to_bf16_kernel<<<1184, 256, 0, st>>>(d->n_entries, d->intens.p, d->intens_bf16.p);
  ADS_LAUNCH_CHECK();
  // searches on other streams may read the copy next
  ADS_CUDA(cudaStreamSynchronize(st));
  return ADS_OK;
}

// Refusal for paths that read f32 intensities of a run that keeps bfloat16 only.
int need_f32_intensities(const AdsDia* d, const char* what) {
  if (!d->bf16_only) return ADS_OK;
  return fail(ADS_ERR_INVALID_ARGUMENT,
              std::string(what) + " needs the run's f32 intensities, but this run keeps bfloat16 "
                                  "intensities only (built with BF16-only storage)");
}

int reserve_candidates(AdsCandidates* c, int64_t cap) {
  if (c->cap >= cap) return ADS_OK;
  const size_t n = (size_t)std::max<int64_t>(cap, 1);
  const size_t col8 = (n * 8 + 255) / 256 * 256, col4 = (n * 4 + 255) / 256 * 256;
  ADS_TRY(c->arena.alloc(5 * col8 + col4 + 256));
  char* q = c->arena.p;
  c->pidx_p = reinterpret_cast<uint64_t*>(q);
  c->rank_p = reinterpret_cast<uint64_t*>(q + col8);
  c->center_p = reinterpret_cast<uint64_t*>(q + 2 * col8);
  c->start_p = reinterpret_cast<uint64_t*>(q + 3 * col8);
  c->stop_p = reinterpret_cast<uint64_t*>(q + 4 * col8);
  c->score_p = reinterpret_cast<float*>(q + 5 * col8);
  c->count_p = reinterpret_cast<int64_t*>(q + 5 * col8 + col4);
  c->err_p = reinterpret_cast<int*>(q + 5 * col8 + col4 + 8);
  c->cap = cap;
  return ADS_OK;
}

// Enqueues one search on the selection's stream.  While `capturing` (stream
// capture for a CUDA graph) it leaves out the cross-stream wait, the stage timing
// and the completion record, which the graph's caller does around each replay.
int enqueue_search(AdsSelection* s, const AdsDia* d, const AdsLib* l, AdsCandidates* c,
                   bool capturing) {
  if (d->device != s->device || l->device != s->device || c->device != s->device)
    return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
  DeviceGuard dg(s->device);
  cudaStream_t st = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
  if (!capturing) ADS_TRY(lib_ready_on(l, st));  // (a captured search replays after this one)
  if (!c->done) {
    ADS_CUDA(cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming));
  } else if (!capturing) {
    // a previous search into these buffers (possibly on another stream) comes first;
    // read-outs are synchronous, so none is in flight
    ADS_CUDA(cudaStreamWaitEvent(st, c->done, 0));
  }
  const int64_t P = l->n_prec;
  const AdsSelectionParams& prm = s->p;
  const int L = (int)s->kernel.size();
  const int64_t n_rt = (int64_t)d->rt.size();
  int64_t launches = 0;

  const float tol_max = l->has_tol ? std::max(l->max_tol, 0.0f) : prm.rt_tolerance;
  const int64_t c_max = std::max<int64_t>(1, max_cycle_span(d->rt, d->delta_t, tol_max, prm.kernel_size));
  // length classes and their cycles per lane (a fixed cycles_per_lane: one class)
  const int S_fixed = s->o.cycles_per_lane;
  if (S_fixed != 0 &&
      std::find(std::begin(kLaneCycles), std::end(kLaneCycles), S_fixed) == std::end(kLaneCycles))
    return fail(ADS_ERR_INVALID_ARGUMENT, "cycles_per_lane must be 0 or one of 4, 8, 10, 12, 16");
  const bool bf16 = s->o.precision == ADS_PRECISION_BF16;
  if (!bf16) ADS_TRY(need_f32_intensities(d, "an FP32 search"));
  LenClasses cls;
  const int n_cls = plan_classes(c_max, S_fixed, &cls);
  const int S_last = cls.S[n_cls - 1];
  const int ncell = (int)((c_max + 32 * S_last - 1) / (32 * S_last) * 32 * S_last);
  const int k_out = (int)std::max<int64_t>(0, std::min<int64_t>(prm.candidate_count, maxima_cap(ncell)));
  const int kf = (int)std::max<int64_t>(1, std::min<int64_t>(prm.top_k_fragments, l->max_frag));
  const int maxw = std::max(1, d->max_overlap);

  ADS_TRY(reserve_candidates(c, P * (int64_t)k_out));
  ADS_CUDA(cudaMemsetAsync(c->count_p, 0, sizeof(int64_t), st));
  ADS_CUDA(cudaMemsetAsync(c->err_p, 0, sizeof(int), st));
  c->pending = true;
  c->count = 0;
  if (P == 0 || k_out == 0) {
    s->last_launches = 0;
    if (!capturing) ADS_CUDA(cudaEventRecord(c->done, st));
    return ADS_OK;
  }

  const size_t Pn = (size_t)P;
  ADS_TRY(s->nf.reserve(Pn));
  ADS_TRY(s->cs.reserve(Pn));
  ADS_TRY(s->ce.reserve(Pn));
  ADS_TRY(s->nwin.reserve(Pn));
  ADS_TRY(s->wins.reserve(Pn * maxw));
  ADS_TRY(s->fw.reserve(Pn * kf));
  ADS_TRY(s->blo.reserve(Pn * kf));
  ADS_TRY(s->bhi.reserve(Pn * kf));
  const int64_t prep_blocks = std::min<int64_t>((P * 32 + kPrepThreads - 1) / kPrepThreads,
                                                 (int64_t)s->num_sms * 16);
  const int64_t keep_stride = std::max<int64_t>(l->max_frag, 1);
  ADS_TRY(s->keep.reserve((size_t)(prep_blocks * (kPrepThreads / 32) * keep_stride)));
  ADS_TRY(s->cand_n.reserve(Pn));
  ADS_TRY(s->cand_score.reserve(Pn * k_out));
  ADS_TRY(s->cand_center.reserve(Pn * k_out));
  ADS_TRY(s->work.reserve(2 * kMaxClasses));  // work counters, then class lengths
  // precursors taken heaviest first when their fragment counts differ (class lists
  // ordered by fragment count; a single class then gets a list too)
  const bool order = std::min<int64_t>(prm.top_k_fragments, l->min_frag) <
                     std::min<int64_t>(prm.top_k_fragments, l->max_frag);
  const bool use_lists = n_cls > 1 || order;
  if (use_lists) ADS_TRY(s->class_lists.reserve(Pn * n_cls));
  if (order) ADS_TRY(s->class_hist.reserve(2 * kMaxClasses * kOrderKeys));
  const int64_t nb = (P + kScanBlock - 1) / kScanBlock;
  ADS_TRY(s->block_sums.reserve((size_t)nb));
  if (s->stats_on) {
    ADS_TRY(s->stats.reserve(kStats));
    ADS_CUDA(cudaMemsetAsync(s->stats.p, 0, kStats * sizeof(unsigned long long), st));
  }

  GridView g;
  ADS_TRY(device_grid(s->device, &g));

  PrepArgs pa;
  pa.n_prec = P;
  pa.pmz = l->pmz_p;
  pa.prt = l->prt_p;
  pa.ptol = l->has_tol ? l->ptol_p : nullptr;
  pa.rt_tol = prm.rt_tolerance;
  pa.fstart = l->fstart_p;
  pa.fstop = l->fstop_p;
  pa.fmz = l->fmz_p;
  pa.fint = l->fint_p;
  pa.fnum = l->fnum_p;
  pa.ftype = l->ftype_p;
  pa.rt = d->rt_dev.p;
  pa.n_rt = (int)n_rt;
  pa.delta_t = d->delta_t;
  pa.pad = (float)prm.kernel_size;
  pa.win = d->win_dev.p;
  pa.n_obs = (int)d->n_obs;
  pa.g = g;
  pa.mass_tol = prm.mass_tolerance;
  pa.top_k = (int)std::min<int64_t>(prm.top_k_fragments, (int64_t)1 << 30);
  pa.kf = kf;
  pa.maxw = maxw;
  pa.min_c = std::max(L + 1, 5);
  pa.keep = s->keep.p;
  pa.keep_stride = keep_stride;
  pa.nf = s->nf.p;
  pa.cs = s->cs.p;
  pa.ce = s->ce.p;
  pa.nwin = s->nwin.p;
  pa.wins = s->wins.p;
  pa.fw = s->fw.p;
  pa.blo = s->blo.p;
  pa.bhi = s->bhi.p;
  pa.err = c->err_p;
  ADS_CUDA(cudaMemsetAsync(s->work.p, 0, 2 * kMaxClasses * sizeof(unsigned long long), st));
  const bool timed = !capturing && s->o.time_stages != 0 && s->stage_used < 65536;
  if (timed) {
    if (s->stage_used == s->stage_pool.size()) {
      std::array<cudaEvent_t, 4> set{};
      for (auto& e : set) ADS_CUDA(cudaEventCreate(&e));
      s->stage_pool.push_back(set);
    }
    s->stage_ev = s->stage_pool[s->stage_used].data();
    ADS_CUDA(cudaEventRecord(s->stage_ev[0], st));
  }
  {
    const size_t prep_smem = plan_prep_smem(&pa);
    prep_kernel<<<(int)prep_blocks, kPrepThreads, prep_smem, st>>>(pa);
    ADS_LAUNCH_CHECK();
    ++launches;
    if (s->stats_on && P > 0) {
      cells_kernel<<<(int)std::min<int64_t>((P + 255) / 256, 1184), 256, 0, st>>>(
          P, s->nf.p, s->cs.p, s->ce.p, s->stats.p + 6);
      ADS_LAUNCH_CHECK();
      ++launches;
    }
  }

  const double2* ln_tab = nullptr;
  ADS_TRY(device_ln_table(s->device, &ln_tab));
  if (bf16) ADS_TRY(ensure_bf16_intensities(const_cast<AdsDia*>(d), st));
  int max_smem = 0;
  ADS_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));

  SearchArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.n_prec = P;
  sa.nf = s->nf.p;
  sa.cs = s->cs.p;
  sa.ce = s->ce.p;
  sa.nwin = s->nwin.p;
  sa.wins = s->wins.p;
  sa.maxw = maxw;
  sa.fw = s->fw.p;
  sa.blo = s->blo.p;
  sa.bhi = s->bhi.p;
  sa.kf = kf;
  sa.win = d->win_dev.p;
  sa.ss = d->slice_starts.p;
  sa.cyc = d->cycles.p;
  sa.inten = d->intens.p;
  sa.inten_bf16 = d->intens_bf16.p;
  sa.ln_tab = ln_tab;
  set_taps(&sa, s->kernel.data(), s->h, s->taps.p);
  sa.h = s->h;
  sa.k_out = k_out;
  sa.gather_mode = s->o.gather_mode;
  sa.scan_thresh = 4 * 32 * (bf16 ? kPrefetchChunks<true> : kPrefetchChunks<false>);
  sa.err = c->err_p;
  sa.cand_n = s->cand_n.p;
  sa.cand_score = s->cand_score.p;
  sa.cand_center = s->cand_center.p;
  sa.stats = s->stats_on ? s->stats.p : nullptr;
  if (timed) ADS_CUDA(cudaEventRecord(s->stage_ev[1], st));
  unsigned int* class_len = reinterpret_cast<unsigned int*>(s->work.p + kMaxClasses);
  if (order) {
    const int cb = (int)std::min<int64_t>((P + 255) / 256, (int64_t)s->num_sms * 8);
    unsigned int* hist = s->class_hist.p;
    unsigned int* cursor = s->class_hist.p + kMaxClasses * kOrderKeys;
    ADS_CUDA(cudaMemsetAsync(hist, 0, (size_t)n_cls * kOrderKeys * sizeof(unsigned int), st));
    class_hist_kernel<<<cb, 256, 0, st>>>(P, s->nf.p, s->cs.p, s->ce.p, n_cls, cls, hist, s->cand_n.p);
    ADS_LAUNCH_CHECK();
    class_offsets_kernel<<<1, kOrderKeys, 0, st>>>(n_cls, hist, cursor, class_len);
    ADS_LAUNCH_CHECK();
    class_scatter_kernel<<<cb, 256, 0, st>>>(P, s->nf.p, s->cs.p, s->ce.p, n_cls, cls, cursor,
                                             s->class_lists.p);
    ADS_LAUNCH_CHECK();
    launches += 3;
  } else if (n_cls > 1) {
    const int cb = (int)std::min<int64_t>((P + 255) / 256, (int64_t)s->num_sms * 8);
    classify_kernel<<<cb, 256, 0, st>>>(P, s->nf.p, s->cs.p, s->ce.p, n_cls, cls,
                                         s->class_lists.p, class_len, s->cand_n.p);
    ADS_LAUNCH_CHECK();
    ++launches;
  }
  for (int b = 0; b < n_cls; ++b) {
    int S = cls.S[b];
    const int cmax_b = cls.bound[b];
    // block shape: warps per block (one precursor per warp at a time); 4 by default,
    // which packs long-window classes into shared memory better than 8
    bool grow = cmax_b > kSmemMaxCycles;
    int nw = s->o.warps_per_block > 0 ? s->o.warps_per_block : kDefaultWarpsPerBlock;
    if (!grow && search_smem_bytes(1, S, s->h, (cmax_b + 32 * S - 1) / (32 * S) * 32 * S, false) >
                     (size_t)max_smem)
      grow = true;  // a very wide kernel: even one warp's plan exceeds shared memory
    if (grow) S = kGrowLaneCycles;
    nw = std::max(1, std::min(nw, max_warps_per_block(bf16, s->h, grow, s->stats_on)));
    const int ncell_b = (cmax_b + 32 * S - 1) / (32 * S) * 32 * S;
    while (nw > 1 && search_smem_bytes(nw, S, s->h, ncell_b, grow) > (size_t)max_smem) --nw;
    const size_t smem = search_smem_bytes(nw, S, s->h, ncell_b, grow);
    if (smem > (size_t)max_smem)
      return fail(ADS_ERR_INTERNAL, "search kernel plan exceeds shared memory (" +
                                        std::to_string(cmax_b) + " cycles)");
    void (*kern)(SearchArgs) = pick_search_kernel(s->h, S, bf16, grow, s->stats_on);
    ADS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    ADS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, nw * 32, smem));
    if (occ <= 0) return fail(ADS_ERR_INTERNAL, "search kernel cannot be resident");
    const int bps = s->o.blocks_per_sm > 0 ? std::min(s->o.blocks_per_sm, occ) : occ;
    sa.list = use_lists ? s->class_lists.p + (int64_t)b * P : nullptr;
    sa.list_len = use_lists ? class_len + b : nullptr;
    sa.c_max = cmax_b;
    sa.ncell = ncell_b;
    sa.work = s->work.p + b;
    int64_t blocks = std::min<int64_t>((int64_t)s->num_sms * bps, (P + nw - 1) / nw);
    sa.grow = nullptr;
    if (grow) {
      const size_t warp_bytes = (size_t)warp_plan(S, s->h, ncell_b).total * 4;
      blocks = grow_blocks(blocks, nw, warp_bytes, (size_t)kGrowBudgetBytes);
      ADS_TRY(s->grow.reserve((size_t)blocks * nw * warp_bytes / 4));
      sa.grow = s->grow.p;
    }
    kern<<<(int)blocks, nw * 32, smem, st>>>(sa);
    ADS_LAUNCH_CHECK();
    ++launches;
  }
  if (timed) ADS_CUDA(cudaEventRecord(s->stage_ev[2], st));

  block_sum_kernel<<<(int)nb, kScanBlock, 0, st>>>(s->cand_n.p, P, s->block_sums.p);
  ADS_LAUNCH_CHECK();
  scan_block_sums_kernel<<<1, kScanBlock, 0, st>>>(s->block_sums.p, nb, c->count_p);
  ADS_LAUNCH_CHECK();
  ScatterArgs ca;
  ca.n_prec = P;
  ca.k_out = k_out;
  ca.peak_length = (uint64_t)prm.peak_length;
  ca.rt_len = (uint64_t)n_rt;
  ca.cand_n = s->cand_n.p;
  ca.cand_score = s->cand_score.p;
  ca.cand_center = s->cand_center.p;
  ca.pidx = l->pidx_p;
  ca.block_off = s->block_sums.p;
  ca.o_pidx = c->pidx_p;
  ca.o_rank = c->rank_p;
  ca.o_score = c->score_p;
  ca.o_center = c->center_p;
  ca.o_start = c->start_p;
  ca.o_stop = c->stop_p;
  scatter_kernel<<<(int)nb, kScanBlock, 0, st>>>(ca);
  ADS_LAUNCH_CHECK();
  launches += 3;
  if (timed) {
    ADS_CUDA(cudaEventRecord(s->stage_ev[3], st));
    ++s->stage_used;
  }
  s->last_launches = launches;
  if (!capturing) ADS_CUDA(cudaEventRecord(c->done, st));
  return ADS_OK;
}

// ------------------------------------------------------------------ autotuner
// Launch shapes of the search kernel: warps per block (precursors in flight per
// CTA) and cycles per lane (0 = length classes, else one fixed width), timed on the
// caller's run and library; the fastest is kept in the selection's options and
// cached per workload shape for the rest of the process.
struct TuneKey {
  int device, precision, h;
  int64_t c_max, P, kf, n_frag;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, precision, h, c_max, P, kf, n_frag) <
           std::tie(o.device, o.precision, o.h, o.c_max, o.P, o.kf, o.n_frag);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::array<float, 3>> g_tune_cache;  // warps, cycles per lane, ms

int autotune(AdsSelection* s, const AdsDia* d, const AdsLib* l, int32_t repeats,
             int32_t* out_warps, int32_t* out_cycles, float* out_ms) {
  if (!s || !d || !l) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
  if (d->device != s->device || l->device != s->device)
    return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
  repeats = std::max(1, std::min<int32_t>(repeats, 100));
  const float tol_max = l->has_tol ? std::max(l->max_tol, 0.0f) : s->p.rt_tolerance;
  const TuneKey key{s->device, s->o.precision, s->h,
                    max_cycle_span(d->rt, d->delta_t, tol_max, s->p.kernel_size), l->n_prec,
                    std::min<int64_t>(s->p.top_k_fragments, l->max_frag), l->n_frag};
  std::array<float, 3> best{0.0f, 0.0f, -1.0f};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) best = it->second;
  }
  if (best[2] < 0.0f) {
    DeviceGuard dg(s->device);
    cudaStream_t st = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
    struct Restore {  // the caller's options come back on every exit path
      AdsSelection* s;
      AdsEngineOptions o;
      ~Restore() { s->o = o; }
    } restore{s, s->o};
    s->o.use_graph = 0;
    s->o.time_stages = 0;
    AdsCandidates scratch;
    scratch.device = s->device;
    int rc = ADS_OK;
    for (int nw : {2, 4, 8}) {
      if (nw > max_warps_per_block(s->o.precision == ADS_PRECISION_BF16, s->h, false, false))
        continue;
      for (int S : {0, 4, 8, 10, 12, 16}) {
        if (S != 0 && (int64_t)32 * S * 8 < key.c_max) continue;  // more than 8 passes
        s->o.warps_per_block = nw;
        s->o.cycles_per_lane = S;
        rc = enqueue_search(s, d, l, &scratch, false);  // warm-up (and buffer sizing)
        float total = 0.0f;
        for (int r = 0; rc == ADS_OK && r < repeats; ++r) {
          ADS_CUDA(cudaEventRecord(s->ev0, st));
          rc = enqueue_search(s, d, l, &scratch, false);
          ADS_CUDA(cudaEventRecord(s->ev1, st));
          ADS_CUDA(cudaEventSynchronize(s->ev1));
          float ms = 0.0f;
          ADS_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
          total += ms;
        }
        if (rc != ADS_OK) break;
        const float ms = total / repeats;
        if (best[2] < 0.0f || ms < best[2]) best = {(float)nw, (float)S, ms};
      }
      if (rc != ADS_OK) break;
    }
    ADS_CUDA(cudaStreamSynchronize(st));
    if (rc != ADS_OK) return rc;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  s->o.warps_per_block = (int32_t)best[0];
  s->o.cycles_per_lane = (int32_t)best[1];
  if (s->graph) {  // captured with the previous shape
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  if (out_warps) *out_warps = (int32_t)best[0];
  if (out_cycles) *out_cycles = (int32_t)best[1];
  if (out_ms) *out_ms = best[2];
  return ADS_OK;
}

// Everything a captured search depends on: the handles and every buffer address.
// Everything a captured pipeline bakes in: the handles, every buffer it reads or
// writes, and the run- and library-derived sizes its launch plan depends on (a handle
// released and another created at the same address must not replay a stale graph).
std::vector<const void*> graph_key(const AdsSelection* s, const AdsDia* d, const AdsLib* l,
                                   const AdsCandidates* c) {
  auto v = [](int64_t x) { return reinterpret_cast<const void*>(static_cast<intptr_t>(x)); };
  uint32_t tol_bits = 0;
  std::memcpy(&tol_bits, &l->max_tol, sizeof(tol_bits));
  return {d, l, c, c->arena.p, s->nf.p, s->cs.p, s->ce.p, s->nwin.p, s->wins.p, s->fw.p,
          s->blo.p, s->bhi.p, s->keep.p, s->cand_n.p, s->cand_score.p, s->cand_center.p,
          s->work.p, s->class_lists.p, s->class_hist.p, s->block_sums.p,
          s->stats_on ? s->stats.p : nullptr,
          d->intens_bf16.p, s->grow.p, s->taps.p,
          d->slice_starts.p, d->cycles.p, d->intens.p, d->win_dev.p, d->rt_dev.p, v(d->n_obs),
          v((int64_t)d->rt.size()), v(d->max_overlap),
          l->arena.p, v(l->n_prec), v(l->n_frag), v(l->max_frag), v(l->min_frag), v(l->has_tol),
          v(tol_bits)};
}

// A search, with use_graph: the first search of a (run, library, collection) runs
// directly (sizing every buffer) and is then captured into a CUDA graph; later
// searches with the same handles and buffers replay the graph in one launch.
int launch_search(AdsSelection* s, const AdsDia* d, const AdsLib* l, AdsCandidates* c) {
  if (!s->o.use_graph) return enqueue_search(s, d, l, c, false);
  DeviceGuard dg(s->device);
  cudaStream_t st = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
  if (s->graph && c->done && graph_key(s, d, l, c) == s->graph_key) {
    ADS_TRY(lib_ready_on(l, st));
    ADS_CUDA(cudaStreamWaitEvent(st, c->done, 0));
    c->pending = true;
    c->count = 0;
    ADS_CUDA(cudaGraphLaunch(s->graph, st));
    s->last_launches = s->graph_launches;
    ADS_CUDA(cudaEventRecord(c->done, st));
    return ADS_OK;
  }
  ADS_TRY(enqueue_search(s, d, l, c, false));
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  const int64_t launches = s->last_launches;
  cudaGraph_t g = nullptr;
  ADS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue_search(s, d, l, c, true);
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (rc != ADS_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  cudaGraphExec_t ex = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate", __FILE__, __LINE__);
  s->graph = ex;
  s->graph_key = graph_key(s, d, l, c);
  s->graph_launches = launches;
  s->last_launches = launches;
  return ADS_OK;
}

int finish(AdsCandidates* c) {
  if (!c->pending) return ADS_OK;
  DeviceGuard dg(c->device);
  int64_t cnt = 0;
  int err = 0;
  ADS_CUDA(cudaStreamWaitEvent(cudaStreamPerThread, c->done, 0));
  ADS_CUDA(cudaMemcpyAsync(&cnt, c->count_p, sizeof(int64_t), cudaMemcpyDeviceToHost,
                           cudaStreamPerThread));
  ADS_CUDA(cudaMemcpyAsync(&err, c->err_p, sizeof(int), cudaMemcpyDeviceToHost, cudaStreamPerThread));
  ADS_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
  c->pending = false;
  if (err)
    return fail(ADS_ERR_INTERNAL, "search kernel reported internal error flags " + std::to_string(err));
  c->count = cnt;
  return ADS_OK;
}

}  // namespace
}  // namespace ads

using namespace ads;

extern "C" {

void ads_selection_params_default(AdsSelectionParams* p) {
  if (!p) return;
  // SelectionParameters::new (src/peak_group_selection/parameters.rs:24-43)
  p->fwhm_rt = 3.0f;
  p->kernel_size = 20;
  p->peak_length = 5;
  p->mass_tolerance = 7.0f;
  p->rt_tolerance = 200.0f;
  p->candidate_count = 3;
  p->top_k_fragments = 12;
}

void ads_engine_options_default(AdsEngineOptions* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
}

int ads_gaussian_kernel(float fwhm_rt, float sigma_scale_rt, int64_t kernel_width,
                        float rt_resolution, float* out, int64_t cap, int64_t* n) {
  return guarded([&] {
    if (kernel_width < 0 || kernel_width > (int64_t(1) << 24))
      return fail(ADS_ERR_INVALID_ARGUMENT, "kernel_width outside [0, 2^24]");
    auto w = gaussian_kernel(fwhm_rt, sigma_scale_rt, kernel_width, rt_resolution);
    if (n) *n = (int64_t)w.size();
    if (out) std::memcpy(out, w.data(), (size_t)std::min<int64_t>(cap, (int64_t)w.size()) * 4);
    return ADS_OK;
  });
}

int ads_selection_create(const AdsSelectionParams* params, const AdsEngineOptions* options,
                         int device, AdsSelection** out) {
  return guarded([&] {
    if (!params || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto s = std::make_unique<AdsSelection>();
    s->p = *params;
    if (options)
      s->o = *options;
    else
      ads_engine_options_default(&s->o);
    if (s->o.precision != ADS_PRECISION_FP32 && s->o.precision != ADS_PRECISION_BF16)
      return fail(ADS_ERR_INVALID_ARGUMENT, "precision must be ADS_PRECISION_FP32 or _BF16");
    if (s->o.gather_mode < 0 || s->o.gather_mode > 2)
      return fail(ADS_ERR_INVALID_ARGUMENT, "gather_mode must be 0, 1 or 2");
    ADS_TRY(check_params(s->p, &s->kernel, &s->h));
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
      cudaGetLastError();
      return fail(ADS_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= n_dev) return fail(ADS_ERR_INVALID_ARGUMENT, "bad device index");
    s->device = device;
    DeviceGuard dg(device);
    ADS_CUDA(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device));
    if (!s->o.stream) {
      ADS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
      s->own_stream = true;
    } else {
      s->stream = (cudaStream_t)s->o.stream;
    }
    ADS_CUDA(cudaEventCreate(&s->ev0));
    ADS_CUDA(cudaEventCreate(&s->ev1));
    if (s->h > kMaxHalf) {  // wide kernels: taps from device memory
      ADS_TRY(s->taps.alloc(s->kernel.size()));
      ADS_CUDA(cudaMemcpy(s->taps.p, s->kernel.data(), s->kernel.size() * 4, cudaMemcpyHostToDevice));
      ADS_CUDA(cudaDeviceSynchronize());  // the upload has landed before any search reads it
    }
    *out = s.release();
    return ADS_OK;
  });
}

int ads_selection_destroy(AdsSelection* s) {
  return guarded([&] {
    if (!s) return ADS_OK;
    DeviceGuard dg(s->device);
    cudaStreamSynchronize(s->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    for (auto& set : s->stage_pool)
      for (auto e : set) cudaEventDestroy(e);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
    return ADS_OK;
  });
}

int ads_selection_kernel(const AdsSelection* s, float* out, int64_t cap, int64_t* n) {
  return guarded([&] {
    if (!s) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    if (n) *n = (int64_t)s->kernel.size();
    if (out) std::memcpy(out, s->kernel.data(), (size_t)std::min<int64_t>(cap, s->kernel.size()) * 4);
    return ADS_OK;
  });
}

int64_t ads_selection_stream(const AdsSelection* s) {
  return s ? (int64_t)(s->o.stream ? (cudaStream_t)s->o.stream : s->stream) : 0;
}

int64_t ads_selection_last_launches(const AdsSelection* s) { return s ? s->last_launches : 0; }

int ads_selection_set_stats(AdsSelection* s, int enabled) {
  if (!s) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
  s->stats_on = enabled != 0;
  return ADS_OK;
}

int ads_selection_stage_times(AdsSelection* s, float* ms, int64_t cap) {
  return guarded([&] {
    if (!s || !ms) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    if (s->stage_used == 0) return fail(ADS_ERR_INVALID_ARGUMENT, "no timed search recorded");
    DeviceGuard dg(s->device);
    ADS_CUDA(cudaEventSynchronize(s->stage_pool[s->stage_used - 1][3]));
    double sum[3] = {0, 0, 0};
    for (size_t k = 0; k < s->stage_used; ++k)
      for (int i = 0; i < 3; ++i) {
        float t = 0.0f;
        ADS_CUDA(cudaEventElapsedTime(&t, s->stage_pool[k][i], s->stage_pool[k][i + 1]));
        sum[i] += t;
      }
    for (int i = 0; i < 3 && i < cap; ++i) ms[i] = (float)sum[i];
    if (cap > 3) ms[3] = (float)s->stage_used;
    s->stage_used = 0;
    return ADS_OK;
  });
}

int ads_selection_last_stats(AdsSelection* s, int64_t* out, int64_t cap) {
  return guarded([&] {
    if (!s || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    if (!s->stats_on || !s->stats.p) return fail(ADS_ERR_INVALID_ARGUMENT, "statistics not enabled");
    DeviceGuard dg(s->device);
    unsigned long long v[kStats];
    cudaStream_t st = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
    ADS_CUDA(cudaMemcpyAsync(v, s->stats.p, sizeof(v), cudaMemcpyDeviceToHost, st));
    ADS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < kStats && i < cap; ++i) out[i] = (int64_t)v[i];
    return ADS_OK;
  });
}

int ads_candidates_create(const AdsSelection* s, AdsCandidates** out) {
  return guarded([&] {
    if (!s || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    auto c = std::make_unique<AdsCandidates>();
    c->device = s->device;
    *out = c.release();
    return ADS_OK;
  });
}

int ads_selection_autotune(AdsSelection* s, const AdsDia* d, const AdsLib* l, int32_t repeats,
                           int32_t* warps_per_block, int32_t* cycles_per_lane, float* best_ms) {
  return guarded([&] { return autotune(s, d, l, repeats, warps_per_block, cycles_per_lane, best_ms); });
}

int ads_select_async(AdsSelection* s, const AdsDia* d, const AdsLib* l, AdsCandidates* c) {
  return guarded([&] {
    if (!s || !d || !l || !c) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    return launch_search(s, d, l, c);
  });
}

int ads_select(AdsSelection* s, const AdsDia* d, const AdsLib* l, AdsCandidates** out) {
  return guarded([&] {
    if (!s || !d || !l || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto c = std::make_unique<AdsCandidates>();
    c->device = s->device;
    DeviceGuard dg(s->device);
    cudaStream_t st = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
    if (s->o.verbose) ADS_CUDA(cudaEventRecord(s->ev0, st));
    ADS_TRY(launch_search(s, d, l, c.get()));
    if (s->o.verbose) ADS_CUDA(cudaEventRecord(s->ev1, st));
    ADS_TRY(finish(c.get()));
    if (s->o.verbose) {
      float ms = 0.0f;
      ADS_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
      // src/peak_group_selection/mod.rs:123-125
      printf("Precursors per second: %.1f\n", (double)l->n_prec / std::max(1e-9, ms * 1e-3));
      printf("Found %lld candidates\n", (long long)c->count);
      fflush(stdout);
    }
    if (s->stats_on) {
      s->last_stats[0] = l->n_prec;
    }
    *out = c.release();
    return ADS_OK;
  });
}

int64_t ads_candidates_size(AdsCandidates* c) {
  if (!c) return -1;
  int rc = guarded([&] { return finish(c); });
  return rc == ADS_OK ? c->count : -1;
}

int ads_candidates_copy_out(AdsCandidates* c, uint64_t* pidx, uint64_t* rank, float* score,
                            uint64_t* scan_center, uint64_t* scan_start, uint64_t* scan_stop,
                            uint64_t* center, uint64_t* start, uint64_t* stop) {
  return guarded([&] {
    if (!c) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    ADS_TRY(finish(c));
    const size_t n = (size_t)c->count;
    if (n == 0) return ADS_OK;
    DeviceGuard dg(c->device);
    struct Col {
      void* dst;
      const void* src;
      size_t bytes;
    } cols[] = {{pidx, c->pidx_p, 8}, {rank, c->rank_p, 8},   {score, c->score_p, 4},
                {center, c->center_p, 8}, {start, c->start_p, 8}, {stop, c->stop_p, 8}};
    for (auto& col : cols)
      if (col.dst)
        ADS_CUDA(cudaMemcpyAsync(col.dst, col.src, n * col.bytes, cudaMemcpyDeviceToHost,
                                 cudaStreamPerThread));
    // the reference's scan_* columns are zero: written on the host while the copies
    // run, one thread per column when they are large (one thread fills about 10 GB/s)
    uint64_t* zeros[3] = {scan_center, scan_start, scan_stop};
    if (n >= ((size_t)1 << 20)) {
      std::vector<std::thread> fill;
      for (uint64_t* z : zeros)
        if (z) fill.emplace_back([z, n] { std::memset(z, 0, n * 8); });
      for (auto& t : fill) t.join();
    } else {
      for (uint64_t* z : zeros)
        if (z) std::memset(z, 0, n * 8);
    }
    ADS_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
    return ADS_OK;
  });
}

int ads_dia_keep_bf16_only(AdsDia* d) {
  return guarded([&] {
    if (!d) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    DeviceGuard dg(d->device);
    cudaStream_t st = nullptr;
    ADS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const int rc = ensure_bf16_intensities(d, st);
    cudaStreamDestroy(st);
    if (rc != ADS_OK) return rc;
    std::lock_guard<std::mutex> lk(d->mu);
    d->intens.release();  // waits for the device to go idle first
    d->bf16_only = true;
    return ADS_OK;
  });
}

int ads_candidates_destroy(AdsCandidates* c) {
  return guarded([&] {
    if (!c) return ADS_OK;
    DeviceGuard dg(c->device);
    delete c;
    return ADS_OK;
  });
}

}  // extern "C"

// ------------------------------------------------------- allocation-free search
//
// ads_select_noalloc serves callers that may not allocate device memory at search
// time: processes whose device memory belongs to another allocator (a framework's
// caching allocator, a serving process on a fixed memory budget), where a
// cudaMalloc from this library could fail or fragment that memory, and loops that
// cannot afford cudaFree's implicit device-wide synchronisation.  Its working
// memory is the fixed array below, which exists once in every GPU context that
// loads this library, for the life of the process.

static __device__ __align__(256) unsigned char g_noalloc_scratch[ADS_NOALLOC_SCRATCH_BYTES];

namespace ads {
namespace {

constexpr size_t kNoAllocLnBytes = kLnTableSize * sizeof(double2);  // first 4 KiB: ln table

std::mutex g_noalloc_mu;
std::map<int, char*> g_noalloc_base;  // device -> device address of g_noalloc_scratch

// The scratch array's device address on the current device, set up on first use:
// host code only knows the array through a stand-in symbol, so the address comes
// from cudaGetSymbolAddress (with the device current), and the ln table is copied
// into the array's first 4 KiB.  The device must be current.
int noalloc_scratch(int device, char** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  auto it = g_noalloc_base.find(device);
  if (it != g_noalloc_base.end()) {
    *out = it->second;
    return ADS_OK;
  }
  void* p = nullptr;
  ADS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  const std::vector<double2> tab = host_ln_table();
  ADS_CUDA(cudaMemcpy(p, tab.data(), kNoAllocLnBytes, cudaMemcpyHostToDevice));
  // a copy from pageable memory may return before its DMA ends; the search kernels
  // run on the caller's stream, which need not wait for the legacy stream
  ADS_CUDA(cudaDeviceSynchronize());
  g_noalloc_base[device] = static_cast<char*>(p);
  *out = static_cast<char*>(p);
  return ADS_OK;
}

// Bump allocator over the scratch array (256-byte aligned pieces); `end` tells
// whether everything fitted.
struct ScratchCarver {
  char* base;
  size_t off;
  template <class T>
  T* take(int64_t n) {
    T* p = reinterpret_cast<T*>(base + off);
    off += ((size_t)std::max<int64_t>(n, 1) * sizeof(T) + 255) / 256 * 256;
    return p;
  }
};

int select_noalloc(const AdsDia* d, const AdsLib* l, const AdsSelectionParams* params,
                   int64_t stream, int64_t capacity, uint64_t* o_pidx, uint64_t* o_rank,
                   float* o_score, uint64_t* o_center, uint64_t* o_start, uint64_t* o_stop,
                   int64_t* o_count, int32_t* o_flags) {
  if (!d || !l || !params || !o_count) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
  if (!o_flags)
    return fail(ADS_ERR_INVALID_ARGUMENT,
                "flags must point to a device int32: the kernels report internal errors there");
  if (d->device != l->device) return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
  std::vector<float> kernel;
  int h = 0;
  ADS_TRY(check_params(*params, &kernel, &h));
  ADS_TRY(need_f32_intensities(d, "ads_select_noalloc (an FP32 search)"));
  const AdsSelectionParams& prm = *params;
  DeviceGuard dg(d->device);
  char* base = nullptr;
  ADS_TRY(noalloc_scratch(d->device, &base));
  const cudaStream_t st = (cudaStream_t)stream;
  // after the library's preparation; a capturing stream cannot wait on work outside
  // its capture, so there the library must be prepared already (documented)
  cudaStreamCaptureStatus capst = cudaStreamCaptureStatusNone;
  ADS_CUDA(cudaStreamIsCapturing(st, &capst));
  if (capst == cudaStreamCaptureStatusNone) ADS_TRY(lib_ready_on(l, st));

  // the same launch shape as ads_select with default engine options
  const int64_t P = l->n_prec;
  const int L = (int)kernel.size();
  const int64_t n_rt = (int64_t)d->rt.size();
  const float tol_max = l->has_tol ? std::max(l->max_tol, 0.0f) : prm.rt_tolerance;
  const int64_t c_max = std::max<int64_t>(1, max_cycle_span(d->rt, d->delta_t, tol_max, prm.kernel_size));
  // windows beyond the shared-memory plan (or a kernel too wide for it): one
  // long-window launch whose warps' working sets are carved from the scratch
  int max_smem = 0;
  ADS_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device));
  const int S0 = best_lane_cycles(c_max);
  const bool grow =
      c_max > kSmemMaxCycles ||
      search_smem_bytes(1, S0, h, (int)((c_max + 32 * S0 - 1) / (32 * S0) * 32 * S0)) > (size_t)max_smem;
  const int S = grow ? kGrowLaneCycles : S0;
  const int ncell = (int)((c_max + 32 * S - 1) / (32 * S) * 32 * S);
  const int k_out = (int)std::max<int64_t>(0, std::min<int64_t>(prm.candidate_count, maxima_cap(ncell)));
  const int kf = (int)std::max<int64_t>(1, std::min<int64_t>(prm.top_k_fragments, l->max_frag));
  const int maxw = std::max(1, d->max_overlap);
  const int64_t rows_needed = P * (int64_t)k_out;
  if (capacity < rows_needed)
    return fail(ADS_ERR_INVALID_ARGUMENT,
                "output capacity " + std::to_string(capacity) + " is below precursors x candidates = " +
                    std::to_string(rows_needed));
  if (rows_needed > 0 && (!o_pidx || !o_rank || !o_score || !o_center || !o_start || !o_stop))
    return fail(ADS_ERR_INVALID_ARGUMENT, "null output array");

  // scratch layout after the ln table
  int n_sms = 0;
  ADS_CUDA(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, d->device));
  const int64_t prep_blocks = std::min<int64_t>((P * 32 + kPrepThreads - 1) / kPrepThreads,
                                                 (int64_t)n_sms * 16);
  const int64_t keep_stride = std::max<int64_t>(l->max_frag, 1);
  const int64_t nb = (P + kScanBlock - 1) / kScanBlock;
  ScratchCarver sc{base, kNoAllocLnBytes};
  auto* work = sc.take<unsigned long long>(1);
  auto* err = sc.take<int>(1);
  auto* nf = sc.take<int>(P);
  auto* cs = sc.take<int>(P);
  auto* ce = sc.take<int>(P);
  auto* nwin = sc.take<int>(P);
  auto* wins = sc.take<int>(P * maxw);
  auto* fw = sc.take<float>(P * kf);
  auto* blo = sc.take<uint32_t>(P * kf);
  auto* bhi = sc.take<uint32_t>(P * kf);
  auto* keep = sc.take<uint8_t>(prep_blocks * (kPrepThreads / 32) * keep_stride);
  auto* cand_n = sc.take<int>(P);
  auto* cand_score = sc.take<float>(P * k_out);
  auto* cand_center = sc.take<int>(P * k_out);
  auto* block_sums = sc.take<int64_t>(nb);
  float* taps = h > kMaxHalf ? sc.take<float>(L) : nullptr;  // wide kernels: taps on the device
  // long windows: at least one block of warps' working sets must fit after the rest
  const int nw0 = kDefaultWarpsPerBlock;
  const size_t grow_warp_bytes = grow ? (size_t)warp_plan(S, h, ncell).total * 4 : 0;
  float* grow_sets = nullptr;
  size_t grow_bytes = 0;
  if (grow) {  // the rest of the array, which must hold one block's working sets
    grow_sets = reinterpret_cast<float*>(sc.base + sc.off);
    const size_t need = (size_t)nw0 * grow_warp_bytes;
    grow_bytes = sc.off < (size_t)ADS_NOALLOC_SCRATCH_BYTES ? (size_t)ADS_NOALLOC_SCRATCH_BYTES - sc.off : 0;
    sc.off += grow_bytes >= need ? grow_bytes : need;
  }
  if (sc.off > (size_t)ADS_NOALLOC_SCRATCH_BYTES)
    return fail(ADS_ERR_INVALID_ARGUMENT,
                "this search needs " + std::to_string(sc.off) + " bytes of scratch, more than the " +
                    std::to_string((size_t)ADS_NOALLOC_SCRATCH_BYTES) +
                    " of ads_select_noalloc; search the library in smaller parts");
  int* flags = reinterpret_cast<int*>(o_flags);
  (void)err;

  // what must start at zero: the work counter, the error flags and the count
  ADS_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned long long), st));
  ADS_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), st));
  ADS_CUDA(cudaMemsetAsync(o_count, 0, sizeof(int64_t), st));
  if (P == 0 || k_out == 0) return ADS_OK;

  // the grid exists: building `d` uploaded it to this device
  GridView g;
  ADS_TRY(device_grid(d->device, &g));
  PrepArgs pa;
  pa.n_prec = P;
  pa.pmz = l->pmz_p;
  pa.prt = l->prt_p;
  pa.ptol = l->has_tol ? l->ptol_p : nullptr;
  pa.rt_tol = prm.rt_tolerance;
  pa.fstart = l->fstart_p;
  pa.fstop = l->fstop_p;
  pa.fmz = l->fmz_p;
  pa.fint = l->fint_p;
  pa.fnum = l->fnum_p;
  pa.ftype = l->ftype_p;
  pa.rt = d->rt_dev.p;
  pa.n_rt = (int)n_rt;
  pa.delta_t = d->delta_t;
  pa.pad = (float)prm.kernel_size;
  pa.win = d->win_dev.p;
  pa.n_obs = (int)d->n_obs;
  pa.g = g;
  pa.mass_tol = prm.mass_tolerance;
  pa.top_k = (int)std::min<int64_t>(prm.top_k_fragments, (int64_t)1 << 30);
  pa.kf = kf;
  pa.maxw = maxw;
  pa.min_c = std::max(L + 1, 5);
  pa.keep = keep;
  pa.keep_stride = keep_stride;
  pa.nf = nf;
  pa.cs = cs;
  pa.ce = ce;
  pa.nwin = nwin;
  pa.wins = wins;
  pa.fw = fw;
  pa.blo = blo;
  pa.bhi = bhi;
  pa.err = flags;
  const size_t prep_smem = plan_prep_smem(&pa);
  prep_kernel<<<(int)prep_blocks, kPrepThreads, prep_smem, st>>>(pa);
  ADS_LAUNCH_CHECK();

  int nw = nw0;
  while (nw > 1 && search_smem_bytes(nw, S, h, ncell, grow) > (size_t)max_smem) --nw;
  const size_t smem = search_smem_bytes(nw, S, h, ncell, grow);
  if (smem > (size_t)max_smem)
    return fail(ADS_ERR_INTERNAL, "search kernel plan exceeds shared memory (" +
                                      std::to_string(c_max) + " cycles)");
  void (*kern)(SearchArgs) = pick_search_kernel(h, S, false, grow, false);
  ADS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  ADS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, nw * 32, smem));
  if (occ <= 0) return fail(ADS_ERR_INTERNAL, "search kernel cannot be resident");
  SearchArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.n_prec = P;
  sa.nf = nf;
  sa.cs = cs;
  sa.ce = ce;
  sa.nwin = nwin;
  sa.wins = wins;
  sa.maxw = maxw;
  sa.fw = fw;
  sa.blo = blo;
  sa.bhi = bhi;
  sa.kf = kf;
  sa.win = d->win_dev.p;
  sa.ss = d->slice_starts.p;
  sa.cyc = d->cycles.p;
  sa.inten = d->intens.p;
  sa.ln_tab = reinterpret_cast<const double2*>(base);
  if (taps)  // from pageable memory: returns once the bytes are staged, ordered on `st`
    ADS_CUDA(cudaMemcpyAsync(taps, kernel.data(), (size_t)L * 4, cudaMemcpyHostToDevice, st));
  set_taps(&sa, kernel.data(), h, taps);
  sa.h = h;
  sa.k_out = k_out;
  sa.c_max = (int)c_max;
  sa.ncell = ncell;
  sa.gather_mode = 0;
  sa.scan_thresh = 4 * 32 * kPrefetchChunks<false>;
  sa.work = work;
  sa.err = flags;
  sa.cand_n = cand_n;
  sa.cand_score = cand_score;
  sa.cand_center = cand_center;
  sa.stats = nullptr;
  int64_t blocks = std::min<int64_t>((int64_t)n_sms * occ, (P + nw - 1) / nw);
  sa.grow = nullptr;
  if (grow) {
    blocks = grow_blocks(blocks, nw, grow_warp_bytes, grow_bytes);
    sa.grow = grow_sets;
  }
  kern<<<(int)blocks, nw * 32, smem, st>>>(sa);
  ADS_LAUNCH_CHECK();

  block_sum_kernel<<<(int)nb, kScanBlock, 0, st>>>(cand_n, P, block_sums);
  ADS_LAUNCH_CHECK();
  scan_block_sums_kernel<<<1, kScanBlock, 0, st>>>(block_sums, nb, o_count);
  ADS_LAUNCH_CHECK();
  ScatterArgs ca;
  ca.n_prec = P;
  ca.k_out = k_out;
  ca.peak_length = (uint64_t)prm.peak_length;
  ca.rt_len = (uint64_t)n_rt;
  ca.cand_n = cand_n;
  ca.cand_score = cand_score;
  ca.cand_center = cand_center;
  ca.pidx = l->pidx_p;
  ca.block_off = block_sums;
  ca.o_pidx = o_pidx;
  ca.o_rank = o_rank;
  ca.o_score = o_score;
  ca.o_center = o_center;
  ca.o_start = o_start;
  ca.o_stop = o_stop;
  scatter_kernel<<<(int)nb, kScanBlock, 0, st>>>(ca);
  ADS_LAUNCH_CHECK();
  return ADS_OK;
}

}  // namespace
}  // namespace ads

extern "C" int ads_select_noalloc(const AdsDia* dia, const AdsLib* lib,
                                  const AdsSelectionParams* params, int64_t stream,
                                  int64_t capacity, uint64_t* precursor_idx, uint64_t* rank,
                                  float* score, uint64_t* cycle_center, uint64_t* cycle_start,
                                  uint64_t* cycle_stop, int64_t* count, int32_t* flags) {
  return ads::guarded([&] {
    return ads::select_noalloc(dia, lib, params, stream, capacity, precursor_idx, rank, score,
                               cycle_center, cycle_start, cycle_stop, count, flags);
  });
}
