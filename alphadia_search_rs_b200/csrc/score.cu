// PeakGroupScoring.score on the device (src/peak_group_scoring/mod.rs:42-340).
//
// One thread per candidate walks the reference's per-candidate steps in their
// order, so every f32 operation rounds as the reference's does:
//   1. the precursor by binary search of its precursor_idx, its fragments filtered
//      (non-zero, no y1), the top-k by intensity and sorted by m/z
//      (src/speclib_flat/mod.rs:240-345, 458-474);
//   2. the dense XIC and intensity-weighted m/z of every fragment over the
//      candidate's cycles (src/dense_xic_observation/mod.rs:97-137,
//      src/quadrupole_observation/mod.rs:152-211), read from the device CSR;
//   3. the 41 features (src/peak_group_scoring/mod.rs:124-338 and the helpers of
//      src/peak_group_scoring/utils.rs, src/utils/mod.rs, src/idf/mod.rs).
// f32::ln and f32::log10 are computed as ln / log10 rounded once from double; the
// reference calls glibc logf / log10f, which can differ in the last bit.  A
// correlation that comes out NaN or infinite, where the reference panics
// (src/peak_group_scoring/utils.rs:164-166), is 0 here.
//
// A thread's matrices (F x C dense XIC, m/z and normalised profiles) and vectors
// live in a global scratch interleaved across threads (element e of thread t at
// e * T + t), so threads working on the same element read consecutive words.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "common.cuh"

// Scored candidates, one row per input candidate (rows whose precursor_idx is not in
// the library are flagged and left out when read).
struct AdsFeatures {
  int device = 0;
  int64_t n = 0;
  int64_t count = 0;
  ads::DevBuf<char> arena;
  uint64_t* pidx_p = nullptr;
  uint64_t* rank_p = nullptr;
  float* feat_p = nullptr;  // feature k of row q at k * n + q
  uint8_t* found_p = nullptr;
  std::vector<uint8_t> found;
  float kernel_ms = 0.0f;  // CUDA-event time of score_kernel
};

// Quantified candidates (SpecLibFlatQuantified, src/speclib_flat_quantified/mod.rs:19-64),
// dense per candidate on the device until ads_quant_copy_out assembles the flat layout.
struct AdsQuant {
  int device = 0;
  int64_t n = 0, n_prec = 0, n_frag = 0;
  int Fm = 1;
  ads::DevBuf<char> arena;
  int* nq_p = nullptr;
  uint32_t* prow_p = nullptr;
  float* rt_p = nullptr;
  uint64_t* pidx_p = nullptr;
  uint64_t* rank_p = nullptr;
  uint64_t* frow_p = nullptr;
  float* fval_p[4] = {nullptr, nullptr, nullptr, nullptr};  // intensity, m/z, correlation, error
  float kernel_ms = 0.0f;
  // the flat SpecLibFlatQuantified layout, assembled on the device
  ads::DevBuf<char> flat;
  uint64_t *p_idx = nullptr, *p_row = nullptr, *p_rank = nullptr, *p_fs = nullptr, *p_fe = nullptr;
  float* p_rt = nullptr;
  uint64_t *f_row = nullptr, *f_pidx = nullptr, *f_rank = nullptr;
  float* f_val[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace ads {
namespace {

constexpr int kFeatures = 41;
constexpr int kScoreBlock = 128;

// src/candidate/features.rs:6-48
const char* const kFeatureNames[kFeatures] = {
    "score", "mean_correlation", "median_correlation", "correlation_std",
    "intensity_correlation", "num_fragments", "num_scans", "num_over_95", "num_over_90",
    "num_over_80", "num_over_50", "num_over_0", "num_over_0_rank_0_5", "num_over_0_rank_6_11",
    "num_over_0_rank_12_17", "num_over_0_rank_18_23", "num_over_50_rank_0_5",
    "num_over_50_rank_6_11", "num_over_50_rank_12_17", "num_over_50_rank_18_23",
    "hyperscore_intensity_observation", "hyperscore_intensity_library",
    "hyperscore_inverse_mass_error", "rt_observed", "delta_rt", "longest_b_series",
    "longest_y_series", "naa", "weighted_mass_error", "log10_b_ion_intensity",
    "log10_y_ion_intensity", "fwhm_rt", "idf_hyperscore", "idf_xic_dot_product",
    "idf_intensity_dot_product", "median_profile_sum", "median_profile_sum_filtered",
    "num_profiles", "num_profiles_filtered", "num_over_0_top6_idf", "num_over_50_top6_idf"};

struct ScoreArgs {
  int64_t n;
  const uint64_t *c_pidx, *c_rank, *c_center, *c_start, *c_stop;
  const float* c_score;
  int64_t P;
  const uint64_t* l_pidx;
  const float *l_pmz, *l_prt;
  const uint8_t* l_naa;
  const uint64_t *l_fs, *l_fe;
  const float *l_fmz, *l_fmzl, *l_fint;
  const uint8_t *l_fnum, *l_ftype;
  const uint32_t* idf_counts;
  float idf_total;
  const WinInfo* win;
  int n_obs;
  const uint32_t* ss;
  const uint16_t* cyc;
  const float* inten;
  const float* rt;
  int64_t n_rt;
  GridView g;
  float tol;
  int64_t top_k;
  int Fm, Fraw, Cm;  // scratch bounds: kept fragments, raw fragments, cycles
  uint32_t* scratch;
  int64_t T;  // threads, the scratch's element stride
  uint64_t* o_pidx;
  uint64_t* o_rank;
  float* o_feat;
  uint8_t* o_found;
  int* err;
  // nullable: the order in which the threads take the candidates (by their precursor's
  // library fragment count, so that the threads of a warp do similar work); results
  // are written at each candidate's own index either way
  const uint32_t* order;
};

// Words of one thread's scratch.
int64_t scratch_words(int Fm, int Fraw, int Cm) {
  return 3 * (int64_t)Fm * Cm + 18 * (int64_t)Fm + 2 * (int64_t)Cm + (int64_t)Fraw;
}

// One thread's view of the interleaved scratch.
struct Scr {
  uint32_t* base;
  int64_t T, t;
  __device__ float f(int64_t e) const { return __uint_as_float(base[e * T + t]); }
  __device__ void sf(int64_t e, float v) const { base[e * T + t] = __float_as_uint(v); }
  __device__ uint32_t u(int64_t e) const { return base[e * T + t]; }
  __device__ void su(int64_t e, uint32_t v) const { base[e * T + t] = v; }
};

__device__ __forceinline__ float log10_rn(float x) { return __double2float_rn(log10((double)x)); }

// Rust 1.88 slice::binary_search on u16 (the LAST of equal elements when found,
// else the insertion point), as fill_xic_and_mz_slice uses it.
__device__ __forceinline__ int64_t bsearch_u16_rust(const uint16_t* a, int64_t n, int x) {
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

// Iterator::sum on f32 (Rust 1.88): a left fold from -0.0.
__device__ float rust_sum(const Scr& s, int64_t e0, int64_t n) {
  float acc = -0.0f;
  for (int64_t i = 0; i < n; ++i) acc = __fadd_rn(acc, s.f(e0 + i));
  return acc;
}

// ndarray 0.16 numeric_util::unrolled_fold with A::add (ArrayBase::sum of a
// contiguous row, as sum_axis(Axis(1)) uses it).
__device__ float ndarray_sum(const Scr& s, int64_t e0, int64_t n) {
  float acc = 0.0f;
  float p[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int64_t i = 0;
  for (; n - i >= 8; i += 8)
#pragma unroll
    for (int k = 0; k < 8; ++k) p[k] = __fadd_rn(p[k], s.f(e0 + i + k));
  acc = __fadd_rn(acc, __fadd_rn(p[0], p[4]));
  acc = __fadd_rn(acc, __fadd_rn(p[1], p[5]));
  acc = __fadd_rn(acc, __fadd_rn(p[2], p[6]));
  acc = __fadd_rn(acc, __fadd_rn(p[3], p[7]));
  for (int64_t k = 0; i + k < n && k < 7; ++k) acc = __fadd_rn(acc, s.f(e0 + i + k));
  return acc;
}

// src/peak_group_scoring/utils.rs:126-172 over scratch vectors
__device__ float correlation_safe(const Scr& s, int64_t ex, int64_t ey, int64_t n) {
  if (n == 0) return 0.0f;
  const float xs = rust_sum(s, ex, n), ys = rust_sum(s, ey, n);
  if (xs == 0.0f || ys == 0.0f) return 0.0f;
  const float xm = __fdiv_rn(xs, (float)n), ym = __fdiv_rn(ys, (float)n);
  float xv = 0.0f, yv = 0.0f, cv = 0.0f;
  for (int64_t i = 0; i < n; ++i) {
    const float dx = __fsub_rn(s.f(ex + i), xm), dy = __fsub_rn(s.f(ey + i), ym);
    xv = __fadd_rn(xv, __fmul_rn(dx, dx));
    yv = __fadd_rn(yv, __fmul_rn(dy, dy));
    cv = __fadd_rn(cv, __fmul_rn(dx, dy));
  }
  if (xv == 0.0f || yv == 0.0f) return 0.0f;
  const float c = __fdiv_rn(cv, __fmul_rn(__fsqrt_rn(xv), __fsqrt_rn(yv)));
  if (isnan(c) || isinf(c)) return 0.0f;
  return fminf(fmaxf(c, -1.0f), 1.0f);
}

// correlation_safe(x, y) for many y against one x: x's sum, mean and squared deviations
// are formed once, in the same order of operations as the one-pair form.
struct XStats {
  float xs, xm, xv;
};

__device__ XStats x_stats(const Scr& s, int64_t ex, int64_t n) {
  XStats r{0.0f, 0.0f, 0.0f};
  if (n == 0) return r;
  r.xs = rust_sum(s, ex, n);
  r.xm = __fdiv_rn(r.xs, (float)n);
  for (int64_t i = 0; i < n; ++i) {
    const float dx = __fsub_rn(s.f(ex + i), r.xm);
    r.xv = __fadd_rn(r.xv, __fmul_rn(dx, dx));
  }
  return r;
}

__device__ float correlation_fixed_x(const Scr& s, const XStats& X, int64_t ex, int64_t ey,
                                     int64_t n) {
  if (n == 0) return 0.0f;
  const float ys = rust_sum(s, ey, n);
  if (X.xs == 0.0f || ys == 0.0f) return 0.0f;
  const float ym = __fdiv_rn(ys, (float)n);
  float yv = 0.0f, cv = 0.0f;
  for (int64_t i = 0; i < n; ++i) {
    const float dx = __fsub_rn(s.f(ex + i), X.xm), dy = __fsub_rn(s.f(ey + i), ym);
    yv = __fadd_rn(yv, __fmul_rn(dy, dy));
    cv = __fadd_rn(cv, __fmul_rn(dx, dy));
  }
  if (X.xv == 0.0f || yv == 0.0f) return 0.0f;
  const float c = __fdiv_rn(cv, __fmul_rn(__fsqrt_rn(X.xv), __fsqrt_rn(yv)));
  if (isnan(c) || isinf(c)) return 0.0f;
  return fminf(fmaxf(c, -1.0f), 1.0f);
}

// Stable ascending insertion sort of n floats at e0 (slice::sort_by(partial_cmp)).
__device__ void sort_floats(const Scr& s, int64_t e0, int64_t n) {
  for (int64_t i = 1; i < n; ++i) {
    const float v = s.f(e0 + i);
    int64_t j = i;
    while (j > 0 && v < s.f(e0 + j - 1)) {
      s.sf(e0 + j, s.f(e0 + j - 1));
      --j;
    }
    s.sf(e0 + j, v);
  }
}

// src/utils/mod.rs:120-143 (v copied into the sort buffer first)
__device__ float median_of(const Scr& s, int64_t ev, int64_t n, int64_t etmp) {
  if (n == 0) return 0.0f;
  for (int64_t i = 0; i < n; ++i) s.sf(etmp + i, s.f(ev + i));
  sort_floats(s, etmp, n);
  const int64_t mid = n / 2;
  return n % 2 == 0 ? __fdiv_rn(__fadd_rn(s.f(etmp + mid - 1), s.f(etmp + mid)), 2.0f)
                    : s.f(etmp + mid);
}

// src/utils/mod.rs:146-173
__device__ float std_of(const Scr& s, int64_t ev, int64_t n) {
  if (n < 2) return 0.0f;
  const float mean = __fdiv_rn(rust_sum(s, ev, n), (float)n);
  float acc = -0.0f;
  for (int64_t i = 0; i < n; ++i) {
    const float d = __fsub_rn(s.f(ev + i), mean);
    acc = __fadd_rn(acc, __fmul_rn(d, d));
  }
  return __fsqrt_rn(__fdiv_rn(acc, (float)(n - 1)));
}

// src/utils/mod.rs:175-221: mask of ranks [r1, r2) by value descending, index ascending.
// The rank of element i is the number of earlier elements not below it (ties and
// unordered pairs go to the lower index) plus the later elements above it.  The two
// halves are separate loops: nvcc 12.9 at -O3 dropped the tie term of the one-loop
// form `(w > v) || (!(w < v) && !(w > v) && j < i)` (every tie ranked 0).
__device__ void ranked_mask(const Scr& s, int64_t ev, int64_t n, int r1, int r2, int64_t em) {
  for (int64_t i = 0; i < n; ++i) {
    const float v = s.f(ev + i);
    int64_t rank = 0;
    for (int64_t j = 0; j < i; ++j) rank += !(s.f(ev + j) < v);
    for (int64_t j = i + 1; j < n; ++j) rank += s.f(ev + j) > v;
    s.su(em + i, (rank >= r1 && rank < r2) ? 1u : 0u);
  }
}


// src/peak_group_scoring/utils.rs:293-312
__device__ float gamma_ln(float x) {
  if (x <= 0.0f) return 0.0f;
  if (fabsf(__fsub_rn(x, 1.0f)) < 1e-6f) return 0.0f;
  if (fabsf(__fsub_rn(x, 2.0f)) < 1e-6f) return 0.0f;
  const float ln_2pi = 1.837877f;
  return __fadd_rn(__fsub_rn(__fmul_rn(__fsub_rn(x, 0.5f), ln_rn(x)), x), __fmul_rn(0.5f, ln_2pi));
}

// src/peak_group_scoring/utils.rs:193-279 (ew < 0: weights 1.0)
__device__ float hyperscore(const Scr& s, int64_t etype, int64_t eint, int64_t emask, int64_t ew,
                            int64_t n) {
  uint32_t nb = 0, ny = 0;
  float sb = 0.0f, sy = 0.0f;
  for (int64_t i = 0; i < n; ++i) {
    const float v = s.f(eint + i);
    if (!s.u(emask + i) || v == 0.0f) continue;
    const float wi = __fmul_rn(v, ew >= 0 ? s.f(ew + i) : 1.0f);
    const uint32_t t = s.u(etype + i);
    if (t == 98) {
      ++nb;
      sb = __fadd_rn(sb, wi);
    } else if (t == 121) {
      ++ny;
      sy = __fadd_rn(sy, wi);
    }
  }
  if (nb == 0 && ny == 0) return 0.0f;
  const float fb = nb > 0 ? gamma_ln(__fadd_rn((float)nb, 1.0f)) : 0.0f;
  const float fy = ny > 0 ? gamma_ln(__fadd_rn((float)ny, 1.0f)) : 0.0f;
  const float lb = sb > 0.0f ? ln_rn(sb) : 0.0f;
  const float ly = sy > 0.0f ? ln_rn(sy) : 0.0f;
  const float h = __fadd_rn(__fadd_rn(__fadd_rn(fb, fy), lb), ly);
  return isfinite(h) ? h : 0.0f;
}

// src/peak_group_scoring/utils.rs:314-372 for one series (numbers sorted in etmp)
__device__ uint32_t longest_series(const Scr& s, int64_t etype, int64_t enum_, int64_t emask,
                                   int64_t n, uint32_t type, int64_t etmp) {
  int64_t m = 0;
  for (int64_t i = 0; i < n; ++i)
    if (s.u(emask + i) && s.u(etype + i) == type) s.su(etmp + m++, s.u(enum_ + i));
  if (m == 0) return 0;
  for (int64_t i = 1; i < m; ++i) {  // sort_unstable: any order of equal numbers
    const uint32_t v = s.u(etmp + i);
    int64_t j = i;
    while (j > 0 && v < s.u(etmp + j - 1)) {
      s.su(etmp + j, s.u(etmp + j - 1));
      --j;
    }
    s.su(etmp + j, v);
  }
  uint32_t mx = 1, cur = 1;  // u8 arithmetic of the reference: wraps
  for (int64_t i = 1; i < m; ++i) {
    if (s.u(etmp + i) == ((s.u(etmp + i - 1) + 1u) & 0xFFu)) {
      cur = (cur + 1u) & 0xFFu;
      mx = max(mx, cur);
    } else {
      cur = 1;
    }
  }
  return mx;
}

// Sort key of each candidate for the work order: its precursor's library fragment count
// (capped at 255; 0 when the precursor is not in the library), and its index.
__global__ void work_key_kernel(int64_t n, const uint64_t* c_pidx, int64_t P, const uint64_t* l_pidx,
                                const uint64_t* l_fs, const uint64_t* l_fe, uint32_t* key,
                                uint32_t* idx) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t x = c_pidx[q];
    uint32_t k = 0;
    if (P > 0) {
      int64_t size = P, base = 0;
      while (size > 1) {
        const int64_t half = size / 2, mid = base + half;
        base = l_pidx[mid] > x ? base : mid;
        size -= half;
      }
      if (l_pidx[base] == x) {
        const uint64_t nraw = l_fe[base] - l_fs[base];
        k = nraw < 255ull ? (uint32_t)nraw : 255u;
      }
    }
    key[q] = k;
    idx[q] = (uint32_t)q;
  }
}

// The candidates' work order (ScoreArgs::order): indices stably sorted by work_key_kernel's
// key.  `buf` receives the order and holds the sort's temporaries.
int work_order(int64_t n, const uint64_t* c_pidx, const AdsLib* l, cudaStream_t st, DevBuf<char>* buf,
               const uint32_t** order) {
  *order = nullptr;
  // nothing to group when every precursor has the same number of library fragments
  if (n <= 1 || n > INT_MAX || l->min_frag == l->max_frag) return ADS_OK;
  size_t sort_bytes = 0;
  ADS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                           (uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, 0, 8, st));
  const size_t b4 = ((size_t)n * 4 + 255) / 256 * 256;
  ADS_TRY(buf->alloc(4 * b4 + sort_bytes));
  uint32_t* key = reinterpret_cast<uint32_t*>(buf->p);
  uint32_t* key_out = reinterpret_cast<uint32_t*>(buf->p + b4);
  uint32_t* idx = reinterpret_cast<uint32_t*>(buf->p + 2 * b4);
  uint32_t* perm = reinterpret_cast<uint32_t*>(buf->p + 3 * b4);
  work_key_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(
      n, c_pidx, l->n_prec, l->pidx_p, l->fstart_p, l->fstop_p, key, idx);
  ADS_LAUNCH_CHECK();
  ADS_CUDA(cub::DeviceRadixSort::SortPairs(buf->p + 4 * b4, sort_bytes, key, key_out, idx, perm,
                                           (int)n, 0, 8, st));
  *order = perm;
  return ADS_OK;
}

__global__ void idf_count_kernel(int64_t n, const float* mzl, GridView g, uint32_t* counts) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(counts + grid_find_closest(g, mzl[i]), 1u);
}

// Largest cycle window of the candidates; error bit 1 when one is out of range.
__global__ void cycle_span_kernel(int64_t n, const uint64_t* center, const uint64_t* start,
                                  const uint64_t* stop, int64_t n_rt, int* span, int* err) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t a = start[q], b = stop[q], c = center[q];
    if (a > b || b > (uint64_t)n_rt || c >= (uint64_t)n_rt) {
      atomicOr(err, 1);
      continue;
    }
    const uint64_t d = b - a;
    atomicMax(span, (int)(d < (uint64_t)INT_MAX ? d : (uint64_t)INT_MAX));
  }
}

// ---- per-candidate steps shared by the scoring and quantification kernels

// filter_sort_fragments (src/speclib_flat/mod.rs:240-345) of the precursor's nraw
// library fragments from fs: kept when non-zero and not y1; the top_k by intensity
// (ties to the lower position); in m/z order (ties keep library order).  Writes the
// kept fragments' m/z to FMZ and their library offsets (from fs) to FRAW; returns F.
__device__ __forceinline__ int64_t select_fragments(const ScoreArgs& a, const Scr& s, int64_t KEEP,
                                                    int64_t FMZ, int64_t FRAW, int64_t fs,
                                                    int64_t nraw) {
  int64_t nk = 0;
  for (int64_t r = 0; r < nraw; ++r) {
    const float I = a.l_fint[fs + r];
    const bool k = I > 0.0f && !(a.l_ftype[fs + r] == 121 && a.l_fnum[fs + r] == 1);
    s.su(KEEP + r, k ? 1u : 0u);
    nk += k;
  }
  const bool topk = nk > a.top_k;
  if (topk) {
    for (int64_t r = 0; r < nraw; ++r) {
      if (!s.u(KEEP + r)) continue;
      const float I = a.l_fint[fs + r];
      int64_t rank = 0;  // earlier not below plus later above
      for (int64_t j = 0; j < r; ++j)
        if (s.u(KEEP + j)) rank += !(a.l_fint[fs + j] < I);
      for (int64_t j = r + 1; j < nraw; ++j)
        if (s.u(KEEP + j)) rank += a.l_fint[fs + j] > I;
      if (rank < a.top_k) s.su(KEEP + r, 2u);
    }
  }
  const uint32_t need = topk ? 2u : 1u;
  for (int64_t r = 0; r < nraw; ++r) {
    if (s.u(KEEP + r) < need) continue;
    const float m = a.l_fmz[fs + r];
    int64_t pos = 0;  // stable: ties keep their library order
    for (int64_t j = 0; j < r; ++j)
      if (s.u(KEEP + j) >= need) pos += !(a.l_fmz[fs + j] > m);
    for (int64_t j = r + 1; j < nraw; ++j)
      if (s.u(KEEP + j) >= need) pos += a.l_fmz[fs + j] < m;
    s.sf(FMZ + pos, m);
    s.su(FRAW + pos, (uint32_t)r);
  }
  return topk ? a.top_k : nk;
}

// DenseXICMZObservation::new (src/dense_xic_observation/mod.rs:97-137) over cycles
// [cs, ce): the F x C dense XIC and intensity-weighted m/z matrices, every window that
// holds the precursor m/z in order, bins in order, entries in cycle order, with Rust's
// binary_search landing on the last entry at the first cycle
// (src/quadrupole_observation/mod.rs:152-211).
__device__ __forceinline__ void gather_xic_mz(const ScoreArgs& a, const Scr& s, int64_t XIC,
                                              int64_t MZO, int64_t FMZ, int64_t F, int cs, int ce,
                                              float pmz) {
  const int64_t C = ce - cs;
  for (int64_t e = 0; e < F * C; ++e) {
    s.sf(XIC + e, 0.0f);
    s.sf(MZO + e, 0.0f);
  }
  for (int w = 0; w < a.n_obs; ++w) {
    const WinInfo wi = a.win[w];
    if (!(wi.lo <= pmz && wi.hi >= pmz) || wi.ss_off < 0) continue;  // empty: no peaks
    const uint32_t* ssw = a.ss + wi.ss_off;
    const uint16_t* cyw = a.cyc + wi.base;
    const float* inw = a.inten + wi.base;
    for (int64_t f = 0; f < F; ++f) {
      const float mz = s.f(FMZ + f);
      const float delta = __fmul_rn(__fmul_rn(mz, a.tol), 1e-6f);
      const uint32_t b0 = grid_lower_bound(a.g, __fsub_rn(mz, delta));
      const uint32_t b1 = max(b0, grid_upper_bound(a.g, __fadd_rn(mz, delta)));
      for (uint32_t b = b0; b < b1; ++b) {
        const float actual = __ldg(a.g.grid + b);
        const int64_t e0 = ssw[b], e1 = ssw[b + 1];
        for (int64_t k = e0 + bsearch_u16_rust(cyw + e0, e1 - e0, cs); k < e1; ++k) {
          const int c = cyw[k];
          if (c >= ce) break;
          const int64_t at = f * C + (c - cs);
          const float v = inw[k];
          const float xs = __fadd_rn(s.f(XIC + at), v);
          s.sf(XIC + at, xs);
          if (v > 0.0f) {
            const float prev = __fsub_rn(xs, v);
            if (prev == 0.0f)
              s.sf(MZO + at, actual);
            else
              s.sf(MZO + at, __fdiv_rn(__fadd_rn(__fmul_rn(s.f(MZO + at), prev),
                                                 __fmul_rn(actual, v)),
                                       xs));
          }
        }
      }
    }
  }
}

// normalize_profiles(xic, 1) (src/peak_group_scoring/utils.rs:71-109) into NRM, and per
// row whether it stays non-zero (NZ).
__device__ __forceinline__ void normalize_rows(const Scr& s, int64_t XIC, int64_t NRM, int64_t NZ,
                                               int64_t F, int64_t C) {
  const int64_t center_c = C / 2;
  const int64_t c0 = center_c > 1 ? center_c - 1 : 0;
  const int64_t c1 = center_c + 2 < C ? center_c + 2 : C;
  for (int64_t f = 0; f < F; ++f) {
    float sum = 0.0f;
    int64_t count = 0;
    for (int64_t j = c0; j < c1; ++j) {
      sum = __fadd_rn(sum, s.f(XIC + f * C + j));
      ++count;
    }
    const float mean = count > 0 ? __fdiv_rn(sum, (float)count) : 0.0f;
    uint32_t nz = 0;
    for (int64_t j = 0; j < C; ++j) {
      const float v = mean > 0.0f ? __fdiv_rn(s.f(XIC + f * C + j), mean) : 0.0f;
      s.sf(NRM + f * C + j, v);
      nz |= v != 0.0f;
    }
    s.su(NZ + f, nz);
  }
}

// ORDERED: threads take the candidates in a.order (else in index order; compiled
// apart because the indirection changes the code of the whole loop).
template <bool ORDERED>
__global__ void __launch_bounds__(kScoreBlock) score_kernel(ScoreArgs a) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.T) return;
  const Scr s{a.scratch, a.T, t};
  const int64_t Fm = a.Fm, Cm = a.Cm;
  // scratch layout (elements)
  const int64_t XIC = 0, MZO = Fm * Cm, NRM = 2 * Fm * Cm, V = 3 * Fm * Cm;
  const int64_t FMZ = V, FMZL = V + Fm, FINT = V + 2 * Fm, FTYPE = V + 3 * Fm, FNUM = V + 4 * Fm,
                OBS = V + 5 * Fm, CORR = V + 6 * Fm, ERR = V + 7 * Fm, IDF = V + 8 * Fm,
                INVW = V + 9 * Fm, M0 = V + 10 * Fm, FRAW = V + 11 * Fm, MATCH = V + 14 * Fm,
                M6 = V + 15 * Fm, TMP = V + 16 * Fm, NZ = V + 17 * Fm, MED = V + 18 * Fm,
                MEDF = MED + Cm, KEEP = MEDF + Cm;

  for (int64_t qq = t; qq < a.n; qq += a.T) {
    const int64_t q = ORDERED ? (int64_t)a.order[qq] : qq;
    a.o_found[q] = 0;
    const uint64_t x = a.c_pidx[q];
    const uint64_t cs64 = a.c_start[q], ce64 = a.c_stop[q], center = a.c_center[q];
    if (cs64 > ce64 || ce64 > (uint64_t)a.n_rt || center >= (uint64_t)a.n_rt ||
        ce64 - cs64 > (uint64_t)Cm) {
      atomicOr(a.err, 1);
      continue;
    }
    // SpecLibFlat::get_precursor_by_idx_filtered: binary search of the sorted idx
    int64_t i = 0;
    {
      int64_t size = a.P, base = 0;
      if (size == 0) continue;
      while (size > 1) {
        const int64_t half = size / 2, mid = base + half;
        base = a.l_pidx[mid] > x ? base : mid;
        size -= half;
      }
      if (a.l_pidx[base] != x) continue;  // skipped, as in the reference
      i = base;
    }
    // filter_sort_fragments, then the kept fragments' library columns
    const int64_t fs = (int64_t)a.l_fs[i], nraw = (int64_t)a.l_fe[i] - fs;
    if (nraw > a.Fraw) {
      atomicOr(a.err, 2);
      continue;
    }
    const int64_t F = select_fragments(a, s, KEEP, FMZ, FRAW, fs, nraw);
    for (int64_t f = 0; f < F; ++f) {
      const int64_t r = fs + (int64_t)s.u(FRAW + f);
      s.sf(FMZL + f, a.l_fmzl[r]);
      s.sf(FINT + f, a.l_fint[r]);
      s.su(FTYPE + f, a.l_ftype[r]);
      s.su(FNUM + f, a.l_fnum[r]);
    }
    const int cs = (int)cs64, ce = (int)ce64;
    const int64_t C = ce - cs;
    gather_xic_mz(a, s, XIC, MZO, FMZ, F, cs, ce, a.l_pmz[i]);
    normalize_rows(s, XIC, NRM, NZ, F, C);
    int64_t n_nz = 0;
    for (int64_t f = 0; f < F; ++f) n_nz += s.u(NZ + f);
    // median profiles of all rows and of the non-zero rows (zeros when none); when every
    // row is non-zero the two are the median of the same values
    const bool all_nz = n_nz == F;
    for (int64_t j = 0; j < C; ++j) {
      for (int pass = 0; pass < (all_nz ? 1 : 2); ++pass) {
        int64_t R = 0;
        for (int64_t f = 0; f < F; ++f)
          if (pass == 0 || s.u(NZ + f)) s.sf(TMP + R++, s.f(NRM + f * C + j));
        float med = 0.0f;
        if (R > 0) {
          sort_floats(s, TMP, R);
          med = R % 2 == 0 ? __fdiv_rn(__fadd_rn(s.f(TMP + R / 2 - 1), s.f(TMP + R / 2)), 2.0f)
                           : s.f(TMP + R / 2);
        }
        s.sf((pass == 0 ? MED : MEDF) + j, med);
        if (all_nz) s.sf(MEDF + j, med);
      }
    }
    const float med_sum = rust_sum(s, MED, C), med_sum_f = rust_sum(s, MEDF, C);
    // calculate_fwhm_rt of the filtered median profile
    float fwhm = 0.0f;
    if (C > 0) {
      const int64_t half = C / 2;
      const float cen = s.f(MEDF + half);
      for (int64_t k = 0; k < half; ++k) {
        const float mean = __fdiv_rn(__fadd_rn(s.f(MEDF + half - k), s.f(MEDF + half + k)), 2.0f);
        if (mean <= __fdiv_rn(cen, 2.0f)) {
          fwhm = __fsub_rn(a.rt[cs + half + k], a.rt[cs + half - k]);
          break;
        }
      }
    }
    // correlations with the filtered median; observed intensities (row sums)
    const XStats xmed = x_stats(s, MEDF, C);
    for (int64_t f = 0; f < F; ++f) {
      s.sf(CORR + f, correlation_fixed_x(s, xmed, MEDF, NRM + f * C, C));
      s.sf(OBS + f, ndarray_sum(s, XIC + f * C, C));
    }
    const float int_corr = correlation_safe(s, OBS, FINT, F);
    const float mean_corr = F > 0 ? __fdiv_rn(rust_sum(s, CORR, F), (float)F) : 0.0f;
    const float med_corr = median_of(s, CORR, F, TMP);
    const float std_corr = std_of(s, CORR, F);
    // create_ranked_mask(intensity, 6r, 6r + 6) for r = 0..3 from one rank per fragment:
    // M0 holds the band rank / 6 (4: none of the four)
    for (int64_t f = 0; f < F; ++f) {
      const float v = s.f(FINT + f);
      int64_t rank = 0;  // earlier not below plus later above (ties to the lower index)
      for (int64_t j = 0; j < f; ++j) rank += !(s.f(FINT + j) < v);
      for (int64_t j = f + 1; j < F; ++j) rank += s.f(FINT + j) > v;
      s.su(M0 + f, (uint32_t)(rank < 24 ? rank / 6 : 4));
    }
    for (int64_t f = 0; f < F; ++f) s.su(MATCH + f, s.f(OBS + f) > 0.0f ? 1u : 0u);
    // fragment m/z and mass errors (ppm), inverse-error weights, IDF
    for (int64_t f = 0; f < F; ++f) {
      float ws = 0.0f, wsum = 0.0f;
      for (int64_t j = 0; j < C; ++j) {
        const float w = s.f(XIC + f * C + j);
        if (w > 0.0f) {
          ws = __fadd_rn(ws, __fmul_rn(s.f(MZO + f * C + j), w));
          wsum = __fadd_rn(wsum, w);
        }
      }
      const float o = wsum > 0.0f ? __fdiv_rn(ws, wsum) : 0.0f;
      const float lib = s.f(FMZ + f);
      const float err = o > 0.0f ? __fmul_rn(__fdiv_rn(__fsub_rn(o, lib), lib), 1e6f) : 0.0f;
      s.sf(ERR + f, err);
      s.sf(INVW + f, __fdiv_rn(1.0f, __fadd_rn(fabsf(err), 0.1f)));
      float idf = 1.0f;
      if (a.idf_total != 0.0f) {
        const uint32_t cnt = a.idf_counts[grid_find_closest(a.g, s.f(FMZL + f))];
        idf = ln_rn(__fdiv_rn(a.idf_total, (float)max(cnt, 1u)));
      }
      s.sf(IDF + f, idf);
    }
    ranked_mask(s, IDF, F, 0, 6, M6);
    float ib = 0.0f, iy = 0.0f, wmae_s = 0.0f, wmae_w = 0.0f;
    for (int64_t f = 0; f < F; ++f) {
      const float o = s.f(OBS + f);
      if (s.u(MATCH + f) && o > 0.0f) {
        if (s.u(FTYPE + f) == 98) ib = __fadd_rn(ib, o);
        if (s.u(FTYPE + f) == 121) iy = __fadd_rn(iy, o);
      }
      const float w = s.f(FINT + f), e = s.f(ERR + f);
      if (w > 0.0f && e != 0.0f) {
        wmae_s = __fadd_rn(wmae_s, __fmul_rn(fabsf(e), w));
        wmae_w = __fadd_rn(wmae_w, w);
      }
    }
    float idf_xic = -0.0f, idf_int = -0.0f;
    for (int64_t f = 0; f < F; ++f) {
      idf_xic = __fadd_rn(idf_xic, __fmul_rn(s.f(IDF + f), s.f(CORR + f)));
      idf_int = __fadd_rn(idf_int, __fmul_rn(s.f(IDF + f), s.f(OBS + f)));
    }
    if (F == 0) idf_xic = idf_int = 0.0f;
    const float rt_obs = a.rt[center];
    float* o = a.o_feat;
    const int64_t n = a.n;
    o[0 * n + q] = a.c_score[q];
    o[1 * n + q] = mean_corr;
    o[2 * n + q] = med_corr;
    o[3 * n + q] = std_corr;
    o[4 * n + q] = int_corr;
    o[5 * n + q] = (float)F;
    o[6 * n + q] = (float)(uint64_t)C;
    // count_values_above (src/utils/mod.rs:223-237) over the correlations, all in one
    // pass (integer counts)
    int c95 = 0, c90 = 0, c80 = 0, c50 = 0, c0 = 0, t0 = 0, t50 = 0;
    int b0[4] = {0, 0, 0, 0}, b50[4] = {0, 0, 0, 0};
    for (int64_t f = 0; f < F; ++f) {
      const float c = s.f(CORR + f);
      const uint32_t band = s.u(M0 + f);
      const bool top = s.u(M6 + f) != 0u;
      c95 += c > 0.95f;
      c90 += c > 0.90f;
      c80 += c > 0.80f;
      c50 += c > 0.50f;
      c0 += c > 0.0f;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        b0[r] += band == (uint32_t)r && c > 0.0f;
        b50[r] += band == (uint32_t)r && c > 0.50f;
      }
      t0 += top && c > 0.0f;
      t50 += top && c > 0.50f;
    }
    o[7 * n + q] = (float)c95;
    o[8 * n + q] = (float)c90;
    o[9 * n + q] = (float)c80;
    o[10 * n + q] = (float)c50;
    o[11 * n + q] = (float)c0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      o[(12 + r) * n + q] = (float)b0[r];
      o[(16 + r) * n + q] = (float)b50[r];
    }
    o[20 * n + q] = hyperscore(s, FTYPE, OBS, MATCH, -1, F);
    o[21 * n + q] = hyperscore(s, FTYPE, FINT, MATCH, -1, F);
    o[22 * n + q] = hyperscore(s, FTYPE, OBS, MATCH, INVW, F);
    o[23 * n + q] = rt_obs;
    o[24 * n + q] = __fsub_rn(rt_obs, a.l_prt[i]);
    o[25 * n + q] = (float)longest_series(s, FTYPE, FNUM, MATCH, F, 98, TMP);
    o[26 * n + q] = (float)longest_series(s, FTYPE, FNUM, MATCH, F, 121, TMP);
    o[27 * n + q] = (float)a.l_naa[i];
    o[28 * n + q] = wmae_w > 0.0f ? __fdiv_rn(wmae_s, wmae_w) : 0.0f;
    o[29 * n + q] = log10_rn(__fadd_rn(ib, 1e-8f));
    o[30 * n + q] = log10_rn(__fadd_rn(iy, 1e-8f));
    o[31 * n + q] = fwhm;
    o[32 * n + q] = hyperscore(s, FTYPE, IDF, MATCH, -1, F);
    o[33 * n + q] = idf_xic;
    o[34 * n + q] = log10_rn(__fadd_rn(idf_int, 1e-8f));
    o[35 * n + q] = med_sum;
    o[36 * n + q] = med_sum_f;
    o[37 * n + q] = (float)F;
    o[38 * n + q] = (float)n_nz;
    o[39 * n + q] = (float)t0;
    o[40 * n + q] = (float)t50;
    a.o_pidx[q] = x;
    a.o_rank[q] = a.c_rank[q];
    a.o_found[q] = 1;
  }
}

// ---------------------------------------------------------------- quantification

// PeakGroupQuantification.quantify per candidate (src/peak_group_quantification/mod.rs:
// 88-167): outputs of candidate q, dense per candidate (slot j of the first o_nq[q]).
struct QuantArgs {
  ScoreArgs s;  // library, run, tolerance, top-k, scratch (o_* and c_score unused)
  int* o_nq;          // fragments kept (observed intensity > 0); 0 drops the candidate
  uint32_t* o_prow;   // input row of the precursor
  float* o_rt;        // rt_observed
  uint64_t* o_frow;   // [n x Fm] input row of the fragment
  float* o_int;       // [n x Fm] observed intensity (row sum of the dense XIC)
  float* o_mzo;       // [n x Fm] observed m/z
  float* o_corr;      // [n x Fm] correlation with the median of the non-zero profiles
  float* o_err;       // [n x Fm] mass error (ppm)
  const uint32_t* l_prow;
};

// Largest cycle range of the candidates that quantification keeps; error bit 1 when a
// range ends beyond the run's RT index (the reference would extract zeros past it, or
// index out of bounds for the centre).
__global__ void quant_span_kernel(int64_t n, const uint64_t* center, const uint64_t* start,
                                  const uint64_t* stop, int64_t n_rt, int* span, int* err) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t a = start[q], b = stop[q], c = center[q];
    if (b <= a || c < a || c >= b) continue;  // dropped (None in the reference)
    if (b > (uint64_t)n_rt) {
      atomicOr(err, 1);
      continue;
    }
    const uint64_t d = b - a;
    atomicMax(span, (int)(d < (uint64_t)INT_MAX ? d : (uint64_t)INT_MAX));
  }
}

template <bool ORDERED>
__global__ void __launch_bounds__(kScoreBlock) quant_kernel(QuantArgs qa) {
  const ScoreArgs& a = qa.s;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.T) return;
  const Scr s{a.scratch, a.T, t};
  const int64_t Fm = a.Fm, Cm = a.Cm;
  // scratch layout (elements), within scratch_words(Fm, Fraw, Cm)
  const int64_t XIC = 0, MZO = Fm * Cm, NRM = 2 * Fm * Cm, V = 3 * Fm * Cm;
  const int64_t FMZ = V, FRAW = V + Fm, NZ = V + 2 * Fm, TMP = V + 3 * Fm, MEDF = V + 18 * Fm,
                KEEP = MEDF + 2 * Cm;

  for (int64_t qq = t; qq < a.n; qq += a.T) {
    const int64_t q = ORDERED ? (int64_t)a.order[qq] : qq;
    qa.o_nq[q] = 0;
    const uint64_t cs64 = a.c_start[q], ce64 = a.c_stop[q], center = a.c_center[q];
    if (ce64 <= cs64 || center < cs64 || center >= ce64) continue;
    if (ce64 > (uint64_t)a.n_rt || ce64 - cs64 > (uint64_t)Cm) {
      atomicOr(a.err, 1);
      continue;
    }
    const uint64_t x = a.c_pidx[q];
    int64_t i = 0;
    {
      int64_t size = a.P, base = 0;
      if (size == 0) continue;
      while (size > 1) {
        const int64_t half = size / 2, mid = base + half;
        base = a.l_pidx[mid] > x ? base : mid;
        size -= half;
      }
      if (a.l_pidx[base] != x) continue;  // get_precursor_by_idx_filtered: None
      i = base;
    }
    // filter_sort_fragments(non-zero, no y1, top-k), as in scoring
    const int64_t fs = (int64_t)a.l_fs[i], nraw = (int64_t)a.l_fe[i] - fs;
    if (nraw > a.Fraw) {
      atomicOr(a.err, 2);
      continue;
    }
    const int64_t F = select_fragments(a, s, KEEP, FMZ, FRAW, fs, nraw);
    const int cs = (int)cs64, ce = (int)ce64;
    const int64_t C = ce - cs;
    gather_xic_mz(a, s, XIC, MZO, FMZ, F, cs, ce, a.l_pmz[i]);
    normalize_rows(s, XIC, NRM, NZ, F, C);
    // filter_non_zero + median_axis_0 (zeros when no row is non-zero)
    for (int64_t j = 0; j < C; ++j) {
      int64_t R = 0;
      for (int64_t f = 0; f < F; ++f)
        if (s.u(NZ + f)) s.sf(TMP + R++, s.f(NRM + f * C + j));
      float med = 0.0f;
      if (R > 0) {
        sort_floats(s, TMP, R);
        med = R % 2 == 0 ? __fdiv_rn(__fadd_rn(s.f(TMP + R / 2 - 1), s.f(TMP + R / 2)), 2.0f)
                         : s.f(TMP + R / 2);
      }
      s.sf(MEDF + j, med);
    }
    // per fragment: observed m/z and mass error, correlation, observed intensity; the
    // fragments with a positive observed intensity are kept in m/z order
    const XStats xmed = x_stats(s, MEDF, C);
    int nq = 0;
    for (int64_t f = 0; f < F; ++f) {
      const float obs = ndarray_sum(s, XIC + f * C, C);
      if (!(obs > 0.0f)) continue;  // PrecursorQuantified::filter_fragments_by_intensity(0.0)
      float ws = 0.0f, wsum = 0.0f;
      for (int64_t j = 0; j < C; ++j) {
        const float w = s.f(XIC + f * C + j);
        if (w > 0.0f) {
          ws = __fadd_rn(ws, __fmul_rn(s.f(MZO + f * C + j), w));
          wsum = __fadd_rn(wsum, w);
        }
      }
      const float o = wsum > 0.0f ? __fdiv_rn(ws, wsum) : 0.0f;
      const float lib = s.f(FMZ + f);
      const int64_t slot = q * Fm + nq;
      qa.o_frow[slot] = (uint64_t)fs + s.u(FRAW + f);
      qa.o_int[slot] = obs;
      qa.o_mzo[slot] = o;
      qa.o_err[slot] = o > 0.0f ? __fmul_rn(__fdiv_rn(__fsub_rn(o, lib), lib), 1e6f) : 0.0f;
      // calculate_correlation_safe(profile, median) is symmetric in its arguments
      qa.o_corr[slot] = correlation_fixed_x(s, xmed, MEDF, NRM + f * C, C);
      ++nq;
    }
    qa.o_nq[q] = nq;
    qa.o_prow[q] = qa.l_prow[i];
    qa.o_rt[q] = a.rt[center];
  }
}

// SpecLibFlatQuantified::from_precursor_quantified_vec (src/speclib_flat_quantified/mod.rs:
// 212-333), step 1: the kept candidates' precursor rows (candidate order, not yet sorted)
// and their fragments, flat in candidate order.
__global__ void quant_flatten_kernel(int64_t n, int Fm, const int* nq, const int* prec_pos,
                                     const uint64_t* frag_off, const uint64_t* pidx,
                                     const uint64_t* rank, const uint32_t* prow, const float* rt,
                                     const uint64_t* frow, const float* v0, const float* v1,
                                     const float* v2, const float* v3, uint64_t* p_idx,
                                     uint64_t* p_row, uint64_t* p_rank, float* p_rt, uint64_t* p_fs,
                                     uint64_t* p_fe, uint32_t* p_perm, uint64_t* f_row, float* f0,
                                     float* f1, float* f2, float* f3, uint64_t* f_pidx,
                                     uint64_t* f_rank) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int k = nq[q];
    if (k <= 0) continue;
    const int j = prec_pos[q];
    const uint64_t o = frag_off[q];
    p_idx[j] = pidx[q];
    p_row[j] = prow[q];
    p_rank[j] = rank[q];
    p_rt[j] = rt[q];
    p_fs[j] = o;
    p_fe[j] = o + (uint64_t)k;
    p_perm[j] = (uint32_t)j;
    for (int m = 0; m < k; ++m) {
      const int64_t slot = q * Fm + m;
      f_row[o + m] = frow[slot];
      f0[o + m] = v0[slot];
      f1[o + m] = v1[slot];
      f2[o + m] = v2[slot];
      f3[o + m] = v3[slot];
      f_pidx[o + m] = pidx[q];
      f_rank[o + m] = rank[q];
    }
  }
}

// Step 2: the precursor columns gathered in the order of the stable sort by precursor_idx.
__global__ void quant_order_kernel(int64_t P, const uint32_t* perm, const uint64_t* row,
                                   const uint64_t* rank, const float* rt, const uint64_t* fs,
                                   const uint64_t* fe, uint64_t* o_row, uint64_t* o_rank,
                                   float* o_rt, uint64_t* o_fs, uint64_t* o_fe) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < P;
       j += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t i = perm[j];
    o_row[j] = row[i];
    o_rank[j] = rank[i];
    o_rt[j] = rt[i];
    o_fs[j] = fs[i];
    o_fe[j] = fe[i];
  }
}

// Assembles the flat layout of a quantification on the device.
struct KeptFragments {
  __host__ __device__ uint64_t operator()(int k) const { return k > 0 ? (uint64_t)k : 0ull; }
};
struct KeptAny {
  __host__ __device__ int operator()(int k) const { return k > 0 ? 1 : 0; }
};

// Totals of the two scans: fragments kept (out[0]) and candidates that kept any (out[1]).
__global__ void quant_totals_kernel(int64_t n, const int* nq, const uint64_t* off, const int* pos,
                                    int64_t* out) {
  const int k = nq[n - 1];
  out[0] = (int64_t)off[n - 1] + (k > 0 ? k : 0);
  out[1] = (int64_t)pos[n - 1] + (k > 0 ? 1 : 0);
}

// d_off / d_pos: each candidate's first fragment row and its precursor row (exclusive
// scans of the kept-fragment counts and of "kept any"), computed on the device.
int quant_assemble(AdsQuant* r, const uint64_t* d_off, const int* d_pos, cudaStream_t st) {
  const int64_t n = r->n, P = r->n_prec, NF = r->n_frag;
  if (P == 0) return ADS_OK;
  size_t sort_bytes = 0;
  ADS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                           (uint32_t*)nullptr, (uint32_t*)nullptr, (int)P, 0, 64, st));
  auto rnd = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t bP8 = rnd((size_t)P * 8), bP4 = rnd((size_t)P * 4), bF8 = rnd((size_t)NF * 8),
               bF4 = rnd((size_t)NF * 4);
  // final columns
  ADS_TRY(r->flat.alloc(5 * bP8 + bP4 + 3 * bF8 + 4 * bF4));
  char* b = r->flat.p;
  auto take = [&](size_t bytes) {
    char* p = b;
    b += bytes;
    return p;
  };
  r->p_idx = reinterpret_cast<uint64_t*>(take(bP8));
  r->p_row = reinterpret_cast<uint64_t*>(take(bP8));
  r->p_rank = reinterpret_cast<uint64_t*>(take(bP8));
  r->p_fs = reinterpret_cast<uint64_t*>(take(bP8));
  r->p_fe = reinterpret_cast<uint64_t*>(take(bP8));
  r->p_rt = reinterpret_cast<float*>(take(bP4));
  r->f_row = reinterpret_cast<uint64_t*>(take(bF8));
  r->f_pidx = reinterpret_cast<uint64_t*>(take(bF8));
  r->f_rank = reinterpret_cast<uint64_t*>(take(bF8));
  for (int k = 0; k < 4; ++k) r->f_val[k] = reinterpret_cast<float*>(take(bF4));
  // temporaries: unsorted precursor columns, permutation, sort space
  DevBuf<char> tmp;
  ADS_TRY(tmp.alloc(6 * bP8 + bP4 + 2 * bP4 + rnd(sort_bytes)));
  b = tmp.p;
  uint64_t* u_idx = reinterpret_cast<uint64_t*>(take(bP8));
  uint64_t* u_row = reinterpret_cast<uint64_t*>(take(bP8));
  uint64_t* u_rank = reinterpret_cast<uint64_t*>(take(bP8));
  uint64_t* u_fs = reinterpret_cast<uint64_t*>(take(bP8));
  uint64_t* u_fe = reinterpret_cast<uint64_t*>(take(bP8));
  uint64_t* u_spare = reinterpret_cast<uint64_t*>(take(bP8));
  float* u_rt = reinterpret_cast<float*>(take(bP4));
  uint32_t* perm_in = reinterpret_cast<uint32_t*>(take(bP4));
  uint32_t* perm = reinterpret_cast<uint32_t*>(take(bP4));
  void* sort_tmp = take(rnd(sort_bytes));
  (void)u_spare;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
  quant_flatten_kernel<<<grid, 256, 0, st>>>(
      n, r->Fm, r->nq_p, d_pos, d_off, r->pidx_p, r->rank_p, r->prow_p, r->rt_p, r->frow_p,
      r->fval_p[0], r->fval_p[1], r->fval_p[2], r->fval_p[3], u_idx, u_row, u_rank, u_rt, u_fs, u_fe,
      perm_in, r->f_row, r->f_val[0], r->f_val[1], r->f_val[2], r->f_val[3], r->f_pidx, r->f_rank);
  ADS_LAUNCH_CHECK();
  // radix sort is stable: equal precursor_idx keep candidate order
  ADS_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, u_idx, r->p_idx, perm_in, perm,
                                           (int)P, 0, 64, st));
  quant_order_kernel<<<(int)std::min<int64_t>((P + 255) / 256, 4096), 256, 0, st>>>(
      P, perm, u_row, u_rank, u_rt, u_fs, u_fe, r->p_row, r->p_rank, r->p_rt, r->p_fs, r->p_fe);
  ADS_LAUNCH_CHECK();
  ADS_CUDA(cudaStreamSynchronize(st));
  r->arena.release();  // the per-candidate slots are no longer needed
  return ADS_OK;
}

// The library's IDF histogram, built once per library on the device.
int ensure_idf(AdsLib* l, const GridView& g, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(l->mu);
  if (l->idf_counts.p) return ADS_OK;
  ADS_TRY(lib_ready_on(l, st));
  ADS_TRY(l->idf_counts.alloc(g.n));
  ADS_CUDA(cudaMemsetAsync(l->idf_counts.p, 0, (size_t)g.n * 4, st));
  if (l->n_frag > 0) {
    idf_count_kernel<<<(int)std::min<int64_t>((l->n_frag + 255) / 256, 4096), 256, 0, st>>>(
        l->n_frag, l->fmzl_p, g, l->idf_counts.p);
    ADS_LAUNCH_CHECK();
  }
  ADS_CUDA(cudaStreamSynchronize(st));
  return ADS_OK;
}

int score_device(const AdsScoringParams* p, const AdsDia* d, AdsLib* l, int64_t n,
                 const uint64_t* pidx, const uint64_t* rank, const float* score,
                 const uint64_t* center, const uint64_t* start, const uint64_t* stop, int64_t c_max,
                 int verbose, AdsFeatures** out) {
  if (d->bf16_only)
    return fail(ADS_ERR_INVALID_ARGUMENT, "scoring needs the run's f32 intensities, but this run "
                                          "keeps bfloat16 intensities only");
  if (!(p->mass_tolerance == p->mass_tolerance))
    return fail(ADS_ERR_INVALID_ARGUMENT, "mass_tolerance is NaN");
  if (p->top_k_fragments < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "top_k_fragments < 0");
  cudaStream_t st = cudaStreamPerThread;
  ADS_TRY(lib_ready_on(l, st));
  GridView g;
  ADS_TRY(device_grid(d->device, &g));
  ADS_TRY(ensure_idf(l, g, st));
  auto f = std::make_unique<AdsFeatures>();
  f->device = d->device;
  f->n = n;
  const size_t n1 = (size_t)std::max<int64_t>(n, 1);
  const size_t b8 = (n1 * 8 + 255) / 256 * 256, b4 = (n1 * 4 * kFeatures + 255) / 256 * 256;
  ADS_TRY(f->arena.alloc(2 * b8 + b4 + n1 + 256));
  f->pidx_p = reinterpret_cast<uint64_t*>(f->arena.p);
  f->rank_p = reinterpret_cast<uint64_t*>(f->arena.p + b8);
  f->feat_p = reinterpret_cast<float*>(f->arena.p + 2 * b8);
  f->found_p = reinterpret_cast<uint8_t*>(f->arena.p + 2 * b8 + b4);
  DevBuf<int> err;
  ADS_TRY(err.alloc(1));
  ADS_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
  struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } ev;
  if (n > 0) {
    const int Fm = (int)std::max<int64_t>(1, std::min<int64_t>(p->top_k_fragments, l->max_frag));
    const int Fraw = (int)std::max<int64_t>(1, l->max_frag);
    const int Cm = (int)std::max<int64_t>(1, c_max);
    const int64_t words = scratch_words(Fm, Fraw, Cm);
    int n_sm = 0;
    ADS_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, d->device));
    int64_t T = std::min<int64_t>(n, (int64_t)n_sm * 16 * kScoreBlock);
    T = std::max<int64_t>(1, std::min<int64_t>(T, ((int64_t)1 << 28) / words));  // <= 1 GiB
    DevBuf<uint32_t> scratch;
    ADS_TRY(scratch.alloc((size_t)(T * words)));
    ScoreArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.c_pidx = pidx;
    a.c_rank = rank;
    a.c_score = score;
    a.c_center = center;
    a.c_start = start;
    a.c_stop = stop;
    a.P = l->n_prec;
    a.l_pidx = l->pidx_p;
    a.l_pmz = l->pmz_p;
    a.l_prt = l->prt_p;
    a.l_naa = l->naa_p;
    a.l_fs = l->fstart_p;
    a.l_fe = l->fstop_p;
    a.l_fmz = l->fmz_p;
    a.l_fmzl = l->fmzl_p;
    a.l_fint = l->fint_p;
    a.l_fnum = l->fnum_p;
    a.l_ftype = l->ftype_p;
    a.idf_counts = l->idf_counts.p;
    a.idf_total = l->idf_total >= 0.0f ? l->idf_total : (float)l->n_frag;
    a.win = d->win_dev.p;
    a.n_obs = (int)d->n_obs;
    a.ss = d->slice_starts.p;
    a.cyc = d->cycles.p;
    a.inten = d->intens.p;
    a.rt = d->rt_dev.p;
    a.n_rt = (int64_t)d->rt.size();
    a.g = g;
    a.tol = p->mass_tolerance;
    a.top_k = p->top_k_fragments;
    a.Fm = Fm;
    a.Fraw = Fraw;
    a.Cm = Cm;
    a.scratch = scratch.p;
    DevBuf<char> order_buf;  // candidates grouped by work (kept until the kernel is done)
    ADS_TRY(work_order(n, pidx, l, st, &order_buf, &a.order));
    a.T = T;
    a.o_pidx = f->pidx_p;
    a.o_rank = f->rank_p;
    a.o_feat = f->feat_p;
    a.o_found = f->found_p;
    a.err = err.p;
    ADS_CUDA(cudaEventCreate(&ev.a));
    ADS_CUDA(cudaEventCreate(&ev.b));
    ADS_CUDA(cudaEventRecord(ev.a, st));
    if (a.order)
      score_kernel<true><<<(int)((T + kScoreBlock - 1) / kScoreBlock), kScoreBlock, 0, st>>>(a);
    else
      score_kernel<false><<<(int)((T + kScoreBlock - 1) / kScoreBlock), kScoreBlock, 0, st>>>(a);
    ADS_LAUNCH_CHECK();
    ADS_CUDA(cudaEventRecord(ev.b, st));
    f->found.resize((size_t)n);
    ADS_CUDA(cudaMemcpyAsync(f->found.data(), f->found_p, (size_t)n, cudaMemcpyDeviceToHost, st));
  }
  int herr = 0;
  ADS_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  ADS_CUDA(cudaStreamSynchronize(st));
  if (herr & 1)
    return fail(ADS_ERR_INVALID_ARGUMENT,
                "candidate cycle range outside the run's RT index (or cycle_start > cycle_stop)");
  if (herr & 2) return fail(ADS_ERR_INTERNAL, "fragment count above the scratch plan");
  for (uint8_t v : f->found) f->count += v;
  if (n > 0) ADS_CUDA(cudaEventElapsedTime(&f->kernel_ms, ev.a, ev.b));
  if (verbose && n > 0) {
    // src/peak_group_scoring/mod.rs:91-98
    printf("Scored %lld candidates at %.2f candidates/second\n", (long long)n,
           (double)n / std::max(1e-9, (double)f->kernel_ms * 1e-3));
    fflush(stdout);
  }
  *out = f.release();
  return ADS_OK;
}

int quant_device(const AdsQuantParams* p, const AdsDia* d, AdsLib* l, int64_t n,
                 const uint64_t* pidx, const uint64_t* rank, const uint64_t* center,
                 const uint64_t* start, const uint64_t* stop, int verbose, AdsQuant** out) {
  if (d->bf16_only)
    return fail(ADS_ERR_INVALID_ARGUMENT, "quantification needs the run's f32 intensities, but "
                                          "this run keeps bfloat16 intensities only");
  if (!(p->tolerance_ppm == p->tolerance_ppm))
    return fail(ADS_ERR_INVALID_ARGUMENT, "tolerance_ppm is NaN");
  if (p->top_k_fragments < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "top_k_fragments < 0");
  cudaStream_t st = cudaStreamPerThread;
  ADS_TRY(lib_ready_on(l, st));
  GridView g;
  ADS_TRY(device_grid(d->device, &g));
  auto r = std::make_unique<AdsQuant>();
  r->device = d->device;
  r->n = n;
  DevBuf<int> tmp;
  ADS_TRY(tmp.alloc(2));
  ADS_CUDA(cudaMemsetAsync(tmp.p, 0, 8, st));
  int64_t c_max = 0;
  if (n > 0) {
    quant_span_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(
        n, center, start, stop, (int64_t)d->rt.size(), tmp.p, tmp.p + 1);
    ADS_LAUNCH_CHECK();
    int h[2];
    ADS_CUDA(cudaMemcpyAsync(h, tmp.p, 8, cudaMemcpyDeviceToHost, st));
    ADS_CUDA(cudaStreamSynchronize(st));
    if (h[1])
      return fail(ADS_ERR_INVALID_ARGUMENT, "candidate cycle range ends beyond the run's RT index");
    c_max = h[0];
  }
  const int Fm = (int)std::max<int64_t>(1, std::min<int64_t>(p->top_k_fragments, l->max_frag));
  const int Fraw = (int)std::max<int64_t>(1, l->max_frag);
  const int Cm = (int)std::max<int64_t>(1, c_max);
  r->Fm = Fm;
  const size_t n1 = (size_t)std::max<int64_t>(n, 1), ns = n1 * (size_t)Fm;
  auto rnd = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_nq = rnd(n1 * 4), b_prow = rnd(n1 * 4), b_rt = rnd(n1 * 4), b_pid = rnd(n1 * 8),
               b_rank = rnd(n1 * 8), b_frow = rnd(ns * 8), b_f = rnd(ns * 4);
  ADS_TRY(r->arena.alloc(b_nq + b_prow + b_rt + b_pid + b_rank + b_frow + 4 * b_f));
  char* base = r->arena.p;
  r->nq_p = reinterpret_cast<int*>(base);
  base += b_nq;
  r->prow_p = reinterpret_cast<uint32_t*>(base);
  base += b_prow;
  r->rt_p = reinterpret_cast<float*>(base);
  base += b_rt;
  r->pidx_p = reinterpret_cast<uint64_t*>(base);
  base += b_pid;
  r->rank_p = reinterpret_cast<uint64_t*>(base);
  base += b_rank;
  r->frow_p = reinterpret_cast<uint64_t*>(base);
  base += b_frow;
  for (int k = 0; k < 4; ++k) {
    r->fval_p[k] = reinterpret_cast<float*>(base);
    base += b_f;
  }
  if (n > 0) {
    ADS_CUDA(cudaMemcpyAsync(r->pidx_p, pidx, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
    ADS_CUDA(cudaMemcpyAsync(r->rank_p, rank, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
    const int64_t words = scratch_words(Fm, Fraw, Cm);
    int n_sm = 0;
    ADS_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, d->device));
    int64_t T = std::min<int64_t>(n, (int64_t)n_sm * 16 * kScoreBlock);
    T = std::max<int64_t>(1, std::min<int64_t>(T, ((int64_t)1 << 28) / words));  // <= 1 GiB
    DevBuf<uint32_t> scratch;
    ADS_TRY(scratch.alloc((size_t)(T * words)));
    QuantArgs qa;
    std::memset(&qa, 0, sizeof(qa));
    ScoreArgs& a = qa.s;
    a.n = n;
    a.c_pidx = pidx;
    a.c_rank = rank;
    a.c_center = center;
    a.c_start = start;
    a.c_stop = stop;
    a.P = l->n_prec;
    a.l_pidx = l->pidx_p;
    a.l_pmz = l->pmz_p;
    a.l_prt = l->prt_p;
    a.l_fs = l->fstart_p;
    a.l_fe = l->fstop_p;
    a.l_fmz = l->fmz_p;
    a.l_fint = l->fint_p;
    a.l_fnum = l->fnum_p;
    a.l_ftype = l->ftype_p;
    a.win = d->win_dev.p;
    a.n_obs = (int)d->n_obs;
    a.ss = d->slice_starts.p;
    a.cyc = d->cycles.p;
    a.inten = d->intens.p;
    a.rt = d->rt_dev.p;
    a.n_rt = (int64_t)d->rt.size();
    a.g = g;
    a.tol = p->tolerance_ppm;
    a.top_k = p->top_k_fragments;
    a.Fm = Fm;
    a.Fraw = Fraw;
    a.Cm = Cm;
    a.scratch = scratch.p;
    DevBuf<char> order_buf;  // candidates grouped by work (kept until the kernel is done)
    ADS_TRY(work_order(n, pidx, l, st, &order_buf, &a.order));
    a.T = T;
    a.err = tmp.p + 1;
    qa.o_nq = r->nq_p;
    qa.o_prow = r->prow_p;
    qa.o_rt = r->rt_p;
    qa.o_frow = r->frow_p;
    qa.o_int = r->fval_p[0];
    qa.o_mzo = r->fval_p[1];
    qa.o_corr = r->fval_p[2];
    qa.o_err = r->fval_p[3];
    qa.l_prow = l->prow_p;
    struct Events {
      cudaEvent_t a = nullptr, b = nullptr;
      ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
      }
    } ev;
    ADS_CUDA(cudaEventCreate(&ev.a));
    ADS_CUDA(cudaEventCreate(&ev.b));
    ADS_CUDA(cudaEventRecord(ev.a, st));
    if (qa.s.order)
      quant_kernel<true><<<(int)((T + kScoreBlock - 1) / kScoreBlock), kScoreBlock, 0, st>>>(qa);
    else
      quant_kernel<false><<<(int)((T + kScoreBlock - 1) / kScoreBlock), kScoreBlock, 0, st>>>(qa);
    ADS_LAUNCH_CHECK();
    ADS_CUDA(cudaEventRecord(ev.b, st));
    // where each candidate's rows go: exclusive scans of the kept-fragment counts
    // and of "kept any fragment", and their totals
    cub::TransformInputIterator<uint64_t, KeptFragments, const int*> frag_in(r->nq_p, KeptFragments());
    cub::TransformInputIterator<int, KeptAny, const int*> prec_in(r->nq_p, KeptAny());
    size_t b1 = 0, b2 = 0;
    ADS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b1, frag_in, (uint64_t*)nullptr, (int)n, st));
    ADS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b2, prec_in, (int*)nullptr, (int)n, st));
    const size_t bo = rnd((size_t)n * 8), bpos = rnd((size_t)n * 4);
    DevBuf<char> scan;
    ADS_TRY(scan.alloc(bo + bpos + 256 + rnd(std::max(b1, b2))));
    uint64_t* d_off = reinterpret_cast<uint64_t*>(scan.p);
    int* d_pos = reinterpret_cast<int*>(scan.p + bo);
    int64_t* d_tot = reinterpret_cast<int64_t*>(scan.p + bo + bpos);
    void* scan_tmp = scan.p + bo + bpos + 256;
    size_t bt = std::max(b1, b2);
    ADS_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, bt, frag_in, d_off, (int)n, st));
    bt = std::max(b1, b2);
    ADS_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, bt, prec_in, d_pos, (int)n, st));
    quant_totals_kernel<<<1, 1, 0, st>>>(n, r->nq_p, d_off, d_pos, d_tot);
    ADS_LAUNCH_CHECK();
    int64_t htot[2] = {0, 0};
    int herr = 0;
    ADS_CUDA(cudaMemcpyAsync(htot, d_tot, sizeof(htot), cudaMemcpyDeviceToHost, st));
    ADS_CUDA(cudaMemcpyAsync(&herr, tmp.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    ADS_CUDA(cudaStreamSynchronize(st));
    if (herr & 1)
      return fail(ADS_ERR_INVALID_ARGUMENT, "candidate cycle range ends beyond the run's RT index");
    if (herr & 2) return fail(ADS_ERR_INTERNAL, "fragment count above the scratch plan");
    ADS_CUDA(cudaEventElapsedTime(&r->kernel_ms, ev.a, ev.b));
    r->n_frag = htot[0];
    r->n_prec = htot[1];
    if (r->n_prec > INT_MAX) return fail(ADS_ERR_INVALID_ARGUMENT, "too many quantified precursors");
    ADS_TRY(quant_assemble(r.get(), d_off, d_pos, st));
  }
  if (verbose) {
    // src/peak_group_quantification/mod.rs:73-78 (the kernel's device time)
    printf("Peak group quantification completed in %.2fs for %lld precursors\n",
           (double)r->kernel_ms * 1e-3, (long long)r->n_prec);
    fflush(stdout);
  }
  *out = r.release();
  return ADS_OK;
}

}  // namespace
}  // namespace ads

using namespace ads;

extern "C" {

void ads_scoring_params_default(AdsScoringParams* p) {
  if (!p) return;
  // ScoringParameters::new (src/peak_group_scoring/parameters.rs:16-25)
  p->mass_tolerance = 7.0f;
  p->top_k_fragments = 100;
}

int ads_score(const AdsScoringParams* params, const AdsDia* dia, AdsLib* lib, AdsCandidates* cand,
              int verbose, AdsFeatures** out) {
  return guarded([&] {
    if (!params || !dia || !lib || !cand || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (dia->device != lib->device || cand->device != lib->device)
      return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
    const int64_t n = ads_candidates_size(cand);  // waits for the search that fills them
    if (n < 0) return fail(ADS_ERR_INTERNAL, ads_last_error());
    DeviceGuard dg(dia->device);
    int64_t c_max = 0;
    if (n > 0) {
      DevBuf<int> tmp;
      ADS_TRY(tmp.alloc(2));
      ADS_CUDA(cudaMemsetAsync(tmp.p, 0, 8, cudaStreamPerThread));
      cycle_span_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, cudaStreamPerThread>>>(
          n, cand->center_p, cand->start_p, cand->stop_p, (int64_t)dia->rt.size(), tmp.p, tmp.p + 1);
      ADS_LAUNCH_CHECK();
      int h[2];
      ADS_CUDA(cudaMemcpyAsync(h, tmp.p, 8, cudaMemcpyDeviceToHost, cudaStreamPerThread));
      ADS_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
      if (h[1]) return fail(ADS_ERR_INVALID_ARGUMENT, "candidate cycle range outside the RT index");
      c_max = h[0];
    }
    return score_device(params, dia, lib, n, cand->pidx_p, cand->rank_p, cand->score_p,
                        cand->center_p, cand->start_p, cand->stop_p, c_max, verbose, out);
  });
}

int ads_score_arrays(const AdsScoringParams* params, const AdsDia* dia, AdsLib* lib, int64_t n,
                     const uint64_t* precursor_idx, const uint64_t* rank, const float* score,
                     const uint64_t* cycle_center, const uint64_t* cycle_start,
                     const uint64_t* cycle_stop, int location, int verbose, AdsFeatures** out) {
  return guarded([&] {
    if (!params || !dia || !lib || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (n < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "negative candidate count");
    if (location != ADS_MEM_HOST && location != ADS_MEM_DEVICE)
      return fail(ADS_ERR_INVALID_ARGUMENT, "location must be ADS_MEM_HOST or ADS_MEM_DEVICE");
    if (n > 0 && (!precursor_idx || !rank || !score || !cycle_center || !cycle_start || !cycle_stop))
      return fail(ADS_ERR_INVALID_ARGUMENT, "null array pointer");
    if (dia->device != lib->device) return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
    DeviceGuard dg(dia->device);
    cudaStream_t st = cudaStreamPerThread;
    const size_t n1 = (size_t)std::max<int64_t>(n, 1);
    DevBuf<uint64_t> cols;
    DevBuf<float> sc;
    ADS_TRY(cols.alloc(5 * n1));
    ADS_TRY(sc.alloc(n1));
    const cudaMemcpyKind kind = location == ADS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    int64_t c_max = 0;
    if (n > 0) {
      const uint64_t* src[5] = {precursor_idx, rank, cycle_center, cycle_start, cycle_stop};
      for (int k = 0; k < 5; ++k)
        ADS_CUDA(cudaMemcpyAsync(cols.p + k * n1, src[k], (size_t)n * 8, kind, st));
      ADS_CUDA(cudaMemcpyAsync(sc.p, score, (size_t)n * 4, kind, st));
      DevBuf<int> tmp;
      ADS_TRY(tmp.alloc(2));
      ADS_CUDA(cudaMemsetAsync(tmp.p, 0, 8, st));
      cycle_span_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(
          n, cols.p + 2 * n1, cols.p + 3 * n1, cols.p + 4 * n1, (int64_t)dia->rt.size(), tmp.p, tmp.p + 1);
      ADS_LAUNCH_CHECK();
      int h[2];
      ADS_CUDA(cudaMemcpyAsync(h, tmp.p, 8, cudaMemcpyDeviceToHost, st));
      ADS_CUDA(cudaStreamSynchronize(st));
      if (h[1]) return fail(ADS_ERR_INVALID_ARGUMENT, "candidate cycle range outside the RT index");
      c_max = h[0];
    }
    return score_device(params, dia, lib, n, cols.p, cols.p + n1, sc.p, cols.p + 2 * n1,
                        cols.p + 3 * n1, cols.p + 4 * n1, c_max, verbose, out);
  });
}

int64_t ads_features_size(const AdsFeatures* f) { return f ? f->count : -1; }

float ads_features_kernel_ms(const AdsFeatures* f) { return f ? f->kernel_ms : -1.0f; }

int ads_features_copy_out(const AdsFeatures* f, uint64_t* precursor_idx, uint64_t* rank,
                          float* features) {
  return guarded([&] {
    if (!f) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    if (f->n == 0) return ADS_OK;
    DeviceGuard dg(f->device);
    const size_t n = (size_t)f->n;
    if (f->count == f->n) {  // every candidate scored: the device layout is the output's
      if (precursor_idx) ADS_CUDA(cudaMemcpy(precursor_idx, f->pidx_p, n * 8, cudaMemcpyDeviceToHost));
      if (rank) ADS_CUDA(cudaMemcpy(rank, f->rank_p, n * 8, cudaMemcpyDeviceToHost));
      if (features) ADS_CUDA(cudaMemcpy(features, f->feat_p, n * 4 * kFeatures, cudaMemcpyDeviceToHost));
      return ADS_OK;
    }
    std::vector<uint64_t> p(n), r(n);
    std::vector<float> x(n * kFeatures);
    ADS_CUDA(cudaMemcpy(p.data(), f->pidx_p, n * 8, cudaMemcpyDeviceToHost));
    ADS_CUDA(cudaMemcpy(r.data(), f->rank_p, n * 8, cudaMemcpyDeviceToHost));
    ADS_CUDA(cudaMemcpy(x.data(), f->feat_p, n * 4 * kFeatures, cudaMemcpyDeviceToHost));
    const size_t m = (size_t)f->count;
    size_t o = 0;
    for (size_t q = 0; q < n; ++q) {
      if (!f->found[q]) continue;
      if (precursor_idx) precursor_idx[o] = p[q];
      if (rank) rank[o] = r[q];
      if (features)
        for (int k = 0; k < kFeatures; ++k) features[(size_t)k * m + o] = x[(size_t)k * n + q];
      ++o;
    }
    return ADS_OK;
  });
}

int ads_features_destroy(AdsFeatures* f) {
  return guarded([&] {
    if (!f) return ADS_OK;
    DeviceGuard dg(f->device);
    delete f;
    return ADS_OK;
  });
}

int ads_feature_names(const char** names, int cap) {
  for (int k = 0; k < kFeatures && k < cap; ++k) names[k] = kFeatureNames[k];
  return kFeatures;
}

void ads_quant_params_default(AdsQuantParams* p) {
  if (!p) return;
  // QuantificationParameters::new (src/peak_group_quantification/parameters.rs:19-28)
  p->tolerance_ppm = 7.0f;
  p->top_k_fragments = 10000;
}

int ads_quantify(const AdsQuantParams* params, const AdsDia* dia, AdsLib* lib, AdsCandidates* cand,
                 int verbose, AdsQuant** out) {
  return guarded([&] {
    if (!params || !dia || !lib || !cand || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (dia->device != lib->device || cand->device != lib->device)
      return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
    const int64_t n = ads_candidates_size(cand);  // waits for the search that fills them
    if (n < 0) return fail(ADS_ERR_INTERNAL, ads_last_error());
    DeviceGuard dg(dia->device);
    return quant_device(params, dia, lib, n, cand->pidx_p, cand->rank_p, cand->center_p,
                        cand->start_p, cand->stop_p, verbose, out);
  });
}

int ads_quantify_arrays(const AdsQuantParams* params, const AdsDia* dia, AdsLib* lib, int64_t n,
                        const uint64_t* precursor_idx, const uint64_t* rank,
                        const uint64_t* cycle_center, const uint64_t* cycle_start,
                        const uint64_t* cycle_stop, int location, int verbose, AdsQuant** out) {
  return guarded([&] {
    if (!params || !dia || !lib || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (n < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "negative candidate count");
    if (location != ADS_MEM_HOST && location != ADS_MEM_DEVICE)
      return fail(ADS_ERR_INVALID_ARGUMENT, "location must be ADS_MEM_HOST or ADS_MEM_DEVICE");
    if (n > 0 && (!precursor_idx || !rank || !cycle_center || !cycle_start || !cycle_stop))
      return fail(ADS_ERR_INVALID_ARGUMENT, "null array pointer");
    if (dia->device != lib->device) return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
    DeviceGuard dg(dia->device);
    cudaStream_t st = cudaStreamPerThread;
    const size_t n1 = (size_t)std::max<int64_t>(n, 1);
    DevBuf<uint64_t> cols;
    ADS_TRY(cols.alloc(5 * n1));
    const cudaMemcpyKind kind = location == ADS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (n > 0) {
      const uint64_t* src[5] = {precursor_idx, rank, cycle_center, cycle_start, cycle_stop};
      for (int k = 0; k < 5; ++k)
        ADS_CUDA(cudaMemcpyAsync(cols.p + k * n1, src[k], (size_t)n * 8, kind, st));
    }
    return quant_device(params, dia, lib, n, cols.p, cols.p + n1, cols.p + 2 * n1, cols.p + 3 * n1,
                        cols.p + 4 * n1, verbose, out);
  });
}

int ads_quant_sizes(const AdsQuant* q, int64_t* n_precursors, int64_t* n_fragments) {
  if (!q) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
  if (n_precursors) *n_precursors = q->n_prec;
  if (n_fragments) *n_fragments = q->n_frag;
  return ADS_OK;
}

float ads_quant_kernel_ms(const AdsQuant* q) { return q ? q->kernel_ms : -1.0f; }

int ads_quant_copy_out(const AdsQuant* q, uint64_t* precursor_idx, uint64_t* precursor_row,
                       uint64_t* rank, float* rt_observed, uint64_t* flat_frag_start_idx,
                       uint64_t* flat_frag_stop_idx, uint64_t* fragment_row, float* intensity,
                       float* mz_observed, float* correlation_observed, float* mass_error_observed,
                       uint64_t* fragment_precursor_idx, uint64_t* fragment_rank) {
  return guarded([&] {
    if (!q) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    if (q->n_prec == 0) return ADS_OK;
    DeviceGuard dg(q->device);
    const size_t P = (size_t)q->n_prec, NF = (size_t)q->n_frag;
    struct Col {
      void* dst;
      const void* src;
      size_t bytes;
    } cols[] = {{precursor_idx, q->p_idx, P * 8},         {precursor_row, q->p_row, P * 8},
                {rank, q->p_rank, P * 8},                 {rt_observed, q->p_rt, P * 4},
                {flat_frag_start_idx, q->p_fs, P * 8},    {flat_frag_stop_idx, q->p_fe, P * 8},
                {fragment_row, q->f_row, NF * 8},         {intensity, q->f_val[0], NF * 4},
                {mz_observed, q->f_val[1], NF * 4},       {correlation_observed, q->f_val[2], NF * 4},
                {mass_error_observed, q->f_val[3], NF * 4}, {fragment_precursor_idx, q->f_pidx, NF * 8},
                {fragment_rank, q->f_rank, NF * 8}};
    for (const Col& c : cols)
      if (c.dst)
        ADS_CUDA(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, cudaStreamPerThread));
    ADS_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
    return ADS_OK;
  });
}

int ads_quant_destroy(AdsQuant* q) {
  return guarded([&] {
    if (!q) return ADS_OK;
    DeviceGuard dg(q->device);
    delete q;
    return ADS_OK;
  });
}

int64_t ads_idf_bins(void) {
  return (int64_t)host_grid().size();
}

int ads_lib_idf_counts(AdsLib* lib, uint32_t* counts, int location) {
  return guarded([&] {
    if (!lib || !counts) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    if (location != ADS_MEM_HOST && location != ADS_MEM_DEVICE)
      return fail(ADS_ERR_INVALID_ARGUMENT, "location must be ADS_MEM_HOST or ADS_MEM_DEVICE");
    DeviceGuard dg(lib->device);
    GridView g;
    ADS_TRY(device_grid(lib->device, &g));
    ADS_TRY(ensure_idf(lib, g, cudaStreamPerThread));
    ADS_CUDA(cudaMemcpy(counts, lib->idf_counts.p, (size_t)g.n * 4,
                        location == ADS_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
    return ADS_OK;
  });
}

int ads_lib_set_idf(AdsLib* lib, const uint32_t* counts, double total_fragments, int location) {
  return guarded([&] {
    if (!lib || !counts) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    if (location != ADS_MEM_HOST && location != ADS_MEM_DEVICE)
      return fail(ADS_ERR_INVALID_ARGUMENT, "location must be ADS_MEM_HOST or ADS_MEM_DEVICE");
    if (!(total_fragments >= 0.0)) return fail(ADS_ERR_INVALID_ARGUMENT, "total_fragments < 0");
    DeviceGuard dg(lib->device);
    GridView g;
    ADS_TRY(device_grid(lib->device, &g));
    ADS_TRY(ensure_idf(lib, g, cudaStreamPerThread));
    std::lock_guard<std::mutex> lk(lib->mu);
    ADS_CUDA(cudaMemcpy(lib->idf_counts.p, counts, (size_t)g.n * 4,
                        location == ADS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice));
    // neither a pageable upload nor a device-to-device copy waits for its DMA, and the
    // scoring kernels read the histogram from other streams
    ADS_CUDA(cudaDeviceSynchronize());
    lib->idf_total = (float)total_fragments;  // usize as f32, as the reference converts
    return ADS_OK;
  });
}

}  // extern "C"
