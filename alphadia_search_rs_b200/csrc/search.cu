// PeakGroupSelection.search on the device (src/peak_group_selection/mod.rs:87-195).
//
// Three stages, all on one stream:
//   1. prep_kernel      one warp per precursor: RT cycle limits, quadrupole
//                       windows, fragment filter / top-k / m/z sort, m/z bin
//                       range of every kept fragment.
//   2. search_kernel    one block per precursor (persistent blocks pulling from
//                       an atomic counter): XIC gather into shared memory,
//                       Gaussian convolution, log-dot score, 5-point local
//                       maxima, top-K.  Arithmetic follows the reference's
//                       operation order with explicitly rounded f32 ops, so the
//                       only difference to the reference is its logf (see ln_rn).
//   3. compaction       order-preserving concatenation of the per-precursor
//                       candidates into the nine to_arrays() columns.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>

#include "common.cuh"

namespace ads {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxHalf = 31;       // kernel half width h <= 31 (2h+1 bits in a u64 mask)
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
__device__ __forceinline__ int rust_bsearch_f32(const float* a, int n, float x) {
  int size = n, base = 0;
  while (size > 1) {
    const int half = size / 2, mid = base + half;
    base = (__ldg(a + mid) > x) ? base : mid;
    size -= half;
  }
  const float v = __ldg(a + base);
  if (v == x) return base;
  return base + (v < x ? 1 : 0);
}

// RTIndex::get_cycle_idx_limits (src/rt_index/mod.rs:89-138).
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
  const float r0 = __ldg(rt), rn = __ldg(rt + n - 1);
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
};

// src/speclib_flat/mod.rs:240-345 (non_zero and y1 filters, top-k by intensity,
// sort by fragment m/z; ties go to the lower library position) followed by the
// ppm bin range of src/quadrupole_observation/mod.rs:79-83 + src/mz_index/mod.rs:95-127.
__device__ int select_fragments(const PrepArgs& a, int64_t p, int lane, uint8_t* keep) {
  const int64_t s = (int64_t)a.fstart[p];
  const int64_t n = (int64_t)a.fstop[p] - s;
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
      int pos = 0;
      for (int64_t j = 0; j < n; ++j) {
        if (keep[j] < need) continue;
        const float m = __ldg(a.fmz + s + j);
        pos += (m < mz) || (m == mz && j < i);
      }
      const float delta = __fmul_rn(__fmul_rn(mz, a.mass_tol), 1e-6f);
      const float lo = __fsub_rn(mz, delta), hi = __fadd_rn(mz, delta);
      const uint32_t b0 = grid_lower_bound(a.g, lo);
      const uint32_t b1 = max(b0, grid_upper_bound(a.g, hi));
      const int64_t o = p * a.kf + pos;
      a.fw[o] = __ldg(a.fint + s + i);
      a.blo[o] = b0;
      a.bhi[o] = b1;
    }
  }
  __syncwarp();
  return F;
}

__global__ void __launch_bounds__(kPrepThreads) prep_kernel(PrepArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = warp0; p < a.n_prec; p += n_warps) {
    const float tol = a.ptol ? __ldg(a.ptol + p) : a.rt_tol;
    int cs, ce;
    rt_limits(a.rt, a.n_rt, a.delta_t, __ldg(a.prt + p), tol, a.pad, &cs, &ce);
    bool skip = (ce - cs) < a.min_c;
    int nw = 0;
    if (!skip) {
      const float pmz = __ldg(a.pmz + p);
      for (int base = 0; base < a.n_obs; base += 32) {
        const int w = base + lane;
        bool hit = false;
        if (w < a.n_obs) {
          const WinInfo wi = a.win[w];
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

// ---------------------------------------------------------------- search

struct SearchArgs {
  int64_t n_prec;
  const int* nf;
  const int* cs;
  const int* ce;
  const int* nwin;
  const int* wins;
  int maxw;
  const float* fw;
  const uint32_t* blo;
  const uint32_t* bhi;
  int kf;
  const WinInfo* win;
  const uint32_t* ss;
  const uint16_t* cyc;
  const float* inten;
  float kw[kMaxHalf + 1];  // kernel taps w[0..h]; w[h] is the centre
  int h;
  int k_out;   // candidates kept per precursor
  int c_max;   // largest cycle range any precursor can have
  int cp;      // c_max rounded up to 32
  int gather_mode;
  int scan_thresh;
  unsigned int* work;
  int* err;
  int* cand_n;
  float* cand_score;
  int* cand_center;
  unsigned long long* stats;  // nullable: [2] fragments [3] entries read [4] accumulated [5] offsets
};

struct Smem {
  float* xrow;    // [nw][cp]
  float* vrow;    // [nw][cp]
  float* score;   // [cp]
  uint32_t* bm;   // [nw][bw]
  float* scr;     // [nw][32]
  float* mval;    // [mx]
  int* midx;      // [mx]
  int* misc;      // [4]
  int bw, mx;
};

__host__ __device__ inline int bitmap_words(int cp) { return cp / 32 + 3; }
__host__ __device__ inline int maxima_cap(int cp) { return cp / 4 + 8; }

__host__ __device__ inline size_t search_smem_bytes(int nw, int cp) {
  const size_t words = (size_t)nw * cp * 2 + cp + (size_t)nw * bitmap_words(cp) + (size_t)nw * 32 +
                       2 * (size_t)maxima_cap(cp) + 4;
  return words * 4;
}

__device__ __forceinline__ Smem carve(float* base, int nw, int cp) {
  Smem s;
  s.bw = bitmap_words(cp);
  s.mx = maxima_cap(cp);
  float* q = base;
  s.xrow = q;
  q += (size_t)nw * cp;
  s.vrow = q;
  q += (size_t)nw * cp;
  s.score = q;
  q += cp;
  s.bm = reinterpret_cast<uint32_t*>(q);
  q += (size_t)nw * s.bw;
  s.scr = q;
  q += (size_t)nw * 32;
  s.mval = q;
  q += s.mx;
  s.midx = reinterpret_cast<int*>(q);
  q += s.mx;
  s.misc = reinterpret_cast<int*>(q);
  return s;
}

// Adds this chunk's accepted entries to the XIC row in lane (= CSR) order: lanes
// that hit the same cycle are summed by their lowest lane, one rounded add per
// entry, exactly like the reference's `dense_xic[c] += intensity`
// (src/quadrupole_observation/mod.rs:96-105).
__device__ __forceinline__ void accumulate(bool inc, int cell, float v, int lane, float* row,
                                           uint32_t* bm, float* scr, unsigned long long& n_acc) {
  const unsigned act = __ballot_sync(kFull, inc);
  if (act == 0) return;
  n_acc += __popc(act);
  const int key = inc ? cell : (-1 - lane);
  const unsigned grp = __match_any_sync(kFull, key);
  scr[lane] = v;
  __syncwarp();
  if (inc && lane == __ffs(grp) - 1) {
    float acc = row[cell];
    unsigned g = grp;
    while (g) {
      const int l = __ffs(g) - 1;
      acc = __fadd_rn(acc, scr[l]);
      g &= g - 1;
    }
    row[cell] = acc;
    atomicOr(bm + (cell >> 5), 1u << (cell & 31));
  }
  __syncwarp();
}

// One (fragment, quadrupole window) pair: fill_xic_slice over the fragment's bin
// range.  Two exact strategies:
//   scan     read every entry of the contiguous CSR range of the bins and keep
//            those with start < cycle < stop, plus the last entry at cycle ==
//            start of each bin (where Rust's binary search lands);
//   bsearch  per bin, binary-search the first kept entry and the first entry
//            at or past stop, then read only the kept entries.
__device__ void gather(const SearchArgs& a, const WinInfo& wi, uint32_t b0, uint32_t b1, int cs,
                       int ce, int lane, float* row, uint32_t* bm, float* scr,
                       unsigned long long& n_read, unsigned long long& n_acc,
                       unsigned long long& n_off, unsigned long long& n_pairs,
                       unsigned long long& n_bins1) {
  if (b1 <= b0) return;
  const uint32_t* ssw = a.ss + wi.ss_off;
  const uint16_t* cy = a.cyc + wi.base;
  const float* in = a.inten + wi.base;
  const int64_t rs = __ldg(ssw + b0), re = __ldg(ssw + b1);
  n_off += 2;
  n_pairs += 1;
  n_bins1 += b1 - b0 + 1;
  const int64_t n = re - rs;
  if (n <= 0) return;
  const bool scan = a.gather_mode == 1 || (a.gather_mode == 0 && n <= a.scan_thresh);
  if (scan) {
    n_read += n;
    for (int64_t q0 = rs; q0 < re; q0 += 32) {
      const int64_t q = q0 + lane;
      const bool valid = q < re;
      const int c = valid ? (int)__ldg(cy + q) : 0;
      bool inc = valid && c > cs && c < ce;
      if (valid && c == cs) {
        const int64_t nxt = q + 1;
        bool last = nxt == re;
        if (!last) {
          // is nxt the first entry of a later bin?  (slice_starts[b] == nxt)
          uint32_t lo = b0 + 1, hi = b1;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if ((int64_t)__ldg(ssw + mid) < nxt)
              lo = mid + 1;
            else
              hi = mid;
          }
          last = (lo < b1) && ((int64_t)__ldg(ssw + lo) == nxt);
          if (!last) last = (int)__ldg(cy + nxt) != cs;
        }
        inc = last;
      }
      const float v = inc ? __ldg(in + q) : 0.0f;
      accumulate(inc, c - cs, v, lane, row, bm, scr, n_acc);
    }
  } else {
    for (uint32_t bb = b0; bb < b1; bb += 32) {
      const uint32_t b = bb + lane;
      const bool vb = b < b1;
      int64_t pos = 0, cnt = 0;
      if (vb) {
        const int64_t s = __ldg(ssw + b), e = __ldg(ssw + b + 1);
        pos = s + rust_bsearch_u16(cy + s, e - s, cs);
        const int64_t end = pos + lower_bound_u16(cy + pos, e - pos, ce);
        cnt = end - pos;
      }
      n_off += 2 * __popc(__ballot_sync(kFull, vb));
      int64_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      const int64_t total = __shfl_sync(kFull, incl, 31);
      const int64_t excl = incl - cnt;
      n_read += total;
      for (int64_t t0 = 0; t0 < total; t0 += 32) {
        const int64_t t = t0 + lane;
        int l = 0;
#pragma unroll
        for (int st = 16; st >= 1; st >>= 1) {
          const int c = l + st;
          const int64_t ec = __shfl_sync(kFull, excl, c);
          if (ec <= t) l = c;
        }
        const int64_t opos = __shfl_sync(kFull, pos, l);
        const int64_t oex = __shfl_sync(kFull, excl, l);
        const bool vt = t < total;
        const int64_t q = opos + (t - oex);
        const int c = vt ? (int)__ldg(cy + q) : 0;
        const float v = vt ? __ldg(in + q) : 0.0f;
        accumulate(vt, c - cs, v, lane, row, bm, scr, n_acc);
      }
    }
  }
}

// 2h+1 bitmap bits starting at bit p0.
__device__ __forceinline__ uint64_t window_bits(const uint32_t* bm, int p0, int nbits) {
  const int w = p0 >> 5, off = p0 & 31;
  const uint64_t lo = (uint64_t)bm[w] | ((uint64_t)bm[w + 1] << 32);
  uint64_t r = lo >> off;
  if (off) r |= (uint64_t)bm[w + 2] << (64 - off);
  return r & ((1ull << nbits) - 1);
}

// convolution_scalar (src/convolution/scalar.rs:5-56) at every output whose
// 2h+1 window holds a nonzero XIC cell, then ln(conv + 1) * w_f
// (src/score/scalar.rs:16-22).  Terms whose inputs are both zero add +0 and are
// skipped; the others are added in the reference's order: centre first, then
// distance h down to 1 with (left + right) * w[h - d].
__device__ __forceinline__ void convolve_row(const SearchArgs& a, const float* x,
                                             const uint32_t* bm, float wf, int C, int lane,
                                             float* vout) {
  const int h = a.h;
  const uint32_t lmask = (1u << h) - 1u;
  for (int j = lane; j < C; j += 32) {
    float v = 0.0f;
    if (j >= h && j < C - h) {
      const uint64_t m = window_bits(bm, j - h, 2 * h + 1);
      if (m) {
        float s = __fadd_rn(0.0f, __fmul_rn(x[j], a.kw[h]));
        const uint32_t lb = (uint32_t)m & lmask;
        const uint32_t rb = (uint32_t)(m >> (h + 1)) & lmask;
        uint32_t D = lb | (__brev(rb) >> (32 - h));
        while (D) {
          const int k = __ffs(D) - 1;
          const int d = h - k;
          s = __fadd_rn(s, __fmul_rn(__fadd_rn(x[j - d], x[j + d]), a.kw[k]));
          D &= D - 1;
        }
        v = __fmul_rn(ln_rn(__fadd_rn(s, 1.0f)), wf);
      }
    }
    vout[j] = v;
  }
}

__global__ void search_kernel(SearchArgs a) {
  extern __shared__ float smem_raw[];
  const int nw = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Smem S = carve(smem_raw, nw, a.cp);
  float* row = S.xrow + (size_t)warp * a.cp;
  float* vrow = S.vrow + (size_t)warp * a.cp;
  uint32_t* bm = S.bm + (size_t)warp * S.bw;
  float* scr = S.scr + warp * 32;
  unsigned long long n_read = 0, n_acc = 0, n_off = 0, n_frag = 0, n_pairs = 0, n_bins1 = 0;

  for (;;) {
    if (threadIdx.x == 0) S.misc[0] = (int)atomicAdd(a.work, 1u);
    __syncthreads();
    const int64_t p = S.misc[0];
    __syncthreads();
    if (p >= a.n_prec) break;
    const int F = a.nf[p];
    const int cs = a.cs[p], ce = a.ce[p];
    const int C = ce - cs;
    if (F == 0 || C <= 0) {
      if (threadIdx.x == 0) a.cand_n[p] = 0;
      continue;
    }
    if (C > a.c_max) {
      if (threadIdx.x == 0) {
        a.cand_n[p] = 0;
        atomicOr(a.err, 2);
      }
      continue;
    }
    const int nwin = a.nwin[p];
    for (int j = threadIdx.x; j < C; j += blockDim.x) S.score[j] = 0.0f;
    n_frag += (warp == 0 && lane == 0) ? F : 0;

    for (int r0 = 0; r0 < F; r0 += nw) {
      const int f = r0 + warp;
      const int nq = min(nw, F - r0);
      if (f < F) {
        for (int j = lane; j < C; j += 32) row[j] = 0.0f;
        for (int j = lane; j < S.bw; j += 32) bm[j] = 0u;
        __syncwarp();
        const int64_t fo = p * a.kf + f;
        const uint32_t b0 = a.blo[fo], b1 = a.bhi[fo];
        for (int wi = 0; wi < nwin; ++wi) {
          const WinInfo w = a.win[a.wins[p * a.maxw + wi]];
          gather(a, w, b0, b1, cs, ce, lane, row, bm, scr, n_read, n_acc, n_off, n_pairs, n_bins1);
        }
        __syncwarp();
        convolve_row(a, row, bm, a.fw[fo], C, lane, vrow);
      }
      __syncthreads();
      // score[j] += v_f[j] in fragment order (src/score/scalar.rs:16-22)
      for (int j = threadIdx.x; j < C; j += blockDim.x) {
        float acc = S.score[j];
        for (int q = 0; q < nq; ++q) acc = __fadd_rn(acc, S.vrow[(size_t)q * a.cp + j]);
        S.score[j] = acc;
      }
      __syncthreads();
    }

    // strict 5-point local maxima (src/peak_group_selection/mod.rs:33-43)
    if (threadIdx.x == 0) S.misc[1] = 0;
    __syncthreads();
    for (int i = threadIdx.x + 2; i < C - 2; i += blockDim.x) {
      const float* sc = S.score;
      if (sc[i - 2] < sc[i - 1] && sc[i - 1] < sc[i] && sc[i] > sc[i + 1] && sc[i + 1] > sc[i + 2]) {
        const int k = atomicAdd(&S.misc[1], 1);
        if (k < S.mx) {
          S.mval[k] = sc[i];
          S.midx[k] = i;
        }
      }
    }
    __syncthreads();
    // top-K by (value descending, cycle ascending): the reference's stable sort
    // by value of maxima found in cycle order (src/peak_group_selection/mod.rs:45-61).
    if (warp == 0) {
      const int nmax = min(S.misc[1], S.mx);
      if (S.misc[1] > S.mx && lane == 0) atomicOr(a.err, 4);
      const int kk = min(a.k_out, nmax);
      for (int r = 0; r < kk; ++r) {
        float bv = 0.0f;
        int bi = -1, bk = -1;
        for (int k = lane; k < nmax; k += 32) {
          const float v = S.mval[k];
          const int i = S.midx[k];
          if (v != v) continue;  // already taken
          if (bk < 0 || v > bv || (v == bv && i < bi)) {
            bv = v;
            bi = i;
            bk = k;
          }
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
          const float ov = __shfl_xor_sync(kFull, bv, o);
          const int oi = __shfl_xor_sync(kFull, bi, o);
          const int ok = __shfl_xor_sync(kFull, bk, o);
          if (ok >= 0 && (bk < 0 || ov > bv || (ov == bv && oi < bi))) {
            bv = ov;
            bi = oi;
            bk = ok;
          }
        }
        if (lane == 0) {
          a.cand_score[p * a.k_out + r] = bv;
          a.cand_center[p * a.k_out + r] = cs + bi;
          S.mval[bk] = __int_as_float(0x7fc00000);
        }
        __syncwarp();
      }
      if (lane == 0) a.cand_n[p] = kk;
    }
    __syncthreads();
  }
  if (a.stats) {
    // the counters are warp-uniform: count them once per warp
    if (lane == 0) {
      atomicAdd(a.stats + 0, n_pairs);
      atomicAdd(a.stats + 1, n_bins1);
      atomicAdd(a.stats + 2, n_frag);
      atomicAdd(a.stats + 3, n_read);
      atomicAdd(a.stats + 4, n_acc);
      atomicAdd(a.stats + 5, n_off);
    }
  }
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
  int64_t last_stats[6] = {0, 0, 0, 0, 0, 0};
  // workspace
  ads::DevBuf<int> nf, cs, ce, nwin, wins, cand_n, cand_center;
  ads::DevBuf<float> fw, cand_score;
  ads::DevBuf<uint32_t> blo, bhi;
  ads::DevBuf<uint8_t> keep;
  ads::DevBuf<unsigned int> work;
  ads::DevBuf<int64_t> block_sums;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // one set of four events per timed search since the last read-out
  std::vector<std::array<cudaEvent_t, 4>> stage_pool;
  size_t stage_used = 0;
  cudaEvent_t* stage_ev = nullptr;  // set of the search being enqueued
};

struct AdsCandidates {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t cap = 0;
  ads::DevBuf<uint64_t> pidx, rank, center, start, stop;
  ads::DevBuf<float> score;
  ads::DevBuf<int64_t> count_dev;
  ads::DevBuf<int> err_dev;
  int64_t count = 0;
  bool pending = false;
};

namespace ads {
namespace {

int check_params(const AdsSelectionParams& p, std::vector<float>* kernel, int* h) {
  if (p.kernel_size < 1)
    return fail(ADS_ERR_INVALID_ARGUMENT, "kernel_size must be >= 1 (the reference panics on 0)");
  if (p.kernel_size > 2 * kMaxHalf)
    return fail(ADS_ERR_INVALID_ARGUMENT, "kernel_size above 62 is not supported");
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

int reserve_candidates(AdsCandidates* c, int64_t cap) {
  if (c->cap >= cap && c->pidx.p) return ADS_OK;
  const size_t n = (size_t)std::max<int64_t>(cap, 1);
  ADS_TRY(c->pidx.alloc(n));
  ADS_TRY(c->rank.alloc(n));
  ADS_TRY(c->score.alloc(n));
  ADS_TRY(c->center.alloc(n));
  ADS_TRY(c->start.alloc(n));
  ADS_TRY(c->stop.alloc(n));
  c->cap = cap;
  return ADS_OK;
}

int launch_search(AdsSelection* s, const AdsDia* d, const AdsLib* l, AdsCandidates* c) {
  if (d->device != s->device || l->device != s->device || c->device != s->device)
    return fail(ADS_ERR_INVALID_ARGUMENT, "handles live on different devices");
  DeviceGuard dg(s->device);
  cudaStream_t st = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
  c->stream = st;
  const int64_t P = l->n_prec;
  const AdsSelectionParams& prm = s->p;
  const int L = (int)s->kernel.size();
  const int64_t n_rt = (int64_t)d->rt.size();
  int64_t launches = 0;

  const float tol_max = l->has_tol ? std::max(l->max_tol, 0.0f) : prm.rt_tolerance;
  const int64_t c_max = std::max<int64_t>(1, max_cycle_span(d->rt, d->delta_t, tol_max, prm.kernel_size));
  const int cp = (int)((c_max + 31) / 32 * 32);
  const int k_out = (int)std::max<int64_t>(0, std::min<int64_t>(prm.candidate_count, maxima_cap(cp)));
  const int kf = (int)std::max<int64_t>(1, std::min<int64_t>(prm.top_k_fragments, l->max_frag));
  const int maxw = std::max(1, d->max_overlap);

  ADS_TRY(c->count_dev.reserve(1));
  ADS_TRY(c->err_dev.reserve(1));
  ADS_TRY(reserve_candidates(c, P * (int64_t)k_out));
  ADS_CUDA(cudaMemsetAsync(c->count_dev.p, 0, sizeof(int64_t), st));
  ADS_CUDA(cudaMemsetAsync(c->err_dev.p, 0, sizeof(int), st));
  c->pending = true;
  c->count = 0;
  if (P == 0 || k_out == 0) {
    s->last_launches = 0;
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
  ADS_TRY(s->work.reserve(1));
  const int64_t nb = (P + kScanBlock - 1) / kScanBlock;
  ADS_TRY(s->block_sums.reserve((size_t)nb));
  if (s->stats_on) {
    ADS_TRY(s->stats.reserve(6));
    ADS_CUDA(cudaMemsetAsync(s->stats.p, 0, 6 * sizeof(unsigned long long), st));
  }

  GridView g;
  ADS_TRY(device_grid(s->device, &g));

  PrepArgs pa;
  pa.n_prec = P;
  pa.pmz = l->pmz.p;
  pa.prt = l->prt.p;
  pa.ptol = l->has_tol ? l->ptol.p : nullptr;
  pa.rt_tol = prm.rt_tolerance;
  pa.fstart = l->fstart.p;
  pa.fstop = l->fstop.p;
  pa.fmz = l->fmz.p;
  pa.fint = l->fint.p;
  pa.fnum = l->fnum.p;
  pa.ftype = l->ftype.p;
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
  pa.err = c->err_dev.p;
  ADS_CUDA(cudaMemsetAsync(s->work.p, 0, sizeof(unsigned int), st));
  const bool timed = s->o.time_stages != 0 && s->stage_used < 65536;
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
    prep_kernel<<<(int)prep_blocks, kPrepThreads, 0, st>>>(pa);
    ADS_LAUNCH_CHECK();
    ++launches;
  }

  int nw = s->o.warps_per_block > 0 ? s->o.warps_per_block : 4;
  nw = std::max(1, std::min(nw, 32));
  size_t smem = search_smem_bytes(nw, cp);
  int max_smem = 0;
  ADS_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
  while (smem > (size_t)max_smem && nw > 1) smem = search_smem_bytes(--nw, cp);
  if (smem > (size_t)max_smem)
    return fail(ADS_ERR_INVALID_ARGUMENT, "RT window too long for shared memory (" +
                                              std::to_string(c_max) + " cycles)");
  ADS_CUDA(cudaFuncSetAttribute(search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  ADS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, search_kernel, nw * 32, smem));
  if (occ <= 0) return fail(ADS_ERR_INTERNAL, "search kernel cannot be resident");
  int bps = s->o.blocks_per_sm > 0 ? std::min(s->o.blocks_per_sm, occ) : occ;

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
  for (int k = 0; k <= s->h; ++k) sa.kw[k] = s->kernel[k];
  sa.h = s->h;
  sa.k_out = k_out;
  sa.c_max = (int)c_max;
  sa.cp = cp;
  sa.gather_mode = s->o.gather_mode;
  sa.scan_thresh = 256;
  sa.work = s->work.p;
  sa.err = c->err_dev.p;
  sa.cand_n = s->cand_n.p;
  sa.cand_score = s->cand_score.p;
  sa.cand_center = s->cand_center.p;
  sa.stats = s->stats_on ? s->stats.p : nullptr;
  if (timed) ADS_CUDA(cudaEventRecord(s->stage_ev[1], st));
  {
    const int64_t blocks = std::min<int64_t>((int64_t)s->num_sms * bps, P);
    search_kernel<<<(int)blocks, nw * 32, smem, st>>>(sa);
    ADS_LAUNCH_CHECK();
    ++launches;
  }
  if (timed) ADS_CUDA(cudaEventRecord(s->stage_ev[2], st));

  block_sum_kernel<<<(int)nb, kScanBlock, 0, st>>>(s->cand_n.p, P, s->block_sums.p);
  ADS_LAUNCH_CHECK();
  scan_block_sums_kernel<<<1, kScanBlock, 0, st>>>(s->block_sums.p, nb, c->count_dev.p);
  ADS_LAUNCH_CHECK();
  ScatterArgs ca;
  ca.n_prec = P;
  ca.k_out = k_out;
  ca.peak_length = (uint64_t)prm.peak_length;
  ca.rt_len = (uint64_t)n_rt;
  ca.cand_n = s->cand_n.p;
  ca.cand_score = s->cand_score.p;
  ca.cand_center = s->cand_center.p;
  ca.pidx = l->pidx.p;
  ca.block_off = s->block_sums.p;
  ca.o_pidx = c->pidx.p;
  ca.o_rank = c->rank.p;
  ca.o_score = c->score.p;
  ca.o_center = c->center.p;
  ca.o_start = c->start.p;
  ca.o_stop = c->stop.p;
  scatter_kernel<<<(int)nb, kScanBlock, 0, st>>>(ca);
  ADS_LAUNCH_CHECK();
  launches += 3;
  if (timed) {
    ADS_CUDA(cudaEventRecord(s->stage_ev[3], st));
    ++s->stage_used;
  }
  s->last_launches = launches;
  return ADS_OK;
}

int finish(AdsCandidates* c) {
  if (!c->pending) return ADS_OK;
  DeviceGuard dg(c->device);
  int64_t cnt = 0;
  int err = 0;
  ADS_CUDA(cudaMemcpyAsync(&cnt, c->count_dev.p, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  ADS_CUDA(cudaMemcpyAsync(&err, c->err_dev.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  ADS_CUDA(cudaStreamSynchronize(c->stream));
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
    if (s->o.precision != ADS_PRECISION_FP32)
      return fail(ADS_ERR_INVALID_ARGUMENT, "only ADS_PRECISION_FP32 is implemented");
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
    *out = s.release();
    return ADS_OK;
  });
}

int ads_selection_destroy(AdsSelection* s) {
  return guarded([&] {
    if (!s) return ADS_OK;
    DeviceGuard dg(s->device);
    cudaStreamSynchronize(s->stream);
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
    unsigned long long v[6];
    cudaStream_t st = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
    ADS_CUDA(cudaMemcpyAsync(v, s->stats.p, sizeof(v), cudaMemcpyDeviceToHost, st));
    ADS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < 6 && i < cap; ++i) out[i] = (int64_t)v[i];
    return ADS_OK;
  });
}

int ads_candidates_create(const AdsSelection* s, AdsCandidates** out) {
  return guarded([&] {
    if (!s || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
    auto c = std::make_unique<AdsCandidates>();
    c->device = s->device;
    c->stream = s->o.stream ? (cudaStream_t)s->o.stream : s->stream;
    *out = c.release();
    return ADS_OK;
  });
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
    } cols[] = {{pidx, c->pidx.p, 8}, {rank, c->rank.p, 8},   {score, c->score.p, 4},
                {center, c->center.p, 8}, {start, c->start.p, 8}, {stop, c->stop.p, 8}};
    for (auto& col : cols)
      if (col.dst)
        ADS_CUDA(cudaMemcpyAsync(col.dst, col.src, n * col.bytes, cudaMemcpyDeviceToHost, c->stream));
    for (uint64_t* z : {scan_center, scan_start, scan_stop})
      if (z) std::memset(z, 0, n * 8);
    ADS_CUDA(cudaStreamSynchronize(c->stream));
    return ADS_OK;
  });
}

int ads_candidates_destroy(AdsCandidates* c) {
  return guarded([&] {
    if (!c) return ADS_OK;
    DeviceGuard dg(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    delete c;
    return ADS_OK;
  });
}

}  // extern "C"
