// The fused per-precursor search kernel: XIC gather -> Gaussian convolution ->
// ln(x + 1) * w -> ordered score sum -> 5-point local maxima -> top-K.
// Included by search.cu inside namespace ads::{anonymous}; uses its helpers
// (kFull, rust_bsearch_u16, lower_bound_u16).
//
// One warp per precursor; warps pull precursors from an atomic counter and never
// wait on each other after the block has staged its tables.  The warp walks the
// precursor's kept fragments in order and, for each one,
//   1. gathers the fragment's XIC row into its shared-memory row: the CSR
//      entries of every (fragment, window) pair are read up to 128 at a time and
//      added to the row in CSR order (the reference's `dense_xic[c] += intensity`);
//   2. convolves the row: lane l owns S consecutive output cycles per pass of
//      32*S cycles and holds the S + 2h inputs they need in registers;
//   3. adds ln(conv + 1) * w_f to its own columns' scores.  Fragments are taken
//      in order, which is the reference's row-major accumulation
//      (src/score/scalar.rs:16-22).
// Then 5-point local maxima over the scores and a warp top-K.  All f32
// arithmetic is explicitly rounded and in the reference's order, so results
// equal the reference's except for its logf (see ln_rn).

struct SearchArgs {
  int64_t n_prec;
  const int* list;                // nullable: the precursors to search, else 0..n_prec-1
  const unsigned int* list_len;   // device length of `list`
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
  const uint16_t* inten_bf16;  // bfloat16 copy of `inten` (BF16-storage searches)
  const double2* ln_tab;
  float kw[kMaxHalf + 1];  // kernel taps w[0..h]; w[h] is the centre (h <= kMaxHalf)
  const float* kw_dev;     // the taps in device memory when h > kMaxHalf, else null
  unsigned long long kw2[kMaxHalf + 1];  // the same taps, each twice (packed f32x2 operands)
  unsigned long long zero2;   // +0.0f twice
  unsigned long long nzero2;  // -0.0f twice
  int h;
  int k_out;   // candidates kept per precursor
  int c_max;   // largest cycle range of the precursors this launch searches
  int ncell;   // cycles a warp's row holds: passes * 32 * S >= c_max
  int gather_mode;
  int scan_thresh;
  float* grow;  // per-warp working sets of a long-window launch (GROW), else null
  unsigned long long* work;
  int* err;
  int* cand_n;
  float* cand_score;
  int* cand_center;
  unsigned long long* stats;  // nullable
};

// CSR entries read per round trip of the scanning gather: 2 x 32 for f32 intensities,
// 3 x 32 for bfloat16 ones (measured: 64-entry batches are 3.7 % faster than 128 on
// 3000 x 300 FP32 data with 301-cycle windows; for BF16 storage 96-entry batches are
// 0.5-1 % faster than 128, 64 and 192 slower).
template <bool FAST>
constexpr int kPrefetchChunks = FAST ? 3 : 2;
constexpr int kBitOff = 32;         // bitmap bit of cycle c is c + kBitOff (room for -h)
constexpr int kSmemMaxCycles = 2048;  // longest RT window (cycles) a warp's shared-memory plan
                                      // holds; longer windows run with GROW
constexpr int kTouchCap = 256;      // cells a row records for clearing; beyond it the row is
                                    // zeroed whole

__host__ __device__ inline int maxima_cap(int ncell) { return ncell / 4 + 8; }

// Shared-memory address of stored index i (cycle + off) in a score array whose
// lanes own S consecutive cycles: one pad word after every S cells, so that the 32
// lanes of a warp, reading at the same offset within their segments, hit 32
// different banks.
template <int S>
__device__ __forceinline__ int xaddr(int i) {
  return i + i / S;
}

// The XIC row is read as 8-byte pairs of cells (u, u + 1), u even within a lane's
// segment, so its segments of S cells (S even) sit at an even stride of
// row_stride(S) words whose half is odd: the 16 lanes of each half-warp then hit 16
// different bank pairs.
__host__ __device__ constexpr int row_stride(int S) {
  return ((S + 2) / 2) % 2 == 1 ? S + 2 : S + 4;
}

template <int S>
__device__ __forceinline__ int raddr(int i) {
  return i + (i / S) * (row_stride(S) - S);
}

// Floor division, for offsets known at compile time.
__host__ __device__ constexpr int floordiv(int a, int b) {
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}

// Per-warp shared-memory plan, in 4-byte words.  The block's ln table (double2 x
// 256 = 1024 words) and kernel taps (h + 1 words, at least 32) come first.
struct WarpPlan {
  int row, tags, bm, scr, score, lst, mval, midx, touched, total;
  int off;        // stored index of cycle c is c + off (off >= h, a multiple of S)
  int row_words;  // words of the row, a multiple of 4
  int lead;       // bitmap words below bm[0]: a window reaching h cycles before cycle 0
                  // reads them (always zero)
  int bw;         // bitmap words from bm[0]
  int mx;         // maxima capacity
};
__host__ __device__ inline int block_header_words(int h) {
  return kLnTableSize * 4 + ((h + 1 + 31) / 32) * 32;
}

__host__ __device__ inline WarpPlan warp_plan(int S, int h, int ncell) {
  WarpPlan w;
  w.off = (h + S - 1) / S * S;
  const int span = ncell + h + w.off + S;  // stored indices [0, span) cover every read
  w.row_words = (span + (span / S + 1) * (row_stride(S) - S) + 3) & ~3;
  int o = 0;
  w.row = o;
  o += w.row_words;
  w.tags = o;  // one byte per cell: the lane that wrote it last
  o += (ncell + 3) / 4;
  w.lead = h > kBitOff ? (h - kBitOff + 31) / 32 : 0;
  w.bw = (ncell + h + kBitOff + 31) / 32 + 2;
  w.bm = o + w.lead;
  o += w.lead + w.bw;
  w.scr = o;
  o += 32;
  w.touched = o;  // cells written by the current row (16 bits each)
  o += kTouchCap / 2;
  w.score = o + 4;  // 4 words of margin below: the maxima scan reads 2 cycles early
  o += ncell + ncell / S + 12;
  o = (o + 1) & ~1;
  w.lst = o;  // one pass of non-zero convolved values: (value, score address) pairs
  o += 2 * 32 * S;
  w.mx = maxima_cap(ncell);
  if (2 * w.mx <= 2 * 32 * S) {
    // the maxima are collected after the precursor's last row is scored, when the
    // output list is free
    w.mval = w.lst;
    w.midx = w.lst + w.mx;
  } else {
    w.mval = o;
    o += w.mx;
    w.midx = o;
    o += w.mx;
  }
  w.total = (o + 3) & ~3;
  return w;
}

__host__ __device__ inline size_t search_smem_bytes(int nw, int S, int h, int ncell, bool grow = false) {
  return (size_t)(block_header_words(h) + (grow ? 0 : nw * warp_plan(S, h, ncell).total)) * 4;
}

// Launch bounds of an instance.  The FP32 shared-memory instances for half widths 10
// and 11 (kernel sizes 20-22) at 128 threads and 5 blocks per SM: up to 102 registers,
// 20 warps (on 3000 x 300 data with 301-cycle windows 9 % faster than 256 x 2, without
// spills worth noting).  Everything else at 256 x 2 (128 registers): the BF16 instances
// (the 20-warp shape was 1.5 % slower on the uneven workload), half width 16 (spilled
// up to 256 bytes and ran 13 % slower at kernel size 31), the generic half width and the
// global-memory (long-window) instances.
template <int H, bool FAST, bool GROW>
struct LaunchShape {
  static constexpr bool narrow = !FAST && !GROW && (H == 10 || H == 11);
  static constexpr int threads = narrow ? 128 : 256;
  static constexpr int blocks = narrow ? 5 : 2;
};
__host__ __device__ constexpr int launch_threads(int h, bool fast, bool grow) {
  return (!fast && !grow && (h == 10 || h == 11)) ? 128 : 256;
}

// Per-warp work counters of the statistics pass (ON); 32 bits suffice for one warp's
// share of a launch.  In the searching instances (ON = false) they hold nothing and
// compile to no instruction.
template <bool ON>
struct Count;
template <>
struct Count<true> {
  unsigned int v = 0;
  __device__ Count& operator+=(unsigned int x) {
    v += x;
    return *this;
  }
  __device__ unsigned int get() const { return v; }
};
template <>
struct Count<false> {
  __device__ Count& operator+=(unsigned int) { return *this; }
  __device__ unsigned int get() const { return 0u; }
};
template <bool ON>
struct Counters {
  Count<ON> read, acc, off, pairs, bins1, frag;
};

// The rare case of add_chunk: lanes that hit the same cycle are grouped and summed
// by their lowest lane in lane order (kept out of line: it is seldom taken).
static __device__ __noinline__ void add_chunk_grouped(bool inc, int cell, int addr, float v,
                                                      int lane, float* row, uint32_t* bm,
                                                      float* scr) {
  const int key = inc ? cell : (-1 - lane);
  const unsigned grp = __match_any_sync(kFull, key);
  scr[lane] = v;
  __syncwarp();
  if (inc && lane == __ffs(grp) - 1) {
    float acc = row[addr];
    unsigned g = grp;
    while (g) {
      const int l = __ffs(g) - 1;
      acc = __fadd_rn(acc, scr[l]);
      g &= g - 1;
    }
    row[addr] = acc;
    const int bit = cell + kBitOff;
    atomicOr(bm + (bit >> 5), 1u << (bit & 31));
  }
}

// Adds one chunk of 32 CSR-consecutive entries to the XIC row in lane order (the
// reference's `dense_xic[c] += intensity`, src/quadrupole_observation/mod.rs:96-105).
// Every accepted lane writes its lane number into its cycle's tag; a lane that
// reads back another number shares the cycle, and only then are the lanes grouped
// and summed by their lowest lane one rounded add at a time.
// Accepted cells are also appended to `touched` (the next row clears them).
template <class Acc>
__device__ __forceinline__ void add_chunk(bool inc, int cell, int addr, float v, int lane,
                                          float* row, uint32_t* bm, uint8_t* tags, float* scr,
                                          Acc& n_acc, uint16_t* touched, int& n_touched) {
  const unsigned act = __ballot_sync(kFull, inc);
  if (act == 0) return;
  n_acc += (unsigned int)__popc(act);
  if (inc) {
    const int at = n_touched + __popc(act & ((1u << lane) - 1u));
    if (at < kTouchCap) touched[at] = (uint16_t)cell;
  }
  n_touched += __popc(act);
  if (inc) tags[cell] = (uint8_t)lane;
  __syncwarp();
  const bool dup = inc && tags[cell] != (uint8_t)lane;
  const int bit = cell + kBitOff;
  if (!__any_sync(kFull, dup)) {
    if (inc) {
      row[addr] = __fadd_rn(row[addr], v);
      atomicOr(bm + (bit >> 5), 1u << (bit & 31));
    }
  } else {
    add_chunk_grouped(inc, cell, addr, v, lane, row, bm, scr);
  }
  __syncwarp();
}

// Is `pos` the first entry of one of the bins (b0, b1)?  (slice_starts[b] == pos)
// Kept out of line: only entries at the window's first cycle ask.
static __device__ __noinline__ bool bin_starts_at(const uint32_t* ssw, uint32_t b0, uint32_t b1,
                                                  uint32_t pos) {
  uint32_t lo = b0 + 1, hi = b1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(ssw + mid) < pos)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo < b1 && __ldg(ssw + lo) == pos;
}

// fill_xic_slice for one (fragment, window) pair whose bin range [b0, b1) spans
// the CSR entries [rs, re) of the window.  Two exact strategies:
//   scan     read every entry of the range, keep start < cycle < stop plus, per
//            bin, the last entry at cycle == start (where Rust's binary_search
//            lands, src/quadrupole_observation/mod.rs:91-94);
//   bsearch  per bin, binary-search the first kept entry and the first entry at or
//            past stop, then read only the kept entries.
// Up to 32 * NC CSR entries (cycle, intensity) of a scanned range, one per lane and
// chunk, -1 / 0 past its end.
template <int NC>
struct ScanBatch {
  int c[NC];
  float v[NC];
};

// Entries of one observation: CSR positions are 32-bit offsets from its base.
struct WinEntries {
  const uint16_t* cy;
  const float* in;
  const uint16_t* in16;  // bfloat16 copy (BF16-storage searches)
};

__device__ __forceinline__ WinEntries win_entries(const SearchArgs& a, int64_t wbase) {
  return WinEntries{a.cyc + wbase, a.inten + wbase, a.inten_bf16 + wbase};
}

// Intensity of entry q: f32, or (BF16 storage) the bfloat16 copy widened.
template <bool FAST>
__device__ __forceinline__ float ld_intensity(const WinEntries& e, uint32_t q) {
  if (FAST) return __uint_as_float((uint32_t)__ldg(e.in16 + q) << 16);
  return __ldg(e.in + q);
}

template <bool FAST>
__device__ __forceinline__ void load_batch(const WinEntries& e, uint32_t q0, uint32_t re, int lane,
                                           ScanBatch<kPrefetchChunks<FAST>>& b) {
#pragma unroll
  for (int u = 0; u < kPrefetchChunks<FAST>; ++u) {
    const uint32_t q = q0 + u * 32 + lane;
    b.c[u] = q < re ? (int)__ldg(e.cy + q) : -1;
    b.v[u] = q < re ? ld_intensity<FAST>(e, q) : 0.0f;
  }
}

__device__ __forceinline__ bool scans(const SearchArgs& a, uint32_t n) {
  return a.gather_mode == 1 || (a.gather_mode == 0 && n <= (uint32_t)a.scan_thresh);
}

// `pre`: the range's first batch, already loaded (or null).
template <int S, bool FAST, bool STATS>
__device__ __forceinline__ void gather_pair(const SearchArgs& a, int wsel, int64_t wbase,
                                            uint32_t b0, uint32_t b1, uint32_t rs, uint32_t re,
                                            int cs, int ce, int lane, float* row, int off,
                                            uint32_t* bm, uint8_t* tags, float* scr,
                                            Counters<STATS>& k,
                                            const ScanBatch<kPrefetchChunks<FAST>>* pre,
                                            uint16_t* touched,
                                            int& n_touched) {
  if (re <= rs) return;
  const uint32_t n = re - rs;
  const WinEntries e = win_entries(a, wbase);
  if (scans(a, n)) {
    k.read += (unsigned int)n;
    constexpr int NC = kPrefetchChunks<FAST>;
    for (uint32_t q0 = rs; q0 < re; q0 += 32 * NC) {
      ScanBatch<NC> bt;
      if (pre != nullptr && q0 == rs)
        bt = *pre;
      else
        load_batch<FAST>(e, q0, re, lane, bt);
#pragma unroll
      for (int u = 0; u < NC; ++u) {
        const uint32_t qb = q0 + u * 32;
        if (qb >= re) break;
        const uint32_t q = qb + lane;
        const int cu = bt.c[u];
        bool inc = q < re && cu > cs && cu < ce;
        const bool at_start = q < re && cu == cs;
        if (__any_sync(kFull, at_start)) {
          int nxt = __shfl_down_sync(kFull, cu, 1);
          const int nxt_first = __shfl_sync(kFull, bt.c[u + 1 < NC ? u + 1 : u], 0);
          if (lane == 31) nxt = (u + 1 < NC) ? nxt_first : -2;
          if (at_start) {
            const uint32_t qn = q + 1;
            bool last = qn >= re;
            if (!last) last = bin_starts_at(a.ss + a.win[wsel].ss_off, b0, b1, qn);
            if (!last) {
              const int cn = nxt == -2 ? (int)__ldg(e.cy + qn) : nxt;
              last = cn != cs;
            }
            inc = last;
          }
        }
        const int cell = cu - cs;
        add_chunk(inc, cell, inc ? raddr<S>(cell + off) : 0, bt.v[u], lane, row, bm, tags, scr,
                  k.acc, touched, n_touched);
      }
    }
  } else {
    const uint32_t* ssw = a.ss + a.win[wsel].ss_off;
    const uint16_t* cy = e.cy;
    for (uint32_t bb = b0; bb < b1; bb += 32) {
      const uint32_t b = bb + lane;
      const bool vb = b < b1;
      int64_t pos = 0, cnt = 0;
      if (vb) {
        const int64_t s0 = __ldg(ssw + b), s1 = __ldg(ssw + b + 1);
        pos = s0 + rust_bsearch_u16(cy + s0, s1 - s0, cs);
        const int64_t end = pos + lower_bound_u16(cy + pos, s1 - pos, ce);
        cnt = end - pos;
      }
      k.off += 2u * (unsigned int)__popc(__ballot_sync(kFull, vb));
      int64_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      const int64_t total = __shfl_sync(kFull, incl, 31);
      const int64_t excl = incl - cnt;
      k.read += (unsigned int)total;
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
        const float v = vt ? ld_intensity<FAST>(e, (uint32_t)q) : 0.0f;
        const int cell = c - cs;
        add_chunk(vt, cell, vt ? raddr<S>(cell + off) : 0, v, lane, row, bm, tags, scr, k.acc,
                  touched, n_touched);
      }
    }
  }
}

// Any bit set in bm[lo, lo + n)?  (n >= 1; lo may be negative: the shift and mask
// below are floor division and remainder on two's-complement ints, and the words
// below bm[0] that such a range reaches are reserved and zero)
__device__ __forceinline__ bool bits_any(const uint32_t* bm, int lo, int n) {
  const int last = lo + n - 1;
  const int w0 = lo >> 5, w1 = last >> 5;
  uint32_t acc = 0;
  for (int w = w0; w <= w1; ++w) {
    uint32_t v = bm[w];
    if (w == w0) v &= 0xffffffffu << (lo & 31);
    if (w == w1) v &= 0xffffffffu >> (31 - (last & 31));
    acc |= v;
  }
  return acc != 0u;
}

// Packed f32x2 arithmetic (sm_100a): one instruction performs two independent f32
// operations, each rounded to nearest exactly like __fadd_rn / __fmul_rn /
// __fmaf_rn, so a packed result is bit-identical to the two scalar ones.
//
// ptxas contracts a packed multiply followed by a packed add into one fused
// multiply-add even with explicit .rn rounding and --fmad=false (measured on
// sm_100a: about half of 12-term chains differed).  The exact path therefore forms
// each rounded product as fma(a, b, -0), with the -0 a kernel argument that ptxas
// cannot see: fma(a, b, -0) = round(a * b) bit for bit, and an fma followed by an
// add is not contractible.  The +0 of the reference's `0 + x * w` is a kernel
// argument for the same reason.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pk2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}

__device__ __forceinline__ void unpk2(f32x2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// One output of convolution_scalar (src/convolution/scalar.rs:30-50) read from the
// row in shared memory: x[j]*w[h] first, then (x[j-d] + x[j+d]) * w[h-d] for
// d = h..1.  Any half width; used off the main path.  FAST (BF16 storage) fuses
// each multiply-add.
template <int S, bool FAST>
__device__ __forceinline__ float conv_at(const float* row, int off, const float* kw_s, int h,
                                         int j) {
  float s = __fadd_rn(0.0f, __fmul_rn(row[raddr<S>(j + off)], kw_s[h]));
  for (int t = 0; t < h; ++t) {
    const float lr = __fadd_rn(row[raddr<S>(j - h + t + off)], row[raddr<S>(j + h - t + off)]);
    s = FAST ? __fmaf_rn(lr, kw_s[t], s) : __fadd_rn(s, __fmul_rn(lr, kw_s[t]));
  }
  return s;
}

// ln(1 + c) for the BF16-storage path: the hardware log2 (absolute error about
// 2^-21) where ln(1 + c) >= ln(17/16), and the series c - c^2/2 + ... + c^7/7
// (relative error below 2^-26) for |c| < 1/16, so that small terms keep their
// relative accuracy.
__device__ __forceinline__ float ln1p_fast(float c) {
  float p = __fmaf_rn(c, -1.0f / 7.0f, 1.0f / 6.0f);
  p = __fmaf_rn(c, p, -1.0f / 5.0f);
  p = __fmaf_rn(c, p, 1.0f / 4.0f);
  p = __fmaf_rn(c, p, -1.0f / 3.0f);
  p = __fmaf_rn(c, p, 1.0f / 2.0f);
  p = __fmaf_rn(c, -p, 1.0f);  // 1 - c/2 + c^2/3 - ...
  const float series = __fmul_rn(c, p);
  return fabsf(c) < 0.0625f ? series : __logf(__fadd_rn(c, 1.0f));
}

// score[j] += ln(c + 1) * w (src/score/scalar.rs:16-22): one rounded operation at a
// time with the exact ln; FAST (BF16 storage) takes the hardware log2 and a fused
// multiply-add.
template <bool FAST>
__device__ __forceinline__ float score_term(float s, float c, float w, const double2* lnt) {
  if (FAST) return __fmaf_rn(ln1p_fast(c), w, s);
  return __fadd_rn(s, __fmul_rn(ln_fast(__fadd_rn(c, 1.0f), lnt), w));
}

template <bool FAST>
__device__ __forceinline__ void score_add(float* score, int addr, float c, float w,
                                          const double2* lnt) {
  if (FAST)
    score[addr] = __fmaf_rn(ln1p_fast(c), w, score[addr]);
  else
    score[addr] = __fadd_rn(score[addr], __fmul_rn(ln_fast(__fadd_rn(c, 1.0f), lnt), w));
}

// Candidate order: value descending, then cycle ascending (maxima values are never
// NaN: every comparison with NaN is false, so NaN is never a strict maximum).
__device__ __forceinline__ bool better(float av, int ai, float bv, int bi) {
  return av > bv || (av == bv && ai < bi);
}

// Compare-exchange between lanes l and l ^ j, the better key going to the lane
// that `keep_best` marks.
__device__ __forceinline__ void cmpx(float& v, int& i, int j, bool keep_best) {
  const float ov = __shfl_xor_sync(kFull, v, j);
  const int oi = __shfl_xor_sync(kFull, i, j);
  if (keep_best ? better(ov, oi, v, i) : better(v, i, ov, oi)) {
    v = ov;
    i = oi;
  }
}

// Bitonic sort of one key per lane, best in lane 0.
__device__ __forceinline__ void warp_sort_best_first(float& v, int& i, int lane) {
#pragma unroll 1
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll 1
    for (int j = k >> 1; j > 0; j >>= 1) cmpx(v, i, j, ((lane & j) == 0) == ((lane & k) == 0));
}

// Sorts a bitonic sequence across the lanes, best in lane 0.
__device__ __forceinline__ void warp_merge_best_first(float& v, int& i, int lane) {
#pragma unroll 1
  for (int j = 16; j > 0; j >>= 1) cmpx(v, i, j, (lane & j) == 0);
}

// The CSR ranges of a precursor's (fragment, window) pairs, fetched 32 at a time
// (lane q holds pair pb + q), and the first batch of the next row's first pair,
// loaded while the current row is convolved.
template <bool FAST>
struct PairCursor {
  int pb = -64;
  uint32_t rs = 0, re = 0, b0 = 0, b1 = 0;
  int wsel = 0;
  int64_t wbase = 0;
  ScanBatch<kPrefetchChunks<FAST>> pre;
  int pre_pi = -1;
};

// Gathers fragment f's XIC row: its (fragment, window) pairs in window order (the
// reference's DenseXICObservation::new, src/dense_xic_observation/mod.rs:30-64),
// then prefetches the first batch of the next fragment's first pair.
template <int S, bool FAST, bool STATS>
__device__ __forceinline__ void gather_row(const SearchArgs& a, int64_t p, int f, int nwin,
                                           int npairs, int cs, int ce, int lane,
                                           PairCursor<FAST>& pc, float* row, int off,
                                           uint32_t* bm, uint8_t* tags, float* scr,
                                           Counters<STATS>& k,
                                           uint16_t* touched, int& n_touched) {
  for (int wi = 0; wi < nwin; ++wi) {
    const int pi = f * nwin + wi;
    if (pi >= pc.pb + 32) {
      pc.pb = pi;
      const int pj = pc.pb + lane;
      pc.rs = pc.re = 0;
      pc.b0 = pc.b1 = 0;
      pc.wsel = 0;
      pc.wbase = 0;
      if (pj < npairs) {
        const int fj = pj / nwin, wj = pj - fj * nwin;
        const int64_t fo = p * a.kf + fj;
        pc.b0 = a.blo[fo];
        pc.b1 = a.bhi[fo];
        pc.wsel = a.wins[p * a.maxw + wj];
        if (pc.b1 > pc.b0) {
          const WinInfo w = a.win[pc.wsel];
          pc.wbase = w.base;
          pc.rs = __ldg(a.ss + w.ss_off + pc.b0);
          pc.re = __ldg(a.ss + w.ss_off + pc.b1);
        }
      }
    }
    const int q = pi - pc.pb;
    const uint32_t qrs = __shfl_sync(kFull, pc.rs, q);
    const uint32_t qre = __shfl_sync(kFull, pc.re, q);
    const uint32_t qb0 = __shfl_sync(kFull, pc.b0, q);
    const uint32_t qb1 = __shfl_sync(kFull, pc.b1, q);
    const int qw = __shfl_sync(kFull, pc.wsel, q);
    const int64_t qbase = __shfl_sync(kFull, pc.wbase, q);
    if (qb1 <= qb0) continue;
    k.off += 2u;
    k.pairs += 1u;
    k.bins1 += qb1 - qb0 + 1;
    gather_pair<S, FAST, STATS>(a, qw, qbase, qb0, qb1, qrs, qre, cs, ce, lane, row, off, bm, tags, scr,
                         k, pi == pc.pre_pi ? &pc.pre : nullptr, touched, n_touched);
  }
  __syncwarp();
  const int pn = (f + 1) * nwin;
  pc.pre_pi = -1;
  if (pn < npairs && pn < pc.pb + 32) {
    const int q = pn - pc.pb;
    const uint32_t nrs = __shfl_sync(kFull, pc.rs, q), nre = __shfl_sync(kFull, pc.re, q);
    const uint32_t nb0 = __shfl_sync(kFull, pc.b0, q), nb1 = __shfl_sync(kFull, pc.b1, q);
    const int64_t nbase = __shfl_sync(kFull, pc.wbase, q);
    if (nb1 > nb0 && nre > nrs && scans(a, nre - nrs)) {
      load_batch<FAST>(win_entries(a, nbase), nrs, nre, lane, pc.pre);
      pc.pre_pi = pn;
    }
  }
}

// Strict 5-point local maxima of a precursor's scores (src/peak_group_selection/mod.rs:33-43),
// collected in cycle order, and the top K of them by (value descending, cycle
// ascending), the reference's stable sort (src/peak_group_selection/mod.rs:45-61),
// written to the candidate slots.  `score` holds cycle j at xaddr<S>(j), with two
// readable words below cycle 0 and S + 2 cycles past C.
template <int S>
__device__ __forceinline__ void pick_top_k(const SearchArgs& a, int64_t p, int cs, int C,
                                           const float* score, float* mval, int* midx, int mx,
                                           int lane) {
  const int passes = (C + 32 * S - 1) / (32 * S);
  // lane l's maxima of a pass go after those of lanes < l
  int nmax = 0;
  for (int ps = 0; ps < passes; ++ps) {
    const int seg = ps * 32 + lane;
    const float* sb = score + seg * (S + 1);
    uint32_t mk = 0;
    if (seg * S < C - 2 && seg * S + S > 2) {
      float v[S + 4];
#pragma unroll
      for (int t = 0; t < S + 4; ++t) v[t] = sb[(t - 2) + floordiv(t - 2, S)];
#pragma unroll
      for (int m = 0; m < S; ++m) {
        const int i = seg * S + m;
        const bool is = i >= 2 && i < C - 2 && v[m] < v[m + 1] && v[m + 1] < v[m + 2] &&
                        v[m + 2] > v[m + 3] && v[m + 3] > v[m + 4];
        mk |= (uint32_t)is << m;
      }
    }
    const int cnt = __popc(mk);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    int pos = nmax + incl - cnt;
    while (mk) {
      const int m = __ffs(mk) - 1;
      if (pos < mx) {
        mval[pos] = sb[m];
        midx[pos] = seg * S + m;
      }
      ++pos;
      mk &= mk - 1;
    }
    nmax += __shfl_sync(kFull, incl, 31);
  }
  __syncwarp();
  if (nmax > mx) {  // cannot happen: maxima are at least 4 cycles apart
    if (lane == 0) atomicOr(a.err, 4);
    nmax = mx;
  }
  const int kk = min(a.k_out, nmax);
  if (a.k_out <= 32) {
    // the best 32 of the maxima, sorted in the lanes: chunks of 32 are sorted
    // and merged into the running best 32
    float bv = -INFINITY;
    int bi = INT_MAX;
    for (int q0 = 0; q0 < nmax; q0 += 32) {
      float v = q0 + lane < nmax ? mval[q0 + lane] : -INFINITY;
      int i = q0 + lane < nmax ? midx[q0 + lane] : INT_MAX;
      warp_sort_best_first(v, i, lane);
      if (q0 == 0) {
        bv = v;
        bi = i;
      } else {
        const float rv = __shfl_sync(kFull, v, 31 - lane);
        const int ri = __shfl_sync(kFull, i, 31 - lane);
        if (better(rv, ri, bv, bi)) {
          bv = rv;
          bi = ri;
        }
        warp_merge_best_first(bv, bi, lane);
      }
    }
    if (lane < kk) {
      a.cand_score[p * a.k_out + lane] = bv;
      a.cand_center[p * a.k_out + lane] = cs + bi;
    }
  }
  for (int r = 0; a.k_out > 32 && r < kk; ++r) {
    float bv = 0.0f;
    int bi = -1, bk = -1;
    for (int q = lane; q < nmax; q += 32) {
      const float v = mval[q];
      const int i = midx[q];
      if (v != v) continue;  // already taken
      if (bk < 0 || v > bv || (v == bv && i < bi)) {
        bv = v;
        bi = i;
        bk = q;
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
      mval[bk] = __int_as_float(0x7fc00000);
    }
    __syncwarp();
  }
  if (lane == 0) a.cand_n[p] = kk;
}

// Per-warp work counters to the statistics pass's totals.
template <bool STATS>
__device__ __forceinline__ void flush_counters(const SearchArgs& a, const Counters<STATS>& k,
                                               int lane) {
  if (STATS && a.stats && lane == 0) {
    atomicAdd(a.stats + 0, (unsigned long long)k.pairs.get());
    atomicAdd(a.stats + 1, (unsigned long long)k.bins1.get());
    atomicAdd(a.stats + 2, (unsigned long long)k.frag.get());
    atomicAdd(a.stats + 3, (unsigned long long)k.read.get());
    atomicAdd(a.stats + 4, (unsigned long long)k.acc.get());
    atomicAdd(a.stats + 5, (unsigned long long)k.off.get());
  }
}

// GROW: the warp's working set (row, tags, bitmap, scores, lists, maxima) lives in
// a global buffer of P.total words per warp (`a.grow`) instead of shared memory, for
// RT windows longer than kSmemMaxCycles; the code and every operation are the same.
// STATS: the statistics pass's work counters (compiled in only for it).
template <int H, int S, bool FAST, bool GROW, bool STATS>
__global__ void __launch_bounds__(LaunchShape<H, FAST, GROW>::threads, LaunchShape<H, FAST, GROW>::blocks)
    search_kernel(SearchArgs a) {
  extern __shared__ __align__(16) float smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int h = H > 0 ? H : a.h;
  const WarpPlan P = warp_plan(S, h, a.ncell);
  double2* lnt = reinterpret_cast<double2*>(smem_raw);
  float* kw_s = smem_raw + kLnTableSize * 4;
  float* wb = GROW ? a.grow + ((size_t)blockIdx.x * (blockDim.x >> 5) + warp) * (size_t)P.total
                   : smem_raw + block_header_words(h) + warp * P.total;
  float* row = wb + P.row;
  uint8_t* tags = reinterpret_cast<uint8_t*>(wb + P.tags);
  uint32_t* bm = reinterpret_cast<uint32_t*>(wb + P.bm);
  float* scr = wb + P.scr;
  float* score = wb + P.score;
  float* mval = wb + P.mval;
  int* midx = reinterpret_cast<int*>(wb + P.midx);
  uint16_t* touched = reinterpret_cast<uint16_t*>(wb + P.touched);
  int n_touched = 0;  // cells the last row wrote (warp-uniform)
  {
    float4* r4 = reinterpret_cast<float4*>(row);
    for (int i = lane; i < P.row_words / 4; i += 32) r4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = lane - P.lead; i < P.bw; i += 32) bm[i] = 0u;
  }

  for (int i = threadIdx.x; i < kLnTableSize; i += blockDim.x) lnt[i] = a.ln_tab[i];
  for (int i = threadIdx.x; i <= a.h; i += blockDim.x) kw_s[i] = a.kw_dev ? a.kw_dev[i] : a.kw[i];
  __syncthreads();
  Counters<STATS> k;

  const unsigned long long n_work = a.list ? (unsigned long long)*a.list_len
                                            : (unsigned long long)a.n_prec;
  for (;;) {
    unsigned long long pw = 0;
    if (lane == 0) pw = atomicAdd(a.work, 1ull);
    pw = __shfl_sync(kFull, pw, 0);
    if (pw >= n_work) break;
    const int64_t p = a.list ? (int64_t)a.list[pw] : (int64_t)pw;
    const int F = a.nf[p];
    const int cs = a.cs[p], ce = a.ce[p];
    const int C = ce - cs;
    if (F == 0 || C <= 0) {
      if (lane == 0) a.cand_n[p] = 0;
      continue;
    }
    if (C > a.c_max) {
      if (lane == 0) {
        a.cand_n[p] = 0;
        atomicOr(a.err, 2);
      }
      continue;
    }
    const int nwin = a.nwin[p];
    const int npairs = F * nwin;
    const int passes = (C + 32 * S - 1) / (32 * S);
    k.frag += F;
    // fragment weights, lane f holding fragment f's (fetched once per precursor)
    const float wf_lane = lane < F ? __ldg(a.fw + p * a.kf + lane) : 0.0f;
    for (int i = lane; i <= C + C / S; i += 32) score[i] = 0.0f;  // cycles [0, C) with pads

    PairCursor<FAST> pc;
    for (int f = 0; f < F; ++f) {
      // the previous row's cells (and bitmap words) back to zero
      if (n_touched > kTouchCap) {
        float4* r4 = reinterpret_cast<float4*>(row);
        for (int i = lane; i < P.row_words / 4; i += 32) r4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int i = lane; i < P.bw; i += 32) bm[i] = 0u;
      } else {
        for (int i = lane; i < n_touched; i += 32) {
          const int c = touched[i];
          row[raddr<S>(c + P.off)] = 0.0f;
          bm[(c + kBitOff) >> 5] = 0u;
        }
      }
      n_touched = 0;
      __syncwarp();
      // ---- 1. gather: the fragment's pairs in window order
      gather_row<S, FAST, STATS>(a, p, f, nwin, npairs, cs, ce, lane, pc, row, P.off, bm, tags,
                                 scr, k, touched, n_touched);
      float wf = __shfl_sync(kFull, wf_lane, f & 31);
      if (f >= 32) wf = __ldg(a.fw + p * a.kf + f);
      if (!isfinite(wf)) {
        // ln(conv + 1) * inf is NaN even where conv is zero: every column takes
        // its term, as in the reference
        for (int j = lane; j < C; j += 32) {
          const float c = (j >= h && j < C - h) ? conv_at<S, FAST>(row, P.off, kw_s, h, j) : 0.0f;
          score_add<FAST>(score, xaddr<S>(j), c, wf, lnt);
        }
        __syncwarp();
        continue;
      }
      if (n_touched == 0) continue;  // no entry accepted: every term is +0
      // ---- 2./3. convolution of this lane's cycles, then the score terms of its
      // non-zero outputs.  A zero output adds ln(1) * w = +0, which leaves a score as
      // it is, so only non-zero outputs of the valid range [h, C - h) are listed
      // (warp-compacted, in lane order) and take a logarithm.
      float2* lst = reinterpret_cast<float2*>(wb + P.lst);
      for (int ps = 0; ps < passes; ++ps) {
        const int j0 = ps * 32 * S + lane * S;
        const bool act = j0 + S > h && j0 < C - h && bits_any(bm, j0 - h + kBitOff, S + 2 * h);
        if (!__any_sync(kFull, act)) continue;
        uint32_t mk = 0;
        float cv[S];
        if (H > 0) {
          if (act) {
            // cells u in [UB, UE) of this lane's segment as 8-byte pairs (u even);
            // every output is formed in the reference's order: 0 + x[j]*w[h], then
            // + (x[j-d] + x[j+d]) * w[h-d] for d = h..1, two outputs (m, m + 1) per
            // packed instruction.  For odd d the pair sums straddle the register
            // pairs and are formed by two scalar adds.
            constexpr int UB = -((H + 1) & ~1);
            constexpr int UE = (S + H + 1) & ~1;
            constexpr int NX = UE - UB;
            const float* rb = row + (ps * 32 + lane + P.off / S) * row_stride(S);
            float xv[NX];
#pragma unroll
            for (int q = 0; q < NX; q += 2) {
              const int u = UB + q;
              const float2 v =
                  *reinterpret_cast<const float2*>(rb + u + floordiv(u, S) * (row_stride(S) - S));
              xv[q] = v.x;
              xv[q + 1] = v.y;
            }
#pragma unroll
            for (int m = 0; m < S; m += 2) {
              f32x2 acc = add2(a.zero2, fma2(pk2(xv[m - UB], xv[m + 1 - UB]), a.kw2[H], a.nzero2));
#pragma unroll
              for (int t = 0; t < H; ++t) {
                const int d = H - t;
                f32x2 lr;
                if (d % 2 == 0)
                  lr = add2(pk2(xv[m - d - UB], xv[m - d + 1 - UB]),
                            pk2(xv[m + d - UB], xv[m + d + 1 - UB]));
                else
                  lr = pk2(__fadd_rn(xv[m - d - UB], xv[m + d - UB]),
                           __fadd_rn(xv[m + 1 - d - UB], xv[m + 1 + d - UB]));
                acc = FAST ? fma2(lr, a.kw2[t], acc) : add2(acc, fma2(lr, a.kw2[t], a.nzero2));
              }
              unpk2(acc, cv[m], cv[m + 1]);
            }
          }
        } else if (act) {
#pragma unroll
          for (int m = 0; m < S; ++m) {
            const int j = j0 + m;
            cv[m] = (j >= h && j < C - h) ? conv_at<S, FAST>(row, P.off, kw_s, h, j) : 0.0f;
          }
        }
        if (act) {
          const int m0 = max(h - j0, 0), m1 = min(C - h - j0, S);
#pragma unroll
          for (int m = 0; m < S; ++m)
            mk |= (uint32_t)(m >= m0 && m < m1 && cv[m] != 0.0f) << m;
        }
        const int cnt = __popc(mk);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += t;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        int pos = incl - cnt;
        const int sbase = (ps * 32 + lane) * (S + 1);  // score address of cycle j0
#pragma unroll
        for (int m = 0; m < S; ++m)
          if ((mk >> m) & 1u) lst[pos++] = make_float2(cv[m], __int_as_float(sbase + m));
        __syncwarp();
        for (int i = lane; i < total; i += 32) {
          const float2 e = lst[i];
          const int at = __float_as_int(e.y);
          score[at] = score_term<FAST>(score[at], e.x, wf, lnt);
        }
        __syncwarp();
      }
      __syncwarp();
    }
    __syncwarp();

    pick_top_k<S>(a, p, cs, C, score, mval, midx, P.mx, lane);
  }
  flush_counters<STATS>(a, k, lane);
}
