// The fused per-precursor search kernel: XIC gather -> Gaussian convolution ->
// ln(x + 1) * w -> ordered score sum -> 5-point local maxima -> top-K.
// Included by search.cu inside namespace ads::{anonymous}; uses its helpers
// (kFull, rust_bsearch_u16, lower_bound_u16).
//
// Per precursor (one block, persistent over an atomic work counter), in rounds of
// `rows` fragments (one round when the whole XIC fits in shared memory):
//   1. gather   warps take fragments round-robin; per (fragment, window) the CSR
//               offsets of all the warp's pairs are fetched together, then up to
//               128 entries of a bin range are read in one round trip and added to
//               the fragment's XIC row in CSR order;
//   2. list     the outputs whose 2h+1 input window holds a nonzero cell (the
//               bitmap of touched cells dilated by h, inside the valid region) are
//               collected into a list; every other output is exactly zero;
//   3. convolve every thread takes list entries: single-input windows take one
//               multiply, the others run the reference's stencil (fully unrolled
//               for the common half widths);
//   4. score    score[j] += ln(conv_f[j] + 1) * w_f in fragment order (logs only
//               for nonzero values);
// then maxima and top-K.  All f32 arithmetic is explicitly rounded and in the
// reference's order, so results equal the reference's except for its logf.

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
  const double2* ln_tab;
  float kw[kMaxHalf + 1];  // kernel taps w[0..h]; w[h] is the centre
  int h;
  int k_out;   // candidates kept per precursor
  int c_max;   // largest cycle range any precursor can have
  int cp;      // c_max rounded up to 32
  int rows;    // XIC rows held in shared memory (fragments per round)
  int gather_mode;
  int scan_thresh;
  unsigned int* work;
  int* err;
  int* cand_n;
  float* cand_score;
  int* cand_center;
  unsigned long long* stats;  // nullable
};

constexpr int kPrefetchChunks = 4;  // 4 x 32 CSR entries read per round trip
constexpr int kListRowShift = 11;   // list entry = row << 11 | cycle (cycle < 2048)

// XIC rows are stored skewed, cycle j at j + j/8, so that reads of neighbouring
// cycles by neighbouring threads spread over the shared-memory banks.
__host__ __device__ __forceinline__ int xs(int j) { return j + (j >> 3); }
__host__ __device__ __forceinline__ int row_stride(int cp) { return cp + cp / 8; }

__host__ __device__ inline int bitmap_words(int cp) { return cp / 32 + 3; }
__host__ __device__ inline int maxima_cap(int cp) { return cp / 4 + 8; }

// Shared-memory plan, in 4-byte words.  The per-warp duplicate tags of the gather
// and the convolved rows of the later phases share one region.
struct SmemPlan {
  int ln, kw, xrow, vrow, tags, list, bm, scr, score, mval, midx, misc, total;
  int bw, mx;
};

__host__ __device__ inline SmemPlan smem_plan(int nw, int cp, int rows) {
  SmemPlan s;
  int o = 0;
  s.bw = bitmap_words(cp);
  s.mx = maxima_cap(cp);
  s.ln = o;
  o += kLnTableSize * 4;
  s.kw = o;
  o += 32;
  s.xrow = o;
  o += rows * row_stride(cp);
  s.vrow = o;
  s.tags = o;
  o += (rows > nw ? rows : nw) * cp;
  s.list = o;
  o += (rows * cp + 1) / 2;  // u16 entries
  s.bm = o;
  o += rows * s.bw;
  s.scr = o;
  o += nw * 32;
  s.score = o;
  o += cp;
  s.mval = o;
  o += s.mx;
  s.midx = o;
  o += s.mx;
  s.misc = o;
  o += 8;
  s.total = o;
  return s;
}

struct Counters {
  unsigned long long read = 0, acc = 0, off = 0, pairs = 0, bins1 = 0, frag = 0;
};

// Adds one chunk of 32 CSR-consecutive entries to the XIC row in lane order (the
// reference's `dense_xic[c] += intensity`, src/quadrupole_observation/mod.rs:96-105).
// A tag per cell detects whether two accepted lanes hit the same cycle; only then
// are the lanes grouped and summed by their lowest lane one rounded add at a time.
// The detection never misses a collision, whatever stale tags hold.
__device__ __forceinline__ void add_chunk(bool inc, int cell, float v, int lane, float* row,
                                          uint32_t* bm, uint32_t* tags, float* scr,
                                          uint32_t& seq, unsigned long long& n_acc) {
  const unsigned act = __ballot_sync(kFull, inc);
  if (act == 0) return;
  n_acc += __popc(act);
  const uint32_t mytag = (seq << 5) | (uint32_t)lane;
  ++seq;
  uint32_t old = 0;
  if (inc) old = atomicMax(tags + cell, mytag);
  __syncwarp();
  const bool dup = inc && (tags[cell] != mytag || (old >> 5) == (mytag >> 5));
  if (!__any_sync(kFull, dup)) {
    if (inc) {
      row[xs(cell)] = __fadd_rn(row[xs(cell)], v);
      atomicOr(bm + (cell >> 5), 1u << (cell & 31));
    }
  } else {
    const int key = inc ? cell : (-1 - lane);
    const unsigned grp = __match_any_sync(kFull, key);
    scr[lane] = v;
    __syncwarp();
    if (inc && lane == __ffs(grp) - 1) {
      float acc = row[xs(cell)];
      unsigned g = grp;
      while (g) {
        const int l = __ffs(g) - 1;
        acc = __fadd_rn(acc, scr[l]);
        g &= g - 1;
      }
      row[xs(cell)] = acc;
      atomicOr(bm + (cell >> 5), 1u << (cell & 31));
    }
  }
  __syncwarp();
}

// Is `pos` the first entry of one of the bins (b0, b1)?  (slice_starts[b] == pos)
__device__ __forceinline__ bool bin_starts_at(const uint32_t* ssw, uint32_t b0, uint32_t b1,
                                              int64_t pos) {
  uint32_t lo = b0 + 1, hi = b1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((int64_t)__ldg(ssw + mid) < pos)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo < b1 && (int64_t)__ldg(ssw + lo) == pos;
}

// fill_xic_slice for one (fragment, window) pair whose bin range [b0, b1) spans
// the CSR entries [rs, re) of the window.  Two exact strategies:
//   scan     read every entry of the range, keep start < cycle < stop plus, per
//            bin, the last entry at cycle == start (where Rust's binary_search
//            lands, src/quadrupole_observation/mod.rs:91-94);
//   bsearch  per bin, binary-search the first kept entry and the first entry at or
//            past stop, then read only the kept entries.
__device__ void gather_pair(const SearchArgs& a, const WinInfo& wi, uint32_t b0, uint32_t b1,
                            int64_t rs, int64_t re, int cs, int ce, int lane, float* row,
                            uint32_t* bm, uint32_t* tags, float* scr, uint32_t& seq,
                            Counters& k) {
  const int64_t n = re - rs;
  if (n <= 0) return;
  const uint32_t* ssw = a.ss + wi.ss_off;
  const uint16_t* cy = a.cyc + wi.base;
  const float* in = a.inten + wi.base;
  const bool scan = a.gather_mode == 1 || (a.gather_mode == 0 && n <= a.scan_thresh);
  if (scan) {
    k.read += n;
    for (int64_t q0 = rs; q0 < re; q0 += 32 * kPrefetchChunks) {
      int c[kPrefetchChunks];
      float v[kPrefetchChunks];
#pragma unroll
      for (int u = 0; u < kPrefetchChunks; ++u) {
        const int64_t q = q0 + u * 32 + lane;
        c[u] = q < re ? (int)__ldg(cy + q) : -1;
        v[u] = q < re ? __ldg(in + q) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kPrefetchChunks; ++u) {
        const int64_t qb = q0 + u * 32;
        if (qb >= re) break;
        const int64_t q = qb + lane;
        const int cu = c[u];
        int nxt = __shfl_down_sync(kFull, cu, 1);
        const int nxt_first = __shfl_sync(kFull, c[u + 1 < kPrefetchChunks ? u + 1 : u], 0);
        if (lane == 31) nxt = (u + 1 < kPrefetchChunks) ? nxt_first : -2;
        bool inc = q < re && cu > cs && cu < ce;
        if (q < re && cu == cs) {
          const int64_t qn = q + 1;
          bool last = qn >= re;
          if (!last) last = bin_starts_at(ssw, b0, b1, qn);
          if (!last) {
            const int cn = nxt == -2 ? (int)__ldg(cy + qn) : nxt;
            last = cn != cs;
          }
          inc = last;
        }
        add_chunk(inc, cu - cs, v[u], lane, row, bm, tags, scr, seq, k.acc);
      }
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
      k.off += 2 * __popc(__ballot_sync(kFull, vb));
      int64_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      const int64_t total = __shfl_sync(kFull, incl, 31);
      const int64_t excl = incl - cnt;
      k.read += total;
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
        add_chunk(vt, c - cs, v, lane, row, bm, tags, scr, seq, k.acc);
      }
    }
  }
}

// nbits (<= 63) bitmap bits starting at bit p0 (p0 may be negative: bits below 0
// are zero).
__device__ __forceinline__ uint64_t window_bits(const uint32_t* bm, int p0, int nbits) {
  int shift = 0;
  if (p0 < 0) {
    shift = -p0;
    nbits -= shift;
    p0 = 0;
    if (nbits <= 0) return 0;
  }
  const int w = p0 >> 5, off = p0 & 31;
  const uint64_t lo = (uint64_t)bm[w] | ((uint64_t)bm[w + 1] << 32);
  uint64_t r = lo >> off;
  if (off) r |= (uint64_t)bm[w + 2] << (64 - off);
  r &= (1ull << nbits) - 1;
  return r << shift;
}


// Active outputs of one 32-cycle word of a row: the touched-cell bitmap dilated
// by h (cycle j is active if a touched cell lies in [j - h, j + h]), limited to the
// valid region [h, C - h) where the reference computes anything.
__device__ __forceinline__ uint32_t active_word(const uint32_t* bm, int w, int h, int C) {
  const uint32_t c = bm[w], p = w > 0 ? bm[w - 1] : 0u, n = bm[w + 1];
  uint32_t act = c;
  for (int d = 1; d <= h; ++d) act |= (c << d) | (p >> (32 - d)) | (c >> d) | (n << (32 - d));
  const int j0 = w * 32;
  const int lo = max(h - j0, 0), hi = min(C - h - j0, 32);  // valid bit range [lo, hi)
  if (hi <= lo) return 0u;
  const uint32_t upper = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
  const uint32_t lower = (1u << lo) - 1u;
  return act & upper & ~lower;
}

// One output of convolution_scalar (src/convolution/scalar.rs:30-50): x[j]*w[h]
// first, then (x[j-d] + x[j+d]) * w[h-d] for d = h..1.  Inputs that are zero add
// +0, so a window with a single nonzero input reduces to that input times its
// tap, exactly.
template <int H>
__device__ __forceinline__ float conv_output(const SearchArgs& a, const float* x,
                                             const uint32_t* bm, const float* kw_s, int j) {
  const int h = H > 0 ? H : a.h;
  const uint64_t m = window_bits(bm, j - h, 2 * h + 1);
  if (__popcll(m) == 1) {
    const int d = abs(__ffsll((long long)m) - 1 - h);
    return __fmul_rn(x[xs(j - h + __ffsll((long long)m) - 1)], kw_s[h - d]);
  }
  if (H > 0) {
    float s = __fadd_rn(0.0f, __fmul_rn(x[xs(j)], a.kw[H]));
#pragma unroll
    for (int k = 0; k < H; ++k)
      s = __fadd_rn(s, __fmul_rn(__fadd_rn(x[xs(j - H + k)], x[xs(j + H - k)]), a.kw[k]));
    return s;
  }
  // any half width: only the nonzero tap pairs, in the reference order
  float s = __fadd_rn(0.0f, __fmul_rn(x[xs(j)], kw_s[h]));
  const uint32_t lmask = (1u << h) - 1u;
  const uint32_t lb = (uint32_t)m & lmask;
  const uint32_t rb = (uint32_t)(m >> (h + 1)) & lmask;
  uint32_t D = lb | (__brev(rb) >> (32 - h));
  while (D) {
    const int k = __ffs(D) - 1;
    const int d = h - k;
    s = __fadd_rn(s, __fmul_rn(__fadd_rn(x[xs(j - d)], x[xs(j + d)]), kw_s[k]));
    D &= D - 1;
  }
  return s;
}

template <int H>
__global__ void __launch_bounds__(256) search_kernel(SearchArgs a) {
  extern __shared__ __align__(16) float smem_raw[];
  const int nw = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const SmemPlan P = smem_plan(nw, a.cp, a.rows);
  uint32_t* sw = reinterpret_cast<uint32_t*>(smem_raw);
  double2* lnt = reinterpret_cast<double2*>(smem_raw + P.ln);
  float* kw_s = smem_raw + P.kw;
  float* xrow = smem_raw + P.xrow;
  float* vrow = smem_raw + P.vrow;
  uint32_t* tags = sw + P.tags + warp * a.cp;
  uint16_t* list = reinterpret_cast<uint16_t*>(sw + P.list);
  uint32_t* bm = sw + P.bm;
  float* scr = smem_raw + P.scr + warp * 32;
  float* score = smem_raw + P.score;
  float* mval = smem_raw + P.mval;
  int* midx = reinterpret_cast<int*>(smem_raw + P.midx);
  int* misc = reinterpret_cast<int*>(smem_raw + P.misc);
  const int cp = a.cp;
  const int h = H > 0 ? H : a.h;
  const int nwords = cp / 32;
  const int n_union = (a.rows > nw ? a.rows : nw) * cp;

  for (int i = threadIdx.x; i < kLnTableSize; i += blockDim.x) lnt[i] = a.ln_tab[i];
  for (int i = threadIdx.x; i <= a.h; i += blockDim.x) kw_s[i] = a.kw[i];
  Counters k;

  for (;;) {
    if (threadIdx.x == 0) misc[0] = (int)atomicAdd(a.work, 1u);
    __syncthreads();
    const int64_t p = misc[0];
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
    if (warp == 0 && lane == 0) k.frag += F;

    for (int r0 = 0; r0 < F; r0 += a.rows) {
      const int nr = min(a.rows, F - r0);
      // zero the XIC rows, the convolved rows (which also clears the gather tags)
      // and the bitmaps
      {
        float4* x4 = reinterpret_cast<float4*>(xrow);
        const int nx4 = nr * row_stride(cp) / 4;
        for (int i = threadIdx.x; i < nx4; i += blockDim.x) x4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        float4* v4 = reinterpret_cast<float4*>(vrow);
        for (int i = threadIdx.x; i < n_union / 4; i += blockDim.x) v4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int i = threadIdx.x; i < nr * P.bw; i += blockDim.x) bm[i] = 0u;
        if (threadIdx.x == 0) misc[2] = 0;
      }
      __syncthreads();
      // ---- 1. gather: this warp's rows, all their windows
      {
        uint32_t seq = 1;
        const int my_rows = nr > warp ? (nr - warp + nw - 1) / nw : 0;
        const int n_pairs = my_rows * nwin;
        for (int pb = 0; pb < n_pairs; pb += 32) {
          // CSR offsets of up to 32 pairs in one round trip
          int64_t rs = 0, re = 0;
          uint32_t b0 = 0, b1 = 0;
          const int pi = pb + lane;
          if (pi < n_pairs) {
            const int f = r0 + warp + (pi / nwin) * nw;
            const int wi = pi % nwin;
            const int64_t fo = p * a.kf + f;
            b0 = a.blo[fo];
            b1 = a.bhi[fo];
            if (b1 > b0) {
              const WinInfo w = a.win[a.wins[p * a.maxw + wi]];
              rs = __ldg(a.ss + w.ss_off + b0);
              re = __ldg(a.ss + w.ss_off + b1);
            }
          }
          const int np = min(32, n_pairs - pb);
          for (int q = 0; q < np; ++q) {
            const int64_t qrs = __shfl_sync(kFull, rs, q);
            const int64_t qre = __shfl_sync(kFull, re, q);
            const uint32_t qb0 = __shfl_sync(kFull, b0, q);
            const uint32_t qb1 = __shfl_sync(kFull, b1, q);
            if (qb1 <= qb0) continue;
            const int pq = pb + q;
            const int fl = warp + (pq / nwin) * nw;  // row within the round
            const WinInfo w = a.win[a.wins[p * a.maxw + pq % nwin]];
            k.off += 2;
            k.pairs += 1;
            k.bins1 += qb1 - qb0 + 1;
            gather_pair(a, w, qb0, qb1, qrs, qre, cs, ce, lane, xrow + (size_t)fl * row_stride(cp),
                        bm + fl * P.bw, tags, scr, seq, k);
          }
        }
      }
      __syncthreads();
      // ---- 2. list of the outputs with a nonzero input window
      for (int it = threadIdx.x; it < nr * nwords; it += blockDim.x) {
        const int fl = it / nwords, w = it - fl * nwords;
        uint32_t act = active_word(bm + fl * P.bw, w, h, C);
        if (act) {
          int pos = atomicAdd(&misc[2], __popc(act));
          while (act) {
            const int b = __ffs(act) - 1;
            list[pos++] = (uint16_t)((fl << kListRowShift) | (w * 32 + b));
            act &= act - 1;
          }
        }
      }
      // the tags region becomes the convolved rows: clear what the gather left
      for (int i = threadIdx.x; i < nw * cp; i += blockDim.x) vrow[i] = 0.0f;
      __syncthreads();
      // ---- 3. convolution of the listed outputs
      const int n_list = misc[2];
      for (int it = threadIdx.x; it < n_list; it += blockDim.x) {
        const int e = list[it];
        const int fl = e >> kListRowShift, j = e & ((1 << kListRowShift) - 1);
        vrow[(size_t)fl * cp + j] =
            conv_output<H>(a, xrow + (size_t)fl * row_stride(cp), bm + fl * P.bw, kw_s, j);
      }
      __syncthreads();
      // ---- 4. score[j] += ln(conv_f[j] + 1) * w_f in fragment order
      // (src/score/scalar.rs:16-22); a zero conv adds ln(1) * w = +0 and is skipped
      const float* fw = a.fw + p * a.kf + r0;
      for (int j = threadIdx.x; j < C; j += blockDim.x) {
        float acc = r0 == 0 ? 0.0f : score[j];
        for (int q = 0; q < nr; ++q) {
          const float c = vrow[(size_t)q * cp + j];
          if (c != 0.0f) acc = __fadd_rn(acc, __fmul_rn(ln_fast(__fadd_rn(c, 1.0f), lnt), __ldg(fw + q)));
        }
        score[j] = acc;
      }
      __syncthreads();
    }

    // strict 5-point local maxima (src/peak_group_selection/mod.rs:33-43)
    if (threadIdx.x == 0) misc[1] = 0;
    __syncthreads();
    for (int i = threadIdx.x + 2; i < C - 2; i += blockDim.x) {
      if (score[i - 2] < score[i - 1] && score[i - 1] < score[i] && score[i] > score[i + 1] &&
          score[i + 1] > score[i + 2]) {
        const int slot = atomicAdd(&misc[1], 1);
        if (slot < P.mx) {
          mval[slot] = score[i];
          midx[slot] = i;
        }
      }
    }
    __syncthreads();
    // top-K by (value descending, cycle ascending): the reference's stable sort by
    // value of maxima found in cycle order (src/peak_group_selection/mod.rs:45-61).
    if (warp == 0) {
      const int nmax = min(misc[1], P.mx);
      if (misc[1] > P.mx && lane == 0) atomicOr(a.err, 4);
      const int kk = min(a.k_out, nmax);
      for (int r = 0; r < kk; ++r) {
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
    __syncthreads();
  }
  if (a.stats && lane == 0) {
    atomicAdd(a.stats + 0, k.pairs);
    atomicAdd(a.stats + 1, k.bins1);
    atomicAdd(a.stats + 2, k.frag);
    atomicAdd(a.stats + 3, k.read);
    atomicAdd(a.stats + 4, k.acc);
    atomicAdd(a.stats + 5, k.off);
  }
}
