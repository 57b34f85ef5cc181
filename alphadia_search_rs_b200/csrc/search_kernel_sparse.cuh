// The BF16-storage search kernel: XIC gather -> scatter convolution -> ln(conv + 1) * w
// on the written outputs -> ordered score sum -> 5-point local maxima -> top-K.
// Included by search.cu after search_kernel.cuh (shares its gather, maxima and
// top-K code).
//
// The BF16 path reads intensities stored as bfloat16 and is compared with the FP64
// oracle, not bit for bit, so it need not keep the reference's order of the
// convolution's additions.  The convolution is linear: the output at cycle j is the
// sum over XIC cells c within h of j of x[c] * w(|j - c|).  A fragment row holds a few
// dozen touched cells among hundreds of cycles, so instead of evaluating the 2h + 1
// taps at every output of a segment (the exact kernel's dense stencil), each touched
// cell adds its x * w to the 2h + 1 outputs around it (shared-memory float atomics;
// the cells of one instruction are distinct, so no two lanes of an instruction add to
// the same output) and marks them in an output bitmap; ln(conv + 1) * w_f is then
// taken only at the marked outputs, one bitmap word (32 outputs) at a time.  XIC cells
// are still summed in CSR order (the exact kernel's gather), and scores in fragment
// order, so results do not depend on the launch shape.  Accumulation, log and score
// stay f32.
//
// Per-warp working set (words): XIC row, tags, touched-cell bitmap, output bitmap,
// convolution row, the unique touched cells of the current row, scores (the exact
// kernel's layout with kSparseS cycles per segment, for pick_top_k) and maxima.

constexpr int kSparseS = 16;            // score segments (pick_top_k layout)
constexpr int kSparseCells = 32 * kSparseS;  // cycles of one maxima pass
constexpr int kSparseHeaderWords = 32;  // the block's kernel taps

struct SparsePlan {
  int row, tags, bm, ob, conv, scr, touched, score, mval, midx, total;
  int bw, ow, mx;
};

// ncell: a multiple of kSparseCells, at least the longest window of the launch.
__host__ __device__ inline SparsePlan sparse_plan(int h, int ncell) {
  SparsePlan w;
  int o = 0;
  w.row = o;  // XIC cell c at row[c]
  o += ncell;
  w.tags = o;
  o += ncell;
  w.bw = (ncell + kBitOff + 31) / 32 + 1;  // touched cells: bit c + kBitOff
  w.bm = o;
  o += w.bw;
  w.ow = (ncell + h + kBitOff + 31) / 32 + 2;  // written outputs: bit j + kBitOff, j in [-h, ncell + h)
  w.ob = o;
  o += w.ow;
  w.conv = o;  // output j at conv[j + h]
  o += ncell + 2 * h;
  w.scr = o;
  o += 32;
  w.touched = o;
  o += kTouchCap / 2;
  w.score = o + 4;  // 4 words of margin below: the maxima scan reads 2 cycles early
  o += ncell + ncell / kSparseS + 12;
  o = (o + 1) & ~1;
  w.mx = maxima_cap(ncell);
  w.mval = o;
  o += w.mx;
  w.midx = o;
  o += w.mx;
  w.total = (o + 3) & ~3;
  return w;
}

__host__ __device__ inline size_t sparse_smem_bytes(int nw, int h, int ncell, bool grow) {
  return (size_t)(kSparseHeaderWords + (grow ? 0 : nw * sparse_plan(h, ncell).total)) * 4;
}

// Cell c's XIC value x added to the outputs c - h .. c + h with weights w(|k|) =
// kernel[h - |k|] (the taps the reference pairs at distance |k|,
// src/convolution/scalar.rs:30-50), and those outputs marked in the bitmap.
template <int H>
__device__ __forceinline__ void scatter_cell(const SearchArgs& a, const float* kw_s, int h,
                                             float* conv, uint32_t* ob, int c, float x) {
  float* cv = conv + c + h;
  if (H > 0) {
#pragma unroll
    for (int k = -H; k <= H; ++k) atomicAdd(cv + k, __fmul_rn(x, a.kw[H - (k < 0 ? -k : k)]));
  } else {
    for (int k = -h; k <= h; ++k) atomicAdd(cv + k, __fmul_rn(x, kw_s[h - (k < 0 ? -k : k)]));
  }
  const int b0 = c - h + kBitOff;  // >= 0: h <= kMaxHalf < kBitOff
  const int w0 = b0 >> 5, sh = b0 & 31;
  const uint64_t m = (1ull << (2 * h + 1)) - 1ull;  // 2h + 1 <= 63 bits
  const uint64_t lo = m << sh;
  atomicOr(ob + w0, (uint32_t)lo);
  atomicOr(ob + w0 + 1, (uint32_t)(lo >> 32));
  if (sh != 0) {
    const uint32_t hi = (uint32_t)(m >> (64 - sh));
    if (hi) atomicOr(ob + w0 + 2, hi);
  }
}

// GROW: the warp's working set lives in a global buffer of P.total words per warp
// (`a.grow`) instead of shared memory, for RT windows longer than kSmemMaxCycles.
template <int H, bool GROW>
__global__ void __launch_bounds__(256, 2) search_kernel_sparse(SearchArgs a) {
  extern __shared__ __align__(16) float smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int h = H > 0 ? H : a.h;
  const SparsePlan P = sparse_plan(h, a.ncell);
  float* kw_s = smem_raw;
  float* wb = GROW ? a.grow + ((size_t)blockIdx.x * (blockDim.x >> 5) + warp) * (size_t)P.total
                   : smem_raw + kSparseHeaderWords + warp * P.total;
  float* row = wb + P.row;
  uint32_t* tags = reinterpret_cast<uint32_t*>(wb + P.tags);
  uint32_t* bm = reinterpret_cast<uint32_t*>(wb + P.bm);
  uint32_t* ob = reinterpret_cast<uint32_t*>(wb + P.ob);
  float* conv = wb + P.conv;
  float* scr = wb + P.scr;
  uint16_t* touched = reinterpret_cast<uint16_t*>(wb + P.touched);
  float* score = wb + P.score;
  float* mval = wb + P.mval;
  int* midx = reinterpret_cast<int*>(wb + P.midx);
  // row, bitmaps and convolution row start at zero and are returned to zero by every
  // fragment row
  for (int i = lane; i < a.ncell; i += 32) row[i] = 0.0f;
  for (int i = lane; i < a.ncell + 2 * h; i += 32) conv[i] = 0.0f;
  for (int i = lane; i < P.bw; i += 32) bm[i] = 0u;
  for (int i = lane; i < P.ow; i += 32) ob[i] = 0u;
  for (int i = threadIdx.x; i <= a.h; i += blockDim.x) kw_s[i] = a.kw[i];
  __syncthreads();
  Counters k;

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
    k.frag += F;
    const float wf_lane = lane < F ? __ldg(a.fw + p * a.kf + lane) : 0.0f;
    for (int i = lane; i <= C + C / kSparseS; i += 32) score[i] = 0.0f;
    // output bitmap words that can hold outputs j in [-h, C + h)
    const int w_hi = (C + h - 1 + kBitOff) >> 5;

    PairCursor<true> pc;
    for (int f = 0; f < F; ++f) {
      int n_touched = 0;
      gather_row<kSparseS, true, true>(a, p, f, nwin, npairs, cs, ce, lane, pc, row, 0, bm, tags,
                                       scr, k, touched, n_touched);
      float wf = __shfl_sync(kFull, wf_lane, f & 31);
      if (f >= 32) wf = __ldg(a.fw + p * a.kf + f);
      const bool finite_w = isfinite(wf);
      if (n_touched == 0 && finite_w) continue;  // empty row: every term is +0
      // ---- scatter every touched cell into the convolution row (and clear the XIC
      // row and the touched bitmap behind it)
      if (n_touched <= kTouchCap) {
        for (int i = lane; i < n_touched; i += 32) {
          const int c = touched[i];
          const float x = row[c];
          row[c] = 0.0f;
          bm[(c + kBitOff) >> 5] = 0u;
          scatter_cell<H>(a, kw_s, h, conv, ob, c, x);
        }
      } else {  // more cells than the list holds: walk the bitmap
        const int b_hi = (C - 1 + kBitOff) >> 5;
        for (int w0 = 0; w0 <= b_hi; w0 += 32) {
          const int wi = w0 + lane;
          uint32_t bits = 0u;
          if (wi <= b_hi) {
            bits = bm[wi];
            bm[wi] = 0u;
          }
          unsigned nz = __ballot_sync(kFull, bits != 0u);
          while (nz) {
            const int src = __ffs(nz) - 1;
            nz &= nz - 1;
            const uint32_t wbits = __shfl_sync(kFull, bits, src);
            if ((wbits >> lane) & 1u) {
              const int c = (w0 + src) * 32 + lane - kBitOff;
              const float x = row[c];
              row[c] = 0.0f;
              scatter_cell<H>(a, kw_s, h, conv, ob, c, x);
            }
          }
        }
      }
      __syncwarp();
      if (finite_w) {
        // ---- score terms at the written outputs: a zero output adds ln(1) * w = +0,
        // so the outputs never written need none.  Outputs outside [h, C - h) are only
        // cleared (the reference leaves them 0).
        for (int w0 = 0; w0 <= w_hi; w0 += 32) {
          const int wi = w0 + lane;
          uint32_t bits = 0u;
          if (wi <= w_hi) {
            bits = ob[wi];
            if (bits) ob[wi] = 0u;
          }
          unsigned nz = __ballot_sync(kFull, bits != 0u);
          while (nz) {
            const int src = __ffs(nz) - 1;
            nz &= nz - 1;
            const uint32_t wbits = __shfl_sync(kFull, bits, src);
            if ((wbits >> lane) & 1u) {
              const int j = (w0 + src) * 32 + lane - kBitOff;
              const float c = conv[j + h];
              conv[j + h] = 0.0f;
              if (j >= h && j < C - h) {
                const int at = xaddr<kSparseS>(j);
                score[at] = __fmaf_rn(ln1p_fast(c), wf, score[at]);
              }
            }
          }
        }
      } else {
        // ln(conv + 1) * inf is NaN even where conv is zero: every column takes its
        // term, as in the reference
        for (int j = lane - h; j < C + h; j += 32) {
          const float c = conv[j + h];
          conv[j + h] = 0.0f;
          if (j >= h && j < C - h) {
            const int at = xaddr<kSparseS>(j);
            score[at] = __fmaf_rn(ln1p_fast(c), wf, score[at]);
          }
        }
        for (int i = lane; i <= w_hi; i += 32) ob[i] = 0u;
      }
      __syncwarp();
    }
    __syncwarp();
    pick_top_k<kSparseS>(a, p, cs, C, score, mval, midx, P.mx, lane);
  }
  flush_counters(a, k, lane);
}
