// CPU oracle for the peak-group-selection path — TEST INFRASTRUCTURE ONLY.
//
// A from-scratch C++17 restatement of the reference crate's scalar CPU path
// (MannLabs/alphadia-search-rs).  Loaded only by tests, smoke() and the CPU
// legs of bench.py, as checker or as timed CPU baseline; never by the product.
// Build: see oracle/Makefile (-O2 -ffp-contract=off, no fast-math).
//
// Each function names the reference file:line it follows.  Third-party
// arithmetic that the reference inherits is restated as follows:
//   * Rust 1.88 `slice::binary_search{,_by}` (rust-toolchain.toml pins 1.88.0):
//     branch-free halving that returns the LAST of several equal elements
//     (see rust_bsearch below).  fill_xic_slice depends on this when a bin holds
//     two peaks at the window's first cycle.
//   * ndarray 0.16.1 `Array1::sum` (Cargo.lock): eight-lane unrolled fold
//     (see ndarray_sum below); used once, for the Gaussian kernel normalisation.
//     Parity at this point is unpinned by the reference tests (they check the
//     kernel sum only to 1e-6).
//   * Rust `f32::ln/exp/sqrt` lower to the platform libm: glibc logf/expf/sqrtf.
//   * Rust `slice::sort_by`/`sort_by_key` are stable; `select_nth_unstable_by`
//     is not, so the kept fragment set under intensity ties is implementation
//     defined.  Here ties keep the lower original position (documented rule).

#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------- helpers

// Rust 1.88 core::slice::binary_search_by restated.  `greater(i)` is true when
// element i compares Greater than the target, `equal(i)` when Equal.  Returns
// the Ok or Err index (callers in the reference use unwrap_or_else(|i| i)).
template <class Greater, class Equal, class Less>
int64_t rust_bsearch(int64_t n, Greater greater, Equal equal, Less less) {
  if (n == 0) return 0;
  int64_t size = n, base = 0;
  while (size > 1) {
    int64_t half = size / 2;
    int64_t mid = base + half;
    base = greater(mid) ? base : mid;
    size -= half;
  }
  if (equal(base)) return base;
  return base + (less(base) ? 1 : 0);
}

// ndarray 0.16.1 numeric_util::unrolled_fold with A::add, as used by
// Array1::sum on contiguous data.
float ndarray_sum(const float* xs, int64_t n) {
  float acc = 0.0f;
  float p0 = 0, p1 = 0, p2 = 0, p3 = 0, p4 = 0, p5 = 0, p6 = 0, p7 = 0;
  while (n >= 8) {
    p0 = p0 + xs[0];
    p1 = p1 + xs[1];
    p2 = p2 + xs[2];
    p3 = p3 + xs[3];
    p4 = p4 + xs[4];
    p5 = p5 + xs[5];
    p6 = p6 + xs[6];
    p7 = p7 + xs[7];
    xs += 8;
    n -= 8;
  }
  acc = acc + (p0 + p4);
  acc = acc + (p1 + p5);
  acc = acc + (p2 + p6);
  acc = acc + (p3 + p7);
  for (int64_t i = 0; i < n && i < 7; ++i) acc = acc + xs[i];
  return acc;
}

inline float log_f32(float x, int mode) {
  if (mode == 0) return logf(x);
  return (float)log((double)x);
}

// --------------------------------------------------------------- m/z grid

// src/mz_index/mod.rs:8-25
std::vector<float> ppm_index(float res, float start, float end) {
  float s = fmaxf(start, 50.0f);
  std::vector<float> v;
  v.push_back(s);
  float cur = s;
  while (cur < end) {
    float step = res / 1e6f;
    cur = cur + cur * step;
    v.push_back(cur);
  }
  return v;
}

// src/mz_index/mod.rs:55-90
int64_t find_closest_index(const float* g, int64_t n, float mz) {
  int64_t left = 0, right = n;
  while (left < right) {
    int64_t mid = left + (right - left) / 2;
    if (g[mid] == mz) return mid;
    if (g[mid] < mz)
      left = mid + 1;
    else
      right = mid;
  }
  if (left == 0) return 0;
  if (left == n) return n - 1;
  float left_diff = fabsf(g[left] - mz);
  float right_diff = fabsf(g[left - 1] - mz);
  return left_diff < right_diff ? left : left - 1;
}

// src/mz_index/mod.rs:95-127
void mz_range_indices(const float* g, int64_t n, float lo, float hi, int64_t* s, int64_t* e) {
  int64_t start = 0, right = n;
  while (start < right) {
    int64_t mid = start + (right - start) / 2;
    if (g[mid] < lo)
      start = mid + 1;
    else
      right = mid;
  }
  int64_t end = start;
  if (start < n) {
    int64_t idx = start;
    while (idx < n && g[idx] <= hi) ++idx;
    end = idx;
  }
  *s = start;
  *e = end;
}

// ---------------------------------------------------------------- RT index

// src/rt_index/mod.rs:20-26
float mean_delta_t(const float* rt, int64_t n) {
  if (n > 1) return (rt[n - 1] - rt[0]) / (float)(n - 1);
  return 1.0f;
}

// src/rt_index/mod.rs:89-138
void rt_limits(const float* rt, int64_t n, float dt, float prt, float tol, int64_t pad,
               int64_t* lo, int64_t* hi) {
  if (n == 0) {
    *lo = 0;
    *hi = 0;
    return;
  }
  float min_tol = (10.0f + (float)pad) * dt;
  float eff = fmaxf(tol, min_tol);
  float lower_rt = prt - eff;
  float upper_rt = prt + eff;
  if (upper_rt < rt[0]) {
    *lo = 0;
    *hi = 0;
    return;
  }
  if (lower_rt > rt[n - 1]) {
    *lo = n;
    *hi = n;
    return;
  }
  auto search = [&](float x) {
    return rust_bsearch(
        n, [&](int64_t i) { return rt[i] > x; }, [&](int64_t i) { return rt[i] == x; },
        [&](int64_t i) { return rt[i] < x; });
  };
  *lo = (lower_rt <= rt[0]) ? 0 : search(lower_rt);
  *hi = (upper_rt >= rt[n - 1]) ? n : search(upper_rt);
}

int64_t bsearch_u16(const uint16_t* a, int64_t n, uint16_t x) {
  return rust_bsearch(
      n, [&](int64_t i) { return a[i] > x; }, [&](int64_t i) { return a[i] == x; },
      [&](int64_t i) { return a[i] < x; });
}

// ---------------------------------------------------------- Gaussian kernel

// src/kernel/mod.rs:13-56
std::vector<float> gaussian_kernel(float fwhm, float scale, int64_t width_in, float res) {
  int64_t width = (int64_t)ceilf((float)width_in / 2.0f) * 2;
  float sigma = fwhm / 2.3548f;
  float rt_sigma = sigma * scale / res;
  int32_t half = (int32_t)(width / 2);
  std::vector<float> w((size_t)width, 0.0f);
  const float pi = 3.14159265358979323846f;
  float norm = 1.0f / (rt_sigma * sqrtf(2.0f * pi));
  for (int32_t x = -half; x < half; ++x) {
    float xf = (float)x;
    float exponent = -0.5f * (xf * xf) / (rt_sigma * rt_sigma);
    float weight = norm * expf(exponent);
    w[(size_t)(x + half)] = weight;
  }
  float sum = ndarray_sum(w.data(), width);
  for (auto& v : w) v = v / sum;
  return w;
}

std::vector<double> gaussian_kernel_f64(float fwhm, float scale, int64_t width_in, float res) {
  int64_t width = (int64_t)ceilf((float)width_in / 2.0f) * 2;
  double sigma = (double)fwhm / 2.3548;
  double rt_sigma = sigma * (double)scale / (double)res;
  int32_t half = (int32_t)(width / 2);
  std::vector<double> w((size_t)width, 0.0);
  const double pi = 3.14159265358979323846;
  double norm = 1.0 / (rt_sigma * std::sqrt(2.0 * pi));
  double sum = 0.0;
  for (int32_t x = -half; x < half; ++x) {
    double xd = (double)x;
    w[(size_t)(x + half)] = norm * std::exp(-0.5 * xd * xd / (rt_sigma * rt_sigma));
    sum += w[(size_t)(x + half)];
  }
  for (auto& v : w) v /= sum;
  return w;
}

// ------------------------------------------------------------- convolution

// src/convolution/scalar.rs:5-56
template <class T>
void convolution(const T* k, int64_t klen, const T* xic, int64_t F, int64_t C, T* out) {
  std::fill(out, out + F * C, T(0));
  int64_t half = klen / 2;
  if (F == 0 || C == 0 || C < klen) return;
  int64_t start = half;
  int64_t end = C > half ? C - half : 0;
  for (int64_t f = 0; f < F; ++f) {
    const T* x = xic + f * C;
    T* o = out + f * C;
    if (start < end) {
      for (int64_t i = start; i < end; ++i) {
        T sum = 0;
        sum = sum + x[i] * k[half];
        for (int64_t j = 0; j < half; ++j) {
          T kv = k[j];
          T l = x[i - (half - j)];
          T r = x[i + (half - j)];
          sum = sum + (l + r) * kv;
        }
        o[i] = sum;
      }
    }
  }
}

// src/score/scalar.rs:4-25
void log_dot(const float* a, int64_t F, int64_t C, const float* w, float* out, int mode) {
  std::fill(out, out + C, 0.0f);
  for (int64_t i = 0; i < F; ++i)
    for (int64_t j = 0; j < C; ++j) {
      float val = log_f32(a[i * C + j] + 1.0f, mode);
      out[j] = out[j] + val * w[i];
    }
}

void log_dot_f64(const double* a, int64_t F, int64_t C, const double* w, double* out) {
  std::fill(out, out + C, 0.0);
  for (int64_t i = 0; i < F; ++i)
    for (int64_t j = 0; j < C; ++j) out[j] = out[j] + std::log(a[i * C + j] + 1.0) * w[i];
}

// ------------------------------------------------------------ local maxima

// src/peak_group_selection/mod.rs:23-64 (stable sort, value descending)
template <class T>
void local_maxima(const T* a, int64_t n, int64_t offset, std::vector<int64_t>& idx,
                  std::vector<T>& val) {
  idx.clear();
  val.clear();
  if (n < 5) return;
  for (int64_t i = 2; i < n - 2; ++i) {
    if (a[i - 2] < a[i - 1] && a[i - 1] < a[i] && a[i] > a[i + 1] && a[i + 1] > a[i + 2]) {
      idx.push_back(i + offset);
      val.push_back(a[i]);
    }
  }
  if (!val.empty()) {
    std::vector<size_t> map(val.size());
    std::iota(map.begin(), map.end(), 0);
    std::stable_sort(map.begin(), map.end(), [&](size_t x, size_t y) { return val[x] > val[y]; });
    std::vector<int64_t> si(map.size());
    std::vector<T> sv(map.size());
    for (size_t q = 0; q < map.size(); ++q) {
      si[q] = idx[map[q]];
      sv[q] = val[map[q]];
    }
    idx.swap(si);
    val.swap(sv);
  }
}

// ---------------------------------------------------------- fragment filter

// src/speclib_flat/mod.rs:240-345.  Returns kept original positions in output
// order (ascending fragment m/z, stable).
std::vector<int64_t> filter_sort_fragments(int64_t n, const float* mz, const float* inten,
                                           const uint8_t* number, const uint8_t* type,
                                           bool non_zero, bool filter_y1, int64_t top_k) {
  std::vector<int64_t> keep;
  keep.reserve((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    if (non_zero && !(inten[i] > 0.0f)) continue;
    if (filter_y1 && type[i] == 121 && number[i] == 1) continue;
    keep.push_back(i);
  }
  int64_t k = std::min<int64_t>(top_k, (int64_t)keep.size());
  if (k < (int64_t)keep.size()) {
    // select_nth_unstable_by(k, intensity descending) + truncate(k): keeps the k
    // largest intensities; ties resolved towards the lower original position.
    std::stable_sort(keep.begin(), keep.end(),
                     [&](int64_t a, int64_t b) { return inten[a] > inten[b]; });
    keep.resize((size_t)k);
    std::sort(keep.begin(), keep.end());
  }
  // Rust's sort_by with partial_cmp().unwrap_or(Equal) leaves NaN placement
  // implementation defined; here NaN sorts after every number (stable).
  auto key = [&](int64_t i) { return std::isnan(mz[i]) ? INFINITY : mz[i]; };
  std::stable_sort(keep.begin(), keep.end(), [&](int64_t a, int64_t b) { return key(a) < key(b); });
  return keep;
}

}  // namespace

// ------------------------------------------------------------ DIA structure

struct OrcObs {
  float iso[2] = {0.0f, 0.0f};
  int64_t num_cycles = 0;
  std::vector<uint32_t> slice_starts;
  std::vector<uint16_t> cycles;
  std::vector<float> intensities;
};

struct OrcDia {
  std::vector<float> grid;
  std::vector<float> rt;
  float delta_t = 1.0f;
  std::vector<OrcObs> obs;
};

struct OrcLib {
  std::vector<uint64_t> precursor_idx;
  std::vector<float> precursor_mz, precursor_rt;
  std::vector<uint64_t> frag_start, frag_stop;
  std::vector<float> fragment_mz, fragment_intensity;
  std::vector<uint8_t> fragment_number, fragment_type;
};

struct OrcCand {
  uint64_t precursor_idx, rank;
  float score;
  double score_f64;
  uint64_t center, start, stop;
};

struct OrcResult {
  std::vector<OrcCand> c;
};

namespace {

template <class Fn>
void parallel_for(int64_t n, int n_threads, int64_t chunk, Fn fn) {
  if (n_threads <= 1 || n <= chunk) {
    for (int64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> ts;
  for (int t = 0; t < n_threads; ++t)
    ts.emplace_back([&] {
      for (;;) {
        int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        int64_t e = std::min(n, b + chunk);
        for (int64_t i = b; i < e; ++i) fn(i);
      }
    });
  for (auto& t : ts) t.join();
}

// src/dia_data_builder/mod.rs:52-139
OrcObs build_observation(int64_t n_spec, const int64_t* dsi, const float* lo, const float* hi,
                         const int64_t* ps, const int64_t* pe, const int64_t* cyc,
                         const float* pmz, const float* pint, const std::vector<float>& grid,
                         int64_t target) {
  OrcObs o;
  const int64_t G = (int64_t)grid.size();
  std::vector<int64_t> spectra;
  for (int64_t s = 0; s < n_spec; ++s)
    if (dsi[s] == target) spectra.push_back(s);
  if (spectra.empty()) {
    o.slice_starts.assign((size_t)G + 1, 0u);
    return o;
  }
  o.iso[0] = lo[spectra[0]];
  o.iso[1] = hi[spectra[0]];
  {
    std::vector<int64_t> cs;
    for (auto s : spectra) cs.push_back(cyc[s]);
    std::sort(cs.begin(), cs.end());
    o.num_cycles = std::unique(cs.begin(), cs.end()) - cs.begin();
  }
  struct P {
    uint32_t bin;
    uint16_t cycle;
    float inten;
  };
  std::vector<P> peaks;
  for (auto s : spectra) {
    uint16_t c = (uint16_t)cyc[s];
    for (int64_t k = ps[s]; k < pe[s]; ++k)
      peaks.push_back({(uint32_t)find_closest_index(grid.data(), G, pmz[k]), c, pint[k]});
  }
  std::stable_sort(peaks.begin(), peaks.end(), [](const P& a, const P& b) {
    return a.bin != b.bin ? a.bin < b.bin : a.cycle < b.cycle;
  });
  o.slice_starts.reserve((size_t)G + 1);
  o.slice_starts.push_back(0);
  o.cycles.reserve(peaks.size());
  o.intensities.reserve(peaks.size());
  size_t pi = 0;
  for (int64_t b = 0; b < G; ++b) {
    while (pi < peaks.size() && peaks[pi].bin == (uint32_t)b) {
      o.cycles.push_back(peaks[pi].cycle);
      o.intensities.push_back(peaks[pi].inten);
      ++pi;
    }
    o.slice_starts.push_back((uint32_t)o.cycles.size());
  }
  return o;
}

// src/quadrupole_observation/mod.rs:70-107
template <class T>
void fill_xic_slice(const OrcObs& o, const std::vector<float>& grid, T* xic, int64_t cs,
                    int64_t ce, float tol, float mz) {
  float delta = mz * tol * 1e-6f;
  float lo = mz - delta;
  float hi = mz + delta;
  int64_t b0, b1;
  mz_range_indices(grid.data(), (int64_t)grid.size(), lo, hi, &b0, &b1);
  for (int64_t b = b0; b < b1; ++b) {
    int64_t s = o.slice_starts[(size_t)b];
    int64_t e = o.slice_starts[(size_t)b + 1];
    const uint16_t* cy = o.cycles.data() + s;
    const float* in = o.intensities.data() + s;
    int64_t pos = bsearch_u16(cy, e - s, (uint16_t)cs);
    for (int64_t i = pos; i < e - s; ++i) {
      int64_t c = cy[i];
      if (c >= ce) break;
      xic[c - cs] = xic[c - cs] + (T)in[i];
    }
  }
}

// src/quadrupole_observation/mod.rs:70-107 over raw arrays (same steps as
// fill_xic_slice above; bins past the observation's last slice are not read
// because the reference tests only query ranges inside it).
void fill_xic_slice_raw(const uint32_t* ss, int64_t n_slices, const uint16_t* cyc,
                        const float* inten, const float* grid, int64_t G, float* xic, int64_t cs,
                        int64_t ce, float tol, float mz) {
  float delta = mz * tol * 1e-6f;
  float lo = mz - delta;
  float hi = mz + delta;
  int64_t b0, b1;
  mz_range_indices(grid, G, lo, hi, &b0, &b1);
  for (int64_t b = b0; b < b1 && b < n_slices; ++b) {
    int64_t s = ss[b], e = ss[b + 1];
    int64_t pos = bsearch_u16(cyc + s, e - s, (uint16_t)cs);
    for (int64_t i = pos; i < e - s; ++i) {
      int64_t c = cyc[s + i];
      if (c >= ce) break;
      xic[c - cs] = xic[c - cs] + inten[s + i];
    }
  }
}

// src/dia_data/mod.rs:79-87
void valid_observations(const OrcDia& d, float mz, std::vector<int64_t>& out) {
  out.clear();
  for (size_t i = 0; i < d.obs.size(); ++i)
    if (d.obs[i].iso[0] <= mz && d.obs[i].iso[1] >= mz) out.push_back((int64_t)i);
}

// src/dense_xic_observation/mod.rs:30-64
template <class T>
void dense_xic(const OrcDia& d, float pmz, int64_t cs, int64_t ce, float tol, const float* fmz,
               int64_t F, T* out) {
  int64_t C = ce - cs;
  std::fill(out, out + F * C, T(0));
  std::vector<int64_t> win;
  valid_observations(d, pmz, win);
  for (auto w : win)
    for (int64_t f = 0; f < F; ++f)
      fill_xic_slice<T>(d.obs[(size_t)w], d.grid, out + f * C, cs, ce, tol, fmz[f]);
}

struct Filtered {
  std::vector<float> mz, w;
};

Filtered filtered_precursor(const OrcLib& l, int64_t i, int64_t top_k) {
  // src/speclib_flat/mod.rs:388-456 with non_zero = filter_y1 = true
  // (src/peak_group_selection/mod.rs:104-109)
  Filtered f;
  int64_t s = (int64_t)l.frag_start[(size_t)i], e = (int64_t)l.frag_stop[(size_t)i];
  auto keep = filter_sort_fragments(e - s, l.fragment_mz.data() + s,
                                    l.fragment_intensity.data() + s,
                                    l.fragment_number.data() + s, l.fragment_type.data() + s,
                                    true, true, top_k);
  for (auto k : keep) {
    f.mz.push_back(l.fragment_mz[(size_t)(s + k)]);
    f.w.push_back(l.fragment_intensity[(size_t)(s + k)]);
  }
  return f;
}

// src/peak_group_selection/mod.rs:131-195 (f32) and its f64 twin.
void search_precursor(const OrcDia& d, const OrcLib& l, const OrcParams& p, float rt_tol,
                      int64_t i, int log_mode, int precision, const std::vector<float>& k32,
                      const std::vector<double>& k64, std::vector<OrcCand>& out) {
  Filtered fr = filtered_precursor(l, i, p.top_k_fragments);
  int64_t cs, ce;
  rt_limits(d.rt.data(), (int64_t)d.rt.size(), d.delta_t, l.precursor_rt[(size_t)i], rt_tol,
            p.kernel_size, &cs, &ce);
  if (ce <= cs) return;
  int64_t F = (int64_t)fr.mz.size(), C = ce - cs;
  std::vector<int64_t> mi;
  std::vector<float> mv32;
  std::vector<double> mv64;
  if (precision == 0) {
    std::vector<float> xic((size_t)(F * C)), conv((size_t)(F * C)), score((size_t)C);
    dense_xic<float>(d, l.precursor_mz[(size_t)i], cs, ce, p.mass_tolerance, fr.mz.data(), F,
                     xic.data());
    convolution<float>(k32.data(), (int64_t)k32.size(), xic.data(), F, C, conv.data());
    log_dot(conv.data(), F, C, fr.w.data(), score.data(), log_mode);
    local_maxima<float>(score.data(), C, cs, mi, mv32);
  } else {
    std::vector<double> xic((size_t)(F * C)), conv((size_t)(F * C)), score((size_t)C);
    std::vector<double> w64(fr.w.begin(), fr.w.end());
    dense_xic<double>(d, l.precursor_mz[(size_t)i], cs, ce, p.mass_tolerance, fr.mz.data(), F,
                      xic.data());
    convolution<double>(k64.data(), (int64_t)k64.size(), xic.data(), F, C, conv.data());
    log_dot_f64(conv.data(), F, C, w64.data(), score.data());
    local_maxima<double>(score.data(), C, cs, mi, mv64);
  }
  int64_t nmax = (int64_t)mi.size();
  int64_t cnt = std::min<int64_t>(p.candidate_count, nmax);
  const uint64_t rt_len = (uint64_t)d.rt.size();
  const uint64_t pl = (uint64_t)p.peak_length;
  for (int64_t r = 0; r < cnt; ++r) {
    uint64_t center = (uint64_t)mi[(size_t)r];
    // usize arithmetic of a release build: wrapping subtraction, then max(0, .)
    uint64_t start = center - pl;
    uint64_t stop = std::min<uint64_t>(center + pl + 1, rt_len);
    OrcCand c;
    c.precursor_idx = l.precursor_idx[(size_t)i];
    c.rank = (uint64_t)r;
    if (precision == 0) {
      c.score = mv32[(size_t)r];
      c.score_f64 = (double)mv32[(size_t)r];
    } else {
      c.score = (float)mv64[(size_t)r];
      c.score_f64 = mv64[(size_t)r];
    }
    c.center = center;
    c.start = start;
    c.stop = stop;
    out.push_back(c);
  }
}

}  // namespace

// =================================================================== C API

extern "C" {

int64_t orc_ppm_index_len(float r, float s, float e) { return (int64_t)ppm_index(r, s, e).size(); }

void orc_ppm_index(float r, float s, float e, float* out) {
  auto v = ppm_index(r, s, e);
  std::memcpy(out, v.data(), v.size() * sizeof(float));
}

int64_t orc_find_closest_index(const float* g, int64_t n, float mz) {
  return find_closest_index(g, n, mz);
}

void orc_mz_range_indices(const float* g, int64_t n, float lo, float hi, int64_t* s, int64_t* e) {
  mz_range_indices(g, n, lo, hi, s, e);
}

float orc_mean_delta_t(const float* rt, int64_t n) { return mean_delta_t(rt, n); }

void orc_rt_limits(const float* rt, int64_t n, float dt, float prt, float tol, int64_t pad,
                   int64_t* lo, int64_t* hi) {
  rt_limits(rt, n, dt, prt, tol, pad, lo, hi);
}

int64_t orc_rust_binary_search_u16(const uint16_t* a, int64_t n, uint16_t x) {
  return bsearch_u16(a, n, x);
}

int64_t orc_gaussian_kernel(float fwhm, float scale, int64_t width, float res, float* out) {
  auto w = gaussian_kernel(fwhm, scale, width, res);
  std::memcpy(out, w.data(), w.size() * sizeof(float));
  return (int64_t)w.size();
}

void orc_convolution(const float* k, int64_t klen, const float* xic, int64_t F, int64_t C,
                     float* out) {
  convolution<float>(k, klen, xic, F, C, out);
}

void orc_log_dot(const float* a, int64_t F, int64_t C, const float* w, float* out, int mode) {
  log_dot(a, F, C, w, out, mode);
}

int64_t orc_local_maxima(const float* a, int64_t n, int64_t offset, int64_t* idx, float* val) {
  std::vector<int64_t> i;
  std::vector<float> v;
  local_maxima<float>(a, n, offset, i, v);
  for (size_t q = 0; q < i.size(); ++q) {
    idx[q] = i[q];
    val[q] = v[q];
  }
  return (int64_t)i.size();
}

int64_t orc_filter_sort_fragments(int64_t n, const float* mz, const float* inten,
                                  const uint8_t* number, const uint8_t* type, int non_zero,
                                  int filter_y1, int64_t top_k, int64_t* out) {
  auto k = filter_sort_fragments(n, mz, inten, number, type, non_zero != 0, filter_y1 != 0, top_k);
  for (size_t q = 0; q < k.size(); ++q) out[q] = k[q];
  return (int64_t)k.size();
}

OrcDia* orc_dia_build(int64_t n_spec, const int64_t* dsi, const float* lo, const float* hi,
                      const int64_t* ps, const int64_t* pe, const int64_t* cyc, const float* srt,
                      int64_t /*n_peaks*/, const float* pmz, const float* pint, int n_threads) {
  auto* d = new OrcDia();
  d->grid = ppm_index(1.0f, 150.0f, 2000.0f);  // src/mz_index/mod.rs:4-6,41-45
  for (int64_t s = 0; s < n_spec; ++s)
    if (dsi[s] == 0) d->rt.push_back(srt[s]);  // src/rt_index/mod.rs:62-66
  d->delta_t = mean_delta_t(d->rt.data(), (int64_t)d->rt.size());
  int64_t max_dsi = 0;
  bool any = false;
  for (int64_t s = 0; s < n_spec; ++s)
    if (!any || dsi[s] > max_dsi) {
      max_dsi = dsi[s];
      any = true;
    }
  int64_t n_obs = any && max_dsi >= 0 ? max_dsi + 1 : (any ? 0 : 1);
  d->obs.resize((size_t)n_obs);
  parallel_for(n_obs, n_threads, 1, [&](int64_t w) {
    d->obs[(size_t)w] = build_observation(n_spec, dsi, lo, hi, ps, pe, cyc, pmz, pint, d->grid, w);
  });
  return d;
}

void orc_dia_free(OrcDia* d) { delete d; }
int64_t orc_dia_num_obs(const OrcDia* d) { return (int64_t)d->obs.size(); }
int64_t orc_dia_grid_len(const OrcDia* d) { return (int64_t)d->grid.size(); }
const float* orc_dia_grid(const OrcDia* d) { return d->grid.data(); }
int64_t orc_dia_rt_len(const OrcDia* d) { return (int64_t)d->rt.size(); }
const float* orc_dia_rt(const OrcDia* d) { return d->rt.data(); }
float orc_dia_delta_t(const OrcDia* d) { return d->delta_t; }
void orc_dia_obs_window(const OrcDia* d, int64_t o, float* lo, float* hi) {
  *lo = d->obs[(size_t)o].iso[0];
  *hi = d->obs[(size_t)o].iso[1];
}
int64_t orc_dia_obs_num_cycles(const OrcDia* d, int64_t o) { return d->obs[(size_t)o].num_cycles; }
int64_t orc_dia_obs_num_peaks(const OrcDia* d, int64_t o) {
  return (int64_t)d->obs[(size_t)o].cycles.size();
}
const uint32_t* orc_dia_obs_slice_starts(const OrcDia* d, int64_t o) {
  return d->obs[(size_t)o].slice_starts.data();
}
const uint16_t* orc_dia_obs_cycles(const OrcDia* d, int64_t o) {
  return d->obs[(size_t)o].cycles.data();
}
const float* orc_dia_obs_intensities(const OrcDia* d, int64_t o) {
  return d->obs[(size_t)o].intensities.data();
}

void orc_fill_xic_slice_raw(const uint32_t* ss, int64_t n_slices, const uint16_t* cyc,
                            const float* inten, const float* grid, int64_t G, float* xic,
                            int64_t cs, int64_t ce, float tol, float mz) {
  fill_xic_slice_raw(ss, n_slices, cyc, inten, grid, G, xic, cs, ce, tol, mz);
}

int64_t orc_dia_valid_observations(const OrcDia* d, float mz, int64_t* out, int64_t cap) {
  std::vector<int64_t> v;
  valid_observations(*d, mz, v);
  for (size_t q = 0; q < v.size() && (int64_t)q < cap; ++q) out[q] = v[q];
  return (int64_t)v.size();
}

void orc_dense_xic(const OrcDia* d, float pmz, int64_t cs, int64_t ce, float tol,
                   const float* fmz, int64_t F, float* out) {
  dense_xic<float>(*d, pmz, cs, ce, tol, fmz, F, out);
}

OrcLib* orc_lib_build(int64_t P, const uint64_t* pidx, const float* pmz, const float* prt,
                      const uint64_t* fs, const uint64_t* fe, int64_t NF, const float* fmz,
                      const float* fint, const uint8_t* fnum, const uint8_t* ftype) {
  // src/speclib_flat/mod.rs:139-163: stable sort of the precursor arrays by
  // precursor_idx; fragment arrays keep their order.
  auto* l = new OrcLib();
  std::vector<int64_t> ord((size_t)P);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return pidx[a] < pidx[b]; });
  for (auto i : ord) {
    l->precursor_idx.push_back(pidx[i]);
    l->precursor_mz.push_back(pmz[i]);
    l->precursor_rt.push_back(prt[i]);
    l->frag_start.push_back(fs[i]);
    l->frag_stop.push_back(fe[i]);
  }
  l->fragment_mz.assign(fmz, fmz + NF);
  l->fragment_intensity.assign(fint, fint + NF);
  l->fragment_number.assign(fnum, fnum + NF);
  l->fragment_type.assign(ftype, ftype + NF);
  return l;
}

void orc_lib_free(OrcLib* l) { delete l; }
int64_t orc_lib_num_precursors(const OrcLib* l) { return (int64_t)l->precursor_idx.size(); }

OrcResult* orc_search(const OrcDia* d, const OrcLib* l, const OrcParams* p, const float* rt_tol_pp,
                      const int64_t* subset, int64_t n_subset, int log_mode, int precision,
                      int n_threads) {
  // src/kernel/mod.rs via src/peak_group_selection/mod.rs:75-85
  auto k32 = gaussian_kernel(p->fwhm_rt, 1.0f, p->kernel_size, 1.0f);
  auto k64 = gaussian_kernel_f64(p->fwhm_rt, 1.0f, p->kernel_size, 1.0f);
  int64_t n = subset ? n_subset : (int64_t)l->precursor_idx.size();
  std::vector<std::vector<OrcCand>> per((size_t)n);
  parallel_for(n, n_threads, 64, [&](int64_t q) {
    int64_t i = subset ? subset[q] : q;
    float tol = rt_tol_pp ? rt_tol_pp[i] : p->rt_tolerance;
    search_precursor(*d, *l, *p, tol, i, log_mode, precision, k32, k64, per[(size_t)q]);
  });
  auto* r = new OrcResult();
  for (auto& v : per) r->c.insert(r->c.end(), v.begin(), v.end());
  return r;
}

int64_t orc_result_len(const OrcResult* r) { return (int64_t)r->c.size(); }

void orc_result_copy(const OrcResult* r, uint64_t* pidx, uint64_t* rank, float* score,
                     double* score64, uint64_t* center, uint64_t* start, uint64_t* stop) {
  for (size_t i = 0; i < r->c.size(); ++i) {
    const auto& c = r->c[i];
    if (pidx) pidx[i] = c.precursor_idx;
    if (rank) rank[i] = c.rank;
    if (score) score[i] = c.score;
    if (score64) score64[i] = c.score_f64;
    if (center) center[i] = c.center;
    if (start) start[i] = c.start;
    if (stop) stop[i] = c.stop;
  }
}

void orc_result_free(OrcResult* r) { delete r; }

int64_t orc_trace_precursor(const OrcDia* d, const OrcLib* l, const OrcParams* p, float rt_tol,
                            int64_t i, int log_mode, int64_t* cs_out, int64_t* ce_out,
                            int64_t* nf_out, float* xic, float* conv, float* score, int64_t cap) {
  Filtered fr = filtered_precursor(*l, i, p->top_k_fragments);
  int64_t cs, ce;
  rt_limits(d->rt.data(), (int64_t)d->rt.size(), d->delta_t, l->precursor_rt[(size_t)i], rt_tol,
            p->kernel_size, &cs, &ce);
  *cs_out = cs;
  *ce_out = ce;
  int64_t F = (int64_t)fr.mz.size();
  *nf_out = F;
  if (ce <= cs) return 0;
  int64_t C = ce - cs;
  if (F * C > cap || C > cap) return -1;
  auto k32 = gaussian_kernel(p->fwhm_rt, 1.0f, p->kernel_size, 1.0f);
  dense_xic<float>(*d, l->precursor_mz[(size_t)i], cs, ce, p->mass_tolerance, fr.mz.data(), F, xic);
  convolution<float>(k32.data(), (int64_t)k32.size(), xic, F, C, conv);
  log_dot(conv, F, C, fr.w.data(), score, log_mode);
  return C;
}

double orc_scores_f64_at(const OrcDia* d, const OrcLib* l, const OrcParams* p, float rt_tol,
                         int64_t i, const int64_t* cycles, int64_t n, double* out) {
  Filtered fr = filtered_precursor(*l, i, p->top_k_fragments);
  int64_t cs, ce;
  rt_limits(d->rt.data(), (int64_t)d->rt.size(), d->delta_t, l->precursor_rt[(size_t)i], rt_tol,
            p->kernel_size, &cs, &ce);
  for (int64_t q = 0; q < n; ++q) out[q] = 0.0;
  if (ce <= cs) return 0.0;
  int64_t F = (int64_t)fr.mz.size(), C = ce - cs;
  auto k64 = gaussian_kernel_f64(p->fwhm_rt, 1.0f, p->kernel_size, 1.0f);
  std::vector<double> xic((size_t)(F * C)), conv((size_t)(F * C)), score((size_t)C);
  std::vector<double> w64(fr.w.begin(), fr.w.end());
  dense_xic<double>(*d, l->precursor_mz[(size_t)i], cs, ce, p->mass_tolerance, fr.mz.data(), F,
                    xic.data());
  convolution<double>(k64.data(), (int64_t)k64.size(), xic.data(), F, C, conv.data());
  log_dot_f64(conv.data(), F, C, w64.data(), score.data());
  double mx = 0.0;
  for (auto v : score) mx = std::max(mx, std::fabs(v));
  for (int64_t q = 0; q < n; ++q) {
    int64_t j = cycles[q] - cs;
    out[q] = (j >= 0 && j < C) ? score[(size_t)j] : 0.0;
  }
  return mx;
}

}  // extern "C"
