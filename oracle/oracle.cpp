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
#include <memory>
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
  std::vector<int64_t> order;  // input position of each sorted precursor
  // PeakGroupScoring inputs (orc_lib_set_scoring): naa in sorted order, library m/z
  std::vector<uint8_t> precursor_naa;
  std::vector<float> fragment_mz_library;
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


// ====================================================================
// PeakGroupScoring.score (src/peak_group_scoring/mod.rs:42-340) and the
// functions it calls.  Rust specifics restated:
//   * `Iterator::sum` on f32 (Rust 1.88): a left fold that starts at -0.0
//     (rust_sum); ndarray `sum_axis(Axis(1))` on a C-ordered matrix sums each
//     contiguous row with ndarray's unrolled fold (ndarray_sum);
//   * `sort_by(partial_cmp)` is stable (std::stable_sort); `powi(2)` is x * x;
//   * `f32::ln`/`log10` are glibc logf/log10f (log_mode 0), or ln/log10 rounded
//     once from double (log_mode 1, what the device computes);
//   * u8 `a + 1` wraps (release build).
// A correlation that comes out NaN or infinite makes the reference panic
// (utils.rs:164-166); here it is 0.
namespace {

inline float log10_f32(float x, int mode) {
  if (mode == 0) return log10f(x);
  return (float)log10((double)x);
}

float rust_sum(const float* xs, int64_t n) {
  float s = -0.0f;
  for (int64_t i = 0; i < n; ++i) s = s + xs[i];
  return s;
}

// src/quadrupole_observation/mod.rs:152-211
void fill_xic_and_mz_slice(const OrcObs& o, const std::vector<float>& grid, float* xic, float* mzo,
                           int64_t cs, int64_t ce, float tol, float mz) {
  float delta = mz * tol * 1e-6f;
  float lo = mz - delta;
  float hi = mz + delta;
  int64_t b0, b1;
  mz_range_indices(grid.data(), (int64_t)grid.size(), lo, hi, &b0, &b1);
  for (int64_t b = b0; b < b1; ++b) {
    float actual = grid[(size_t)b];
    int64_t s = o.slice_starts[(size_t)b];
    int64_t e = o.slice_starts[(size_t)b + 1];
    const uint16_t* cy = o.cycles.data() + s;
    const float* in = o.intensities.data() + s;
    int64_t pos = bsearch_u16(cy, e - s, (uint16_t)cs);
    for (int64_t i = pos; i < e - s; ++i) {
      int64_t c = cy[i];
      if (c >= ce) break;
      int64_t r = c - cs;
      float v = in[i];
      xic[r] = xic[r] + v;
      if (v > 0.0f) {
        float prev = xic[r] - v;
        if (prev == 0.0f)
          mzo[r] = actual;
        else
          mzo[r] = (mzo[r] * prev + actual * v) / xic[r];
      }
    }
  }
}

// src/dense_xic_observation/mod.rs:97-137
void dense_xic_mz(const OrcDia& d, float pmz, int64_t cs, int64_t ce, float tol, const float* fmz,
                  int64_t F, float* xic, float* mzo) {
  int64_t C = ce - cs;
  std::fill(xic, xic + F * C, 0.0f);
  std::fill(mzo, mzo + F * C, 0.0f);
  std::vector<int64_t> win;
  valid_observations(d, pmz, win);
  for (auto w : win)
    for (int64_t f = 0; f < F; ++f)
      fill_xic_and_mz_slice(d.obs[(size_t)w], d.grid, xic + f * C, mzo + f * C, cs, ce, tol, fmz[f]);
}

// src/peak_group_scoring/utils.rs:71-109
void normalize_profiles(const float* x, int64_t R, int64_t C, int64_t dil, float* out) {
  int64_t center = C / 2;
  int64_t a = center > dil ? center - dil : 0;
  int64_t b = std::min(center + dil + 1, C);
  for (int64_t i = 0; i < R; ++i) {
    float sum = 0.0f;
    int64_t count = 0;
    for (int64_t j = a; j < b; ++j) {
      sum = sum + x[i * C + j];
      ++count;
    }
    float mean = count > 0 ? sum / (float)count : 0.0f;
    for (int64_t j = 0; j < C; ++j) out[i * C + j] = mean > 0.0f ? x[i * C + j] / mean : 0.0f;
  }
}

// src/peak_group_scoring/utils.rs:7-29 (rows with a non-zero value, in order)
std::vector<int64_t> non_zero_rows(const float* x, int64_t R, int64_t C) {
  std::vector<int64_t> rows;
  for (int64_t i = 0; i < R; ++i)
    for (int64_t j = 0; j < C; ++j)
      if (x[i * C + j] != 0.0f) {
        rows.push_back(i);
        break;
      }
  return rows;
}

bool partial_less(float a, float b) { return a < b; }  // NaN compares Equal

// src/peak_group_scoring/utils.rs:35-66 over the given rows
void median_axis_0(const float* x, const std::vector<int64_t>& rows, int64_t C, float* out) {
  const int64_t R = (int64_t)rows.size();
  std::vector<float> col((size_t)R);
  for (int64_t j = 0; j < C; ++j) {
    if (R == 0) {
      out[j] = 0.0f;
      continue;
    }
    for (int64_t i = 0; i < R; ++i) col[(size_t)i] = x[rows[(size_t)i] * C + j];
    std::stable_sort(col.begin(), col.end(), partial_less);
    out[j] = R % 2 == 0 ? (col[(size_t)(R / 2 - 1)] + col[(size_t)(R / 2)]) / 2.0f : col[(size_t)(R / 2)];
  }
}

// src/peak_group_scoring/utils.rs:126-172
float correlation_safe(const float* x, const float* y, int64_t n) {
  if (n == 0) return 0.0f;
  float xs = rust_sum(x, n), ys = rust_sum(y, n);
  if (xs == 0.0f || ys == 0.0f) return 0.0f;
  float xm = xs / (float)n, ym = ys / (float)n;
  float xv = 0.0f, yv = 0.0f, cv = 0.0f;
  for (int64_t i = 0; i < n; ++i) {
    float dx = x[i] - xm, dy = y[i] - ym;
    xv = xv + dx * dx;
    yv = yv + dy * dy;
    cv = cv + dx * dy;
  }
  if (xv == 0.0f || yv == 0.0f) return 0.0f;
  float c = cv / (sqrtf(xv) * sqrtf(yv));
  if (std::isnan(c) || std::isinf(c)) return 0.0f;
  return std::min(std::max(c, -1.0f), 1.0f);
}

// src/peak_group_scoring/utils.rs:293-312
float gamma_ln(float x, int mode) {
  if (x <= 0.0f) return 0.0f;
  if (fabsf(x - 1.0f) < 1e-6f) return 0.0f;
  if (fabsf(x - 2.0f) < 1e-6f) return 0.0f;
  const float ln_2pi = 1.837877f;
  return (x - 0.5f) * log_f32(x, mode) - x + 0.5f * ln_2pi;
}

// src/peak_group_scoring/utils.rs:193-279 (weights null: 1.0)
float hyperscore_weighted(const uint8_t* type, const float* inten, const bool* mask,
                          const float* w, int64_t n, int mode) {
  uint32_t nb = 0, ny = 0;
  float sb = 0.0f, sy = 0.0f;
  for (int64_t i = 0; i < n; ++i) {
    if (!mask[i] || inten[i] == 0.0f) continue;
    float wi = inten[i] * (w ? w[i] : 1.0f);
    if (type[i] == 98) {
      ++nb;
      sb = sb + wi;
    } else if (type[i] == 121) {
      ++ny;
      sy = sy + wi;
    }
  }
  if (nb == 0 && ny == 0) return 0.0f;
  float fb = nb > 0 ? gamma_ln((float)nb + 1.0f, mode) : 0.0f;
  float fy = ny > 0 ? gamma_ln((float)ny + 1.0f, mode) : 0.0f;
  float lb = sb > 0.0f ? log_f32(sb, mode) : 0.0f;
  float ly = sy > 0.0f ? log_f32(sy, mode) : 0.0f;
  float h = fb + fy + lb + ly;
  return std::isfinite(h) ? h : 0.0f;
}

// src/peak_group_scoring/utils.rs:314-372
void longest_ion_series(const uint8_t* type, const uint8_t* number, const bool* mask, int64_t n,
                        uint8_t* lb, uint8_t* ly) {
  std::vector<uint8_t> b, y;
  for (int64_t i = 0; i < n; ++i) {
    if (!mask[i]) continue;
    if (type[i] == 98) b.push_back(number[i]);
    if (type[i] == 121) y.push_back(number[i]);
  }
  auto longest = [](std::vector<uint8_t> v) -> uint8_t {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    uint8_t mx = 1, cur = 1;
    for (size_t i = 1; i < v.size(); ++i) {
      if (v[i] == (uint8_t)(v[i - 1] + 1)) {
        cur = (uint8_t)(cur + 1);
        mx = std::max(mx, cur);
      } else {
        cur = 1;
      }
    }
    return mx;
  };
  *lb = longest(b);
  *ly = longest(y);
}

// src/peak_group_scoring/utils.rs:402-429
float intensity_ion_series(const uint8_t* type, const float* inten, const bool* mask, int64_t n,
                           uint8_t target) {
  float t = 0.0f;
  for (int64_t i = 0; i < n; ++i)
    if (mask[i] && inten[i] > 0.0f && type[i] == target) t = t + inten[i];
  return t;
}

// src/peak_group_scoring/utils.rs:431-437
float dot_product(const float* a, const float* b, int64_t n) {
  if (n == 0) return 0.0f;
  float s = -0.0f;
  for (int64_t i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

// src/peak_group_scoring/utils.rs:453-476
float fwhm_rt(const float* prof, int64_t C, int64_t cs, const float* rt) {
  if (C == 0) return 0.0f;
  int64_t half = C / 2;
  float center = prof[half];
  for (int64_t i = 0; i < half; ++i) {
    float mean = (prof[half - i] + prof[half + i]) / 2.0f;
    if (mean <= center / 2.0f) return rt[cs + half + i] - rt[cs + half - i];
  }
  return 0.0f;
}

// src/utils/mod.rs:41-75 and :11-39
void fragment_mz_errors(const float* dmz, const float* dxic, int64_t F, int64_t C,
                        const float* mz_lib, float* mz_obs, float* err) {
  for (int64_t f = 0; f < F; ++f) {
    float ws = 0.0f, wsum = 0.0f;
    for (int64_t j = 0; j < C; ++j) {
      float w = dxic[f * C + j];
      if (w > 0.0f) {
        ws = ws + dmz[f * C + j] * w;
        wsum = wsum + w;
      }
    }
    float o = wsum > 0.0f ? ws / wsum : 0.0f;
    mz_obs[f] = o;
    err[f] = o > 0.0f ? ((o - mz_lib[f]) / mz_lib[f]) * 1e6f : 0.0f;
  }
}

// src/utils/mod.rs:83-117
float weighted_mean_abs_error(const float* err, const float* w, int64_t n) {
  if (n == 0) return 0.0f;
  float ws = 0.0f, wsum = 0.0f;
  for (int64_t i = 0; i < n; ++i)
    if (w[i] > 0.0f && err[i] != 0.0f) {
      ws = ws + fabsf(err[i]) * w[i];
      wsum = wsum + w[i];
    }
  return wsum > 0.0f ? ws / wsum : 0.0f;
}

// src/utils/mod.rs:120-143
float median_of(const float* v, int64_t n) {
  if (n == 0) return 0.0f;
  std::vector<float> s(v, v + n);
  std::stable_sort(s.begin(), s.end(), partial_less);
  int64_t mid = n / 2;
  return n % 2 == 0 ? (s[(size_t)(mid - 1)] + s[(size_t)mid]) / 2.0f : s[(size_t)mid];
}

// src/utils/mod.rs:146-173
float std_of(const float* v, int64_t n) {
  if (n < 2) return 0.0f;
  float mean = rust_sum(v, n) / (float)n;
  float acc = -0.0f;
  for (int64_t i = 0; i < n; ++i) acc = acc + (v[i] - mean) * (v[i] - mean);
  return sqrtf(acc / (float)(n - 1));
}

// src/utils/mod.rs:175-221
void ranked_mask(const float* v, int64_t n, int64_t r1, int64_t r2, bool* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = false;
  if (n == 0 || r1 >= r2) return;
  std::vector<int64_t> idx((size_t)n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
    if (v[b] < v[a]) return true;   // value descending
    if (v[a] < v[b]) return false;
    return a < b;                   // then index ascending (NaN compares Equal)
  });
  for (int64_t r = std::min(r1, n); r < std::min(r2, n); ++r) out[idx[(size_t)r]] = true;
}

// src/utils/mod.rs:223-237
int64_t count_above(const float* v, int64_t n, float thr, const bool* mask) {
  int64_t c = 0;
  for (int64_t i = 0; i < n; ++i)
    if ((!mask || mask[i]) && v[i] > thr) ++c;
  return c;
}

constexpr int kNumFeatures = 41;

struct OrcFeatureRow {
  uint64_t precursor_idx, rank;
  float f[kNumFeatures];
};

struct Idf {
  std::vector<uint32_t> counts;
  float total = 0.0f;
};

// src/idf/mod.rs:13-33 over the library's fragment_mz_library
Idf build_idf(const OrcDia& d, const OrcLib& l) {
  Idf idf;
  idf.counts.assign(d.grid.size(), 0u);
  idf.total = (float)l.fragment_mz_library.size();
  for (float mz : l.fragment_mz_library)
    ++idf.counts[(size_t)find_closest_index(d.grid.data(), (int64_t)d.grid.size(), mz)];
  return idf;
}

// src/idf/mod.rs:35-48
float idf_of(const Idf& idf, const OrcDia& d, float mz, int mode) {
  if (idf.total == 0.0f) return 1.0f;
  uint32_t c = idf.counts[(size_t)find_closest_index(d.grid.data(), (int64_t)d.grid.size(), mz)];
  return log_f32(idf.total / (float)std::max(c, 1u), mode);
}

// src/peak_group_scoring/mod.rs:104-340 for one candidate whose precursor sits at
// sorted position i.
void score_candidate(const OrcDia& d, const OrcLib& l, const Idf& idf, float tol, int64_t top_k,
                     int64_t i, uint64_t pidx, uint64_t rank, float cand_score, uint64_t center,
                     uint64_t cstart, uint64_t cstop, int mode, OrcFeatureRow& out) {
  // get_precursor_by_idx_filtered(idx, non_zero = true, y1 = true, top_k)
  const int64_t s = (int64_t)l.frag_start[(size_t)i], e = (int64_t)l.frag_stop[(size_t)i];
  auto keep = filter_sort_fragments(e - s, l.fragment_mz.data() + s, l.fragment_intensity.data() + s,
                                    l.fragment_number.data() + s, l.fragment_type.data() + s,
                                    true, true, top_k);
  const int64_t F = (int64_t)keep.size();
  std::vector<float> fmz, fmzl, fint;
  std::vector<uint8_t> ftype, fnum;
  for (auto k : keep) {
    fmz.push_back(l.fragment_mz[(size_t)(s + k)]);
    fmzl.push_back(l.fragment_mz_library[(size_t)(s + k)]);
    fint.push_back(l.fragment_intensity[(size_t)(s + k)]);
    ftype.push_back(l.fragment_type[(size_t)(s + k)]);
    fnum.push_back(l.fragment_number[(size_t)(s + k)]);
  }
  const int64_t cs = (int64_t)cstart, C = (int64_t)cstop - (int64_t)cstart;
  std::vector<float> xic((size_t)(F * C)), mzo((size_t)(F * C)), norm((size_t)(F * C));
  dense_xic_mz(d, l.precursor_mz[(size_t)i], cs, (int64_t)cstop, tol, fmz.data(), F, xic.data(),
               mzo.data());
  normalize_profiles(xic.data(), F, C, 1, norm.data());
  std::vector<int64_t> all((size_t)F);
  std::iota(all.begin(), all.end(), 0);
  auto nz = non_zero_rows(norm.data(), F, C);
  std::vector<float> med((size_t)C), med_f((size_t)C);
  median_axis_0(norm.data(), all, C, med.data());
  median_axis_0(norm.data(), nz, C, med_f.data());
  const float med_sum = rust_sum(med.data(), C), med_sum_f = rust_sum(med_f.data(), C);
  const float fwhm = fwhm_rt(med_f.data(), C, cs, d.rt.data());
  std::vector<float> corr((size_t)F);
  for (int64_t f = 0; f < F; ++f) corr[(size_t)f] = correlation_safe(med_f.data(), norm.data() + f * C, C);
  std::vector<float> obs((size_t)F);
  for (int64_t f = 0; f < F; ++f) obs[(size_t)f] = ndarray_sum(xic.data() + f * C, C);
  const float int_corr = correlation_safe(obs.data(), fint.data(), F);
  const float mean_corr = F > 0 ? rust_sum(corr.data(), F) / (float)F : 0.0f;
  const float med_corr = median_of(corr.data(), F);
  const float std_corr = std_of(corr.data(), F);
  std::unique_ptr<bool[]> m0(new bool[(size_t)F + 1]), m1(new bool[(size_t)F + 1]),
      m2(new bool[(size_t)F + 1]), m3(new bool[(size_t)F + 1]), matched(new bool[(size_t)F + 1]),
      m6(new bool[(size_t)F + 1]);
  ranked_mask(fint.data(), F, 0, 6, m0.get());
  ranked_mask(fint.data(), F, 6, 12, m1.get());
  ranked_mask(fint.data(), F, 12, 18, m2.get());
  ranked_mask(fint.data(), F, 18, 24, m3.get());
  for (int64_t f = 0; f < F; ++f) matched[(size_t)f] = obs[(size_t)f] > 0.0f;
  std::vector<float> mz_obs((size_t)F), err((size_t)F), inv_w((size_t)F), idf_v((size_t)F);
  fragment_mz_errors(mzo.data(), xic.data(), F, C, fmz.data(), mz_obs.data(), err.data());
  for (int64_t f = 0; f < F; ++f) inv_w[(size_t)f] = 1.0f / (fabsf(err[(size_t)f]) + 0.1f);
  for (int64_t f = 0; f < F; ++f) idf_v[(size_t)f] = idf_of(idf, d, fmzl[(size_t)f], mode);
  ranked_mask(idf_v.data(), F, 0, 6, m6.get());
  const float rt_obs = d.rt[(size_t)center];
  const float ib = intensity_ion_series(ftype.data(), obs.data(), matched.get(), F, 98);
  const float iy = intensity_ion_series(ftype.data(), obs.data(), matched.get(), F, 121);
  const float idf_int_dot = dot_product(idf_v.data(), obs.data(), F);
  uint8_t lb = 0, ly = 0;
  longest_ion_series(ftype.data(), fnum.data(), matched.get(), F, &lb, &ly);
  const float* c = corr.data();
  float* o = out.f;
  out.precursor_idx = pidx;
  out.rank = rank;
  o[0] = cand_score;
  o[1] = mean_corr;
  o[2] = med_corr;
  o[3] = std_corr;
  o[4] = int_corr;
  o[5] = (float)F;
  o[6] = (float)(uint64_t)C;
  o[7] = (float)count_above(c, F, 0.95f, nullptr);
  o[8] = (float)count_above(c, F, 0.90f, nullptr);
  o[9] = (float)count_above(c, F, 0.80f, nullptr);
  o[10] = (float)count_above(c, F, 0.50f, nullptr);
  o[11] = (float)count_above(c, F, 0.0f, nullptr);
  o[12] = (float)count_above(c, F, 0.0f, m0.get());
  o[13] = (float)count_above(c, F, 0.0f, m1.get());
  o[14] = (float)count_above(c, F, 0.0f, m2.get());
  o[15] = (float)count_above(c, F, 0.0f, m3.get());
  o[16] = (float)count_above(c, F, 0.50f, m0.get());
  o[17] = (float)count_above(c, F, 0.50f, m1.get());
  o[18] = (float)count_above(c, F, 0.50f, m2.get());
  o[19] = (float)count_above(c, F, 0.50f, m3.get());
  o[20] = hyperscore_weighted(ftype.data(), obs.data(), matched.get(), nullptr, F, mode);
  o[21] = hyperscore_weighted(ftype.data(), fint.data(), matched.get(), nullptr, F, mode);
  o[22] = hyperscore_weighted(ftype.data(), obs.data(), matched.get(), inv_w.data(), F, mode);
  o[23] = rt_obs;
  o[24] = rt_obs - l.precursor_rt[(size_t)i];
  o[25] = (float)lb;
  o[26] = (float)ly;
  o[27] = (float)l.precursor_naa[(size_t)i];
  o[28] = weighted_mean_abs_error(err.data(), fint.data(), F);
  o[29] = log10_f32(ib + 1e-8f, mode);
  o[30] = log10_f32(iy + 1e-8f, mode);
  o[31] = fwhm;
  o[32] = hyperscore_weighted(ftype.data(), idf_v.data(), matched.get(), nullptr, F, mode);
  o[33] = dot_product(idf_v.data(), c, F);
  o[34] = log10_f32(idf_int_dot + 1e-8f, mode);
  o[35] = med_sum;
  o[36] = med_sum_f;
  o[37] = (float)F;
  o[38] = (float)nz.size();
  o[39] = (float)count_above(c, F, 0.0f, m6.get());
  o[40] = (float)count_above(c, F, 0.50f, m6.get());
}


// ---- PeakGroupQuantification (src/peak_group_quantification/mod.rs:49-168)

struct OrcQuantFrag {
  uint64_t frow;  // input position of the fragment in the library arrays
  float intensity, mz_observed, correlation, mass_error;
};

struct OrcQuantRow {
  bool ok = false;
  uint64_t pidx = 0, prow = 0, rank = 0;
  float rt_observed = 0.0f;
  std::vector<OrcQuantFrag> frags;
};

// quantify_precursor (src/peak_group_quantification/mod.rs:88-167) for one candidate
// whose precursor sits at sorted position i; false when the reference returns None.
bool quantify_candidate(const OrcDia& d, const OrcLib& l, float tol, int64_t top_k, int64_t i,
                        uint64_t pidx, uint64_t rank, uint64_t center, uint64_t cstart,
                        uint64_t cstop, OrcQuantRow& out) {
  if (cstop <= cstart || center < cstart || center >= cstop) return false;
  if (center >= d.rt.size()) return false;  // the reference indexes out of bounds
  const int64_t s = (int64_t)l.frag_start[(size_t)i], e = (int64_t)l.frag_stop[(size_t)i];
  auto keep = filter_sort_fragments(e - s, l.fragment_mz.data() + s, l.fragment_intensity.data() + s,
                                    l.fragment_number.data() + s, l.fragment_type.data() + s,
                                    true, true, top_k);
  const int64_t F = (int64_t)keep.size();
  std::vector<float> fmz;
  for (auto k : keep) fmz.push_back(l.fragment_mz[(size_t)(s + k)]);
  const int64_t C = (int64_t)(cstop - cstart);
  std::vector<float> xic((size_t)(F * C)), mzo((size_t)(F * C)), norm((size_t)(F * C));
  dense_xic_mz(d, l.precursor_mz[(size_t)i], (int64_t)cstart, (int64_t)cstop, tol, fmz.data(), F,
               xic.data(), mzo.data());
  std::vector<float> mz_obs((size_t)F), err((size_t)F);
  fragment_mz_errors(mzo.data(), xic.data(), F, C, fmz.data(), mz_obs.data(), err.data());
  normalize_profiles(xic.data(), F, C, 1, norm.data());
  auto nz = non_zero_rows(norm.data(), F, C);
  std::vector<float> med_f((size_t)C);
  median_axis_0(norm.data(), nz, C, med_f.data());  // filter_non_zero + median_axis_0
  out.ok = false;
  out.frags.clear();
  for (int64_t f = 0; f < F; ++f) {
    const float corr = correlation_safe(norm.data() + f * C, med_f.data(), C);
    const float obs = ndarray_sum(xic.data() + f * C, C);
    if (obs > 0.0f)  // PrecursorQuantified::filter_fragments_by_intensity(0.0)
      out.frags.push_back({(uint64_t)(s + keep[(size_t)f]), obs, mz_obs[(size_t)f], corr,
                           err[(size_t)f]});
  }
  if (out.frags.empty()) return false;
  out.ok = true;
  out.pidx = pidx;
  out.prow = (uint64_t)l.order[(size_t)i];
  out.rank = rank;
  out.rt_observed = d.rt[(size_t)center];
  return true;
}

}  // namespace

struct OrcFeatures {
  std::vector<OrcFeatureRow> rows;
};

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
  l->order = ord;
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


// ---- PeakGroupScoring (src/peak_group_scoring/mod.rs:42-340)

void orc_lib_set_scoring(OrcLib* l, const uint8_t* naa, int64_t n_frag, const float* fmz_library) {
  // SpecLibFlat::from_arrays (src/speclib_flat/mod.rs:100-188): precursor_naa follows the
  // stable precursor sort, fragment_mz_library keeps the input order
  l->precursor_naa.clear();
  for (auto i : l->order) l->precursor_naa.push_back(naa ? naa[i] : 0);
  l->fragment_mz_library.assign(fmz_library, fmz_library + n_frag);
}

OrcFeatures* orc_score(const OrcDia* d, const OrcLib* l, float mass_tolerance, int64_t top_k,
                       const uint64_t* pidx, const uint64_t* rank, const float* score,
                       const uint64_t* center, const uint64_t* start, const uint64_t* stop,
                       int64_t n, int log_mode, int n_threads) {
  Idf idf = build_idf(*d, *l);
  std::vector<OrcFeatureRow> rows((size_t)n);
  std::vector<char> found((size_t)n, 0);
  const int64_t P = (int64_t)l->precursor_idx.size();
  const uint64_t* keys = l->precursor_idx.data();
  parallel_for(n, n_threads, 64, [&](int64_t q) {
    // SpecLibFlat::get_precursor_by_idx_filtered: binary_search on the sorted idx
    const uint64_t x = pidx[q];
    int64_t i = rust_bsearch(
        P, [&](int64_t m) { return keys[m] > x; }, [&](int64_t m) { return keys[m] == x; },
        [&](int64_t m) { return keys[m] < x; });
    if (i >= P || keys[i] != x) return;  // skipped with a warning in the reference
    score_candidate(*d, *l, idf, mass_tolerance, top_k, i, x, rank[q], score[q], center[q],
                    start[q], stop[q], log_mode, rows[(size_t)q]);
    found[(size_t)q] = 1;
  });
  auto* r = new OrcFeatures();
  for (int64_t q = 0; q < n; ++q)
    if (found[(size_t)q]) r->rows.push_back(rows[(size_t)q]);
  return r;
}

int64_t orc_features_len(const OrcFeatures* r) { return (int64_t)r->rows.size(); }

void orc_features_copy(const OrcFeatures* r, uint64_t* pidx, uint64_t* rank, float* feats) {
  for (size_t q = 0; q < r->rows.size(); ++q) {
    pidx[q] = r->rows[q].precursor_idx;
    rank[q] = r->rows[q].rank;
    for (int k = 0; k < kNumFeatures; ++k) feats[q * kNumFeatures + k] = r->rows[q].f[k];
  }
}

void orc_features_free(OrcFeatures* r) { delete r; }

// SpecLibFlatQuantified::from_precursor_quantified_vec (src/speclib_flat_quantified/mod.rs:
// 212-333): fragments in candidate order, precursors stably sorted by precursor_idx with
// their fragment ranges.
struct OrcQuant {
  std::vector<uint64_t> p_idx, p_row, p_rank, p_start, p_stop;
  std::vector<float> p_rt_observed;
  std::vector<uint64_t> f_row, f_pidx, f_rank;
  std::vector<float> f_intensity, f_mz_observed, f_correlation, f_mass_error;
};

OrcQuant* orc_quantify(const OrcDia* d, const OrcLib* l, float tolerance_ppm, int64_t top_k,
                       const uint64_t* pidx, const uint64_t* rank, const uint64_t* center,
                       const uint64_t* start, const uint64_t* stop, int64_t n, int n_threads) {
  std::vector<OrcQuantRow> rows((size_t)n);
  const int64_t P = (int64_t)l->precursor_idx.size();
  const uint64_t* keys = l->precursor_idx.data();
  parallel_for(n, n_threads, 64, [&](int64_t q) {
    const uint64_t x = pidx[q];
    int64_t i = rust_bsearch(
        P, [&](int64_t m) { return keys[m] > x; }, [&](int64_t m) { return keys[m] == x; },
        [&](int64_t m) { return keys[m] < x; });
    if (i >= P || keys[i] != x) return;  // get_precursor_by_idx_filtered: None
    quantify_candidate(*d, *l, tolerance_ppm, top_k, i, x, rank[q], center[q], start[q], stop[q],
                       rows[(size_t)q]);
  });
  auto* r = new OrcQuant();
  std::vector<size_t> kept;
  uint64_t at = 0;
  std::vector<uint64_t> fs, fe;
  for (size_t q = 0; q < rows.size(); ++q) {
    const auto& w = rows[q];
    if (!w.ok) continue;
    kept.push_back(q);
    fs.push_back(at);
    for (const auto& f : w.frags) {
      r->f_row.push_back(f.frow);
      r->f_intensity.push_back(f.intensity);
      r->f_mz_observed.push_back(f.mz_observed);
      r->f_correlation.push_back(f.correlation);
      r->f_mass_error.push_back(f.mass_error);
      r->f_pidx.push_back(w.pidx);
      r->f_rank.push_back(w.rank);
    }
    at += w.frags.size();
    fe.push_back(at);
  }
  std::vector<size_t> ord(kept.size());
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](size_t a, size_t b) { return rows[kept[a]].pidx < rows[kept[b]].pidx; });
  for (size_t k : ord) {
    const auto& w = rows[kept[k]];
    r->p_idx.push_back(w.pidx);
    r->p_row.push_back(w.prow);
    r->p_rank.push_back(w.rank);
    r->p_rt_observed.push_back(w.rt_observed);
    r->p_start.push_back(fs[k]);
    r->p_stop.push_back(fe[k]);
  }
  return r;
}

void orc_quant_sizes(const OrcQuant* r, int64_t* n_prec, int64_t* n_frag) {
  *n_prec = (int64_t)r->p_idx.size();
  *n_frag = (int64_t)r->f_row.size();
}

void orc_quant_copy(const OrcQuant* r, uint64_t* p_idx, uint64_t* p_row, uint64_t* p_rank,
                    float* p_rt_observed, uint64_t* p_start, uint64_t* p_stop, uint64_t* f_row,
                    float* f_intensity, float* f_mz_observed, float* f_correlation,
                    float* f_mass_error, uint64_t* f_pidx, uint64_t* f_rank) {
  auto cp = [](const auto& v, auto* dst) { std::copy(v.begin(), v.end(), dst); };
  cp(r->p_idx, p_idx);
  cp(r->p_row, p_row);
  cp(r->p_rank, p_rank);
  cp(r->p_rt_observed, p_rt_observed);
  cp(r->p_start, p_start);
  cp(r->p_stop, p_stop);
  cp(r->f_row, f_row);
  cp(r->f_intensity, f_intensity);
  cp(r->f_mz_observed, f_mz_observed);
  cp(r->f_correlation, f_correlation);
  cp(r->f_mass_error, f_mass_error);
  cp(r->f_pidx, f_pidx);
  cp(r->f_rank, f_rank);
}

void orc_quant_free(OrcQuant* r) { delete r; }

// ---- the scoring helpers on raw arrays (for the reference's unit-test values)

void orc_sc_normalize_profiles(const float* x, int64_t R, int64_t C, int64_t dil, float* out) {
  normalize_profiles(x, R, C, dil, out);
}
void orc_sc_median_axis0(const float* x, int64_t R, int64_t C, int non_zero_only, float* out) {
  std::vector<int64_t> rows;
  if (non_zero_only) {
    rows = non_zero_rows(x, R, C);
  } else {
    rows.resize((size_t)R);
    std::iota(rows.begin(), rows.end(), 0);
  }
  median_axis_0(x, rows, C, out);
}
float orc_sc_correlation(const float* x, const float* y, int64_t n) { return correlation_safe(x, y, n); }
float orc_sc_gamma_ln(float x, int mode) { return gamma_ln(x, mode); }
float orc_sc_hyperscore(const uint8_t* type, const float* inten, const uint8_t* mask,
                        const float* w, int64_t n, int mode) {
  std::unique_ptr<bool[]> m(new bool[(size_t)n + 1]);
  for (int64_t i = 0; i < n; ++i) m[(size_t)i] = mask[i] != 0;
  return hyperscore_weighted(type, inten, m.get(), w, n, mode);
}
void orc_sc_longest_ion_series(const uint8_t* type, const uint8_t* number, const uint8_t* mask,
                               int64_t n, uint8_t* lb, uint8_t* ly) {
  std::unique_ptr<bool[]> m(new bool[(size_t)n + 1]);
  for (int64_t i = 0; i < n; ++i) m[(size_t)i] = mask[i] != 0;
  longest_ion_series(type, number, m.get(), n, lb, ly);
}
float orc_sc_intensity_ion_series(const uint8_t* type, const float* inten, const uint8_t* mask,
                                  int64_t n, uint8_t target) {
  std::unique_ptr<bool[]> m(new bool[(size_t)n + 1]);
  for (int64_t i = 0; i < n; ++i) m[(size_t)i] = mask[i] != 0;
  return intensity_ion_series(type, inten, m.get(), n, target);
}
float orc_sc_fwhm_rt(const float* prof, int64_t C, int64_t cs, const float* rt) {
  return fwhm_rt(prof, C, cs, rt);
}
void orc_sc_fragment_mz_errors(const float* dmz, const float* dxic, int64_t F, int64_t C,
                               const float* mz_lib, float* mz_obs, float* err) {
  fragment_mz_errors(dmz, dxic, F, C, mz_lib, mz_obs, err);
}
float orc_sc_weighted_mae(const float* err, const float* w, int64_t n) {
  return weighted_mean_abs_error(err, w, n);
}
float orc_sc_median(const float* v, int64_t n) { return median_of(v, n); }
float orc_sc_std(const float* v, int64_t n) { return std_of(v, n); }
void orc_sc_ranked_mask(const float* v, int64_t n, int64_t r1, int64_t r2, uint8_t* out) {
  std::unique_ptr<bool[]> m(new bool[(size_t)n + 1]);
  ranked_mask(v, n, r1, r2, m.get());
  for (int64_t i = 0; i < n; ++i) out[i] = m[(size_t)i] ? 1 : 0;
}
int64_t orc_sc_count_above(const float* v, int64_t n, float thr, const uint8_t* mask) {
  if (!mask) return count_above(v, n, thr, nullptr);
  std::unique_ptr<bool[]> m(new bool[(size_t)n + 1]);
  for (int64_t i = 0; i < n; ++i) m[(size_t)i] = mask[i] != 0;
  return count_above(v, n, thr, m.get());
}
float orc_sc_dot(const float* a, const float* b, int64_t n) { return dot_product(a, b, n); }
void orc_sc_dense_xic_mz(const OrcDia* d, float pmz, int64_t cs, int64_t ce, float tol,
                         const float* fmz, int64_t F, float* xic, float* mzo) {
  dense_xic_mz(*d, pmz, cs, ce, tol, fmz, F, xic, mzo);
}
void orc_sc_idf(const OrcDia* d, const OrcLib* l, const float* mz, int64_t n, int mode, float* out) {
  Idf idf = build_idf(*d, *l);
  for (int64_t i = 0; i < n; ++i) out[i] = idf_of(idf, *d, mz[i], mode);
}

}  // extern "C"
