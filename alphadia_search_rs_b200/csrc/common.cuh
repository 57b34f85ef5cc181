// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "ads_gpu.h"

namespace ads {

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
void clear_error();
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define ADS_TRY(expr)                   \
  do {                                  \
    int _rc = (expr);                   \
    if (_rc != ADS_OK) return _rc;      \
  } while (0)

#define ADS_CUDA(expr)                                                  \
  do {                                                                  \
    cudaError_t _e = (expr);                                            \
    if (_e != cudaSuccess) return ::ads::cuda_fail(_e, #expr, __FILE__, __LINE__); \
  } while (0)

#define ADS_LAUNCH_CHECK() ADS_CUDA(cudaGetLastError())

// Runs `body` and converts C++ exceptions to status codes so nothing crosses
// the C boundary.
template <class F>
int guarded(F&& body) {
  try {
    clear_error();
    return body();
  } catch (const std::bad_alloc&) {
    return fail(ADS_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(ADS_ERR_INTERNAL, e.what());
  } catch (...) {
    return fail(ADS_ERR_INTERNAL, "unknown exception");
  }
}

// Device-current guard: restores the previous device on scope exit.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (dev != prev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// ------------------------------------------------------------ device memory
// Every device buffer of the engine comes from one memory pool per device that
// keeps up to kPoolKeepBytes of freed memory for reuse, so that building a
// library or a candidate collection per call does not map and unmap device pages
// each time.  Allocation and release are ordered on a private stream of the pool;
// a release first waits for the device to go idle (the guarantee cudaFree gives),
// so no kernel still in flight can see its memory handed out again.
constexpr uint64_t kPoolKeepBytes = uint64_t(4) << 30;
int pool_alloc(int device, size_t bytes, void** out);
void pool_free(int device, void* p);
// Frees p once the work enqueued on `st` so far is done (no host synchronisation): for
// memory that only `st` uses.
void pool_free_async(int device, void* p, cudaStream_t st);

// Owning device buffer (move-only) on the current device's pool.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  int dev = -1;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), dev(o.dev) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      dev = o.dev;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) pool_free(dev, p);
    p = nullptr;
    n = 0;
  }
  // release() for a buffer that only `st` has used: ordered after its work on `st`.
  void release_async(cudaStream_t st) {
    if (p) pool_free_async(dev, p, st);
    p = nullptr;
    n = 0;
  }
  // Allocates exactly `count` elements on the current device (frees the previous
  // buffer).
  int alloc(size_t count) {
    release();
    if (count == 0) return ADS_OK;
    int d = 0;
    ADS_CUDA(cudaGetDevice(&d));
    void* q = nullptr;
    ADS_TRY(pool_alloc(d, count * sizeof(T), &q));
    p = static_cast<T*>(q);
    n = count;
    dev = d;
    return ADS_OK;
  }
  // Grows to at least `count` elements, keeping nothing.
  int reserve(size_t count) { return count <= n ? ADS_OK : alloc(count); }
  size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------- m/z grid
// The global 1-ppm grid (src/mz_index/mod.rs:4-25) and a coarse lookup table
// over the grid's float bit patterns that brackets any lower/upper bound to a
// handful of grid points.
constexpr int kLutShift = 6;

struct GridView {
  const float* grid = nullptr;
  const uint32_t* lut = nullptr;
  uint32_t n = 0;       // grid length
  uint32_t n_lut = 0;   // lut length
  uint32_t bits0 = 0;   // bit pattern of grid[0]
  float first = 0.0f;
  float last = 0.0f;
};

const std::vector<float>& host_grid();
int device_grid(int device, GridView* out);

// Gaussian kernel of PeakGroupSelection::new (src/kernel/mod.rs:13-56).
std::vector<float> gaussian_kernel(float fwhm_rt, float sigma_scale_rt, int64_t kernel_width,
                                   float rt_resolution);

__device__ __forceinline__ uint32_t f2bits(float x) { return __float_as_uint(x); }

// First i with grid[i] >= x (lower_bound), exact for every float x, NaN -> 0.
__device__ __forceinline__ uint32_t grid_lower_bound(const GridView& g, float x) {
  if (!(x > g.first)) return 0;
  if (x > g.last) return g.n;
  uint32_t k = (f2bits(x) - g.bits0) >> kLutShift;
  uint32_t lo = __ldg(g.lut + k), hi = __ldg(g.lut + k + 1);
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(g.grid + mid) < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// First i with grid[i] > x (upper_bound), exact, NaN -> 0.
__device__ __forceinline__ uint32_t grid_upper_bound(const GridView& g, float x) {
  if (!(x >= g.first)) return 0;
  if (!(x < g.last)) return g.n;
  uint32_t k = (f2bits(x) - g.bits0) >> kLutShift;
  uint32_t lo = __ldg(g.lut + k), hi = __ldg(g.lut + k + 1);
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(g.grid + mid) <= x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// MZIndex::find_closest_index (src/mz_index/mod.rs:55-90): nearest grid point,
// ties to the lower index, clamped to the ends.
__device__ __forceinline__ uint32_t grid_find_closest(const GridView& g, float mz) {
  uint32_t left = grid_lower_bound(g, mz);
  if (left == 0) return 0;
  if (left == g.n) return g.n - 1;
  float a = __ldg(g.grid + left);
  if (a == mz) return left;
  float ld = fabsf(__fsub_rn(a, mz));
  float rd = fabsf(__fsub_rn(__ldg(g.grid + left - 1), mz));
  return ld < rd ? left : left - 1;
}

// ln(x) of a float rounded to the nearest float: evaluated in double and rounded
// once.  (The reference calls glibc logf, which is not correctly rounded for
// about 1e-3 of its inputs: there the two differ by one ulp.)
__device__ __forceinline__ float ln_rn(float x) { return __double2float_rn(log((double)x)); }

// The same, kept out of line for rarely taken paths (keeps hot loops small).
static __device__ __noinline__ float ln_rn_slow(float x) {
  return __double2float_rn(log((double)x));
}

// Table for ln_fast: for j in [0, 256), c_j = 1 + j/256, {1/c_j, ln(c_j)} in double.
constexpr int kLnTableBits = 8;
constexpr int kLnTableSize = 1 << kLnTableBits;
int device_ln_table(int device, const double2** out);
std::vector<double2> host_ln_table();  // the values device_ln_table uploads

// The same value as ln_rn(x) for every float x, computed faster: x = 2^e * m,
// m = c_j * (1 + r) with 0 <= r < 2^-8, ln(1 + r) by its Taylor series to r^5,
// all in double; e*ln2 + ln(c_j) and r*p(r) are non-negative for x > 1, so the
// result y carries a relative error below 2^-42.  Rounding y to float is then correct unless the 29
// bits of y's significand below float precision lie within 2^14 units of the
// halfway pattern (about one input in 2^14); there ln_rn decides.  Checked against
// ln_rn for every float in (1, inf).  `tab` is the table of device_ln_table
// (usually staged in shared memory).
__device__ __forceinline__ float ln_fast(float x, const double2* tab, bool* slow = nullptr) {
  const uint32_t b = __float_as_uint(x);
  if (b <= 0x3F800000u || b >= 0x7F800000u) {  // x <= 1, negative, inf or NaN
    return b == 0x3F800000u ? 0.0f : ln_rn_slow(x);
  }
  const int e = (int)(b >> 23) - 127;
  const uint32_t j = (b >> (23 - kLnTableBits)) & (kLnTableSize - 1);
  const double m = (double)__uint_as_float((b & 0x007FFFFFu) | 0x3F800000u);
  const double2 t = tab[j];
  const double r = fma(m, t.x, -1.0);
  // 1 - r/2 + r^2/3 - r^3/4 + r^4/5 as (1 - r/2) + r^2 * ((1/3 - r/4) + r^2/5): three
  // dependent steps after r instead of four; e*ln2 + ln(c_j) forms alongside
  const double r2 = r * r;
  const double c0 = fma(r, -1.0 / 2.0, 1.0);
  const double c1 = fma(r, -1.0 / 4.0, 1.0 / 3.0);
  const double p = fma(r2, fma(r2, 1.0 / 5.0, c1), c0);
  const double ln2 = 0.6931471805599453094172321;
  const double y = fma(p, r, fma((double)e, ln2, t.y));
  const uint32_t low = (uint32_t)__double2loint(y) & 0x1FFFFFFFu;
  if (low - (0x10000000u - 0x4000u) < 0x8000u) {
    if (slow) *slow = true;
    return ln_rn_slow(x);
  }
  return __double2float_rn(y);
}

// ------------------------------------------------------------- structures
struct WinInfo {
  float lo, hi;      // isolation window, inclusive at both ends
  int64_t base;      // first entry of this observation in the entry arrays
  int64_t ss_off;    // element offset of its slice_starts, -1 if it holds no peaks
};

}  // namespace ads

struct AdsDia {
  int device = 0;
  int64_t n_obs = 0;
  int64_t grid_len = 0;
  std::vector<ads::WinInfo> win;
  std::vector<int64_t> num_cycles, num_peaks;
  ads::DevBuf<ads::WinInfo> win_dev;
  ads::DevBuf<uint32_t> slice_starts;  // [slots x (grid_len + 1)]
  ads::DevBuf<uint16_t> cycles;
  ads::DevBuf<float> intens;
  ads::DevBuf<uint16_t> intens_bf16;   // built on first BF16 search
  bool bf16_only = false;              // f32 intensities released (ads_dia_keep_bf16_only)
  int64_t n_entries = 0;
  int max_overlap = 0;                 // max number of non-empty windows covering one m/z
  std::vector<float> rt;               // MS1 retention times (RT index)
  float delta_t = 1.0f;
  ads::DevBuf<float> rt_dev;
  std::vector<float> rt_values;        // every spectrum's RT (DIAData.rt_values)
  std::vector<float> cycle;
  int64_t cycle_shape[4] = {0, 0, 0, 0};
  std::mutex mu;
};

struct AdsLib {
  int device = 0;
  int64_t n_prec = 0, n_frag = 0;
  int64_t max_frag = 0;  // max fragments of one precursor
  int64_t min_frag = 0;  // min fragments of one precursor
  ads::DevBuf<char> arena;  // every array below lives in this one allocation
  uint64_t* pidx_p = nullptr;  // precursor arrays, sorted by precursor_idx
  float* pmz_p = nullptr;
  float* prt_p = nullptr;
  float* ptol_p = nullptr;     // optional per-precursor RT half-window
  uint32_t* prow_p = nullptr;  // input row of each sorted precursor
  uint64_t* fstart_p = nullptr;
  uint64_t* fstop_p = nullptr;
  uint8_t* naa_p = nullptr;    // precursor_naa (scoring), sorted like the other precursor arrays
  float* fmz_p = nullptr;      // fragment arrays, input order
  float* fmzl_p = nullptr;     // fragment_mz_library (scoring's IDF)
  float* fint_p = nullptr;
  uint8_t* fnum_p = nullptr;
  uint8_t* ftype_p = nullptr;
  bool has_tol = false;
  float max_tol = 0.0f;
  // recorded after the library's device-side preparation (the precursor sort); every
  // stream that reads the arrays waits on it (lib_ready_on)
  cudaEvent_t ready = nullptr;
  // InverseDocumentFrequency (src/idf/mod.rs:13-33): fragments of the library per
  // m/z grid bin, built on the first scoring call
  std::mutex mu;
  ads::DevBuf<uint32_t> idf_counts;
  float idf_total = -1.0f;  // fragments the histogram counts (< 0: this library's own)
  AdsLib() = default;
  AdsLib(const AdsLib&) = delete;
  AdsLib& operator=(const AdsLib&) = delete;
  ~AdsLib() {
    if (ready) cudaEventDestroy(ready);
  }
};

namespace ads {
// Orders `st` after the library's preparation (from_arrays returns once its uploads
// have landed; the sort behind them may still be queued).
inline int lib_ready_on(const AdsLib* l, cudaStream_t st) {
  if (l->ready) ADS_CUDA(cudaStreamWaitEvent(st, l->ready, 0));
  return ADS_OK;
}
}  // namespace ads

// Candidate columns on the device (CandidateCollection, src/candidate/entry.rs:41-179).
struct AdsCandidates {
  int device = 0;
  cudaEvent_t done = nullptr;
  int64_t cap = -1;
  ads::DevBuf<char> arena;  // all columns and counters in one allocation
  uint64_t* pidx_p = nullptr;
  uint64_t* rank_p = nullptr;
  uint64_t* center_p = nullptr;
  uint64_t* start_p = nullptr;
  uint64_t* stop_p = nullptr;
  float* score_p = nullptr;
  int64_t* count_p = nullptr;
  int* err_p = nullptr;
  int64_t count = 0;
  bool pending = false;
  ~AdsCandidates() {
    if (done) {
      cudaEventSynchronize(done);
      cudaEventDestroy(done);
    }
  }
};

