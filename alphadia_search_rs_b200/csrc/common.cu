// Errors, the global m/z grid and the Gaussian kernel (host side).
#include <cmath>
#include <cstring>
#include <map>

#include "common.cuh"

namespace ads {

thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e),
           what, file, line);
  g_last_error = buf;
  cudaGetLastError();  // a non-sticky error must not resurface in a later, unrelated call
  return e == cudaErrorMemoryAllocation ? ADS_ERR_OUT_OF_MEMORY : ADS_ERR_CUDA;
}

// ------------------------------------------------------------ device memory

namespace {
struct DevicePool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t stream = nullptr;
};
std::mutex g_pool_mu;
std::map<int, DevicePool> g_pools;

int device_pool(int device, DevicePool* out) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(device);
  if (it != g_pools.end()) {
    *out = it->second;
    return ADS_OK;
  }
  DeviceGuard dg(device);
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  DevicePool dp;
  ADS_CUDA(cudaMemPoolCreate(&dp.pool, &props));
  uint64_t keep = kPoolKeepBytes;
  ADS_CUDA(cudaMemPoolSetAttribute(dp.pool, cudaMemPoolAttrReleaseThreshold, &keep));
  ADS_CUDA(cudaStreamCreateWithFlags(&dp.stream, cudaStreamNonBlocking));
  g_pools[device] = dp;
  *out = dp;
  return ADS_OK;
}
// The pool's release threshold counts all memory it holds, in use or not; keeping it
// at (bytes in use + kPoolKeepBytes) keeps up to kPoolKeepBytes of freed memory for
// reuse however much long-lived data (a run, a library) the pool holds.
void update_release_threshold(cudaMemPool_t pool) {
  uint64_t used = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  uint64_t keep = used + kPoolKeepBytes;
  if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
    cudaGetLastError();
}
}  // namespace

int pool_alloc(int device, size_t bytes, void** out) {
  *out = nullptr;
  DevicePool dp;
  ADS_TRY(device_pool(device, &dp));
  cudaError_t e = cudaMallocFromPoolAsync(out, bytes, dp.pool, dp.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(dp.stream);  // usable on every stream
  if (e != cudaSuccess) {
    *out = nullptr;
    return cuda_fail(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
  }
  update_release_threshold(dp.pool);
  return ADS_OK;
}

void pool_free(int device, void* p) {
  DevicePool dp;
  if (device_pool(device, &dp) != ADS_OK) return;
  DeviceGuard dg(device);
  cudaDeviceSynchronize();  // nothing in flight may still read or write p
  cudaFreeAsync(p, dp.stream);
  update_release_threshold(dp.pool);
  cudaStreamSynchronize(dp.stream);
  cudaGetLastError();
}

void pool_free_async(int device, void* p, cudaStream_t st) {
  DevicePool dp;
  if (device_pool(device, &dp) != ADS_OK) return;
  DeviceGuard dg(device);
  cudaFreeAsync(p, st);
  update_release_threshold(dp.pool);
  cudaGetLastError();
}

// ---------------------------------------------------------------- m/z grid

// MZIndex::new / ppm_index (src/mz_index/mod.rs:8-25, 41-45): f32 geometric
// sequence from max(150, 50) while below 2000, each step adding cur * (1/1e6)
// rounded separately (this file is compiled with -ffp-contract=off).
const std::vector<float>& host_grid() {
  static const std::vector<float> grid = [] {
    const float resolution_ppm = 1.0f, mz_start = 150.0f, mz_end = 2000.0f;
    std::vector<float> v;
    v.reserve(2600000);
    float cur = std::fmax(mz_start, 50.0f);
    v.push_back(cur);
    while (cur < mz_end) {
      volatile float step = resolution_ppm / 1e6f;
      volatile float inc = cur * step;
      cur = cur + inc;
      v.push_back(cur);
    }
    return v;
  }();
  return grid;
}

namespace {
struct DeviceGridStore {
  float* grid = nullptr;
  uint32_t* lut = nullptr;
  GridView view;
};
std::mutex g_grid_mu;
std::map<int, DeviceGridStore> g_grids;

uint32_t bits_of(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return u;
}
float float_of(uint32_t u) {
  float x;
  std::memcpy(&x, &u, 4);
  return x;
}
}  // namespace

int device_grid(int device, GridView* out) {
  std::lock_guard<std::mutex> lk(g_grid_mu);
  auto it = g_grids.find(device);
  if (it != g_grids.end()) {
    *out = it->second.view;
    return ADS_OK;
  }
  const auto& g = host_grid();
  const uint32_t n = (uint32_t)g.size();
  const uint32_t b0 = bits_of(g[0]);
  const uint32_t n_lut = ((bits_of(g[n - 1]) - b0) >> kLutShift) + 2;
  std::vector<uint32_t> lut(n_lut);
  size_t pos = 0;
  for (uint32_t k = 0; k < n_lut; ++k) {
    float t = float_of(b0 + (k << kLutShift));
    while (pos < n && g[pos] < t) ++pos;  // lower_bound, monotone in k
    lut[k] = (uint32_t)pos;
  }
  DeviceGuard dg(device);
  DeviceGridStore st;
  ADS_CUDA(cudaMalloc(&st.grid, n * sizeof(float)));
  ADS_CUDA(cudaMalloc(&st.lut, n_lut * sizeof(uint32_t)));
  ADS_CUDA(cudaMemcpy(st.grid, g.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  ADS_CUDA(cudaMemcpy(st.lut, lut.data(), n_lut * sizeof(uint32_t), cudaMemcpyHostToDevice));
  // copies from pageable memory may return before their DMA ends, and the kernels
  // that read the grid run on non-blocking streams
  ADS_CUDA(cudaDeviceSynchronize());
  st.view.grid = st.grid;
  st.view.lut = st.lut;
  st.view.n = n;
  st.view.n_lut = n_lut;
  st.view.bits0 = b0;
  st.view.first = g[0];
  st.view.last = g[n - 1];
  g_grids[device] = st;
  *out = st.view;
  return ADS_OK;
}

namespace {
std::mutex g_ln_mu;
std::map<int, double2*> g_ln_tables;
}  // namespace

std::vector<double2> host_ln_table() {
  std::vector<double2> tab(kLnTableSize);
  for (int j = 0; j < kLnTableSize; ++j) {
    const double c = 1.0 + (double)j / kLnTableSize;
    tab[j].x = 1.0 / c;
    tab[j].y = std::log(c);
  }
  return tab;
}

int device_ln_table(int device, const double2** out) {
  std::lock_guard<std::mutex> lk(g_ln_mu);
  auto it = g_ln_tables.find(device);
  if (it != g_ln_tables.end()) {
    *out = it->second;
    return ADS_OK;
  }
  const std::vector<double2> tab = host_ln_table();
  DeviceGuard dg(device);
  double2* d = nullptr;
  ADS_CUDA(cudaMalloc(&d, kLnTableSize * sizeof(double2)));
  ADS_CUDA(cudaMemcpy(d, tab.data(), kLnTableSize * sizeof(double2), cudaMemcpyHostToDevice));
  ADS_CUDA(cudaDeviceSynchronize());  // as for the grid: the DMA has landed before any use
  g_ln_tables[device] = d;
  *out = d;
  return ADS_OK;
}

// ----------------------------------------------------------- Gaussian kernel

namespace {
// ndarray 0.16.1 `Array1::sum` on contiguous data: an eight-lane unrolled fold,
// the lanes combined pairwise (0,4),(1,5),(2,6),(3,7), then the tail added in
// order.
float ndarray_sum(const float* xs, int64_t n) {
  volatile float p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  while (n >= 8) {
    for (int i = 0; i < 8; ++i) p[i] = p[i] + xs[i];
    xs += 8;
    n -= 8;
  }
  volatile float acc = 0.0f;
  acc = acc + (p[0] + p[4]);
  acc = acc + (p[1] + p[5]);
  acc = acc + (p[2] + p[6]);
  acc = acc + (p[3] + p[7]);
  for (int64_t i = 0; i < n && i < 7; ++i) acc = acc + xs[i];
  return acc;
}
}  // namespace

// GaussianKernel::new / gaussian_kernel_1d (src/kernel/mod.rs:13-56).
std::vector<float> gaussian_kernel(float fwhm_rt, float sigma_scale_rt, int64_t kernel_width,
                                   float rt_resolution) {
  const int64_t width = (int64_t)std::ceil((float)kernel_width / 2.0f) * 2;
  const float sigma = fwhm_rt / 2.3548f;
  const float rt_sigma = sigma * sigma_scale_rt / rt_resolution;
  const int32_t half = (int32_t)(width / 2);
  std::vector<float> w((size_t)width, 0.0f);
  const float pi = 3.14159265358979323846f;
  const float two_pi = 2.0f * pi;
  const float normalization = 1.0f / (rt_sigma * std::sqrt(two_pi));
  for (int32_t x = -half; x < half; ++x) {
    const float xf = (float)x;
    volatile float x2 = xf * xf;
    volatile float s2 = rt_sigma * rt_sigma;
    volatile float num = -0.5f * x2;
    const float exponent = num / s2;
    volatile float e = std::exp(exponent);
    w[(size_t)(x + half)] = normalization * e;
  }
  const float sum = ndarray_sum(w.data(), width);
  for (auto& v : w) v = v / sum;
  return w;
}

}  // namespace ads

extern "C" const char* ads_last_error(void) { return ads::g_last_error.c_str(); }

namespace {
__global__ void selftest_ln_kernel(uint32_t lo, uint32_t hi, const double2* tab,
                                   unsigned long long* out) {
  unsigned long long bad = 0, slow = 0;
  const uint64_t n = (uint64_t)hi - lo;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float x = __uint_as_float(lo + (uint32_t)i);
    bool s = false;
    const float a = ads::ln_fast(x, tab, &s);
    const float b = ads::ln_rn(x);
    bad += __float_as_uint(a) != __float_as_uint(b);
    slow += s;
  }
  atomicAdd(out, bad);
  atomicAdd(out + 1, slow);
}
}  // namespace

extern "C" int ads_selftest_ln(int device, uint32_t lo_bits, uint32_t hi_bits, int64_t* mismatches,
                               int64_t* slow_path) {
  using namespace ads;
  return guarded([&] {
    if (hi_bits < lo_bits) return fail(ADS_ERR_INVALID_ARGUMENT, "hi_bits < lo_bits");
    DeviceGuard dg(device);
    const double2* tab = nullptr;
    ADS_TRY(device_ln_table(device, &tab));
    DevBuf<unsigned long long> out;
    ADS_TRY(out.alloc(2));
    ADS_CUDA(cudaMemset(out.p, 0, 16));
    selftest_ln_kernel<<<148 * 16, 256>>>(lo_bits, hi_bits, tab, out.p);
    ADS_LAUNCH_CHECK();
    unsigned long long h[2];
    ADS_CUDA(cudaMemcpy(h, out.p, 16, cudaMemcpyDeviceToHost));
    if (mismatches) *mismatches = (int64_t)h[0];
    if (slow_path) *slow_path = (int64_t)h[1];
    return ADS_OK;
  });
}
