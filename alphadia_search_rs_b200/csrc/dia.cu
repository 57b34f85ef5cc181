// DIAData construction on the device (DIADataBuilder::from_alpha_raw,
// src/dia_data_builder/mod.rs:11-139) and the DIAData getters.
//
// Layout in HBM, per quadrupole observation w (= delta_scan_idx):
//   slice_starts[slot(w)][b]  u32, b in [0, grid_len], CSR offsets by m/z bin
//   cycles[base(w) + i]       u16 cycle index of entry i
//   intens[base(w) + i]       f32 intensity of entry i
// Entries are ordered by (bin, cycle), ties in the order the reference visits
// peaks (spectrum index, then peak index), exactly like its stable sort_by_key.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace ads {
namespace {

constexpr int kBinShift = 16;
constexpr int kWinShift = 38;  // 22 bits of m/z bin above 16 bits of cycle

// One block per spectrum: every peak gets its (window, bin, cycle) key and its
// peak index as value, written at the spectrum's slot in the reference's visit
// order.
template <class V>
__global__ void bin_peaks_kernel(int64_t n_spec, const int64_t* __restrict__ item_off,
                                 const int64_t* __restrict__ pstart,
                                 const int64_t* __restrict__ pstop, const int32_t* __restrict__ win,
                                 const uint16_t* __restrict__ cyc, const float* __restrict__ mz,
                                 GridView g, uint64_t* __restrict__ keys, V* __restrict__ vals) {
  for (int64_t s = blockIdx.x; s < n_spec; s += gridDim.x) {
    const int32_t w = win[s];
    if (w < 0) continue;
    const int64_t off = item_off[s], b = pstart[s], e = pstop[s];
    const uint64_t hi = ((uint64_t)w << kWinShift) | (uint64_t)cyc[s];
    for (int64_t k = threadIdx.x; k < e - b; k += blockDim.x) {
      const int64_t i = b + k;
      const uint32_t bin = grid_find_closest(g, __ldg(mz + i));
      keys[off + k] = hi | ((uint64_t)bin << kBinShift);
      vals[off + k] = (V)i;
    }
  }
}

// counts[slot(w)][bin] += 1 for every sorted entry; cycles/intensities gathered.
template <class V>
__global__ void scatter_entries_kernel(int64_t n, const uint64_t* __restrict__ keys,
                                       const V* __restrict__ vals,
                                       const float* __restrict__ pint,
                                       const int64_t* __restrict__ slot_of_win, int64_t stride,
                                       uint32_t* __restrict__ counts, uint16_t* __restrict__ cycles,
                                       float* __restrict__ intens) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const int64_t w = (int64_t)(k >> kWinShift);
    const uint32_t bin = (uint32_t)((k >> kBinShift) & ((1u << 22) - 1));
    cycles[i] = (uint16_t)(k & 0xFFFFu);
    intens[i] = __ldg(pint + vals[i]);
    atomicAdd(counts + slot_of_win[w] * stride + bin, 1u);
  }
}

struct SegmentOf {
  int64_t stride;
  __host__ __device__ int64_t operator()(int64_t i) const { return i / stride; }
};

struct SpectrumTable {
  std::vector<int64_t> dsi, start, stop, cyc;
  std::vector<float> lo, hi, rt;
};

template <class T>
int fetch(const T* src, int64_t n, int loc, std::vector<T>& dst) {
  dst.resize((size_t)n);
  if (n == 0) return ADS_OK;
  if (!src) return fail(ADS_ERR_INVALID_ARGUMENT, "null array pointer");
  if (loc == ADS_MEM_DEVICE) {
    ADS_CUDA(cudaMemcpy(dst.data(), src, (size_t)n * sizeof(T), cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(dst.data(), src, (size_t)n * sizeof(T));
  }
  return ADS_OK;
}

template <class V>
int build_entries(AdsDia* d, const AdsRawArrays* raw, const std::vector<int32_t>& win_of_spec,
                  const std::vector<uint16_t>& cyc16, const std::vector<int64_t>& item_off,
                  int64_t n_items, const std::vector<int64_t>& slot_of_win, int64_t n_slots,
                  const GridView& g, cudaStream_t st) {
  const int64_t n_spec = raw->n_spectra;
  const int64_t stride = d->grid_len + 1;
  // device copies of the spectrum table and, if needed, the peak arrays
  DevBuf<int64_t> d_off, d_start, d_stop, d_slot;
  DevBuf<int32_t> d_win;
  DevBuf<uint16_t> d_cyc;
  DevBuf<float> d_mz, d_int;
  const float* mz = raw->peak_mz;
  const float* pint = raw->peak_intensity;
  ADS_TRY(d_off.alloc(n_spec));
  ADS_TRY(d_win.alloc(n_spec));
  ADS_TRY(d_cyc.alloc(n_spec));
  ADS_TRY(d_slot.alloc(slot_of_win.size()));
  ADS_CUDA(cudaMemcpyAsync(d_off.p, item_off.data(), n_spec * 8, cudaMemcpyHostToDevice, st));
  ADS_CUDA(cudaMemcpyAsync(d_win.p, win_of_spec.data(), n_spec * 4, cudaMemcpyHostToDevice, st));
  ADS_CUDA(cudaMemcpyAsync(d_cyc.p, cyc16.data(), n_spec * 2, cudaMemcpyHostToDevice, st));
  ADS_CUDA(cudaMemcpyAsync(d_slot.p, slot_of_win.data(), slot_of_win.size() * 8,
                           cudaMemcpyHostToDevice, st));
  if (raw->location == ADS_MEM_DEVICE) {
    ADS_TRY(d_start.alloc(n_spec));
    ADS_TRY(d_stop.alloc(n_spec));
    ADS_CUDA(cudaMemcpyAsync(d_start.p, raw->spectrum_peak_start_idx, n_spec * 8,
                             cudaMemcpyDeviceToDevice, st));
    ADS_CUDA(cudaMemcpyAsync(d_stop.p, raw->spectrum_peak_stop_idx, n_spec * 8,
                             cudaMemcpyDeviceToDevice, st));
  } else {
    ADS_TRY(d_start.alloc(n_spec));
    ADS_TRY(d_stop.alloc(n_spec));
    ADS_CUDA(cudaMemcpyAsync(d_start.p, raw->spectrum_peak_start_idx, n_spec * 8,
                             cudaMemcpyHostToDevice, st));
    ADS_CUDA(cudaMemcpyAsync(d_stop.p, raw->spectrum_peak_stop_idx, n_spec * 8,
                             cudaMemcpyHostToDevice, st));
    ADS_TRY(d_mz.alloc(raw->n_peaks));
    ADS_TRY(d_int.alloc(raw->n_peaks));
    if (raw->n_peaks) {
      ADS_CUDA(cudaMemcpyAsync(d_mz.p, raw->peak_mz, raw->n_peaks * 4, cudaMemcpyHostToDevice, st));
      ADS_CUDA(cudaMemcpyAsync(d_int.p, raw->peak_intensity, raw->n_peaks * 4,
                               cudaMemcpyHostToDevice, st));
    }
    mz = d_mz.p;
    pint = d_int.p;
  }

  DevBuf<uint64_t> keys_a, keys_b;
  DevBuf<V> vals_a, vals_b;
  ADS_TRY(keys_a.alloc(n_items));
  ADS_TRY(keys_b.alloc(n_items));
  ADS_TRY(vals_a.alloc(n_items));
  ADS_TRY(vals_b.alloc(n_items));
  if (n_spec > 0 && n_items > 0) {
    const int grid = (int)std::min<int64_t>(n_spec, 1 << 20);
    bin_peaks_kernel<V><<<grid, 128, 0, st>>>(n_spec, d_off.p, d_start.p, d_stop.p, d_win.p,
                                               d_cyc.p, mz, g, keys_a.p, vals_a.p);
    ADS_LAUNCH_CHECK();
  }
  // stable LSD radix sort on (window, bin, cycle): equal keys keep visit order
  int n_win_bits = 1;
  while ((int64_t(1) << n_win_bits) < (int64_t)slot_of_win.size()) ++n_win_bits;
  const int end_bit = kWinShift + n_win_bits;
  size_t tmp_bytes = 0;
  ADS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys_a.p, keys_b.p, vals_a.p,
                                           vals_b.p, n_items, kBinShift - 16, end_bit, st));
  DevBuf<unsigned char> tmp;
  ADS_TRY(tmp.alloc(tmp_bytes + 16));
  if (n_items > 0)
    ADS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys_a.p, keys_b.p, vals_a.p,
                                             vals_b.p, n_items, 0, end_bit, st));
  keys_a.release();
  vals_a.release();
  tmp.release();

  ADS_TRY(d->cycles.alloc(n_items));
  ADS_TRY(d->intens.alloc(n_items));
  DevBuf<uint32_t> counts;
  ADS_TRY(counts.alloc((size_t)(n_slots * stride)));
  ADS_TRY(d->slice_starts.alloc((size_t)(n_slots * stride)));
  if (n_slots > 0) {
    ADS_CUDA(cudaMemsetAsync(counts.p, 0, counts.bytes(), st));
    if (n_items > 0) {
      scatter_entries_kernel<V><<<4 * 148 * 8, 256, 0, st>>>(n_items, keys_b.p, vals_b.p, pint,
                                                             d_slot.p, stride, counts.p,
                                                             d->cycles.p, d->intens.p);
      ADS_LAUNCH_CHECK();
    }
    // per-observation exclusive scan of the bin counts -> slice_starts
    cub::CountingInputIterator<int64_t> idx(0);
    cub::TransformInputIterator<int64_t, SegmentOf, cub::CountingInputIterator<int64_t>> seg(
        idx, SegmentOf{stride});
    size_t sb = 0;
    const int64_t total = n_slots * stride;
    ADS_CUDA(cub::DeviceScan::ExclusiveSumByKey(nullptr, sb, seg, counts.p, d->slice_starts.p,
                                                total, ::cuda::std::equal_to<>(), st));
    DevBuf<unsigned char> stmp;
    ADS_TRY(stmp.alloc(sb + 16));
    ADS_CUDA(cub::DeviceScan::ExclusiveSumByKey(stmp.p, sb, seg, counts.p, d->slice_starts.p,
                                                total, ::cuda::std::equal_to<>(), st));
    ADS_CUDA(cudaStreamSynchronize(st));
  }
  ADS_CUDA(cudaStreamSynchronize(st));
  return ADS_OK;
}

int dia_create(const AdsRawArrays* raw, int device, AdsDia** out) {
  if (!raw || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (raw->location != ADS_MEM_HOST && raw->location != ADS_MEM_DEVICE)
    return fail(ADS_ERR_INVALID_ARGUMENT, "location must be ADS_MEM_HOST or ADS_MEM_DEVICE");
  const int64_t n_spec = raw->n_spectra, n_peaks = raw->n_peaks;
  if (n_spec <= 0)
    return fail(ADS_ERR_INVALID_ARGUMENT, "DIAData needs at least one spectrum");
  if (n_peaks < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "n_peaks < 0");
  if (n_peaks > 0 && (!raw->peak_mz || !raw->peak_intensity))
    return fail(ADS_ERR_INVALID_ARGUMENT, "null peak array");
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
    cudaGetLastError();
    return fail(ADS_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= n_dev) return fail(ADS_ERR_INVALID_ARGUMENT, "bad device index");
  DeviceGuard dg(device);

  SpectrumTable t;
  const int L = raw->location;
  ADS_TRY(fetch(raw->spectrum_delta_scan_idx, n_spec, L, t.dsi));
  ADS_TRY(fetch(raw->spectrum_peak_start_idx, n_spec, L, t.start));
  ADS_TRY(fetch(raw->spectrum_peak_stop_idx, n_spec, L, t.stop));
  ADS_TRY(fetch(raw->spectrum_cycle_idx, n_spec, L, t.cyc));
  ADS_TRY(fetch(raw->isolation_lower_mz, n_spec, L, t.lo));
  ADS_TRY(fetch(raw->isolation_upper_mz, n_spec, L, t.hi));
  ADS_TRY(fetch(raw->spectrum_rt, n_spec, L, t.rt));

  // validation the reference leaves to panics or silent truncation
  int64_t max_dsi = t.dsi[0];
  for (int64_t s = 0; s < n_spec; ++s) {
    if (t.start[s] < 0 || t.stop[s] < t.start[s] || t.stop[s] > n_peaks)
      return fail(ADS_ERR_INVALID_ARGUMENT,
                  "spectrum " + std::to_string(s) + ": peak range outside [0, n_peaks] or start > stop");
    if (t.cyc[s] < 0 || t.cyc[s] > 65535)
      return fail(ADS_ERR_INVALID_ARGUMENT,
                  "spectrum " + std::to_string(s) + ": cycle index outside [0, 65535]");
    max_dsi = std::max(max_dsi, t.dsi[s]);
  }
  if (max_dsi > (int64_t(1) << 20))
    return fail(ADS_ERR_INVALID_ARGUMENT, "delta_scan_idx above 2^20");
  const int64_t n_obs = max_dsi >= 0 ? max_dsi + 1 : 0;

  auto d = new AdsDia();
  std::unique_ptr<AdsDia> guard(d);
  d->device = device;
  d->n_obs = n_obs;
  d->grid_len = (int64_t)host_grid().size();
  d->win.assign((size_t)n_obs, WinInfo{0.0f, 0.0f, 0, -1});
  d->num_cycles.assign((size_t)n_obs, 0);
  d->num_peaks.assign((size_t)n_obs, 0);
  d->rt_values = t.rt;

  // RT index from MS1 scans (src/rt_index/mod.rs:53-75)
  for (int64_t s = 0; s < n_spec; ++s)
    if (t.dsi[s] == 0) d->rt.push_back(t.rt[s]);
  const int64_t n_rt = (int64_t)d->rt.size();
  d->delta_t = n_rt > 1 ? (d->rt[n_rt - 1] - d->rt[0]) / (float)(n_rt - 1) : 1.0f;

  // per observation: isolation window of the first spectrum, unique cycles,
  // peak counts (src/dia_data_builder/mod.rs:57-91)
  std::vector<char> seen_first((size_t)n_obs, 0);
  std::vector<std::pair<int64_t, int64_t>> wc;
  wc.reserve((size_t)n_spec);
  std::vector<int32_t> win_of_spec((size_t)n_spec, -1);
  std::vector<uint16_t> cyc16((size_t)n_spec);
  for (int64_t s = 0; s < n_spec; ++s) {
    cyc16[s] = (uint16_t)t.cyc[s];
    const int64_t w = t.dsi[s];
    if (w < 0) continue;
    win_of_spec[s] = (int32_t)w;
    if (!seen_first[w]) {
      seen_first[w] = 1;
      d->win[w].lo = t.lo[s];
      d->win[w].hi = t.hi[s];
    }
    d->num_peaks[w] += t.stop[s] - t.start[s];
    wc.emplace_back(w, t.cyc[s]);
  }
  std::sort(wc.begin(), wc.end());
  for (size_t i = 0; i < wc.size(); ++i)
    if (i == 0 || wc[i] != wc[i - 1]) d->num_cycles[wc[i].first]++;

  // entry bases and slice_starts slots (observations without peaks get none)
  std::vector<int64_t> slot_of_win((size_t)std::max<int64_t>(n_obs, 1), 0);
  int64_t n_slots = 0, n_items = 0;
  for (int64_t w = 0; w < n_obs; ++w) {
    if (d->num_peaks[w] > 0xFFFFFFFFll)
      return fail(ADS_ERR_INVALID_ARGUMENT, "more than 2^32-1 peaks in one observation");
    d->win[w].base = n_items;
    n_items += d->num_peaks[w];
    if (d->num_peaks[w] > 0) {
      d->win[w].ss_off = n_slots * (d->grid_len + 1);
      slot_of_win[w] = n_slots++;
    }
  }
  std::vector<int64_t> item_off((size_t)n_spec, 0);
  {
    std::vector<int64_t> cursor((size_t)std::max<int64_t>(n_obs, 1), 0);
    for (int64_t w = 0; w < n_obs; ++w) cursor[w] = d->win[w].base;
    for (int64_t s = 0; s < n_spec; ++s) {
      const int64_t w = t.dsi[s];
      if (w < 0) continue;
      item_off[s] = cursor[w];
      cursor[w] += t.stop[s] - t.start[s];
    }
  }
  d->n_entries = n_items;

  // maximum depth of overlapping (non-empty) isolation windows, closed intervals
  {
    std::vector<std::pair<float, int>> ev;
    for (int64_t w = 0; w < n_obs; ++w)
      if (d->num_peaks[w] > 0 && d->win[w].lo <= d->win[w].hi) {
        ev.emplace_back(d->win[w].lo, -1);  // opens sort first at equal m/z
        ev.emplace_back(d->win[w].hi, +1);
      }
    std::sort(ev.begin(), ev.end());
    int depth = 0, best = 0;
    for (auto& e : ev) {
      depth += (e.second < 0) ? 1 : -1;
      best = std::max(best, depth);
    }
    d->max_overlap = best;
  }

  if (raw->cycle) {
    int64_t nc = 1;
    for (int i = 0; i < 4; ++i) {
      if (raw->cycle_shape[i] < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "negative cycle shape");
      nc *= raw->cycle_shape[i];
      d->cycle_shape[i] = raw->cycle_shape[i];
    }
    d->cycle.assign(raw->cycle, raw->cycle + nc);
  }

  GridView g;
  ADS_TRY(device_grid(device, &g));
  cudaStream_t st;
  ADS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int rc;
  if (n_peaks < (int64_t(1) << 32))
    rc = build_entries<uint32_t>(d, raw, win_of_spec, cyc16, item_off, n_items, slot_of_win,
                                 n_slots, g, st);
  else
    rc = build_entries<uint64_t>(d, raw, win_of_spec, cyc16, item_off, n_items, slot_of_win,
                                 n_slots, g, st);
  cudaStreamDestroy(st);
  if (rc != ADS_OK) return rc;

  ADS_TRY(d->win_dev.alloc(std::max<int64_t>(n_obs, 1)));
  if (n_obs)
    ADS_CUDA(cudaMemcpy(d->win_dev.p, d->win.data(), n_obs * sizeof(WinInfo), cudaMemcpyHostToDevice));
  ADS_TRY(d->rt_dev.alloc(std::max<int64_t>(n_rt, 1)));
  if (n_rt) ADS_CUDA(cudaMemcpy(d->rt_dev.p, d->rt.data(), n_rt * 4, cudaMemcpyHostToDevice));
  // copies from pageable memory may return before their DMA ends; searches read these
  // tables from non-blocking streams
  ADS_CUDA(cudaDeviceSynchronize());
  *out = guard.release();
  return ADS_OK;
}

}  // namespace
}  // namespace ads

using namespace ads;

extern "C" {

const char* ads_version(void) { return "alphadia-search-b200 0.1.0"; }

int ads_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int ads_dia_create(const AdsRawArrays* raw, int device, AdsDia** out) {
  return guarded([&] { return dia_create(raw, device, out); });
}

int ads_dia_destroy(AdsDia* dia) {
  return guarded([&] {
    if (dia) {
      DeviceGuard dg(dia->device);
      delete dia;
    }
    return ADS_OK;
  });
}

int64_t ads_dia_num_observations(const AdsDia* dia) { return dia ? dia->n_obs : 0; }

int64_t ads_dia_memory_footprint_bytes(const AdsDia* dia) {
  if (!dia) return 0;
  // src/dia_data/mod.rs:90-105 + src/quadrupole_observation/mod.rs:110-128 with
  // 64-bit Rust layouts: Vec = 24 bytes, usize = 8, [f32; 2] = 8.
  int64_t total = (int64_t)dia->rt.size() * 4 + 24;
  for (int64_t w = 0; w < dia->n_obs; ++w)
    total += 8 + 8 + 3 * 24 + (dia->grid_len + 1) * 4 + dia->num_peaks[w] * (2 + 4);
  return total;
}

int64_t ads_dia_device_bytes(const AdsDia* dia) {
  if (!dia) return 0;
  return (int64_t)(dia->slice_starts.bytes() + dia->cycles.bytes() + dia->intens.bytes() +
                   dia->intens_bf16.bytes() + dia->win_dev.bytes() + dia->rt_dev.bytes());
}

int ads_dia_rt_values(const AdsDia* dia, float* out, int64_t cap, int64_t* n) {
  return guarded([&] {
    if (!dia) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    const int64_t m = (int64_t)dia->rt_values.size();
    if (n) *n = m;
    if (out) std::memcpy(out, dia->rt_values.data(), (size_t)std::min(m, cap) * 4);
    return ADS_OK;
  });
}

int ads_dia_cycle(const AdsDia* dia, float* out, int64_t cap, int64_t shape[4]) {
  return guarded([&] {
    if (!dia) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    if (shape)
      for (int i = 0; i < 4; ++i) shape[i] = dia->cycle_shape[i];
    if (out)
      std::memcpy(out, dia->cycle.data(),
                  (size_t)std::min<int64_t>((int64_t)dia->cycle.size(), cap) * 4);
    return ADS_OK;
  });
}

int ads_dia_rt_index(const AdsDia* dia, float* out, int64_t cap, int64_t* n, float* delta_t) {
  return guarded([&] {
    if (!dia) return fail(ADS_ERR_INVALID_ARGUMENT, "null handle");
    const int64_t m = (int64_t)dia->rt.size();
    if (n) *n = m;
    if (delta_t) *delta_t = dia->delta_t;
    if (out) std::memcpy(out, dia->rt.data(), (size_t)std::min(m, cap) * 4);
    return ADS_OK;
  });
}

int ads_dia_observation_info(const AdsDia* dia, int64_t obs, float* lo, float* hi,
                             int64_t* num_cycles, int64_t* num_peaks) {
  return guarded([&] {
    if (!dia || obs < 0 || obs >= dia->n_obs)
      return fail(ADS_ERR_INVALID_ARGUMENT, "bad observation index");
    if (lo) *lo = dia->win[obs].lo;
    if (hi) *hi = dia->win[obs].hi;
    if (num_cycles) *num_cycles = dia->num_cycles[obs];
    if (num_peaks) *num_peaks = dia->num_peaks[obs];
    return ADS_OK;
  });
}

int ads_dia_copy_observation(const AdsDia* dia, int64_t obs, uint32_t* ss, uint16_t* cyc,
                             float* inten) {
  return guarded([&] {
    if (!dia || obs < 0 || obs >= dia->n_obs)
      return fail(ADS_ERR_INVALID_ARGUMENT, "bad observation index");
    DeviceGuard dg(dia->device);
    const auto& w = dia->win[obs];
    const int64_t n = dia->num_peaks[obs];
    if (ss) {
      if (w.ss_off < 0)
        std::memset(ss, 0, (size_t)(dia->grid_len + 1) * 4);
      else
        ADS_CUDA(cudaMemcpy(ss, dia->slice_starts.p + w.ss_off, (dia->grid_len + 1) * 4,
                            cudaMemcpyDeviceToHost));
    }
    if (cyc && n)
      ADS_CUDA(cudaMemcpy(cyc, dia->cycles.p + w.base, n * 2, cudaMemcpyDeviceToHost));
    if (inten && n) {
      if (dia->bf16_only) {  // the stored bfloat16 values, widened
        std::vector<uint16_t> b((size_t)n);
        ADS_CUDA(cudaMemcpy(b.data(), dia->intens_bf16.p + w.base, n * 2, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; ++i) {
          const uint32_t bits = (uint32_t)b[(size_t)i] << 16;
          std::memcpy(inten + i, &bits, 4);
        }
      } else {
        ADS_CUDA(cudaMemcpy(inten, dia->intens.p + w.base, n * 4, cudaMemcpyDeviceToHost));
      }
    }
    return ADS_OK;
  });
}

int64_t ads_mz_grid_len(void) { return (int64_t)host_grid().size(); }

int ads_mz_grid(float* out, int64_t cap) {
  return guarded([&] {
    const auto& g = host_grid();
    if (!out) return fail(ADS_ERR_INVALID_ARGUMENT, "null output");
    std::memcpy(out, g.data(), (size_t)std::min<int64_t>((int64_t)g.size(), cap) * 4);
    return ADS_OK;
  });
}

}  // extern "C"
