// SpecLibFlat on the device (SpecLibFlat::from_arrays, src/speclib_flat/mod.rs:100-188).
// Precursor arrays are stably sorted by precursor_idx; fragment arrays keep their
// order and are addressed through flat_frag_start/stop_idx.  All device arrays of a
// library live in one allocation.
#include <cub/cub.cuh>

#include <cmath>
#include <cstring>
#include <memory>

#include "common.cuh"

namespace ads {
namespace {

template <class T>
__global__ void gather_kernel(int64_t n, const uint32_t* __restrict__ perm,
                              const T* __restrict__ src, T* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

__global__ void iota_kernel(int64_t n, uint32_t* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)i;
}

// Bump allocator over one device allocation (256-byte aligned pieces).
struct Carver {
  char* base = nullptr;
  size_t off = 0;
  template <class T>
  T* take(int64_t n) {
    T* p = reinterpret_cast<T*>(base + off);
    off += ((size_t)std::max<int64_t>(n, 1) * sizeof(T) + 255) / 256 * 256;
    return p;
  }
};

template <class T>
int copy_in(T* dst, const T* src, int64_t n, int loc, cudaStream_t st) {
  if (n == 0) return ADS_OK;
  if (!src) return fail(ADS_ERR_INVALID_ARGUMENT, "null array pointer");
  ADS_CUDA(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(T),
                           loc == ADS_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           st));
  return ADS_OK;
}

// Host view of a small per-precursor array: the caller's memory when it is on the
// host, a copy when it is on the device.
template <class T>
int host_view(const T* src, int64_t n, int loc, std::vector<T>& store, const T** out) {
  if (n > 0 && !src) return fail(ADS_ERR_INVALID_ARGUMENT, "null array pointer");
  if (loc == ADS_MEM_HOST) {
    *out = src;
    return ADS_OK;
  }
  store.resize((size_t)n);
  if (n) ADS_CUDA(cudaMemcpy(store.data(), src, (size_t)n * sizeof(T), cudaMemcpyDeviceToHost));
  *out = store.data();
  return ADS_OK;
}

template <class T>
void launch_gather(int64_t n, const uint32_t* perm, const T* src, T* dst, cudaStream_t st) {
  gather_kernel<T><<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(n, perm, src, dst);
}

int lib_create(const AdsLibArrays* a, int device, AdsLib** out) {
  if (!a || !out) return fail(ADS_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (a->location != ADS_MEM_HOST && a->location != ADS_MEM_DEVICE)
    return fail(ADS_ERR_INVALID_ARGUMENT, "location must be ADS_MEM_HOST or ADS_MEM_DEVICE");
  const int64_t P = a->n_precursors, NF = a->n_fragments;
  if (P < 0 || NF < 0) return fail(ADS_ERR_INVALID_ARGUMENT, "negative array length");
  if (P >= (int64_t(1) << 32)) return fail(ADS_ERR_INVALID_ARGUMENT, "more than 2^32-1 precursors");
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
    cudaGetLastError();
    return fail(ADS_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= n_dev) return fail(ADS_ERR_INVALID_ARGUMENT, "bad device index");
  DeviceGuard dg(device);
  const int L = a->location;

  // host views of the per-precursor arrays the host validates below
  std::vector<uint64_t> fs_store, fe_store;
  std::vector<float> rt_store, tol_store;
  const uint64_t *fs = nullptr, *fe = nullptr;
  const float *prt = nullptr, *tol = nullptr;
  ADS_TRY(host_view(a->flat_frag_start_idx, P, L, fs_store, &fs));
  ADS_TRY(host_view(a->flat_frag_stop_idx, P, L, fe_store, &fe));
  ADS_TRY(host_view(a->precursor_rt, P, L, rt_store, &prt));
  auto lib = std::make_unique<AdsLib>();
  lib->device = device;
  lib->n_prec = P;
  lib->n_frag = NF;
  lib->has_tol = a->precursor_rt_tolerance != nullptr;

  cudaStream_t st;
  ADS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};

  // one allocation for the library; a second, temporary one for the sort
  auto plan_lib = [&](Carver& c) {
    lib->pidx_p = c.take<uint64_t>(P);
    lib->pmz_p = c.take<float>(P);
    lib->prt_p = c.take<float>(P);
    lib->ptol_p = lib->has_tol ? c.take<float>(P) : nullptr;
    lib->prow_p = c.take<uint32_t>(P);
    lib->fstart_p = c.take<uint64_t>(P);
    lib->fstop_p = c.take<uint64_t>(P);
    lib->naa_p = c.take<uint8_t>(P);
    lib->fmz_p = c.take<float>(NF);
    lib->fmzl_p = c.take<float>(NF);
    lib->fint_p = c.take<float>(NF);
    lib->fnum_p = c.take<uint8_t>(NF);
    lib->ftype_p = c.take<uint8_t>(NF);
  };
  Carver sizing;
  plan_lib(sizing);
  ADS_TRY(lib->arena.alloc(sizing.off));
  Carver c{lib->arena.p, 0};
  plan_lib(c);

  DevBuf<char> tmp;
  Carver t;
  uint64_t* pidx_in = nullptr;
  float *pmz_in = nullptr, *prt_in = nullptr, *ptol_in = nullptr;
  uint64_t *fs_in = nullptr, *fe_in = nullptr;
  uint32_t *pos_in = nullptr, *pos_out = nullptr;
  uint8_t* naa_in = nullptr;
  void* sort_tmp = nullptr;
  size_t sort_bytes = 0;
  // host arrays already in precursor_idx order (non-decreasing) need no sort: the
  // stable sort would keep them as they are
  bool in_order = false;
  if (L == ADS_MEM_HOST && P > 1 && a->precursor_idx) {
    const uint64_t* pi = a->precursor_idx;
    in_order = true;
    for (int64_t i = 1; i < P && in_order; ++i) in_order = pi[i - 1] <= pi[i];
  }
  const bool sort = P > 1 && !in_order;
  if (sort) {
    ADS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint64_t*)nullptr,
                                             (uint64_t*)nullptr, (uint32_t*)nullptr,
                                             (uint32_t*)nullptr, P, 0, 64, st));
    auto plan_tmp = [&](Carver& q) {
      pidx_in = q.take<uint64_t>(P);
      pmz_in = q.take<float>(P);
      prt_in = q.take<float>(P);
      ptol_in = lib->has_tol ? q.take<float>(P) : nullptr;
      fs_in = q.take<uint64_t>(P);
      fe_in = q.take<uint64_t>(P);
      naa_in = q.take<uint8_t>(P);
      pos_in = q.take<uint32_t>(P);
      sort_tmp = q.take<char>((int64_t)sort_bytes);
    };
    Carver tsize;
    plan_tmp(tsize);
    ADS_TRY(tmp.alloc(tsize.off));
    t.base = tmp.p;
    plan_tmp(t);
  }
  // precursor arrays land in the temporary area when they still need sorting
  ADS_TRY(copy_in(sort ? pidx_in : lib->pidx_p, a->precursor_idx, P, L, st));
  ADS_TRY(copy_in(sort ? pmz_in : lib->pmz_p, a->precursor_mz, P, L, st));
  ADS_TRY(copy_in(sort ? prt_in : lib->prt_p, a->precursor_rt, P, L, st));
  ADS_TRY(copy_in(sort ? fs_in : lib->fstart_p, a->flat_frag_start_idx, P, L, st));
  ADS_TRY(copy_in(sort ? fe_in : lib->fstop_p, a->flat_frag_stop_idx, P, L, st));
  if (lib->has_tol) ADS_TRY(copy_in(sort ? ptol_in : lib->ptol_p, a->precursor_rt_tolerance, P, L, st));
  if (a->precursor_naa)
    ADS_TRY(copy_in(sort ? naa_in : lib->naa_p, a->precursor_naa, P, L, st));
  else if (P)
    ADS_CUDA(cudaMemsetAsync(sort ? naa_in : lib->naa_p, 0, (size_t)P, st));
  ADS_TRY(copy_in(lib->fmz_p, a->fragment_mz, NF, L, st));
  // fragment_mz_library (the IDF of scoring reads it) defaults to fragment_mz; when it
  // is fragment_mz's own array it is copied on the device instead of uploaded again
  if (!a->fragment_mz_library || a->fragment_mz_library == a->fragment_mz) {
    if (NF) ADS_CUDA(cudaMemcpyAsync(lib->fmzl_p, lib->fmz_p, (size_t)NF * sizeof(float),
                                     cudaMemcpyDeviceToDevice, st));
  } else {
    ADS_TRY(copy_in(lib->fmzl_p, a->fragment_mz_library, NF, L, st));
  }
  ADS_TRY(copy_in(lib->fint_p, a->fragment_intensity, NF, L, st));
  ADS_TRY(copy_in(lib->fnum_p, a->fragment_number, NF, L, st));
  ADS_TRY(copy_in(lib->ftype_p, a->fragment_type, NF, L, st));
  // the caller's arrays may be released once the copies above have landed
  cudaEvent_t copied = nullptr;
  ADS_CUDA(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
  struct EventGuard {
    cudaEvent_t e;
    ~EventGuard() { cudaEventDestroy(e); }
  } eg{copied};
  ADS_CUDA(cudaEventRecord(copied, st));

  // validation of the per-precursor arrays (the reference panics on these), on the
  // host while the copies above are in flight; on failure the buffers are released
  // only after the device is idle
  for (int64_t i = 0; i < P; ++i) {
    if (fs[i] > fe[i] || fe[i] > (uint64_t)NF)
      return fail(ADS_ERR_INVALID_ARGUMENT,
                  "precursor " + std::to_string(i) + ": fragment range outside [0, n_fragments]");
    if (!std::isfinite(prt[i]))
      return fail(ADS_ERR_INVALID_ARGUMENT, "precursor " + std::to_string(i) + ": RT is not finite");
    lib->max_frag = std::max<int64_t>(lib->max_frag, (int64_t)(fe[i] - fs[i]));
    lib->min_frag = i == 0 ? (int64_t)(fe[i] - fs[i]) : std::min<int64_t>(lib->min_frag, (int64_t)(fe[i] - fs[i]));
  }
  if (a->precursor_rt_tolerance) {
    ADS_TRY(host_view(a->precursor_rt_tolerance, P, L, tol_store, &tol));
    for (int64_t i = 0; i < P; ++i) {
      const float v = tol[i];
      if (std::isfinite(v))
        lib->max_tol = std::max(lib->max_tol, v);
      else if (!std::isnan(v))
        lib->max_tol = INFINITY;
    }
  }

  if (sort) {
    // stable radix sort of (precursor_idx, position): equal keys keep input order
    iota_kernel<<<(int)std::min<int64_t>((P + 255) / 256, 4096), 256, 0, st>>>(P, pos_in);
    ADS_LAUNCH_CHECK();
    pos_out = lib->prow_p;  // kept: the input row of every sorted precursor
    ADS_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, pidx_in, lib->pidx_p, pos_in,
                                             pos_out, P, 0, 64, st));
    launch_gather(P, pos_out, pmz_in, lib->pmz_p, st);
    launch_gather(P, pos_out, prt_in, lib->prt_p, st);
    launch_gather(P, pos_out, fs_in, lib->fstart_p, st);
    launch_gather(P, pos_out, fe_in, lib->fstop_p, st);
    launch_gather(P, pos_out, naa_in, lib->naa_p, st);
    if (lib->has_tol) launch_gather(P, pos_out, ptol_in, lib->ptol_p, st);
    ADS_LAUNCH_CHECK();
    // the sort's temporary area is freed behind its last use on this stream: a
    // library built while searches run elsewhere on the device does not wait for them
    tmp.release_async(st);
  } else if (P > 0) {
    iota_kernel<<<(int)std::min<int64_t>((P + 255) / 256, 4096), 256, 0, st>>>(P, lib->prow_p);
    ADS_LAUNCH_CHECK();
  }
  // The sort and gathers need SMs, which a search already running elsewhere on the
  // device may hold until it ends: waiting for them here would keep the caller from
  // enqueueing its next search behind that one.  Readers of the library wait on
  // `ready` instead; the host waits for the uploads only.
  ADS_CUDA(cudaEventCreateWithFlags(&lib->ready, cudaEventDisableTiming));
  ADS_CUDA(cudaEventRecord(lib->ready, st));
  ADS_CUDA(cudaEventSynchronize(copied));
  *out = lib.release();
  return ADS_OK;
}

}  // namespace
}  // namespace ads

using namespace ads;

extern "C" {

int ads_lib_create(const AdsLibArrays* arrays, int device, AdsLib** out) {
  return guarded([&] { return lib_create(arrays, device, out); });
}

int ads_lib_destroy(AdsLib* lib) {
  return guarded([&] {
    if (lib) {
      DeviceGuard dg(lib->device);
      delete lib;
    }
    return ADS_OK;
  });
}

int64_t ads_lib_num_precursors(const AdsLib* lib) { return lib ? lib->n_prec : 0; }
int64_t ads_lib_num_fragments(const AdsLib* lib) { return lib ? lib->n_frag : 0; }

}  // extern "C"
