// SpecLibFlat on the device (SpecLibFlat::from_arrays, src/speclib_flat/mod.rs:100-188).
// Precursor arrays are stably sorted by precursor_idx; fragment arrays keep their
// order and are addressed through flat_frag_start/stop_idx.
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

template <class T>
int upload(DevBuf<T>& dst, const T* src, int64_t n, int loc, cudaStream_t st) {
  ADS_TRY(dst.alloc((size_t)std::max<int64_t>(n, 1)));
  if (n == 0) return ADS_OK;
  if (!src) return fail(ADS_ERR_INVALID_ARGUMENT, "null array pointer");
  ADS_CUDA(cudaMemcpyAsync(dst.p, src, (size_t)n * sizeof(T),
                           loc == ADS_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           st));
  return ADS_OK;
}

template <class T>
int permute(DevBuf<T>& buf, const uint32_t* perm, int64_t n, cudaStream_t st) {
  if (n == 0) return ADS_OK;
  DevBuf<T> out;
  ADS_TRY(out.alloc((size_t)n));
  gather_kernel<T><<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(n, perm, buf.p,
                                                                                   out.p);
  ADS_LAUNCH_CHECK();
  ADS_CUDA(cudaStreamSynchronize(st));
  buf = std::move(out);
  return ADS_OK;
}

template <class T>
int host_copy(const T* src, int64_t n, int loc, std::vector<T>& dst) {
  dst.resize((size_t)n);
  if (n == 0) return ADS_OK;
  if (!src) return fail(ADS_ERR_INVALID_ARGUMENT, "null array pointer");
  if (loc == ADS_MEM_DEVICE)
    ADS_CUDA(cudaMemcpy(dst.data(), src, (size_t)n * sizeof(T), cudaMemcpyDeviceToHost));
  else
    std::memcpy(dst.data(), src, (size_t)n * sizeof(T));
  return ADS_OK;
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

  // validation on host copies of the small per-precursor arrays
  std::vector<uint64_t> fs, fe;
  std::vector<float> prt, tol;
  ADS_TRY(host_copy(a->flat_frag_start_idx, P, L, fs));
  ADS_TRY(host_copy(a->flat_frag_stop_idx, P, L, fe));
  ADS_TRY(host_copy(a->precursor_rt, P, L, prt));
  auto lib = std::make_unique<AdsLib>();
  lib->device = device;
  lib->n_prec = P;
  lib->n_frag = NF;
  for (int64_t i = 0; i < P; ++i) {
    if (fs[i] > fe[i] || fe[i] > (uint64_t)NF)
      return fail(ADS_ERR_INVALID_ARGUMENT,
                  "precursor " + std::to_string(i) + ": fragment range outside [0, n_fragments]");
    if (!std::isfinite(prt[i]))
      return fail(ADS_ERR_INVALID_ARGUMENT, "precursor " + std::to_string(i) + ": RT is not finite");
    lib->max_frag = std::max<int64_t>(lib->max_frag, (int64_t)(fe[i] - fs[i]));
  }
  if (a->precursor_rt_tolerance) {
    ADS_TRY(host_copy(a->precursor_rt_tolerance, P, L, tol));
    lib->has_tol = true;
    for (float v : tol)
      if (std::isfinite(v)) lib->max_tol = std::max(lib->max_tol, v);
      else if (!std::isnan(v)) lib->max_tol = INFINITY;
  }

  cudaStream_t st;
  ADS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};

  ADS_TRY(upload(lib->pidx, a->precursor_idx, P, L, st));
  ADS_TRY(upload(lib->pmz, a->precursor_mz, P, L, st));
  ADS_TRY(upload(lib->prt, a->precursor_rt, P, L, st));
  ADS_TRY(upload(lib->fstart, a->flat_frag_start_idx, P, L, st));
  ADS_TRY(upload(lib->fstop, a->flat_frag_stop_idx, P, L, st));
  if (lib->has_tol) ADS_TRY(upload(lib->ptol, a->precursor_rt_tolerance, P, L, st));
  ADS_TRY(upload(lib->fmz, a->fragment_mz, NF, L, st));
  ADS_TRY(upload(lib->fint, a->fragment_intensity, NF, L, st));
  ADS_TRY(upload(lib->fnum, a->fragment_number, NF, L, st));
  ADS_TRY(upload(lib->ftype, a->fragment_type, NF, L, st));

  if (P > 1) {
    // stable radix sort of (precursor_idx, position): equal keys keep input order
    DevBuf<uint64_t> keys_out;
    DevBuf<uint32_t> pos_in, pos_out;
    ADS_TRY(keys_out.alloc(P));
    ADS_TRY(pos_in.alloc(P));
    ADS_TRY(pos_out.alloc(P));
    std::vector<uint32_t> iota((size_t)P);
    for (int64_t i = 0; i < P; ++i) iota[i] = (uint32_t)i;
    ADS_CUDA(cudaMemcpyAsync(pos_in.p, iota.data(), P * 4, cudaMemcpyHostToDevice, st));
    size_t tb = 0;
    ADS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, lib->pidx.p, keys_out.p, pos_in.p,
                                             pos_out.p, P, 0, 64, st));
    DevBuf<unsigned char> tmp;
    ADS_TRY(tmp.alloc(tb + 16));
    ADS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, lib->pidx.p, keys_out.p, pos_in.p,
                                             pos_out.p, P, 0, 64, st));
    ADS_CUDA(cudaStreamSynchronize(st));
    lib->pidx = std::move(keys_out);
    ADS_TRY(permute(lib->pmz, pos_out.p, P, st));
    ADS_TRY(permute(lib->prt, pos_out.p, P, st));
    ADS_TRY(permute(lib->fstart, pos_out.p, P, st));
    ADS_TRY(permute(lib->fstop, pos_out.p, P, st));
    if (lib->has_tol) ADS_TRY(permute(lib->ptol, pos_out.p, P, st));
  }
  ADS_CUDA(cudaStreamSynchronize(st));
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
