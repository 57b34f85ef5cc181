/*
 * ads_gpu.h — C ABI of the B200-native peak-group-selection engine.
 *
 * Drop-in boundary for `PeakGroupSelection.search` of MannLabs/alphadia-search-rs.
 * Each entry point names the reference interface it replaces (file:line in the
 * reference crate).  The ABI is plain C: opaque handles, plain pointers and sizes,
 * int status codes.  Nothing here throws or aborts across the boundary.
 *
 * Ownership: input arrays are borrowed for the duration of a call only (the
 * reference copies its numpy inputs too).  Handles own their device buffers and are
 * released by the matching *_destroy.  Candidate arrays are copied into
 * caller-allocated memory by ads_candidates_copy_out.
 *
 * Threading: calls on different handles may run concurrently.  A selection handle
 * owns one CUDA stream; calls that share a selection handle must be serialised by
 * the caller.  Error text is kept per host thread (ads_last_error).
 *
 * Device state: per device the library keeps a memory pool, the m/z grid and a log
 * table for the life of the process.  A cudaDeviceReset while the library is in use
 * invalidates them and is not supported.
 */
#ifndef ADS_GPU_H
#define ADS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define ADS_OK 0
#define ADS_ERR_INVALID_ARGUMENT 1 /* Python: ValueError */
#define ADS_ERR_OUT_OF_MEMORY 2    /* Python: MemoryError */
#define ADS_ERR_CUDA 3             /* Python: RuntimeError */
#define ADS_ERR_DEVICE_TIMEOUT 4   /* a bounded device-side wait ran out */
#define ADS_ERR_INTERNAL 5

#define ADS_MEM_HOST 0   /* array pointers are host memory */
#define ADS_MEM_DEVICE 1 /* array pointers are device memory of the handle's device */

#define ADS_PRECISION_FP32 0 /* f32 intensities, XIC and convolution (reference numerics) */
#define ADS_PRECISION_BF16 1 /* bf16-stored intensities; f32 accumulation, log and score */

/* Error text of the last failing call on this host thread ("" if none). */
const char* ads_last_error(void);
/* Library version string. */
const char* ads_version(void);
/* Number of CUDA devices visible (0 when there is none); never fails. */
int ads_device_count(void);

/* ------------------------------------------------------------------ DIAData
 * Replaces DIAData::from_arrays (src/dia_data/mod.rs:43-72), which builds through
 * DIADataBuilder::from_alpha_raw (src/dia_data_builder/mod.rs:11-139).  Argument
 * meaning follows the reference's numpy arrays; `cycle` is the 4-D float array the
 * reference stores and returns unchanged (may be NULL with all dims 0).
 */
typedef struct AdsDia AdsDia;

typedef struct {
  int32_t location; /* ADS_MEM_HOST or ADS_MEM_DEVICE for the spectrum and peak arrays */
  int64_t n_spectra;
  const int64_t* spectrum_delta_scan_idx;
  const float* isolation_lower_mz;
  const float* isolation_upper_mz;
  const int64_t* spectrum_peak_start_idx;
  const int64_t* spectrum_peak_stop_idx;
  const int64_t* spectrum_cycle_idx;
  const float* spectrum_rt;
  int64_t n_peaks;
  const float* peak_mz;
  const float* peak_intensity;
  const float* cycle; /* host memory always */
  int64_t cycle_shape[4];
} AdsRawArrays;

int ads_dia_create(const AdsRawArrays* raw, int device, AdsDia** out);
int ads_dia_destroy(AdsDia* dia);
/* DIAData.num_observations (src/dia_data/mod.rs:74-77) */
int64_t ads_dia_num_observations(const AdsDia* dia);
/* DIAData.memory_footprint_bytes (src/dia_data/mod.rs:90-105): same accounting
 * (rt index + per-observation slice_starts/cycle_indices/intensities + fixed parts). */
int64_t ads_dia_memory_footprint_bytes(const AdsDia* dia);
/* DIAData.rt_values / cycle getters (src/dia_data/mod.rs:127-135).  Copies into host
 * memory; returns the element count in *n (pass out = NULL to query). */
int ads_dia_rt_values(const AdsDia* dia, float* out, int64_t cap, int64_t* n);
int ads_dia_cycle(const AdsDia* dia, float* out, int64_t cap, int64_t shape[4]);
/* RT index of MS1 scans (src/rt_index/mod.rs:53-75). */
int ads_dia_rt_index(const AdsDia* dia, float* out, int64_t cap, int64_t* n, float* delta_t);
/* One quadrupole observation (src/quadrupole_observation/mod.rs:12-25):
 * isolation window, number of unique cycles, number of peaks. */
int ads_dia_observation_info(const AdsDia* dia, int64_t obs, float* iso_lower, float* iso_upper,
                             int64_t* num_cycles, int64_t* num_peaks);
/* Copies one observation's CSR to host: slice_starts (grid_len + 1 entries),
 * cycle_indices and intensities (num_peaks entries each).  Any pointer may be NULL. */
int ads_dia_copy_observation(const AdsDia* dia, int64_t obs, uint32_t* slice_starts,
                             uint16_t* cycle_indices, float* intensities);
/* Bytes of device memory the run holds (CSR offsets, cycles, intensities in the
 * stored precisions, windows, RT index).  An addition: the reference reports only
 * its own accounting (memory_footprint_bytes). */
int64_t ads_dia_device_bytes(const AdsDia* dia);
/* BF16-only storage (an addition, for runs searched with ADS_PRECISION_BF16 only):
 * rounds the intensities to bfloat16 (nearest even) once and releases the f32 array,
 * so the run holds 4 bytes per peak (u16 cycle + bf16 intensity) instead of 6 or 8.
 * Afterwards FP32 searches, scoring and quantification of this run fail with
 * ADS_ERR_INVALID_ARGUMENT; BF16 searches give the same results as on the f32 run;
 * ads_dia_copy_observation returns the stored bfloat16 values widened to f32. */
int ads_dia_keep_bf16_only(AdsDia* dia);
/* Length of the global 1-ppm m/z grid (src/mz_index/mod.rs:4-6,27). */
int64_t ads_mz_grid_len(void);
int ads_mz_grid(float* out, int64_t cap);

/* Self-test of the device logarithm (no reference counterpart): evaluates the
 * search kernel's ln over every float whose bit pattern lies in [lo_bits, hi_bits)
 * and counts results that differ from ln rounded once from double precision, and
 * inputs that took the slow path. */
int ads_selftest_ln(int device, uint32_t lo_bits, uint32_t hi_bits, int64_t* mismatches,
                    int64_t* slow_path);

/* ---------------------------------------------------------------- SpecLibFlat
 * Replaces SpecLibFlat::from_arrays (src/speclib_flat/mod.rs:100-188): precursor
 * arrays are stably sorted by precursor_idx, fragment arrays keep their order.
 * Arrays the selection path never reads (library m/z and RT, nAA, cardinality,
 * charge, loss type, position) may be NULL.  precursor_rt_tolerance is an
 * extension: an optional per-precursor RT half-window in seconds that replaces
 * SelectionParameters.rt_tolerance for that precursor (NULL = the global value).
 * ads_lib_create returns once the arrays have been copied (the caller may release
 * them); the sort on the device may still be queued behind other work, and every
 * call that reads the library orders itself after it.  Inside a stream capture
 * (ads_select_noalloc) the library must already be prepared: synchronise, or search
 * it once outside the capture, first.
 */
typedef struct AdsLib AdsLib;

typedef struct {
  int32_t location; /* ADS_MEM_HOST or ADS_MEM_DEVICE */
  int64_t n_precursors;
  const uint64_t* precursor_idx;
  const float* precursor_mz_library;
  const float* precursor_mz;
  const float* precursor_rt_library;
  const float* precursor_rt;
  const uint8_t* precursor_naa;
  const uint64_t* flat_frag_start_idx;
  const uint64_t* flat_frag_stop_idx;
  int64_t n_fragments;
  const float* fragment_mz_library;
  const float* fragment_mz;
  const float* fragment_intensity;
  const uint8_t* fragment_cardinality;
  const uint8_t* fragment_charge;
  const uint8_t* fragment_loss_type;
  const uint8_t* fragment_number;
  const uint8_t* fragment_position;
  const uint8_t* fragment_type;
  const float* precursor_rt_tolerance; /* extension, may be NULL */
} AdsLibArrays;

int ads_lib_create(const AdsLibArrays* arrays, int device, AdsLib** out);
int ads_lib_destroy(AdsLib* lib);
/* SpecLibFlat.num_precursors / num_fragments (src/speclib_flat/mod.rs:190-198) */
int64_t ads_lib_num_precursors(const AdsLib* lib);
int64_t ads_lib_num_fragments(const AdsLib* lib);

/* ------------------------------------------------------- PeakGroupSelection
 * SelectionParameters (src/peak_group_selection/parameters.rs:4-43): same seven
 * fields, same meaning, same defaults (ads_selection_params_default).
 */
typedef struct {
  float fwhm_rt;
  int64_t kernel_size;
  int64_t peak_length;
  float mass_tolerance;
  float rt_tolerance;
  int64_t candidate_count;
  int64_t top_k_fragments;
} AdsSelectionParams;

/* Engine options beyond the reference's parameters. */
typedef struct {
  int32_t precision;   /* ADS_PRECISION_FP32 (default) or ADS_PRECISION_BF16 */
  int32_t verbose;     /* 1: print the reference's two lines after each search
                          (src/peak_group_selection/mod.rs:123-125) */
  int32_t use_graph;   /* 1: capture the search pipeline in a CUDA graph and replay it */
  int32_t warps_per_block; /* 0 = default (4); else 1..8 warps, one precursor each
                              (FP32 searches: at most 4) */
  int32_t blocks_per_sm;   /* 0 = autotuned/default */
  int32_t gather_mode;     /* 0 = automatic, 1 = always scan bin ranges, 2 = always
                              binary-search each bin (both are exact; for testing) */
  int32_t time_stages;     /* 1: record CUDA events around each stage of a search */
  int32_t cycles_per_lane; /* 0 = chosen from the longest RT window; else 4, 8, 10, 12
                              or 16 consecutive cycles per lane of the search kernel */
  int64_t stream;          /* cudaStream_t to run on, 0 = the handle's own stream */
} AdsEngineOptions;

void ads_selection_params_default(AdsSelectionParams* p);
void ads_engine_options_default(AdsEngineOptions* o);

/* GaussianKernel::new(fwhm_rt, sigma_scale_rt, kernel_width, rt_resolution)
 * (src/kernel/mod.rs:13-56) on the host: writes the weights and their count (the
 * width rounded up to even).  Needs no device. */
int ads_gaussian_kernel(float fwhm_rt, float sigma_scale_rt, int64_t kernel_width,
                        float rt_resolution, float* out, int64_t cap, int64_t* n);

typedef struct AdsSelection AdsSelection;
typedef struct AdsCandidates AdsCandidates;

/* PeakGroupSelection::new (src/peak_group_selection/mod.rs:74-85): validates the
 * parameters and builds the Gaussian kernel (src/kernel/mod.rs:13-56) once. */
int ads_selection_create(const AdsSelectionParams* params, const AdsEngineOptions* options,
                         int device, AdsSelection** out);
int ads_selection_destroy(AdsSelection* sel);
/* Kernel weights the selection uses (length returned in *n). */
int ads_selection_kernel(const AdsSelection* sel, float* out, int64_t cap, int64_t* n);

/* PeakGroupSelection.search (src/peak_group_selection/mod.rs:87-128): returns a
 * new candidate collection in the reference's order (library order of
 * precursor_idx, then rank).  Blocks until the search is done. */
int ads_select(AdsSelection* sel, const AdsDia* dia, const AdsLib* lib, AdsCandidates** out);

/* Same search, enqueued on the selection's stream without waiting, into an existing
 * collection whose device buffers are reused (grown if needed).  The collection's
 * size is read (and the stream synchronised) by ads_candidates_size. */
int ads_select_async(AdsSelection* sel, const AdsDia* dia, const AdsLib* lib,
                     AdsCandidates* reuse);
/* Allocation-free search.  No counterpart in the reference: an addition for callers
 * that may not allocate device memory while they search -- processes whose device
 * memory belongs to another allocator (a framework's caching allocator, a serving
 * process on a fixed budget), where an allocation from this library could fail or
 * fragment that memory, and loops that cannot afford cudaFree's implicit
 * device-wide synchronisation.
 *
 * Runs the search of ads_select with default engine options and writes the
 * candidates, in the same order and with the same values, into caller-owned
 * device arrays of `capacity` rows (capacity >= precursors x min(candidate_count,
 * maxima capacity)); the row count goes to the device int64 *count and the kernels'
 * internal error flags (0 = none; anything else means the output is not to be
 * trusted) to the device int32 *flags, which must not be NULL.  The scan_* columns
 * of the reference are zero and not written.  Everything is enqueued on `stream` (a
 * cudaStream_t as integer, 0 = the legacy default stream) and the call returns
 * without waiting.
 *
 * Working memory is a fixed device array of ADS_NOALLOC_SCRATCH_BYTES that every
 * GPU context loading this library holds until the process exits; a search that
 * needs more (about 200 bytes per precursor with 12 fragments and 3 candidates;
 * RT windows longer than 2048 cycles also need about 60 KB per 1000 cycles for each
 * of at least four warps) fails with ADS_ERR_INVALID_ARGUMENT and should be split
 * over smaller libraries.  The first call on a device sets the array up (looks up its
 * device address and copies a 4 KiB table into it, then synchronises the device);
 * make that first call before any stream capture.  A cudaDeviceReset after it is
 * not supported (the address is kept for the process).  Calls whose work overlaps
 * on the GPU share the array and race: issue them on one stream or order them with
 * events. */
#define ADS_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int ads_select_noalloc(const AdsDia* dia, const AdsLib* lib, const AdsSelectionParams* params,
                       int64_t stream, int64_t capacity, uint64_t* precursor_idx, uint64_t* rank,
                       float* score, uint64_t* cycle_center, uint64_t* cycle_start,
                       uint64_t* cycle_stop, int64_t* count, int32_t* flags);

/* Empty collection bound to a selection's device, for ads_select_async. */
int ads_candidates_create(const AdsSelection* sel, AdsCandidates** out);
/* cudaStream_t (as integer) that a selection enqueues its work on. */
int64_t ads_selection_stream(const AdsSelection* sel);
/* Number of kernels the last search launched (for launch accounting). */
int64_t ads_selection_last_launches(const AdsSelection* sel);
/* Per-search counters of the last search: [0] (fragment, window) pairs gathered,
 * [1] sum over those pairs of (m/z bins + 1), [2] fragments searched, [3] XIC peak
 * entries read, [4] XIC peak entries accumulated (n_in), [5] CSR offsets read,
 * [6] XIC cells convolved and scored (sum of kept fragments x cycles).
 * Collected only while enabled with ads_selection_set_stats. */
int ads_selection_set_stats(AdsSelection* sel, int enabled);
int ads_selection_last_stats(AdsSelection* sel, int64_t* out, int64_t cap);
/* Device time in ms of the stages of every search since the previous call, measured
 * with CUDA events on the selection's stream when created with time_stages = 1:
 * [0] prep kernel, [1] search kernel, [2] compaction kernels (sums), [3] number of
 * searches.  Waits for the last recorded search. */
int ads_selection_stage_times(AdsSelection* sel, float* ms, int64_t cap);
/* Autotuner (an engine addition; the reference has no launch shapes to tune).
 * Times the search of `dia` x `lib` (`repeats` timed searches per shape, after
 * one warm-up) for warps per block 2, 4, 8 (precursors in flight per CTA; 2 and 4 for
 * FP32) and cycles
 * per lane 0 (length classes), 4, 8, 10, 12, 16 (cycles per tile = 32 x that),
 * keeps the fastest in the selection's options and caches it per workload shape
 * (device, precision, kernel half width, longest RT window, precursors, fragments)
 * for the process.  Writes the choice and its mean ms where the pointers are not
 * NULL.  Blocks until done. */
int ads_selection_autotune(AdsSelection* sel, const AdsDia* dia, const AdsLib* lib,
                           int32_t repeats, int32_t* warps_per_block, int32_t* cycles_per_lane,
                           float* best_ms);

/* ------------------------------------------------------- CandidateCollection
 * CandidateCollection.len / to_arrays (src/candidate/entry.rs:61-173). */
int64_t ads_candidates_size(AdsCandidates* cand);
/* Copies into caller arrays of ads_candidates_size() elements, in the tuple order of
 * to_arrays: precursor_idx, rank, score, scan_center, scan_start, scan_stop,
 * cycle_center, cycle_start, cycle_stop (u64 except score f32).  Any pointer may be
 * NULL to skip that array (the scan_* arrays are always zero, as in the reference). */
int ads_candidates_copy_out(AdsCandidates* cand, uint64_t* precursor_idx, uint64_t* rank,
                            float* score, uint64_t* scan_center, uint64_t* scan_start,
                            uint64_t* scan_stop, uint64_t* cycle_center, uint64_t* cycle_start,
                            uint64_t* cycle_stop);
int ads_candidates_destroy(AdsCandidates* cand);

/* ---------------------------------------------------------------- scoring */

/* ScoringParameters (src/peak_group_scoring/parameters.rs:4-40). */
typedef struct {
  float mass_tolerance;    /* ppm; default 7.0 */
  int64_t top_k_fragments; /* default 100 */
} AdsScoringParams;
void ads_scoring_params_default(AdsScoringParams* p);

/* CandidateFeatureCollection (src/candidate/features.rs:192-431): 41 f32 features per
 * candidate, device resident. */
typedef struct AdsFeatures AdsFeatures;

/* PeakGroupScoring.score (src/peak_group_scoring/mod.rs:42-101) of the candidates of a
 * search (waits for that search).  Candidates whose precursor_idx is not in the library
 * are left out, as in the reference; the others keep their order.  verbose: print the
 * reference's "Scored N candidates at R candidates/second" line.  The library's IDF
 * histogram (src/idf/mod.rs:13-33) is built on its first scoring call. */
int ads_score(const AdsScoringParams* params, const AdsDia* dia, AdsLib* lib, AdsCandidates* cand,
              int verbose, AdsFeatures** out);
/* The same for candidate columns given as arrays (CandidateCollection.from_arrays),
 * host or device memory.  Cycle ranges outside the run's RT index are an
 * ADS_ERR_INVALID_ARGUMENT (the reference indexes out of bounds). */
int ads_score_arrays(const AdsScoringParams* params, const AdsDia* dia, AdsLib* lib, int64_t n,
                     const uint64_t* precursor_idx, const uint64_t* rank, const float* score,
                     const uint64_t* cycle_center, const uint64_t* cycle_start,
                     const uint64_t* cycle_stop, int location, int verbose, AdsFeatures** out);
/* Scored candidates (rows that to_dict_arrays returns). */
int64_t ads_features_size(const AdsFeatures* features);
/* Device time of the scoring kernel that filled the handle, in milliseconds (CUDA
 * events on the launching stream); 0 for an empty collection, -1 for a null handle.
 * The reference prints the same figure as candidates per second
 * (src/peak_group_scoring/mod.rs:91-98). */
float ads_features_kernel_ms(const AdsFeatures* features);
/* Copies into host arrays of ads_features_size() elements; `features` holds the 41
 * columns one after another, in the order of ads_feature_names (CandidateFeatureCollection
 * .get_feature_names, src/candidate/features.rs:6-48). */
int ads_features_copy_out(const AdsFeatures* features, uint64_t* precursor_idx, uint64_t* rank,
                          float* features_out);
int ads_features_destroy(AdsFeatures* features);
/* Writes up to cap feature names; returns their number (41). */
int ads_feature_names(const char** names, int cap);

/* Sharded scoring.  The IDF of scoring (src/idf/mod.rs:13-33) counts the fragments of
 * the whole library per m/z grid bin.  A library split across ranks gives each rank's
 * SpecLibFlat only its own counts; the ranks sum their histograms (one all-reduce of
 * ads_idf_bins() 32-bit counts) and their fragment totals and set the sums back, after
 * which each rank scores its candidates as the unsplit library would. */
int64_t ads_idf_bins(void);
/* This library's own histogram (n = ads_idf_bins()) into host or device memory. */
int ads_lib_idf_counts(AdsLib* lib, uint32_t* counts, int location);
/* Replaces the histogram and the fragment total scoring uses for this library. */
int ads_lib_set_idf(AdsLib* lib, const uint32_t* counts, double total_fragments, int location);

/* ---- PeakGroupQuantification (src/peak_group_quantification/mod.rs:49-168) ---- */

/* QuantificationParameters (src/peak_group_quantification/parameters.rs:4-37). */
typedef struct AdsQuantParams {
  float tolerance_ppm;     /* default 7.0 */
  int64_t top_k_fragments; /* default 10000 */
} AdsQuantParams;
void ads_quant_params_default(AdsQuantParams* p);

/* SpecLibFlatQuantified (src/speclib_flat_quantified/mod.rs:19-64), device resident
 * until copied out. */
typedef struct AdsQuant AdsQuant;
/* PeakGroupQuantification.quantify of the candidates a search left on the device: per
 * candidate its precursor's fragments (filtered, top-k, m/z order) with the dense XIC's
 * row sums as observed intensity, the intensity-weighted observed m/z and its ppm error,
 * and the correlation with the median of the non-zero normalised profiles; fragments
 * with an observed intensity of 0 are dropped, and so is a candidate left without any
 * (as are unknown precursors, empty cycle ranges and centres outside them).  A range
 * that ends beyond the run's RT index is an ADS_ERR_INVALID_ARGUMENT. */
int ads_quantify(const AdsQuantParams* params, const AdsDia* dia, AdsLib* lib, AdsCandidates* cand,
                 int verbose, AdsQuant** out);
/* The same for candidate columns given as arrays, host or device memory. */
int ads_quantify_arrays(const AdsQuantParams* params, const AdsDia* dia, AdsLib* lib, int64_t n,
                        const uint64_t* precursor_idx, const uint64_t* rank,
                        const uint64_t* cycle_center, const uint64_t* cycle_start,
                        const uint64_t* cycle_stop, int location, int verbose, AdsQuant** out);
int ads_quant_sizes(const AdsQuant* quant, int64_t* n_precursors, int64_t* n_fragments);
/* Device time of the quantification kernel in ms (an addition). */
float ads_quant_kernel_ms(const AdsQuant* quant);
/* Copies the SpecLibFlatQuantified layout into host arrays (any may be NULL): per
 * precursor (n_precursors, sorted by precursor_idx, ties in candidate order)
 * precursor_idx, the precursor's row in the arrays given to ads_lib_create, rank,
 * rt_observed and its [start, stop) range of fragments; per fragment (n_fragments, in
 * candidate order) its row in the library's fragment arrays, observed intensity,
 * observed m/z, correlation, mass error, precursor_idx and rank.  The library's
 * pass-through columns (m/z, RT, naa, fragment annotations) are the caller's arrays at
 * those rows (src/speclib_flat_quantified/mod.rs:126-210). */
int ads_quant_copy_out(const AdsQuant* quant, uint64_t* precursor_idx, uint64_t* precursor_row,
                       uint64_t* rank, float* rt_observed, uint64_t* flat_frag_start_idx,
                       uint64_t* flat_frag_stop_idx, uint64_t* fragment_row, float* intensity,
                       float* mz_observed, float* correlation_observed, float* mass_error_observed,
                       uint64_t* fragment_precursor_idx, uint64_t* fragment_rank);
int ads_quant_destroy(AdsQuant* quant);

#ifdef __cplusplus
}
#endif
#endif /* ADS_GPU_H */
