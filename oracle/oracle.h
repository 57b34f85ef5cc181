/*
 * CPU oracle for the peak-group-selection path — TEST INFRASTRUCTURE ONLY.
 *
 * A from-scratch C++17 restatement of the reference crate's scalar CPU path
 * (MannLabs/alphadia-search-rs).  Only tests, `__graft_entry__.smoke()` and the
 * CPU legs of `bench.py` may load it, and only as the checker or the timed CPU
 * baseline.  The product (libads_gpu.so) never links or calls it.
 *
 * Every function cites the reference file:line it restates.  Arithmetic is
 * plain IEEE f32 in the reference's operation order; the library is compiled
 * with -ffp-contract=off and without fast-math so no FMA contraction or
 * re-association happens, and it calls glibc logf/expf/sqrtf exactly where the
 * reference calls f32::ln/exp/sqrt (Rust lowers those to the platform libm).
 *
 * Parity pin: the known-answer tests of the reference crate for this path
 * (grid length, RT limits, window membership, builder ordering, XIC sums,
 * log-dot values, local maxima, fragment filter, candidate arrays) are ported
 * as tests against this library.  No reference test pins an end-to-end
 * search() result; the whole-path result is pinned only piecewise.
 */
#ifndef ADS_ORACLE_H
#define ADS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- m/z grid: src/mz_index/mod.rs:8-25, :55-90, :95-127 ---- */
int64_t orc_ppm_index_len(float resolution_ppm, float mz_start, float mz_end);
/* writes orc_ppm_index_len(...) values */
void orc_ppm_index(float resolution_ppm, float mz_start, float mz_end, float* out);
int64_t orc_find_closest_index(const float* grid, int64_t n, float mz);
void orc_mz_range_indices(const float* grid, int64_t n, float lower_mz, float upper_mz,
                          int64_t* start, int64_t* stop);

/* ---- RT index: src/rt_index/mod.rs:20-26, :89-138 ---- */
float orc_mean_delta_t(const float* rt, int64_t n);
void orc_rt_limits(const float* rt, int64_t n, float delta_t, float precursor_rt,
                   float rt_tolerance, int64_t num_cycles_padding, int64_t* lower, int64_t* upper);

/* Rust 1.88 `slice::binary_search` on sorted u16 values (returns Ok/Err index). */
int64_t orc_rust_binary_search_u16(const uint16_t* a, int64_t n, uint16_t x);

/* ---- Gaussian kernel: src/kernel/mod.rs:13-56; returns the array length ---- */
int64_t orc_gaussian_kernel(float fwhm_rt, float sigma_scale_rt, int64_t kernel_width,
                            float rt_resolution, float* out /* capacity >= kernel_width + 2 */);

/* ---- convolution: src/convolution/scalar.rs:5-56 ---- */
void orc_convolution(const float* kernel, int64_t klen, const float* xic, int64_t n_rows,
                     int64_t n_cols, float* out);

/* ---- log-dot score: src/score/scalar.rs:4-25.
 * log_mode 0: glibc logf (what the reference calls on Linux).
 * log_mode 1: logf correctly rounded, i.e. (float)log((double)x). ---- */
void orc_log_dot(const float* a, int64_t n_rows, int64_t n_cols, const float* w, float* out,
                 int log_mode);

/* ---- local maxima: src/peak_group_selection/mod.rs:23-64; returns the count ---- */
int64_t orc_local_maxima(const float* a, int64_t n, int64_t offset, int64_t* idx, float* val);

/* ---- fragment filter: src/speclib_flat/mod.rs:240-345.
 * Writes the original positions of the kept fragments in output order and
 * returns how many were kept. ---- */
int64_t orc_filter_sort_fragments(int64_t n, const float* mz, const float* intensity,
                                  const uint8_t* number, const uint8_t* type, int non_zero,
                                  int filter_y1, int64_t top_k, int64_t* out_pos);

/* ---- DIAData build: src/dia_data_builder/mod.rs:11-139, src/rt_index/mod.rs:53-75 ---- */
typedef struct OrcDia OrcDia;
OrcDia* orc_dia_build(int64_t n_spectra, const int64_t* delta_scan_idx, const float* iso_lower,
                      const float* iso_upper, const int64_t* peak_start, const int64_t* peak_stop,
                      const int64_t* cycle_idx, const float* spectrum_rt, int64_t n_peaks,
                      const float* peak_mz, const float* peak_intensity, int n_threads);
void orc_dia_free(OrcDia* d);
int64_t orc_dia_num_obs(const OrcDia* d);
int64_t orc_dia_grid_len(const OrcDia* d);
const float* orc_dia_grid(const OrcDia* d);
int64_t orc_dia_rt_len(const OrcDia* d);
const float* orc_dia_rt(const OrcDia* d);
float orc_dia_delta_t(const OrcDia* d);
void orc_dia_obs_window(const OrcDia* d, int64_t obs, float* lower, float* upper);
int64_t orc_dia_obs_num_cycles(const OrcDia* d, int64_t obs);
int64_t orc_dia_obs_num_peaks(const OrcDia* d, int64_t obs);
const uint32_t* orc_dia_obs_slice_starts(const OrcDia* d, int64_t obs);
const uint16_t* orc_dia_obs_cycles(const OrcDia* d, int64_t obs);
const float* orc_dia_obs_intensities(const OrcDia* d, int64_t obs);
/* src/quadrupole_observation/mod.rs:70-107 on a caller-built observation
 * (slice_starts has n_slices+1 entries); adds into xic[stop-start]. */
void orc_fill_xic_slice_raw(const uint32_t* slice_starts, int64_t n_slices, const uint16_t* cycles,
                            const float* intensities, const float* grid, int64_t grid_len,
                            float* xic, int64_t cycle_start, int64_t cycle_stop,
                            float mass_tolerance, float mz);
/* src/dia_data/mod.rs:79-87; returns count, writes up to cap indices */
int64_t orc_dia_valid_observations(const OrcDia* d, float precursor_mz, int64_t* out, int64_t cap);
/* src/dense_xic_observation/mod.rs:30-64 — out is n_frag x (stop-start), row-major */
void orc_dense_xic(const OrcDia* d, float precursor_mz, int64_t cycle_start, int64_t cycle_stop,
                   float mass_tolerance, const float* fragment_mz, int64_t n_frag, float* out);

/* ---- SpecLibFlat: src/speclib_flat/mod.rs:100-188 (stable sort by precursor_idx) ---- */
typedef struct OrcLib OrcLib;
OrcLib* orc_lib_build(int64_t n_prec, const uint64_t* precursor_idx, const float* precursor_mz,
                      const float* precursor_rt, const uint64_t* frag_start,
                      const uint64_t* frag_stop, int64_t n_frag, const float* fragment_mz,
                      const float* fragment_intensity, const uint8_t* fragment_number,
                      const uint8_t* fragment_type);
void orc_lib_free(OrcLib* l);
int64_t orc_lib_num_precursors(const OrcLib* l);

/* ---- search: src/peak_group_selection/mod.rs:94-195 ---- */
typedef struct {
  float fwhm_rt;
  int64_t kernel_size;
  int64_t peak_length;
  float mass_tolerance;
  float rt_tolerance;
  int64_t candidate_count;
  int64_t top_k_fragments;
} OrcParams;

typedef struct OrcResult OrcResult;
/* rt_tolerance_per_precursor: optional (NULL = params.rt_tolerance for all), indexed in
 * sorted-library order.  subset: optional list of sorted-library positions to search
 * (NULL = all, in order).  precision 0 = f32 (reference), 1 = f64 variant (same control
 * flow, XIC/kernel/convolution/log/score in double). */
OrcResult* orc_search(const OrcDia* d, const OrcLib* l, const OrcParams* p,
                      const float* rt_tolerance_per_precursor, const int64_t* subset,
                      int64_t n_subset, int log_mode, int precision, int n_threads);
int64_t orc_result_len(const OrcResult* r);
void orc_result_copy(const OrcResult* r, uint64_t* precursor_idx, uint64_t* rank, float* score,
                     double* score_f64, uint64_t* cycle_center, uint64_t* cycle_start,
                     uint64_t* cycle_stop);
void orc_result_free(OrcResult* r);

/* Per-precursor trace for debugging: fills the filtered fragment count, the cycle
 * limits and (if the buffers are large enough) the XIC, convolved XIC and score. */
int64_t orc_trace_precursor(const OrcDia* d, const OrcLib* l, const OrcParams* p,
                            float rt_tolerance, int64_t lib_pos, int log_mode,
                            int64_t* cycle_start, int64_t* cycle_stop, int64_t* n_frag,
                            float* xic, float* conv, float* score, int64_t cap);

/* f64 score of one precursor at given absolute cycles (for BF16 error reports). Writes
 * scores and returns max_j |score_f64[j]| over the whole cycle window. */
double orc_scores_f64_at(const OrcDia* d, const OrcLib* l, const OrcParams* p,
                         float rt_tolerance, int64_t lib_pos, const int64_t* cycles, int64_t n,
                         double* out);


/* ---- PeakGroupScoring: src/peak_group_scoring/mod.rs:42-340 ---- */
typedef struct OrcFeatures OrcFeatures;
/* precursor_naa in input order; fragment_mz_library (n_frag, input order) */
void orc_lib_set_scoring(OrcLib* l, const uint8_t* precursor_naa, int64_t n_frag,
                         const float* fragment_mz_library);
/* Candidates in the order given; those whose precursor_idx is not in the library are
 * skipped.  41 features per row in FEATURE_NAMES order (src/candidate/features.rs:6-48). */
OrcFeatures* orc_score(const OrcDia* d, const OrcLib* l, float mass_tolerance, int64_t top_k,
                       const uint64_t* precursor_idx, const uint64_t* rank, const float* score,
                       const uint64_t* cycle_center, const uint64_t* cycle_start,
                       const uint64_t* cycle_stop, int64_t n, int log_mode, int n_threads);
int64_t orc_features_len(const OrcFeatures* r);
void orc_features_copy(const OrcFeatures* r, uint64_t* precursor_idx, uint64_t* rank, float* feats);
void orc_features_free(OrcFeatures* r);

// PeakGroupQuantification.quantify (src/peak_group_quantification/mod.rs:49-168) into the
// SpecLibFlatQuantified layout (src/speclib_flat_quantified/mod.rs:212-333): precursor
// rows (stably sorted by precursor_idx) and fragment rows (candidate order), with the
// input rows of the library's precursor and fragment arrays for the pass-through columns.
typedef struct OrcQuant OrcQuant;
OrcQuant* orc_quantify(const OrcDia* d, const OrcLib* l, float tolerance_ppm, int64_t top_k,
                       const uint64_t* pidx, const uint64_t* rank, const uint64_t* center,
                       const uint64_t* start, const uint64_t* stop, int64_t n, int n_threads);
void orc_quant_sizes(const OrcQuant* r, int64_t* n_prec, int64_t* n_frag);
void orc_quant_copy(const OrcQuant* r, uint64_t* p_idx, uint64_t* p_row, uint64_t* p_rank,
                    float* p_rt_observed, uint64_t* p_start, uint64_t* p_stop, uint64_t* f_row,
                    float* f_intensity, float* f_mz_observed, float* f_correlation,
                    float* f_mass_error, uint64_t* f_pidx, uint64_t* f_rank);
void orc_quant_free(OrcQuant* r);
/* the scoring helpers, for the reference's unit-test values */
void orc_sc_normalize_profiles(const float* x, int64_t rows, int64_t cols, int64_t dil, float* out);
void orc_sc_median_axis0(const float* x, int64_t rows, int64_t cols, int non_zero_only, float* out);
float orc_sc_correlation(const float* x, const float* y, int64_t n);
float orc_sc_gamma_ln(float x, int log_mode);
float orc_sc_hyperscore(const uint8_t* type, const float* inten, const uint8_t* mask,
                        const float* weights, int64_t n, int log_mode);
void orc_sc_longest_ion_series(const uint8_t* type, const uint8_t* number, const uint8_t* mask,
                               int64_t n, uint8_t* longest_b, uint8_t* longest_y);
float orc_sc_intensity_ion_series(const uint8_t* type, const float* inten, const uint8_t* mask,
                                  int64_t n, uint8_t target);
float orc_sc_fwhm_rt(const float* profile, int64_t n, int64_t cycle_start, const float* rt);
void orc_sc_fragment_mz_errors(const float* dense_mz, const float* dense_xic, int64_t F, int64_t C,
                               const float* mz_library, float* mz_observed, float* mass_error);
float orc_sc_weighted_mae(const float* err, const float* weights, int64_t n);
float orc_sc_median(const float* v, int64_t n);
float orc_sc_std(const float* v, int64_t n);
void orc_sc_ranked_mask(const float* v, int64_t n, int64_t r1, int64_t r2, uint8_t* out);
int64_t orc_sc_count_above(const float* v, int64_t n, float threshold, const uint8_t* mask);
float orc_sc_dot(const float* a, const float* b, int64_t n);
void orc_sc_dense_xic_mz(const OrcDia* d, float precursor_mz, int64_t cycle_start,
                         int64_t cycle_stop, float mass_tolerance, const float* fragment_mz,
                         int64_t F, float* xic, float* mz);
void orc_sc_idf(const OrcDia* d, const OrcLib* l, const float* mz, int64_t n, int log_mode,
                float* out);

#ifdef __cplusplus
}
#endif
#endif
