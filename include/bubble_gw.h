/*
 * bubble_gw.h -- C ABI of the generalized bulk-flow many-bubble GW spectrum.
 *
 * Drop-in replacement for the bulk-flow subset of the reference crate
 * `c-bubble-gw` (rust/c-bubble-gw/src/lib.rs, header generated from
 * rust/c-bubble-gw/cbindgen.toml).  Same symbol names, argument meaning,
 * ownership and error behaviour; the computation runs on an sm_100a GPU.
 *
 * Conventions (rust/c-bubble-gw/README.md:36-44):
 *   - the library owns handles; arrays are caller-owned, C-contiguous,
 *     row-major; bubble arrays are (n, 4) with columns (t, x, y, z);
 *   - a zero-length array may be NULL;
 *   - every failure other than a NULL `out` in ..._new returns
 *     BGW_STATUS_CALCULATION_ERROR and sets a thread-local message readable
 *     with bgw_last_error_message();
 *   - NAN stands for "None" in optional f64 arguments.
 */
#pragma once
#ifndef BUBBLE_GW_H
#define BUBBLE_GW_H

#include <stdbool.h>
#include <stddef.h>

/* rust/c-bubble-gw/src/lib.rs:18-26 */
typedef enum BgwStatus {
    BGW_STATUS_OK = 0,
    BGW_STATUS_NULL_POINTER = 1,
    BGW_STATUS_INVALID_ARGUMENT = 2,
    BGW_STATUS_CALCULATION_ERROR = 3,
    BGW_STATUS_PANIC = 4,
} BgwStatus;

/* rust/c-bubble-gw/src/lib.rs:65-68 */
typedef enum BgwTimeCutoffKind {
    BGW_TIME_CUTOFF_KIND_UNIT = 0,
    BGW_TIME_CUTOFF_KIND_EXPONENTIAL = 1,
} BgwTimeCutoffKind;

/* rust/c-bubble-gw/src/lib.rs:70-77.  ratio_t_cut / ratio_t_0 = NAN -> defaults
 * 0.999999999 and 0.25 (rust/bubble-gw/src/time_cutoff.rs:22-30). */
typedef struct BgwTimeCutoffConfig {
    BgwTimeCutoffKind kind;
    double smax;
    double ratio_t_cut;
    double ratio_t_0;
} BgwTimeCutoffConfig;

/* rust/c-bubble-gw/src/lib.rs:79-84 */
typedef struct BgwComplex64 {
    double re;
    double im;
} BgwComplex64;

/* Opaque handle, rust/c-bubble-gw/src/lib.rs:91-94 */
typedef struct bgw_generalized_bulk_flow bgw_generalized_bulk_flow;

#ifdef __cplusplus
extern "C" {
#endif

/* Version string, NUL-terminated, static.  Replaces rust/c-bubble-gw/src/lib.rs:219-223. */
const char *bgw_version(void);

/* Thread-local message of the most recent failing call ("" after a success).
 * Replaces rust/c-bubble-gw/src/lib.rs:225-229 (interior NULs become spaces). */
const char *bgw_last_error_message(void);

/* Creates a calculator over an EmptyLattice: the caller passes any boundary
 * images as exterior bubbles.  Validates causality (no interior-interior or
 * interior-exterior pair with negative Minkowski interval).  *out is set to
 * NULL before any work; a NULL `out` returns BGW_STATUS_NULL_POINTER.
 * Replaces rust/c-bubble-gw/src/lib.rs:386-422. */
BgwStatus bgw_generalized_bulk_flow_empty_lattice_new(bgw_generalized_bulk_flow **out,
                                                      const double *bubbles_interior, size_t n_interior,
                                                      const double *bubbles_exterior, size_t n_exterior);

/* Frees a handle; NULL is allowed.  Replaces rust/c-bubble-gw/src/lib.rs:424-430. */
void bgw_generalized_bulk_flow_free(bgw_generalized_bulk_flow *bulk_flow);

/* Host threads used for host-side preparation; 0 is an error.
 * Replaces rust/c-bubble-gw/src/lib.rs:432-446. */
BgwStatus bgw_generalized_bulk_flow_set_num_threads(bgw_generalized_bulk_flow *bulk_flow, size_t num_threads);

/* Angular patch grid n_cos_thetax x n_phix (both >= 2).  With
 * precompute_first_bubbles the first-collider masks for k = z are computed
 * on the GPU at the first spectrum call and kept on the device.
 * Replaces rust/c-bubble-gw/src/lib.rs:448-461. */
BgwStatus bgw_generalized_bulk_flow_set_resolution(bgw_generalized_bulk_flow *bulk_flow, size_t n_cos_thetax,
                                                   size_t n_phix, bool precompute_first_bubbles);

/* Post-collision scaling f = sum_k a[s,k] (dt_c/dt)^p[s,k] * exp(-dt(1-r)/damping),
 * row-major (n_sets, n_terms); damping_width NAN = no damping.
 * Replaces rust/c-bubble-gw/src/lib.rs:463-494. */
BgwStatus bgw_generalized_bulk_flow_set_gradient_scaling_params(bgw_generalized_bulk_flow *bulk_flow,
                                                                const double *coefficients, const double *powers,
                                                                size_t n_sets, size_t n_terms,
                                                                double damping_width);

/* C_{+,x}(w) summed over `selected_bubbles` (NULL = all interior bubbles),
 * k-hat = z.  out: (2, n_sets, n_w) row-major, [0] = C_+, [1] = C_x;
 * out_len must equal 2*n_sets*n_w.  t_begin is used only if has_t_begin
 * (default 0).  Replaces rust/c-bubble-gw/src/lib.rs:526-574. */
BgwStatus bgw_generalized_bulk_flow_compute_c_integral(bgw_generalized_bulk_flow *bulk_flow, const double *w_arr,
                                                       size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                       size_t n_t, const size_t *selected_bubbles,
                                                       size_t n_selected_bubbles, BgwTimeCutoffConfig time_cutoff,
                                                       BgwComplex64 *out, size_t out_len);

#ifdef __cplusplus
}
#endif

#endif /* BUBBLE_GW_H */
