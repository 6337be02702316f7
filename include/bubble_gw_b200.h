/*
 * bubble_gw_b200.h -- extensions of the bubble_gw C ABI for the B200 build.
 *
 * Everything here is additive: the reference-compatible surface is
 * bubble_gw.h.  Each entry point names the reference interface it serves
 * (file:line in the reference tree) or says that it has no counterpart.
 * Status codes, error messages and array conventions are those of
 * bubble_gw.h.
 */
#pragma once
#ifndef BUBBLE_GW_B200_H
#define BUBBLE_GW_B200_H

#include "bubble_gw.h"

#include <stdint.h>

/* Lattice kinds (rust/bubble-gw/src/many_bubbles/lattice/built_in_lattice.rs:20).
 * Parameters (LatticeGeometry::parameters):
 *   PARALLELEPIPED / CARTESIAN: origin(3), e1(3), e2(3), e3(3)   (12 doubles)
 *   SPHERICAL: center(3), radius                                  (4 doubles)
 *   EMPTY: none                                                   (0 doubles) */
typedef enum BgwxLatticeKind {
    BGWX_LATTICE_PARALLELEPIPED = 0,
    BGWX_LATTICE_CARTESIAN = 1,
    BGWX_LATTICE_SPHERICAL = 2,
    BGWX_LATTICE_EMPTY = 3,
} BgwxLatticeKind;

/* rust/bubble-gw/src/many_bubbles/lattice/boundary_condition.rs:3 */
typedef enum BgwxBoundaryCondition {
    BGWX_BC_PERIODIC = 0,
    BGWX_BC_REFLECTION = 1,
    BGWX_BC_NONE = 2,
} BgwxBoundaryCondition;

/* Spectrum kernels.  FP64_DIRECT: plain FP64, one complex phase per
 * (bubble, cos-theta row, t, w), as the reference's loop nest.
 * FP64_FACTORED: FP64 with the time phase shared across bubbles (register
 * tiled).  MIXED: FP64 phases, tables and final sums; the time-phase product
 * runs on the tensor cores as an exact integer product of four int8 digits
 * per operand (relative error about 2^-32 of the operands' scales per term,
 * n_t at most 32767).  MIXED_SIMT: FP32 operands with the product on the FP32
 * CUDA cores and FP32 partial sums folded into FP64 every 16 steps. */
typedef enum BgwxKernel {
    BGWX_KERNEL_FP64_DIRECT = 0,
    BGWX_KERNEL_FP64_FACTORED = 1,
    BGWX_KERNEL_MIXED = 2,
    BGWX_KERNEL_MIXED_SIMT = 3,
} BgwxKernel;

/* Per-call device timings (milliseconds, CUDA events on the handle's stream). */
typedef struct BgwxTimings {
    double masks_ms;    /* first-collider search (all k-hat chunks) */
    double spectrum_ms; /* spectrum kernels (all k-hat chunks) */
    double total_ms;    /* whole device section of the last call */
    double h2d_bytes;   /* host->device bytes copied by the last call */
    double d2h_bytes;   /* device->host bytes copied by the last call */
    uint64_t launches;  /* kernels launched by the last call */
    uint64_t directions;/* patch directions searched by the mask kernel */
    uint64_t fallbacks; /* directions resolved by the exact slow path */
    double beta_ms;     /* factored kernels: beta producer */
    double gemm_ms;     /* factored kernels: time-phase GEMM and epilogue */
    uint64_t graph_replays; /* batched ensemble: 1 when the call replayed its captured CUDA graph */
} BgwxTimings;

#ifdef __cplusplus
extern "C" {
#endif

/* Lattice containment, one byte per point (1 = inside).  EMPTY reports
 * n_points = 0 semantics: out is left untouched and *n_out = 0.
 * Replaces LatticeGeometry::contains (parallelepiped_lattice.rs:161-186,
 * spherical_lattice.rs, empty_lattice.rs:31). */
BgwStatus bgwx_lattice_contains(BgwxLatticeKind kind, const double *params, const double *points_xyz,
                                size_t n_points, uint8_t *out, size_t *n_out);

/* Boundary images of interior bubbles: periodic = 6 face shifts, reflection
 * = 6 face mirrors (parallelepiped) or 2 tangent-plane mirrors (sphere).
 * Writes at most `capacity` rows of (t, x, y, z) and the row count to *n_out.
 * Replaces GenerateBubblesExterior (parallelepiped_lattice.rs:189-299,
 * spherical_lattice.rs:72-131, empty_lattice.rs:38-46). */
BgwStatus bgwx_lattice_exterior(BgwxLatticeKind kind, const double *params, BgwxBoundaryCondition bc,
                                const double *interior, size_t n_interior, double *out, size_t capacity,
                                size_t *n_out);

/* Causality check of LatticeBubbles::new (lattice_bubbles.rs:71-119): no
 * interior-interior or interior-exterior pair may have a negative interval. */
BgwStatus bgwx_check_causality(const double *interior, size_t n_interior, const double *exterior,
                               size_t n_exterior);

/* As bgw_generalized_bulk_flow_empty_lattice_new without the causality check:
 * the Python LatticeBubbles validates at construction and adds boundary
 * images afterwards without re-validating (lattice_bubbles.rs:323-365), and
 * GeneralizedBulkFlow::new (generalized_bulk_flow.rs:86-108) checks nothing. */
BgwStatus bgwx_generalized_bulk_flow_new_unchecked(bgw_generalized_bulk_flow **out, const double *interior,
                                                   size_t n_interior, const double *exterior, size_t n_exterior);

/* Selects the spectrum kernel used by every compute call on this handle.
 * No counterpart in the reference (it has one f64 CPU path). */
BgwStatus bgwx_generalized_bulk_flow_set_kernel(bgw_generalized_bulk_flow *bulk_flow, BgwxKernel kernel);

/* Launch shape of the spectrum calls on this handle (compute_c_integral and
 * the k-hat forms; not the ensemble or the adjoint): at most frames_per_launch
 * k-hat frames per launch (0 = as many as the memory budget allows) and
 * row_parts cos-theta row parts per tensor-core GEMM tile (0 = the wave-fill
 * model's choice; at most 16; the mixed kernel only).  A non-zero value here
 * takes precedence over autotuning.  The spectrum does not depend on the shape
 * beyond the order of FP64 partial sums.  No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_set_launch_shape(bgw_generalized_bulk_flow *bulk_flow, size_t frames_per_launch,
                                                      size_t row_parts);

/* Measured launch shapes: with enabled, the first spectrum call of each problem
 * shape (device, kernel, bubble counts, grids, coefficient sets) on a factored
 * kernel times candidate shapes around the automatic one on its own first
 * frames (frames per launch, GEMM row parts, then the mixed kernel's GEMM
 * stages) and keeps the fastest for the process; with the environment variable
 * BGWX_AUTOTUNE_CACHE naming a file, choices are also read from and appended
 * to it.  The FP64 direct kernel has no tunable shape.  Off by default.
 * No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_set_autotune(bgw_generalized_bulk_flow *bulk_flow, bool enabled);

/* The launch shape the last spectrum call on this handle used (frames per
 * launch, GEMM row parts; zeros before the first call).  No counterpart. */
BgwStatus bgwx_generalized_bulk_flow_last_launch_shape(const bgw_generalized_bulk_flow *bulk_flow,
                                                       size_t *out_frames_per_launch, size_t *out_row_parts);

/* Pipeline stages of 32 time steps in the mixed kernel's tensor-core GEMM:
 * 3, 4 or 5 (0 = automatic: 4, or the autotuner's measured choice).  The
 * stage count changes only the overlap of copies and MMAs, not the result.
 * No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_set_gemm_stages(bgw_generalized_bulk_flow *bulk_flow, size_t stages);

/* GEMM stages of the last spectrum call (0 when it did not run the mixed
 * kernel's GEMM).  No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_last_gemm_stages(const bgw_generalized_bulk_flow *bulk_flow, size_t *out_stages);

/* Chunking of the first-collider search: 1, 2 or 4 times the automatic number
 * of blocks per (radiating bubble, k-hat frame), each over a range of whole
 * cos-theta rows (0 = automatic: 1, or the autotuner's measured choice).  The
 * masks are the same for every choice.  No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_set_mask_chunking(bgw_generalized_bulk_flow *bulk_flow, size_t chunking);

/* Mask-search chunking of the last spectrum call.  No counterpart in the
 * reference. */
BgwStatus bgwx_generalized_bulk_flow_last_mask_chunking(const bgw_generalized_bulk_flow *bulk_flow,
                                                        size_t *out_chunking);

/* With `enabled`, each k-hat spectrum call keeps every frame's collision
 * delays and first-collider codes on the device (when they fit in a third of
 * the free device memory), and a following
 * bgwx_generalized_bulk_flow_spectrum_vjp on the same bubbles, selection,
 * directions and grid reads them instead of searching again.  The gradients
 * are the same bits either way.  No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_set_keep_masks(bgw_generalized_bulk_flow *bulk_flow, bool enabled);

/* First-collider codes (-1 None, i Interior(i), -(i+2) Exterior(i)) and the
 * collision delays of compute_delta_tab for interior bubbles [a_begin, a_end)
 * at k-hat = z, computed on the GPU.  out_codes: (a_end-a_begin, n_cos, n_phi)
 * int32; out_delta_tab (may be NULL): same shape, f64.
 * Replaces GeneralizedBulkFlow::compute_first_colliding_bubble and
 * compute_delta_tab (generalized_bulk_flow.rs:127-206, 421-471). */
BgwStatus bgwx_generalized_bulk_flow_first_colliding(bgw_generalized_bulk_flow *bulk_flow, size_t a_begin,
                                                     size_t a_end, int32_t *out_codes, double *out_delta_tab);

/* Spectrum for K directions k-hat (row-major (K, 3), unit vectors).  For each
 * k-hat the configuration is rotated by the Rodrigues rotation R(k) taking
 * k-hat to z (about k x z; identity for +z; pi about x for -z), and the
 * result equals bgw_generalized_bulk_flow_compute_c_integral on the rotated
 * configuration with the same `selected_bubbles` (NULL = all interior
 * bubbles).  out: (K, 2, n_sets, n_w); out_len = K*2*n_sets*n_w.
 * Serves the reference's per-direction recipe of rotating LatticeBubbles
 * (lattice_bubbles.rs:144-197) and recomputing (generalized_bulk_flow.rs:928-984). */
BgwStatus bgwx_generalized_bulk_flow_compute_c_integral_khat(
    bgw_generalized_bulk_flow *bulk_flow, const double *w_arr, size_t n_w, bool has_t_begin, double t_begin,
    double t_end, size_t n_t, const double *khat, size_t n_khat, const size_t *selected_bubbles,
    size_t n_selected_bubbles, BgwTimeCutoffConfig time_cutoff, BgwComplex64 *out, size_t out_len);

/* As bgwx_generalized_bulk_flow_compute_c_integral_khat with the result
 * written to device memory `out_device` ((K, 2, n_sets, n_w) complex128,
 * out_len elements) and the work left in flight on the handle's stream: the
 * call returns after enqueueing, inputs that did not change since the previous
 * call are not copied again (they stay resident in HBM).  No counterpart in
 * the reference. */
BgwStatus bgwx_generalized_bulk_flow_compute_c_integral_khat_device(
    bgw_generalized_bulk_flow *bulk_flow, const double *w_arr, size_t n_w, bool has_t_begin, double t_begin,
    double t_end, size_t n_t, const double *khat, size_t n_khat, const size_t *selected_bubbles,
    size_t n_selected_bubbles, BgwTimeCutoffConfig time_cutoff, void *out_device, size_t out_len);

/* Batched ensemble: the spectra of R independent nucleation realizations in
 * one call, each along the same K directions k-hat.  Realization r's bubbles
 * are rows interior_offsets[r] .. interior_offsets[r+1]-1 of `interior` and
 * rows exterior_offsets[r] .. exterior_offsets[r+1]-1 of `exterior` (both
 * (n, 4) row-major (t, x, y, z); offsets have R+1 non-decreasing entries
 * starting at 0).  Every interior bubble of a realization radiates.  The
 * resolution, gradient scaling parameters and kernel come from `bulk_flow`
 * (its own bubbles are not used).  With `validate` each realization passes
 * the causality check of bgw_generalized_bulk_flow_empty_lattice_new.
 * out: (R, K, 2, n_sets, n_w); out_len = R*K*2*n_sets*n_w.  Block r equals
 * bgwx_generalized_bulk_flow_compute_c_integral_khat on a handle holding
 * realization r, bit for bit.  Replaces a caller's loop that builds one
 * GeneralizedBulkFlow per realization and calls compute_c_integral on each
 * (generalized_bulk_flow.rs:928-984, used as in
 * docs/examples/generalized_bulkflow.py:679-703).  No counterpart in the
 * reference's C ABI. */
BgwStatus bgwx_generalized_bulk_flow_compute_ensemble_khat(
    bgw_generalized_bulk_flow *bulk_flow, const double *interior, const size_t *interior_offsets,
    const double *exterior, const size_t *exterior_offsets, size_t n_realizations, bool validate,
    const double *w_arr, size_t n_w, bool has_t_begin, double t_begin, double t_end, size_t n_t,
    const double *khat, size_t n_khat, BgwTimeCutoffConfig time_cutoff, BgwComplex64 *out, size_t out_len);

/* Adjoint (vector-Jacobian product) of the spectrum of every interior bubble
 * along K directions k-hat (n_khat = 0: the unrotated frame, K = 1).
 * grad_out: (K, 2, n_sets, n_w) cotangents dL/dRe C + i dL/dIm C of a real
 * loss L, grad_len = K*2*n_sets*n_w.  Writes dL/d(coefficients) and
 * dL/d(powers) ((n_sets, n_terms) each) and dL/d(bubbles) ((n_interior +
 * n_exterior, 4), columns (t, x, y, z); a caller whose exterior rows are
 * images of interior rows adds each image row's gradient to its source row).
 * FP64, except that with a mixed kernel selected the depth-n_w products of
 * the cotangents with the phases run in FP32, folded into FP64 every 16
 * frequencies; the first-collider search is recomputed, phases are
 * recomputed rather than stored.  Collision status and first-collider identity
 * are piecewise constant in the inputs and carry no gradient.  Differentiates
 * generalized_bulk_flow.rs:481-873 and the delays of :421-471.  No counterpart
 * in the reference. */
BgwStatus bgwx_generalized_bulk_flow_spectrum_vjp(bgw_generalized_bulk_flow *bulk_flow, const double *w_arr,
                                                  size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                  size_t n_t, const double *khat, size_t n_khat,
                                                  BgwTimeCutoffConfig time_cutoff, const BgwComplex64 *grad_out,
                                                  size_t grad_len, double *grad_coefficients, double *grad_powers,
                                                  double *grad_bubbles);

/* Replaces the handle's bubbles (no causality check, as
 * bgwx_generalized_bulk_flow_new_unchecked), keeping its settings and device
 * state: fitting loops move bubbles between calls.  No counterpart. */
BgwStatus bgwx_generalized_bulk_flow_set_bubbles(bgw_generalized_bulk_flow *bulk_flow, const double *interior,
                                                 size_t n_interior, const double *exterior, size_t n_exterior);

/* Time-resolved integrand of the spectrum: out (2, n_sets, n_w, n_t), the
 * sum over `selected_bubbles` (NULL = all interior bubbles; an empty selection
 * gives zeros) of each bubble's A_{+,x}(w, t) e^{i w (t - z_a)} times the
 * trapezoid dt weight and 1/(6 pi), zero at steps t <= t_a; no time cutoff.
 * Summing over the last axis gives compute_c_integral without cutoff.
 * Errors as the reference: n_t < 2, then an index out of range, then (for a
 * bubble with t_a < t_end) t_begin > t_end.  Replaces
 * GeneralizedBulkFlow::compute_c_integrand and, with a one-bubble selection,
 * compute_c_integrand_fixed_bubble (generalized_bulk_flow.rs:776-920). */
BgwStatus bgwx_generalized_bulk_flow_compute_c_integrand(bgw_generalized_bulk_flow *bulk_flow, const double *w_arr,
                                                         size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                         size_t n_t, const size_t *selected_bubbles,
                                                         size_t n_selected_bubbles, BgwComplex64 *out,
                                                         size_t out_len);

/* The tensor form of the reference's NewGeneralizedBulkFlow::compute_c_tensor
 * (rust/bubble-gw/src/many_bubbles/new_generalized_bulk_flow.rs:1205-1275,
 * Python rust/py-bubble-gw/src/py_many_bubbles/py_new_generalized_bulk_flow.rs:265-313):
 * C_ij(w) = 1/(6 pi) sum_n int dt e^{i w (t - z_n)} A_n,ij with the phi
 * integral of x_i x_j (t - t_n)^3 f in six components, out (K, 6, S, W) in the
 * order xx, xy, xz, yy, yz, zz, for each k-hat row of `khat` (its rotated
 * configuration, the convention of ..._compute_c_integral_khat) or, with
 * khat NULL, the configuration as given (K = 1, the reference's call).  No
 * time cutoff (the tensor form has none); plain FP64 (the direct kernel) for
 * every kernel selection.  The handle's bubbles, resolution and scaling
 * parameters are those of the scalar form. */
BgwStatus bgwx_generalized_bulk_flow_compute_c_tensor_khat(bgw_generalized_bulk_flow *bulk_flow, const double *w_arr,
                                                          size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                          size_t n_t, const double *khat, size_t n_khat,
                                                          const size_t *selected_bubbles, size_t n_selected_bubbles,
                                                          BgwComplex64 *out, size_t out_len);

/* The time-resolved tensor integrand (the reference's
 * NewGeneralizedBulkFlow::compute_c_tensor_integrand,
 * new_generalized_bulk_flow.rs:832-1065): out (6, S, W, n_t), each step's
 * A_ij e^{i w (t - z_a)} (trapezoid dt weight) / (6 pi) summed over the
 * selected bubbles (NULL = all); plain FP64, unrotated configuration. */
BgwStatus bgwx_generalized_bulk_flow_compute_c_tensor_integrand(bgw_generalized_bulk_flow *bulk_flow,
                                                                const double *w_arr, size_t n_w, bool has_t_begin,
                                                                double t_begin, double t_end, size_t n_t,
                                                                const size_t *selected_bubbles,
                                                                size_t n_selected_bubbles, BgwComplex64 *out,
                                                                size_t out_len);

/* Draws the bubbles of n_realizations nucleation Monte Carlo realizations on
 * the GPU (one block per realization): exponential-rate nucleation in a
 * periodic cube of side box_side, candidates arriving as a Poisson process
 * with rate Gamma0 V e^{beta t} (Gamma0 V / beta = gamma_scale n), rejected
 * inside an accepted bubble's wall at the nearest periodic copy, the rejection
 * against bubbles and images of the reference's
 * rust/bubble-gw/src/many_bubbles/bubbles_nucleation/fixed_rate_nucleation.rs;
 * after max_rejections rejections the prefactor doubles and the draw restarts
 * (at most 40 times).  Random numbers: Philox4x32-10 keyed by seeds[r].
 * interior: (sum n, 4) rows [t, x, y, z], times relative to each realization's
 * first bubble; exterior: (6 sum n, 4), the +x, -x, +y, -y, +z, -z images of
 * every bubble; attempts (n_realizations, may be NULL): prefactor attempts
 * used.  The ensemble sampler of the benchmark configurations, moved to the
 * device; no counterpart in the reference's C ABI. */
BgwStatus bgwx_nucleate_exponential(const int64_t *n_bubbles, const double *beta, const uint64_t *seeds,
                                    size_t n_realizations, double box_side, double gamma_scale,
                                    size_t max_rejections, double *interior, size_t interior_len, double *exterior,
                                    size_t exterior_len, int32_t *attempts);

/* Energy spectrum of bulk-flow output, the post-processing the reference's
 * consumer applies to compute_c_integral results
 * (src/gw_fopt/bubble_dynamics/utils/data_gw_bulkflow.py:26-146,
 * DataGwBulkFlow.de_dlogw_dcosthetak and de_dlogw), on this handle's GPU:
 *   C_+/x(w) = sum_s set_weights[s] C_{+/x,s}(w)          (sets with weight 0 are skipped)
 *   spectra[k, w] = 8 pi w^3 (|C_+|^2 + |C_x|^2)           per k-hat direction k
 *   de_dlogw[w]   = 2 trapezoid(spectra[:, w], x = sorted(cos_thetak))
 * The rows enter the trapezoid in the order given (the reference sorts only x).
 * c: (n_khat, 2, n_sets, n_w) complex128 (the layout of
 * bgwx_generalized_bulk_flow_compute_c_integral_khat); spectra: (n_khat, n_w)
 * or NULL; de_dlogw: (n_w).  Host pointers.  Errors: CalculationError. */
BgwStatus bgwx_generalized_bulk_flow_power_spectrum(bgw_generalized_bulk_flow *bulk_flow, const BgwComplex64 *c,
                                                    size_t n_khat, size_t n_sets, const double *w_arr, size_t n_w,
                                                    const double *set_weights, const double *cos_thetak,
                                                    double *spectra, double *de_dlogw);

/* The same with c, spectra and de_dlogw in device memory (for example the
 * output of bgwx_generalized_bulk_flow_compute_c_integral_khat_device), so the
 * spectrum never leaves the GPU; w_arr, set_weights and cos_thetak are host
 * arrays.  Runs on the handle's stream and returns when the results are
 * written.  No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_power_spectrum_device(bgw_generalized_bulk_flow *bulk_flow,
                                                           const void *c_device, size_t n_khat, size_t n_sets,
                                                           const double *w_arr, size_t n_w,
                                                           const double *set_weights, const double *cos_thetak,
                                                           void *spectra_device, void *de_dlogw_device);

/* Runs this handle's device work on `stream` (a cudaStream_t created by the
 * caller; NULL selects the handle's own non-blocking stream, so the legacy
 * default stream cannot be chosen).  No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_set_stream(bgw_generalized_bulk_flow *bulk_flow, void *stream);

/* Forgets which inputs are resident on the device, so that the next call
 * copies every input from the host again (used to measure end-to-end cost).
 * No counterpart in the reference. */
BgwStatus bgwx_generalized_bulk_flow_drop_resident_inputs(bgw_generalized_bulk_flow *bulk_flow);

/* Measured device throughput of FP64 FMA (flop/s), FP32 FMA (flop/s) and the
 * SFU (sin/cos operations/s), the peaks of the spectrum kernels' roofline.
 * No counterpart in the reference. */
BgwStatus bgwx_measure_compute_peaks(double *fp64_flops, double *fp32_flops, double *sfu_ops);

/* First-collider codes and collision delays, as bgwx_generalized_bulk_flow_first_colliding
 * returns them, for callers that cannot allocate device memory: frameworks that
 * serve all device memory from their own pool and long-running services that
 * must not allocate after start-up.  Everything is caller-owned device memory:
 *   d_bubbles   (n_total, 4) rows (t, x, y, z), interior rows first;
 *   d_selected  (n_selected) uint32 interior indices, n_selected <= 512 (an index
 *               >= n_interior yields codes INT32_MIN and delays NaN for that row);
 *   d_dirs      (n_dirs, 4) patch directions (1, s cos(phi), s sin(phi), c) with
 *               c = -1 + i*(2/(n_cos-1)), s = |sqrt(1 - c*c)|, phi = j*(2 pi/(n_phi-1)),
 *               row i*n_phi + j, sin/cos from the C library;
 *   d_codes     (n_selected, n_dirs) int32 out: -1 None, i Interior(i), -(i+2) Exterior(i);
 *   d_delta_tab (n_selected, n_dirs) f64 out.
 * The work runs on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * is left in flight.  The library's only work array, the per-bubble candidate
 * lists, is a fixed static device array of 512 entries (about 3.2 MB on every
 * GPU that loads the library, until exit); more than 512 selected bubbles is
 * rejected with an error.  The first call on each device looks up that array's
 * device address, so make the first call before any stream capture.  All calls
 * share the array: calls whose work overlaps on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.
 * No counterpart in the reference. */
BgwStatus bgwx_first_colliding_noalloc(const double *d_bubbles, size_t n_interior, size_t n_total,
                                       const uint32_t *d_selected, size_t n_selected, const double *d_dirs,
                                       size_t n_dirs, int32_t *d_codes, double *d_delta_tab, void *stream);

/* The rotation R(k) used above, row-major 3x3.  No counterpart in the reference. */
void bgwx_rotation_for_khat(double kx, double ky, double kz, double *R);

/* Device timings of the last compute call on this handle.  No counterpart. */
BgwStatus bgwx_generalized_bulk_flow_last_timings(const bgw_generalized_bulk_flow *bulk_flow, BgwxTimings *out);

/* Number of CUDA devices visible (0 on a machine without a GPU).  No counterpart. */
int bgwx_device_count(void);

#ifdef __cplusplus
}
#endif

#endif /* BUBBLE_GW_B200_H */
