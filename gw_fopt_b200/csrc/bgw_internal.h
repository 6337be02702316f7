// Internal interfaces shared by the C ABI (capi.cpp), the lattice geometry
// (lattice.cpp) and the device pipeline (pipeline.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/bubble_gw.h"
#include "../../include/bubble_gw_b200.h"

namespace bgw {

// Raised inside the library; converted to BGW_STATUS_CALCULATION_ERROR plus
// the message by the C ABI wrapper (rust/c-bubble-gw/src/lib.rs:119-134).
struct Error {
    std::string msg;
    bool index_error = false;  // GeneralizedBulkFlowError::InvalidIndex
};

// Rust's `Display` for f64: shortest round-trip digits, positional notation,
// no trailing ".0" ("1", "0.5", "-0", "inf", "NaN").
std::string rust_f64(double x);

// Everything the device pipeline needs for one spectrum call.  Host arrays
// are owned by the caller of run_spectrum.
struct SpectrumJob {
    // bubbles: interior then exterior, (n_tot, 4) rows (t, x, y, z)
    const double* bubbles = nullptr;
    size_t n_int = 0, n_tot = 0;
    // angular grid (generalized_bulk_flow.rs:221-238): cos(theta) rows,
    // phi columns, direction table (n_cos*n_phi, 4) = (1, sx, sy, c)
    size_t n_cos = 0, n_phi = 0;
    const double* cos_thetax = nullptr;
    const double* dirs = nullptr;
    const double* sin2phi = nullptr;  // sin(2 phi_j)
    const double* cos2phi = nullptr;  // cos(2 phi_j)
    const double* sinphi = nullptr;   // sin(phi_j), cos(phi_j): the tensor form
    const double* cosphi = nullptr;
    bool tensor = false;              // NewGeneralizedBulkFlow: (6, S, W) per k-hat, FP64 direct only
    // scaling functions
    size_t n_sets = 0, n_terms = 0;
    const double* coeffs = nullptr;
    const double* powers = nullptr;
    bool has_damping = false;
    double damping = 0.0;
    // time grid
    size_t n_t = 0;
    const double* t_arr = nullptr;
    const double* cutoff = nullptr;  // cutoff weight at each t
    double dt = 0.0;
    // frequencies
    size_t n_w = 0;
    const double* w = nullptr;
    // radiating bubbles (interior indices, duplicates allowed)
    const uint32_t* sel = nullptr;
    size_t n_sel = 0;
    // k-hat rotations, (K, 9) row-major; nullptr = the unrotated frame (K = 1)
    const double* rot = nullptr;
    size_t n_k = 1;
    BgwxKernel kernel = BGWX_KERNEL_FP64_DIRECT;
    // launch shape; 0 = automatic (frames per launch from the memory budget,
    // row parts from the wave-fill model, 4 GEMM stages).  frames_per_launch is
    // capped by the budget; row_parts (at most 16) and gemm_stages (3 to 5)
    // apply to the tensor-core GEMM only.
    size_t frames_per_launch = 0;
    int row_parts = 0;
    int gemm_stages = 0;
    // mask search: the automatic number of blocks per (bubble, frame) times 1, 2 or 4 (0: 1);
    // finer direction ranges per block give shorter tails, coarser ones fewer list gathers
    int mask_chunking = 0;
    // keep every frame's collision delays and first-collider codes on the device (when they fit in
    // the mask budget) for a following adjoint call on the same bubbles, directions and grid
    bool keep_masks = false;
    // Several realizations in one call (the batched ensemble, factored kernels): `bubbles` holds
    // them one after another (n_tot rows in all; n_int = n_tot), `sel` has one slot per radiating
    // bubble, padded so that each realization starts a GEMM column tile (padding slots hold
    // kNoSlot), `ranges` (n_sel pairs) gives each slot's realization rows (first, count) and
    // `real_tiles` (n_real + 1) the first column tile of each realization.  The output is then
    // (n_real, n_k, 2, n_sets, n_w).
    const uint32_t* ranges = nullptr;
    const uint32_t* real_tiles = nullptr;
    size_t n_real = 0;
};

// A padding slot of a batched job.
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

// Radiating bubbles per GEMM column tile of a factored-kernel job (each batched
// realization starts a tile).
size_t factored_bubbles_per_tile(const SpectrumJob& job);

// The launch shape a spectrum call used (or is to use).
struct LaunchShape {
    size_t frames_per_launch = 0;
    int row_parts = 0;
    int gemm_stages = 0;
    int mask_chunking = 0;
};

struct MaskJob {
    const double* bubbles = nullptr;
    size_t n_int = 0, n_tot = 0;
    size_t n_cos = 0, n_phi = 0;
    const double* dirs = nullptr;
    const uint32_t* sel = nullptr;
    size_t n_sel = 0;
};

// Device state owned by one handle (one CUDA stream, grow-only buffers).
struct Device;
Device* device_create();  // throws Error when no CUDA device is usable
void device_destroy(Device*);

// Runs the spectrum; out: (n_k, 2, n_sets, n_w) complex as interleaved
// doubles.  With out_is_device the result is written to device memory and
// only the device's error counters are read back (timings are then not
// filled).  A call waits for its work and throws Error when a kernel reported
// a failed wait.  `nested` calls (the batched ensemble) neither clear nor read
// the error counters and return without synchronising: their caller does
// both once.
void run_spectrum(Device* dev, const SpectrumJob& job, double* out, bool out_is_device, BgwxTimings* timings,
                  bool nested = false, bool uploads_only = false);

// The launch shape of the last run_spectrum on this device (frames per launch
// and GEMM row parts actually used).
LaunchShape last_launch_shape(const Device* dev);

// Frames per launch that the memory budget allows for this job.
size_t spectrum_max_frames_per_launch(const SpectrumJob& job);

// Row parts the wave-fill model picks for kn frames per launch (1 unless the
// job runs the tensor-core GEMM).
int factored_auto_row_parts(const Device* dev, const SpectrumJob& job, size_t kn);

// Measured launch shape for a factored-kernel spectrum job: candidate frame
// counts per launch and GEMM row splits are timed on the device on a sample of
// the job's frames, once per (device, problem shape); the choice is kept for
// the process and, when the environment variable BGWX_AUTOTUNE_CACHE names a
// file, in that file.  The FP64 direct kernel has no tunable shape and gets
// the automatic one.  Throws Error.
LaunchShape autotune_launch_shape(Device* dev, const SpectrumJob& job);

// The spectra of R realizations that share every setting but their bubbles,
// into one device array copied out once; out: (R, n_k, 2, n_sets, n_w)
// complex as interleaved doubles.  On the factored kernels all realizations
// form one batched job (each pipeline launch covers every realization of its
// frames; the launch shape of jobs[0], or a measured one when `autotune`); the
// FP64 direct kernel runs one job per realization back to back.  Realizations
// with no radiating bubble yield zeros.
void run_ensemble(Device* dev, const std::vector<SpectrumJob>& jobs, double* out, BgwxTimings* timings,
                  bool autotune = false);

// Vector-Jacobian product of the spectrum: gbar (n_k, 2, n_sets, n_w)
// complex cotangents dL/dRe C + i dL/dIm C (interleaved doubles) ->
// g_par (coefficients then powers, 2 n_sets n_terms) and g_bub ((n_tot, 4),
// gradients with respect to every bubble row, exterior rows included).
void run_adjoint(Device* dev, const SpectrumJob& job, const double* gbar, double* g_par, double* g_bub,
                 BgwxTimings* timings);

// Time-resolved integrand of the unrotated frame (job.rot ignored): out
// (2, n_sets, n_w, n_t) complex as interleaved doubles, the sum over the
// selected bubbles in selection order; job.cutoff must be all ones (the
// reference applies no time cutoff to the integrand).
void run_integrand(Device* dev, const SpectrumJob& job, double* out, BgwxTimings* timings);

// Uses `stream` (a cudaStream_t) for all later work; nullptr = own stream.
void device_set_stream(Device* dev, void* stream);

// Marks every uploaded input as stale (the next call copies it again).
void device_drop_resident(Device* dev);

// First-collider codes and delays for the selected bubbles at the
// unrotated frame.  out_codes (n_sel, n_cos*n_phi) int32; out_tau may be null.
void run_masks(Device* dev, const MaskJob& job, int32_t* out_codes, double* out_tau, BgwxTimings* timings);

int device_count();

// Exponential-rate nucleation of R realizations on the GPU (nucleation.cu).
// interior (sum n, 4), exterior (6 sum n, 4), rows of realization r from the
// running sum of n; attempts (R): prefactor doublings used + 1, or -1.
void run_nucleation(const int64_t* n, const double* beta, const uint64_t* seed, size_t R, double L,
                    double gamma_scale, int64_t max_rejections, int max_attempts, double* interior,
                    double* exterior, int32_t* attempts);

// Energy spectrum per k-hat and its cos(theta_k) integral (postprocess.cu).
// c: (K, 2, S, W) complex128, on the device or the host; w (W), set weights
// (S) and x = sorted cos(theta_k) (K) on the host; spectra (K, W) may be null.
void run_power_spectrum(Device* dev, const void* c, bool c_on_device, size_t K, size_t S, size_t W,
                        const double* w, const double* a, const double* x_sorted, double* spectra, double* de,
                        bool out_on_device);

// Thread-local message of bgw_last_error_message (capi.cpp).
void set_last_error(std::string message);
void clear_last_error();

// Lattice geometry (lattice.cpp).
void lattice_contains(BgwxLatticeKind kind, const double* params, const double* pts, size_t n, uint8_t* out);
std::vector<double> lattice_exterior(BgwxLatticeKind kind, const double* params, BgwxBoundaryCondition bc,
                                     const double* interior, size_t n);
void check_causality(const double* interior, size_t n_int, const double* exterior, size_t n_ext);

// Host reference-arithmetic helpers (no FMA contraction in this library's
// host translation units: compiled with -ffp-contract=off).
std::vector<double> linspace(double a, double b, size_t n);
void rotation_for_khat(double kx, double ky, double kz, double* R);

}  // namespace bgw
