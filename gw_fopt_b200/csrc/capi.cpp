// The C ABI: reference-compatible bgw_* entry points (rust/c-bubble-gw/src/lib.rs)
// and the bgwx_* extensions.  Host-side validation and grids live here; all
// numerical work on the path runs on the GPU (pipeline.cu).  There is no CPU
// fallback: without a usable CUDA device the compute calls fail with
// BGW_STATUS_CALCULATION_ERROR.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "bgw_internal.h"

#define BGW_VERSION_STRING "0.1.0+b200"

using bgw::Error;

// Opaque handle (rust/c-bubble-gw/src/lib.rs:100-102 holds a
// GeneralizedBulkFlow<EmptyLattice>; generalized_bulk_flow.rs:65-80).
struct bgw_generalized_bulk_flow {
    std::vector<double> bubbles;  // interior rows then exterior rows, (n, 4)
    size_t n_int = 0, n_ext = 0;
    bool has_res = false;
    bool precompute = false;
    size_t n_cos = 0, n_phi = 0;
    std::vector<double> cos_thetax, phix, dirs, sin2phi, cos2phi, sinphi, cosphi;
    // generalized_bulk_flow.rs:98-99 defaults: coefficients [[1.0]], powers [[3.0]]
    size_t n_sets = 1, n_terms = 1;
    std::vector<double> coeffs{1.0}, powers{3.0};
    bool has_damping = false;
    double damping = 0.0;
    size_t num_threads = 1;
    BgwxKernel kernel = BGWX_KERNEL_FP64_DIRECT;
    // launch shape of spectrum calls: fixed (non-zero), measured (autotune) or automatic
    size_t frames_per_launch = 0, row_parts = 0, gemm_stages = 0, mask_chunking = 0;
    bool autotune = false;
    bool keep_masks = false;  // spectrum calls keep their masks for a following adjoint call
    bgw::Device* dev = nullptr;
    BgwxTimings timings{};
    ~bgw_generalized_bulk_flow() {
        if (dev) bgw::device_destroy(dev);
    }
};

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace bgw {
void set_last_error(std::string m) {
    for (auto& ch : m)
        if (ch == '\0') ch = ' ';
    g_last_error = std::move(m);
}
void clear_last_error() { g_last_error.clear(); }
}  // namespace bgw

namespace {
using bgw::set_last_error;

// rust/c-bubble-gw/src/lib.rs:119-134: Ok -> clear; Err -> CalculationError.
template <class F>
BgwStatus run_ffi(F&& f) {
    try {
        f();
        g_last_error.clear();
        return BGW_STATUS_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return BGW_STATUS_CALCULATION_ERROR;
    } catch (const std::bad_alloc&) {
        set_last_error("memory allocation failed");
        return BGW_STATUS_CALCULATION_ERROR;
    } catch (const std::exception& e) {
        set_last_error(std::string("internal error crossed the C ABI boundary: ") + e.what());
        return BGW_STATUS_PANIC;
    } catch (...) {
        set_last_error("internal error crossed the C ABI boundary");
        return BGW_STATUS_PANIC;
    }
}

// rust/c-bubble-gw/src/lib.rs:140-148: a zero-length slice may be NULL.
template <class T>
const T* slice(const T* p, size_t len, const char* name) {
    if (len == 0) return nullptr;
    if (!p) throw Error{std::string(name) + " must not be null"};
    return p;
}

size_t checked_mul(size_t a, size_t b, const char* name) {
    if (a != 0 && b > (size_t)-1 / a) throw Error{std::string(name) + " length overflow"};
    return a * b;
}

bgw_generalized_bulk_flow* handle(bgw_generalized_bulk_flow* h) {
    if (!h) throw Error{"bulk_flow must not be null"};
    return h;
}

bgw_generalized_bulk_flow* make_handle(const double* interior, size_t n_int, const double* exterior, size_t n_ext,
                                       bool validate) {
    size_t li = checked_mul(n_int, 4, "interior bubbles");
    size_t le = checked_mul(n_ext, 4, "exterior bubbles");
    const double* pi = slice(interior, li, "bubbles_interior");
    const double* pe = slice(exterior, le, "bubbles_exterior");
    if (validate) bgw::check_causality(pi, n_int, pe, n_ext);
    auto* h = new bgw_generalized_bulk_flow();
    h->bubbles.resize(li + le);
    if (li) std::memcpy(h->bubbles.data(), pi, li * sizeof(double));
    if (le) std::memcpy(h->bubbles.data() + li, pe, le * sizeof(double));
    h->n_int = n_int;
    h->n_ext = n_ext;
    return h;
}

void require_resolution(const bgw_generalized_bulk_flow* h) {
    if (!h->has_res) throw Error{"Field 'n_cos_thetax' is not initialized"};
}

bgw::Device* device(bgw_generalized_bulk_flow* h) {
    if (!h->dev) h->dev = bgw::device_create();
    return h->dev;
}

// time_cutoff.rs:15-43.
struct Cutoff {
    bool exponential = false;
    double t_cut = 0, inv_t_0_sq = 0;
    double eval(double t) const {
        if (!exponential || t < t_cut) return 1.0;
        double d = t - t_cut;
        return std::exp(-(d * d) * inv_t_0_sq);
    }
};

Cutoff make_cutoff(const BgwTimeCutoffConfig& c) {
    Cutoff k;
    if (c.kind == BGW_TIME_CUTOFF_KIND_UNIT) return k;
    if (c.kind != BGW_TIME_CUTOFF_KIND_EXPONENTIAL) throw Error{"invalid time cutoff kind"};
    double rc = std::isnan(c.ratio_t_cut) ? 0.999999999 : c.ratio_t_cut;
    double r0 = std::isnan(c.ratio_t_0) ? 0.25 : c.ratio_t_0;
    k.exponential = true;
    k.t_cut = rc * c.smax;
    double t0 = r0 * (c.smax - k.t_cut);
    k.inv_t_0_sq = 1.0 / (t0 * t0);
    return k;
}

// The parts of a spectrum job that come from the handle's settings and the
// call's grids (everything except the bubbles and the radiating selection).
bgw::SpectrumJob settings_job(const bgw_generalized_bulk_flow* h, const std::vector<double>& t_arr,
                              const std::vector<double>& cw, const double* w, size_t n_w, const double* rot,
                              size_t n_k) {
    bgw::SpectrumJob job;
    job.n_cos = h->n_cos;
    job.n_phi = h->n_phi;
    job.cos_thetax = h->cos_thetax.data();
    job.dirs = h->dirs.data();
    job.sin2phi = h->sin2phi.data();
    job.cos2phi = h->cos2phi.data();
    job.sinphi = h->sinphi.data();
    job.cosphi = h->cosphi.data();
    job.n_sets = h->n_sets;
    job.n_terms = h->n_terms;
    job.coeffs = h->coeffs.data();
    job.powers = h->powers.data();
    job.has_damping = h->has_damping;
    job.damping = h->damping;
    job.n_t = t_arr.size();
    job.t_arr = t_arr.data();
    job.cutoff = cw.data();
    job.dt = t_arr[1] - t_arr[0];
    job.n_w = n_w;
    job.w = w;
    job.rot = rot;
    job.n_k = n_k;
    job.kernel = h->kernel;
    job.keep_masks = h->keep_masks;
    return job;
}

// The handle's launch shape into a spectrum job: a fixed shape when one is
// set, else the measured one when autotuning is on, else automatic.
void apply_launch_shape(bgw_generalized_bulk_flow* h, bgw::SpectrumJob& job) {
    if (h->frames_per_launch || h->row_parts || h->gemm_stages || h->mask_chunking) {
        job.frames_per_launch = h->frames_per_launch;
        job.row_parts = (int)h->row_parts;
        job.gemm_stages = (int)h->gemm_stages;
        job.mask_chunking = (int)h->mask_chunking;
    } else if (h->autotune) {
        const bgw::LaunchShape s = bgw::autotune_launch_shape(device(h), job);
        job.frames_per_launch = s.frames_per_launch;
        job.row_parts = s.row_parts;
        job.gemm_stages = s.gemm_stages;
        job.mask_chunking = s.mask_chunking;
    }
}

// Rotations R(k) of the (n_khat, 3) unit rows.
std::vector<double> khat_rotations(const double* khat, size_t n_khat) {
    const double* k = slice(khat, checked_mul(n_khat, 3, "khat"), "khat");
    std::vector<double> rot(9 * n_khat);
    for (size_t q = 0; q < n_khat; ++q) {
        double kx = k[3 * q], ky = k[3 * q + 1], kz = k[3 * q + 2];
        double n2 = kx * kx + ky * ky + kz * kz;
        if (!(std::fabs(n2 - 1.0) <= 1e-9)) throw Error{"khat rows must be unit vectors"};
        bgw::rotation_for_khat(kx, ky, kz, &rot[9 * q]);
    }
    return rot;
}

// Shared body of compute_c_integral (generalized_bulk_flow.rs:928-984) for
// n_k frames; rot == nullptr means the unrotated frame.
void compute_common(bgw_generalized_bulk_flow* h, const double* w_arr, size_t n_w, bool has_t_begin, double t_begin,
                    double t_end, size_t n_t, const size_t* selected, size_t n_selected, bool has_selected,
                    const BgwTimeCutoffConfig& cutoff, const double* rot, size_t n_k, BgwComplex64* out,
                    size_t out_len, void* out_device = nullptr) {
    const double* w = slice(w_arr, n_w, "w_arr");
    Cutoff cut = make_cutoff(cutoff);
    size_t S = h->n_sets;
    size_t expected = checked_mul(checked_mul(checked_mul(n_k, 2, "out"), S, "out"), n_w, "out");
    if (n_t < 2) throw Error{"Invalid resolution: n_t must be >= 2 for integration"};
    std::vector<uint32_t> ids;
    if (has_selected) {
        const size_t* sel = slice(selected, n_selected, "selected_bubbles");
        for (size_t q = 0; q < n_selected; ++q) {
            if (sel[q] >= h->n_int) {
                Error e{"Index " + std::to_string(sel[q]) + " out of bounds for max " + std::to_string(h->n_int)};
                e.index_error = true;
                throw e;
            }
            ids.push_back((uint32_t)sel[q]);
        }
    } else {
        for (size_t a = 0; a < h->n_int; ++a) ids.push_back((uint32_t)a);
    }
    if (out_device && out_len != expected)
        throw Error{"out_len=" + std::to_string(out_len) + " does not match expected length " +
                    std::to_string(expected)};
    std::vector<double> result(out_device ? 0 : 2 * expected, 0.0);
    h->timings = BgwxTimings{};
    bool device_written = false;
    if (!ids.empty()) {
        double tb = has_t_begin ? t_begin : 0.0;
        if (tb > t_end)
            throw Error{"Invalid time range: t_begin=" + bgw::rust_f64(tb) + " > t_end=" + bgw::rust_f64(t_end)};
        require_resolution(h);
        if (S > 0 && n_w > 0) {
            std::vector<double> t_arr = bgw::linspace(tb, t_end, n_t);
            std::vector<double> cw(n_t);
            for (size_t k = 0; k < n_t; ++k) cw[k] = cut.eval(t_arr[k]);
            bgw::SpectrumJob job = settings_job(h, t_arr, cw, w, n_w, rot, n_k);
            job.bubbles = h->bubbles.data();
            job.n_int = h->n_int;
            job.n_tot = h->n_int + h->n_ext;
            job.sel = ids.data();
            job.n_sel = ids.size();
            apply_launch_shape(h, job);
            if (out_device) {
                bgw::run_spectrum(device(h), job, static_cast<double*>(out_device), true, &h->timings);
                device_written = true;
            } else {
                bgw::run_spectrum(device(h), job, result.data(), false, &h->timings);
            }
        }
    }
    if (out_device) {
        if (!device_written && expected)
            throw Error{"nothing to compute for a device output (empty selection, n_sets or n_w)"};
        return;
    }
    if (out_len != expected)
        throw Error{"out_len=" + std::to_string(out_len) + " does not match expected length " +
                    std::to_string(expected)};
    BgwComplex64* o = const_cast<BgwComplex64*>(slice(out, out_len, "out"));
    for (size_t q = 0; q < expected; ++q) o[q] = BgwComplex64{result[2 * q], result[2 * q + 1]};
}

}  // namespace

extern "C" {

const char* bgw_version(void) { return BGW_VERSION_STRING; }

const char* bgw_last_error_message(void) { return g_last_error.c_str(); }

BgwStatus bgw_generalized_bulk_flow_empty_lattice_new(bgw_generalized_bulk_flow** out, const double* bubbles_interior,
                                                      size_t n_interior, const double* bubbles_exterior,
                                                      size_t n_exterior) {
    if (!out) {
        set_last_error("out must not be null");
        return BGW_STATUS_NULL_POINTER;
    }
    *out = nullptr;
    return run_ffi([&] { *out = make_handle(bubbles_interior, n_interior, bubbles_exterior, n_exterior, true); });
}

BgwStatus bgwx_generalized_bulk_flow_new_unchecked(bgw_generalized_bulk_flow** out, const double* interior,
                                                   size_t n_interior, const double* exterior, size_t n_exterior) {
    if (!out) {
        set_last_error("out must not be null");
        return BGW_STATUS_NULL_POINTER;
    }
    *out = nullptr;
    return run_ffi([&] { *out = make_handle(interior, n_interior, exterior, n_exterior, false); });
}

void bgw_generalized_bulk_flow_free(bgw_generalized_bulk_flow* bulk_flow) { delete bulk_flow; }

BgwStatus bgw_generalized_bulk_flow_set_num_threads(bgw_generalized_bulk_flow* bulk_flow, size_t num_threads) {
    return run_ffi([&] {
        if (num_threads == 0) throw Error{"num_threads must be > 0"};
        handle(bulk_flow)->num_threads = num_threads;
    });
}

// generalized_bulk_flow.rs:208-270.  The direction table uses glibc sin/cos
// on the host so that it is bitwise the reference's.
BgwStatus bgw_generalized_bulk_flow_set_resolution(bgw_generalized_bulk_flow* bulk_flow, size_t n_cos_thetax,
                                                   size_t n_phix, bool precompute_first_bubbles) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (n_cos_thetax < 2 || n_phix < 2)
            throw Error{"Invalid resolution: Angular resolutions must be greater than one"};
        h->n_cos = n_cos_thetax;
        h->n_phi = n_phix;
        h->cos_thetax = bgw::linspace(-1.0, 1.0, n_cos_thetax);
        h->phix = bgw::linspace(0.0, 2.0 * M_PI, n_phix);
        h->dirs.assign(4 * n_cos_thetax * n_phix, 0.0);
        for (size_t i = 0; i < n_cos_thetax; ++i) {
            double c = h->cos_thetax[i];
            double s = std::fabs(std::sqrt(1.0 - c * c));
            for (size_t j = 0; j < n_phix; ++j) {
                double phi = h->phix[j];
                double sp = std::sin(phi), cp = std::cos(phi);
                double* d = &h->dirs[4 * (i * n_phix + j)];
                d[0] = 1.0;
                d[1] = s * cp;
                d[2] = s * sp;
                d[3] = c;
            }
        }
        h->sin2phi.resize(n_phix);
        h->cos2phi.resize(n_phix);
        h->sinphi.resize(n_phix);
        h->cosphi.resize(n_phix);
        for (size_t j = 0; j < n_phix; ++j) {  // new_generalized_bulk_flow.rs:640-644
            h->sinphi[j] = std::sin(h->phix[j]);
            h->cosphi[j] = std::cos(h->phix[j]);
        }
        for (size_t j = 0; j < n_phix; ++j) {
            h->sin2phi[j] = std::sin(2.0 * h->phix[j]);
            h->cos2phi[j] = std::cos(2.0 * h->phix[j]);
        }
        h->precompute = precompute_first_bubbles;
        h->has_res = true;
    });
}

BgwStatus bgw_generalized_bulk_flow_set_gradient_scaling_params(bgw_generalized_bulk_flow* bulk_flow,
                                                                const double* coefficients, const double* powers,
                                                                size_t n_sets, size_t n_terms,
                                                                double damping_width) {
    // rust/c-bubble-gw/src/lib.rs:465-494: chunks(n_terms) panics for n_terms == 0.
    if (n_terms == 0) {
        set_last_error("internal error crossed the C ABI boundary: chunk size must be non-zero");
        return BGW_STATUS_PANIC;
    }
    return run_ffi([&] {
        size_t len = checked_mul(n_sets, n_terms, "gradient scaling");
        const double* c = slice(coefficients, len, "coefficients");
        const double* p = slice(powers, len, "powers");
        auto* h = handle(bulk_flow);
        h->n_sets = n_sets;
        h->n_terms = n_sets ? n_terms : 0;
        h->coeffs.assign(c, c + len);
        h->powers.assign(p, p + len);
        h->has_damping = !std::isnan(damping_width);
        h->damping = damping_width;
    });
}

BgwStatus bgw_generalized_bulk_flow_compute_c_integral(bgw_generalized_bulk_flow* bulk_flow, const double* w_arr,
                                                       size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                       size_t n_t, const size_t* selected_bubbles,
                                                       size_t n_selected_bubbles, BgwTimeCutoffConfig time_cutoff,
                                                       BgwComplex64* out, size_t out_len) {
    return run_ffi([&] {
        compute_common(handle(bulk_flow), w_arr, n_w, has_t_begin, t_begin, t_end, n_t, selected_bubbles,
                       n_selected_bubbles, selected_bubbles != nullptr, time_cutoff, nullptr, 1, out, out_len);
    });
}

BgwStatus bgwx_generalized_bulk_flow_compute_c_integral_khat(bgw_generalized_bulk_flow* bulk_flow,
                                                             const double* w_arr, size_t n_w, bool has_t_begin,
                                                             double t_begin, double t_end, size_t n_t,
                                                             const double* khat, size_t n_khat,
                                                             const size_t* selected_bubbles,
                                                             size_t n_selected_bubbles,
                                                             BgwTimeCutoffConfig time_cutoff, BgwComplex64* out,
                                                             size_t out_len) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        std::vector<double> rot = khat_rotations(khat, n_khat);
        if (n_khat == 0) {
            if (out_len != 0)
                throw Error{"out_len=" + std::to_string(out_len) + " does not match expected length 0"};
            return;
        }
        compute_common(h, w_arr, n_w, has_t_begin, t_begin, t_end, n_t, selected_bubbles, n_selected_bubbles,
                       selected_bubbles != nullptr, time_cutoff, rot.data(), n_khat, out, out_len);
    });
}

BgwStatus bgwx_generalized_bulk_flow_compute_c_integral_khat_device(
    bgw_generalized_bulk_flow* bulk_flow, const double* w_arr, size_t n_w, bool has_t_begin, double t_begin,
    double t_end, size_t n_t, const double* khat, size_t n_khat, const size_t* selected_bubbles,
    size_t n_selected_bubbles, BgwTimeCutoffConfig time_cutoff, void* out_device, size_t out_len) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (!out_device) throw Error{"out_device must not be null"};
        if (n_khat == 0) throw Error{"khat must hold at least one direction"};
        std::vector<double> rot = khat_rotations(khat, n_khat);
        compute_common(h, w_arr, n_w, has_t_begin, t_begin, t_end, n_t, selected_bubbles, n_selected_bubbles,
                       selected_bubbles != nullptr, time_cutoff, rot.data(), n_khat, nullptr, out_len, out_device);
    });
}

BgwStatus bgwx_generalized_bulk_flow_compute_ensemble_khat(
    bgw_generalized_bulk_flow* bulk_flow, const double* interior, const size_t* interior_offsets,
    const double* exterior, const size_t* exterior_offsets, size_t n_realizations, bool validate,
    const double* w_arr, size_t n_w, bool has_t_begin, double t_begin, double t_end, size_t n_t,
    const double* khat, size_t n_khat, BgwTimeCutoffConfig time_cutoff, BgwComplex64* out, size_t out_len) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        const size_t R = n_realizations;
        const size_t S = h->n_sets;
        const size_t per_r = checked_mul(checked_mul(checked_mul(n_khat, 2, "out"), S, "out"), n_w, "out");
        const size_t expected = checked_mul(R, per_r, "out");
        if (out_len != expected)
            throw Error{"out_len=" + std::to_string(out_len) + " does not match expected length " +
                        std::to_string(expected)};
        if (expected == 0) return;
        const size_t* io = slice(interior_offsets, R + 1, "interior_offsets");
        const size_t* eo = slice(exterior_offsets, R + 1, "exterior_offsets");
        if (io[0] != 0 || eo[0] != 0) throw Error{"offsets must start at 0"};
        for (size_t r = 0; r < R; ++r)
            if (io[r + 1] < io[r] || eo[r + 1] < eo[r]) throw Error{"offsets must be non-decreasing"};
        const double* pi = slice(interior, checked_mul(io[R], 4, "interior bubbles"), "interior");
        const double* pe = slice(exterior, checked_mul(eo[R], 4, "exterior bubbles"), "exterior");
        if (n_t < 2) throw Error{"Invalid resolution: n_t must be >= 2 for integration"};
        const double tb = has_t_begin ? t_begin : 0.0;
        if (tb > t_end)
            throw Error{"Invalid time range: t_begin=" + bgw::rust_f64(tb) + " > t_end=" + bgw::rust_f64(t_end)};
        require_resolution(h);
        std::vector<double> rot = khat_rotations(khat, n_khat);
        const double* w = slice(w_arr, n_w, "w_arr");
        Cutoff cut = make_cutoff(time_cutoff);
        std::vector<double> t_arr = bgw::linspace(tb, t_end, n_t);
        std::vector<double> cw(n_t);
        for (size_t k = 0; k < n_t; ++k) cw[k] = cut.eval(t_arr[k]);
        // per realization: interior rows then exterior rows, as a handle holds them
        std::vector<std::vector<double>> bubbles(R);
        std::vector<std::vector<uint32_t>> ids(R);
        std::vector<bgw::SpectrumJob> jobs(R);
        for (size_t r = 0; r < R; ++r) {
            const size_t ni = io[r + 1] - io[r], ne = eo[r + 1] - eo[r];
            const double* ri = pi ? pi + 4 * io[r] : nullptr;
            const double* re = pe ? pe + 4 * eo[r] : nullptr;
            if (validate) bgw::check_causality(ri, ni, re, ne);
            if (ni > 0xffffffffULL) throw Error{"too many interior bubbles in one realization"};
            bubbles[r].resize(4 * (ni + ne));
            if (ni) std::memcpy(bubbles[r].data(), ri, 4 * ni * sizeof(double));
            if (ne) std::memcpy(bubbles[r].data() + 4 * ni, re, 4 * ne * sizeof(double));
            ids[r].resize(ni);
            for (size_t a = 0; a < ni; ++a) ids[r][a] = (uint32_t)a;
            jobs[r] = settings_job(h, t_arr, cw, w, n_w, rot.data(), n_khat);
            jobs[r].bubbles = bubbles[r].data();
            jobs[r].n_int = ni;
            jobs[r].n_tot = ni + ne;
            jobs[r].sel = ids[r].data();
            jobs[r].n_sel = ni;
            // a fixed launch shape applies to the batched launches (the measured one is taken there)
            jobs[r].frames_per_launch = h->frames_per_launch;
            jobs[r].row_parts = (int)h->row_parts;
            jobs[r].gemm_stages = (int)h->gemm_stages;
            jobs[r].mask_chunking = (int)h->mask_chunking;
        }
        const bool fixed = h->frames_per_launch || h->row_parts || h->gemm_stages || h->mask_chunking;
        h->timings = BgwxTimings{};
        std::vector<double> result(2 * expected, 0.0);
        bgw::run_ensemble(device(h), jobs, result.data(), &h->timings, h->autotune && !fixed);
        BgwComplex64* o = const_cast<BgwComplex64*>(slice(out, out_len, "out"));
        for (size_t q = 0; q < expected; ++q) o[q] = BgwComplex64{result[2 * q], result[2 * q + 1]};
    });
}

BgwStatus bgwx_generalized_bulk_flow_spectrum_vjp(bgw_generalized_bulk_flow* bulk_flow, const double* w_arr,
                                                  size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                  size_t n_t, const double* khat, size_t n_khat,
                                                  BgwTimeCutoffConfig time_cutoff, const BgwComplex64* grad_out,
                                                  size_t grad_len, double* grad_coefficients, double* grad_powers,
                                                  double* grad_bubbles) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        const size_t S = h->n_sets, M = h->n_terms, SM = S * M;
        const size_t K = n_khat ? n_khat : 1;
        const size_t expected = checked_mul(checked_mul(checked_mul(K, 2, "grad_out"), S, "grad_out"), n_w,
                                            "grad_out");
        if (grad_len != expected)
            throw Error{"grad_len=" + std::to_string(grad_len) + " does not match expected length " +
                        std::to_string(expected)};
        const size_t n_tot = h->n_int + h->n_ext;
        double* gc = const_cast<double*>(slice<double>(grad_coefficients, SM, "grad_coefficients"));
        double* gp = const_cast<double*>(slice<double>(grad_powers, SM, "grad_powers"));
        double* gb = const_cast<double*>(slice<double>(grad_bubbles, checked_mul(n_tot, 4, "grad_bubbles"),
                                                       "grad_bubbles"));
        if (SM) std::fill(gc, gc + SM, 0.0), std::fill(gp, gp + SM, 0.0);
        if (n_tot) std::fill(gb, gb + 4 * n_tot, 0.0);
        if (n_t < 2) throw Error{"Invalid resolution: n_t must be >= 2 for integration"};
        const double tb = has_t_begin ? t_begin : 0.0;
        if (tb > t_end)
            throw Error{"Invalid time range: t_begin=" + bgw::rust_f64(tb) + " > t_end=" + bgw::rust_f64(t_end)};
        require_resolution(h);
        if (expected == 0 || h->n_int == 0) return;
        const BgwComplex64* g = slice(grad_out, grad_len, "grad_out");
        std::vector<double> rot = khat_rotations(khat, n_khat);
        const double* w = slice(w_arr, n_w, "w_arr");
        Cutoff cut = make_cutoff(time_cutoff);
        std::vector<double> t_arr = bgw::linspace(tb, t_end, n_t);
        std::vector<double> cw(n_t);
        for (size_t k = 0; k < n_t; ++k) cw[k] = cut.eval(t_arr[k]);
        std::vector<uint32_t> ids(h->n_int);
        for (size_t a = 0; a < h->n_int; ++a) ids[a] = (uint32_t)a;
        bgw::SpectrumJob job = settings_job(h, t_arr, cw, w, n_w, n_khat ? rot.data() : nullptr, K);
        job.bubbles = h->bubbles.data();
        job.n_int = h->n_int;
        job.n_tot = n_tot;
        job.sel = ids.data();
        job.n_sel = ids.size();
        std::vector<double> gbar(2 * expected);
        for (size_t q = 0; q < expected; ++q) {
            gbar[2 * q] = g[q].re;
            gbar[2 * q + 1] = g[q].im;
        }
        std::vector<double> gpar(2 * SM);
        h->timings = BgwxTimings{};
        bgw::run_adjoint(device(h), job, gbar.data(), gpar.data(), gb, &h->timings);
        for (size_t q = 0; q < SM; ++q) {
            gc[q] = gpar[q];
            gp[q] = gpar[SM + q];
        }
    });
}

namespace {
// Validates the post-processing arguments and returns x = sorted cos(theta_k)
// (data_gw_bulkflow.py:23: np.sort of the rows' cos_theta_k).
std::vector<double> power_spectrum_args(size_t n_khat, size_t n_sets, const double* w_arr, size_t n_w,
                                        const double* set_weights, const double* cos_thetak) {
    if (n_khat == 0) throw Error{"cos_thetak must hold at least one direction"};
    if (n_sets == 0) throw Error{"n_sets must be > 0"};
    slice(w_arr, n_w, "w_arr");
    const double* a = slice(set_weights, n_sets, "set_weights");
    const double* ck = slice(cos_thetak, n_khat, "cos_thetak");
    checked_mul(checked_mul(checked_mul(n_khat, 2, "c"), n_sets, "c"), n_w, "c");
    for (size_t s = 0; s < n_sets; ++s)
        if (!std::isfinite(a[s])) throw Error{"set_weights must be finite"};
    std::vector<double> x(ck, ck + n_khat);
    for (double v : x)
        if (std::isnan(v)) throw Error{"cos_thetak must not contain NaN"};
    std::sort(x.begin(), x.end());
    return x;
}
}  // namespace

BgwStatus bgwx_generalized_bulk_flow_power_spectrum(bgw_generalized_bulk_flow* bulk_flow, const BgwComplex64* c,
                                                    size_t n_khat, size_t n_sets, const double* w_arr, size_t n_w,
                                                    const double* set_weights, const double* cos_thetak,
                                                    double* spectra, double* de_dlogw) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        const std::vector<double> x = power_spectrum_args(n_khat, n_sets, w_arr, n_w, set_weights, cos_thetak);
        if (n_w == 0) return;
        const BgwComplex64* pc = slice(c, n_khat * 2 * n_sets * n_w, "c");
        if (!de_dlogw) throw Error{"de_dlogw must not be null"};
        bgw::run_power_spectrum(device(h), pc, false, n_khat, n_sets, n_w, w_arr, set_weights, x.data(), spectra,
                                de_dlogw, false);
    });
}

BgwStatus bgwx_generalized_bulk_flow_power_spectrum_device(bgw_generalized_bulk_flow* bulk_flow,
                                                           const void* c_device, size_t n_khat, size_t n_sets,
                                                           const double* w_arr, size_t n_w,
                                                           const double* set_weights, const double* cos_thetak,
                                                           void* spectra_device, void* de_dlogw_device) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        const std::vector<double> x = power_spectrum_args(n_khat, n_sets, w_arr, n_w, set_weights, cos_thetak);
        if (n_w == 0) return;
        if (!c_device || !de_dlogw_device) throw Error{"c_device and de_dlogw_device must not be null"};
        bgw::run_power_spectrum(device(h), c_device, true, n_khat, n_sets, n_w, w_arr, set_weights, x.data(),
                                static_cast<double*>(spectra_device), static_cast<double*>(de_dlogw_device), true);
    });
}

BgwStatus bgwx_generalized_bulk_flow_compute_c_tensor_khat(bgw_generalized_bulk_flow* bulk_flow, const double* w_arr,
                                                          size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                          size_t n_t, const double* khat, size_t n_khat,
                                                          const size_t* selected_bubbles, size_t n_selected_bubbles,
                                                          BgwComplex64* out, size_t out_len) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        const double* w = slice(w_arr, n_w, "w_arr");
        const size_t K = khat ? n_khat : 1;
        if (khat && n_khat == 0) throw Error{"khat must hold at least one direction"};
        std::vector<double> rot = khat ? khat_rotations(khat, n_khat) : std::vector<double>();
        const size_t S = h->n_sets;
        const size_t expected = checked_mul(checked_mul(checked_mul(K, 6, "out"), S, "out"), n_w, "out");
        if (out_len != expected)
            throw Error{"out_len=" + std::to_string(out_len) + " does not match expected length " +
                        std::to_string(expected)};
        if (n_t < 2) throw Error{"n_t must be >= 2 for integration"};
        std::vector<uint32_t> ids;
        if (selected_bubbles) {
            const size_t* sel = slice(selected_bubbles, n_selected_bubbles, "selected_bubbles");
            for (size_t q = 0; q < n_selected_bubbles; ++q) {
                if (sel[q] >= h->n_int) {
                    Error e{"Index " + std::to_string(sel[q]) + " out of bounds for max " + std::to_string(h->n_int)};
                    e.index_error = true;
                    throw e;
                }
                ids.push_back((uint32_t)sel[q]);
            }
        } else {
            for (size_t a = 0; a < h->n_int; ++a) ids.push_back((uint32_t)a);
        }
        std::vector<double> result(2 * expected, 0.0);
        h->timings = BgwxTimings{};
        const double tb = has_t_begin ? t_begin : 0.0;
        if (tb > t_end)
            throw Error{"Invalid time range: t_begin=" + bgw::rust_f64(tb) + " > t_end=" + bgw::rust_f64(t_end)};
        if (!ids.empty() && S > 0 && n_w > 0) {
            require_resolution(h);
            std::vector<double> t_arr = bgw::linspace(tb, t_end, n_t);
            std::vector<double> cw(n_t, 1.0);  // the tensor form has no time cutoff
            bgw::SpectrumJob job = settings_job(h, t_arr, cw, w, n_w, khat ? rot.data() : nullptr, K);
            job.bubbles = h->bubbles.data();
            job.n_int = h->n_int;
            job.n_tot = h->n_int + h->n_ext;
            job.sel = ids.data();
            job.n_sel = ids.size();
            job.tensor = true;
            job.kernel = BGWX_KERNEL_FP64_DIRECT;
            bgw::run_spectrum(device(h), job, result.data(), false, &h->timings);
        }
        BgwComplex64* o = const_cast<BgwComplex64*>(slice(out, out_len, "out"));
        for (size_t q = 0; q < expected; ++q) o[q] = BgwComplex64{result[2 * q], result[2 * q + 1]};
    });
}

BgwStatus bgwx_nucleate_exponential(const int64_t* n_bubbles, const double* beta, const uint64_t* seeds,
                                    size_t n_realizations, double box_side, double gamma_scale,
                                    size_t max_rejections, double* interior, size_t interior_len, double* exterior,
                                    size_t exterior_len, int32_t* attempts) {
    return run_ffi([&] {
        const size_t R = n_realizations;
        const int64_t* n = slice(n_bubbles, R, "n_bubbles");
        const double* b = slice(beta, R, "beta");
        const uint64_t* sd = slice(seeds, R, "seeds");
        if (!(box_side > 0.0) || !std::isfinite(box_side)) throw Error{"box_side must be positive and finite"};
        if (!(gamma_scale > 0.0) || !std::isfinite(gamma_scale)) throw Error{"gamma_scale must be positive and finite"};
        if (max_rejections == 0 || max_rejections > (size_t)INT64_MAX) throw Error{"max_rejections must be > 0"};
        size_t rows = 0;
        for (size_t r = 0; r < R; ++r) {
            if (n[r] < 0) throw Error{"n_bubbles must be >= 0"};
            if (!(b[r] > 0.0) || !std::isfinite(b[r])) throw Error{"beta must be positive and finite"};
            rows += (size_t)n[r];
        }
        if (interior_len != checked_mul(rows, 4, "interior") || exterior_len != checked_mul(rows, 24, "exterior"))
            throw Error{"interior_len / exterior_len must be 4 and 24 times the total bubble count " +
                        std::to_string(rows)};
        std::vector<int32_t> att(R, 0);
        if (rows) {
            slice(interior, interior_len, "interior");
            slice(exterior, exterior_len, "exterior");
        }
        bgw::run_nucleation(n, b, sd, R, box_side, gamma_scale, (int64_t)max_rejections, 40, interior, exterior,
                            att.data());
        for (size_t r = 0; r < R; ++r)
            if (att[r] < 0)
                throw Error{"realization " + std::to_string(r) +
                            ": the false vacuum ran out before every bubble was placed, after 40 doublings of "
                            "the rate prefactor"};
        if (attempts) std::memcpy(attempts, att.data(), R * sizeof(int32_t));
    });
}

BgwStatus bgwx_generalized_bulk_flow_set_bubbles(bgw_generalized_bulk_flow* bulk_flow, const double* interior,
                                                 size_t n_interior, const double* exterior, size_t n_exterior) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        size_t li = checked_mul(n_interior, 4, "interior bubbles");
        size_t le = checked_mul(n_exterior, 4, "exterior bubbles");
        const double* pi = slice(interior, li, "bubbles_interior");
        const double* pe = slice(exterior, le, "bubbles_exterior");
        h->bubbles.resize(li + le);
        if (li) std::memcpy(h->bubbles.data(), pi, li * sizeof(double));
        if (le) std::memcpy(h->bubbles.data() + li, pe, le * sizeof(double));
        h->n_int = n_interior;
        h->n_ext = n_exterior;
    });
}

namespace {
// compute_c_integrand (GBF:875-920) and its tensor form (NGBF:993-1065): out
// (NG, S, W, n_t) with NG = 2 (C_+, C_x) or 6 (xx, xy, xz, yy, yz, zz).
void integrand_common(bgw_generalized_bulk_flow* bulk_flow, const double* w_arr, size_t n_w, bool has_t_begin,
                      double t_begin, double t_end, size_t n_t, const size_t* selected_bubbles,
                      size_t n_selected_bubbles, BgwComplex64* out, size_t out_len, bool tensor) {
    {
        auto* h = handle(bulk_flow);
        const size_t S = h->n_sets;
        const size_t expected =
            checked_mul(checked_mul(checked_mul(tensor ? 6 : 2, S, "out"), n_w, "out"), n_t, "out");
        // generalized_bulk_flow.rs:883-906: n_t, then the selection
        if (n_t < 2) throw Error{"Invalid resolution: n_t must be >= 2"};
        std::vector<uint32_t> ids;
        if (selected_bubbles) {
            const size_t* sel = slice(selected_bubbles, n_selected_bubbles, "selected_bubbles");
            for (size_t q = 0; q < n_selected_bubbles; ++q) {
                if (sel[q] >= h->n_int) {
                    Error e{"Index " + std::to_string(sel[q]) + " out of bounds for max " + std::to_string(h->n_int)};
                    e.index_error = true;
                    throw e;
                }
                ids.push_back((uint32_t)sel[q]);
            }
        } else {
            for (size_t a = 0; a < h->n_int; ++a) ids.push_back((uint32_t)a);
        }
        if (out_len != expected)
            throw Error{"out_len=" + std::to_string(out_len) + " does not match expected length " +
                        std::to_string(expected)};
        BgwComplex64* o = const_cast<BgwComplex64*>(slice(out, out_len, "out"));
        for (size_t q = 0; q < expected; ++q) o[q] = BgwComplex64{0.0, 0.0};
        const double tb = has_t_begin ? t_begin : 0.0;
        // bubbles nucleating at or after t_end contribute zeros before the range check (:786-797)
        std::vector<uint32_t> live;
        for (uint32_t a : ids)
            if (h->bubbles[4 * (size_t)a] < t_end) live.push_back(a);
        if (live.empty() || S == 0 || n_w == 0) return;
        if (tb > t_end)
            throw Error{"Invalid time range: t_begin=" + bgw::rust_f64(tb) + " > t_end=" + bgw::rust_f64(t_end)};
        require_resolution(h);
        const double* w = slice(w_arr, n_w, "w_arr");
        std::vector<double> t_arr = bgw::linspace(tb, t_end, n_t);
        std::vector<double> ones(n_t, 1.0);  // no time cutoff on the integrand
        bgw::SpectrumJob job = settings_job(h, t_arr, ones, w, n_w, nullptr, 1);
        job.bubbles = h->bubbles.data();
        job.n_int = h->n_int;
        job.n_tot = h->n_int + h->n_ext;
        job.sel = live.data();
        job.n_sel = live.size();
        job.tensor = tensor;
        std::vector<double> result(2 * expected);
        h->timings = BgwxTimings{};
        bgw::run_integrand(device(h), job, result.data(), &h->timings);
        for (size_t q = 0; q < expected; ++q) o[q] = BgwComplex64{result[2 * q], result[2 * q + 1]};
    }
}
}  // namespace

BgwStatus bgwx_generalized_bulk_flow_compute_c_integrand(bgw_generalized_bulk_flow* bulk_flow, const double* w_arr,
                                                         size_t n_w, bool has_t_begin, double t_begin, double t_end,
                                                         size_t n_t, const size_t* selected_bubbles,
                                                         size_t n_selected_bubbles, BgwComplex64* out,
                                                         size_t out_len) {
    return run_ffi([&] {
        integrand_common(bulk_flow, w_arr, n_w, has_t_begin, t_begin, t_end, n_t, selected_bubbles,
                         n_selected_bubbles, out, out_len, false);
    });
}

BgwStatus bgwx_generalized_bulk_flow_compute_c_tensor_integrand(bgw_generalized_bulk_flow* bulk_flow,
                                                                const double* w_arr, size_t n_w, bool has_t_begin,
                                                                double t_begin, double t_end, size_t n_t,
                                                                const size_t* selected_bubbles,
                                                                size_t n_selected_bubbles, BgwComplex64* out,
                                                                size_t out_len) {
    return run_ffi([&] {
        integrand_common(bulk_flow, w_arr, n_w, has_t_begin, t_begin, t_end, n_t, selected_bubbles,
                         n_selected_bubbles, out, out_len, true);
    });
}

BgwStatus bgwx_generalized_bulk_flow_drop_resident_inputs(bgw_generalized_bulk_flow* bulk_flow) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (h->dev) bgw::device_drop_resident(h->dev);
    });
}

BgwStatus bgwx_generalized_bulk_flow_set_stream(bgw_generalized_bulk_flow* bulk_flow, void* stream) {
    return run_ffi([&] { bgw::device_set_stream(device(handle(bulk_flow)), stream); });
}

BgwStatus bgwx_generalized_bulk_flow_set_kernel(bgw_generalized_bulk_flow* bulk_flow, BgwxKernel kernel) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (kernel != BGWX_KERNEL_FP64_DIRECT && kernel != BGWX_KERNEL_FP64_FACTORED && kernel != BGWX_KERNEL_MIXED &&
            kernel != BGWX_KERNEL_MIXED_SIMT)
            throw Error{"unknown kernel " + std::to_string((int)kernel)};
        h->kernel = kernel;
    });
}

BgwStatus bgwx_generalized_bulk_flow_set_launch_shape(bgw_generalized_bulk_flow* bulk_flow, size_t frames_per_launch,
                                                      size_t row_parts) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (row_parts > 16) throw Error{"row_parts must be at most 16"};
        h->frames_per_launch = frames_per_launch;
        h->row_parts = row_parts;
    });
}

BgwStatus bgwx_generalized_bulk_flow_set_gemm_stages(bgw_generalized_bulk_flow* bulk_flow, size_t stages) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (stages != 0 && (stages < 3 || stages > 5)) throw Error{"gemm stages must be 0 (automatic) or 3 to 5"};
        h->gemm_stages = stages;
    });
}

BgwStatus bgwx_generalized_bulk_flow_last_gemm_stages(const bgw_generalized_bulk_flow* bulk_flow, size_t* out_stages) {
    return run_ffi([&] {
        if (!bulk_flow) throw Error{"bulk_flow must not be null"};
        if (!out_stages) throw Error{"outputs must not be null"};
        *out_stages = bulk_flow->dev ? (size_t)bgw::last_launch_shape(bulk_flow->dev).gemm_stages : 0;
    });
}

BgwStatus bgwx_generalized_bulk_flow_set_mask_chunking(bgw_generalized_bulk_flow* bulk_flow, size_t chunking) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (chunking != 0 && chunking != 1 && chunking != 2 && chunking != 4)
            throw Error{"mask chunking must be 0 (automatic), 1, 2 or 4"};
        h->mask_chunking = chunking;
    });
}

BgwStatus bgwx_generalized_bulk_flow_last_mask_chunking(const bgw_generalized_bulk_flow* bulk_flow,
                                                        size_t* out_chunking) {
    return run_ffi([&] {
        if (!bulk_flow) throw Error{"bulk_flow must not be null"};
        if (!out_chunking) throw Error{"outputs must not be null"};
        *out_chunking = bulk_flow->dev ? (size_t)bgw::last_launch_shape(bulk_flow->dev).mask_chunking : 0;
    });
}

BgwStatus bgwx_generalized_bulk_flow_set_keep_masks(bgw_generalized_bulk_flow* bulk_flow, bool enabled) {
    return run_ffi([&] { handle(bulk_flow)->keep_masks = enabled; });
}

BgwStatus bgwx_generalized_bulk_flow_set_autotune(bgw_generalized_bulk_flow* bulk_flow, bool enabled) {
    return run_ffi([&] { handle(bulk_flow)->autotune = enabled; });
}

BgwStatus bgwx_generalized_bulk_flow_last_launch_shape(const bgw_generalized_bulk_flow* bulk_flow,
                                                       size_t* out_frames_per_launch, size_t* out_row_parts) {
    return run_ffi([&] {
        if (!bulk_flow) throw Error{"bulk_flow must not be null"};
        if (!out_frames_per_launch || !out_row_parts) throw Error{"outputs must not be null"};
        const bgw_generalized_bulk_flow* h = bulk_flow;
        *out_frames_per_launch = 0;
        *out_row_parts = 0;
        if (h->dev) {
            const bgw::LaunchShape s = bgw::last_launch_shape(h->dev);
            *out_frames_per_launch = s.frames_per_launch;
            *out_row_parts = (size_t)s.row_parts;
        }
    });
}

BgwStatus bgwx_generalized_bulk_flow_first_colliding(bgw_generalized_bulk_flow* bulk_flow, size_t a_begin,
                                                     size_t a_end, int32_t* out_codes, double* out_delta_tab) {
    return run_ffi([&] {
        auto* h = handle(bulk_flow);
        if (a_end > h->n_int || a_begin > a_end) {
            Error e{"Index " + std::to_string(a_end > h->n_int ? a_end : a_begin) + " out of bounds for max " +
                    std::to_string(h->n_int)};
            e.index_error = true;
            throw e;
        }
        require_resolution(h);
        size_t n = a_end - a_begin;
        if (n == 0) return;
        size_t nd = h->n_cos * h->n_phi;
        slice(out_codes, checked_mul(n, nd, "out_codes"), "out_codes");
        std::vector<uint32_t> ids(n);
        for (size_t q = 0; q < n; ++q) ids[q] = (uint32_t)(a_begin + q);
        bgw::MaskJob job;
        job.bubbles = h->bubbles.data();
        job.n_int = h->n_int;
        job.n_tot = h->n_int + h->n_ext;
        job.n_cos = h->n_cos;
        job.n_phi = h->n_phi;
        job.dirs = h->dirs.data();
        job.sel = ids.data();
        job.n_sel = n;
        h->timings = BgwxTimings{};
        bgw::run_masks(device(h), job, out_codes, out_delta_tab, &h->timings);
    });
}

void bgwx_rotation_for_khat(double kx, double ky, double kz, double* R) { bgw::rotation_for_khat(kx, ky, kz, R); }

BgwStatus bgwx_generalized_bulk_flow_last_timings(const bgw_generalized_bulk_flow* bulk_flow, BgwxTimings* out) {
    return run_ffi([&] {
        if (!bulk_flow) throw Error{"bulk_flow must not be null"};
        if (!out) throw Error{"out must not be null"};
        *out = bulk_flow->timings;
    });
}

BgwStatus bgwx_lattice_contains(BgwxLatticeKind kind, const double* params, const double* points_xyz,
                                size_t n_points, uint8_t* out, size_t* n_out) {
    return run_ffi([&] {
        if (!n_out) throw Error{"n_out must not be null"};
        if (kind == BGWX_LATTICE_EMPTY) {
            *n_out = 0;
            return;
        }
        size_t np = kind == BGWX_LATTICE_SPHERICAL ? 4 : 12;
        if ((int)kind < 0 || (int)kind > 3) throw Error{"unknown lattice kind"};
        const double* p = slice(params, np, "params");
        const double* pts = slice(points_xyz, checked_mul(n_points, 3, "points"), "points");
        uint8_t* o = const_cast<uint8_t*>(slice(out, n_points, "out"));
        bgw::lattice_contains(kind, p, pts, n_points, o);
        *n_out = n_points;
    });
}

BgwStatus bgwx_lattice_exterior(BgwxLatticeKind kind, const double* params, BgwxBoundaryCondition bc,
                                const double* interior, size_t n_interior, double* out, size_t capacity,
                                size_t* n_out) {
    return run_ffi([&] {
        if (!n_out) throw Error{"n_out must not be null"};
        if ((int)kind < 0 || (int)kind > 3) throw Error{"unknown lattice kind"};
        if ((int)bc < 0 || (int)bc > 2) throw Error{"unknown boundary condition"};
        size_t np = kind == BGWX_LATTICE_EMPTY ? 0 : (kind == BGWX_LATTICE_SPHERICAL ? 4 : 12);
        const double* p = slice(params, np, "params");
        const double* in = slice(interior, checked_mul(n_interior, 4, "interior"), "interior");
        std::vector<double> ext = bgw::lattice_exterior(kind, p, bc, in, n_interior);
        size_t rows = ext.size() / 4;
        *n_out = rows;
        if (rows > capacity)
            throw Error{"capacity " + std::to_string(capacity) + " is smaller than " + std::to_string(rows) +
                        " exterior rows"};
        double* o = const_cast<double*>(slice(out, ext.size(), "out"));
        if (!ext.empty()) std::memcpy(o, ext.data(), ext.size() * sizeof(double));
    });
}

BgwStatus bgwx_check_causality(const double* interior, size_t n_interior, const double* exterior,
                               size_t n_exterior) {
    return run_ffi([&] {
        const double* pi = slice(interior, checked_mul(n_interior, 4, "interior"), "bubbles_interior");
        const double* pe = slice(exterior, checked_mul(n_exterior, 4, "exterior"), "bubbles_exterior");
        bgw::check_causality(pi, n_interior, pe, n_exterior);
    });
}

int bgwx_device_count(void) { return bgw::device_count(); }

}  // extern "C"
