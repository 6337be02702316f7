// Adjoint (vector-Jacobian product) of the spectrum, adjoint.cu.
#pragma once

#include "device_common.cuh"

namespace bgw {

// Work arrays of one k-hat chunk of the adjoint, sized by adjoint_bytes_per_frame.
struct AdjointScratch {
    double* bbar;     // (kn, n_sel, n_cos, n_t, 2S)  dL/dT: cotangent of each (bubble, row, step) term
    double* imq;      // (kn, n_sel, n_cos, n_t, 2S)  Im sum_w w conj(G) e^{i phi}
    double* taubar;   // (kn, n_sel, n_cos*n_phi)     dL/dtau
    double* rowpart;  // (kn, n_sel, n_cos, 2 + 2 S M) per-row partial sums
    double* bubpart;  // (kn, n_sel, 4) gradient of each radiating bubble's own terms (t, x, y, z)
    long long* gfix;  // (n_tot, 4, 2) bubble gradients of the chunk as fixed-point (high, low) integer sums
    int* gexp;        // every contribution of the chunk is below 2^gexp in magnitude
};

// Launches the adjoint kernels of kn frames whose rotated bubbles, masks
// (delays and first-collider codes) and cotangents are on the device, and
// accumulates into g_bub ((n_tot, 4), the unrotated frame) and g_par
// (coefficients then powers, 2 S M).  Returns the number of launches.
uint64_t launch_adjoint_chunk(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                              const double* tau, const int32_t* codes, const D4* dirs, const double* cos_t,
                              const double* sin2, const double* cos2, const double* coeffs, const double* powers,
                              const double* t_arr, const double* cutw, const double* w, const double* rot,
                              const double2* gbar, size_t kn, const AdjointScratch& s, const double2* mt,
                              const double* tt, double* g_bub, double* g_par);

// Frame-independent tables: mt (n_cos, n_w, n_t) time phases e^{i w t_k (1 - c_i)};
// tt (n_sel, n_t, 4 + S M) per (bubble, step) factors of the collided scaling.
uint64_t launch_adjoint_tables(Device* dev, const SpectrumJob& job, const D4* bub, const uint32_t* sel,
                               const double* cos_t, const double* t_arr, const double* w, const double* powers,
                               double2* mt, double* tt);

size_t adjoint_bytes_per_frame(const SpectrumJob& job);

}  // namespace bgw
