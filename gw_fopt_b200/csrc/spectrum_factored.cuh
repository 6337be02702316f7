// Factored spectrum kernels (FP64 and mixed precision), spectrum_factored.cu.
#pragma once

#include "device_common.cuh"

namespace bgw {

// Launches the factored spectrum for kn frames whose masks are in `tau`;
// writes (kn, 2, S, W) complex sums into out.  Returns the number of kernel
// launches.
uint64_t launch_factored(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                         const double* tau, const double* cos_t, const double* sin2, const double* cos2,
                         const double* coeffs, const double* powers, const double* t_arr, const double* cutw,
                         const double* w, size_t kn, double2* out, cudaEvent_t* ev3);

// Device bytes per k-hat frame of the factored path's work arrays.
size_t factored_bytes_per_frame(const SpectrumJob& job);

}  // namespace bgw
