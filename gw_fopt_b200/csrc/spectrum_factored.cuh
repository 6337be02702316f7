// Factored spectrum kernels (FP64 and mixed precision), spectrum_factored.cu.
#pragma once

#include "device_common.cuh"

namespace bgw {

// sin/cos of an FP64 argument: FP64 kernel uses sincos; the mixed kernel
// reduces the argument modulo 2 pi in FP64 and evaluates sincosf on the
// reduced FP32 argument.
template <class Real>
__device__ __forceinline__ void phase(double arg, double& s, double& c);

template <>
__device__ __forceinline__ void phase<double>(double arg, double& s, double& c) {
    sincos(arg, &s, &c);
}

template <>
__device__ __forceinline__ void phase<float>(double arg, double& s, double& c) {
    // Cody & Waite (1980) additive reduction with 2 pi = C1 + C2; the fused
    // multiply-add forms n*C1 exactly, so one constant pair suffices.
    const double inv2pi = 0.15915494309189535;
    const double C1 = 6.283185307179586;      // 2 pi rounded to double
    const double C2 = 2.4492935982947064e-16;  // 2 pi - C1
    const double n = rint(arg * inv2pi);
    const double r = fma(-n, C2, fma(-n, C1, arg));
    float sf, cf;
    sincosf((float)r, &sf, &cf);
    s = sf;
    c = cf;
}


// Launches the factored spectrum for frames [k0, k0 + kn) whose masks are in
// `tau`; writes (kn, 2, S, W) complex sums into out + k0 (2 S W), or, for a
// batched job (job.n_real > 0; real_tiles on the device), frame k of
// realization r into out + (r n_k + k) (2 S W).  Returns the number of kernel
// launches.
uint64_t launch_factored(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                         const double* tau, const double* cos_t, const double* sin2, const double* cos2,
                         const double* coeffs, const double* powers, const double* t_arr, const double* cutw,
                         const double* w, size_t k0, size_t kn, double2* out, const uint32_t* real_tiles,
                         cudaEvent_t* ev3);

// Device bytes per k-hat frame of the factored path's work arrays.
size_t factored_bytes_per_frame(const SpectrumJob& job);

}  // namespace bgw
