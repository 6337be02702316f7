// Spectrum post-processing on the device: the energy spectrum per k-hat
// direction and its integral over cos(theta_k), as the reference's
// downstream consumer forms them from the bulk-flow output
// (src/gw_fopt/bubble_dynamics/utils/data_gw_bulkflow.py:26-146):
//   C_+/x(w) = sum_s a_s C_{+/x, s}(w)                        (:67-106)
//   dE/dlnw dcos(theta_k) = 8 pi w^3 (|C_+|^2 + |C_x|^2)       (:108-114)
//   dE/dlnw = 2 trapezoid(dE/dlnw dcos(theta_k), x = sorted cos(theta_k))   (:143-146)
// The rows enter the trapezoid in the order given while x is sorted, as there.
// One thread per frequency walks the k-hat directions in order (a fixed
// summation order); the work is O(K S W), read once from HBM.

#include <cuda_runtime.h>
#include <math_constants.h>

#include "bgw_internal.h"
#include "device_common.cuh"

namespace bgw {

__global__ void k_power_spectrum(const double2* __restrict__ c, int K, int S, int W, const double* __restrict__ w,
                                 const double* __restrict__ a, const double* __restrict__ x,
                                 double* __restrict__ spectra, double* __restrict__ de) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= W) return;
    const double om = w[q];
    const double f = (8.0 * CUDART_PI) * (om * om * om);
    double acc = 0.0, yprev = 0.0;
    for (int k = 0; k < K; ++k) {
        double pr = 0.0, pi = 0.0, xr = 0.0, xi = 0.0;
        for (int s = 0; s < S; ++s) {
            const double as = a[s];
            if (as == 0.0) continue;  // a set that no weight names
            const double2 cp = c[((size_t)(2 * k) * S + s) * W + q];
            const double2 cx = c[((size_t)(2 * k + 1) * S + s) * W + q];
            pr += as * cp.x;
            pi += as * cp.y;
            xr += as * cx.x;
            xi += as * cx.y;
        }
        const double y = f * ((pr * pr + pi * pi) + (xr * xr + xi * xi));
        if (spectra) spectra[(size_t)k * W + q] = y;
        if (k > 0) acc += (x[k] - x[k - 1]) * (yprev + y) / 2.0;
        yprev = y;
    }
    de[q] = 2.0 * acc;
}

void launch_power_spectrum(cudaStream_t st, const void* c, size_t K, size_t S, size_t W, const double* w,
                           const double* a, const double* x, double* spectra, double* de) {
    if (K > 0x7fffffffULL || S > 0x7fffffffULL || W > 0x7fffffffULL) throw Error{"power spectrum: sizes too large"};
    if (W == 0) return;
    const unsigned blocks = (unsigned)((W + 127) / 128);
    k_power_spectrum<<<blocks, 128, 0, st>>>(static_cast<const double2*>(c), (int)K, (int)S, (int)W, w, a, x,
                                              spectra, de);
    CUDA_OK(cudaGetLastError());
}

}  // namespace bgw

namespace bgw {

void run_power_spectrum(Device* dev, const void* c, bool c_on_device, size_t K, size_t S, size_t W,
                        const double* w, const double* a, const double* x_sorted, double* spectra, double* de,
                        bool out_on_device) {
    CUDA_OK(cudaSetDevice(dev->id));
    const cudaStream_t st = dev->stream;
    const size_t c_bytes = K * 2 * S * W * sizeof(double2);
    const void* c_dev = c;
    if (!c_on_device) {
        dev->pp_in.ensure(c_bytes);
        CUDA_OK(cudaMemcpyAsync(dev->pp_in.p, c, c_bytes, cudaMemcpyHostToDevice, st));
        c_dev = dev->pp_in.p;
    }
    // small inputs, one buffer: w (W), set weights (S), sorted cos(theta_k) (K)
    dev->pp_small.ensure((W + S + K) * sizeof(double));
    double* small = static_cast<double*>(dev->pp_small.p);
    CUDA_OK(cudaMemcpyAsync(small, w, W * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(small + W, a, S * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(small + W + S, x_sorted, K * sizeof(double), cudaMemcpyHostToDevice, st));
    double* spec_dev = spectra;
    double* de_dev = de;
    if (!out_on_device) {
        dev->pp_out.ensure((K * W + W) * sizeof(double));
        de_dev = static_cast<double*>(dev->pp_out.p);
        spec_dev = spectra ? de_dev + W : nullptr;
    }
    launch_power_spectrum(st, c_dev, K, S, W, small, small + W, small + W + S, spec_dev, de_dev);
    if (!out_on_device) {
        CUDA_OK(cudaMemcpyAsync(de, de_dev, W * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (spectra)
            CUDA_OK(cudaMemcpyAsync(spectra, spec_dev, K * W * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    CUDA_OK(cudaStreamSynchronize(st));
}

}  // namespace bgw
