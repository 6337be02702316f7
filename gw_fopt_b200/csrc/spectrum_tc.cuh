// Tensor-core (tcgen05, TF32 split) time-phase GEMM of the mixed kernel, spectrum_tc.cu.
#pragma once

#include "device_common.cuh"

namespace bgw {

struct TcArgs {
    const D4* bub;          // rotated frames (kn, n_tot)
    size_t n_tot;
    const uint32_t* sel;
    int n_sel;
    int n_cos, n_t, n_w, S;
    const double* t_arr;
    const double* w;
    const double* cos_t;
    const int* kfirst;      // (n_sel) first step with t_k > t_a
    const float* beta;      // (kn, n_cos, cols_pad, t_pad)
    long cols_pad;
    int t_pad;
    double dt;
    int bpt;                // bubbles per 128-column tile
    int tiles_per_frame;
    double2* partial;       // (kn, tiles_per_frame, 2, S, W)
    unsigned int* err;      // set non-zero when a pipeline wait gave up
};

// Launches the GEMM + epilogue for kn frames on `st`.
void launch_gemm_tc(const TcArgs& A, size_t kn, cudaStream_t st);

}  // namespace bgw
