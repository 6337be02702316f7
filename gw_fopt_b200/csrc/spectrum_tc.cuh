// Tensor-core (tcgen05, TF32 split) time-phase GEMM of the mixed kernel, spectrum_tc.cu.
#pragma once

#include "device_common.cuh"

namespace bgw {

// Operand blocks in HBM: 128 rows x 32 time steps of TF32 in the K-major
// 128-byte-swizzled layout of the UMMA descriptor (16 KB each), as a hi part
// followed by a lo part (x = hi + lo).  Float index of (row n, step k) inside
// a block; k in [0, 32).
__host__ __device__ inline size_t tc_swz(int n, int k) {
    return (size_t)(n >> 3) * 256 + (n & 7) * 32 + ((((k >> 2) ^ (n & 7))) << 2) + (k & 3);
}
constexpr int kTcBlockFloats = 128 * 32;

struct TcArgs {
    const D4* bub;          // rotated frames (kn, n_tot)
    size_t n_tot;
    const uint32_t* sel;
    int n_sel;
    int n_cos, n_t, n_w, S;
    const double* w;
    const double* cos_t;
    const int* kfirst;      // (n_sel) first step with t_k > t_a
    const float* atab;      // time phases: (n_cos, n_wt, nkb, hi|lo) blocks
    const float* btab;      // beta: (kn, n_cos, tiles, nkb, hi|lo) blocks
    int n_wt, nkb;
    int bpt;                // bubbles per 128-column tile
    int tiles_per_frame;
    int row_parts;          // CTAs per (frequency tile, column tile), each over a range of cos-theta rows
    double2* partial;       // (kn, tiles_per_frame, row_parts, 2, S, W)
    unsigned int* err;      // set non-zero when a pipeline wait gave up
};

// Fills atab (n_cos * n_wt * nkb * 2 blocks) with M_i[w, k] = e^{i w (1 - c_i) t_k}
// (rows 2 l + {0: cos, 1: sin} of frequency tile wt, zero past n_w and n_t).
void launch_tc_phase_table(const double* w, const double* cos_t, const double* t_arr, int n_cos, int n_w, int n_t,
                           float* atab, cudaStream_t st);

// Launches the GEMM + epilogue for kn frames on `st`.
void launch_gemm_tc(const TcArgs& A, size_t kn, cudaStream_t st);

// Row parts that make n_ctas x parts CTAs fill whole waves of one CTA per SM
// best (at most n_cos / 8 parts).
int tc_row_parts(size_t n_ctas, int n_cos, int n_sm);

}  // namespace bgw
