// Tensor-core (tcgen05, int8 digit slices) time-phase GEMM of the mixed kernel, spectrum_tc.cu.
#pragma once

#include <cstdint>

#include "device_common.cuh"

namespace bgw {

// Operand blocks in HBM: 128 rows x 32 time steps of int8 in the K-major
// 32-byte-swizzled layout of the UMMA descriptor (4 KB per block): row n of a
// block at byte (n/8)*256 + (n%8)*32, its 16-byte half h (steps 16h..16h+15)
// at half position h ^ ((n/4) % 2).  Byte index of (row n, step k), k in [0, 32).
__host__ __device__ inline int i8_swz(int n, int k) {
    return (n >> 3) * 256 + (n & 7) * 32 + ((((k >> 4) ^ (n >> 2)) & 1) << 4) + (k & 15);
}
constexpr int kI8Slices = 4;                       // int8 digits per value
constexpr int kI8Block = 128 * 32;                 // bytes of one digit block
constexpr int kI8BlockSet = kI8Slices * kI8Block;  // the four digit blocks of one (rows, 32 steps) block

// Digits of x in [-1, 1]: X = rint(x F) with F = 0x7F7F7F7F (|X| <= F < 2^31)
// written in balanced base 256, x F = sum_s d_s 256^(3-s) with the top digit
// d_0 in [-127, 127] and d_1, d_2, d_3 in [-128, 127]; the representation error
// is |e| <= 0.5 / F (2^-32 about).  Adding 128 to every digit gives the
// ordinary base-256 digits of Y = X + 0x80808080, which lies in
// [0x01010101, 0xFFFFFFFF] and so needs no carry beyond 32 bits: the digits are
// the bytes of Y with the top bit flipped.  Returned packed, byte s = digit
// d_s (d_0 the most significant).
constexpr double kI8Full = 2139062143.0;  // F = 0x7F7F7F7F
// x y = (256^6 / F^2) sum_L 256^-L sum_{s+r=L} d_s(x) d_r(y) for the digit
// pairs of level L = s + r
constexpr double kI8PairScale = 281474976710656.0 / (kI8Full * kI8Full);
// X is the low word of x F + 1.5 2^52: the sum lies in [2^52, 2^53), where the
// spacing of doubles is 1, so the fused multiply-add rounds x F to an integer
// and the low 32 mantissa bits hold it in two's complement.
__device__ __forceinline__ uint32_t i8_digits(double x) {
    const double r = fma(x, kI8Full, 6755399441055744.0);
    const uint32_t y = (uint32_t)__double2loint(r) + 0x80808080u;
    return __byte_perm(y ^ 0x80808080u, 0u, 0x0123);
}

// Four packed digit words (one step each, byte s = digit s) transposed into
// four slice words (one digit each, byte m = step m).
__device__ __forceinline__ void i8_transpose4(uint32_t p0, uint32_t p1, uint32_t p2, uint32_t p3,
                                              uint32_t (&w)[4]) {
    const uint32_t t0 = __byte_perm(p0, p1, 0x5140), t1 = __byte_perm(p2, p3, 0x5140);
    const uint32_t t2 = __byte_perm(p0, p1, 0x7362), t3 = __byte_perm(p2, p3, 0x7362);
    w[0] = __byte_perm(t0, t1, 0x5410);
    w[1] = __byte_perm(t0, t1, 0x7632);
    w[2] = __byte_perm(t2, t3, 0x5410);
    w[3] = __byte_perm(t2, t3, 0x7632);
}

struct TcArgs {
    const D4* bub;          // rotated frames (kn, n_tot)
    size_t n_tot;
    const uint32_t* sel;
    int n_sel;
    int n_cos, n_t, n_w, S;
    const double* w;
    const double* cos_t;
    const int* kfirst;      // (n_sel) first step with t_k > t_a
    const int8_t* atab;     // time-phase digits: (n_cos, n_wt, nkb) block sets
    const int8_t* btab;     // beta digits: (kn, n_cos, tiles, nkb) block sets
    const double* bscale;   // (kn, n_sel, n_cos): beta of row (frame, slot, i) = scale x digits
    int n_wt, nkb;
    int bpt;                // bubbles per 128-column tile
    int tiles_per_frame;
    int row_parts;          // CTAs per (frequency tile, column tile), each over a range of cos-theta rows
    int stages;             // pipeline stages of 32 steps (3 to 5; 0: 4)
    double2* partial;       // (kn, tiles_per_frame, row_parts, 2, S, W)
    unsigned int* err;      // set non-zero when a pipeline wait gave up
};

// Fills atab (n_cos * n_wt * nkb block sets) with the digits of
// M_i[w, k] = e^{i w (1 - c_i) t_k} (rows 2 l + {0: cos, 1: sin} of frequency
// tile wt, zero past n_w and n_t).
void launch_tc_phase_table(const double* w, const double* cos_t, const double* t_arr, int n_cos, int n_w, int n_t,
                           int8_t* atab, cudaStream_t st);

// Launches the GEMM + epilogue for kn frames on `st`.
void launch_gemm_tc(const TcArgs& A, size_t kn, cudaStream_t st);

// Row parts that make n_ctas x parts CTAs fill whole waves of one CTA per SM
// best (at most n_cos / 8 parts).
int tc_row_parts(size_t n_ctas, int n_cos, int n_sm);

// Largest n_t the int8 GEMM accumulates exactly in 32-bit integers: a level
// sums at most 4 n_t products of magnitude <= 128^2, and 4 128^2 32767 < 2^31.
constexpr int kI8MaxSteps = 32767;

}  // namespace bgw
