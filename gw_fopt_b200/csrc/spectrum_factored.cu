// Factored spectrum kernels (FP64 and mixed precision).
//
// The reference accumulates, per bubble a, cos-theta row i and time t_k,
//   B_{s,g}(a,i,k) e^{-i w dt_k c_i} dc v_i  x  e^{i w (t_k - z_a)} u_k cut_k dt / (6 pi)
// (generalized_bulk_flow.rs:481-873).  The phase splits as
//   w [(t_k - z_a) - (t_k - t_a) c_i] = w t_k (1 - c_i) + w (t_a c_i - z_a),
// so for a fixed row i the time phase M_i[w, k] = e^{i w (1 - c_i) t_k} is the
// same for every bubble and every k-hat frame, and
//   C_{s,g}(w) = sum_i sum_a e^{i w (t_a c_i - z_a)} Y_i[w, (a,s,g)],
//   Y_i = M_i (W x T complex)  .  beta_i (T x columns real),
// a GEMM per row (columns = frame x bubble x set x {+,x}) followed by a
// per-(w, bubble) phase in the epilogue.
//
// beta comes from the collision structure without evaluating every patch at
// every t: with q_j = w_j g(phi_j) (g = cos 2phi, sin 2phi) and
//   f = sum_m a_m (tau_j / dt)^{p_m} exp(-(dt - tau_j) / width)   (collided),
//   dt^3 sum_j q_j f_j = dt^3 U(k) + sum_m a_m dt^{3-p_m} e^{-dt/width} Pm(k),
// where U(k) sums q_j over the patches not yet collided at step k and Pm(k)
// sums q_j tau_j^{p_m} e^{tau_j/width} over those already collided.  k_events
// sorts each row's collided patches by the first time step at which the
// reference's test (t_k - t_a) >= tau_j holds (exact FP64 comparisons), in
// buckets of kKC steps, and stores U at every bucket boundary as a backward
// sum of the remaining terms (forming it as total minus collided cancels
// catastrophically once most patches have collided); the GEMM kernel turns
// running prefix sums into beta tile by tile.
//
// Kernels:
//   k_time_tables   per bubble and t: dt^3 and dt^{3-p} e^{-dt/width}
//   k_events        per (frame, bubble, row): bucketed, stably sorted events
//   k_spec_factored per (w tile, column tile): loop over rows i, GEMM over t
//                   in chunks of kKC with beta produced in shared memory,
//                   FP64 epilogue; Real = double (FP64) or float (mixed)
//   k_reduce_tiles  deterministic sum of the column-tile partials per frame

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "bgw_internal.h"
#include "device_common.cuh"
#include "spectrum_factored.cuh"
#include "spectrum_tc.cuh"
#include "tc_ptx.cuh"

namespace bgw {

constexpr int kKC = 32;          // time steps per GEMM k-tile
constexpr int kFold = 16;        // mixed: FP32 partial sums are folded into FP64 every kFold steps
constexpr int kWT = 64;          // frequencies per CTA
constexpr int kRows = 2 * kWT;   // GEMM rows: (Re, Im) of each frequency
constexpr int kThreads = 256;
constexpr int kTM = 8;           // register tile rows per thread (columns: TN = 8 FP32, 4 FP64)

// ---------------------------------------------------------------------------
__global__ void k_time_tables(const D4* __restrict__ bub, const uint32_t* __restrict__ sel, int n_sel,
                              const double* __restrict__ t_arr, int n_t, const double* __restrict__ powers,
                              const double* __restrict__ coeffs, const double* __restrict__ cutw, int SM,
                              int has_damp, double damp, double* __restrict__ D, int* __restrict__ kfirst) {
    const int slot = blockIdx.x;
    const int k = blockIdx.y * blockDim.x + threadIdx.x;
    if (slot >= n_sel || k >= n_t || sel[slot] == kNoSlot) return;
    const double ta = bub[sel[slot]].t;
    const double dt = t_arr[k] - ta;
    double* row = D + ((size_t)slot * n_t + k) * (1 + SM);
    const bool on = dt > 0.0;
    // step weight (time cutoff x trapezoid end weight) folded into the table
    const double wk = cutw[k] * ((k == 0 || k == n_t - 1) ? 0.5 : 1.0);
    const double d3 = on ? dt * (dt * dt) : 0.0;
    row[0] = wk * d3;
    const double e = has_damp ? exp(-dt / damp) : 1.0;
    for (int q = 0; q < SM; ++q) row[1 + q] = d3 != 0.0 ? wk * coeffs[q] * (pow(dt, 3.0 - powers[q]) * e) : 0.0;
    // first active step (t_a <= t_k and dt > 0): monotone in k
    if (on && (k == 0 || !(t_arr[k - 1] - ta > 0.0))) kfirst[slot] = k;
    if (k == n_t - 1 && !on) kfirst[slot] = n_t;
}

// Per (bubble, block of 32 steps): the least and the largest D_q(k) of each
// table column over the block's steps k < n_t (one warp, lane = step), stored
// as (min, max) pairs.
__global__ void k_time_maxima(const double* __restrict__ D, int n_sel, int n_t, int nblk, int Q,
                              double* __restrict__ Dmax) {
    const long wid = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (wid >= (long)n_sel * nblk) return;
    const int slot = (int)(wid / nblk), b = (int)(wid % nblk);
    const int k = (b << 5) + lane;
    for (int q = 0; q < Q; ++q) {
        const double v = k < n_t ? D[((size_t)slot * n_t + k) * Q + q] : 0.0;
        double lo = v, hi = v;
        for (int o = 16; o > 0; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            Dmax[((size_t)wid * Q + q) * 2] = lo;
            Dmax[((size_t)wid * Q + q) * 2 + 1] = hi;
        }
    }
}

// ---------------------------------------------------------------------------
// k_beta: one warp per row (frame, slot, i).  The row's collided patches
// become events at the first step k_j with (t_k - t_a) >= tau_j (exact FP64
// comparisons, GBF:405), counting-sorted (stable in j) into blocks of 32
// steps.  Block b covers k = 32 b + lane: each lane gathers its step's event
// weights, a warp inclusive scan gives the collided sums Pm(k) and a warp
// exclusive suffix scan plus the backward block totals gives the uncollided
// sums U(k) -- both are sums of the terms they stand for, never differences.
// beta(k) = rf_i u_k cut_k [dt^3 U(k) + sum_m a_m dt^{3-p_m} e^{-dt/w} Pm(k)]
// is written to beta[frame][i][col][k], col = slot*2S + 2s + g.
struct BetaArgs {
    const double* tau;     // (kn, n_sel, n_cos*n_phi)
    const D4* bub;         // bubbles (frame 0; times are frame independent)
    const uint32_t* sel;
    int n_sel, n_cos, n_phi, n_t, S, M;
    const double* t_arr;
    const double* cutw;
    const double* cos_t;
    const double* cos2;
    const double* sin2;
    const double* powers;  // (S*M)
    const double* coeffs;  // (S*M)
    const double* D;       // (n_sel, n_t, 1+S*M)
    int has_damp;
    double damp;
    double dphi, dcos, dt;
    long n_rows;           // kn * n_sel * n_cos
    int nblk;              // ceil(n_t / 32)
    long cols_pad;         // columns per (frame, i): tiles_per_frame * tile_cols
    int tile_cols;         // columns of one GEMM tile
    int bpt;               // bubbles per tile
    int t_pad;             // row length of beta
    int per_warp_bytes;
    int tiles;             // column tiles per frame (int8 digit layout)
    double* scale;         // int8 digit layout: (kn, n_sel, n_cos) row scales, max |beta| of the row
    const double* Dmax;    // int8 digit layout: (n_sel, nblk, 1+S*M, 2) least and largest D over each block's steps
};

// x^p: binary powering for integral |p| <= 32 (a few ulp), pow() otherwise.
__device__ __forceinline__ double tpow(double x, double p) {
    const double r = rint(p);
    if (r == p && fabs(r) <= 32.0) {
        unsigned n = (unsigned)fabs(r);
        double acc = 1.0, b = x;
        while (n) {
            if (n & 1u) acc *= b;
            b *= b;
            n >>= 1;
        }
        return r < 0.0 ? 1.0 / acc : acc;
    }
    return pow(x, p);
}

template <class Real, int SMC>
__global__ void __launch_bounds__(256, std::is_same<Real, int8_t>::value ? 3 : 1) k_beta(BetaArgs A, Real* __restrict__ beta) {
    extern __shared__ __align__(16) unsigned char sm_b[];
    constexpr int NQ = 2 + 2 * SMC;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long row = (long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (row >= A.n_rows) return;
    const int NB = A.nblk;
    const int EV = A.n_phi;  // event capacity: one event per patch at most
    unsigned char* base = sm_b + (size_t)warp * A.per_warp_bytes;
    double* evq = reinterpret_cast<double*>(base);             // [NQ][n_phi]: weight q of event e at q * n_phi + e
    double* btot = evq + (size_t)A.n_phi * NQ;                  // [NQ][NB] block totals
    double* uend = btot + (size_t)NQ * NB;                      // [NB][2] uncollided after block
    double* pbeg = uend + 2 * NB;                               // [NB][2 SMC] collided before block
    int* boff = reinterpret_cast<int*>(pbeg + (size_t)2 * SMC * NB);  // [NB+1]
    int* brun = boff + NB + 1;                                  // [NB]
    uint8_t* evs = reinterpret_cast<uint8_t*>(brun + NB);       // [n_phi + 4] step of each event within its block
    // a crowded event block's per-step counts and running offsets [2][32], and its events in step order [n_phi]
    int* scnt = reinterpret_cast<int*>(evs + ((A.n_phi + 4 + 3) & ~3));
    uint16_t* sperm = reinterpret_cast<uint16_t*>(scnt + 64);
    const int slot = (int)((row / A.n_cos) % A.n_sel);
    if (A.sel[slot] == kNoSlot) return;  // a padding slot of a batched job: its columns are never read
    const int i = (int)(row % A.n_cos);
    const long frame = row / ((long)A.n_cos * A.n_sel);
    const double* trow = A.tau + (size_t)row * A.n_phi;
    // The delays of patches j = lane + 32 jj, jj < kMaxJ, are loaded first, all at once (one
    // memory latency for the row), and kept for both passes over the patches.
    constexpr int kMaxJ = 6;
    double tj_c[kMaxJ];
#pragma unroll
    for (int jj = 0; jj < kMaxJ; ++jj) {
        const int j = 32 * jj + lane;
        tj_c[jj] = j < A.n_phi ? __ldcs(trow + j) : 0.0;
    }
    const double ta = A.bub[A.sel[slot]].t;
    const unsigned full = 0xffffffffu;
    const double inv_dt = 1.0 / A.dt;  // the estimate below is only a starting point
    auto block_of = [&](int j, double tj, int& kj) -> int {
        kj = A.n_t;
        if (j >= A.n_phi) return -2;  // not a patch
        if (!(tj > 0.0)) return -1;    // never collides
        // first k with (t_k - t_a) >= tau_j: arithmetic estimate, then exact
        // comparisons (the predicate is monotone in k) settle the boundary
        const double est = ceil((ta + tj - A.t_arr[0]) * inv_dt);
        int lo = est < 0.0 ? 0 : (est > (double)A.n_t ? A.n_t : (int)est);
        while (lo > 0 && A.t_arr[lo - 1] - ta >= tj) --lo;
        while (lo < A.n_t && !(A.t_arr[lo] - ta >= tj)) ++lo;
        kj = lo;
        return lo < A.n_t ? lo >> 5 : -1;
    };
    for (int b = lane; b < NB; b += 32) boff[b] = 0;
    __syncwarp();
    // pass 1: events per block; never-colliding weights (lane sums, fixed-order reduction).
    // The first collided step of patches j = lane + 32 jj, jj < kMaxJ, is kept for pass 2.
    int kj_c[kMaxJ], b_c[kMaxJ];
    double nc = 0.0, ns = 0.0;
    auto pass1 = [&](int j, int b) {
        if (b == -1) {
            const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
            nc += wj * A.cos2[j];
            ns += wj * A.sin2[j];
        }
        const unsigned m = __match_any_sync(full, b);
        if (b >= 0 && lane == __ffs(m) - 1) boff[b] += __popc(m);
        __syncwarp();
    };
#pragma unroll
    for (int jj = 0; jj < kMaxJ; ++jj) {
        if (32 * jj >= A.n_phi) break;
        const int j = 32 * jj + lane;
        kj_c[jj] = 0;
        b_c[jj] = block_of(j, tj_c[jj], kj_c[jj]);
        pass1(j, b_c[jj]);
    }
    for (int j0 = 32 * kMaxJ; j0 < A.n_phi; j0 += 32) {
        int kj;
        const int j = j0 + lane;
        const int b = block_of(j, j < A.n_phi ? trow[j] : 0.0, kj);
        pass1(j, b);
    }
    for (int o = 16; o > 0; o >>= 1) {
        nc += __shfl_down_sync(full, nc, o);
        ns += __shfl_down_sync(full, ns, o);
    }
    // block counts -> first event of each block: an exclusive warp scan over 32 blocks at a time
    {
        int carry = 0;
        for (int bc = 0; bc < NB; bc += 32) {
            const int b = bc + lane;
            const int c = b < NB ? boff[b] : 0;
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(full, incl, o);
                if (lane >= o) incl += t;
            }
            if (b < NB) {
                boff[b] = carry + incl - c;
                brun[b] = carry + incl - c;
            }
            carry += __shfl_sync(full, incl, 31);
        }
        __syncwarp();
        if (lane == 0) boff[NB] = carry;
    }
    __syncwarp();
    // pass 2: scatter events (stable in j within a block)
    const unsigned lt = (1u << lane) - 1u;
    auto pass2 = [&](int j, double tj, int kj, int b) {
        const unsigned m = __match_any_sync(full, b);
        int pos = 0;
        if (b >= 0) pos = brun[b] + __popc(m & lt);
        __syncwarp();
        if (b >= 0 && lane == __ffs(m) - 1) brun[b] += __popc(m);
        __syncwarp();
        if (b >= 0) {
            evs[pos] = (uint8_t)(kj & 31);
            const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
            const double qc = wj * A.cos2[j], qs = wj * A.sin2[j];
            double* q = evq + pos;
            q[0] = qc;
            q[EV] = qs;
            const double ed = A.has_damp ? exp(tj / A.damp) : 1.0;
#pragma unroll
            for (int t = 0; t < SMC; ++t) {
                const double f = tpow(tj, A.powers[t]) * ed;
                q[(2 + 2 * t) * EV] = qc * f;
                q[(3 + 2 * t) * EV] = qs * f;
            }
        }
    };
#pragma unroll
    for (int jj = 0; jj < kMaxJ; ++jj) {
        if (32 * jj >= A.n_phi) break;
        pass2(32 * jj + lane, tj_c[jj], kj_c[jj], b_c[jj]);
    }
    for (int j0 = 32 * kMaxJ; j0 < A.n_phi; j0 += 32) {
        int kj;
        const int j = j0 + lane;
        const double tj = j < A.n_phi ? trow[j] : 0.0;
        const int b = block_of(j, tj, kj);
        pass2(j, tj, kj, b);
    }
    __syncwarp();
    // block totals of every weight: the lanes take a block's events in strides
    // of 32 and a butterfly reduction adds the lane sums (a fixed order for a
    // given event count); then the collided sums before each block (exclusive
    // prefix over blocks) and the uncollided sums after each block (exclusive
    // suffix plus the never-colliding weights), as warp scans over lanes = blocks
    for (int b = lane; b < NB; b += 32)
        if (boff[b] == boff[b + 1]) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) btot[(size_t)q * NB + b] = 0.0;
        }
    for (int bc = 0; bc < NB; bc += 32) {
        const int bl = bc + lane;
        for (unsigned h = __ballot_sync(full, bl < NB && boff[bl] != boff[bl + 1]); h; h &= h - 1) {
            const int b = bc + __ffs(h) - 1;
            double t[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) t[q] = 0.0;
            for (int e = boff[b] + lane; e < boff[b + 1]; e += 32) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) t[q] += evq[(size_t)q * EV + e];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) t[q] += __shfl_xor_sync(full, t[q], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) btot[(size_t)q * NB + b] = t[q];
            }
        }
    }
    __syncwarp();
    {
        double carry[2 * SMC];
#pragma unroll
        for (int q = 0; q < 2 * SMC; ++q) carry[q] = 0.0;
        for (int bc = 0; bc < NB; bc += 32) {
            const int b = bc + lane;
            double v[2 * SMC];
#pragma unroll
            for (int q = 0; q < 2 * SMC; ++q) v[q] = b < NB ? btot[(size_t)(2 + q) * NB + b] : 0.0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
                for (int q = 0; q < 2 * SMC; ++q) {
                    const double u = __shfl_up_sync(full, v[q], o);
                    if (lane >= o) v[q] += u;
                }
            }
#pragma unroll
            for (int q = 0; q < 2 * SMC; ++q) {
                double ex = __shfl_up_sync(full, v[q], 1);
                if (lane == 0) ex = 0.0;
                if (b < NB) pbeg[(size_t)b * 2 * SMC + q] = carry[q] + ex;
                carry[q] += __shfl_sync(full, v[q], 31);
            }
        }
        // the never-colliding sums were reduced into lane 0
        double cc = __shfl_sync(full, nc, 0), cs = __shfl_sync(full, ns, 0);
        for (int bc = ((NB - 1) >> 5) << 5; bc >= 0; bc -= 32) {
            const int b = bc + lane;
            double vc = b < NB ? btot[b] : 0.0, vs = b < NB ? btot[(size_t)NB + b] : 0.0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double uc = __shfl_down_sync(full, vc, o), us = __shfl_down_sync(full, vs, o);
                if (lane + o < 32) {
                    vc += uc;
                    vs += us;
                }
            }
            double xc = __shfl_down_sync(full, vc, 1), xs = __shfl_down_sync(full, vs, 1);
            if (lane == 31) xc = xs = 0.0;
            if (b < NB) {
                uend[2 * b] = cc + xc;
                uend[2 * b + 1] = cs + xs;
            }
            cc += __shfl_sync(full, vc, 0);
            cs += __shfl_sync(full, vs, 0);
        }
    }
    __syncwarp();
    // pass 3.  Blocks holding events ("event blocks") are formed one at a time
    // with lane = step: each lane sums the events at its own step (their block
    // offsets are compared four at a time as bytes), then warp scans give the
    // collided sums up to and the uncollided sums after every step.  Blocks
    // without events have constant sums: each lane forms 4 consecutive steps,
    // 8 lanes a block, 4 such blocks at a time (int8 digits: 16 steps, 2 lanes
    // a block, 16 blocks at a time).  The int8 digit layout needs the row's
    // scale, max |beta| over its steps and columns, before any digit: a first
    // sweep forms every value and keeps only the maximum.
    constexpr bool kI8 = std::is_same<Real, int8_t>::value;
    const double ci = A.cos_t[i];
    const double vi = (i == 0 || i == A.n_cos - 1) ? 0.5 : 1.0;
    const double rf = (0.5 * (1.0 - ci * ci) * A.dphi) * (A.dcos * vi) * A.dt * (1.0 / (6.0 * CUDART_PI));
    const long col = (long)(slot / A.bpt) * A.tile_cols + (long)(slot % A.bpt) * 2 * A.S;
    Real* brow = kI8 ? nullptr : beta + (((size_t)frame * A.n_cos + i) * A.cols_pad + col) * A.t_pad;
    const double* Dslot = A.D + (size_t)slot * A.n_t * (1 + SMC);
    const int nbase = (slot % A.bpt) * 2 * A.S;
    int8_t* blk_row =
        kI8 ? reinterpret_cast<int8_t*>(beta) +
                  (((size_t)frame * A.n_cos + i) * A.tiles + slot / A.bpt) * (size_t)NB * kI8BlockSet
            : nullptr;
    // beta of coefficient set s at step k from the sums there: the table row
    // holds the step weight times dt^3 and times a_m dt^{3-p_m} e^{-dt/w}
    auto value = [&](int k, int s, const double* P, double Uc, double Us, double mul, double& xc, double& xs) {
        const double* Dk = Dslot + (size_t)min(k, A.n_t - 1) * (1 + SMC);
        double g[1 + SMC];
        if constexpr ((1 + SMC) % 2 == 0) {
#pragma unroll
            for (int q = 0; q < 1 + SMC; q += 2) {
                const double2 v = __ldg(reinterpret_cast<const double2*>(Dk + q));
                g[q] = v.x;
                g[q + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 1 + SMC; ++q) g[q] = __ldg(Dk + q);
        }
        double vc = g[0] * Uc, vs = g[0] * Us;
        const int t0 = s * A.M, t1 = t0 + A.M;  // the terms of set s
#pragma unroll
        for (int t = 0; t < SMC; ++t) {
            if (t < t0 || t >= t1) continue;
            vc += g[1 + t] * P[2 * t];
            vs += g[1 + t] * P[2 * t + 1];
        }
        const double r = k < A.n_t ? mul : 0.0;
        xc = r * vc;
        xs = r * vs;
    };
    // Collided sums through step (b << 5) + lane and uncollided sums after it, for
    // block b, lane = step (the whole warp calls it with the same b).
    auto step_sums = [&](int b, double (&P)[2 * SMC], double& Uc, double& Us) {
        const int e0 = boff[b], e1 = boff[b + 1];
        if (e0 == e1) {  // a block without events: constant sums
#pragma unroll
            for (int q = 0; q < 2 * SMC; ++q) P[q] = pbeg[(size_t)b * 2 * SMC + q];
            Uc = uend[2 * b];
            Us = uend[2 * b + 1];
            return;
        }
        double dq[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) dq[q] = 0.0;
        if (e1 - e0 > 32) {
            // Many events: the block's events are counting-sorted by their step (stable in event
            // order; ranks within 32 events from __match_any groups), then each lane adds the
            // events of its own step in event order.
            int* run = scnt + 32;
            scnt[lane] = 0;
            __syncwarp();
            for (int r0 = e0; r0 < e1; r0 += 32) {
                const int e = r0 + lane;
                const int se = e < e1 ? (int)evs[e] : 32 + lane;
                const unsigned m = __match_any_sync(full, se);
                if (e < e1 && lane == __ffs(m) - 1) scnt[se] += __popc(m);
                __syncwarp();
            }
            const int c = scnt[lane];
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(full, incl, o);
                if (lane >= o) incl += t;
            }
            const int ex = incl - c;  // first position of this lane's step
            run[lane] = ex;
            __syncwarp();
            const unsigned lt = (1u << lane) - 1u;
            for (int r0 = e0; r0 < e1; r0 += 32) {
                const int e = r0 + lane;
                const bool v = e < e1;
                const int se = v ? (int)evs[e] : 32 + lane;
                const unsigned m = __match_any_sync(full, se);
                if (v) sperm[run[se] + __popc(m & lt)] = (uint16_t)e;
                __syncwarp();
                if (v && lane == __ffs(m) - 1) run[se] += __popc(m);
                __syncwarp();
            }
            for (int r = 0; r < c; ++r) {
                const double* qe = evq + sperm[ex + r];
#pragma unroll
                for (int q = 0; q < NQ; ++q) dq[q] += qe[(size_t)q * EV];
            }
            __syncwarp();
        } else {
            const uint32_t pat = 0x01010101u * (uint32_t)lane;
            for (int e4 = e0 & ~3; e4 < e1; e4 += 4) {
                uint32_t eq = __vcmpeq4(*reinterpret_cast<const uint32_t*>(evs + e4), pat);
                if (e4 < e0) eq &= 0xffffffffu << (8 * (e0 - e4));
                if (e1 - e4 < 4) eq &= (1u << (8 * (e1 - e4))) - 1u;
                while (eq) {
                    const int by = (__ffs(eq) - 1) >> 3;
                    eq &= ~(0xffu << (8 * by));
                    const double* qe = evq + (e4 + by);
#pragma unroll
                    for (int q = 0; q < NQ; ++q) dq[q] += qe[(size_t)q * EV];
                }
            }
        }
        // collided sums through this step (inclusive scan), uncollided after it (suffix scan)
        double uc = dq[0], us = dq[1];
#pragma unroll
        for (int q = 0; q < 2 * SMC; ++q) P[q] = dq[2 + q];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
            for (int q = 0; q < 2 * SMC; ++q) {
                const double v = __shfl_up_sync(full, P[q], o);
                if (lane >= o) P[q] += v;
            }
            const double vc = __shfl_down_sync(full, uc, o), vs = __shfl_down_sync(full, us, o);
            if (lane + o < 32) {
                uc += vc;
                us += vs;
            }
        }
        // uncollided after this step: the next step's inclusive suffix sum
        Uc = __shfl_down_sync(full, uc, 1);
        Us = __shfl_down_sync(full, us, 1);
        if (lane == 31) Uc = Us = 0.0;
        Uc += uend[2 * b];
        Us += uend[2 * b + 1];
#pragma unroll
        for (int q = 0; q < 2 * SMC; ++q) P[q] = pbeg[(size_t)b * 2 * SMC + q] + P[q];
    };
    if constexpr (kI8) {
        // The row's scale is max |beta| over its steps and columns, found exactly without
        // forming every value.
        // (a) Every event block is formed once (lane = step) and its 2S values are kept for the
        //     digits: a block of at least 32 events in its own weight slots (plane 2s + g, slots
        //     boff[b] + lane; its weights are not read again), smaller blocks in the block-total
        //     table while it has room (the rest are formed again in (c)).
        // (b) In a block without events U and Pm are constant, so beta = rf (D0(k) U + sum_m Dm(k)
        //     Pm) is bounded by interval arithmetic over the per-block ranges of the time table;
        //     such blocks are formed (lane = step) in decreasing order of their bound until no
        //     bound exceeds the largest value found (most often one block: the last one, where
        //     dt^3 peaks).
        // (c) Digits of every block.
        double vmax = 0.0;
        const double* Dmx = A.Dmax + (size_t)slot * NB * (1 + SMC) * 2;
        int* where = brun;  // per event block: -1 not kept, -2 own slots, c >= 0 table slot c
        const int n_tab = (NQ * NB) / (64 * A.S);
        int used_tab = 0;
        auto kept = [&](int b, int& stride) -> double* {
            const int w = where[b];
            if (w == -2) {
                stride = EV;
                return evq + boff[b];
            }
            stride = 32;
            return w >= 0 ? btot + (size_t)w * 64 * A.S : nullptr;
        };
        for (int bc = 0; bc < NB; bc += 32) {
            const int bl = bc + lane;
            for (unsigned h = __ballot_sync(full, bl < NB && boff[bl] != boff[bl + 1]); h; h &= h - 1) {
                const int b = bc + __ffs(h) - 1;
                double P[2 * SMC], Uc, Us;
                step_sums(b, P, Uc, Us);
                const int k = (b << 5) + lane;
                const int code = boff[b + 1] - boff[b] >= 32 ? -2 : (used_tab < n_tab ? used_tab++ : -1);
                __syncwarp();
                if (lane == 0) where[b] = code;
                __syncwarp();
                int stride = 0;
                double* dst = kept(b, stride);
                for (int s2 = 0; s2 < A.S; ++s2) {
                    double xc, xs;
                    value(k, s2, P, Uc, Us, rf, xc, xs);
                    vmax = fmax(vmax, fmax(fabs(xc), fabs(xs)));
                    if (dst) {
                        dst[(size_t)(2 * s2) * stride + lane] = xc;
                        dst[(size_t)(2 * s2 + 1) * stride + lane] = xs;
                    }
                }
                __syncwarp();
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(full, vmax, o));
        for (int bc = 0; bc < NB; bc += 32) {
            const int bl = bc + lane;
            double bnd = -1.0;  // this lane's block's bound (-1: none or an event block)
            if (bl < NB && boff[bl] == boff[bl + 1]) {
                // beta of set s, column g lies in rf (D0 [U] + sum_m Dm [Pm]) with D in [min, max]
                // over the block and U, Pm the block's constants
                const double* mx = Dmx + (size_t)bl * (1 + SMC) * 2;
                auto term = [&](double dlo, double dhi, double c, double& lo, double& hi, double& sa) {
                    const double p0 = dlo * c, p1 = dhi * c;
                    lo += fmin(p0, p1);
                    hi += fmax(p0, p1);
                    sa += fmax(fabs(dlo), fabs(dhi)) * fabs(c);
                };
                for (int s2 = 0; s2 < A.S; ++s2) {
                    const int t0 = s2 * A.M, t1 = t0 + A.M;
#pragma unroll
                    for (int g = 0; g < 2; ++g) {
                        double lo = 0.0, hi = 0.0, sa = 0.0;
                        term(mx[0], mx[1], uend[2 * bl + g], lo, hi, sa);
#pragma unroll
                        for (int q = 0; q < SMC; ++q)
                            if (q >= t0 && q < t1)
                                term(mx[2 + 2 * q], mx[3 + 2 * q], pbeg[(size_t)bl * 2 * SMC + 2 * q + g], lo, hi, sa);
                        // relative and absolute margins cover the rounding of these sums and of
                        // the values themselves (a few ulp of the summed magnitudes)
                        bnd = fmax(bnd, (fmax(fabs(lo), fabs(hi)) * (1.0 + 1e-12) + 1e-13 * sa) * rf);
                    }
                }
            }
            for (;;) {
                double bb = bnd;
                int bi = lane;
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(full, bb, o);
                    const int oi = __shfl_xor_sync(full, bi, o);
                    if (ob > bb || (ob == bb && oi < bi)) {
                        bb = ob;
                        bi = oi;
                    }
                }
                // Every remaining bound is covered once no bound exceeds vmax (1 + 1e-10): a value up
                // to that much above the scale still maps to |x F| <= F + 0.22, which rounds into the
                // digit range.  (Without the slack, blocks whose values all equal the maximum, as after
                // the last collision with powers = 3, would each be formed.)
                if (!(bb > vmax * (1.0 + 1e-10))) break;
                {
                    const int b = bc + bi, k = (b << 5) + lane;
                    const double* P = pbeg + (size_t)b * 2 * SMC;
                    const double Uc = uend[2 * b], Us = uend[2 * b + 1];
                    double m = 0.0;
                    for (int s2 = 0; s2 < A.S; ++s2) {
                        double xc, xs;
                        value(k, s2, P, Uc, Us, rf, xc, xs);
                        m = fmax(m, fmax(fabs(xc), fabs(xs)));
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(full, m, o));
                    vmax = fmax(vmax, m);
                }
                if (lane == bi) bnd = -1.0;
            }
        }
        if (lane == 0) A.scale[row] = vmax;
        const double inv = vmax > 0.0 ? 1.0 / vmax : 0.0;
        const double rinv = rf * inv;
        // digits (streaming stores: the GEMM reads them back from DRAM).  Event blocks: lane = step; a
        // quad of lanes transposes its packed digit
        // words so that lane 4q + d holds digit d of steps 4q .. 4q + 3.  Blocks without
        // events: 4 steps per lane (8 lanes a block, 4 blocks at a time), transposed in
        // registers.  Either way a store instruction fills whole 32-byte rows of the blocks.
        const bool odd = lane & 1, hi = lane & 2;
        auto quad_transpose = [&](uint32_t p) {
            const uint32_t t1 = __shfl_xor_sync(full, p, 1);
            p = __byte_perm(p, t1, odd ? 0x3715 : 0x6240);
            const uint32_t t2 = __shfl_xor_sync(full, p, 2);
            return __byte_perm(p, t2, hi ? 0x3276 : 0x5410);
        };
        const int dg = lane & 3, s4 = (lane >> 2) * 4;
        for (int bc = 0; bc < NB; bc += 32) {
            const int bl = bc + lane;
            const bool has = bl < NB && boff[bl] != boff[bl + 1];
            const unsigned ev_blocks = __ballot_sync(full, has);
            unsigned quiet = __ballot_sync(full, bl < NB && !has);
            for (unsigned h = ev_blocks; h; h &= h - 1) {
                const int b = bc + __ffs(h) - 1;
                const int k = (b << 5) + lane;
                int stride = 0;
                const double* src = kept(b, stride);
                double P[2 * SMC], Uc = 0.0, Us = 0.0;
                if (!src) step_sums(b, P, Uc, Us);
                int8_t* blk = blk_row + (size_t)b * kI8BlockSet + dg * kI8Block;
                for (int s2 = 0; s2 < A.S; ++s2) {
                    double xc, xs;
                    if (src) {
                        xc = src[(size_t)(2 * s2) * stride + lane];
                        xs = src[(size_t)(2 * s2 + 1) * stride + lane];
                    } else {
                        value(k, s2, P, Uc, Us, rf, xc, xs);
                    }
                    const uint32_t wc = quad_transpose(i8_digits(xc * inv));
                    const uint32_t ws = quad_transpose(i8_digits(xs * inv));
                    __stcs(reinterpret_cast<unsigned int*>(blk + i8_swz(nbase + 2 * s2, s4)), wc);
                    __stcs(reinterpret_cast<unsigned int*>(blk + i8_swz(nbase + 2 * s2 + 1, s4)), ws);
                }
            }
            const int sub = lane >> 3, s0 = (lane & 7) * 4;
            while (quiet) {
                unsigned t = quiet;
                for (int g = 0; g < sub && t; ++g) t &= t - 1;
                const int b = t ? bc + __ffs(t) - 1 : -1;
                for (int g = 0; g < 4 && quiet; ++g) quiet &= quiet - 1;
                if (b < 0) continue;
                const int k0 = (b << 5) + s0;
                // the block's constant sums, with rf / scale folded in: 1 + SMC products per
                // value (steps past n_t, in the last block only, go through value())
                const bool tail = k0 + 4 > A.n_t;
                double P[2 * SMC];
#pragma unroll
                for (int q = 0; q < 2 * SMC; ++q) P[q] = rinv * pbeg[(size_t)b * 2 * SMC + q];
                const double Uc = rinv * uend[2 * b], Us = rinv * uend[2 * b + 1];
                const double* Db = Dslot + (size_t)k0 * (1 + SMC);
                int8_t* blk = blk_row + (size_t)b * kI8BlockSet;
                for (int s2 = 0; s2 < A.S; ++s2) {
                    uint32_t pc[4], ps[4];
                    const int t0 = s2 * A.M, t1 = t0 + A.M;  // the terms of set s2
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        double xc, xs;
                        if (tail) {
                            value(k0 + m, s2, P, Uc, Us, 1.0, xc, xs);
                        } else {
                            const double* Dk = Db + (size_t)m * (1 + SMC);
                            double g[1 + SMC];
                            if constexpr ((1 + SMC) % 2 == 0) {
#pragma unroll
                                for (int q = 0; q < 1 + SMC; q += 2) {
                                    const double2 v = __ldg(reinterpret_cast<const double2*>(Dk + q));
                                    g[q] = v.x;
                                    g[q + 1] = v.y;
                                }
                            } else {
#pragma unroll
                                for (int q = 0; q < 1 + SMC; ++q) g[q] = __ldg(Dk + q);
                            }
                            xc = g[0] * Uc;
                            xs = g[0] * Us;
#pragma unroll
                            for (int q = 0; q < SMC; ++q) {
                                if (SMC > 1 && (q < t0 || q >= t1)) continue;
                                xc = fma(g[1 + q], P[2 * q], xc);
                                xs = fma(g[1 + q], P[2 * q + 1], xs);
                            }
                        }
                        pc[m] = i8_digits(xc);
                        ps[m] = i8_digits(xs);
                    }
                    uint32_t wc[4], ws[4];
                    i8_transpose4(pc[0], pc[1], pc[2], pc[3], wc);
                    i8_transpose4(ps[0], ps[1], ps[2], ps[3], ws);
                    const int oc = i8_swz(nbase + 2 * s2, s0), os = i8_swz(nbase + 2 * s2 + 1, s0);
#pragma unroll
                    for (int d = 0; d < kI8Slices; ++d) {
                        __stcs(reinterpret_cast<unsigned int*>(blk + d * kI8Block + oc), wc[d]);
                        __stcs(reinterpret_cast<unsigned int*>(blk + d * kI8Block + os), ws[d]);
                    }
                }
            }
        }
    } else {
        for (int bc = 0; bc < NB; bc += 32) {
            const int bl = bc + lane;
            const bool has = bl < NB && boff[bl] != boff[bl + 1];
            const unsigned ev_blocks = __ballot_sync(full, has);
            unsigned quiet = __ballot_sync(full, bl < NB && !has);
            // ---- event blocks, lane = step
            for (unsigned h = ev_blocks; h; h &= h - 1) {
                const int b = bc + __ffs(h) - 1;
                double P[2 * SMC], Uc, Us;
                step_sums(b, P, Uc, Us);
                const int k = (b << 5) + lane;
                for (int s2 = 0; s2 < A.S; ++s2) {
                    double xc, xs;
                    value(k, s2, P, Uc, Us, rf, xc, xs);
                    if (k < A.t_pad) {
                        brow[(size_t)(2 * s2) * A.t_pad + k] = (Real)xc;
                        brow[(size_t)(2 * s2 + 1) * A.t_pad + k] = (Real)xs;
                    }
                }
            }
            // ---- blocks without events, 4 steps per lane
            const int sub = lane >> 3, s0 = (lane & 7) * 4;
            while (quiet) {
                unsigned t = quiet;
                for (int g = 0; g < sub && t; ++g) t &= t - 1;
                const int b = t ? bc + __ffs(t) - 1 : -1;
                for (int g = 0; g < 4 && quiet; ++g) quiet &= quiet - 1;
                if (b < 0) continue;
                const double* P = pbeg + (size_t)b * 2 * SMC;
                const double Uc = uend[2 * b], Us = uend[2 * b + 1];
                const int k0 = (b << 5) + s0;
                for (int s2 = 0; s2 < A.S; ++s2) {
                    double xc[4], xs[4];
#pragma unroll
                    for (int m = 0; m < 4; ++m) value(k0 + m, s2, P, Uc, Us, rf, xc[m], xs[m]);
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        const int k = k0 + m;
                        if (k < A.t_pad) {
                            brow[(size_t)(2 * s2) * A.t_pad + k] = (Real)xc[m];
                            brow[(size_t)(2 * s2 + 1) * A.t_pad + k] = (Real)xs[m];
                        }
                    }
                }
            }
        }
    }
}

template <class Real, int SMC>
static void launch_beta_smc(const BetaArgs& B, Real* out, size_t smem, unsigned blocks, int threads,
                            cudaStream_t st) {
    CUDA_OK(cudaFuncSetAttribute(k_beta<Real, SMC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // three blocks per SM need the largest shared-memory carveout; without the preference the
    // driver may pick a smaller one (two blocks per SM) depending on the kernels run before
    CUDA_OK(cudaFuncSetAttribute(k_beta<Real, SMC>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    k_beta<Real, SMC><<<blocks, threads, smem, st>>>(B, out);
}

template <class Real>
static void launch_beta(int SM, const BetaArgs& B, Real* out, size_t smem, unsigned blocks, int threads,
                        cudaStream_t st) {
    switch (SM) {
        case 1: launch_beta_smc<Real, 1>(B, out, smem, blocks, threads, st); break;
        case 2: launch_beta_smc<Real, 2>(B, out, smem, blocks, threads, st); break;
        case 3: launch_beta_smc<Real, 3>(B, out, smem, blocks, threads, st); break;
        case 4: launch_beta_smc<Real, 4>(B, out, smem, blocks, threads, st); break;
        case 5: launch_beta_smc<Real, 5>(B, out, smem, blocks, threads, st); break;
        case 6: launch_beta_smc<Real, 6>(B, out, smem, blocks, threads, st); break;
        case 7: launch_beta_smc<Real, 7>(B, out, smem, blocks, threads, st); break;
        case 8: launch_beta_smc<Real, 8>(B, out, smem, blocks, threads, st); break;
        default: throw Error{"at most 8 (set, term) pairs in the factored kernels"};
    }
}

// ---------------------------------------------------------------------------
struct FactArgs {
    const D4* bub;  // rotated frames (kn, n_tot)
    size_t n_tot;
    const uint32_t* sel;
    int n_sel;
    int n_cos, n_t, n_w;
    int S;
    const double* t_arr;
    const double* w;
    const double* cos_t;
    const int* kfirst;     // (n_sel)
    const void* beta;      // (kn, n_cos, cols_pad, t_pad) Real
    long cols_pad;
    int t_pad;
    double dt;
    int bpt;               // bubbles per column tile
    int tiles_per_frame;
    double2* partial;      // (kn, tiles_per_frame, 2, S, W)
};

// One CTA per (64-frequency tile, column tile), looping over the rows i.
// Thread (ty, tx) of 16 x 16 owns rows ty*8 .. ty*8+7 (frequencies ty*4 .. +3,
// Re/Im interleaved) and TN columns in two groups of TN/2: tx*TN/2 + u and
// COLS/2 + tx*TN/2 + u, so that consecutive threads read consecutive 16-byte
// words of a beta-tile row (no shared-memory bank conflicts).
template <int TN, int COLS>
__device__ __forceinline__ int thread_col(int tx, int u) {
    return u < TN / 2 ? tx * (TN / 2) + u : COLS / 2 + tx * (TN / 2) + (u - TN / 2);
}

template <class Real, int TN>
__global__ void __launch_bounds__(kThreads, 1) k_gemm(FactArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int COLS = 16 * TN;                                  // 128 (FP32) or 64 (FP64)
    constexpr int BS = COLS + 16 / (int)sizeof(Real);              // padded row of the beta tile
    constexpr int VEC = 16 / (int)sizeof(Real);                    // elements per 16-byte load
    constexpr int NPRE = COLS * kKC / VEC / kThreads;              // 16-byte loads per thread per tile
    Real* Msm = reinterpret_cast<Real*>(smem);                     // [kKC][kRows]
    Real* Bsm = Msm + kKC * kRows;                                 // [kKC][BS]
    double* Pn_re = reinterpret_cast<double*>(Bsm + kKC * BS);      // [kKC][kWT]
    double* Pn_im = Pn_re + kKC * kWT;
    double* anc = Pn_im + kKC * kWT;                               // [2][kWT]
    double2* red = reinterpret_cast<double2*>(anc + 2 * kWT);       // [kThreads][4][2S]
    double2* Cacc = red + kThreads * 4 * 2 * A.S;                  // [kWT][2S]
    int* binfo = reinterpret_cast<int*>(Cacc + kWT * 2 * A.S);      // [bpt]: slot or -1
    double* bt = reinterpret_cast<double*>(binfo + 64);            // [bpt] t_a
    double* bz = bt + 64;                                          // [bpt] z_a

    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;
    const int w0 = blockIdx.x * kWT;
    const int frame = blockIdx.y / A.tiles_per_frame;
    const int tile = blockIdx.y % A.tiles_per_frame;
    const int cpb = 2 * A.S;  // columns per bubble
    const D4* B = A.bub + (size_t)frame * A.n_tot;
    const Real* beta = static_cast<const Real*>(A.beta);

    if (tid < 64) {
        const int slot = tile * A.bpt + tid;
        const bool ok = tid < A.bpt && slot < A.n_sel && A.sel[slot] != kNoSlot;
        binfo[tid] = ok ? slot : -1;
        if (ok) {
            const D4 xa = B[A.sel[slot]];
            bt[tid] = xa.t;
            bz[tid] = xa.z;
        }
    }
    for (int q = tid; q < kWT * cpb; q += kThreads) Cacc[q] = make_double2(0.0, 0.0);
    __syncthreads();
    int kstart = A.n_t;
    for (int b = 0; b < A.bpt; ++b)
        if (binfo[b] >= 0) kstart = min(kstart, A.kfirst[binfo[b]]);
    const int c_start = kstart / kKC;
    const int n_chunks = (A.n_t + kKC - 1) / kKC;
    const long col0 = (long)tile * COLS;

    for (int i = 0; i < A.n_cos; ++i) {
        const double ci = A.cos_t[i];
        const double one_m_c = 1.0 - ci;
        for (int q = tid; q < kKC * kWT; q += kThreads) {
            const int n = q / kWT, wl = q % kWT;
            const int wi = w0 + wl;
            double sn = 0.0, cs = 1.0;
            if (wi < A.n_w) phase<Real>(A.w[wi] * one_m_c * (n * A.dt), sn, cs);
            Pn_re[q] = cs;
            Pn_im[q] = sn;
        }
        const Real* bi = beta + (((size_t)frame * A.n_cos + i) * A.cols_pad + col0) * A.t_pad;
        // 16-byte loads of the beta tile: column q / (kKC/VEC), steps VEC*(q % (kKC/VEC)) ...
        using Vec = typename std::conditional<sizeof(Real) == 4, float4, double2>::type;
        Vec pre[NPRE];
        auto fetch = [&](int k0) {
#pragma unroll
            for (int v = 0; v < NPRE; ++v) {
                const int q = tid + v * kThreads;
                const int col = q / (kKC / VEC), n = (q % (kKC / VEC)) * VEC;
                const int k = k0 + n;  // t_pad is a multiple of VEC: a load is all in or all out
                if (k < A.t_pad) pre[v] = __ldg(reinterpret_cast<const Vec*>(bi + (size_t)col * A.t_pad + k));
                else pre[v] = Vec{};
            }
        };
        double acc[kTM][TN];
#pragma unroll
        for (int r = 0; r < kTM; ++r)
#pragma unroll
            for (int u = 0; u < TN; ++u) acc[r][u] = 0.0;
        if (c_start < n_chunks) fetch(c_start * kKC);
        __syncthreads();

        for (int ch = c_start; ch < n_chunks; ++ch) {
            const int k0 = ch * kKC;
            if (tid < kWT) {
                const int wi = w0 + tid;
                double sn = 0.0, cs = 0.0;
                if (wi < A.n_w) phase<Real>(A.w[wi] * one_m_c * A.t_arr[k0], sn, cs);
                anc[tid] = cs;
                anc[kWT + tid] = sn;
            }
#pragma unroll
            for (int v = 0; v < NPRE; ++v) {
                const int q = tid + v * kThreads;
                const int col = q / (kKC / VEC), n = (q % (kKC / VEC)) * VEC;
                const Real* pv = reinterpret_cast<const Real*>(&pre[v]);
#pragma unroll
                for (int e = 0; e < VEC; ++e) Bsm[(n + e) * BS + col] = pv[e];
            }
            __syncthreads();
            for (int q = tid; q < kKC * kWT; q += kThreads) {
                const int n = q / kWT, wl = q % kWT;
                const double ar = anc[wl], ai = anc[kWT + wl];
                const double pr = Pn_re[q], pi = Pn_im[q];
                const bool valid = k0 + n < A.n_t;
                Msm[n * kRows + 2 * wl] = valid ? (Real)(ar * pr - ai * pi) : (Real)0;
                Msm[n * kRows + 2 * wl + 1] = valid ? (Real)(ar * pi + ai * pr) : (Real)0;
            }
            __syncthreads();
            if (ch + 1 < n_chunks) fetch(k0 + kKC);  // in flight during the GEMM below
            if constexpr (sizeof(Real) == 8) {
#pragma unroll 4
                for (int n = 0; n < kKC; ++n) {
                    double a[kTM], bb[TN];
                    const double2* ap = reinterpret_cast<const double2*>(Msm + n * kRows + ty * kTM);
                    const double2* bp0 = reinterpret_cast<const double2*>(Bsm + n * BS + tx * (TN / 2));
                    const double2* bp1 = reinterpret_cast<const double2*>(Bsm + n * BS + COLS / 2 + tx * (TN / 2));
#pragma unroll
                    for (int r = 0; r < kTM / 2; ++r) {
                        const double2 v = ap[r];
                        a[2 * r] = v.x;
                        a[2 * r + 1] = v.y;
                    }
#pragma unroll
                    for (int u = 0; u < TN / 4; ++u) {
                        const double2 v0 = bp0[u], v1 = bp1[u];
                        bb[2 * u] = v0.x;
                        bb[2 * u + 1] = v0.y;
                        bb[TN / 2 + 2 * u] = v1.x;
                        bb[TN / 2 + 2 * u + 1] = v1.y;
                    }
#pragma unroll
                    for (int r = 0; r < kTM; ++r)
#pragma unroll
                        for (int u = 0; u < TN; ++u) acc[r][u] = fma(a[r], bb[u], acc[r][u]);
                }
            } else {
#pragma unroll 1
                for (int n0 = 0; n0 < kKC; n0 += kFold) {
                    float cacc[kTM][TN];
#pragma unroll
                    for (int r = 0; r < kTM; ++r)
#pragma unroll
                        for (int u = 0; u < TN; ++u) cacc[r][u] = 0.0f;
#pragma unroll
                    for (int n = n0; n < n0 + kFold; ++n) {
                        float a[kTM], bb[TN];
                        const float4* ap = reinterpret_cast<const float4*>(Msm + n * kRows + ty * kTM);
                        const float4 b0 = *reinterpret_cast<const float4*>(Bsm + n * BS + tx * (TN / 2));
                        const float4 b1 = *reinterpret_cast<const float4*>(Bsm + n * BS + COLS / 2 + tx * (TN / 2));
#pragma unroll
                        for (int r = 0; r < kTM / 4; ++r) {
                            const float4 v = ap[r];
                            a[4 * r] = v.x;
                            a[4 * r + 1] = v.y;
                            a[4 * r + 2] = v.z;
                            a[4 * r + 3] = v.w;
                        }
                        bb[0] = b0.x;
                        bb[1] = b0.y;
                        bb[2] = b0.z;
                        bb[3] = b0.w;
                        bb[4] = b1.x;
                        bb[5] = b1.y;
                        bb[6] = b1.z;
                        bb[7] = b1.w;
#pragma unroll
                        for (int r = 0; r < kTM; ++r)
#pragma unroll
                            for (int u = 0; u < TN; ++u) cacc[r][u] = fmaf(a[r], bb[u], cacc[r][u]);
                    }
#pragma unroll
                    for (int r = 0; r < kTM; ++r)
#pragma unroll
                        for (int u = 0; u < TN; ++u) acc[r][u] += (double)cacc[r][u];
                }
            }
            __syncthreads();
        }
        // epilogue: per thread, C_{s,g}(w) partials of its columns in fixed order
        // partials in structure-of-arrays order red[(q*cpb + sg)*kThreads + tid]
        for (int q = 0; q < 4 * cpb; ++q) red[(size_t)q * kThreads + tid] = make_double2(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < kTM / 2; ++q) {
            const int wl = ty * (kTM / 2) + q;
            const int wi = w0 + wl;
#pragma unroll
            for (int u = 0; u < TN; ++u) {
                const int col = thread_col<TN, COLS>(tx, u);
                const int b = col / cpb;
                if (b >= A.bpt || binfo[b] < 0 || wi >= A.n_w) continue;
                double sn, cs;
                phase<Real>(A.w[wi] * (bt[b] * ci - bz[b]), sn, cs);
                const double yr = acc[2 * q][u], yi = acc[2 * q + 1][u];
                double2& d = red[(size_t)(q * cpb + (col % cpb)) * kThreads + tid];
                d.x += cs * yr - sn * yi;
                d.y += cs * yi + sn * yr;
            }
        }
        __syncthreads();
        for (int q = tid; q < kWT * cpb; q += kThreads) {
            const int wl = q / cpb, sg = q % cpb;
            const int tyw = wl / (kTM / 2), qq = wl % (kTM / 2);
            double2 sum = Cacc[q];
            for (int t = 0; t < 16; ++t) {
                const double2 v = red[(size_t)(qq * cpb + sg) * kThreads + tyw * 16 + t];
                sum.x += v.x;
                sum.y += v.y;
            }
            Cacc[q] = sum;
        }
        __syncthreads();
    }
    for (int q = tid; q < kWT * cpb; q += kThreads) {
        const int wl = q / cpb, sg = q % cpb;
        const int s = sg >> 1, g = sg & 1;
        const int wi = w0 + wl;
        if (wi >= A.n_w) continue;
        const size_t o = ((((size_t)frame * A.tiles_per_frame + tile) * 2 + g) * A.S + s) * A.n_w + wi;
        A.partial[o] = Cacc[q];
    }
}

__global__ void k_reduce_tiles(const double2* __restrict__ partial, int tiles, size_t per, int kn,
                               double2* __restrict__ out) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (q >= per || k >= kn) return;
    double2 acc = make_double2(0.0, 0.0);
    const double2* p = partial + (size_t)k * tiles * per + q;
    for (int t = 0; t < tiles; ++t) {
        const double2 v = p[(size_t)t * per];
        acc.x += v.x;
        acc.y += v.y;
    }
    out[(size_t)k * per + q] = acc;
}

// Batched jobs: frame k of realization r is the sum of its own column tiles'
// partials, in the order of k_reduce_tiles (tiles, then row parts).
__global__ void k_reduce_real(const double2* __restrict__ partial, const uint32_t* __restrict__ real_tiles,
                              int tiles_per_frame, int parts, size_t per, int kn, size_t n_k, size_t k0,
                              double2* __restrict__ out) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    const int r = blockIdx.z;
    if (q >= per || k >= kn) return;
    double2 acc = make_double2(0.0, 0.0);
    const double2* p = partial + (size_t)k * tiles_per_frame * parts * per + q;
    for (size_t t = (size_t)real_tiles[r] * parts; t < (size_t)real_tiles[r + 1] * parts; ++t) {
        const double2 v = p[t * per];
        acc.x += v.x;
        acc.y += v.y;
    }
    out[((size_t)r * n_k + k0 + k) * per + q] = acc;
}

// ---------------------------------------------------------------------------
template <class Real, int TN>
static size_t gemm_smem_bytes(int S) {
    constexpr int COLS = 16 * TN;
    constexpr int BS = COLS + 16 / (int)sizeof(Real);
    size_t b = (size_t)kKC * kRows * sizeof(Real) + (size_t)kKC * BS * sizeof(Real);
    b = (b + 15) & ~(size_t)15;
    b += 2 * (size_t)kKC * kWT * sizeof(double);   // step table
    b += 2 * (size_t)kWT * sizeof(double);         // anchors
    b += (size_t)kThreads * 4 * 2 * S * sizeof(double2);  // epilogue partials
    b += (size_t)kWT * 2 * S * sizeof(double2);    // C accumulator
    b += 64 * sizeof(int) + 2 * 64 * sizeof(double);
    return b;
}

template <class Real>
constexpr int gemm_tn() { return sizeof(Real) == 4 ? 8 : 4; }

struct FactGeom {
    int bpt, tiles_per_frame, t_pad, nblk, tile_cols;
    long cols_pad;
};

// real_size: 8 (FP64 GEMM, 64-column tiles), 4 (FP32 GEMM) or 1 (int8 tensor-core GEMM), 128-column tiles
static FactGeom fact_geom(const SpectrumJob& job, size_t real_size) {
    FactGeom g;
    const int S = (int)job.n_sets;
    const int cols = real_size == 8 ? 64 : 128;
    g.tile_cols = cols;
    g.bpt = std::min(64, cols / (2 * S));
    g.tiles_per_frame = (int)((job.n_sel + g.bpt - 1) / g.bpt);
    g.cols_pad = (long)g.tiles_per_frame * cols;  // every tile is `cols` wide; unused columns stay zero
    const int align = real_size == 4 ? 4 : 2;
    g.t_pad = (int)((job.n_t + align - 1) / align * align);
    g.nblk = (int)((job.n_t + 31) / 32);
    return g;
}

// Sums the column-tile partials of kn frames: per frame (single job) or per
// (realization, frame) (batched job).
static uint64_t reduce_tiles(Device* dev, const SpectrumJob& job, const double2* partial, int tiles_per_frame,
                             int parts, size_t per, size_t k0, size_t kn, double2* out, const uint32_t* real_tiles) {
    if (job.n_real > 0) {
        if (job.n_real > 65535) throw Error{"too many realizations in one batched call"};
        dim3 gr((unsigned)((per + 255) / 256), (unsigned)kn, (unsigned)job.n_real);
        k_reduce_real<<<gr, 256, 0, dev->stream>>>(partial, real_tiles, tiles_per_frame, parts, per, (int)kn,
                                                   job.n_k, k0, out);
    } else {
        dim3 gr((unsigned)((per + 255) / 256), (unsigned)kn);
        k_reduce_tiles<<<gr, 256, 0, dev->stream>>>(partial, tiles_per_frame * parts, per, (int)kn, out + k0 * per);
    }
    CUDA_OK(cudaGetLastError());
    return 1;
}

template <class Real>
static uint64_t launch_typed(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                             const double* tau, const double* cos_t, const double* sin2, const double* cos2,
                             const double* coeffs, const double* powers, const double* t_arr, const double* cutw,
                             const double* w, size_t k0, size_t kn, double2* out, const uint32_t* real_tiles,
                             cudaEvent_t* ev3) {
    const int S = (int)job.n_sets, M = (int)job.n_terms, SM = S * M;
    const int n_t = (int)job.n_t, n_cos = (int)job.n_cos, n_phi = (int)job.n_phi, n_w = (int)job.n_w;
    const int n_sel = (int)job.n_sel;
    constexpr bool tc = std::is_same<Real, int8_t>::value;
    if (SM > 8 || 2 * S > (sizeof(Real) == 8 ? 64 : 128))
        throw Error{"the factored kernels support at most 8 (set, term) pairs; use the fp64_direct kernel"};
    if (job.has_damping) {
        const double span = job.t_arr[job.n_t - 1] - job.t_arr[0] + 4.0;
        if (!(std::fabs(span / job.damping) < 600.0))
            throw Error{"damping width too small for the factored kernels (exp overflow); use fp64_direct"};
    }
    const FactGeom G = fact_geom(job, sizeof(Real));
    uint64_t launches = 0;
    // per-bubble time tables (frame independent)
    dev->fact_D.ensure((size_t)n_sel * n_t * (1 + SM) * sizeof(double));
    dev->fact_kfirst.ensure((size_t)n_sel * sizeof(int));
    if ((n_t + 127) / 128 > 65535) throw Error{"too many time steps for the time-table grid"};
    {
        dim3 g((unsigned)n_sel, (unsigned)((n_t + 127) / 128));
        k_time_tables<<<g, 128, 0, dev->stream>>>(bub_frames, sel, n_sel, t_arr, n_t, powers, coeffs, cutw, SM,
                                                  job.has_damping ? 1 : 0, job.damping, (double*)dev->fact_D.p,
                                                  (int*)dev->fact_kfirst.p);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    // beta
    record_event(dev, ev3[0]);
    const int nkb = G.nblk;
    const size_t beta_elems = tc ? (size_t)kn * n_cos * G.tiles_per_frame * nkb * kI8BlockSet
                                 : (size_t)kn * n_cos * G.cols_pad * G.t_pad;
    if (tc) {
        // row scales, and the per-block maxima of the time table that bound them
        dev->beta_scale.ensure((size_t)kn * n_sel * n_cos * sizeof(double));
        dev->fact_Dmax.ensure((size_t)n_sel * nkb * (1 + SM) * 2 * sizeof(double));
        const long warps = (long)n_sel * nkb;
        k_time_maxima<<<(unsigned)((warps + 7) / 8), 256, 0, dev->stream>>>((const double*)dev->fact_D.p, n_sel, n_t,
                                                                            nkb, 1 + SM, (double*)dev->fact_Dmax.p);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    dev->beta.ensure(beta_elems * sizeof(Real));
    if ((long)n_sel * 2 * S != G.cols_pad) {  // unused tile columns must read as zero
        // padding columns of the last tile are read by the GEMM: keep them zero
        CUDA_OK(cudaMemsetAsync(dev->beta.p, 0, beta_elems * sizeof(Real), dev->stream));
    }
    {
        BetaArgs B;
        B.tau = tau;
        B.bub = bub_frames;
        B.sel = sel;
        B.n_sel = n_sel;
        B.n_cos = n_cos;
        B.n_phi = n_phi;
        B.n_t = n_t;
        B.S = S;
        B.M = M;
        B.t_arr = t_arr;
        B.cutw = cutw;
        B.cos_t = cos_t;
        B.cos2 = cos2;
        B.sin2 = sin2;
        B.powers = powers;
        B.coeffs = coeffs;
        B.D = (const double*)dev->fact_D.p;
        B.has_damp = job.has_damping ? 1 : 0;
        B.damp = job.damping;
        B.dphi = 2.0 * M_PI / (double)n_phi;
        B.dcos = 2.0 / (double)(n_cos - 1);
        B.dt = job.dt;
        B.n_rows = (long)kn * n_sel * n_cos;
        B.nblk = G.nblk;
        B.cols_pad = G.cols_pad;
        B.tile_cols = G.tile_cols;
        B.bpt = G.bpt;
        B.t_pad = G.t_pad;
        const int NQ = 2 + 2 * SM;
        size_t pw = (size_t)n_phi * NQ * sizeof(double) + 2 * (size_t)NQ * G.nblk * sizeof(double) +
                    (2 * (size_t)G.nblk + 1) * sizeof(int) + (((size_t)n_phi + 4 + 3) & ~(size_t)3) +
                    64 * sizeof(int) + (size_t)n_phi * sizeof(uint16_t);
        pw = (pw + 15) & ~(size_t)15;
        B.per_warp_bytes = (int)pw;
        B.tiles = G.tiles_per_frame;
        B.scale = tc ? (double*)dev->beta_scale.p : nullptr;
        B.Dmax = tc ? (const double*)dev->fact_Dmax.p : nullptr;
        int warps = (int)std::min<size_t>(8, (200 * 1024) / pw);
        if (warps < 1) throw Error{"n_phi too large for the beta kernel"};
        const size_t smem = (size_t)warps * pw;
        const unsigned blocks = (unsigned)((B.n_rows + warps - 1) / warps);
        launch_beta<Real>(SM, B, (Real*)dev->beta.p, smem, blocks, warps * 32, dev->stream);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    // GEMM + epilogue
    record_event(dev, ev3[1]);
    FactArgs A;
    A.bub = bub_frames;
    A.n_tot = job.n_tot;
    A.sel = sel;
    A.n_sel = n_sel;
    A.n_cos = n_cos;
    A.n_t = n_t;
    A.n_w = n_w;
    A.S = S;
    A.t_arr = t_arr;
    A.w = w;
    A.cos_t = cos_t;
    A.kfirst = (const int*)dev->fact_kfirst.p;
    A.beta = dev->beta.p;
    A.cols_pad = G.cols_pad;
    A.t_pad = G.t_pad;
    A.dt = job.dt;
    A.bpt = G.bpt;
    A.tiles_per_frame = G.tiles_per_frame;
    const size_t per = (size_t)2 * S * n_w;
    // tensor-core path: each column tile's CTAs split the cos-theta rows so that
    // the grid fills whole waves of one CTA per SM
    const int row_parts =
        !tc ? 1
            : job.row_parts > 0 ? std::min(std::min(job.row_parts, 16), n_cos)
                                : tc_row_parts((size_t)((n_w + 63) / 64) * kn * G.tiles_per_frame, n_cos, dev->n_sm);
    dev->last_row_parts = row_parts;
    dev->fact_partial.ensure((size_t)kn * G.tiles_per_frame * row_parts * per * sizeof(double2));
    A.partial = (double2*)dev->fact_partial.p;
    if constexpr (tc) {
        // time-phase digits: frame independent, built by the first launch chunk of each call
        // (0.8 ms at config 3) and reused by the others
        const int n_wt = (n_w + 63) / 64;
        const size_t atab_bytes = (size_t)n_cos * n_wt * nkb * kI8BlockSet;
        if (!dev->tc_atab_valid || dev->tc_atab.cap < atab_bytes) {
            dev->tc_atab.ensure(atab_bytes);
            launch_tc_phase_table(w, cos_t, t_arr, n_cos, n_w, n_t, (int8_t*)dev->tc_atab.p, dev->stream);
            ++launches;
            dev->tc_atab_valid = true;
        }
        TcArgs T;
        T.bub = bub_frames;
        T.n_tot = job.n_tot;
        T.sel = sel;
        T.n_sel = n_sel;
        T.n_cos = n_cos;
        T.n_t = n_t;
        T.n_w = n_w;
        T.S = S;
        T.w = w;
        T.cos_t = cos_t;
        T.kfirst = (const int*)dev->fact_kfirst.p;
        T.atab = (const int8_t*)dev->tc_atab.p;
        T.btab = (const int8_t*)dev->beta.p;
        T.bscale = (const double*)dev->beta_scale.p;
        T.n_wt = n_wt;
        T.nkb = nkb;
        T.bpt = G.bpt;
        T.tiles_per_frame = G.tiles_per_frame;
        T.row_parts = row_parts;
        T.stages = job.gemm_stages > 0 ? job.gemm_stages : 4;
        dev->last_gemm_stages = T.stages;
        T.partial = A.partial;
        T.err = reinterpret_cast<unsigned int*>(static_cast<unsigned char*>(dev->counters.p) + 8);
        launch_gemm_tc(T, kn, dev->stream);
        ++launches;
        record_event(dev, ev3[2]);
        launches += reduce_tiles(dev, job, A.partial, G.tiles_per_frame, row_parts, per, k0, kn, out, real_tiles);
        return launches;
    } else {
        constexpr int TN = gemm_tn<Real>();
        const size_t smem = gemm_smem_bytes<Real, TN>(S);
        if (smem > 227 * 1024) throw Error{"too many coefficient sets for the factored kernel's shared memory"};
        CUDA_OK(cudaFuncSetAttribute(k_gemm<Real, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const size_t gy = (size_t)kn * G.tiles_per_frame;
        if (gy > 65535) throw Error{"too many column tiles in one k-hat chunk"};
        dim3 grid((unsigned)((n_w + kWT - 1) / kWT), (unsigned)gy);
        k_gemm<Real, TN><<<grid, kThreads, smem, dev->stream>>>(A);
        CUDA_OK(cudaGetLastError());
        ++launches;
        record_event(dev, ev3[2]);
        launches += reduce_tiles(dev, job, A.partial, G.tiles_per_frame, 1, per, k0, kn, out, real_tiles);
        return launches;
    }
}

uint64_t launch_factored(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                         const double* tau, const double* cos_t, const double* sin2, const double* cos2,
                         const double* coeffs, const double* powers, const double* t_arr, const double* cutw,
                         const double* w, size_t k0, size_t kn, double2* out, const uint32_t* real_tiles,
                         cudaEvent_t* ev3) {
    if (job.kernel == BGWX_KERNEL_MIXED)
        return launch_typed<int8_t>(dev, job, bub_frames, sel, tau, cos_t, sin2, cos2, coeffs, powers, t_arr, cutw, w,
                                    k0, kn, out, real_tiles, ev3);
    if (job.kernel == BGWX_KERNEL_MIXED_SIMT)
        return launch_typed<float>(dev, job, bub_frames, sel, tau, cos_t, sin2, cos2, coeffs, powers, t_arr, cutw, w,
                                   k0, kn, out, real_tiles, ev3);
    return launch_typed<double>(dev, job, bub_frames, sel, tau, cos_t, sin2, cos2, coeffs, powers, t_arr, cutw, w, k0,
                                kn, out, real_tiles, ev3);
}

size_t factored_bubbles_per_tile(const SpectrumJob& job) {
    const size_t real = job.kernel == BGWX_KERNEL_MIXED        ? 1
                        : job.kernel == BGWX_KERNEL_MIXED_SIMT ? sizeof(float)
                                                               : sizeof(double);
    return (size_t)fact_geom(job, real).bpt;
}

int factored_auto_row_parts(const Device* dev, const SpectrumJob& job, size_t kn) {
    if (job.kernel != BGWX_KERNEL_MIXED) return 1;
    const FactGeom G = fact_geom(job, 1);
    return tc_row_parts((size_t)((job.n_w + 63) / 64) * kn * G.tiles_per_frame, (int)job.n_cos, dev->n_sm);
}

size_t factored_bytes_per_frame(const SpectrumJob& job) {
    const size_t real = job.kernel == BGWX_KERNEL_MIXED        ? 1
                        : job.kernel == BGWX_KERNEL_MIXED_SIMT ? sizeof(float)
                                                               : sizeof(double);
    const FactGeom G = fact_geom(job, real);
    // int8 tensor-core path: the digit block sets and one FP64 scale per (bubble, row)
    const size_t beta = job.kernel == BGWX_KERNEL_MIXED
                            ? (size_t)job.n_cos * G.tiles_per_frame * G.nblk * kI8BlockSet +
                                  (size_t)job.n_sel * job.n_cos * sizeof(double)
                            : (size_t)job.n_cos * G.cols_pad * G.t_pad * real;
    // partials: up to 16 row parts per column tile on the tensor-core path
    const size_t parts = job.kernel == BGWX_KERNEL_MIXED ? 16 : 1;
    return beta + (size_t)G.tiles_per_frame * parts * 2 * job.n_sets * job.n_w * sizeof(double2);
}

}  // namespace bgw
