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
#include <vector>

#include "bgw_internal.h"
#include "device_common.cuh"
#include "spectrum_factored.cuh"

namespace bgw {

constexpr int kKC = 16;          // time steps per chunk (GEMM k-tile, event bucket)
constexpr int kWT = 64;          // frequencies per CTA
constexpr int kRows = 2 * kWT;   // GEMM rows: (Re, Im) of each frequency
constexpr int kCols = 64;        // GEMM columns per CTA
constexpr int kThreads = 256;
constexpr int kTM = 8, kTN = 4;  // register tile per thread
constexpr int kMaxQ = 2 + 2 * 8; // q values per event: (P0 cos, P0 sin) + 2 per (set, term), <= 8 terms

// ---------------------------------------------------------------------------
__global__ void k_time_tables(const D4* __restrict__ bub, const uint32_t* __restrict__ sel, int n_sel,
                              const double* __restrict__ t_arr, int n_t, const double* __restrict__ powers, int SM,
                              int has_damp, double damp, double* __restrict__ D, int* __restrict__ kfirst) {
    const int slot = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= n_sel || k >= n_t) return;
    const double ta = bub[sel[slot]].t;
    const double dt = t_arr[k] - ta;
    double* row = D + ((size_t)slot * n_t + k) * (1 + SM);
    const bool on = dt > 0.0;
    row[0] = on ? dt * (dt * dt) : 0.0;
    const double e = has_damp ? exp(-dt / damp) : 1.0;
    for (int q = 0; q < SM; ++q) row[1 + q] = on ? pow(dt, 3.0 - powers[q]) * e : 0.0;
    // first active step (t_a <= t_k and dt > 0): monotone in k
    if (on && (k == 0 || !(t_arr[k - 1] - ta > 0.0))) kfirst[slot] = k;
    if (k == n_t - 1 && !on) kfirst[slot] = n_t;
}

// ---------------------------------------------------------------------------
// One warp per row (frame, slot, i): events sorted by bucket, stable in j.
template <class Real>
__global__ void __launch_bounds__(256)
    k_events(const double* __restrict__ tau, const D4* __restrict__ bub, const uint32_t* __restrict__ sel,
             int n_sel, int n_cos, int n_phi, const double* __restrict__ t_arr, int n_t,
             const double* __restrict__ cos2, const double* __restrict__ sin2, const double* __restrict__ powers,
             int SM, int has_damp, double damp, long n_rows, int NB, int* __restrict__ ev_off,
             int* __restrict__ ev_k, Real* __restrict__ ev_q, double2* __restrict__ ev_unc) {
    extern __shared__ int sm_ev[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long row = (long)blockIdx.x * (blockDim.x >> 5) + warp;
    const int per_warp = 2 * (NB + 1) + 4 * NB + 2;  // ints: hist, run, then 2*NB doubles (8-byte aligned)
    int* hist = sm_ev + warp * per_warp;
    int* run = hist + (NB + 1);
    if (row >= n_rows) return;
    const int slot = (int)((row / n_cos) % n_sel);
    const double ta = bub[sel[slot]].t;
    const double* trow = tau + (size_t)row * n_phi;
    const int NQ = 2 + 2 * SM;
    for (int b = lane; b <= NB; b += 32) hist[b] = 0;
    __syncwarp();
    auto bucket_of = [&](int j, int& kj) -> int {
        kj = n_t;
        if (j >= n_phi) return -1;
        const double tj = trow[j];
        if (!(tj > 0.0)) return -1;
        int lo = 0, hi = n_t;  // first k with (t_k - t_a) >= tau_j (GBF:405)
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (t_arr[mid] - ta >= tj) hi = mid;
            else lo = mid + 1;
        }
        kj = lo;
        return lo < n_t ? lo / kKC : -1;
    };
    const unsigned full = 0xffffffffu;
    for (int j0 = 0; j0 < n_phi; j0 += 32) {
        int kj;
        const int b = bucket_of(j0 + lane, kj);
        const unsigned m = __match_any_sync(full, b);
        if (b >= 0 && lane == __ffs(m) - 1) hist[b] += __popc(m);
        __syncwarp();
    }
    if (lane == 0) {
        int acc = 0;
        for (int b = 0; b < NB; ++b) {
            int c = hist[b];
            hist[b] = acc;
            run[b] = acc;
            acc += c;
        }
        hist[NB] = acc;
    }
    __syncwarp();
    int* off = ev_off + (size_t)row * (NB + 1);
    for (int b = lane; b <= NB; b += 32) off[b] = hist[b];
    const unsigned lt = (1u << lane) - 1u;
    for (int j0 = 0; j0 < n_phi; j0 += 32) {
        const int j = j0 + lane;
        int kj;
        const int b = bucket_of(j, kj);
        const unsigned m = __match_any_sync(full, b);
        int pos = 0;
        if (b >= 0) pos = run[b] + __popc(m & lt);
        __syncwarp();
        if (b >= 0 && lane == __ffs(m) - 1) run[b] += __popc(m);
        __syncwarp();
        if (b >= 0) {
            const size_t e = (size_t)row * n_phi + pos;
            ev_k[e] = kj;
            const double tj = trow[j];
            const double wj = (j == 0 || j == n_phi - 1) ? 0.5 : 1.0;
            const double qc = wj * cos2[j], qs = wj * sin2[j];
            Real* q = ev_q + e * NQ;
            q[0] = (Real)qc;
            q[1] = (Real)qs;
            const double ed = has_damp ? exp(tj / damp) : 1.0;
            for (int t = 0; t < SM; ++t) {
                const double f = pow(tj, powers[t]) * ed;
                q[2 + 2 * t] = (Real)(qc * f);
                q[3 + 2 * t] = (Real)(qs * f);
            }
        }
    }
    __syncwarp();
    // Uncollided sums U[c] = sum of q over the patches not collided before
    // bucket c: the never-colliding patches plus the events of buckets >= c,
    // accumulated backwards (a sum of the remaining terms, never a difference
    // of two large sums).  Per-bucket sums are formed in lane order.
    double* bsum = reinterpret_cast<double*>(run + (NB + 1));  // [NB][2] after hist/run
    for (int b = lane; b < NB; b += 32) {
        bsum[2 * b] = 0.0;
        bsum[2 * b + 1] = 0.0;
    }
    __syncwarp();
    double nc = 0.0, ns = 0.0;  // never collided within the grid (lane 0 accumulates)
    for (int j0 = 0; j0 < n_phi; j0 += 32) {
        const int j = j0 + lane;
        int kj;
        const int b = bucket_of(j, kj);
        double qc = 0.0, qs = 0.0;
        if (j < n_phi) {
            const double wj = (j == 0 || j == n_phi - 1) ? 0.5 : 1.0;
            qc = wj * cos2[j];
            qs = wj * sin2[j];
        }
        const unsigned m = __match_any_sync(full, b);
        const bool leader = lane == __ffs(m) - 1;
        double gc = 0.0, gs = 0.0;
        for (int l = 0; l < 32; ++l) {
            const double vc = __shfl_sync(full, qc, l), vs = __shfl_sync(full, qs, l);
            const int bl = __shfl_sync(full, b, l);
            const bool valid_l = j0 + l < n_phi;
            if (leader && valid_l && bl == b) {
                gc += vc;
                gs += vs;
            }
            if (lane == 0 && valid_l && bl < 0) {
                nc += vc;
                ns += vs;
            }
        }
        if (leader && b >= 0) {
            bsum[2 * b] += gc;
            bsum[2 * b + 1] += gs;
        }
        __syncwarp();
    }
    if (lane == 0) {
        double2* U = ev_unc + (size_t)row * (NB + 1);
        double uc = nc, us = ns;
        U[NB] = make_double2(uc, us);
        for (int c = NB - 1; c >= 0; --c) {
            uc += bsum[2 * c];
            us += bsum[2 * c + 1];
            U[c] = make_double2(uc, us);
        }
    }
}

// ---------------------------------------------------------------------------
struct FactArgs {
    const D4* bub;  // rotated frames (kn, n_tot)
    size_t n_tot;
    const uint32_t* sel;
    int n_sel;
    int n_cos, n_phi, n_t, n_w;
    int S, M;
    const double* cos_t;
    const double* t_arr;
    const double* cutw;
    const double* w;
    const double* coeffs;  // (S, M)
    const double* D;       // (n_sel, n_t, 1+S*M)
    const int* kfirst;     // (n_sel)
    const int* ev_off;     // (rows, NB+1)
    const int* ev_k;       // (rows, n_phi)
    const void* ev_q;      // (rows, n_phi, NQ) Real
    const double2* ev_unc; // (rows, NB+1): uncollided sums of q before bucket c
    int NB;
    double dt, dphi, dcos;
    int bpt;               // bubbles per column tile
    int tiles_per_frame;
    double2* partial;      // (kn, tiles_per_frame, 2, S, W)
};

struct SmemF {
    double anchor_re[kWT], anchor_im[kWT];
};

// sin/cos of an FP64 argument: FP64 kernel uses sincos; the mixed kernel
// reduces the argument modulo 2 pi in FP64 (Cody-Waite, two constants) and
// evaluates sincosf on the reduced FP32 argument.
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

template <class Real>
__global__ void __launch_bounds__(kThreads, 1) k_spec_factored(FactArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    // shared-memory layout
    Real* Msm = reinterpret_cast<Real*>(smem);                       // [kKC][kRows]
    Real* Bsm = Msm + kKC * kRows;                                   // [kKC][kCols]
    double* Pn_re = reinterpret_cast<double*>(Bsm + kKC * kCols);     // [kKC][kWT]
    double* Pn_im = Pn_re + kKC * kWT;
    double* E_re = Pn_im + kKC * kWT;                                // [kWT][bpt]
    double* E_im = E_re + kWT * 32;
    double2* Yt = reinterpret_cast<double2*>(E_im + kWT * 32);        // [kCols][kWT]
    double2* Cacc = Yt + kCols * kWT;                                // [kWT][S][2]
    double* Pst = reinterpret_cast<double*>(Cacc + kWT * A.S * 2);    // [bpt][NQ]
    double* anc = Pst + 32 * kMaxQ;                                  // [2][kWT]
    int* binfo = reinterpret_cast<int*>(anc + 2 * kWT);               // [bpt]: slot or -1

    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;
    const int w0 = blockIdx.x * kWT;
    const int frame = blockIdx.y / A.tiles_per_frame;
    const int tile = blockIdx.y % A.tiles_per_frame;
    const int NQ = 2 + 2 * A.S * A.M;
    const int SM = A.S * A.M;
    const int cols_per_b = 2 * A.S;
    const D4* B = A.bub + (size_t)frame * A.n_tot;
    const Real* evq = static_cast<const Real*>(A.ev_q);

    if (tid < A.bpt) {
        const int slot = tile * A.bpt + tid;
        binfo[tid] = slot < A.n_sel ? slot : -1;
    }
    for (int q = tid; q < kWT * A.S * 2; q += kThreads) Cacc[q] = make_double2(0.0, 0.0);
    __syncthreads();
    int kstart = A.n_t;
    for (int b = 0; b < A.bpt; ++b)
        if (binfo[b] >= 0) kstart = min(kstart, A.kfirst[binfo[b]]);
    const int c_start = kstart / kKC;
    const int n_chunks = (A.n_t + kKC - 1) / kKC;
    const double inv6pi = 1.0 / (6.0 * CUDART_PI);

    for (int i = 0; i < A.n_cos; ++i) {
        const double ci = A.cos_t[i];
        const double one_m_c = 1.0 - ci;
        const double vi = (i == 0 || i == A.n_cos - 1) ? 0.5 : 1.0;
        const double row_factor = (0.5 * (1.0 - ci * ci) * A.dphi) * (A.dcos * vi) * A.dt * inv6pi;
        // within-chunk phase steps P_n(w) = e^{i w (1-c_i) n dt}, and epilogue phases
        for (int q = tid; q < kKC * kWT; q += kThreads) {
            const int n = q / kWT, wl = q % kWT;
            const int wi = w0 + wl;
            double s = 0.0, c = 1.0;
            if (wi < A.n_w) phase<Real>(A.w[wi] * one_m_c * (n * A.dt), s, c);
            Pn_re[q] = c;
            Pn_im[q] = s;
        }
        for (int q = tid; q < kWT * A.bpt; q += kThreads) {
            const int wl = q / A.bpt, b = q % A.bpt;
            const int wi = w0 + wl;
            double s = 0.0, c = 0.0;
            if (wi < A.n_w && binfo[b] >= 0) {
                const D4 xa = B[A.sel[binfo[b]]];
                phase<Real>(A.w[wi] * (xa.t * ci - xa.z), s, c);
            }
            E_re[wl * 32 + b] = c;
            E_im[wl * 32 + b] = s;
        }
        for (int q = tid; q < 32 * kMaxQ; q += kThreads) Pst[q] = 0.0;  // layout [bubble][kMaxQ]
        double acc[kTM][kTN];
        Real cacc[kTM][kTN];
#pragma unroll
        for (int r = 0; r < kTM; ++r)
#pragma unroll
            for (int u = 0; u < kTN; ++u) acc[r][u] = 0.0;
        __syncthreads();

        for (int ch = c_start; ch < n_chunks; ++ch) {
            const int k0 = ch * kKC;
            // (1) anchors e^{i w (1-c_i) t_k0} and the M tile
            if (tid < kWT) {
                const int wi = w0 + tid;
                double s = 0.0, c = 0.0;
                if (wi < A.n_w) phase<Real>(A.w[wi] * one_m_c * A.t_arr[k0], s, c);
                anc[tid] = c;
                anc[kWT + tid] = s;
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
            // (2) the beta tile from running prefix sums and this bucket's events
            for (int q = tid; q < kKC * kCols; q += kThreads) {
                const int n = q / kCols, col = q % kCols;
                const int k = k0 + n;
                const int b = col / cols_per_b, sg = col % cols_per_b;
                const int s = sg >> 1, g = sg & 1;
                double beta = 0.0;
                if (b < A.bpt && binfo[b] >= 0 && k < A.n_t) {
                    const int slot = binfo[b];
                    const double* Drow = A.D + ((size_t)slot * A.n_t + k) * (1 + SM);
                    const double d3 = Drow[0];
                    if (d3 != 0.0) {
                        const long row = ((long)frame * A.n_sel + slot) * A.n_cos + i;
                        const int* off = A.ev_off + (size_t)row * (A.NB + 1);
                        const int e0 = off[ch], e1 = off[ch + 1];
                        const int* ek = A.ev_k + (size_t)row * A.n_phi;
                        const Real* eq = evq + (size_t)row * A.n_phi * NQ;
                        // uncollided patches: those of later buckets plus this bucket's with k_e > k
                        double unc = g ? A.ev_unc[(size_t)row * (A.NB + 1) + ch + 1].y
                                       : A.ev_unc[(size_t)row * (A.NB + 1) + ch + 1].x;
                        double pm[8];
                        for (int m = 0; m < A.M; ++m) pm[m] = Pst[b * kMaxQ + 2 + 2 * (s * A.M + m) + g];
                        for (int e = e0; e < e1; ++e) {
                            if (ek[e] > k) {
                                unc += (double)eq[(size_t)e * NQ + g];
                            } else {
                                for (int m = 0; m < A.M; ++m)
                                    pm[m] += (double)eq[(size_t)e * NQ + 2 + 2 * (s * A.M + m) + g];
                            }
                        }
                        double v = d3 * unc;
                        for (int m = 0; m < A.M; ++m) v += A.coeffs[s * A.M + m] * Drow[1 + s * A.M + m] * pm[m];
                        beta = row_factor * A.cutw[k] * ((k == 0 || k == A.n_t - 1) ? 0.5 : 1.0) * v;
                    }
                }
                Bsm[n * kCols + col] = (Real)beta;
            }
            __syncthreads();
            // (3) fold this bucket into the running prefix sums
            for (int q = tid; q < A.bpt * NQ; q += kThreads) {
                const int b = q / NQ, qi = q % NQ;
                if (binfo[b] < 0) continue;
                const long row = ((long)frame * A.n_sel + binfo[b]) * A.n_cos + i;
                const int* off = A.ev_off + (size_t)row * (A.NB + 1);
                const Real* eq = evq + (size_t)row * A.n_phi * NQ;
                double p = Pst[b * kMaxQ + qi];
                for (int e = off[ch]; e < off[ch + 1]; ++e) p += (double)eq[(size_t)e * NQ + qi];
                Pst[b * kMaxQ + qi] = p;
            }
            // (4) register-tiled GEMM over the chunk
#pragma unroll
            for (int r = 0; r < kTM; ++r)
#pragma unroll
                for (int u = 0; u < kTN; ++u) cacc[r][u] = (Real)0;
#pragma unroll 4
            for (int n = 0; n < kKC; ++n) {
                Real a[kTM], bb[kTN];
#pragma unroll
                for (int r = 0; r < kTM; ++r) a[r] = Msm[n * kRows + ty * kTM + r];
#pragma unroll
                for (int u = 0; u < kTN; ++u) bb[u] = Bsm[n * kCols + tx * kTN + u];
#pragma unroll
                for (int r = 0; r < kTM; ++r)
#pragma unroll
                    for (int u = 0; u < kTN; ++u) cacc[r][u] = fma(a[r], bb[u], cacc[r][u]);
            }
#pragma unroll
            for (int r = 0; r < kTM; ++r)
#pragma unroll
                for (int u = 0; u < kTN; ++u) acc[r][u] += (double)cacc[r][u];
            __syncthreads();
        }
        // epilogue: C_{s,g}(w) += sum_b E(w, b) Y(w, (b, s, g))
#pragma unroll
        for (int q = 0; q < kTM / 2; ++q) {
            const int wl = (ty * kTM) / 2 + q;
#pragma unroll
            for (int u = 0; u < kTN; ++u) {
                const int col = tx * kTN + u;
                const int b = col / cols_per_b;
                double2 v = make_double2(0.0, 0.0);
                if (b < A.bpt) {
                    const double er = E_re[wl * 32 + b], ei = E_im[wl * 32 + b];
                    const double yr = acc[2 * q][u], yi = acc[2 * q + 1][u];
                    v = make_double2(er * yr - ei * yi, er * yi + ei * yr);
                }
                Yt[col * kWT + wl] = v;
            }
        }
        __syncthreads();
        for (int q = tid; q < kWT * A.S * 2; q += kThreads) {
            const int wl = q / (A.S * 2), sg = q % (A.S * 2);
            double2 sum = Cacc[q];
            for (int b = 0; b < A.bpt; ++b) {
                const double2 v = Yt[(b * cols_per_b + sg) * kWT + wl];
                sum.x += v.x;
                sum.y += v.y;
            }
            Cacc[q] = sum;
        }
        __syncthreads();
    }
    // partial (frame, tile, g, s, w)
    for (int q = tid; q < kWT * A.S * 2; q += kThreads) {
        const int wl = q / (A.S * 2), sg = q % (A.S * 2);
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

// ---------------------------------------------------------------------------
static size_t fact_smem_bytes(int real_size, int S) {
    size_t b = (size_t)kKC * kRows * real_size + (size_t)kKC * kCols * real_size;
    b = (b + 15) & ~(size_t)15;
    b += 2 * (size_t)kKC * kWT * sizeof(double);
    b += 2 * (size_t)kWT * 32 * sizeof(double);
    b += (size_t)kCols * kWT * sizeof(double2);
    b += (size_t)kWT * S * 2 * sizeof(double2);
    b += 32 * kMaxQ * sizeof(double);
    b += 2 * kWT * sizeof(double);
    b += 32 * sizeof(int);
    return b;
}

template <class Real>
static uint64_t launch_typed(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                             const double* tau, const double* cos_t, const double* sin2, const double* cos2,
                             const double* coeffs, const double* powers, const double* t_arr, const double* cutw,
                             const double* w, size_t kn, double2* out) {
    const int S = (int)job.n_sets, M = (int)job.n_terms, SM = S * M;
    const int n_t = (int)job.n_t, n_cos = (int)job.n_cos, n_phi = (int)job.n_phi, n_w = (int)job.n_w;
    const int n_sel = (int)job.n_sel;
    if (M > 8 || 2 + 2 * SM > kMaxQ || 2 * S > kCols)
        throw Error{"the factored kernels support at most 8 (set, term) pairs; use the fp64_direct kernel"};
    if (job.has_damping) {
        double max_tau_over = job.t_arr[job.n_t - 1] / job.damping;
        if (!(std::fabs(max_tau_over) < 600.0))
            throw Error{"damping width too small for the factored kernels (exp overflow); use fp64_direct"};
    }
    const int NB = (n_t + kKC - 1) / kKC;
    const int NQ = 2 + 2 * SM;
    const long rows = (long)kn * n_sel * n_cos;
    uint64_t launches = 0;
    // per-bubble time tables (frame independent)
    dev->fact_D.ensure((size_t)n_sel * n_t * (1 + SM) * sizeof(double));
    dev->fact_kfirst.ensure((size_t)n_sel * sizeof(int));
    // bubble times are frame independent: frame 0 of bub_frames serves
    {
        dim3 g((unsigned)((n_t + 127) / 128), (unsigned)n_sel);
        k_time_tables<<<g, 128, 0, dev->stream>>>(bub_frames, sel, n_sel, t_arr, n_t, powers, SM,
                                                  job.has_damping ? 1 : 0, job.damping, (double*)dev->fact_D.p,
                                                  (int*)dev->fact_kfirst.p);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    // events
    dev->ev_off.ensure((size_t)rows * (NB + 1) * sizeof(int));
    dev->ev_k.ensure((size_t)rows * n_phi * sizeof(int));
    dev->ev_q.ensure((size_t)rows * n_phi * NQ * sizeof(Real));
    dev->ev_unc.ensure((size_t)rows * (NB + 1) * sizeof(double2));
    {
        const int warps = 8;
        size_t smem = (size_t)warps * (2 * (NB + 1) + 4 * NB + 2) * sizeof(int);
        if (smem > 200 * 1024) throw Error{"n_t too large for the event kernel"};
        CUDA_OK(cudaFuncSetAttribute(k_events<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        unsigned blocks = (unsigned)((rows + warps - 1) / warps);
        k_events<Real><<<blocks, warps * 32, smem, dev->stream>>>(
            tau, bub_frames, sel, n_sel, n_cos, n_phi, t_arr, n_t, cos2, sin2, powers, SM, job.has_damping ? 1 : 0,
            job.damping, rows, NB, (int*)dev->ev_off.p, (int*)dev->ev_k.p, (Real*)dev->ev_q.p,
            (double2*)dev->ev_unc.p);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    // GEMM + epilogue
    FactArgs A;
    A.bub = bub_frames;
    A.n_tot = job.n_tot;
    A.sel = sel;
    A.n_sel = n_sel;
    A.n_cos = n_cos;
    A.n_phi = n_phi;
    A.n_t = n_t;
    A.n_w = n_w;
    A.S = S;
    A.M = M;
    A.cos_t = cos_t;
    A.t_arr = t_arr;
    A.cutw = cutw;
    A.w = w;
    A.coeffs = coeffs;
    A.D = (const double*)dev->fact_D.p;
    A.kfirst = (const int*)dev->fact_kfirst.p;
    A.ev_off = (const int*)dev->ev_off.p;
    A.ev_k = (const int*)dev->ev_k.p;
    A.ev_q = dev->ev_q.p;
    A.ev_unc = (const double2*)dev->ev_unc.p;
    A.NB = NB;
    A.dt = job.dt;
    A.dphi = 2.0 * M_PI / (double)n_phi;
    A.dcos = 2.0 / (double)(n_cos - 1);
    A.bpt = std::min(32, kCols / (2 * S));
    A.tiles_per_frame = (n_sel + A.bpt - 1) / A.bpt;
    const size_t per = (size_t)2 * S * n_w;
    dev->fact_partial.ensure((size_t)kn * A.tiles_per_frame * per * sizeof(double2));
    A.partial = (double2*)dev->fact_partial.p;
    const size_t smem = fact_smem_bytes((int)sizeof(Real), S);
    CUDA_OK(cudaFuncSetAttribute(k_spec_factored<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const size_t gy = (size_t)kn * A.tiles_per_frame;
    if (gy > 65535) throw Error{"too many column tiles in one k-hat chunk"};
    dim3 grid((unsigned)((n_w + kWT - 1) / kWT), (unsigned)gy);
    k_spec_factored<Real><<<grid, kThreads, smem, dev->stream>>>(A);
    CUDA_OK(cudaGetLastError());
    ++launches;
    dim3 gr((unsigned)((per + 255) / 256), (unsigned)kn);
    k_reduce_tiles<<<gr, 256, 0, dev->stream>>>(A.partial, A.tiles_per_frame, per, (int)kn, out);
    CUDA_OK(cudaGetLastError());
    ++launches;
    return launches;
}

uint64_t launch_factored(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                         const double* tau, const double* cos_t, const double* sin2, const double* cos2,
                         const double* coeffs, const double* powers, const double* t_arr, const double* cutw,
                         const double* w, size_t kn, double2* out) {
    if (job.kernel == BGWX_KERNEL_MIXED)
        return launch_typed<float>(dev, job, bub_frames, sel, tau, cos_t, sin2, cos2, coeffs, powers, t_arr, cutw, w,
                                   kn, out);
    return launch_typed<double>(dev, job, bub_frames, sel, tau, cos_t, sin2, cos2, coeffs, powers, t_arr, cutw, w, kn,
                                out);
}

size_t factored_bytes_per_frame(const SpectrumJob& job) {
    const size_t NB = (job.n_t + kKC - 1) / kKC;
    const size_t NQ = 2 + 2 * job.n_sets * job.n_terms;
    const size_t real = job.kernel == BGWX_KERNEL_MIXED ? sizeof(float) : sizeof(double);
    const size_t rows = job.n_sel * job.n_cos;
    const size_t bpt = std::min<size_t>(32, kCols / (2 * job.n_sets));
    const size_t tiles = (job.n_sel + bpt - 1) / bpt;
    return rows * ((NB + 1) * (sizeof(int) + sizeof(double2)) + job.n_phi * (sizeof(int) + NQ * real)) +
           tiles * 2 * job.n_sets * job.n_w * sizeof(double2);
}

}  // namespace bgw
