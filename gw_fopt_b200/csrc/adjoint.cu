// Adjoint of the generalized bulk-flow spectrum (FP64).
//
// Forward (generalized_bulk_flow.rs:481-873, per k-hat frame on the rotated
// configuration, bubble a with t_a, z_a, row i with c_i, step k with t_k and
// dt_k = t_k - t_a > 0):
//   C_{g,s}(w) = sum_{a,i,k} e^{i phi} T_{g,s}(a,i,k),
//   phi        = w [(t_k - z_a) - dt_k c_i],
//   T_{g,s}    = pre_{i,k} dt_k^3 sum_j q_g(j) f_s(a,i,j,k),
//   pre_{i,k}  = 1/2 (1 - c_i^2) dphi dc v_i u_k cut_k dt / (6 pi),  q_g(j) = w_j {cos 2phi_j, sin 2phi_j},
//   f_s        = 1 before the collision, sum_m a_{sm} r^{p_{sm}} D after it (tau > 0 and dt_k >= tau),
//   r = tau/dt_k, D = exp(-(dt_k - tau)/width) (1 without damping),
//   tau        = Delta^2 / (2 Delta.x_hat), Delta = x_b - x_a for the first collider b (Minkowski products).
// Given the cotangent G_{g,s}(w) = dL/dRe C + i dL/dIm C (so dL = Re sum conj(G) dC):
//   P_{g,s}(a,i,k) = sum_w conj(G) e^{i phi},   Q_{g,s}(a,i,k) = sum_w w conj(G) e^{i phi},
//   dL/dT_{g,s}    = Re P,
//   dL/dt_a       += sum T (-c_i Im Q) - sum Re P dT/d(dt_k),
//   dL/dz_a       += sum T Im Q,
//   dL/da_{sm}     = sum Re P pre dt^3 q_g r^p D,   dL/dp_{sm} = sum Re P pre dt^3 q_g a r^p ln(r) D,
//   dL/dtau_{aij}  = sum_k Re P pre dt^3 q_g sum_m a r^p D (p/tau + 1/width),
// and tau's derivative with respect to Delta moves dL/dtau onto the radiating
// bubble (-) and its first collider (+).  Spatial gradients of a rotated frame
// are rotated back with R^T.  The collision status and the first-collider
// identity are piecewise constant in the inputs and carry no gradient.
//
// Kernels:
//   k_adj_mtab    the time-phase table M_i(w, k), once per call
//   k_adj_pq      per (frame, row): Re P and Im Q as two real products of depth W
//   k_adj_rows    one warp per (frame, bubble, row): the patch sums above in event form (suffix
//                 sums over the steps read at each patch's collision step), dL/dtau per patch
//   k_adj_bubble  per (frame, bubble): the row partials of t_a and z_a
//   k_adj_geom    per (frame, bubble, patch): dL/dtau -> both bubbles of the collision, and the
//                 bubble parts above, summed as fixed-point integers (deterministic; two passes:
//                 exponent bound, then sums) and added to the gradients by k_adj_fixout
//   k_adj_params  per parameter: fixed-order sum of the row partials

#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <type_traits>

#include "adjoint.cuh"
#include "bgw_internal.h"
#include "device_common.cuh"

namespace bgw {

constexpr int kAdjThreads = 256;

struct AdjArgs {
    const D4* bub;        // rotated bubbles of the chunk's frames, (kn, n_tot)
    size_t n_tot;
    int n_int;
    const uint32_t* sel;
    int n_sel, n_cos, n_phi, n_t, n_w, S, M;
    const double* tau;    // (kn, n_sel, nd)
    const int32_t* codes; // (kn, n_sel, nd)
    const D4* dirs;       // (nd) (1, nx, ny, nz)
    const double* cos_t;
    const double* sin2;
    const double* cos2;
    const double* coeffs; // (S*M)
    const double* powers; // (S*M)
    const double* t_arr;
    const double* cutw;
    const double* w;
    const double* rot;    // (kn, 9) rotations of the chunk's frames; nullptr = identity
    const double2* gbar;  // (kn, 2, S, W) cotangents of the chunk's frames
    int kn;               // frames in the chunk
    int f32pq;            // k_adj_pq: FP32 products folded into FP64 every kPqW frequencies (mixed kernels)
    int has_damp;
    double damp;
    double dphi, dcos, dt;
    AdjointScratch s;
    double* g_bub;        // (n_tot, 4)
    double* g_par;        // (2 S M)
};

// ---------------------------------------------------------------------------
// The phase factorises as e^{i phi} = M_i(w, k) E_{a,i}(w) with
// M_i = e^{i w t_k (1 - c_i)} (frame and bubble independent) and
// E_{a,i} = e^{i w (t_a c_i - z_a)}, so for each row i
//   P_{a,gs}(k) = sum_w H_{a,gs}(w) M_i(w, k),   H = conj(G_gs(w)) E_{a,i}(w),
//   Re P = sum_w (Hr Mr - Hi Mi),   Im Q = sum_w w (Hr Mi + Hi Mr):
// two real products of depth W per (frame, row), computed by k_adj_pq.
__global__ void k_adj_mtab(const double* __restrict__ cos_t, const double* __restrict__ t_arr,
                           const double* __restrict__ w, int n_cos, int n_w, int n_t, double2* __restrict__ mt) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)n_cos * n_w * n_t) return;
    const int k = (int)(q % n_t);
    const int wi = (int)((q / n_t) % n_w);
    const int i = (int)(q / ((size_t)n_t * n_w));
    double sn, cs;
    sincos(w[wi] * (t_arr[k] * (1.0 - cos_t[i])), &sn, &cs);
    mt[q] = make_double2(cs, sn);
}

constexpr int kPqRows = 64;   // (bubble, set, g) rows per tile
constexpr int kPqCols = 64;   // time steps per tile
constexpr int kPqW = 16;      // frequencies per shared-memory stage

// One CTA per (row tile x step tile, cos-theta row i, frame).  Thread
// (ty, tx) of 16 x 16 owns rows ty + 16 u and steps tx + 16 v (u, v < 4).
// F32: the products run in FP32 (H and M rounded to FP32, one FP32 sum per stage of kPqW
// frequencies), each stage's sums added to FP64 accumulators: about 16 x 2^-24 of the terms
// per stage instead of FP64 rounding, at twice the FMA rate.
template <int S, bool F32>
__global__ void __launch_bounds__(kAdjThreads) k_adj_pq(AdjArgs A, const double2* __restrict__ mt, int row_tiles) {
    constexpr int S2 = 2 * S;
    using V2 = typename std::conditional<F32, float2, double2>::type;
    using R = typename std::conditional<F32, float, double>::type;
    __shared__ V2 Hs[kPqW][kPqRows];
    __shared__ V2 Ms[kPqW][kPqCols];
    __shared__ R ws[kPqW];
    const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
    const int rt = blockIdx.x % row_tiles, kt = blockIdx.x / row_tiles;
    const int i = blockIdx.y, f = blockIdx.z;
    const int W = A.n_w;
    const int n_rows = A.n_sel * S2;
    const int r0 = rt * kPqRows, k0 = kt * kPqCols;
    // k_adj_rows reads P and Q only at steps after a row's bubble nucleated: a tile whose steps
    // all precede that for every bubble of its rows has nothing to compute
    __shared__ int s_kmin;
    if (tid == 0) s_kmin = A.n_t;
    __syncthreads();
    if (tid < kPqRows / S2) {
        const int slot = r0 / S2 + tid;
        if (slot < A.n_sel) {
            const double ta = A.bub[(size_t)f * A.n_tot + A.sel[slot]].t;
            int lo = 0, hi = A.n_t;  // first step with t_k - t_a > 0 (monotone in k)
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (A.t_arr[mid] - ta > 0.0) hi = mid;
                else lo = mid + 1;
            }
            atomicMin(&s_kmin, lo);
        }
    }
    __syncthreads();
    if (k0 + kPqCols <= s_kmin) return;
    const double ci = A.cos_t[i];
    double P[4][4], Q[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) P[u][v] = Q[u][v] = 0.0;
    for (int w0 = 0; w0 < W; w0 += kPqW) {
        R Ps[4][4], Qs[4][4];  // this stage's sums
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) Ps[u][v] = Qs[u][v] = R(0);
        __syncthreads();
        // H tile: row r = slot * S2 + gs
        for (int q = tid; q < kPqW * kPqRows; q += blockDim.x) {
            const int wl = q / kPqRows, rl = q % kPqRows;
            const int wi = w0 + wl, r = r0 + rl;
            double2 h = make_double2(0.0, 0.0);
            if (wi < W && r < n_rows) {
                const int slot = r / S2, gs = r % S2;
                const D4 xa = A.bub[(size_t)f * A.n_tot + A.sel[slot]];
                double sn, cs;
                sincos(A.w[wi] * (xa.t * ci - xa.z), &sn, &cs);
                const double2 g = A.gbar[((size_t)f * S2 + gs) * W + wi];
                // conj(g) * (cs + i sn)
                h = make_double2(g.x * cs + g.y * sn, g.x * sn - g.y * cs);
            }
            Hs[wl][rl] = V2{(R)h.x, (R)h.y};
        }
        for (int q = tid; q < kPqW * kPqCols; q += blockDim.x) {
            const int wl = q / kPqCols, kl = q % kPqCols;
            const int wi = w0 + wl, k = k0 + kl;
            const double2 m = (wi < W && k < A.n_t) ? mt[((size_t)i * W + wi) * A.n_t + k] : make_double2(0.0, 0.0);
            Ms[wl][kl] = V2{(R)m.x, (R)m.y};
        }
        if (tid < kPqW) ws[tid] = (R)(w0 + tid < W ? A.w[w0 + tid] : 0.0);
        __syncthreads();
#pragma unroll 4
        for (int wl = 0; wl < kPqW; ++wl) {
            V2 h[4], m[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) h[u] = Hs[wl][ty + 16 * u];
#pragma unroll
            for (int v = 0; v < 4; ++v) m[v] = Ms[wl][tx + 16 * v];
            const R om = ws[wl];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    Ps[u][v] = fma(h[u].x, m[v].x, fma(-h[u].y, m[v].y, Ps[u][v]));
                    Qs[u][v] = fma(om, fma(h[u].x, m[v].y, h[u].y * m[v].x), Qs[u][v]);
                }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                P[u][v] += (double)Ps[u][v];
                Q[u][v] += (double)Qs[u][v];
            }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int r = r0 + ty + 16 * u;
        if (r >= n_rows) continue;
        const int slot = r / S2, gs = r % S2;
        const size_t row = ((size_t)f * A.n_sel + slot) * A.n_cos + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int k = k0 + tx + 16 * v;
            if (k >= A.n_t) continue;
            const size_t o = (row * A.n_t + k) * S2 + gs;
            A.s.bbar[o] = P[u][v];
            A.s.imq[o] = Q[u][v];
        }
    }
}

// ---------------------------------------------------------------------------
// Per (bubble, step) factors of the collided scaling, frame independent:
// with r = tau/dt, a r^p D = a (tau^p e^{tau/w}) (dt^{-p} e^{-dt/w}), so the
// patch factor tau^p e^{tau/w} is formed once per patch and the step factor
// once per (bubble, step).  Row layout: dt^2, dt^3, ln dt, 1/dt, then
// dt^{-p_q} e^{-dt/w} for every (set, term) q; zeros where dt <= 0.
__global__ void k_adj_ttab(const D4* __restrict__ bub, const uint32_t* __restrict__ sel, int n_sel,
                           const double* __restrict__ t_arr, int n_t, const double* __restrict__ powers, int SM,
                           int has_damp, double damp, double* __restrict__ tt) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)n_sel * n_t) return;
    const int slot = (int)(q / n_t), k = (int)(q % n_t);
    const double dtk = t_arr[k] - bub[sel[slot]].t;
    double* row = tt + q * (4 + SM);
    const bool on = dtk > 0.0;
    row[0] = on ? dtk * dtk : 0.0;
    row[1] = on ? dtk * dtk * dtk : 0.0;
    row[2] = on ? log(dtk) : 0.0;
    row[3] = on ? 1.0 / dtk : 0.0;
    const double e = has_damp ? exp(-dtk / damp) : 1.0;
    for (int m = 0; m < SM; ++m) row[4 + m] = on ? exp(-powers[m] * log(dtk)) * e : 0.0;
}

// ---------------------------------------------------------------------------
// Row sums in event form.  The time grid is non-decreasing (t_begin <= t_end),
// so dt_k = t_k - t_a is too, and the collided steps of patch j are the
// suffix k >= kc_j: kc_j is the first step with dt_k >= tau_j (n_t when
// tau_j <= 0 or the wall is never reached).  Every double sum over (patch j,
// step k) of the direct form is then sum_j X_j . Y(kc_j), Y(k) = sum_{k'>=k}
// y_k' a suffix sum of per-step vectors.  Per step k (zero where dt_k <= 0),
// with g = 0, 1 the cos 2phi and sin 2phi weights, s_q the set of term q,
// be_q = dt^{-p_q} e^{-dt/w} and c1_q = -p_q/dt - 1/w:
//   T[g,q] = pre bb[g,s_q] be_q (3 d2 + d3 c1_q) + c_i Z[g,q]
//   Z[g,q] = pd3 iq[g,s_q] be_q,   B[g,q] = pd3 bb[g,s_q] be_q,   L[g,q] = B[g,q] ln dt
//   U[g]   = 3 pre d2 sum_s bb[g,s] + c_i V[g],   V[g] = pd3 sum_s iq[g,s]
// and with x_jg = q_g(j), y_jq = tau_j^{p_q} e^{tau_j/w} (a_q r^p D = a_q y_jq be_q):
//   acc_t  -= sum_j sum_g x_jg [sum_q a_q y_jq T(kc_j) + U(0) - U(kc_j)]
//   acc_z  += sum_j sum_g x_jg [sum_q a_q y_jq Z(kc_j) + V(0) - V(kc_j)]
//   tbar_j  = sum_g x_jg sum_q a_q y_jq (p_q/tau_j + 1/w) B(kc_j)
//   abar_q += sum_j sum_g x_jg y_jq B(kc_j)
//   pbar_q += a_q sum_j sum_g x_jg y_jq (ln tau_j B(kc_j) - L(kc_j))
// One warp per (frame, bubble, row) walks the steps in chunks of 32 from the
// last (lane = step): a warp suffix scan of each component plus the carry of
// the later chunks, the chunk's suffix sums to shared memory, and each patch
// whose kc_j falls in the chunk reads its entry once.  Work per row is
// O(n_t + n_phi) where the direct form is O(n_t n_phi).
constexpr int kRowWarps = 4;

template <int SMC>
__host__ __device__ constexpr int row_components() {
    return 8 * SMC + 4;
}

template <int S, int SMC, int JPL>
__global__ void __launch_bounds__(32 * kRowWarps) k_adj_rows(AdjArgs A, const double* __restrict__ tt) {
    constexpr int S2 = 2 * S;
    constexpr int M = SMC / S;
    constexpr int TW = 4 + SMC;
    constexpr int C = row_components<SMC>();
    constexpr int oT = 0, oZ = 2 * SMC, oB = 4 * SMC, oL = 6 * SMC, oU = 8 * SMC, oV = 8 * SMC + 2;
    extern __shared__ double rows_smem[];
    const unsigned full = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* sw = rows_smem + (size_t)warp * C * 32;  // [component][step in chunk]
    const long row = (long)blockIdx.x * kRowWarps + warp;
    const long R = (long)A.n_sel * A.n_cos;  // rows per frame
    const int f = (int)(row / R);
    if (f >= A.kn) return;
    const int slot = (int)((row % R) / A.n_cos);
    const int i = (int)(row % A.n_cos);
    const int n_t = A.n_t;
    const int nd = A.n_cos * A.n_phi;
    const double ta = A.bub[(size_t)f * A.n_tot + A.sel[slot]].t;
    const double ci = A.cos_t[i];
    const double vi = (i == 0 || i == A.n_cos - 1) ? 0.5 : 1.0;
    const double rowc = 0.5 * (1.0 - ci * ci) * A.dphi * A.dcos * vi * A.dt / (6.0 * M_PI);
    const double invw = A.has_damp ? 1.0 / A.damp : 0.0;
    const size_t pbase = ((size_t)f * A.n_sel + slot) * nd + (size_t)i * A.n_phi;

    double a_c[SMC], p_c[SMC];
#pragma unroll
    for (int q = 0; q < SMC; ++q) {
        a_c[q] = A.coeffs[q];
        p_c[q] = A.powers[q];
    }
    // collision step of this lane's patches j = lane + 32 jj (a monotone predicate: binary search)
    double tau_j[JPL], tbar[JPL];
    int kc[JPL];
    double xs0 = 0.0, xs1 = 0.0;  // sum over the lane's patches of the two weights
#pragma unroll
    for (int jj = 0; jj < JPL; ++jj) {
        const int j = lane + 32 * jj;
        const double tj = j < A.n_phi ? A.tau[pbase + j] : 0.0;
        tau_j[jj] = tj;
        tbar[jj] = 0.0;
        int lo = n_t;
        if (tj > 0.0) {
            lo = 0;
            int hi = n_t;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (A.t_arr[mid] - ta >= tj) hi = mid;
                else lo = mid + 1;
            }
        }
        kc[jj] = lo;
        if (j < A.n_phi) {
            const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
            xs0 += wj * A.cos2[j];
            xs1 += wj * A.sin2[j];
        }
    }
    // first step after the bubble's nucleation (dt_k > 0)
    int k0 = 0;
    {
        int hi = n_t;
        while (k0 < hi) {
            const int mid = (k0 + hi) >> 1;
            if (A.t_arr[mid] - ta > 0.0) hi = mid;
            else k0 = mid + 1;
        }
    }

    // sw[32 c] holds the suffix sum of component c from the start of the last chunk
    // done (the carry into the next one): zero before the first
#pragma unroll
    for (int c = 0; c < C; ++c) sw[c * 32 + lane] = 0.0;
    __syncwarp();
    double acc_t = 0.0, acc_z = 0.0, abar[SMC], pbar[SMC];
#pragma unroll
    for (int q = 0; q < SMC; ++q) abar[q] = pbar[q] = 0.0;

    const size_t base = ((size_t)f * A.n_sel + slot) * A.n_cos + i;
    const double* trow = tt + (size_t)slot * n_t * TW;
    for (int c0 = ((n_t - 1) >> 5) << 5; c0 >= (k0 & ~31); c0 -= 32) {
        const int k = c0 + lane;
        double y[C];
#pragma unroll
        for (int c = 0; c < C; ++c) y[c] = 0.0;
        if (k >= k0 && k < n_t) {
            const double* tk = trow + (size_t)k * TW;
            const double d2 = tk[0], d3 = tk[1], ld = tk[2], invd = tk[3];
            const double uk = (k == 0 || k == n_t - 1) ? 0.5 : 1.0;
            const double pre = rowc * uk * A.cutw[k];
            const double pd3 = pre * d3;
            const size_t o = (base * n_t + k) * S2;
            double bb[S2], iq[S2];
#pragma unroll
            for (int g = 0; g < S2; ++g) {
                bb[g] = A.s.bbar[o + g];
                iq[g] = A.s.imq[o + g];
            }
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                double sb = 0.0, si = 0.0;
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    sb += bb[g * S + s];
                    si += iq[g * S + s];
                }
                y[oV + g] = pd3 * si;
                y[oU + g] = 3.0 * pre * d2 * sb + ci * y[oV + g];
#pragma unroll
                for (int q = 0; q < SMC; ++q) {
                    const int s = q / M;
                    const double be = tk[4 + q];
                    const double c1 = -p_c[q] * invd - invw;
                    const double zq = pd3 * iq[g * S + s] * be;
                    const double bq = pd3 * bb[g * S + s] * be;
                    y[oZ + g * SMC + q] = zq;
                    y[oB + g * SMC + q] = bq;
                    y[oL + g * SMC + q] = bq * ld;
                    y[oT + g * SMC + q] = pre * bb[g * S + s] * be * (3.0 * d2 + d3 * c1) + ci * zq;
                }
            }
        }
        // inclusive suffix sums within the chunk, then the later chunks' total
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const double v = __shfl_down_sync(full, y[c], off);
                if (lane + off < 32) y[c] += v;
            }
        }
#pragma unroll
        for (int c = 0; c < C; ++c) y[c] += sw[c * 32];
        __syncwarp();
#pragma unroll
        for (int c = 0; c < C; ++c) sw[c * 32 + lane] = y[c];
        __syncwarp();
#pragma unroll
        for (int jj = 0; jj < JPL; ++jj) {
            const int kj = kc[jj];
            if (kj < c0 || kj >= c0 + 32 || kj >= n_t) continue;
            const double* e = sw + (kj - c0);  // component c at e[32 c]
            const int j = lane + 32 * jj;
            const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
            const double x0 = wj * A.cos2[j], x1 = wj * A.sin2[j];
            // the uncollided steps k < kc_j: the totals U(0) and V(0) are added after the loop
            acc_t += x0 * e[32 * oU] + x1 * e[32 * (oU + 1)];
            acc_z -= x0 * e[32 * oV] + x1 * e[32 * (oV + 1)];
            const double tj = tau_j[jj];
            const double lt = log(tj);
            const double et = A.has_damp ? exp(tj * invw) : 1.0;
            double tb = 0.0;
#pragma unroll
            for (int q = 0; q < SMC; ++q) {
                const double yq = exp(p_c[q] * lt) * et;
                const double c2 = p_c[q] / tj + invw;
                const double Tx = x0 * e[32 * (oT + q)] + x1 * e[32 * (oT + SMC + q)];
                const double Zx = x0 * e[32 * (oZ + q)] + x1 * e[32 * (oZ + SMC + q)];
                const double Bx = x0 * e[32 * (oB + q)] + x1 * e[32 * (oB + SMC + q)];
                const double Lx = x0 * e[32 * (oL + q)] + x1 * e[32 * (oL + SMC + q)];
                const double ay = a_c[q] * yq;
                acc_t -= ay * Tx;
                acc_z += ay * Zx;
                tb += ay * c2 * Bx;
                abar[q] += yq * Bx;
                pbar[q] += a_c[q] * yq * (lt * Bx - Lx);
            }
            tbar[jj] = tb;
        }
        __syncwarp();
    }
    // every patch's uncollided part starts from the totals U(0), V(0)
    acc_t -= xs0 * sw[32 * oU] + xs1 * sw[32 * (oU + 1)];
    acc_z += xs0 * sw[32 * oV] + xs1 * sw[32 * (oV + 1)];
#pragma unroll
    for (int jj = 0; jj < JPL; ++jj) {
        const int j = lane + 32 * jj;
        if (j < A.n_phi) A.s.taubar[pbase + j] = tbar[jj];
    }
    // fixed-order warp reduction of the row partials
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc_t += __shfl_down_sync(full, acc_t, off);
        acc_z += __shfl_down_sync(full, acc_z, off);
#pragma unroll
        for (int q = 0; q < SMC; ++q) {
            abar[q] += __shfl_down_sync(full, abar[q], off);
            pbar[q] += __shfl_down_sync(full, pbar[q], off);
        }
    }
    if (lane == 0) {
        double* rp = A.s.rowpart + base * (2 + 2 * SMC);
        rp[0] = acc_t;
        rp[1] = acc_z;
#pragma unroll
        for (int q = 0; q < SMC; ++q) {
            rp[2 + q] = abar[q];
            rp[2 + SMC + q] = pbar[q];
        }
    }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ void rotate_back(const double* R, double& gx, double& gy, double& gz) {
    // X' = R X  =>  dL/dX = R^T dL/dX'
    if (!R) return;
    const double ux = R[0] * gx + R[3] * gy + R[6] * gz;
    const double uy = R[1] * gx + R[4] * gy + R[7] * gz;
    const double uz = R[2] * gx + R[5] * gy + R[8] * gz;
    gx = ux;
    gy = uy;
    gz = uz;
}

// Bubble gradients are summed deterministically (the same bits on every run,
// whatever the order in which blocks run): every contribution v becomes the
// integer X = rint(v 2^(61 - E)), E the chunk's exponent bound (|v| < 2^E),
// split as X = H 2^31 + L with 0 <= L < 2^31, and H and L are added with
// 64-bit integer atomics, which are exact and so order-independent.  X keeps
// v to double precision relative to the chunk's largest contribution; the
// sums cannot overflow while a chunk has fewer than 2^31 contributions.

// Contribution of item q of frame f: q < n_sel*nd is a patch whose dL/dtau
// moves onto its first collider (kb, +g) and its radiating bubble (ka, -g);
// q = n_sel*nd + slot is the radiating bubble's own (t, x, y, z) part.
__device__ __forceinline__ void geom_item(const AdjArgs& A, int f, size_t q, long& ka, long& kb, double (&g)[4]) {
    const size_t nd = (size_t)A.n_cos * A.n_phi;
    ka = kb = -1;
    g[0] = g[1] = g[2] = g[3] = 0.0;
    if (q < (size_t)A.n_sel * nd) {
        const int slot = (int)(q / nd), d = (int)(q % nd);
        const size_t o = ((size_t)f * A.n_sel + slot) * nd + d;
        const double tb = A.s.taubar[o];
        const int32_t code = A.codes[o];
        const double tau = A.tau[o];
        if (tb != 0.0 && code != -1 && tau > 0.0) {
            const size_t b = code >= 0 ? (size_t)code : (size_t)A.n_int + (size_t)(-(code + 2));
            const uint32_t a = A.sel[slot];
            const D4 xa = A.bub[(size_t)f * A.n_tot + a];
            const D4 xb = A.bub[(size_t)f * A.n_tot + b];
            const D4 n = A.dirs[d];
            const double Dt = xb.t - xa.t, Dx = xb.x - xa.x, Dy = xb.y - xa.y, Dz = xb.z - xa.z;
            const double dot = -Dt + Dx * n.x + Dy * n.y + Dz * n.z;
            if (fabs(dot) >= 1e-10) {
                const double D2 = -Dt * Dt + Dx * Dx + Dy * Dy + Dz * Dz;
                const double inv = 1.0 / dot;
                const double h = 0.5 * D2 * inv * inv;
                g[0] = tb * (-Dt * inv + h);
                g[1] = tb * (Dx * inv - h * n.x);
                g[2] = tb * (Dy * inv - h * n.y);
                g[3] = tb * (Dz * inv - h * n.z);
                rotate_back(A.rot ? A.rot + 9 * f : nullptr, g[1], g[2], g[3]);
                ka = (long)a;
                kb = (long)b;
            }
        }
    } else if (q < (size_t)A.n_sel * nd + A.n_sel) {
        const int slot = (int)(q - (size_t)A.n_sel * nd);
        const double* bp = A.s.bubpart + ((size_t)f * A.n_sel + slot) * 4;
        g[0] = bp[0];
        g[1] = bp[1];
        g[2] = bp[2];
        g[3] = bp[3];
        ka = (long)A.sel[slot];
    }
}

// Adds each lane's fixed-point 4-vector (high and low parts) to gfix[key]
// (key < 0: nothing) with one atomic per run of equal keys in consecutive
// lanes: neighbouring patches mostly share their radiating bubble and their
// first collider.  Integer sums: exact in any order.  Call with the full warp.
__device__ __forceinline__ void warp_runs_add(long long* gfix, long key, const long long (&h_in)[4],
                                              const long long (&l_in)[4]) {
    const int lane = threadIdx.x & 31;
    long long h[4], l[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        h[c] = h_in[c];
        l[c] = l_in[c];
    }
    const long prev = __shfl_up_sync(0xffffffffu, key, 1);
    const bool head = lane == 0 || prev != key;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const int run = __popc(heads & (0xffffffffu >> (31 - lane)));  // runs started at or before this lane
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int r_up = __shfl_up_sync(0xffffffffu, run, off);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const long long uh = __shfl_up_sync(0xffffffffu, h[c], off);
            const long long ul = __shfl_up_sync(0xffffffffu, l[c], off);
            if (lane >= off && r_up == run) {
                h[c] += uh;
                l[c] += ul;
            }
        }
    }
    const int r_dn = __shfl_down_sync(0xffffffffu, run, 1);
    const bool tail = lane == 31 || r_dn != run;
    if (tail && key >= 0) {
        unsigned long long* g = reinterpret_cast<unsigned long long*>(gfix + 8 * key);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            atomicAdd(g + 2 * c, (unsigned long long)h[c]);
            atomicAdd(g + 2 * c + 1, (unsigned long long)l[c]);
        }
    }
}

__global__ void k_adj_gexp_init(int* gexp) { *gexp = -2000; }

// PASS 0: the exponent bound of the chunk's contributions; PASS 1: their fixed-point sums.
template <int PASS>
__global__ void k_adj_geom(AdjArgs A) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    long ka, kb;
    double g[4];
    geom_item(A, f, q, ka, kb, g);
    if constexpr (PASS == 0) {
        int e = -2000;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            int ex;
            if (g[c] != 0.0 && isfinite(g[c])) {
                frexp(g[c], &ex);  // |g| < 2^ex
                e = max(e, ex);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
        if ((threadIdx.x & 31) == 0 && e > -2000) atomicMax(A.s.gexp, e);
    } else {
        const int sh = 61 - *A.s.gexp;
        long long h[4], l[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            long long X = 0;
            if (isfinite(g[c])) {
                X = __double2ll_rn(ldexp(g[c], sh));
            } else if (kb >= 0 || ka >= 0) {
                // a non-finite gradient is passed on as it is
                if (kb >= 0) atomicAdd(A.g_bub + 4 * kb + c, g[c]);
                if (ka >= 0 && kb >= 0) atomicAdd(A.g_bub + 4 * ka + c, -g[c]);
                else if (ka >= 0) atomicAdd(A.g_bub + 4 * ka + c, g[c]);
            }
            h[c] = X >> 31;
            l[c] = X & 0x7fffffffLL;
        }
        // a patch adds +g to its collider and -g to its radiating bubble; a bubble part adds +g
        const bool patch = kb >= 0;
        warp_runs_add(A.s.gfix, kb, h, l);
        if (patch) {
            // -X = (-H - 1) 2^31 + (2^31 - L) for L > 0, and -H 2^31 for L = 0
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const long long X = h[c] * (1LL << 31) + l[c];
                h[c] = (-X) >> 31;
                l[c] = (-X) & 0x7fffffffLL;
            }
        }
        warp_runs_add(A.s.gfix, ka, h, l);
    }
}

// g_bub += the chunk's fixed-point sums; the accumulators are cleared for the next chunk.
__global__ void k_adj_fixout(AdjArgs A) {
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= 4 * A.n_tot) return;
    const int sh = 61 - *A.s.gexp;
    long long* p = A.s.gfix + 2 * c;
    const long long H = p[0], L = p[1];
    if (H != 0 || L != 0) A.g_bub[c] += ldexp((double)H, 31 - sh) + ldexp((double)L, -sh);
    p[0] = 0;
    p[1] = 0;
}

template <int SMC>
__global__ void k_adj_bubble(AdjArgs A) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (slot >= A.n_sel) return;
    double st = 0.0, sz = 0.0;
    for (int i = 0; i < A.n_cos; ++i) {
        const double* rp = A.s.rowpart + (((size_t)f * A.n_sel + slot) * A.n_cos + i) * (2 + 2 * SMC);
        st += rp[0];
        sz += rp[1];
    }
    // z' = R[2,:] . x  =>  dL/dx += dL/dz' R[2,:]
    double gx = 0.0, gy = 0.0, gz = sz;
    rotate_back(A.rot ? A.rot + 9 * f : nullptr, gx, gy, gz);
    double* bp = A.s.bubpart + ((size_t)f * A.n_sel + slot) * 4;
    bp[0] = st;
    bp[1] = gx;
    bp[2] = gy;
    bp[3] = gz;
}

template <int SMC>
__global__ void k_adj_params(AdjArgs A, long n_rows) {
    __shared__ double red[kAdjThreads];
    const int q = blockIdx.x;  // 0 .. 2*SMC-1
    double s = 0.0;
    for (long r = threadIdx.x; r < n_rows; r += blockDim.x) s += A.s.rowpart[r * (2 + 2 * SMC) + 2 + q];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) A.g_par[q] += red[0];
}

// ---------------------------------------------------------------------------
template <int S, int SMC, int JPL>
static void launch_rows(const AdjArgs& A, long rows, cudaStream_t st, const double* tt) {
    const size_t smem = (size_t)kRowWarps * row_components<SMC>() * 32 * sizeof(double);
    static_assert(kRowWarps * row_components<4>() * 32 * sizeof(double) <= 48 * 1024, "row kernel shared memory");
    k_adj_rows<S, SMC, JPL><<<(unsigned)((rows + kRowWarps - 1) / kRowWarps), 32 * kRowWarps, smem, st>>>(A, tt);
}

template <int S, int SMC>
static uint64_t launch_typed(const AdjArgs& A, size_t kn, cudaStream_t st, const double2* mt, const double* tt) {
    uint64_t launches = 0;
    {
        const int row_tiles = (A.n_sel * 2 * S + kPqRows - 1) / kPqRows;
        const int col_tiles = (A.n_t + kPqCols - 1) / kPqCols;
        if ((long)row_tiles * col_tiles > 0x7fffffffL) throw Error{"adjoint grid too large"};
        dim3 g((unsigned)(row_tiles * col_tiles), (unsigned)A.n_cos, (unsigned)kn);
        if (A.f32pq)
            k_adj_pq<S, true><<<g, kAdjThreads, 0, st>>>(A, mt, row_tiles);
        else
            k_adj_pq<S, false><<<g, kAdjThreads, 0, st>>>(A, mt, row_tiles);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    {
        const long rows = (long)kn * A.n_sel * A.n_cos;
        if (A.n_phi <= 32) launch_rows<S, SMC, 1>(A, rows, st, tt);
        else if (A.n_phi <= 64) launch_rows<S, SMC, 2>(A, rows, st, tt);
        else if (A.n_phi <= 128) launch_rows<S, SMC, 4>(A, rows, st, tt);
        else launch_rows<S, SMC, 8>(A, rows, st, tt);
        CUDA_OK(cudaGetLastError());
        ++launches;
        dim3 gb((unsigned)((A.n_sel + 127) / 128), (unsigned)kn);
        k_adj_bubble<SMC><<<gb, 128, 0, st>>>(A);
        CUDA_OK(cudaGetLastError());
        // every bubble gradient of the chunk: fixed-point sums (deterministic)
        const size_t per = (size_t)A.n_sel * A.n_cos * A.n_phi + A.n_sel;
        dim3 gg((unsigned)((per + 255) / 256), (unsigned)kn);
        k_adj_gexp_init<<<1, 1, 0, st>>>(A.s.gexp);
        k_adj_geom<0><<<gg, 256, 0, st>>>(A);
        k_adj_geom<1><<<gg, 256, 0, st>>>(A);
        k_adj_fixout<<<(unsigned)((4 * A.n_tot + 255) / 256), 256, 0, st>>>(A);
        CUDA_OK(cudaGetLastError());
        launches += 5;
        k_adj_params<SMC><<<2 * SMC, kAdjThreads, 0, st>>>(A, rows);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    return launches;
}

template <int S, int M>
static uint64_t dispatch_m(const AdjArgs& A, size_t kn, cudaStream_t st, const double2* mt, const double* tt) {
    return launch_typed<S, S * M>(A, kn, st, mt, tt);
}

uint64_t launch_adjoint_tables(Device* dev, const SpectrumJob& job, const D4* bub, const uint32_t* sel,
                               const double* cos_t, const double* t_arr, const double* w, const double* powers,
                               double2* mt, double* tt) {
    if (job.has_damping) {
        const double span = job.t_arr[job.n_t - 1] - job.t_arr[0] + 4.0;
        if (!(std::fabs(span / job.damping) < 600.0))
            throw Error{"damping width too small for the adjoint (exp overflow)"};
    }
    const size_t n = job.n_cos * job.n_w * job.n_t;
    k_adj_mtab<<<(unsigned)((n + 255) / 256), 256, 0, dev->stream>>>(cos_t, t_arr, w, (int)job.n_cos,
                                                                       (int)job.n_w, (int)job.n_t, mt);
    CUDA_OK(cudaGetLastError());
    const size_t nt = job.n_sel * job.n_t;
    k_adj_ttab<<<(unsigned)((nt + 255) / 256), 256, 0, dev->stream>>>(
        bub, sel, (int)job.n_sel, t_arr, (int)job.n_t, powers, (int)(job.n_sets * job.n_terms),
        job.has_damping ? 1 : 0, job.damping, tt);
    CUDA_OK(cudaGetLastError());
    return 2;
}

uint64_t launch_adjoint_chunk(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                              const double* tau, const int32_t* codes, const D4* dirs, const double* cos_t,
                              const double* sin2, const double* cos2, const double* coeffs, const double* powers,
                              const double* t_arr, const double* cutw, const double* w, const double* rot,
                              const double2* gbar, size_t kn, const AdjointScratch& s, const double2* mt,
                              const double* tt, double* g_bub, double* g_par) {
    AdjArgs A;
    A.bub = bub_frames;
    A.n_tot = job.n_tot;
    A.n_int = (int)job.n_int;
    A.sel = sel;
    A.n_sel = (int)job.n_sel;
    A.n_cos = (int)job.n_cos;
    A.n_phi = (int)job.n_phi;
    A.n_t = (int)job.n_t;
    A.n_w = (int)job.n_w;
    A.S = (int)job.n_sets;
    A.M = (int)job.n_terms;
    A.tau = tau;
    A.codes = codes;
    A.dirs = dirs;
    A.cos_t = cos_t;
    A.sin2 = sin2;
    A.cos2 = cos2;
    A.coeffs = coeffs;
    A.powers = powers;
    A.t_arr = t_arr;
    A.cutw = cutw;
    A.w = w;
    A.rot = rot;
    A.gbar = gbar;
    A.kn = (int)kn;
    // the backward's precision follows the forward's kernel: FP32 products of depth kPqW for the
    // mixed kernels, FP64 otherwise
    A.f32pq = (job.kernel == BGWX_KERNEL_MIXED || job.kernel == BGWX_KERNEL_MIXED_SIMT) ? 1 : 0;
    A.has_damp = job.has_damping ? 1 : 0;
    A.damp = job.damping;
    A.dphi = 2.0 * M_PI / (double)job.n_phi;
    A.dcos = 2.0 / (double)(job.n_cos - 1);
    A.dt = job.dt;
    A.s = s;
    A.g_bub = g_bub;
    A.g_par = g_par;
    if (job.n_phi > 256) throw Error{"the adjoint supports n_phi <= 256"};
    if (kn > 65535 || job.n_sel > 65535 || job.n_cos > 65535) throw Error{"adjoint grid too large"};
    const cudaStream_t st = dev->stream;
    const int S = A.S, M = A.M;
    // (S, M) pairs with S*M <= 8
    switch (S) {
        case 1:
            switch (M) {
                case 1: return dispatch_m<1, 1>(A, kn, st, mt, tt);
                case 2: return dispatch_m<1, 2>(A, kn, st, mt, tt);
                case 3: return dispatch_m<1, 3>(A, kn, st, mt, tt);
                case 4: return dispatch_m<1, 4>(A, kn, st, mt, tt);
                default: break;
            }
            break;
        case 2:
            switch (M) {
                case 1: return dispatch_m<2, 1>(A, kn, st, mt, tt);
                case 2: return dispatch_m<2, 2>(A, kn, st, mt, tt);
                default: break;
            }
            break;
        case 3:
            if (M == 1) return dispatch_m<3, 1>(A, kn, st, mt, tt);
            break;
        case 4:
            if (M == 1) return dispatch_m<4, 1>(A, kn, st, mt, tt);
            break;
        default: break;
    }
    throw Error{"the adjoint supports (n_sets, n_terms) with n_sets*n_terms <= 4"};
}

size_t adjoint_bytes_per_frame(const SpectrumJob& job) {
    const size_t S2 = 2 * job.n_sets, SM = job.n_sets * job.n_terms;
    const size_t rows = job.n_sel * job.n_cos;
    const size_t nd = job.n_cos * job.n_phi;
    return rows * job.n_t * S2 * 2 * sizeof(double) + job.n_sel * nd * (2 * sizeof(double) + sizeof(int32_t)) +
           rows * (2 + 2 * SM) * sizeof(double) + job.n_tot * sizeof(D4);
}

}  // namespace bgw
