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
//   k_adj_phase   per (frame, bubble, row, step): Re P and Im Q (one FP64 sincos per w)
//   k_adj_rows    one warp per (frame, bubble, row): the patch sums above, dL/dtau per patch
//   k_adj_geom    per (frame, bubble, patch): dL/dtau -> both bubbles of the collision (atomics)
//   k_adj_bubble  per (frame, bubble): the row partials of t_a and z_a (atomics)
//   k_adj_params  per parameter: fixed-order sum of the row partials

#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "adjoint.cuh"
#include "bgw_internal.h"
#include "device_common.cuh"

namespace bgw {

constexpr int kAdjThreads = 256;
constexpr int kMaxJPerLane = 8;  // n_phi <= 256

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
    int has_damp;
    double damp;
    double dphi, dcos, dt;
    AdjointScratch s;
    double* g_bub;        // (n_tot, 4)
    double* g_par;        // (2 S M)
};

// ---------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(kAdjThreads) k_adj_phase(AdjArgs A) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    constexpr int S2 = 2 * S;
    const int W = A.n_w;
    double2* G = reinterpret_cast<double2*>(sm_raw);  // [S2][W]
    double* ws = reinterpret_cast<double*>(G + S2 * W);
    const int i = blockIdx.x, slot = blockIdx.y, f = blockIdx.z;
    for (int q = threadIdx.x; q < S2 * W; q += blockDim.x) G[q] = A.gbar[(size_t)f * S2 * W + q];
    for (int q = threadIdx.x; q < W; q += blockDim.x) ws[q] = A.w[q];
    __syncthreads();
    const D4 xa = A.bub[(size_t)f * A.n_tot + A.sel[slot]];
    const double ci = A.cos_t[i];
    const size_t row = ((size_t)f * A.n_sel + slot) * A.n_cos + i;
    for (int k = threadIdx.x; k < A.n_t; k += blockDim.x) {
        const double tk = A.t_arr[k];
        const double dtk = tk - xa.t;
        const size_t o = (row * A.n_t + k) * S2;
        double P[S2], Q[S2];
#pragma unroll
        for (int g = 0; g < S2; ++g) P[g] = Q[g] = 0.0;
        if (dtk > 0.0) {
            const double theta = (tk - xa.z) - dtk * ci;
            for (int q = 0; q < W; ++q) {
                double sn, cs;
                sincos(ws[q] * theta, &sn, &cs);
#pragma unroll
                for (int g = 0; g < S2; ++g) {
                    const double2 gv = G[g * W + q];
                    P[g] += gv.x * cs + gv.y * sn;
                    Q[g] += ws[q] * (gv.x * sn - gv.y * cs);
                }
            }
        }
#pragma unroll
        for (int g = 0; g < S2; ++g) {
            A.s.bbar[o + g] = P[g];
            A.s.imq[o + g] = Q[g];
        }
    }
}

// ---------------------------------------------------------------------------
template <int S, int SMC>
__global__ void __launch_bounds__(kAdjThreads) k_adj_rows(AdjArgs A) {
    constexpr int S2 = 2 * S;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long row = (long)blockIdx.x * (blockDim.x >> 5) + warp;
    const long R = (long)A.n_sel * A.n_cos;  // rows per frame
    const int f = (int)(row / R);
    if (f >= A.kn) return;
    const int slot = (int)((row % R) / A.n_cos);
    const int i = (int)(row % A.n_cos);
    const int M = A.M;
    const int nd = A.n_cos * A.n_phi;
    const D4 xa = A.bub[(size_t)f * A.n_tot + A.sel[slot]];
    const double ci = A.cos_t[i];
    const double vi = (i == 0 || i == A.n_cos - 1) ? 0.5 : 1.0;
    const double rowc = 0.5 * (1.0 - ci * ci) * A.dphi * A.dcos * vi * A.dt / (6.0 * M_PI);
    const double invw = A.has_damp ? 1.0 / A.damp : 0.0;

    double tau_j[kMaxJPerLane], q0[kMaxJPerLane], q1[kMaxJPerLane], tbar[kMaxJPerLane];
#pragma unroll
    for (int jj = 0; jj < kMaxJPerLane; ++jj) {
        const int j = lane + 32 * jj;
        const bool ok = j < A.n_phi;
        const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
        tau_j[jj] = ok ? A.tau[((size_t)f * A.n_sel + slot) * nd + (size_t)i * A.n_phi + j] : 0.0;
        q0[jj] = ok ? wj * A.cos2[j] : 0.0;
        q1[jj] = ok ? wj * A.sin2[j] : 0.0;
        tbar[jj] = 0.0;
    }
    double a_c[SMC], p_c[SMC];
#pragma unroll
    for (int q = 0; q < SMC; ++q) {
        a_c[q] = A.coeffs[q];
        p_c[q] = A.powers[q];
    }
    double acc_t = 0.0, acc_z = 0.0, abar[SMC], pbar[SMC];
#pragma unroll
    for (int q = 0; q < SMC; ++q) abar[q] = pbar[q] = 0.0;

    const size_t base = ((size_t)f * A.n_sel + slot) * A.n_cos + i;
    for (int k = 0; k < A.n_t; ++k) {
        const double dtk = A.t_arr[k] - xa.t;
        if (!(dtk > 0.0)) continue;
        const double uk = (k == 0 || k == A.n_t - 1) ? 0.5 : 1.0;
        const double pre = rowc * uk * A.cutw[k];
        const double d2 = dtk * dtk, d3 = d2 * dtk;
        const size_t o = (base * A.n_t + k) * S2;
        double bb[S2], iq[S2];
#pragma unroll
        for (int g = 0; g < S2; ++g) {
            bb[g] = A.s.bbar[o + g];
            iq[g] = A.s.imq[o + g];
        }
#pragma unroll
        for (int jj = 0; jj < kMaxJPerLane; ++jj) {
            if (lane + 32 * jj >= A.n_phi) break;
            double Bs[S], Is[S];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                Bs[s] = bb[s] * q0[jj] + bb[S + s] * q1[jj];
                Is[s] = iq[s] * q0[jj] + iq[S + s] * q1[jj];
            }
            const double tj = tau_j[jj];
            if (tj > 0.0 && dtk >= tj) {
                const double r = tj / dtk;
                const double lr = log(r);
                const double D = A.has_damp ? exp(-(dtk - tj) * invw) : 1.0;
                double fs[S], dfdt[S], dfdtau[S];
#pragma unroll
                for (int s = 0; s < S; ++s) fs[s] = dfdt[s] = dfdtau[s] = 0.0;
#pragma unroll
                for (int q = 0; q < SMC; ++q) {
                    const int s = q / M;
                    const double rpD = exp(p_c[q] * lr) * D;
                    const double e = a_c[q] * rpD;
                    fs[s] += e;
                    dfdt[s] += e * (-p_c[q] / dtk - invw);
                    dfdtau[s] += e * (p_c[q] / tj + invw);
                    const double wgt = pre * d3 * Bs[s] * rpD;
                    abar[q] += wgt;
                    pbar[q] += wgt * a_c[q] * lr;
                }
                double st = 0.0, sz = 0.0, sx = 0.0;
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    st += Bs[s] * (3.0 * d2 * fs[s] + d3 * dfdt[s]);
                    sz += Is[s] * fs[s];
                    sx += Bs[s] * dfdtau[s];
                }
                acc_t += pre * (-st - ci * d3 * sz);
                acc_z += pre * d3 * sz;
                tbar[jj] += pre * d3 * sx;
            } else {
                double sb = 0.0, sz = 0.0;
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    sb += Bs[s];
                    sz += Is[s];
                }
                acc_t += pre * (-3.0 * d2 * sb - ci * d3 * sz);
                acc_z += pre * d3 * sz;
            }
        }
    }
#pragma unroll
    for (int jj = 0; jj < kMaxJPerLane; ++jj) {
        const int j = lane + 32 * jj;
        if (j < A.n_phi) A.s.taubar[((size_t)f * A.n_sel + slot) * nd + (size_t)i * A.n_phi + j] = tbar[jj];
    }
    // fixed-order warp reduction of the row partials
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc_t += __shfl_down_sync(0xffffffffu, acc_t, off);
        acc_z += __shfl_down_sync(0xffffffffu, acc_z, off);
#pragma unroll
        for (int q = 0; q < SMC; ++q) {
            abar[q] += __shfl_down_sync(0xffffffffu, abar[q], off);
            pbar[q] += __shfl_down_sync(0xffffffffu, pbar[q], off);
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
__device__ __forceinline__ void add_rotated_back(double* g, const double* R, double gt, double gx, double gy,
                                                 double gz, double sign) {
    // X' = R X  =>  dL/dX = R^T dL/dX'
    double ux = gx, uy = gy, uz = gz;
    if (R) {
        ux = R[0] * gx + R[3] * gy + R[6] * gz;
        uy = R[1] * gx + R[4] * gy + R[7] * gz;
        uz = R[2] * gx + R[5] * gy + R[8] * gz;
    }
    atomicAdd(g + 0, sign * gt);
    atomicAdd(g + 1, sign * ux);
    atomicAdd(g + 2, sign * uy);
    atomicAdd(g + 3, sign * uz);
}

__global__ void k_adj_geom(AdjArgs A) {
    const int nd = A.n_cos * A.n_phi;
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (q >= (size_t)A.n_sel * nd) return;
    const int slot = (int)(q / nd), d = (int)(q % nd);
    const size_t o = ((size_t)f * A.n_sel + slot) * nd + d;
    const double tb = A.s.taubar[o];
    if (tb == 0.0) return;
    const int32_t code = A.codes[o];
    const double tau = A.tau[o];
    if (code == -1 || !(tau > 0.0)) return;
    const size_t b = code >= 0 ? (size_t)code : (size_t)A.n_int + (size_t)(-(code + 2));
    const uint32_t a = A.sel[slot];
    const D4 xa = A.bub[(size_t)f * A.n_tot + a];
    const D4 xb = A.bub[(size_t)f * A.n_tot + b];
    const D4 n = A.dirs[d];
    const double Dt = xb.t - xa.t, Dx = xb.x - xa.x, Dy = xb.y - xa.y, Dz = xb.z - xa.z;
    const double dot = -Dt + Dx * n.x + Dy * n.y + Dz * n.z;
    if (fabs(dot) < 1e-10) return;
    const double D2 = -Dt * Dt + Dx * Dx + Dy * Dy + Dz * Dz;
    const double inv = 1.0 / dot;
    const double h = 0.5 * D2 * inv * inv;
    const double gt = tb * (-Dt * inv + h);
    const double gx = tb * (Dx * inv - h * n.x);
    const double gy = tb * (Dy * inv - h * n.y);
    const double gz = tb * (Dz * inv - h * n.z);
    const double* R = A.rot ? A.rot + 9 * f : nullptr;
    add_rotated_back(A.g_bub + 4 * b, R, gt, gx, gy, gz, 1.0);
    add_rotated_back(A.g_bub + 4 * (size_t)a, R, gt, gx, gy, gz, -1.0);
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
    const double* R = A.rot ? A.rot + 9 * f : nullptr;
    // z' = R[2,:] . x  =>  dL/dx += dL/dz' R[2,:]
    add_rotated_back(A.g_bub + 4 * (size_t)A.sel[slot], R, st, 0.0, 0.0, sz, 1.0);
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
template <int S, int SMC>
static uint64_t launch_typed(const AdjArgs& A, size_t kn, cudaStream_t st) {
    uint64_t launches = 0;
    {
        const size_t smem = (size_t)2 * S * A.n_w * sizeof(double2) + (size_t)A.n_w * sizeof(double);
        if (smem > 200 * 1024) throw Error{"too many frequencies for the adjoint's shared memory"};
        CUDA_OK(cudaFuncSetAttribute(k_adj_phase<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        dim3 g((unsigned)A.n_cos, (unsigned)A.n_sel, (unsigned)kn);
        k_adj_phase<S><<<g, kAdjThreads, smem, st>>>(A);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    {
        const long rows = (long)kn * A.n_sel * A.n_cos;
        const int warps = kAdjThreads / 32;
        k_adj_rows<S, SMC><<<(unsigned)((rows + warps - 1) / warps), kAdjThreads, 0, st>>>(A);
        CUDA_OK(cudaGetLastError());
        ++launches;
        const size_t per = (size_t)A.n_sel * A.n_cos * A.n_phi;
        dim3 gg((unsigned)((per + 255) / 256), (unsigned)kn);
        k_adj_geom<<<gg, 256, 0, st>>>(A);
        CUDA_OK(cudaGetLastError());
        ++launches;
        dim3 gb((unsigned)((A.n_sel + 127) / 128), (unsigned)kn);
        k_adj_bubble<SMC><<<gb, 128, 0, st>>>(A);
        CUDA_OK(cudaGetLastError());
        ++launches;
        k_adj_params<SMC><<<2 * SMC, kAdjThreads, 0, st>>>(A, rows);
        CUDA_OK(cudaGetLastError());
        ++launches;
    }
    return launches;
}

template <int S, int M>
static uint64_t dispatch_m(const AdjArgs& A, size_t kn, cudaStream_t st) {
    return launch_typed<S, S * M>(A, kn, st);
}

uint64_t launch_adjoint_chunk(Device* dev, const SpectrumJob& job, const D4* bub_frames, const uint32_t* sel,
                              const double* tau, const int32_t* codes, const D4* dirs, const double* cos_t,
                              const double* sin2, const double* cos2, const double* coeffs, const double* powers,
                              const double* t_arr, const double* cutw, const double* w, const double* rot,
                              const double2* gbar, size_t kn, const AdjointScratch& s, double* g_bub,
                              double* g_par) {
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
    A.has_damp = job.has_damping ? 1 : 0;
    A.damp = job.damping;
    A.dphi = 2.0 * M_PI / (double)job.n_phi;
    A.dcos = 2.0 / (double)(job.n_cos - 1);
    A.dt = job.dt;
    A.s = s;
    A.g_bub = g_bub;
    A.g_par = g_par;
    if (job.n_phi > 32 * kMaxJPerLane) throw Error{"the adjoint supports n_phi <= 256"};
    if (kn > 65535 || job.n_sel > 65535 || job.n_cos > 65535) throw Error{"adjoint grid too large"};
    const cudaStream_t st = dev->stream;
    const int S = A.S, M = A.M;
    // (S, M) pairs with S*M <= 8
    switch (S) {
        case 1:
            switch (M) {
                case 1: return dispatch_m<1, 1>(A, kn, st);
                case 2: return dispatch_m<1, 2>(A, kn, st);
                case 3: return dispatch_m<1, 3>(A, kn, st);
                case 4: return dispatch_m<1, 4>(A, kn, st);
                default: break;
            }
            break;
        case 2:
            switch (M) {
                case 1: return dispatch_m<2, 1>(A, kn, st);
                case 2: return dispatch_m<2, 2>(A, kn, st);
                default: break;
            }
            break;
        case 3:
            if (M == 1) return dispatch_m<3, 1>(A, kn, st);
            break;
        case 4:
            if (M == 1) return dispatch_m<4, 1>(A, kn, st);
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
