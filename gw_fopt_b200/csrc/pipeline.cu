// Device pipeline of the generalized bulk-flow spectrum (sm_100a).
//
// Stages, per chunk of k-hat frames:
//   k_rotate       bubbles (t, x, y, z) rotated by R(k)            [optional]
//   k_neighbors, k_masks_list (masks.cu)
//                  exact first-collider search per (k, bubble, patch)
//   k_spec_direct  plain FP64 spectrum: one complex phase per
//                  (bubble, cos-theta row, t, w), the reference's loop nest
//   k_reduce       deterministic sum of per-bubble partial spectra
//
// Reference: rust/bubble-gw/src/many_bubbles/generalized_bulk_flow.rs (GBF).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bgw_internal.h"
#include "device_common.cuh"
#include "masks.cuh"
#include "spectrum_factored.cuh"
#include "adjoint.cuh"

namespace bgw {

int device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

Device* device_create() {
    int n = device_count();
    if (n <= 0)
        throw Error{"no CUDA device is available: the bulk-flow spectrum runs only on the GPU (no CPU fallback)"};
    auto* d = new Device();
    try {
        CUDA_OK(cudaGetDevice(&d->id));
        CUDA_OK(cudaDeviceGetAttribute(&d->n_sm, cudaDevAttrMultiProcessorCount, d->id));
        CUDA_OK(cudaStreamCreateWithFlags(&d->own_stream, cudaStreamNonBlocking));
        d->stream = d->own_stream;
        for (auto& e : d->ev) CUDA_OK(cudaEventCreate(&e));
    } catch (...) {
        delete d;
        throw;
    }
    return d;
}

void device_destroy(Device* d) { delete d; }

void device_set_stream(Device* d, void* stream) {
    CUDA_OK(cudaStreamSynchronize(d->stream));
    d->stream = stream ? static_cast<cudaStream_t>(stream) : d->own_stream;
}

void device_drop_resident(Device* d) {
    for (DevBuf* b : {&d->bub, &d->dirs, &d->cos_t, &d->sin2, &d->cos2, &d->coeffs, &d->powers, &d->t_arr,
                      &d->cutw, &d->w, &d->sel, &d->rot, &d->cosphi, &d->sinphi})
        b->shadow_valid = false;
}

Device::~Device() {
    if (stream) cudaStreamSynchronize(stream);
    if (ens_graph) cudaGraphExecDestroy(ens_graph);
    if (own_stream) cudaStreamDestroy(own_stream);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : chunk_ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : fact_ev)
        if (e) cudaEventDestroy(e);
}

// ---------------------------------------------------------------------------
// k_rotate: x' = R x with x'_i = (R_i0 x + R_i1 y) + R_i2 z, unfused.
// ---------------------------------------------------------------------------
__global__ void k_rotate(const D4* __restrict__ bub, const double* __restrict__ rot, size_t n_tot,
                         D4* __restrict__ out) {
    size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    int k = blockIdx.y;
    if (b >= n_tot) return;
    const double* R = rot + 9 * k;
    D4 v = bub[b];
    D4 o;
    o.t = v.t;
    o.x = dadd(dadd(dmul(R[0], v.x), dmul(R[1], v.y)), dmul(R[2], v.z));
    o.y = dadd(dadd(dmul(R[3], v.x), dmul(R[4], v.y)), dmul(R[5], v.z));
    o.z = dadd(dadd(dmul(R[6], v.x), dmul(R[7], v.y)), dmul(R[8], v.z));
    out[(size_t)k * n_tot + b] = o;
}

// ---------------------------------------------------------------------------
// Plain FP64 spectrum (GBF:481-586, 588-664, 775-873), one block per
// (k-hat, radiating bubble).  Per t: the B stage evaluates every patch of
// every cos-theta row into shared memory; the A stage gives each thread one w
// and a stride of rows (rows split across thread groups when n_w < 256) and
// forms sum_i B_i e^{-i w dt c_i} dc v_i; the C stage multiplies by
// e^{i w (t - z_a)} u_t cut(t) dt.  The block writes its bubble's
// (2, S, W) contribution times 1/(6 pi).
// ---------------------------------------------------------------------------
constexpr int kSpecThreads = 256;
constexpr int kSetChunk = 4;

struct SpecArgs {
    const D4* bub;
    size_t n_tot;
    const uint32_t* sel;
    size_t n_sel;
    const double* tau;
    int n_cos, n_phi;
    const double* cos_thetax;
    const double* sin2phi;
    const double* cos2phi;
    const double* coeffs;
    const double* powers;
    int n_sets, n_terms;
    int has_damping;
    double damping;
    const double* t_arr;
    const double* cutw;
    int n_t;
    double dt;
    const double* w;
    int n_w;
    double2* partial;  // (K, n_sel, 2, S, W); with PER_T: (n_sel, 2, S, W, n_t); tensor: (K, n_sel, 6, S, W)
    int tau_in_smem;
    const double* cosphi;  // tensor form
    const double* sinphi;
};

// Combination step of ndarray's unrolled_fold:
// acc = (((0 + (p0+p4)) + (p1+p5)) + (p2+p6)) + (p3+p7), then + tail.
__device__ __forceinline__ double unrolled_sum8(const double* p8, double tail) {
    double acc = 0.0;
    acc = __dadd_rn(acc, __dadd_rn(p8[0], p8[4]));
    acc = __dadd_rn(acc, __dadd_rn(p8[1], p8[5]));
    acc = __dadd_rn(acc, __dadd_rn(p8[2], p8[6]));
    acc = __dadd_rn(acc, __dadd_rn(p8[3], p8[7]));
    return __dadd_rn(acc, tail);
}

// PER_T: the time-resolved integrand of compute_c_integrand_fixed_bubble
// (generalized_bulk_flow.rs:776-866): each step's A e^{i w (t - z_a)} times the
// trapezoid dt weight and 1/(6 pi), one output per step (no time cutoff),
// instead of the sum over steps.
template <bool PER_T>
__global__ void __launch_bounds__(kSpecThreads) k_spec_direct(SpecArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int k = blockIdx.y;
    const size_t slot = blockIdx.x;
    const int nd = A.n_cos * A.n_phi;
    const double* tau_g = A.tau + ((size_t)k * A.n_sel + slot) * nd;
    double* tau_s = reinterpret_cast<double*>(smem_raw);
    // even number of doubles before Bsm keeps the double2 array below 16-byte aligned
    double* Bsm = tau_s + (A.tau_in_smem ? ((nd + 1) & ~1) : 0);  // [n_cos][kSetChunk][2]
    double2* red = reinterpret_cast<double2*>(Bsm + (size_t)A.n_cos * kSetChunk * 2);  // [256][kSetChunk][2]
    const double* tau = A.tau_in_smem ? tau_s : tau_g;
    if (A.tau_in_smem)
        for (int q = threadIdx.x; q < nd; q += kSpecThreads) tau_s[q] = tau_g[q];
    __syncthreads();

    const uint32_t a = A.sel[slot];
    const D4 xa = A.bub[(size_t)k * A.n_tot + a];
    const double ta = xa.t, za = xa.z;
    const int W_eff = min(A.n_w, kSpecThreads);
    const int n_ig = kSpecThreads / W_eff;
    const int wl = threadIdx.x % W_eff;
    const int ig = threadIdx.x / W_eff;
    const bool wthread = ig < n_ig;
    const double dphi = 2.0 * CUDART_PI / (double)A.n_phi;
    const double dcos = 2.0 / (double)(A.n_cos - 1);
    const double inv6pi = 1.0 / (6.0 * CUDART_PI);

    for (int s0 = 0; s0 < A.n_sets; s0 += kSetChunk) {
        const int sc = min(kSetChunk, A.n_sets - s0);
        for (int wb = 0; wb < A.n_w; wb += W_eff) {
            const int wi = wb + wl;
            const bool wvalid = wthread && wi < A.n_w;
            const double wv = wvalid ? A.w[wi] : 0.0;
            double2 cacc[kSetChunk][2];
#pragma unroll
            for (int s = 0; s < kSetChunk; ++s) cacc[s][0] = cacc[s][1] = make_double2(0.0, 0.0);

            for (int kt = 0; kt < A.n_t; ++kt) {
                const double t = A.t_arr[kt];
                if (!(ta <= t)) continue;  // GBF:821
                const double dta = t - ta;
                // ---- B stage (GBF:481-586) ----
                for (int i = threadIdx.x; i < A.n_cos; i += kSpecThreads) {
                    const double c = A.cos_thetax[i];
                    const double sin_sq = 1.0 - c * c;
                    const double cubed = dta * (dta * dta);
                    for (int s = 0; s < sc; ++s) {
                        double bp = 0.0, bm = 0.0;
                        if (dta > 0.0) {
                            const double* trow = tau + (size_t)i * A.n_phi;
                            const int sidx = (s0 + s) * A.n_terms;
                            // f(t, t_n, t_nc) for patch j (GBF:549-567)
                            auto factor = [&](int j) {
                                const double tj = trow[j];
                                double f = 1.0;
                                if (tj > 0.0 && dta >= tj) {
                                    const double ratio = tj / dta;
                                    f = 0.0;
                                    for (int m = 0; m < A.n_terms; ++m)
                                        f += A.coeffs[sidx + m] * pow(ratio, A.powers[sidx + m]);
                                    if (A.has_damping) f *= exp(-dta * (1.0 - ratio) / A.damping);
                                }
                                return f;
                            };
                            // ndarray's eight-way unrolled sum over phi (GBF:578-579)
                            double pc[8], ps[8];
#pragma unroll
                            for (int u = 0; u < 8; ++u) pc[u] = ps[u] = 0.0;
                            const int nfull = A.n_phi & ~7;
                            for (int j0 = 0; j0 < nfull; j0 += 8) {
#pragma unroll
                                for (int u = 0; u < 8; ++u) {
                                    const int j = j0 + u;
                                    const double f = factor(j);
                                    const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
                                    pc[u] = __dadd_rn(pc[u], __dmul_rn(__dmul_rn(A.cos2phi[j], f), wj));
                                    ps[u] = __dadd_rn(ps[u], __dmul_rn(__dmul_rn(A.sin2phi[j], f), wj));
                                }
                            }
                            double sum_c = unrolled_sum8(pc, 0.0);
                            double sum_s = unrolled_sum8(ps, 0.0);
                            for (int j = nfull; j < A.n_phi; ++j) {
                                const double f = factor(j);
                                const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
                                sum_c = __dadd_rn(sum_c, __dmul_rn(__dmul_rn(A.cos2phi[j], f), wj));
                                sum_s = __dadd_rn(sum_s, __dmul_rn(__dmul_rn(A.sin2phi[j], f), wj));
                            }
                            bp = 0.5 * sin_sq * (sum_c * dphi * cubed);
                            bm = 0.5 * sin_sq * (sum_s * dphi * cubed);
                        }
                        Bsm[((size_t)i * kSetChunk + s) * 2 + 0] = bp;
                        Bsm[((size_t)i * kSetChunk + s) * 2 + 1] = bm;
                    }
                }
                __syncthreads();
                // ---- A stage (GBF:635-661) ----
                double2 aacc[kSetChunk][2];
#pragma unroll
                for (int s = 0; s < kSetChunk; ++s) aacc[s][0] = aacc[s][1] = make_double2(0.0, 0.0);
                if (wvalid) {
                    for (int i = ig; i < A.n_cos; i += n_ig) {
                        const double base_im = -dta * A.cos_thetax[i];
                        double sn, cs;
                        sincos(wv * base_im, &sn, &cs);
                        const double vi = (i == 0 || i == A.n_cos - 1) ? 0.5 : 1.0;
                        const double pr = (cs * dcos) * vi, pim = (sn * dcos) * vi;
#pragma unroll
                        for (int s = 0; s < kSetChunk; ++s) {
                            if (s < sc) {
                                const double bp = Bsm[((size_t)i * kSetChunk + s) * 2 + 0];
                                const double bm = Bsm[((size_t)i * kSetChunk + s) * 2 + 1];
                                aacc[s][0].x += bp * pr;
                                aacc[s][0].y += bp * pim;
                                aacc[s][1].x += bm * pr;
                                aacc[s][1].y += bm * pim;
                            }
                        }
                    }
                }
#pragma unroll
                for (int s = 0; s < kSetChunk; ++s) {
                    red[((size_t)threadIdx.x * kSetChunk + s) * 2 + 0] = aacc[s][0];
                    red[((size_t)threadIdx.x * kSetChunk + s) * 2 + 1] = aacc[s][1];
                }
                __syncthreads();
                // ---- C stage (GBF:832-851) ----
                if (PER_T && wvalid && ig == 0) {
                    double sn, cs;
                    sincos(wv * (t - za), &sn, &cs);
                    const double dtw = A.dt * ((kt == 0 || kt == A.n_t - 1) ? 0.5 : 1.0);
                    for (int s = 0; s < sc; ++s) {
                        for (int g = 0; g < 2; ++g) {
                            double2 at = make_double2(0.0, 0.0);
                            for (int q = 0; q < n_ig; ++q) {
                                const double2 v = red[((size_t)(q * W_eff + wl) * kSetChunk + s) * 2 + g];
                                at.x += v.x;
                                at.y += v.y;
                            }
                            // (A e^{i w (t - z_a)}) (dt w_t) / (6 pi), GBF:832-840 and 862-863
                            const double re = (at.x * cs - at.y * sn) * dtw * inv6pi;
                            const double im = (at.x * sn + at.y * cs) * dtw * inv6pi;
                            const size_t o = ((((size_t)slot * 2 + g) * A.n_sets + (s0 + s)) * A.n_w + wi) * A.n_t + kt;
                            A.partial[o] = make_double2(re, im);
                        }
                    }
                }
                if (!PER_T && wvalid && ig == 0) {
                    double sn, cs;
                    sincos(wv * (t - za), &sn, &cs);
                    const double uw = (kt == 0 || kt == A.n_t - 1) ? 0.5 : 1.0;
                    const double cw = A.cutw[kt];
                    for (int s = 0; s < sc; ++s) {
                        for (int g = 0; g < 2; ++g) {
                            double2 at = make_double2(0.0, 0.0);
                            for (int q = 0; q < n_ig; ++q) {
                                const double2 v = red[((size_t)(q * W_eff + wl) * kSetChunk + s) * 2 + g];
                                at.x += v.x;
                                at.y += v.y;
                            }
                            double re = (at.x * cs - at.y * sn) * uw * cw;
                            double im = (at.x * sn + at.y * cs) * uw * cw;
                            cacc[s][g].x += re * A.dt;
                            cacc[s][g].y += im * A.dt;
                        }
                    }
                }
                __syncthreads();
            }
            if (!PER_T && wvalid && ig == 0) {
                for (int s = 0; s < sc; ++s)
                    for (int g = 0; g < 2; ++g) {
                        size_t o = ((((size_t)k * A.n_sel + slot) * 2 + g) * A.n_sets + (s0 + s)) * A.n_w + wi;
                        A.partial[o] = make_double2(cacc[s][g].x * inv6pi, cacc[s][g].y * inv6pi);
                    }
            }
        }
    }
}

// The tensor form of new_generalized_bulk_flow.rs (NGBF:592-1203): the phi
// integral of x_i x_j (t - t_n)^3 f in six components (xx, xy, xz, yy, yz, zz,
// NGBF:634-727), the same A and C stages with NGBF's factor placement
// (NGBF:782-826, 1145-1168), no time cutoff; one coefficient set at a time.
// PER_T: the time-resolved integrand (NGBF:832-991), each step's
// A e^{i w (t - z_a)} (dt w_t) / (6 pi), partial (n_sel, 6, S, W, n_t).
template <bool PER_T>
__global__ void __launch_bounds__(kSpecThreads) k_tensor_direct(SpecArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NG = 6;
    const int k = blockIdx.y;
    const size_t slot = blockIdx.x;
    const int nd = A.n_cos * A.n_phi;
    const double* tau_g = A.tau + ((size_t)k * A.n_sel + slot) * nd;
    double* tau_s = reinterpret_cast<double*>(smem_raw);
    double* Bsm = tau_s + (A.tau_in_smem ? ((nd + 1) & ~1) : 0);                      // [n_cos][6]
    double2* red = reinterpret_cast<double2*>(Bsm + (size_t)A.n_cos * NG);            // [256][6]
    const double* tau = A.tau_in_smem ? tau_s : tau_g;
    if (A.tau_in_smem)
        for (int q = threadIdx.x; q < nd; q += kSpecThreads) tau_s[q] = tau_g[q];
    __syncthreads();

    const uint32_t a = A.sel[slot];
    const D4 xa = A.bub[(size_t)k * A.n_tot + a];
    const double ta = xa.t, za = xa.z;
    const int W_eff = min(A.n_w, kSpecThreads);
    const int n_ig = kSpecThreads / W_eff;
    const int wl = threadIdx.x % W_eff;
    const int ig = threadIdx.x / W_eff;
    const bool wthread = ig < n_ig;
    const double dphi = 2.0 * CUDART_PI / (double)A.n_phi;
    const double dcos = A.n_cos > 1 ? 2.0 / (double)(A.n_cos - 1) : 1.0;
    const double inv6pi = 1.0 / (6.0 * CUDART_PI);

    for (int s = 0; s < A.n_sets; ++s) {
        for (int wb = 0; wb < A.n_w; wb += W_eff) {
            const int wi = wb + wl;
            const bool wvalid = wthread && wi < A.n_w;
            const double wv = wvalid ? A.w[wi] : 0.0;
            double2 cacc[NG];
#pragma unroll
            for (int g = 0; g < NG; ++g) cacc[g] = make_double2(0.0, 0.0);
            for (int kt = 0; kt < A.n_t; ++kt) {
                const double t = A.t_arr[kt];
                if (t <= ta) continue;  // NGBF:1130
                const double dta = t - ta;
                // ---- B stage (NGBF:592-727) ----
                for (int i = threadIdx.x; i < A.n_cos; i += kSpecThreads) {
                    const double c = A.cos_thetax[i];
                    const double st = sqrt(fmax(__dsub_rn(1.0, __dmul_rn(c, c)), 0.0));
                    const double s2 = __dmul_rn(st, st), c2 = __dmul_rn(c, c), scz = __dmul_rn(st, c);
                    const double cubed = __dmul_rn(__dmul_rn(dta, dta), dta);
                    const double* trow = tau + (size_t)i * A.n_phi;
                    const int sidx = s * A.n_terms;
                    auto factor = [&](int j) {
                        const double tj = trow[j];
                        double f = 1.0;
                        if (tj > 0.0 && dta >= tj) {
                            const double ratio = tj / dta;
                            f = 0.0;
                            for (int m = 0; m < A.n_terms; ++m) f += A.coeffs[sidx + m] * pow(ratio, A.powers[sidx + m]);
                            if (A.has_damping) f *= exp(-dta * (1.0 - ratio) / A.damping);
                        }
                        return f;
                    };
                    auto basis = [&](int j, int g) {
                        const double cp = A.cosphi[j], sp = A.sinphi[j];
                        switch (g) {
                            case 0: return __dmul_rn(__dmul_rn(cp, cp), s2);
                            case 1: return __dmul_rn(__dmul_rn(cp, sp), s2);
                            case 2: return __dmul_rn(cp, scz);
                            case 3: return __dmul_rn(__dmul_rn(sp, sp), s2);
                            case 4: return __dmul_rn(sp, scz);
                            default: return c2;
                        }
                    };
                    // ndarray's eight-way unrolled sum over phi, per component
                    double p8[NG][8];
#pragma unroll
                    for (int g = 0; g < NG; ++g)
#pragma unroll
                        for (int u = 0; u < 8; ++u) p8[g][u] = 0.0;
                    const int nfull = A.n_phi & ~7;
                    for (int j0 = 0; j0 < nfull; j0 += 8) {
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            const int j = j0 + u;
                            const double f = factor(j);
                            const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
#pragma unroll
                            for (int g = 0; g < NG; ++g) p8[g][u] = __dadd_rn(p8[g][u], __dmul_rn(__dmul_rn(basis(j, g), f), wj));
                        }
                    }
                    double sums[NG];
#pragma unroll
                    for (int g = 0; g < NG; ++g) sums[g] = unrolled_sum8(p8[g], 0.0);
                    for (int j = nfull; j < A.n_phi; ++j) {
                        const double f = factor(j);
                        const double wj = (j == 0 || j == A.n_phi - 1) ? 0.5 : 1.0;
#pragma unroll
                        for (int g = 0; g < NG; ++g) sums[g] = __dadd_rn(sums[g], __dmul_rn(__dmul_rn(basis(j, g), f), wj));
                    }
#pragma unroll
                    for (int g = 0; g < NG; ++g) Bsm[(size_t)i * NG + g] = __dmul_rn(__dmul_rn(sums[g], dphi), cubed);
                }
                __syncthreads();
                // ---- A stage (NGBF:782-826): phase e^{-i w dt c_i} (dcos w_theta) ----
                double2 aacc[NG];
#pragma unroll
                for (int g = 0; g < NG; ++g) aacc[g] = make_double2(0.0, 0.0);
                if (wvalid) {
                    for (int i = ig; i < A.n_cos; i += n_ig) {
                        double sn, cs;
                        sincos(wv * (-dta * A.cos_thetax[i]), &sn, &cs);
                        const double vi = A.n_cos == 1 ? 1.0 : ((i == 0 || i == A.n_cos - 1) ? 0.5 : 1.0);
                        const double pfs = dcos * vi;
                        const double pr = cs * pfs, pim = sn * pfs;
#pragma unroll
                        for (int g = 0; g < NG; ++g) {
                            const double b = Bsm[(size_t)i * NG + g];
                            aacc[g].x += b * pr;
                            aacc[g].y += b * pim;
                        }
                    }
                }
#pragma unroll
                for (int g = 0; g < NG; ++g) red[(size_t)threadIdx.x * NG + g] = aacc[g];
                __syncthreads();
                // ---- C stage (NGBF:1145-1168): A e^{i w (t - z_a)} (dt w_t) ----
                if (PER_T && wvalid && ig == 0) {
                    double sn, cs;
                    sincos(wv * (t - za), &sn, &cs);
                    const double dtw = A.dt * ((kt == 0 || kt == A.n_t - 1) ? 0.5 : 1.0);
                    const double fr = cs * dtw, fi = sn * dtw;
                    for (int g = 0; g < NG; ++g) {
                        double2 at = make_double2(0.0, 0.0);
                        for (int q = 0; q < n_ig; ++q) {
                            const double2 v = red[(size_t)(q * W_eff + wl) * NG + g];
                            at.x += v.x;
                            at.y += v.y;
                        }
                        const size_t o = ((((size_t)slot * NG + g) * A.n_sets + s) * A.n_w + wi) * A.n_t + kt;
                        A.partial[o] = make_double2((at.x * fr - at.y * fi) * inv6pi, (at.x * fi + at.y * fr) * inv6pi);
                    }
                }
                if (!PER_T && wvalid && ig == 0) {
                    double sn, cs;
                    sincos(wv * (t - za), &sn, &cs);
                    const double dtw = A.dt * ((kt == 0 || kt == A.n_t - 1) ? 0.5 : 1.0);
                    const double fr = cs * dtw, fi = sn * dtw;
                    for (int g = 0; g < NG; ++g) {
                        double2 at = make_double2(0.0, 0.0);
                        for (int q = 0; q < n_ig; ++q) {
                            const double2 v = red[(size_t)(q * W_eff + wl) * NG + g];
                            at.x += v.x;
                            at.y += v.y;
                        }
                        cacc[g].x += at.x * fr - at.y * fi;
                        cacc[g].y += at.x * fi + at.y * fr;
                    }
                }
                __syncthreads();
            }
            if (!PER_T && wvalid && ig == 0) {
                for (int g = 0; g < NG; ++g) {
                    const size_t o = ((((size_t)k * A.n_sel + slot) * NG + g) * A.n_sets + s) * A.n_w + wi;
                    A.partial[o] = make_double2(cacc[g].x * inv6pi, cacc[g].y * inv6pi);
                }
            }
        }
    }
}

// Sum over radiating bubbles in index order (GBF:971-981).
__global__ void k_reduce(const double2* __restrict__ partial, size_t n_sel, size_t per, size_t kc,
                         double2* __restrict__ out) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t k = blockIdx.y;
    if (q >= per || k >= kc) return;
    double2 acc = make_double2(0.0, 0.0);
    const double2* p = partial + k * n_sel * per + q;
    for (size_t s = 0; s < n_sel; ++s) {
        double2 v = p[s * per];
        acc.x += v.x;
        acc.y += v.y;
    }
    out[k * per + q] = acc;
}

// ---------------------------------------------------------------------------
// Host orchestration.
// ---------------------------------------------------------------------------
namespace {

// Host -> device copy that is skipped when the bytes equal those of the
// previous upload into the same buffer (inputs stay resident in HBM).
template <class T>
T* upload(Device* dev, DevBuf& buf, const T* host, size_t n, BgwxTimings* tm) {
    const size_t bytes = n * sizeof(T);
    buf.ensure(bytes);
    if (bytes) {
        const unsigned char* hb = reinterpret_cast<const unsigned char*>(host);
        if (buf.shadow_valid && buf.shadow.size() == bytes && std::memcmp(buf.shadow.data(), hb, bytes) == 0)
            return static_cast<T*>(buf.p);
        buf.shadow.assign(hb, hb + bytes);
        CUDA_OK(cudaMemcpyAsync(buf.p, buf.shadow.data(), bytes, cudaMemcpyHostToDevice, dev->stream));
        buf.shadow_valid = true;
        if (tm) tm->h2d_bytes += (double)bytes;
    }
    return static_cast<T*>(buf.p);
}

size_t mask_budget_bytes() {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return (size_t)1 << 30;
    size_t b = free_b / 3;
    const size_t cap = (size_t)64 << 30;
    return std::max<size_t>((size_t)256 << 20, std::min(b, cap));
}

}  // namespace

size_t spectrum_max_frames_per_launch(const SpectrumJob& job) {
    const size_t nd = job.n_cos * job.n_phi;
    const size_t per = (job.tensor ? 6 : 2) * job.n_sets * job.n_w;
    const size_t per_k = job.n_sel * nd * sizeof(double) +
                         (job.kernel == BGWX_KERNEL_FP64_DIRECT ? job.n_sel * per * sizeof(double2)
                                                                : factored_bytes_per_frame(job));
    const size_t kc = std::max<size_t>(1, mask_budget_bytes() / std::max<size_t>(per_k, 1));
    return std::min<size_t>(kc, 65535);
}

LaunchShape last_launch_shape(const Device* dev) {
    LaunchShape s;
    s.frames_per_launch = dev->last_frames_per_launch;
    s.row_parts = dev->last_row_parts;
    s.gemm_stages = dev->last_gemm_stages;
    s.mask_chunking = dev->last_mask_chunking;
    return s;
}

void run_masks(Device* dev, const MaskJob& job, int32_t* out_codes, double* out_tau, BgwxTimings* tm) {
    CUDA_OK(cudaSetDevice(dev->id));
    const size_t nd = job.n_cos * job.n_phi;
    D4* bub = reinterpret_cast<D4*>(upload(dev, dev->bub, job.bubbles, 4 * job.n_tot, tm));
    D4* dirs = reinterpret_cast<D4*>(upload(dev, dev->dirs, job.dirs, 4 * nd, tm));
    uint32_t* sel = upload(dev, dev->sel, job.sel, job.n_sel, tm);
    dev->tau.ensure(job.n_sel * nd * sizeof(double));
    dev->codes.ensure(job.n_sel * nd * sizeof(int32_t));
    dev->counters.ensure(64);
    CUDA_OK(cudaMemsetAsync(dev->counters.p, 0, 64, dev->stream));
    CUDA_OK(cudaEventRecord(dev->ev[0], dev->stream));
    uint64_t nl = 0;
    launch_mask_pipeline(dev, bub, bub, job.n_int, job.n_tot, sel, nullptr, job.n_sel, dirs, nd, job.n_phi, 1, (double*)dev->tau.p,
                         (int32_t*)dev->codes.p, (unsigned long long*)dev->counters.p, true, &nl);
    CUDA_OK(cudaEventRecord(dev->ev[1], dev->stream));
    CUDA_OK(cudaMemcpyAsync(out_codes, dev->codes.p, job.n_sel * nd * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            dev->stream));
    if (out_tau)
        CUDA_OK(cudaMemcpyAsync(out_tau, dev->tau.p, job.n_sel * nd * sizeof(double), cudaMemcpyDeviceToHost,
                                dev->stream));
    unsigned long long fb = 0;
    CUDA_OK(cudaMemcpyAsync(&fb, dev->counters.p, sizeof fb, cudaMemcpyDeviceToHost, dev->stream));
    CUDA_OK(cudaStreamSynchronize(dev->stream));
    float ms = 0;
    CUDA_OK(cudaEventElapsedTime(&ms, dev->ev[0], dev->ev[1]));
    if (tm) {
        tm->masks_ms += ms;
        tm->total_ms += ms;
        tm->launches += nl;
        tm->directions += job.n_sel * nd;
        tm->fallbacks += fb;
        tm->d2h_bytes += (double)(job.n_sel * nd * (sizeof(int32_t) + (out_tau ? sizeof(double) : 0)));
    }
}

// The inputs the masks of a job depend on: bubbles, frame rotations, radiating selection, interior
// count and angular grid (the direction table follows from the grid).
static std::vector<unsigned char> masks_key(const SpectrumJob& job) {
    std::vector<unsigned char> k;
    auto put = [&](const void* p, size_t bytes) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        k.insert(k.end(), b, b + bytes);
    };
    const size_t sizes[6] = {job.n_int, job.n_tot, job.n_sel, job.n_cos, job.n_phi, job.rot ? job.n_k : 0};
    put(sizes, sizeof sizes);
    put(job.bubbles, 4 * job.n_tot * sizeof(double));
    put(job.sel, job.n_sel * sizeof(uint32_t));
    if (job.rot) put(job.rot, 9 * job.n_k * sizeof(double));
    return k;
}

// Per-stage device times of the last run_spectrum's launch chunks (masks, then
// spectrum = beta + GEMM for the factored kernels), once its work is complete.
static void add_stage_times(Device* dev, BgwxTimings* tm) {
    float ms_masks = 0, ms_spec = 0, ms_beta = 0, ms_gemm = 0;
    // diagnostic only: an event that was not recorded leaves the stage times at zero
    auto el = [](float& acc, cudaEvent_t a, cudaEvent_t b) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess)
            acc += ms;
        else
            cudaGetLastError();
    };
    for (size_t ci = 0; ci < dev->last_n_chunks; ++ci) {
        el(ms_masks, dev->chunk_ev[3 * ci], dev->chunk_ev[3 * ci + 1]);
        el(ms_spec, dev->chunk_ev[3 * ci + 1], dev->chunk_ev[3 * ci + 2]);
        if (dev->last_factored) {
            el(ms_beta, dev->fact_ev[3 * ci], dev->fact_ev[3 * ci + 1]);
            el(ms_gemm, dev->fact_ev[3 * ci + 1], dev->fact_ev[3 * ci + 2]);
        }
    }
    tm->masks_ms += ms_masks;
    tm->spectrum_ms += ms_spec;
    tm->beta_ms += ms_beta;
    tm->gemm_ms += ms_gemm;
}

// Error counters of a call: [0] mask fallbacks (u64), [1] non-zero when a
// tensor-core pipeline wait gave up.
static void check_counters(Device* dev, unsigned long long* fallbacks) {
    unsigned long long cnt[2] = {0, 0};
    CUDA_OK(cudaMemcpyAsync(cnt, dev->counters.p, sizeof cnt, cudaMemcpyDeviceToHost, dev->stream));
    CUDA_OK(cudaStreamSynchronize(dev->stream));
    if (cnt[1] != 0) throw Error{"tensor-core GEMM: a pipeline wait gave up; the result is invalid"};
    if (fallbacks) *fallbacks = cnt[0];
}

void run_spectrum(Device* dev, const SpectrumJob& job, double* out, bool out_is_device, BgwxTimings* tm,
                  bool nested, bool uploads_only) {
    CUDA_OK(cudaSetDevice(dev->id));
    const size_t nd = job.n_cos * job.n_phi;
    const size_t S = job.n_sets, W = job.n_w, K = job.n_k;
    const size_t per = (job.tensor ? 6 : 2) * S * W;
    if (job.tensor && job.kernel != BGWX_KERNEL_FP64_DIRECT)
        throw Error{"the tensor form runs only on the FP64 direct kernel"};
    if (job.n_cos > 4096 || job.n_phi > 65536) throw Error{"angular resolution too large for the GPU kernels"};
    if (job.n_t > (size_t)0x7fffffff || W > (size_t)0x7fffffff) throw Error{"n_t or n_w too large"};

    D4* bub = reinterpret_cast<D4*>(upload(dev, dev->bub, job.bubbles, 4 * job.n_tot, tm));
    D4* dirs = reinterpret_cast<D4*>(upload(dev, dev->dirs, job.dirs, 4 * nd, tm));
    double* cos_t = upload(dev, dev->cos_t, job.cos_thetax, job.n_cos, tm);
    double* sin2 = upload(dev, dev->sin2, job.sin2phi, job.n_phi, tm);
    double* cos2 = upload(dev, dev->cos2, job.cos2phi, job.n_phi, tm);
    double* coeffs = upload(dev, dev->coeffs, job.coeffs, S * job.n_terms, tm);
    double* powers = upload(dev, dev->powers, job.powers, S * job.n_terms, tm);
    double* t_arr = upload(dev, dev->t_arr, job.t_arr, job.n_t, tm);
    double* cutw = upload(dev, dev->cutw, job.cutoff, job.n_t, tm);
    double* w = upload(dev, dev->w, job.w, W, tm);
    uint32_t* sel = upload(dev, dev->sel, job.sel, job.n_sel, tm);
    double* rot = job.rot ? upload(dev, dev->rot, job.rot, 9 * K, tm) : nullptr;
    const bool batched = job.n_real > 0;
    if (batched && (job.kernel == BGWX_KERNEL_FP64_DIRECT || job.tensor))
        throw Error{"batched realizations run on the factored kernels only"};
    const uint2* ranges =
        batched ? reinterpret_cast<const uint2*>(upload(dev, dev->ranges, job.ranges, 2 * job.n_sel, tm)) : nullptr;
    const uint32_t* real_tiles = batched ? upload(dev, dev->real_tiles, job.real_tiles, job.n_real + 1, tm) : nullptr;
    const size_t out_blocks = batched ? job.n_real * K : K;  // (realization,) frame blocks of the output
    double* cosphi = job.tensor ? upload(dev, dev->cosphi, job.cosphi, job.n_phi, tm) : nullptr;
    double* sinphi = job.tensor ? upload(dev, dev->sinphi, job.sinphi, job.n_phi, tm) : nullptr;
    if (uploads_only) return;  // the inputs are resident; a captured launch sequence follows

    // frames per chunk: bounded by the mask buffer budget (and by the job's launch shape)
    size_t kc = std::min(K, spectrum_max_frames_per_launch(job));
    if (job.frames_per_launch) kc = std::min(kc, job.frames_per_launch);
    dev->last_frames_per_launch = kc;
    dev->last_row_parts = job.kernel == BGWX_KERNEL_FP64_DIRECT ? 1 : 0;  // the factored launch records its own
    dev->last_gemm_stages = 0;
    dev->last_mask_chunking = job.mask_chunking > 0 ? job.mask_chunking : 1;
    // masks kept for an adjoint call: every frame's delays and codes, written in place
    const bool keep = job.keep_masks && !batched && !job.tensor &&
                      K * job.n_sel * nd * (sizeof(double) + sizeof(int32_t)) <= mask_budget_bytes();
    if (keep) {
        dev->kept_valid = false;
        dev->kept_tau.ensure(K * job.n_sel * nd * sizeof(double));
        dev->kept_codes.ensure(K * job.n_sel * nd * sizeof(int32_t));
    } else {
        dev->tau.ensure(kc * job.n_sel * nd * sizeof(double));
    }
    if (job.kernel == BGWX_KERNEL_FP64_DIRECT) dev->partial.ensure(kc * job.n_sel * per * sizeof(double2));
    double2* final_out = out_is_device ? reinterpret_cast<double2*>(out) : nullptr;
    if (!final_out) {
        dev->out.ensure(out_blocks * per * sizeof(double2));
        final_out = (double2*)dev->out.p;
    }
    const size_t n_chunks = (K + kc - 1) / kc;
    while (dev->chunk_ev.size() < 3 * n_chunks) {
        cudaEvent_t e;
        CUDA_OK(cudaEventCreate(&e));
        dev->chunk_ev.push_back(e);
    }
    while (dev->fact_ev.size() < 3 * n_chunks) {
        cudaEvent_t e;
        CUDA_OK(cudaEventCreate(&e));
        dev->fact_ev.push_back(e);
    }
    if (rot) dev->bubrot.ensure(kc * job.n_tot * sizeof(D4));
    dev->tc_atab_valid = false;  // the time-phase digits are built by this call's first chunk
    if (!nested) {
        dev->counters.ensure(64);
        CUDA_OK(cudaMemsetAsync(dev->counters.p, 0, 64, dev->stream));
    }

    // shared memory of the direct kernel
    size_t smem_fixed = job.tensor ? (size_t)job.n_cos * 6 * sizeof(double) + (size_t)kSpecThreads * 6 * sizeof(double2)
                                   : (size_t)job.n_cos * kSetChunk * 2 * sizeof(double) +
                                         (size_t)kSpecThreads * kSetChunk * 2 * sizeof(double2);
    size_t smem_tau = ((nd + 1) & ~(size_t)1) * sizeof(double);
    int max_optin = 0;
    CUDA_OK(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev->id));
    int tau_in_smem = smem_fixed + smem_tau <= (size_t)max_optin ? 1 : 0;
    size_t smem = smem_fixed + (tau_in_smem ? smem_tau : 0);
    if (smem > (size_t)max_optin) throw Error{"n_cos_thetax too large for the shared-memory layout"};
    CUDA_OK(cudaFuncSetAttribute(k_spec_direct<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (job.tensor)
        CUDA_OK(cudaFuncSetAttribute(k_tensor_direct<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

    uint64_t launches = 0;
    record_event(dev, dev->ev[4]);
    for (size_t k0 = 0, ci = 0; k0 < K; k0 += kc, ++ci) {
        const size_t kn = std::min(kc, K - k0);
        cudaEvent_t* cev = &dev->chunk_ev[3 * ci];
        const D4* fb = bub;
        if (rot) {
            dim3 g((unsigned)((job.n_tot + 255) / 256), (unsigned)kn);
            k_rotate<<<g, 256, 0, dev->stream>>>(bub, rot + 9 * k0, job.n_tot, (D4*)dev->bubrot.p);
            CUDA_OK(cudaGetLastError());
            ++launches;
            fb = (const D4*)dev->bubrot.p;
        }
        record_event(dev, cev[0]);
        double* tau_k = keep ? (double*)dev->kept_tau.p + k0 * job.n_sel * nd : (double*)dev->tau.p;
        int32_t* codes_k = keep ? (int32_t*)dev->kept_codes.p + k0 * job.n_sel * nd : nullptr;
        launch_mask_pipeline(dev, bub, fb, job.n_int, job.n_tot, sel, ranges, job.n_sel, dirs, nd, job.n_phi, kn,
                             tau_k, codes_k, (unsigned long long*)dev->counters.p, k0 == 0, &launches,
                             job.mask_chunking);
        record_event(dev, cev[1]);
        if (job.kernel == BGWX_KERNEL_FP64_DIRECT) {
            SpecArgs A;
            A.bub = fb;
            A.n_tot = job.n_tot;
            A.sel = sel;
            A.n_sel = job.n_sel;
            A.tau = tau_k;
            A.n_cos = (int)job.n_cos;
            A.n_phi = (int)job.n_phi;
            A.cos_thetax = cos_t;
            A.sin2phi = sin2;
            A.cos2phi = cos2;
            A.coeffs = coeffs;
            A.powers = powers;
            A.n_sets = (int)S;
            A.n_terms = (int)job.n_terms;
            A.has_damping = job.has_damping ? 1 : 0;
            A.damping = job.damping;
            A.t_arr = t_arr;
            A.cutw = cutw;
            A.n_t = (int)job.n_t;
            A.dt = job.dt;
            A.w = w;
            A.n_w = (int)W;
            A.partial = (double2*)dev->partial.p;
            A.tau_in_smem = tau_in_smem;
            A.cosphi = cosphi;
            A.sinphi = sinphi;
            if (job.n_sel > 0x7fffffffULL) throw Error{"too many radiating bubbles"};
            dim3 g((unsigned)job.n_sel, (unsigned)kn);
            if (job.tensor)
                k_tensor_direct<false><<<g, kSpecThreads, smem, dev->stream>>>(A);
            else
                k_spec_direct<false><<<g, kSpecThreads, smem, dev->stream>>>(A);
            CUDA_OK(cudaGetLastError());
            ++launches;
            dim3 gr((unsigned)((per + 255) / 256), (unsigned)kn);
            k_reduce<<<gr, 256, 0, dev->stream>>>((const double2*)dev->partial.p, job.n_sel, per, kn,
                                                  final_out + k0 * per);
            CUDA_OK(cudaGetLastError());
            ++launches;
        } else {
            launches += launch_factored(dev, job, fb, sel, tau_k, cos_t, sin2, cos2, coeffs,
                                        powers, t_arr, cutw, w, k0, kn, final_out, real_tiles, &dev->fact_ev[3 * ci]);
        }
        record_event(dev, cev[2]);
    }
    record_event(dev, dev->ev[5]);
    if (keep) {
        dev->kept_key = masks_key(job);
        dev->kept_valid = true;
    }
    dev->last_n_chunks = n_chunks;
    dev->last_factored = job.kernel != BGWX_KERNEL_FP64_DIRECT;
    if (out_is_device) {
        if (tm) tm->launches += launches;
        if (!nested) check_counters(dev, nullptr);
        return;
    }
    CUDA_OK(cudaMemcpyAsync(out, final_out, out_blocks * per * sizeof(double2), cudaMemcpyDeviceToHost, dev->stream));
    unsigned long long fbk = 0;
    check_counters(dev, &fbk);
    float total = 0;
    CUDA_OK(cudaEventElapsedTime(&total, dev->ev[4], dev->ev[5]));
    if (tm) {
        add_stage_times(dev, tm);
        tm->total_ms += total;
        tm->launches += launches;
        tm->directions += K * job.n_sel * nd;
        tm->fallbacks += fbk;
        tm->d2h_bytes += (double)(out_blocks * per * sizeof(double2));
    }
}

// The launch sequence of a batched job as a CUDA graph.  Its kernels take the
// job's sizes and scalars by value and the device buffers by address, so a
// graph serves later calls whose key (every size, scalar and launch-shape
// choice) and buffer generation match; the inputs themselves are uploaded
// before each launch.  The first call of a key runs eagerly and sizes the
// grow-only buffers, the second captures the sequence (no allocation can
// happen during the capture then), later calls replay it.
static std::string batched_key(const SpectrumJob& b) {
    std::string k;
    auto put = [&](double v) {
        char buf[32];
        std::snprintf(buf, sizeof buf, "%a:", v);
        k += buf;
    };
    for (double v : {(double)b.kernel, (double)b.n_tot, (double)b.n_sel, (double)b.n_real, (double)b.n_cos,
                     (double)b.n_phi, (double)b.n_t, (double)b.n_w, (double)b.n_sets, (double)b.n_terms,
                     (double)b.has_damping, b.damping, b.dt, (double)b.n_k, (double)b.frames_per_launch,
                     (double)b.row_parts, (double)b.gemm_stages, (double)b.mask_chunking})
        put(v);
    return k;
}

static void run_batched(Device* dev, SpectrumJob b, double2* eo, BgwxTimings* local) {
    // the frames per launch are fixed here: a captured sequence must not depend on free memory
    if (!b.frames_per_launch) b.frames_per_launch = std::min(b.n_k, spectrum_max_frames_per_launch(b));
    const std::string key = batched_key(b);
    double* out = reinterpret_cast<double*>(eo);
    run_spectrum(dev, b, out, true, local, true, true);  // uploads what changed
    if (dev->ens_graph && dev->ens_graph_key == key && dev->ens_graph_gen == dev->buffers_generation()) {
        CUDA_OK(cudaGraphLaunch(dev->ens_graph, dev->stream));
        local->launches += dev->ens_graph_launches;
        dev->last_n_chunks = dev->ens_graph_chunks;
        dev->last_factored = true;
        ++local->graph_replays;
        return;
    }
    if (dev->ens_sized_key != key || dev->ens_sized_gen != dev->buffers_generation()) {
        run_spectrum(dev, b, out, true, local, true);
        dev->ens_sized_key = key;
        dev->ens_sized_gen = dev->buffers_generation();
        return;
    }
    if (dev->ens_graph) {
        CUDA_OK(cudaGraphExecDestroy(dev->ens_graph));
        dev->ens_graph = nullptr;
    }
    BgwxTimings cap{};
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(dev->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGetLastError();  // a stream that cannot be captured: run eagerly
        run_spectrum(dev, b, out, true, local, true);
        return;
    }
    dev->capturing = true;
    try {
        run_spectrum(dev, b, out, true, &cap, true);
    } catch (...) {
        dev->capturing = false;
        cudaStreamEndCapture(dev->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
    }
    dev->capturing = false;
    CUDA_OK(cudaStreamEndCapture(dev->stream, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    CUDA_OK(e);
    if (dev->buffers_generation() != dev->ens_sized_gen) {  // a buffer moved during the capture: do not keep it
        cudaGraphExecDestroy(exec);
        throw Error{"batched ensemble: a device buffer was reallocated while the launch sequence was captured"};
    }
    dev->ens_graph = exec;
    dev->ens_graph_key = key;
    dev->ens_graph_gen = dev->buffers_generation();
    dev->ens_graph_launches = cap.launches;
    dev->ens_graph_chunks = dev->last_n_chunks;
    CUDA_OK(cudaGraphLaunch(exec, dev->stream));
    local->launches += cap.launches;
}

void run_ensemble(Device* dev, const std::vector<SpectrumJob>& jobs, double* out, BgwxTimings* tm, bool autotune) {
    CUDA_OK(cudaSetDevice(dev->id));
    const size_t R = jobs.size();
    if (R == 0) return;
    const SpectrumJob& j0 = jobs[0];
    const size_t per_r = j0.n_k * 2 * j0.n_sets * j0.n_w;  // complex values per realization
    const bool batched = j0.kernel != BGWX_KERNEL_FP64_DIRECT;
    // One job over every realization: bubbles one realization after another, radiating slots
    // padded so that each realization starts a GEMM column tile; each launch of the pipeline
    // (rotation, masks, beta, GEMM, reduction) then covers all realizations of its frames.
    SpectrumJob b = j0;
    std::vector<double> bub;
    std::vector<uint32_t> sel, ranges, real_tiles(R + 1, 0);
    size_t radiating = 0;
    if (batched) {
        const size_t bpt = factored_bubbles_per_tile(j0);
        size_t rows = 0, tiles = 0;
        for (size_t r = 0; r < R; ++r) {
            const SpectrumJob& j = jobs[r];
            real_tiles[r] = (uint32_t)tiles;
            bub.insert(bub.end(), j.bubbles, j.bubbles + 4 * j.n_tot);
            const size_t nt = (j.n_sel + bpt - 1) / bpt;
            for (size_t q = 0; q < nt * bpt; ++q) {
                sel.push_back(q < j.n_sel ? (uint32_t)(rows + j.sel[q]) : kNoSlot);
                ranges.push_back((uint32_t)rows);
                ranges.push_back((uint32_t)j.n_tot);
            }
            rows += j.n_tot;
            tiles += nt;
            radiating += j.n_sel;
            if (rows > 0xFFFFFFF0ULL || sel.size() > 0x7FFFFFFFULL) throw Error{"ensemble too large for one call"};
        }
        real_tiles[R] = (uint32_t)tiles;
        b.bubbles = bub.data();
        b.n_tot = rows;
        b.n_int = rows;  // sel holds indices into the whole array; padding slots are kNoSlot
        b.sel = sel.data();
        b.n_sel = sel.size();
        b.ranges = ranges.data();
        b.real_tiles = real_tiles.data();
        b.n_real = R;
        if (autotune && radiating > 0) {
            const LaunchShape s = autotune_launch_shape(dev, b);
            b.frames_per_launch = s.frames_per_launch;
            b.row_parts = s.row_parts;
            b.gemm_stages = s.gemm_stages;
            b.mask_chunking = s.mask_chunking;
        }
    }
    dev->ens_out.ensure(R * per_r * sizeof(double2));
    double2* eo = (double2*)dev->ens_out.p;
    CUDA_OK(cudaMemsetAsync(eo, 0, R * per_r * sizeof(double2), dev->stream));
    BgwxTimings local{};
    dev->counters.ensure(64);
    CUDA_OK(cudaMemsetAsync(dev->counters.p, 0, 64, dev->stream));
    CUDA_OK(cudaEventRecord(dev->ev[6], dev->stream));
    if (batched) {
        if (radiating > 0) run_batched(dev, b, eo, &local);
    } else {
        std::vector<size_t> order(R);
        for (size_t r = 0; r < R; ++r) order[r] = r;
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
            return jobs[x].n_sel * jobs[x].n_tot > jobs[y].n_sel * jobs[y].n_tot;
        });
        for (size_t r : order) {
            if (jobs[r].n_sel == 0) continue;
            run_spectrum(dev, jobs[r], reinterpret_cast<double*>(eo + r * per_r), true, &local, true);
        }
    }
    CUDA_OK(cudaEventRecord(dev->ev[7], dev->stream));
    CUDA_OK(cudaMemcpyAsync(out, eo, R * per_r * sizeof(double2), cudaMemcpyDeviceToHost, dev->stream));
    check_counters(dev, nullptr);
    float total = 0;
    CUDA_OK(cudaEventElapsedTime(&total, dev->ev[6], dev->ev[7]));
    if (tm) {
        if (batched && radiating > 0) add_stage_times(dev, tm);  // the one batched run's stages
        tm->graph_replays += local.graph_replays;
        tm->total_ms += total;
        tm->launches += local.launches;
        tm->h2d_bytes += local.h2d_bytes;
        tm->d2h_bytes += (double)(R * per_r * sizeof(double2));
        for (const auto& j : jobs) tm->directions += j.n_k * j.n_sel * j.n_cos * j.n_phi;
    }
}

void run_adjoint(Device* dev, const SpectrumJob& job, const double* gbar, double* g_par, double* g_bub,
                 BgwxTimings* tm) {
    CUDA_OK(cudaSetDevice(dev->id));
    const size_t nd = job.n_cos * job.n_phi;
    const size_t S = job.n_sets, W = job.n_w, K = job.n_k;
    const size_t per = 2 * S * W;
    const size_t SM = S * job.n_terms;
    if (job.n_t > (size_t)0x7fffffff || W > (size_t)0x7fffffff) throw Error{"n_t or n_w too large"};
    D4* bub = reinterpret_cast<D4*>(upload(dev, dev->bub, job.bubbles, 4 * job.n_tot, tm));
    D4* dirs = reinterpret_cast<D4*>(upload(dev, dev->dirs, job.dirs, 4 * nd, tm));
    double* cos_t = upload(dev, dev->cos_t, job.cos_thetax, job.n_cos, tm);
    double* sin2 = upload(dev, dev->sin2, job.sin2phi, job.n_phi, tm);
    double* cos2 = upload(dev, dev->cos2, job.cos2phi, job.n_phi, tm);
    double* coeffs = upload(dev, dev->coeffs, job.coeffs, SM, tm);
    double* powers = upload(dev, dev->powers, job.powers, SM, tm);
    double* t_arr = upload(dev, dev->t_arr, job.t_arr, job.n_t, tm);
    double* cutw = upload(dev, dev->cutw, job.cutoff, job.n_t, tm);
    double* w = upload(dev, dev->w, job.w, W, tm);
    uint32_t* sel = upload(dev, dev->sel, job.sel, job.n_sel, tm);
    double* rot = job.rot ? upload(dev, dev->rot, job.rot, 9 * K, tm) : nullptr;
    double2* gb = reinterpret_cast<double2*>(upload(dev, dev->adj_gbar, gbar, 2 * K * per, tm));

    const size_t per_k = adjoint_bytes_per_frame(job);
    size_t kc = std::max<size_t>(1, std::min(K, mask_budget_bytes() / std::max<size_t>(per_k, 1)));
    kc = std::min<size_t>(kc, 65535);
    const size_t rows = job.n_sel * job.n_cos;
    // the masks kept by the last spectrum call on the same inputs are reused (same stream, so that
    // call's kernels have finished before this call's read them)
    const bool reuse = dev->kept_valid && dev->kept_key == masks_key(job);
    if (!reuse) {
        dev->tau.ensure(kc * job.n_sel * nd * sizeof(double));
        dev->codes.ensure(kc * job.n_sel * nd * sizeof(int32_t));
    }
    // the fixed-point gradient sums of a chunk hold fewer than 2^31 contributions
    const size_t per_frame_contrib = 2 * job.n_sel * nd + job.n_sel;
    kc = std::max<size_t>(1, std::min(kc, ((size_t)1 << 31) / std::max<size_t>(per_frame_contrib, 1)));
    if (per_frame_contrib >= ((size_t)1 << 31)) throw Error{"adjoint: too many (bubble, patch) pairs per frame"};
    const size_t n_dbl = kc * (2 * rows * job.n_t * 2 * S + job.n_sel * nd + rows * (2 + 2 * SM) + job.n_sel * 4);
    dev->adj_scratch.ensure(n_dbl * sizeof(double) + job.n_tot * 8 * sizeof(long long) + 64);
    AdjointScratch sc;
    sc.bbar = (double*)dev->adj_scratch.p;
    sc.imq = sc.bbar + kc * rows * job.n_t * 2 * S;
    sc.taubar = sc.imq + kc * rows * job.n_t * 2 * S;
    sc.rowpart = sc.taubar + kc * job.n_sel * nd;
    sc.bubpart = sc.rowpart + kc * rows * (2 + 2 * SM);
    sc.gfix = reinterpret_cast<long long*>(sc.bubpart + kc * job.n_sel * 4);
    sc.gexp = reinterpret_cast<int*>(sc.gfix + job.n_tot * 8);
    CUDA_OK(cudaMemsetAsync(sc.gfix, 0, job.n_tot * 8 * sizeof(long long), dev->stream));
    dev->adj_grad.ensure((4 * job.n_tot + 2 * SM) * sizeof(double));
    double* d_gbub = (double*)dev->adj_grad.p;
    double* d_gpar = d_gbub + 4 * job.n_tot;
    CUDA_OK(cudaMemsetAsync(d_gbub, 0, (4 * job.n_tot + 2 * SM) * sizeof(double), dev->stream));
    if (rot) dev->bubrot.ensure(kc * job.n_tot * sizeof(D4));
    dev->counters.ensure(64);
    CUDA_OK(cudaMemsetAsync(dev->counters.p, 0, 64, dev->stream));

    uint64_t launches = 0;
    CUDA_OK(cudaEventRecord(dev->ev[4], dev->stream));
    const size_t mt_bytes = (job.n_cos * W * job.n_t * sizeof(double2) + 255) & ~(size_t)255;
    dev->adj_mtab.ensure(mt_bytes + job.n_sel * job.n_t * (4 + SM) * sizeof(double));
    double2* mt = (double2*)dev->adj_mtab.p;
    double* tt = (double*)((unsigned char*)dev->adj_mtab.p + mt_bytes);
    launches += launch_adjoint_tables(dev, job, bub, sel, cos_t, t_arr, w, powers, mt, tt);
    for (size_t k0 = 0; k0 < K; k0 += kc) {
        const size_t kn = std::min(kc, K - k0);
        const D4* fb = bub;
        if (rot) {
            dim3 g((unsigned)((job.n_tot + 255) / 256), (unsigned)kn);
            k_rotate<<<g, 256, 0, dev->stream>>>(bub, rot + 9 * k0, job.n_tot, (D4*)dev->bubrot.p);
            CUDA_OK(cudaGetLastError());
            ++launches;
            fb = (const D4*)dev->bubrot.p;
        }
        const double* tau_k = reuse ? (const double*)dev->kept_tau.p + k0 * job.n_sel * nd : (const double*)dev->tau.p;
        const int32_t* codes_k =
            reuse ? (const int32_t*)dev->kept_codes.p + k0 * job.n_sel * nd : (const int32_t*)dev->codes.p;
        if (!reuse)
            launch_mask_pipeline(dev, bub, fb, job.n_int, job.n_tot, sel, nullptr, job.n_sel, dirs, nd, job.n_phi, kn,
                                 (double*)dev->tau.p, (int32_t*)dev->codes.p, (unsigned long long*)dev->counters.p,
                                 k0 == 0, &launches);
        launches += launch_adjoint_chunk(dev, job, fb, sel, tau_k, codes_k,
                                         dirs, cos_t, sin2, cos2, coeffs, powers, t_arr, cutw, w,
                                         rot ? rot + 9 * k0 : nullptr, gb + k0 * per, kn, sc, mt, tt, d_gbub,
                                         d_gpar);
    }
    CUDA_OK(cudaEventRecord(dev->ev[5], dev->stream));
    CUDA_OK(cudaMemcpyAsync(g_bub, d_gbub, 4 * job.n_tot * sizeof(double), cudaMemcpyDeviceToHost, dev->stream));
    CUDA_OK(cudaMemcpyAsync(g_par, d_gpar, 2 * SM * sizeof(double), cudaMemcpyDeviceToHost, dev->stream));
    CUDA_OK(cudaStreamSynchronize(dev->stream));
    float total = 0;
    CUDA_OK(cudaEventElapsedTime(&total, dev->ev[4], dev->ev[5]));
    if (tm) {
        tm->total_ms += total;
        tm->launches += launches;
        tm->directions += K * job.n_sel * nd;
        tm->d2h_bytes += (double)((4 * job.n_tot + 2 * SM) * sizeof(double));
    }
}

// out += sum over the chunk's bubbles, in slot order, of their per-step values.
__global__ void k_reduce_integrand(const double2* __restrict__ partial, size_t n, size_t per, double2* __restrict__ out) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= per) return;
    double2 acc = out[q];
    for (size_t a = 0; a < n; ++a) {
        const double2 v = partial[a * per + q];
        acc.x += v.x;
        acc.y += v.y;
    }
    out[q] = acc;
}

void run_integrand(Device* dev, const SpectrumJob& job, double* out, BgwxTimings* tm) {
    CUDA_OK(cudaSetDevice(dev->id));
    const size_t nd = job.n_cos * job.n_phi;
    const size_t S = job.n_sets, W = job.n_w, T = job.n_t;
    const size_t per = (job.tensor ? 6 : 2) * S * W * T;  // complex values of one bubble's integrand
    if (job.n_cos > 4096 || job.n_phi > 65536) throw Error{"angular resolution too large for the GPU kernels"};
    D4* bub = reinterpret_cast<D4*>(upload(dev, dev->bub, job.bubbles, 4 * job.n_tot, tm));
    D4* dirs = reinterpret_cast<D4*>(upload(dev, dev->dirs, job.dirs, 4 * nd, tm));
    double* cos_t = upload(dev, dev->cos_t, job.cos_thetax, job.n_cos, tm);
    double* sin2 = upload(dev, dev->sin2, job.sin2phi, job.n_phi, tm);
    double* cos2 = upload(dev, dev->cos2, job.cos2phi, job.n_phi, tm);
    double* coeffs = upload(dev, dev->coeffs, job.coeffs, S * job.n_terms, tm);
    double* powers = upload(dev, dev->powers, job.powers, S * job.n_terms, tm);
    double* t_arr = upload(dev, dev->t_arr, job.t_arr, T, tm);
    double* cutw = upload(dev, dev->cutw, job.cutoff, T, tm);
    double* w = upload(dev, dev->w, job.w, W, tm);
    uint32_t* sel = upload(dev, dev->sel, job.sel, job.n_sel, tm);
    double* cosphi = job.tensor ? upload(dev, dev->cosphi, job.cosphi, job.n_phi, tm) : nullptr;
    double* sinphi = job.tensor ? upload(dev, dev->sinphi, job.sinphi, job.n_phi, tm) : nullptr;
    // bubbles per chunk: bounded by the per-bubble integrand buffer
    const size_t budget = mask_budget_bytes();
    size_t chunk = std::max<size_t>(1, std::min(job.n_sel, budget / std::max<size_t>(per * sizeof(double2), 1)));
    chunk = std::min<size_t>(chunk, 65535);
    dev->tau.ensure(job.n_sel * nd * sizeof(double));
    dev->partial.ensure(chunk * per * sizeof(double2));
    dev->out.ensure(per * sizeof(double2));
    dev->counters.ensure(64);
    CUDA_OK(cudaMemsetAsync(dev->counters.p, 0, 64, dev->stream));
    CUDA_OK(cudaMemsetAsync(dev->out.p, 0, per * sizeof(double2), dev->stream));
    size_t smem = job.tensor ? (size_t)job.n_cos * 6 * sizeof(double) + (size_t)kSpecThreads * 6 * sizeof(double2)
                             : (size_t)job.n_cos * kSetChunk * 2 * sizeof(double) +
                                   (size_t)kSpecThreads * kSetChunk * 2 * sizeof(double2);
    const size_t smem_tau = ((nd + 1) & ~(size_t)1) * sizeof(double);
    int max_optin = 0;
    CUDA_OK(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev->id));
    const int tau_in_smem = smem + smem_tau <= (size_t)max_optin ? 1 : 0;
    if (tau_in_smem) smem += smem_tau;
    if (smem > (size_t)max_optin) throw Error{"n_cos_thetax too large for the shared-memory layout"};
    CUDA_OK(cudaFuncSetAttribute(k_spec_direct<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (job.tensor)
        CUDA_OK(cudaFuncSetAttribute(k_tensor_direct<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    uint64_t launches = 0;
    CUDA_OK(cudaEventRecord(dev->ev[4], dev->stream));
    launch_mask_pipeline(dev, bub, bub, job.n_int, job.n_tot, sel, nullptr, job.n_sel, dirs, nd, job.n_phi, 1, (double*)dev->tau.p,
                         nullptr, (unsigned long long*)dev->counters.p, true, &launches);
    for (size_t s0 = 0; s0 < job.n_sel; s0 += chunk) {
        const size_t n = std::min(chunk, job.n_sel - s0);
        CUDA_OK(cudaMemsetAsync(dev->partial.p, 0, n * per * sizeof(double2), dev->stream));
        SpecArgs A;
        A.bub = bub;
        A.n_tot = job.n_tot;
        A.sel = sel + s0;
        A.n_sel = n;
        A.tau = (const double*)dev->tau.p + s0 * nd;
        A.n_cos = (int)job.n_cos;
        A.n_phi = (int)job.n_phi;
        A.cos_thetax = cos_t;
        A.sin2phi = sin2;
        A.cos2phi = cos2;
        A.coeffs = coeffs;
        A.powers = powers;
        A.n_sets = (int)S;
        A.n_terms = (int)job.n_terms;
        A.has_damping = job.has_damping ? 1 : 0;
        A.damping = job.damping;
        A.t_arr = t_arr;
        A.cutw = cutw;
        A.n_t = (int)T;
        A.dt = job.dt;
        A.w = w;
        A.n_w = (int)W;
        A.partial = (double2*)dev->partial.p;
        A.tau_in_smem = tau_in_smem;
        A.cosphi = cosphi;
        A.sinphi = sinphi;
        if (job.tensor)
            k_tensor_direct<true><<<dim3((unsigned)n, 1), kSpecThreads, smem, dev->stream>>>(A);
        else
            k_spec_direct<true><<<dim3((unsigned)n, 1), kSpecThreads, smem, dev->stream>>>(A);
        CUDA_OK(cudaGetLastError());
        k_reduce_integrand<<<(unsigned)((per + 255) / 256), 256, 0, dev->stream>>>((const double2*)dev->partial.p, n,
                                                                                   per, (double2*)dev->out.p);
        CUDA_OK(cudaGetLastError());
        launches += 2;
    }
    CUDA_OK(cudaEventRecord(dev->ev[5], dev->stream));
    CUDA_OK(cudaMemcpyAsync(out, dev->out.p, per * sizeof(double2), cudaMemcpyDeviceToHost, dev->stream));
    CUDA_OK(cudaStreamSynchronize(dev->stream));
    float total = 0;
    CUDA_OK(cudaEventElapsedTime(&total, dev->ev[4], dev->ev[5]));
    if (tm) {
        tm->total_ms += total;
        tm->spectrum_ms += total;
        tm->launches += launches;
        tm->directions += job.n_sel * nd;
        tm->d2h_bytes += (double)(per * sizeof(double2));
    }
}

}  // namespace bgw
