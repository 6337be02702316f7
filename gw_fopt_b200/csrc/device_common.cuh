// Device-side building blocks shared by the kernels: the spacetime 4-vector,
// unfused FP64 arithmetic for the collision decisions, buffers and the
// per-handle device state.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include <string>
#include <vector>

#include "bgw_internal.h"

namespace bgw {

#define CUDA_OK(x)                                                                                  \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess)                                                                      \
            throw ::bgw::Error{std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" #x ")"}; \
    } while (0)

// Spacetime event / interval (t, x, y, z); 32-byte aligned rows in HBM.
struct __align__(16) D4 {
    double t, x, y, z;
};

// Unfused IEEE operations: the collision decisions must reproduce Rust's
// f64 arithmetic (no a*b+c contraction), so they never use plain operators.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Minkowski scalar product, signature (-,+,+,+), summed left to right
// (rust/bubble-gw/src/many_bubbles/spacetime.rs:593-600 via nalgebra's U4 dot).
__device__ __forceinline__ double mdot(const D4& a, const D4& b) {
    double p0 = dmul(-a.t, b.t);
    double p1 = dmul(a.x, b.x);
    double p2 = dmul(a.y, b.y);
    double p3 = dmul(a.z, b.z);
    return dadd(dadd(dadd(p0, p1), p2), p3);
}

__device__ __forceinline__ D4 dsub4(const D4& b, const D4& a) {
    return D4{dsub(b.t, a.t), dsub(b.x, a.x), dsub(b.y, a.y), dsub(b.z, a.z)};
}

// Grow-only device buffer.  `shadow` keeps the bytes last uploaded from the
// host so that unchanged inputs stay resident in HBM across calls.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    std::vector<unsigned char> shadow;
    bool shadow_valid = false;
    unsigned long long gen = 0;  // (re)allocations of this buffer
    void ensure(size_t bytes) {
        if (bytes <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes < 256 ? 256 : bytes;
        CUDA_OK(cudaMalloc(&p, want));
        cap = want;
        shadow_valid = false;
        ++gen;
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

struct Device {
    int id = 0;
    int n_sm = 148;                 // multiprocessors of this device
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;  // own_stream or a caller-provided stream
    cudaEvent_t ev[8] = {};
    std::vector<cudaEvent_t> chunk_ev;  // 3 per k-hat chunk
    std::vector<cudaEvent_t> fact_ev;   // 3 per k-hat chunk: before beta, before GEMM, after GEMM
    DevBuf bub, bubrot, dirs, cos_t, sin2, cos2, coeffs, powers, t_arr, cutw, w, sel, rot, cosphi, sinphi;
    DevBuf tau, codes, partial, out, counters, nblists;
    DevBuf ranges, real_tiles;  // batched jobs: per-slot realization rows, first tile per realization
    DevBuf fact_D, fact_kfirst, beta, fact_partial;  // factored-kernel work arrays
    DevBuf ens_out;                                  // batched ensemble: all realizations' spectra
    DevBuf pp_in, pp_small, pp_out;                  // spectrum post-processing: input, small tables, output
    DevBuf beta_scale;                               // int8 tensor-core GEMM: per-(bubble, row) beta scales
    DevBuf fact_Dmax;                                // int8 tensor-core GEMM: per-(bubble, block) time-table maxima
    DevBuf tc_atab;                                  // int8 tensor-core GEMM: time-phase digits
    bool capturing = false;      // the stream is being captured into a CUDA graph
    size_t last_n_chunks = 0;    // launch chunks of the last run_spectrum (their events hold its stage times)
    // the batched ensemble's launch sequence: sized by an eager run of a shape, captured by the
    // next call of that shape and replayed by later ones
    std::string ens_sized_key, ens_graph_key;
    unsigned long long ens_sized_gen = 0, ens_graph_gen = 0;
    cudaGraphExec_t ens_graph = nullptr;
    uint64_t ens_graph_launches = 0;
    size_t ens_graph_chunks = 0;
    bool last_factored = false;
    bool tc_atab_valid = false;  // tc_atab holds the current call's time-phase digits
    DevBuf adj_gbar, adj_scratch, adj_grad, adj_mtab; // adjoint: cotangents, work arrays, gradients, phases
    // masks kept by a spectrum call for the adjoint: (K, n_sel, n_cos n_phi) delays and codes, and the
    // inputs they were computed from (bubbles, rotations, selection, grid sizes)
    DevBuf kept_tau, kept_codes;
    std::vector<unsigned char> kept_key;
    bool kept_valid = false;
    size_t last_frames_per_launch = 0;               // launch shape of the last spectrum call
    int last_row_parts = 0;
    int last_gemm_stages = 0;
    int last_mask_chunking = 0;
    // Changes whenever one of this device's buffers is reallocated: a captured CUDA graph holds
    // buffer addresses and stays valid only while the count is unchanged.
    unsigned long long buffers_generation() const {
        unsigned long long g = 0;
        for (const DevBuf* b : {&bub, &bubrot, &dirs, &cos_t, &sin2, &cos2, &coeffs, &powers, &t_arr, &cutw, &w, &sel,
                                &rot, &cosphi, &sinphi, &tau, &codes, &partial, &out, &counters, &nblists, &ranges,
                                &real_tiles, &fact_D, &fact_kfirst, &beta, &fact_partial, &ens_out, &beta_scale,
                                &fact_Dmax, &tc_atab})
            g += b->gen;
        return g;
    }
    ~Device();
};

// Records a timing event on the device's stream.  Inside a stream capture a
// plain record only orders the graph's nodes; an external record becomes a
// node that records the event whenever the graph runs.
inline void record_event(Device* d, cudaEvent_t e) {
    CUDA_OK(d->capturing ? cudaEventRecordWithFlags(e, d->stream, cudaEventRecordExternal)
                         : cudaEventRecord(e, d->stream));
}

}  // namespace bgw
