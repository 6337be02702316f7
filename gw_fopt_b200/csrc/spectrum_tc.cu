// Mixed-precision time-phase GEMM on the 5th-generation tensor cores.
//
// For each cos-theta row i the factored spectrum needs Y_i = M_i beta_i with
// M_i[w, k] = e^{i w (1 - c_i) t_k} (rows: Re and Im of 64 frequencies) and
// beta_i[k, col] (columns: bubble x set x {+, x}); the epilogue applies
// e^{i w (t_a c_i - z_a)} per (w, bubble) and sums over the tile's bubbles
// (spectrum_factored.cu holds the derivation).  Here the product runs as
// tcgen05.mma kind::tf32 with FP32 accumulation in tensor memory, each FP32
// operand split into two TF32 parts, x = x_hi + x_lo, and three products
// A_hi B_lo + A_lo B_hi + A_hi B_hi per K step (the A_lo B_lo term is below
// FP32 rounding), which keeps FP32-level operand accuracy.
//
// One CTA per (64-frequency tile, 128-column tile), looping over the rows i;
// per row the K dimension is the time steps from the tile's first active
// block of 32 steps on.  Warp roles (13 warps):
//   0-3   A producers: thread = tensor-memory lane = GEMM row (w, Re|Im).  The
//         time phase of step 32 kb + n is z_kb P_n: the block anchor z_kb
//         advances by an FP64 complex recurrence from an FP64 sincos at the
//         row's first block, P_n = e^{i w' n dt} is a per-row FP32 table; the
//         FP32 value is split and stored to tensor memory (tcgen05.st).
//   4-7   B producers: beta (FP32, HBM) -> split -> shared memory in the
//         K-major 128-byte-swizzled layout, 32 steps per stage.
//   8-11  epilogue: thread = lane.  Per row the phases e^{i w (t_a c_i - z_a)}
//         (FP64 argument reduction, FP32 sincos) go to a shared-memory table;
//         every block of 32 steps the accumulator (tcgen05.ld) is multiplied by
//         them and summed per (w, set, +/x) in FP64.
//   12    MMA issue (one thread) and tensor-memory allocation.
// Stages: 4 (A in tensor memory, B in shared memory), full/empty mbarriers;
// the accumulator is double-buffered across blocks of 32 steps.  Every wait is bounded:
// on a timeout the block records an error flag, tells the other roles to
// stop, waits for its issued MMAs to finish and frees its tensor memory.
//
// Tensor memory (512 columns): accumulators at columns 0 and 128; stage s's
// A_hi at 256 + 64 s and A_lo at 256 + 64 s + 32.

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "bgw_internal.h"
#include "device_common.cuh"
#include "spectrum_factored.cuh"
#include "spectrum_tc.cuh"
#include "tc_ptx.cuh"

namespace bgw {

namespace {

constexpr int kTcRows = 128;     // GEMM rows: 64 frequencies x (Re, Im)
constexpr int kTcWT = 64;        // frequencies per CTA
constexpr int kTcCols = 128;     // GEMM columns per CTA
constexpr int kTcKB = 32;        // time steps per stage (128 bytes of TF32)
constexpr int kTcStages = 4;
constexpr int kTcFoldKB = 1;     // blocks of 32 steps accumulated in tensor memory before the FP64 fold
constexpr int kTcWarps = 13;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr uint32_t kTmemCols = 512;
constexpr int kBTileBytes = kTcCols * kTcKB * 4;  // 16 KB per (stage, hi|lo)
constexpr int kEStride = 66;     // phase-table row (one frequency, 64 bubbles) padded against bank conflicts

struct SmemLayout {
    static constexpr int b_hi = 0;
    static constexpr int b_lo = kTcStages * kBTileBytes;
    static constexpr int bars = 2 * kTcStages * kBTileBytes;  // full[S], empty[S], accf[2], acce[2], drain
    static constexpr int n_bars = 2 * kTcStages + 5;
    static constexpr int tslot = bars + 8 * n_bars;
    static constexpr int abort_flag = tslot + 4;
    static constexpr int binfo = tslot + 16;                  // int[64]
    static constexpr int bt = binfo + 64 * 4;                 // double[64]
    static constexpr int bz = bt + 64 * 8;                    // double[64]
    static constexpr int etab = bz + 64 * 8;                  // float2[64 w][kEStride] (bubbles)
    static constexpr int ptab = etab + 64 * 66 * 8;           // float2[32 steps][64 w]
    static constexpr int total = ptab + 32 * 64 * 8;
};

__device__ __forceinline__ uint32_t swz128(int n, int c) {
    return (uint32_t)((n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4));
}

template <int S>
__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_tc(TcArgs A) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                         ~static_cast<uintptr_t>(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + SmemLayout::bars);
    uint64_t* full = bars;
    uint64_t* empty = bars + kTcStages;
    uint64_t* accf = bars + 2 * kTcStages;
    uint64_t* acce = accf + 2;
    uint64_t* drain = acce + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SmemLayout::tslot);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + SmemLayout::abort_flag);
    int* binfo = reinterpret_cast<int*>(sm + SmemLayout::binfo);
    double* bt = reinterpret_cast<double*>(sm + SmemLayout::bt);
    double* bz = reinterpret_cast<double*>(sm + SmemLayout::bz);

    constexpr int CPB = 2 * S;  // columns per bubble
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int w0 = blockIdx.x * kTcWT;
    const int frame = blockIdx.y / A.tiles_per_frame;
    const int tile = blockIdx.y % A.tiles_per_frame;
    const D4* B = A.bub + (size_t)frame * A.n_tot;

    if (tid < 64) {
        const int slot = tile * A.bpt + tid;
        const bool ok = tid < A.bpt && slot < A.n_sel;
        binfo[tid] = ok ? slot : -1;
        bt[tid] = 0.0;
        bz[tid] = 0.0;
        if (ok) {
            const D4 xa = B[A.sel[slot]];
            bt[tid] = xa.t;
            bz[tid] = xa.z;
        }
    }
    if (tid == 0) {
        for (int q = 0; q < 2 * kTcStages; ++q) tc::mbar_init(&bars[q], q < kTcStages ? 8u : 1u);
        tc::mbar_init(&accf[0], 1);
        tc::mbar_init(&accf[1], 1);
        tc::mbar_init(&acce[0], 4);
        tc::mbar_init(&acce[1], 4);
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::mbar_fence_init();
    }
    if (warp == kTcWarps - 1) {
        tc::tmem_alloc(tslot, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tbase = *tslot;

    int kstart = A.n_t;
    for (int b = 0; b < A.bpt && b < 64; ++b)
        if (binfo[b] >= 0) kstart = min(kstart, A.kfirst[binfo[b]]);
    const int nkb = (A.n_t + kTcKB - 1) / kTcKB;
    const int kb0 = kstart / kTcKB;
    const bool active = kb0 < nkb;
    const long col0 = (long)tile * kTcCols;
    bool failed = false;

    if (warp < 4) {
        // ---------------- A producers ----------------
        const int r = 32 * warp + lane;
        const int wl = r >> 1, part = r & 1;
        const int wi = w0 + wl;
        const bool wok = wi < A.n_w;
        const uint32_t lanebase = (uint32_t)(32 * warp) << 16;
        float2* ptab = reinterpret_cast<float2*>(sm + SmemLayout::ptab);
        int it = 0;
        for (int i = 0; active && i < A.n_cos && !failed; ++i) {
            // M[w, k] = z_kb P_n, k = 32 kb + n: the block anchor z_kb = e^{i w' t_k}
            // advances in FP64 by e^{i w' 32 dt}; P_n = e^{i w' n dt} (FP32 table,
            // each warp fills the entries of its own 16 frequencies).
            const double om1 = 1.0 - A.cos_t[i];
            __syncwarp();
            for (int q = lane; q < 32 * 16; q += 32) {
                const int n = q >> 4, l = 16 * warp + (q & 15);
                const double oml = (w0 + l < A.n_w) ? A.w[w0 + l] * om1 : 0.0;
                double sn, cs;
                sincos(oml * (n * A.dt), &sn, &cs);
                ptab[n * kTcWT + l] = make_float2((float)cs, (float)sn);
            }
            __syncwarp();
            const double om = wok ? A.w[wi] * om1 : 0.0;
            double zr, zi, sr, si;
            sincos(om * A.t_arr[kb0 * kTcKB], &zi, &zr);
            sincos(om * (kTcKB * A.dt), &si, &sr);
            for (int kb = kb0; kb < nkb; ++kb, ++it) {
                const float ar = (float)zr, ai = (float)zi;
                const bool tail = (kb + 1) * kTcKB > A.n_t;
                const double nr = fma(zr, sr, -zi * si);
                const double ni = fma(zr, si, zi * sr);
                zr = nr;
                zi = ni;
                const int st = it % kTcStages;
                if (!tc::warp_wait_bounded(&empty[st], ((it / kTcStages) & 1) ^ 1, abort_flag)) {
                    failed = true;
                    break;
                }
                const uint32_t acol = tbase + 256 + 64 * st;
#pragma unroll
                for (int h = 0; h < 2; ++h) {  // 16 steps at a time
                    uint32_t hi[16], lo[16];
#pragma unroll
                    for (int n = 0; n < 16; ++n) {
                        const int nn = 16 * h + n;
                        const float2 p = ptab[nn * kTcWT + wl];
                        float v = part ? fmaf(ar, p.y, ai * p.x) : fmaf(ar, p.x, -ai * p.y);
                        if (tail && kb * kTcKB + nn >= A.n_t) v = 0.0f;
                        tc::split_tf32_fast(v, hi[n], lo[n]);
                    }
                    tc::tmem_st16((acol + 16 * h) | lanebase, hi);
                    tc::tmem_st16((acol + 32 + 16 * h) | lanebase, lo);
                }
                tc::tmem_wait_st();
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&full[st]);
            }
        }
    } else if (warp < 8) {
        // ---------------- B producers ----------------
        const int tb = tid - 128;
        const float* beta = A.beta;
        int it = 0;
        for (int i = 0; active && i < A.n_cos && !failed; ++i) {
            const float* brow = beta + (((size_t)frame * A.n_cos + i) * A.cols_pad + col0) * A.t_pad;
            for (int kb = kb0; kb < nkb; ++kb, ++it) {
                float4 v[8];
                const bool tail = (kb + 1) * kTcKB > A.n_t;
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int q = tb + 128 * u;
                    const int n = q >> 3, c = q & 7;
                    const int k = kb * kTcKB + 4 * c;
                    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (!tail) {
                        x = __ldg(reinterpret_cast<const float4*>(brow + (size_t)n * A.t_pad + k));
                    } else {
                        if (k < A.t_pad) x = __ldg(reinterpret_cast<const float4*>(brow + (size_t)n * A.t_pad + k));
                        if (k + 0 >= A.n_t) x.x = 0.f;
                        if (k + 1 >= A.n_t) x.y = 0.f;
                        if (k + 2 >= A.n_t) x.z = 0.f;
                        if (k + 3 >= A.n_t) x.w = 0.f;
                    }
                    v[u] = x;
                }
                const int st = it % kTcStages;
                if (!tc::warp_wait_bounded(&empty[st], ((it / kTcStages) & 1) ^ 1, abort_flag)) {
                    failed = true;
                    break;
                }
                unsigned char* bh = sm + SmemLayout::b_hi + st * kBTileBytes;
                unsigned char* bl = sm + SmemLayout::b_lo + st * kBTileBytes;
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int q = tb + 128 * u;
                    const int n = q >> 3, c = q & 7;
                    uint4 h, l;
                    tc::split_tf32_fast(v[u].x, h.x, l.x);
                    tc::split_tf32_fast(v[u].y, h.y, l.y);
                    tc::split_tf32_fast(v[u].z, h.z, l.z);
                    tc::split_tf32_fast(v[u].w, h.w, l.w);
                    const uint32_t off = swz128(n, c);
                    *reinterpret_cast<uint4*>(bh + off) = h;
                    *reinterpret_cast<uint4*>(bl + off) = l;
                }
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&full[st]);
            }
        }
    } else if (warp < 12) {
        // ---------------- epilogue ----------------
        // Tensor-core FP32 accumulation rounds each addition into a growing
        // sum, so the accumulator is handed over every kTcFoldKB blocks of 32
        // steps and its contribution, phase included (the phase is constant
        // along a row), is added to FP64 sums per (w, set, +/x).  Each lane
        // holds one GEMM row, Re (even lane) or Im (odd lane) of its
        // frequency, and accumulates sum_b cos_b Y_b and sum_b sin_b Y_b of
        // that row; Re C = sum cos Yr - sum sin Yi and Im C = sum cos Yi +
        // sum sin Yr are formed once at the end.  Products are summed in FP32
        // over the bubbles of a 32-column chunk (two interleaved chains), then
        // added to the FP64 sums.
        const int q4 = warp - 8;
        const int r = 32 * q4 + lane;
        const int wl = r >> 1, part = r & 1;
        const int wi = w0 + wl;
        const uint32_t lanebase = (uint32_t)(32 * q4) << 16;
        float2* etab = reinterpret_cast<float2*>(sm + SmemLayout::etab);
        double accC[CPB], accS[CPB];
#pragma unroll
        for (int c = 0; c < CPB; ++c) accC[c] = accS[c] = 0.0;
        int seg = 0;
        for (int i = 0; active && i < A.n_cos && !failed; ++i) {
            // e^{i w (t_a c_i - z_a)} per (w, bubble) of this row; zero for empty
            // columns (each warp fills and reads only its own 16 frequencies)
            const double ci = A.cos_t[i];
            __syncwarp();
#pragma unroll 4
            for (int q = lane; q < 64 * 16; q += 32) {
                const int b = q & 63, l = 16 * q4 + (q >> 6);
                float2 e = make_float2(0.f, 0.f);
                if (b < A.bpt && binfo[b] >= 0 && w0 + l < A.n_w) {
                    double sn, cs;
                    phase<float>(A.w[w0 + l] * (bt[b] * ci - bz[b]), sn, cs);
                    e = make_float2((float)cs, (float)sn);
                }
                etab[l * kEStride + b] = e;
            }
            __syncwarp();
            const float2* erow = etab + wl * kEStride;
            const int nseg = (nkb - kb0 + kTcFoldKB - 1) / kTcFoldKB;
            for (int g = 0; g < nseg; ++g, ++seg) {
                const int buf = seg & 1;
                if (!tc::warp_wait_bounded(&accf[buf], (seg >> 1) & 1, abort_flag)) {
                    failed = true;
                    break;
                }
                tc::tc_fence_after();
                // columns [n0, n0 + 32) from y; the chunk's phases are loaded first
                auto consume = [&](const uint32_t (&y)[32], const int n0) {
                    constexpr int NB = 32 / CPB + 2;
                    const int b_first = n0 / CPB;
                    float2 ev[NB];
#pragma unroll
                    for (int j = 0; j < NB; ++j)
                        if (b_first + j <= (n0 + 31) / CPB) ev[j] = erow[b_first + j];
                    float pc[2][CPB], ps[2][CPB];
#pragma unroll
                    for (int c = 0; c < CPB; ++c) pc[0][c] = ps[0][c] = pc[1][c] = ps[1][c] = 0.f;
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const int n = n0 + c;
                        const int b = n / CPB, sc = n % CPB, h2 = b & 1;
                        const float2 e = ev[b - b_first];
                        const float yv = __uint_as_float(y[c]);
                        pc[h2][sc] = fmaf(e.x, yv, pc[h2][sc]);
                        ps[h2][sc] = fmaf(e.y, yv, ps[h2][sc]);
                    }
#pragma unroll
                    for (int q = 0; q < CPB; ++q) {
                        accC[q] += (double)(pc[0][q] + pc[1][q]);
                        accS[q] += (double)(ps[0][q] + ps[1][q]);
                    }
                };
                const uint32_t dcol = (tbase + 128 * buf) | lanebase;
#pragma unroll
                for (int ch = 0; ch < kTcCols / 32; ++ch) {
                    uint32_t y[32];
                    tc::tmem_ld32(dcol + 32 * ch, y);
                    tc::tmem_wait_ld();
                    if (ch == kTcCols / 32 - 1) {  // every column is in registers: release the buffer
                        tc::tc_fence_before();
                        __syncwarp();
                        if (lane == 0) tc::mbar_arrive(&acce[buf]);
                    }
                    consume(y, 32 * ch);
                }
            }
        }
        // even lane: (sum cos Yr, sum sin Yr); odd lane: (sum cos Yi, sum sin Yi)
#pragma unroll
        for (int sg = 0; sg < CPB; ++sg) {
            const double oc = __shfl_xor_sync(0xffffffffu, accC[sg], 1);
            const double os = __shfl_xor_sync(0xffffffffu, accS[sg], 1);
            if (part == 0 && wi < A.n_w) {
                const int s_ = sg >> 1, g = sg & 1;
                const size_t o = ((((size_t)frame * A.tiles_per_frame + tile) * 2 + g) * S + s_) * A.n_w + wi;
                A.partial[o] = make_double2(accC[sg] - os, oc + accS[sg]);
            }
        }
    } else {
        // ---------------- MMA issue ----------------
        if (lane == 0 && active) {
            const uint32_t idesc = tc::idesc_tf32(kTcRows, kTcCols);
            int it = 0, seg = 0;
            for (int i = 0; i < A.n_cos && !failed; ++i) {
                uint32_t dcol = 0, accumulate = 0;
                for (int kb = kb0; kb < nkb; ++kb, ++it) {
                    if ((kb - kb0) % kTcFoldKB == 0) {  // a new accumulation segment
                        const int buf = seg & 1;
                        if (!tc::mbar_wait_bounded(&acce[buf], ((seg >> 1) & 1) ^ 1, abort_flag)) {
                            failed = true;
                            break;
                        }
                        tc::tc_fence_after();
                        dcol = tbase + 128 * buf;
                        accumulate = 0;
                    }
                    const int st = it % kTcStages;
                    if (!tc::mbar_wait_bounded(&full[st], (it / kTcStages) & 1, abort_flag)) {
                        failed = true;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t a_hi = tbase + 256 + 64 * st, a_lo = a_hi + 32;
                    const uint32_t b_hi = tc::smem_u32(sm + SmemLayout::b_hi + st * kBTileBytes);
                    const uint32_t b_lo = tc::smem_u32(sm + SmemLayout::b_lo + st * kBTileBytes);
#pragma unroll
                    for (int j = 0; j < kTcKB / 8; ++j) {
                        tc::mma_tf32_ts(dcol, a_hi + 8 * j, tc::sdesc_k128(b_lo + 32 * j), idesc, accumulate);
                        accumulate = 1;
                        tc::mma_tf32_ts(dcol, a_lo + 8 * j, tc::sdesc_k128(b_hi + 32 * j), idesc, 1);
                        tc::mma_tf32_ts(dcol, a_hi + 8 * j, tc::sdesc_k128(b_hi + 32 * j), idesc, 1);
                    }
                    tc::mma_commit(&empty[st]);
                    if ((kb - kb0) % kTcFoldKB == kTcFoldKB - 1 || kb == nkb - 1) {
                        tc::mma_commit(&accf[seg & 1]);
                        ++seg;
                    }
                }
            }
            // wait for every MMA issued by this thread before the memory is freed
            tc::mma_commit(drain);
            volatile int never = 0;
            if (!tc::mbar_wait_bounded(drain, 0, &never)) failed = true;
        }
    }
    if (failed) {
        *abort_flag = 1;
        atomicOr(A.err, 1u);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == kTcWarps - 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tbase, kTmemCols);
    }
}

template <int S>
void launch_s(const TcArgs& A, dim3 grid, size_t smem, cudaStream_t st) {
    CUDA_OK(cudaFuncSetAttribute(k_gemm_tc<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gemm_tc<S><<<grid, kTcThreads, smem, st>>>(A);
}

}  // namespace

void launch_gemm_tc(const TcArgs& A, size_t kn, cudaStream_t st) {
    if (A.bpt * 2 * A.S > kTcCols) throw Error{"tensor-core GEMM: too many columns per tile"};
    const size_t smem = SmemLayout::total + 1024;
    const size_t gy = kn * (size_t)A.tiles_per_frame;
    if (gy > 65535) throw Error{"too many column tiles in one k-hat chunk"};
    dim3 grid((unsigned)((A.n_w + kTcWT - 1) / kTcWT), (unsigned)gy);
    switch (A.S) {
        case 1: launch_s<1>(A, grid, smem, st); break;
        case 2: launch_s<2>(A, grid, smem, st); break;
        case 3: launch_s<3>(A, grid, smem, st); break;
        case 4: launch_s<4>(A, grid, smem, st); break;
        case 5: launch_s<5>(A, grid, smem, st); break;
        case 6: launch_s<6>(A, grid, smem, st); break;
        case 7: launch_s<7>(A, grid, smem, st); break;
        case 8: launch_s<8>(A, grid, smem, st); break;
        default: throw Error{"tensor-core GEMM supports at most 8 coefficient sets"};
    }
    CUDA_OK(cudaGetLastError());
}

}  // namespace bgw
