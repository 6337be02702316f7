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
// Both operands arrive pre-split and pre-swizzled from HBM: the time phases
// from a per-call table (k_tc_phase_table, frame and bubble independent), beta
// from k_beta, in 16 KB blocks of 128 rows x 32 steps.  One thread streams the
// blocks of a 32-step stage into shared memory with bulk copies that complete
// on the stage's mbarrier (transaction bytes); one thread issues the MMAs with
// both operands in shared memory.
//
// One CTA per (64-frequency tile, 128-column tile), looping over the rows i;
// per row the K dimension is the time steps from the tile's first active
// block of 32 steps on.  Warp roles (10 warps):
//   0     bulk-copy producer (one thread)
//   1     MMA issue (one thread) and tensor-memory allocation
//   2-9   epilogue, two warpgroups of 64 columns each: thread = tensor-memory
//         lane.  Per row the phases e^{i w (t_a c_i - z_a)} (FP64 argument
//         reduction, FP32 sincos) go to a shared-memory table; every block of
//         32 steps the accumulator (tcgen05.ld) is multiplied by them and
//         summed per (w, set, +/x) in FP64.
// Stages: 3 x 64 KB (A hi/lo, B hi/lo); the FP32 accumulator is double-
// buffered in tensor memory across blocks of 32 steps.  Every wait is bounded:
// on a timeout the block records an error flag, tells the other roles to stop,
// waits for its issued MMAs and copies to finish and frees its tensor memory.
//
// Tensor memory: 256 columns, accumulators at columns 0 and 128.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <type_traits>

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
constexpr int kTcStages = 3;
constexpr int kTcFoldKB = 1;     // blocks of 32 steps accumulated in tensor memory before the FP64 fold
constexpr int kTcWarps = 10;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr uint32_t kTmemCols = 256;
constexpr int kBlockBytes = kTcBlockFloats * 4;   // 16 KB
constexpr int kStageBytes = 4 * kBlockBytes;      // A hi, A lo, B hi, B lo

struct SmemLayout {
    static constexpr int stages = 0;
    static constexpr int bars = kTcStages * kStageBytes;      // full[S], empty[S], accf[2], acce[2], drain
    static constexpr int n_bars = 2 * kTcStages + 5;
    static constexpr int tslot = bars + 8 * n_bars;
    static constexpr int abort_flag = tslot + 4;
    static constexpr int binfo = tslot + 16;                   // int[64]
    static constexpr int bt = binfo + 64 * 4;                  // double[64]
    static constexpr int bz = bt + 64 * 8;                     // double[64]
    static constexpr int etab = bz + 64 * 8;                   // float2[64 w][64 bubbles], XOR-swizzled
    static constexpr int total = etab + 64 * 64 * 8;
};

// Phase-table slot of (frequency l, bubble b): rows of 64 bubbles, the bubble
// index XORed with l % 16 so that the 16 frequencies read by a warp fall in
// distinct banks.
__device__ __forceinline__ int eslot(int l, int b) { return l * 64 + (b ^ (l & 15)); }

__global__ void k_tc_phase_table(const double* __restrict__ w, const double* __restrict__ cos_t,
                                 const double* __restrict__ t_arr, int n_cos, int n_w, int n_t, int n_wt, int nkb,
                                 float* __restrict__ atab) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n_el = (size_t)n_cos * n_wt * nkb * kTcBlockFloats;
    if (q >= n_el) return;
    const int e = (int)(q % kTcBlockFloats);
    const size_t blk = q / kTcBlockFloats;  // (i, wt, kb)
    const int kb = (int)(blk % nkb);
    const int wt = (int)((blk / nkb) % n_wt);
    const int i = (int)(blk / ((size_t)nkb * n_wt));
    const int r = e >> 5, kk = e & 31;
    const int wi = wt * kTcWT + (r >> 1), k = kb * kTcKB + kk;
    float v = 0.0f;
    if (wi < n_w && k < n_t) {
        double sn, cs;
        sincos(w[wi] * ((1.0 - cos_t[i]) * t_arr[k]), &sn, &cs);
        v = (float)((r & 1) ? sn : cs);
    }
    uint32_t hi, lo;
    tc::split_tf32_fast(v, hi, lo);
    float* out = atab + blk * 2 * kTcBlockFloats;
    const size_t o = tc_swz(r, kk);
    out[o] = __uint_as_float(hi);
    out[kTcBlockFloats + o] = __uint_as_float(lo);
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
    const int wt = blockIdx.x;
    const int w0 = wt * kTcWT;
    // blockIdx.y = (frame, tile, part): part p takes the rows [i0, i1)
    const int part_ = blockIdx.y % A.row_parts;
    const int frame = blockIdx.y / A.row_parts / A.tiles_per_frame;
    const int tile = (blockIdx.y / A.row_parts) % A.tiles_per_frame;
    const int i0 = A.n_cos * part_ / A.row_parts, i1 = A.n_cos * (part_ + 1) / A.row_parts;
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
        for (int q = 0; q < kTcStages; ++q) {
            tc::mbar_init(&full[q], 1);   // the producer's arrive; the copies' bytes complete the phase
            tc::mbar_init(&empty[q], 1);  // the MMA thread's commit
        }
        tc::mbar_init(&accf[0], 1);
        tc::mbar_init(&accf[1], 1);
        tc::mbar_init(&acce[0], 8);
        tc::mbar_init(&acce[1], 8);
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::mbar_fence_init();
    }
    if (warp == 1) {
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
    const int nkb = A.nkb;
    const int kb0 = kstart / kTcKB;
    const bool active = kb0 < nkb;
    bool failed = false;

    if (warp == 0) {
        // ---------------- bulk-copy producer ----------------
        if (lane == 0 && active) {
            int it = 0;
            for (int i = i0; i < i1 && !failed; ++i) {
                const float* arow = A.atab + ((size_t)(i * A.n_wt + wt) * nkb) * 2 * kTcBlockFloats;
                const float* brow =
                    A.btab + ((((size_t)frame * A.n_cos + i) * A.tiles_per_frame + tile) * nkb) * 2 * kTcBlockFloats;
                for (int kb = kb0; kb < nkb; ++kb, ++it) {
                    const int st = it % kTcStages;
                    if (!tc::mbar_wait_bounded_poll(&empty[st], ((it / kTcStages) & 1) ^ 1, abort_flag)) {
                        failed = true;
                        break;
                    }
                    unsigned char* dst = sm + SmemLayout::stages + st * kStageBytes;
                    tc::mbar_arrive_expect_tx(&full[st], kStageBytes);
                    tc::bulk_g2s(dst, arow + (size_t)kb * 2 * kTcBlockFloats, 2 * kBlockBytes, &full[st]);
                    tc::bulk_g2s(dst + 2 * kBlockBytes, brow + (size_t)kb * 2 * kTcBlockFloats, 2 * kBlockBytes,
                                 &full[st]);
                }
            }
            // before the block ends, the copies this thread issued must have landed:
            // wait (bounded) for the last phase of every stage it filled
            const int n_it = it;
            for (int q = 0; q < kTcStages && q < n_it; ++q) {
                const int last = n_it - 1 - q;  // the last kTcStages iterations cover each used stage once
                volatile int never = 0;
                if (!tc::mbar_wait_bounded_poll(&full[last % kTcStages], (last / kTcStages) & 1, &never)) failed = true;
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issue ----------------
        if (lane == 0 && active) {
            const uint32_t idesc = tc::idesc_tf32(kTcRows, kTcCols);
            int it = 0, seg = 0;
            for (int i = i0; i < i1 && !failed; ++i) {
                uint32_t dcol = 0, accumulate = 0;
                for (int kb = kb0; kb < nkb; ++kb, ++it) {
                    if ((kb - kb0) % kTcFoldKB == 0) {  // a new accumulation segment
                        const int buf = seg & 1;
                        if (!tc::mbar_wait_bounded_poll(&acce[buf], ((seg >> 1) & 1) ^ 1, abort_flag)) {
                            failed = true;
                            break;
                        }
                        tc::tc_fence_after();
                        dcol = tbase + 128 * buf;
                        accumulate = 0;
                    }
                    const int st = it % kTcStages;
                    if (!tc::mbar_wait_bounded_poll(&full[st], (it / kTcStages) & 1, abort_flag)) {
                        failed = true;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t base = tc::smem_u32(sm + SmemLayout::stages + st * kStageBytes);
                    const uint32_t a_hi = base, a_lo = base + kBlockBytes;
                    const uint32_t b_hi = base + 2 * kBlockBytes, b_lo = base + 3 * kBlockBytes;
#pragma unroll
                    for (int j = 0; j < kTcKB / 8; ++j) {
                        tc::mma_tf32_ss(dcol, tc::sdesc_k128(a_hi + 32 * j), tc::sdesc_k128(b_lo + 32 * j), idesc,
                                        accumulate);
                        accumulate = 1;
                        tc::mma_tf32_ss(dcol, tc::sdesc_k128(a_lo + 32 * j), tc::sdesc_k128(b_hi + 32 * j), idesc, 1);
                        tc::mma_tf32_ss(dcol, tc::sdesc_k128(a_hi + 32 * j), tc::sdesc_k128(b_hi + 32 * j), idesc, 1);
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
            if (!tc::mbar_wait_bounded_poll(drain, 0, &never)) failed = true;
        }
    } else {
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
        const int q4 = warp & 3;             // tensor-memory lane quadrant of this warp
        const int half = (warp - 2) >> 2;    // which 64 columns
        const int r = 32 * q4 + lane;
        const int wl = r >> 1, part = r & 1;
        const int wi = w0 + wl;
        const uint32_t lanebase = (uint32_t)(32 * q4) << 16;
        float2* etab = reinterpret_cast<float2*>(sm + SmemLayout::etab);
        double accC[CPB], accS[CPB];
#pragma unroll
        for (int c = 0; c < CPB; ++c) accC[c] = accS[c] = 0.0;
        // the column offset is a compile-time constant in each instance, so that
        // every per-column index below is too (no dynamically indexed arrays)
        auto run = [&](auto half_c) {
            constexpr int c_lo = decltype(half_c)::value * (kTcCols / 2);
            constexpr int b_lo = c_lo / CPB, b_hi = (c_lo + kTcCols / 2 - 1) / CPB;
            constexpr int nb = b_hi - b_lo + 1;
            int seg = 0;
            for (int i = i0; active && i < i1 && !failed; ++i) {
                // e^{i w (t_a c_i - z_a)} per (w, bubble) of this row; zero for empty columns.
                // Each warp fills the entries it reads (its 16 frequencies, its bubbles).
                const double ci = A.cos_t[i];
                __syncwarp();
#pragma unroll 4
                for (int q = lane; q < 16 * nb; q += 32) {
                    const int b = b_lo + q % nb, l = 16 * q4 + q / nb;
                    float2 e = make_float2(0.f, 0.f);
                    if (b < A.bpt && binfo[b] >= 0 && w0 + l < A.n_w) {
                        double sn, cs;
                        phase<float>(A.w[w0 + l] * (bt[b] * ci - bz[b]), sn, cs);
                        e = make_float2((float)cs, (float)sn);
                    }
                    etab[eslot(l, b)] = e;
                }
                __syncwarp();
                // this lane's phases for the whole row stay in registers
                float2 evr[nb];
#pragma unroll
                for (int j = 0; j < nb; ++j) evr[j] = etab[eslot(wl, b_lo + j)];
                const int nseg = (nkb - kb0 + kTcFoldKB - 1) / kTcFoldKB;
                for (int g = 0; g < nseg; ++g, ++seg) {
                    const int buf = seg & 1;
                    if (!tc::warp_wait_bounded(&accf[buf], (seg >> 1) & 1, abort_flag)) {
                        failed = true;
                        break;
                    }
                    tc::tc_fence_after();
                    // columns [n0, n0 + 32) from y; the chunk's phases are loaded first
                    auto consume = [&](const uint32_t (&y)[32], auto n0_c) {
                        constexpr int n0 = decltype(n0_c)::value;
                        float pc[2][CPB], ps[2][CPB];
#pragma unroll
                        for (int c = 0; c < CPB; ++c) pc[0][c] = ps[0][c] = pc[1][c] = ps[1][c] = 0.f;
#pragma unroll
                        for (int c = 0; c < 32; ++c) {
                            const int n = n0 + c;
                            const int b = n / CPB, sc = n % CPB, h2 = b & 1;
                            const float2 e = evr[b - b_lo];
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
                    const uint32_t dcol = (tbase + 128 * buf + c_lo) | lanebase;
                    uint32_t y0[32], y1[32];
                    tc::tmem_ld32(dcol, y0);
                    tc::tmem_ld32(dcol + 32, y1);
                    tc::tmem_wait_ld();
                    tc::tc_fence_before();
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&acce[buf]);  // this warp's columns are in registers
                    consume(y0, std::integral_constant<int, c_lo>{});
                    consume(y1, std::integral_constant<int, c_lo + 32>{});
                }
            }
        };
        if (half == 0)
            run(std::integral_constant<int, 0>{});
        else
            run(std::integral_constant<int, 1>{});
        // The second warpgroup hands its sums to the first through the stage
        // area: once the last accumulator is ready every MMA and copy has
        // completed, so no stage is in use any more.
        double* xch = reinterpret_cast<double*>(sm + SmemLayout::stages);
        if (half == 1) {
#pragma unroll
            for (int sg = 0; sg < CPB; ++sg) {
                xch[(2 * sg) * kTcRows + r] = accC[sg];
                xch[(2 * sg + 1) * kTcRows + r] = accS[sg];
            }
        }
        asm volatile("bar.sync 1, 256;" ::: "memory");  // the eight epilogue warps only
        if (half == 0) {
            // even lane: (sum cos Yr, sum sin Yr); odd lane: (sum cos Yi, sum sin Yi)
#pragma unroll
            for (int sg = 0; sg < CPB; ++sg) {
                const double ac = accC[sg] + xch[(2 * sg) * kTcRows + r];
                const double as = accS[sg] + xch[(2 * sg + 1) * kTcRows + r];
                const double oc = __shfl_xor_sync(0xffffffffu, ac, 1);
                const double os = __shfl_xor_sync(0xffffffffu, as, 1);
                if (part == 0 && wi < A.n_w) {
                    const int s_ = sg >> 1, g = sg & 1;
                    const size_t o = (((((size_t)frame * A.tiles_per_frame + tile) * A.row_parts + part_) * 2 + g) * S +
                                       s_) * A.n_w + wi;
                    A.partial[o] = make_double2(ac - os, oc + as);
                }
            }
        }
    }
    if (failed) {
        *abort_flag = 1;
        atomicOr(A.err, 1u);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
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

void launch_tc_phase_table(const double* w, const double* cos_t, const double* t_arr, int n_cos, int n_w, int n_t,
                           float* atab, cudaStream_t st) {
    const int n_wt = (n_w + kTcWT - 1) / kTcWT, nkb = (n_t + kTcKB - 1) / kTcKB;
    const size_t n_el = (size_t)n_cos * n_wt * nkb * kTcBlockFloats;
    if (n_el / 256 + 1 > 0x7fffffffULL) throw Error{"time-phase table too large"};
    k_tc_phase_table<<<(unsigned)((n_el + 255) / 256), 256, 0, st>>>(w, cos_t, t_arr, n_cos, n_w, n_t, n_wt, nkb,
                                                                     atab);
    CUDA_OK(cudaGetLastError());
}

int tc_row_parts(size_t n_ctas, int n_cos, int n_sm) {
    int best = 1;
    double best_eff = 0.0;
    const int max_parts = std::max(1, std::min(16, n_cos / 8));
    for (int p = 1; p <= max_parts; ++p) {
        const double c = (double)n_ctas * p;
        const double waves = std::ceil(c / n_sm);
        const double eff = c / (waves * n_sm);
        if (eff > best_eff + 0.01) {
            best_eff = eff;
            best = p;
        }
    }
    return best;
}

void launch_gemm_tc(const TcArgs& A, size_t kn, cudaStream_t st) {
    if (A.bpt * 2 * A.S > kTcCols) throw Error{"tensor-core GEMM: too many columns per tile"};
    if (A.row_parts < 1 || A.row_parts > A.n_cos) throw Error{"tensor-core GEMM: bad row split"};
    const size_t smem = SmemLayout::total + 1024;
    const size_t gy = kn * (size_t)A.tiles_per_frame * A.row_parts;
    if (gy > 65535) throw Error{"too many column tiles in one k-hat chunk"};
    dim3 grid((unsigned)A.n_wt, (unsigned)gy);
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
