// Mixed-precision time-phase GEMM on the 5th-generation tensor cores, as an
// exact integer product of digit slices.
//
// For each cos-theta row i the factored spectrum needs Y_i = M_i beta_i with
// M_i[w, k] = e^{i w (1 - c_i) t_k} (rows: Re and Im of 64 frequencies) and
// beta_i[k, col] (columns: bubble x set x {+, x}); the epilogue applies
// e^{i w (t_a c_i - z_a)} per (w, bubble) and sums over the tile's bubbles
// (spectrum_factored.cu holds the derivation).
//
// Both operands are written as four signed 8-bit digits in balanced base 256
// (spectrum_tc.cuh): M F = sum_p m_p 256^(3-p) and beta F = s_a sum_q b_q
// 256^(3-q) with F = 0x7F7F7F7F, one scale s_a per (frame, bubble, row) =
// max |beta| over the row's steps and columns.  The product keeps the ten
// digit pairs (p, q) with p + q <= 3 (p = 0 the most significant digit); the
// pairs of one level L = p + q share the weight 256^-L, so
//   Y = s_a 256^6 / F^2  sum_L 256^-L D_L,   D_L = sum_k sum_{p+q=L} m_p b_q,
// and each D_L is accumulated EXACTLY by tcgen05.mma kind::i8 in a 32-bit
// integer accumulator of tensor memory (|D_L| <= 4 * 128^2 * n_t < 2^31 for
// n_t <= 32767).  The error is the digit truncation, about 2^-32 of the
// operands' scales per term, against 2^-24 for FP32 operands; there is no
// rounding in the accumulation at all, so the accumulators run over a whole
// row of time steps and are read once per row.
//
// Both operands arrive pre-split and pre-swizzled from HBM: the time phases
// from a per-call table (k_tc_phase_table, FP64 sincos, frame and bubble
// independent), beta from k_beta, as sets of four 4 KB digit blocks of 128
// rows x 32 steps.  One thread streams each 32-step stage (A digits, B digits:
// 32 KB) into shared memory with two bulk copies that complete on the stage's
// mbarrier (transaction bytes); one thread issues the ten MMAs per stage.
//
// One CTA per (64-frequency tile, 128-column tile, range of cos-theta rows);
// per row the K dimension is the time steps from the tile's first active block
// of 32 steps on.  Warp roles (10 warps):
//   0     bulk-copy producer (one thread)
//   1     MMA issue (one thread) and tensor-memory allocation
//   2-9   epilogue, two warpgroups of 64 columns each: thread = tensor-memory
//         lane.  While a row's MMAs run, each warp fills its part of the FP64
//         table s_a 256^6/F^2 e^{i w (t_a c_i - z_a)} (64 w x 64 bubbles, shared
//         memory); when the row's accumulators are complete it reads the four
//         levels (tcgen05.ld), combines them (level 0 in FP64, levels 1-3 in
//         FP32, whose rounding lies below the truncation) and adds
//         phase x value to FP64 sums per (w, set, +/x).
// Stages: 4 x 32 KB.  Tensor memory: 512 columns, level L at columns 128 L.
// Every wait is bounded: on a timeout the block records an error flag, tells
// the other roles to stop, waits for its issued MMAs and copies to finish and
// frees its tensor memory.

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
constexpr int kTcKB = 32;        // time steps per stage (32 bytes of int8)
constexpr int kTcWarps = 10;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr uint32_t kTmemCols = 512;
constexpr int kStageBytes = 2 * kI8BlockSet;  // A digits, B digits

// Shared memory of a GEMM CTA with ST pipeline stages (3 to 5 fit next to the phase table).
template <int ST>
struct SmemLayout {
    static constexpr int stages = 0;
    static constexpr int etab = ST * kStageBytes;              // double2[64 w][64 bubbles], XOR-swizzled
    static constexpr int bars = etab + 64 * 64 * 16;          // full[ST], empty[ST], accf, acce, drain
    static constexpr int n_bars = 2 * ST + 3;
    static constexpr int tslot = bars + 8 * n_bars;
    static constexpr int abort_flag = tslot + 4;
    static constexpr int binfo = tslot + 16;                   // int[64]
    static constexpr int bt = binfo + 64 * 4;                  // double[64]
    static constexpr int bz = bt + 64 * 8;                     // double[64]
    static constexpr int total = bz + 64 * 8;
};
static_assert(SmemLayout<5>::total + 1024 <= 227 * 1024, "shared memory budget");

// Phase-table slot of (frequency l, bubble b): rows of 64 bubbles, the bubble
// index XORed with l % 8 so that the 16 frequencies read by a warp fall in
// distinct 16-byte bank groups (two wavefronts for 16 x 16 bytes).
__device__ __forceinline__ int eslot(int l, int b) { return l * 64 + (b ^ (l & 7)); }

// Shared-memory descriptor of a K-major, 32-byte-swizzled digit block (256-byte
// aligned): bits [0,14) address >> 4, [16,30) leading byte offset >> 4 (unused
// for this layout, 1), [32,46) stride byte offset >> 4 (256 bytes between
// 8-row groups), [46,48) version 1, [61,64) layout 6 = 32-byte swizzle.
__device__ __forceinline__ uint64_t sdesc_sw32(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}

// Instruction descriptor of kind::i8: S32 accumulator (bits [4,6) = 2), A and
// B signed 8-bit (bits [7,10) and [10,13) = 1), K-major, dense, N >> 3 at
// [17,23), M >> 4 at [24,29).
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T in 32-bit integers; issued by one thread.
__device__ __forceinline__ void mma_i8_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// 16 consecutive 32-bit columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__global__ void k_tc_phase_table(const double* __restrict__ w, const double* __restrict__ cos_t,
                                 const double* __restrict__ t_arr, int n_cos, int n_w, int n_t, int n_wt, int nkb,
                                 int8_t* __restrict__ atab) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n_el = (size_t)n_cos * n_wt * nkb * kI8Block;
    if (q >= n_el) return;
    const int e = (int)(q % kI8Block);
    const size_t blk = q / kI8Block;  // (i, wt, kb)
    const int kb = (int)(blk % nkb);
    const int wt = (int)((blk / nkb) % n_wt);
    const int i = (int)(blk / ((size_t)nkb * n_wt));
    const int r = e >> 5, kk = e & 31;
    const int wi = wt * kTcWT + (r >> 1), k = kb * kTcKB + kk;
    double v = 0.0;
    if (wi < n_w && k < n_t) {
        double sn, cs;
        sincos(w[wi] * ((1.0 - cos_t[i]) * t_arr[k]), &sn, &cs);
        v = (r & 1) ? sn : cs;
    }
    const uint32_t d = i8_digits(v);
    int8_t* out = atab + blk * kI8BlockSet + i8_swz(r, kk);
#pragma unroll
    for (int s = 0; s < kI8Slices; ++s) out[(size_t)s * kI8Block] = (int8_t)(d >> (8 * s));
}

template <int S, int ST>
__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_i8(TcArgs A) {
    constexpr int kTcStages = ST;
    using SmemLayout = bgw::SmemLayout<ST>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                         ~static_cast<uintptr_t>(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + SmemLayout::bars);
    uint64_t* full = bars;
    uint64_t* empty = bars + kTcStages;
    uint64_t* accf = bars + 2 * kTcStages;
    uint64_t* acce = accf + 1;
    uint64_t* drain = acce + 1;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SmemLayout::tslot);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + SmemLayout::abort_flag);
    int* binfo = reinterpret_cast<int*>(sm + SmemLayout::binfo);
    double* bt = reinterpret_cast<double*>(sm + SmemLayout::bt);
    double* bz = reinterpret_cast<double*>(sm + SmemLayout::bz);

    constexpr int CPB = 2 * S;  // columns per bubble
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wt = blockIdx.x;
    const int w0 = wt * kTcWT;
    // blockIdx.y = (frame, part, tile), tile fastest: part p takes the rows [i0, i1).  CTAs
    // resident together then share the time-phase digits of their rows (one part, many
    // column tiles) and each column tile's beta (its frequency tiles) in L2.
    const int tile = blockIdx.y % A.tiles_per_frame;
    const int part_ = (blockIdx.y / A.tiles_per_frame) % A.row_parts;
    const int frame = blockIdx.y / A.tiles_per_frame / A.row_parts;
    const int i0 = A.n_cos * part_ / A.row_parts, i1 = A.n_cos * (part_ + 1) / A.row_parts;
    const D4* B = A.bub + (size_t)frame * A.n_tot;

    if (tid < 64) {
        const int slot = tile * A.bpt + tid;
        const bool ok = tid < A.bpt && slot < A.n_sel && A.sel[slot] != kNoSlot;
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
        tc::mbar_init(accf, 1);  // the MMA thread's commit after a row's last stage
        tc::mbar_init(acce, 8);  // every epilogue warp, once it holds the row's accumulators
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
                const int8_t* arow = A.atab + ((size_t)(i * A.n_wt + wt) * nkb) * kI8BlockSet;
                const int8_t* brow =
                    A.btab + ((((size_t)frame * A.n_cos + i) * A.tiles_per_frame + tile) * nkb) * kI8BlockSet;
                for (int kb = kb0; kb < nkb; ++kb, ++it) {
                    const int st = it % kTcStages;
                    if (!tc::mbar_wait_bounded_poll(&empty[st], ((it / kTcStages) & 1) ^ 1, abort_flag)) {
                        failed = true;
                        break;
                    }
                    unsigned char* dst = sm + SmemLayout::stages + st * kStageBytes;
                    tc::mbar_arrive_expect_tx(&full[st], kStageBytes);
                    tc::bulk_g2s(dst, arow + (size_t)kb * kI8BlockSet, kI8BlockSet, &full[st]);
                    tc::bulk_g2s(dst + kI8BlockSet, brow + (size_t)kb * kI8BlockSet, kI8BlockSet, &full[st]);
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
            const uint32_t idesc = idesc_i8(kTcRows, kTcCols);
            int it = 0, row = 0;
            for (int i = i0; i < i1 && !failed; ++i, ++row) {
                // the epilogue has read the previous row's accumulators
                if (!tc::mbar_wait_bounded_poll(acce, (row & 1) ^ 1, abort_flag)) {
                    failed = true;
                    break;
                }
                tc::tc_fence_after();
                for (int kb = kb0; kb < nkb; ++kb, ++it) {
                    const int st = it % kTcStages;
                    if (!tc::mbar_wait_bounded_poll(&full[st], (it / kTcStages) & 1, abort_flag)) {
                        failed = true;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t base = tc::smem_u32(sm + SmemLayout::stages + st * kStageBytes);
                    // the ten digit pairs (p, q), p + q <= 3, into level p + q; the first
                    // pair of each level in the row's first block starts that level's sum
                    const uint32_t acc = kb == kb0 ? 0u : 1u;
                    auto mma = [&](int p, int q, uint32_t a) {
                        mma_i8_ss(tbase + 128 * (p + q), sdesc_sw32(base + p * kI8Block),
                                  sdesc_sw32(base + kI8BlockSet + q * kI8Block), idesc, a);
                    };
                    mma(0, 0, acc);
                    mma(0, 1, acc);
                    mma(1, 0, 1u);
                    mma(0, 2, acc);
                    mma(1, 1, 1u);
                    mma(2, 0, 1u);
                    mma(0, 3, acc);
                    mma(1, 2, 1u);
                    mma(2, 1, 1u);
                    mma(3, 0, 1u);
                    tc::mma_commit(&empty[st]);
                }
                if (failed) break;
                tc::mma_commit(accf);
            }
            // wait for every MMA issued by this thread before the memory is freed
            tc::mma_commit(drain);
            volatile int never = 0;
            if (!tc::mbar_wait_bounded_poll(drain, 0, &never)) failed = true;
        }
    } else {
        // ---------------- epilogue ----------------
        // Each lane holds one GEMM row, Re (even lane) or Im (odd lane) of its
        // frequency, and accumulates sum_b cos_b Y_b and sum_b sin_b Y_b of that
        // row in FP64; Re C = sum cos Yr - sum sin Yi and Im C = sum cos Yi +
        // sum sin Yr are formed once at the end.
        const int q4 = warp & 3;             // tensor-memory lane quadrant of this warp
        const int half = (warp - 2) >> 2;    // which 64 columns
        const int r = 32 * q4 + lane;
        const int wl = r >> 1, part = r & 1;
        const int wi = w0 + wl;
        const uint32_t lanebase = (uint32_t)(32 * q4) << 16;
        double2* etab = reinterpret_cast<double2*>(sm + SmemLayout::etab);
        double accC[CPB], accS[CPB];
#pragma unroll
        for (int c = 0; c < CPB; ++c) accC[c] = accS[c] = 0.0;
        constexpr float kInv256 = 1.0f / 256.0f;
        // the column offset is a compile-time constant in each instance, so that
        // every per-column index below is too (no dynamically indexed arrays)
        auto run = [&](auto half_c) {
            constexpr int c_lo = decltype(half_c)::value * (kTcCols / 2);
            constexpr int b_lo = c_lo / CPB, b_hi = (c_lo + kTcCols / 2 - 1) / CPB;
            constexpr int nb = b_hi - b_lo + 1;
            int row = 0;
            for (int i = i0; active && i < i1 && !failed; ++i, ++row) {
                // s_a 256^6 / F^2 e^{i w (t_a c_i - z_a)} per (w, bubble) of this row; zero for
                // empty columns.  Each warp fills the entries it reads (its 16
                // frequencies, its bubbles) while the row's MMAs run.
                const double ci = A.cos_t[i];
                __syncwarp();
                for (int q = lane; q < 16 * nb; q += 32) {
                    const int b = b_lo + q % nb, l = 16 * q4 + q / nb;
                    double2 e = make_double2(0.0, 0.0);
                    if (b < A.bpt && binfo[b] >= 0 && w0 + l < A.n_w) {
                        const double sc =
                            A.bscale[((size_t)frame * A.n_sel + binfo[b]) * A.n_cos + i] * kI8PairScale;
                        double sn, cs;
                        sincos(A.w[w0 + l] * (bt[b] * ci - bz[b]), &sn, &cs);
                        e = make_double2(sc * cs, sc * sn);
                    }
                    etab[eslot(l, b)] = e;
                }
                __syncwarp();
                if (!tc::warp_wait_bounded(accf, row & 1, abort_flag)) {
                    failed = true;
                    break;
                }
                tc::tc_fence_after();
                // columns [n0, n0 + 16): the four levels' integer sums combined
                auto consume = [&](const uint32_t (&d0)[16], const uint32_t (&d1)[16], const uint32_t (&d2)[16],
                                   const uint32_t (&d3)[16], auto n0_c) {
                    constexpr int n0 = decltype(n0_c)::value;
#pragma unroll
                    for (int c = 0; c < 16; ++c) {
                        const int n = n0 + c;
                        const int b = n / CPB, sc = n % CPB;
                        const float lo = fmaf(fmaf(fmaf((float)(int)d3[c], kInv256, (float)(int)d2[c]), kInv256,
                                                   (float)(int)d1[c]),
                                              kInv256, 0.0f);
                        const double y = (double)(int)d0[c] + (double)lo;
                        const double2 e = etab[eslot(wl, b)];
                        accC[sc] = fma(e.x, y, accC[sc]);
                        accS[sc] = fma(e.y, y, accS[sc]);
                    }
                };
                auto chunk = [&](auto n0_c, bool last) {
                    constexpr int n0 = decltype(n0_c)::value;
                    const uint32_t col = (tbase + n0) | lanebase;
                    uint32_t d0[16], d1[16], d2[16], d3[16];
                    tc::tc_fence_after();
                    tmem_ld16(col, d0);
                    tmem_ld16(col + 128, d1);
                    tmem_ld16(col + 256, d2);
                    tmem_ld16(col + 384, d3);
                    tc::tmem_wait_ld();
                    if (last) {
                        // this warp's columns of the row are in registers
                        tc::tc_fence_before();
                        __syncwarp();
                        if (lane == 0) tc::mbar_arrive(acce);
                    }
                    consume(d0, d1, d2, d3, n0_c);
                };
                chunk(std::integral_constant<int, c_lo>{}, false);
                chunk(std::integral_constant<int, c_lo + 16>{}, false);
                chunk(std::integral_constant<int, c_lo + 32>{}, false);
                chunk(std::integral_constant<int, c_lo + 48>{}, true);
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

template <int S, int ST>
void launch_st(const TcArgs& A, dim3 grid, cudaStream_t st) {
    const size_t smem = SmemLayout<ST>::total + 1024;
    CUDA_OK(cudaFuncSetAttribute(k_gemm_i8<S, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gemm_i8<S, ST><<<grid, kTcThreads, smem, st>>>(A);
}

template <int S>
void launch_s(const TcArgs& A, dim3 grid, cudaStream_t st) {
    switch (A.stages) {
        case 3: launch_st<S, 3>(A, grid, st); break;
        case 5: launch_st<S, 5>(A, grid, st); break;
        default: launch_st<S, 4>(A, grid, st); break;
    }
}

}  // namespace

void launch_tc_phase_table(const double* w, const double* cos_t, const double* t_arr, int n_cos, int n_w, int n_t,
                           int8_t* atab, cudaStream_t st) {
    const int n_wt = (n_w + kTcWT - 1) / kTcWT, nkb = (n_t + kTcKB - 1) / kTcKB;
    const size_t n_el = (size_t)n_cos * n_wt * nkb * kI8Block;
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
    if (A.n_t > kI8MaxSteps) throw Error{"the mixed kernel accumulates at most 32767 time steps exactly; use fp64_factored"};
    if (A.stages != 0 && (A.stages < 3 || A.stages > 5)) throw Error{"tensor-core GEMM: 3 to 5 pipeline stages"};
    const size_t gy = kn * (size_t)A.tiles_per_frame * A.row_parts;
    if (gy > 65535) throw Error{"too many column tiles in one k-hat chunk"};
    dim3 grid((unsigned)A.n_wt, (unsigned)gy);
    switch (A.S) {
        case 1: launch_s<1>(A, grid, st); break;
        case 2: launch_s<2>(A, grid, st); break;
        case 3: launch_s<3>(A, grid, st); break;
        case 4: launch_s<4>(A, grid, st); break;
        case 5: launch_s<5>(A, grid, st); break;
        case 6: launch_s<6>(A, grid, st); break;
        case 7: launch_s<7>(A, grid, st); break;
        case 8: launch_s<8>(A, grid, st); break;
        default: throw Error{"tensor-core GEMM supports at most 8 coefficient sets"};
    }
    CUDA_OK(cudaGetLastError());
}

}  // namespace bgw
