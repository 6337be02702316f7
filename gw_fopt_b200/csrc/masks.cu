// First-collider search with per-bubble candidate lists (exact).
//
// For interior bubble a and a collider c with Delta = x_c - x_a (t, x, y, z),
// the collision delay along any direction x-hat = (1, n) is
//   tau_c(n) = s_c / (2 d_c),  s_c = -dt^2 + |dx|^2,  d_c = -dt + dx.n,
// and because d_c <= D_c = |dx| - dt and s_c = D_c (|dx| + dt),
//   tau_c(n) >= key_c = (|dx| + dt) / 2        for every n with d_c > 0.
// k_neighbors builds, once per radiating bubble (frame independent, the keys
// are rotation invariant), the list of the colliders with the smallest keys
// (radix select on the float keys, then a bitonic sort by (key, index)),
// kmax = a lower bound of every key outside the list, and
//   rho1 = max_c (dt^2 + |dx|^2) / D_c,  rho2 = max_c (|dt| + |dx|) / D_c.
//
// k_masks_list then decides each direction exactly as the reference
// (generalized_bulk_flow.rs:127-206, 1003-1018) does -- the unique b passing
// check(b, c) against every c, or None -- but evaluates only what can matter:
//   1. argmin m of tau over the list in key order, stopping once
//      key > tau_best (1 + 1e-12): no later collider can have a smaller tau;
//   2. check(m, c) for the listed c with key_c <= theta_m, where
//        theta_m = tau_m (1 + 1e-12) + 64 u (A_m rho1 + Q_m rho2) / d_m
//      (u = 2^-53).  The rounding error of the reference's check expression is
//      below 20 u (A_m Q_c + A_c Q_m) while its exact value is at least
//      2 d_m D_c (key_c - tau_m), so every c with key_c > theta_m passes in
//      floating point as well and needs no evaluation;
//   3. if m fails, the passer (if any) is one of the c that m failed against
//      (r(c, m) = -r(m, c) exactly in IEEE arithmetic); each is verified the
//      same way.
// Whenever a bound reaches past the list (or the list has no candidate and is
// not complete) the direction falls back to the exhaustive scan over all
// colliders.  Colliders with a near-lightlike interval (D_c tiny) are kept in
// a small always-checked set; too many of them make the bubble use the
// exhaustive scan for every direction.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "bgw_internal.h"
#include "device_common.cuh"
#include "masks.cuh"

namespace bgw {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ bool check_pt(const D4& dba, double nb, const D4& dca, const D4& x) {
    const double nc = mdot(dca, dca);
    D4 cv;
    cv.t = dsub(dmul(dba.t, nc), dmul(dca.t, nb));
    cv.x = dsub(dmul(dba.x, nc), dmul(dca.x, nb));
    cv.y = dsub(dmul(dba.y, nc), dmul(dca.y, nb));
    cv.z = dsub(dmul(dba.z, nc), dmul(dca.z, nb));
    return mdot(cv, x) > 0.0;
}

// check(b, c) with both Minkowski norms precomputed (same values as check_pt).
__device__ __forceinline__ bool check_pre(const D4& dba, double nb, const D4& dca, double nc, const D4& x) {
    D4 cv;
    cv.t = dsub(dmul(dba.t, nc), dmul(dca.t, nb));
    cv.x = dsub(dmul(dba.x, nc), dmul(dca.x, nb));
    cv.y = dsub(dmul(dba.y, nc), dmul(dca.y, nb));
    cv.z = dsub(dmul(dba.z, nc), dmul(dca.z, nb));
    return mdot(cv, x) > 0.0;
}

// Exhaustive decision for one direction, by a whole warp (all 32 lanes call it
// with the same arguments).  It returns what the sequential procedure returns:
// the argmin of tau in collider order (first index on ties), checked against
// every collider; when it fails, the first of its failures (in collider order)
// that passes every check, or the reference loop (GBF:162-199) when it failed
// more than kMaxFail times.  Lanes take colliders lane, lane + 32, ...; a
// check over all colliders is the AND of the lanes' checks, so its order does
// not matter.
__device__ __forceinline__ double tau_of(const D4& dba, const D4& x, bool& ok) {
    const double dot = mdot(dba, x);
    ok = false;
    double tau = CUDART_INF;
    if (dot > 1e-10) {
        tau = __ddiv_rn(mdot(dba, dba), dmul(2.0, dot));
        ok = tau > 0.0;
    }
    return tau;
}

// true when check(b, c) passes for every collider c other than a and b
__device__ bool warp_all_pass(const D4* __restrict__ B, size_t n_tot, uint32_t a, size_t b, const D4& xa,
                              const D4& dba, double nb, const D4& x) {
    const unsigned full = 0xffffffffu;
    for (size_t base = 0; base < n_tot; base += 32) {
        const size_t c = base + (threadIdx.x & 31);
        bool pass = true;
        if (c < n_tot && c != a && c != b) pass = check_pt(dba, nb, dsub4(B[c], xa), x);
        if (!__all_sync(full, pass)) return false;
    }
    return true;
}

__device__ long exhaustive_warp(const D4* __restrict__ B, size_t n_tot, uint32_t a, const D4& xa, const D4& x) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // 1. argmin: lane-local first minimum, then the (tau, index) minimum over lanes
    double bt = CUDART_INF;
    long bi = -1;
    for (size_t b = lane; b < n_tot; b += 32) {
        if (b == a) continue;
        bool ok;
        const double tau = tau_of(dsub4(B[b], xa), x, ok);
        if (ok && tau < bt) {
            bt = tau;
            bi = (long)b;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double t2 = __shfl_xor_sync(full, bt, o);
        const long i2 = __shfl_xor_sync(full, bi, o);
        if (i2 >= 0 && (bi < 0 || t2 < bt || (t2 == bt && i2 < bi))) {
            bt = t2;
            bi = i2;
        }
    }
    if (bi < 0) return -1;
    const long best = bi;
    // 2. check the argmin against every collider; keep its first kMaxFail failures
    const D4 dm = dsub4(B[best], xa);
    const double nm = mdot(dm, dm);
    long my_fail = -1;  // lane f holds failure f
    int nfail = 0;
    for (size_t base = 0; base < n_tot; base += 32) {
        const size_t c = base + lane;
        bool fail = false;
        if (c < n_tot && c != a && (long)c != best) fail = !check_pt(dm, nm, dsub4(B[c], xa), x);
        unsigned m = __ballot_sync(full, fail);
        while (m && nfail < kMaxFail) {
            const int bit = __ffs(m) - 1;
            m &= m - 1;
            if (lane == nfail) my_fail = (long)(base + bit);
            ++nfail;
        }
        nfail += __popc(m);
    }
    if (nfail == 0) return best;
    if (nfail > kMaxFail) {
        // the reference loop (GBF:162-199): candidates in collider order with tau below the current result's
        long r = -1;
        double rt = CUDART_INF;
        for (size_t base = 0; base < n_tot; base += 32) {
            const size_t b = base + lane;
            bool ok = false;
            double tau = CUDART_INF;
            if (b < n_tot && b != a) {
                // the reference's skips: dot <= 1e-10, tau <= 0 (NaN goes on, as there)
                const D4 dba = dsub4(B[b], xa);
                const double dot = mdot(dba, x);
                if (!(dot <= 1e-10)) {
                    tau = __ddiv_rn(mdot(dba, dba), dmul(2.0, dot));
                    ok = !(tau <= 0.0);
                }
            }
            unsigned m = __ballot_sync(full, ok);
            while (m) {
                const int bit = __ffs(m) - 1;
                m &= m - 1;
                const double tb = __shfl_sync(full, tau, bit);
                if (tb >= rt) continue;
                const size_t cb = base + bit;
                const D4 dba = dsub4(B[cb], xa);
                if (warp_all_pass(B, n_tot, a, cb, xa, dba, mdot(dba, dba), x)) {
                    r = (long)cb;
                    rt = tb;
                }
            }
        }
        return r;
    }
    // 3. the first failure (in collider order) that passes every check
    for (int f = 0; f < nfail; ++f) {
        const long c = __shfl_sync(full, my_fail, f);
        const D4 dc = dsub4(B[c], xa);
        bool ok;
        tau_of(dc, x, ok);
        if (!ok) continue;
        if (warp_all_pass(B, n_tot, a, (size_t)c, xa, dc, mdot(dc, dc), x)) return c;
    }
    return -1;
}

// ------------------------------------------------------------ k_neighbors
__device__ __forceinline__ void collider_bounds(const D4& d, double& key, double& D, double& Q, double& A) {
    const double dx = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    key = fmax(0.5 * (dx + d.t), 0.0);
    D = dx - d.t;
    Q = d.t * d.t + dx * dx;
    A = fabs(d.t) + dx;
}

__global__ void __launch_bounds__(kNbThreads)
    k_neighbors(const D4* __restrict__ bub, size_t n_int, size_t n_tot, const uint32_t* __restrict__ sel,
                const uint2* __restrict__ ranges, NbList* __restrict__ out) {
    __shared__ unsigned hist[2048];
    __shared__ unsigned s_prefix, s_mask, s_need, s_count, s_nout;
    __shared__ double s_key[kList];
    __shared__ int s_idx[kList];
    __shared__ double s_r1[kNbThreads], s_r2[kNbThreads];
    const int slot = blockIdx.x;
    uint32_t a = sel[slot];
    NbList* L = out + slot;
    if (a >= n_int) {  // not an interior bubble: marked, never dereferenced
        if (threadIdx.x == 0) L->count = -1;
        return;
    }
    if (ranges) {  // several realizations: this slot's colliders are its own realization's rows
        const uint2 r = ranges[slot];
        bub += r.x;
        n_tot = r.y;
        a -= r.x;
    }
    const D4 xa = bub[a];
    const size_t n_c = n_tot - 1;  // colliders other than a
    const bool complete = n_c <= (size_t)kList;
    auto fbits = [&](size_t c) -> unsigned {
        double key, D, Q, A;
        collider_bounds(dsub4(bub[c], xa), key, D, Q, A);
        return __float_as_uint(__double2float_rd(key));
    };
    if (threadIdx.x == 0) {
        s_prefix = 0;
        s_mask = 0;
        s_need = kList;  // rank of the cut value (1-based)
        s_count = 0;
        s_nout = 0;
    }
    __syncthreads();
    unsigned cut = 0xffffffffu;  // list = {c : fbits(c) < cut}
    if (!complete) {
        const int shifts[3] = {21, 10, 0};
        const unsigned widths[3] = {11, 11, 10};
        for (int p = 0; p < 3; ++p) {
            const unsigned dmask = (1u << widths[p]) - 1u;
            for (int q = threadIdx.x; q < 2048; q += kNbThreads) hist[q] = 0;
            __syncthreads();
            const unsigned pre = s_prefix, pm = s_mask;
            for (size_t c = threadIdx.x; c < n_tot; c += kNbThreads) {
                if (c == a) continue;
                const unsigned v = fbits(c);
                if ((v & pm) == pre) atomicAdd(&hist[(v >> shifts[p]) & dmask], 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned need = s_need, acc = 0, dsel = 0;
                for (unsigned dg = 0; dg <= dmask; ++dg) {
                    if (acc + hist[dg] >= need) {
                        dsel = dg;
                        break;
                    }
                    acc += hist[dg];
                }
                s_need = need - acc;
                s_prefix = pre | (dsel << shifts[p]);
                s_mask = pm | (dmask << shifts[p]);
            }
            __syncthreads();
        }
        cut = s_prefix;  // the kList-th smallest float key (bits)
    }
    // collect the list (unordered), then sort by (key, index)
    for (size_t c = threadIdx.x; c < n_tot; c += kNbThreads) {
        if (c == a) continue;
        double key, D, Q, A;
        collider_bounds(dsub4(bub[c], xa), key, D, Q, A);
        if (complete || __float_as_uint(__double2float_rd(key)) < cut) {
            const unsigned pos = atomicAdd(&s_count, 1u);
            if (pos < (unsigned)kList) {
                s_key[pos] = key;
                s_idx[pos] = (int)c;
            }
        }
    }
    __syncthreads();
    const int n = (int)min(s_count, (unsigned)kList);
    for (int q = n + threadIdx.x; q < kList; q += kNbThreads) {
        s_key[q] = CUDART_INF;
        s_idx[q] = 0x7fffffff;
    }
    __syncthreads();
    // bitonic sort of kList entries (kList a power of two <= 2 * kNbThreads)
    for (int size = 2; size <= kList; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int q = threadIdx.x; q < kList; q += kNbThreads) {
                const int p = q ^ stride;
                if (p > q) {
                    const bool up = (q & size) == 0;
                    const double kq = s_key[q], kp = s_key[p];
                    const int iq = s_idx[q], ip = s_idx[p];
                    const bool gt = kq > kp || (kq == kp && iq > ip);
                    if (gt == up) {
                        s_key[q] = kp;
                        s_key[p] = kq;
                        s_idx[q] = ip;
                        s_idx[p] = iq;
                    }
                }
            }
            __syncthreads();
        }
    }
    // rho bounds over every collider; near-lightlike colliders are kept aside
    double r1 = 0.0, r2 = 0.0;
    for (size_t c = threadIdx.x; c < n_tot; c += kNbThreads) {
        if (c == a) continue;
        double key, D, Q, A;
        collider_bounds(dsub4(bub[c], xa), key, D, Q, A);
        if (D > 1e-6 * A) {
            r1 = fmax(r1, Q / D);
            r2 = fmax(r2, A / D);
        } else {
            const unsigned pos = atomicAdd(&s_nout, 1u);
            if (pos < (unsigned)kMaxOutliers) L->outlier[pos] = (int)c;
        }
    }
    s_r1[threadIdx.x] = r1;
    s_r2[threadIdx.x] = r2;
    __syncthreads();
    for (int q = threadIdx.x; q < kList; q += kNbThreads) {
        L->key[q] = s_key[q];
        L->idx[q] = s_idx[q];
    }
    if (threadIdx.x == 0) {
        double m1 = 0.0, m2 = 0.0;
        for (int q = 0; q < kNbThreads; ++q) {
            m1 = fmax(m1, s_r1[q]);
            m2 = fmax(m2, s_r2[q]);
        }
        L->rho1 = m1 * (1.0 + 1e-12);
        L->rho2 = m2 * (1.0 + 1e-12);
        L->count = n;
        L->kmax = complete ? CUDART_INF : (double)__uint_as_float(cut);
        const unsigned no = s_nout;
        L->n_outliers = no <= (unsigned)kMaxOutliers ? (int)no : -1;
    }
}

// ------------------------------------------------------------ k_masks_list
// One block per (radiating bubble, direction range, frame): the candidate list
// is gathered into shared memory once, then every warp walks 32-direction
// chunks of the range independently (no block barrier after the prologue).
__global__ void __launch_bounds__(kMaskListThreads)
    k_masks_list(const D4* __restrict__ bub, size_t n_int, size_t n_tot, const uint32_t* __restrict__ sel,
                 const uint2* __restrict__ ranges, size_t n_sel, const NbList* __restrict__ lists,
                 const D4* __restrict__ dirs, size_t nd,
                 size_t row_len, unsigned n_split, double* __restrict__ tau_out, int32_t* __restrict__ code_out,
                 unsigned long long* __restrict__ counters) {
    // per listed collider: Delta = x_c - x_a and its Minkowski norm, computed once
    // per block with the reference's operations (direction independent)
    __shared__ D4 s_pos[kList];
    // per listed collider e: its Minkowski norm n_e and |n_e| + L1(Delta_e), the factor of e in
    // the sign filter's error bound (L1 = |dt| + |dx| + |dy| + |dz|), read together
    __shared__ double2 s_ns[kList];
    __shared__ double s_thr[kList]; // direction-independent part of the verification bound, see theta_of
    __shared__ double s_key[kList];
    __shared__ int s_idx[kList];
    __shared__ D4 s_opos[kMaxOutliers];
    __shared__ double s_onrm[kMaxOutliers];
    __shared__ int s_oidx[kMaxOutliers];
    const int k = blockIdx.y;
    const size_t slot = blockIdx.x / n_split;
    const unsigned part = blockIdx.x % n_split;
    // the block's directions: whole rows [r_begin, r_end) of row_len directions (one cos-theta row)
    const size_t n_rows = nd / row_len;
    const size_t rpb = (n_rows + n_split - 1) / n_split;
    const size_t r_begin = min(n_rows, rpb * part), r_end = min(n_rows, rpb * (part + 1));
    const size_t d_begin = r_begin * row_len, d_end = r_end * row_len;
    const int lane = threadIdx.x & 31;
    constexpr int kBatch = 2;
    // rows walked by a warp in one strip item; an item's first row has no seed, so longer items miss
    // fewer seeds (16 rows with 8192-direction blocks: 5 % faster than 8 rows with 4096)
    constexpr int kRowsPerItem = 16;
    const D4* B = bub + (size_t)k * n_tot;  // frame k
    uint32_t a = sel[slot];
    const NbList* L = lists + slot;
    const int n = L->count;
    __shared__ bool s_big;  // a listed Delta too large for the candidate filter's margin
    __shared__ unsigned s_next;  // the block's work queue of strip items
    if (threadIdx.x == 0) {
        s_big = false;
        s_next = 0;
    }
    __syncthreads();
    double* tau_row = tau_out + ((size_t)k * n_sel + slot) * nd;
    int32_t* code_row = code_out ? code_out + ((size_t)k * n_sel + slot) * nd : nullptr;
    if (a >= n_int || n < 0) {  // invalid radiating bubble: sentinel outputs
        for (size_t d = d_begin + threadIdx.x; d < d_end; d += kMaskListThreads) {
            tau_row[d] = CUDART_NAN;
            if (code_row) code_row[d] = INT32_MIN;
        }
        return;
    }
    if (ranges) {  // several realizations: this slot's colliders are its own realization's rows
        const uint2 r = ranges[slot];
        B += r.x;
        n_tot = r.y;
        a -= r.x;
    }
    const int no = L->n_outliers;
    const D4 xa = B[a];
    for (int q = threadIdx.x; q < n; q += kMaskListThreads) {
        const int c = L->idx[q];
        s_idx[q] = c;
        s_key[q] = L->key[q];
        const D4 dc = dsub4(B[c], xa);
        s_pos[q] = dc;
        const double nrm_q = mdot(dc, dc);
        const double l1_q = fabs(dc.t) + fabs(dc.x) + fabs(dc.y) + fabs(dc.z);
        s_ns[q] = make_double2(nrm_q, fabs(nrm_q) + l1_q);
        {
            // theta = tau (1 + 1e-12) + 64 u (A rho1 + Q rho2) / dot with 1 / dot = 2 tau / nrm
            // for a collider (nrm > 0): theta = tau (1 + 1e-12 + s_thr)
            const double dx = sqrt(dc.x * dc.x + dc.y * dc.y + dc.z * dc.z);
            const double Ac = fabs(dc.t) + dx, Qc = dc.t * dc.t + dx * dx;
            s_thr[q] = nrm_q > 0.0 ? 2.0 * (64.0 * 1.1102230246251565e-16) * (Ac * L->rho1 + Qc * L->rho2) / nrm_q
                                      : CUDART_INF;
        }
        if (!(l1_q < 1e5)) s_big = true;  // benign race: every writer stores true
    }
    for (int q = threadIdx.x; q < no; q += kMaskListThreads) {
        s_oidx[q] = L->outlier[q];
        const D4 dc = dsub4(B[L->outlier[q]], xa);
        s_opos[q] = dc;
        s_onrm[q] = mdot(dc, dc);
    }
    __syncthreads();
    const double kmax = L->kmax;
    unsigned long long n_full = 0;
    // Work items: 32 consecutive directions of a row (a strip) over up to kRowsPerItem
    // consecutive rows.  A lane walks its column down the rows; each result, when it came
    // from the list, seeds the next row's candidate (the neighbouring patch in cos theta
    // most often has the same first collider).  Warps take items from a shared counter.
    const size_t n_strips = (row_len + 31) / 32;
    const size_t n_groups = (r_end - r_begin + kRowsPerItem - 1) / kRowsPerItem;
    const size_t n_items = n_strips * n_groups;
    for (;;) {
      unsigned item = 0;
      if (lane == 0) item = atomicAdd(&s_next, 1u);
      item = __shfl_sync(0xffffffffu, item, 0);
      if (item >= n_items) break;
      const size_t strip = item % n_strips, group = item / n_strips;
      const size_t col = strip * 32 + lane;
      const bool live = col < row_len;
      int seed = -1;
      // each row's direction is loaded one row ahead, so that its latency overlaps the search
      D4 x_next = dirs[(r_begin + group * kRowsPerItem) * row_len + (live ? col : 0)];
      for (int rr = 0; rr < kRowsPerItem; ++rr) {
        const size_t rw = r_begin + group * kRowsPerItem + rr;
        if (rw >= r_end) break;  // warp-uniform
        // the barrier reconverges lanes whose searches ended at different steps
        __syncwarp();
        const size_t d = rw * row_len + (live ? col : 0);
        const D4 x = x_next;
        if (rr + 1 < kRowsPerItem && rw + 1 < r_end) x_next = dirs[d + row_len];
        long result = -1;
        int res_pos = -1;      // list position of the result, when it came from the list
        double res_tau = 0.0;  // tau of the result when it came from the list (same operations)
        bool full = no < 0 || s_big;

        // Approximate Minkowski product with the direction (FMA chain): within
        // 4.01 u L1(d) of the exact value, since |x_i| <= 1.
        auto adot = [&](const D4& p) { return fma(p.z, x.z, fma(p.y, x.y, fma(p.x, x.x, -(p.t * x.t)))); };

        // Verifies candidate c (Delta dc, norm nc) against the list up to key theta and the
        // outliers.  check(c, e) is the sign of the reference's expression V_ref; the filter value
        //   V = fma(ne, adot(c), -(nc adot(e)))
        // is within 6.03 u S of the exact value and V_ref within 6.01 u S, where
        // S = |ne| L1(c) + |nc| L1(e); |V| > 32 u S (plus an underflow guard) fixes
        // the sign, otherwise the reference's expression is evaluated.  The bound is taken as
        // 32 u max(L1(c), |nc|) (|ne| + L1(e)) >= 32 u S: looser, which only sends a few more
        // values near zero to the exact evaluation.  c is the candidate's collider index, cpos its
        // list position (the list holds each collider once).
        auto verify = [&](int c, int cpos, const D4& dc, double nc, double theta, int* fails, int& nfail,
                          int* first_fail = nullptr) -> bool {
            const double dotc = adot(dc);
            const double l1c = fabs(dc.t) + fabs(dc.x) + fabs(dc.y) + fabs(dc.z);
            const double mc = 32.0 * 1.1102230246251565e-16 * fmax(l1c, fabs(nc));
            bool ok = true;
            // entries in batches of kBatch: their filter values are independent
            // (instruction-level parallelism); decisions are taken in list order
            bool done = false;
            for (int e0 = 0; e0 < n && !done; e0 += kBatch) {
                double vb[kBatch], bb[kBatch], kb[kBatch];
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
                    const int e = min(e0 + j, n - 1);
                    kb[j] = s_key[e];
                    const D4 pe = s_pos[e];
                    const double2 ns = s_ns[e];
                    vb[j] = fma(ns.x, dotc, -(nc * adot(pe)));
                    bb[j] = fma(ns.y, mc, 1e-300);
                }
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
                    const int e = e0 + j;
                    if (e >= n || kb[j] > theta) {
                        done = true;
                        break;
                    }
                    if (e == cpos) continue;
                    bool pass;
                    if (vb[j] > bb[j]) pass = true;
                    else if (vb[j] < -bb[j]) pass = false;
                    else pass = check_pre(dc, nc, s_pos[e], s_ns[e].x, x);
                    if (!pass) {
                        ok = false;
                        if (fails) {
                            if (nfail < kMaxFail) fails[nfail] = e;
                            ++nfail;
                        } else {
                            if (first_fail) *first_fail = e;
                            return false;
                        }
                    }
                }
            }
            for (int e = 0; e < no; ++e) {
                const int ce = s_oidx[e];
                if (ce == c) continue;
                bool in_list = false;  // already checked above when listed with key <= theta
                for (int q = 0; q < n && s_key[q] <= theta; ++q) in_list |= (s_idx[q] == ce);
                if (in_list) continue;
                if (!check_pre(dc, nc, s_opos[e], s_onrm[e], x)) {
                    ok = false;
                    if (!fails) return false;
                    nfail = kMaxFail + 1;  // outliers are resolved by the exhaustive path
                }
            }
            return ok;
        };
        // The verification bound of listed candidate e with delay tau (the 1e-12 relative slack
        // covers the few roundings of this form)
        auto theta_of = [&](int e, double tau) { return tau * ((1.0 + 1e-12) + s_thr[e]); };

        // 0. the previous row's result at this column (the neighbouring patch in cos theta
        //    most often has the same first collider): checked against every listed collider up
        //    to its bound and the outliers, stopping at the first failure.  If it passes it is
        //    the exact answer (the passer is unique).  If it fails against a listed collider,
        //    that collider (where the first-collider region most often moved to between the
        //    rows) is checked the same way.  Otherwise the direction takes steps 1-3.
        bool seeded = false;
        auto try_seed = [&](int q, int* first_fail) {
            const D4 dq = s_pos[q];
            const double dd = mdot(dq, x);
            if (!(dd > 1e-10)) return false;
            const double tq = __ddiv_rn(s_ns[q].x, dmul(2.0, dd));
            if (!(tq > 0.0)) return false;
            const double th = theta_of(q, tq);
            int dummy = 0;
            if (!(th < kmax) || !verify(s_idx[q], q, dq, s_ns[q].x, th, nullptr, dummy, first_fail)) return false;
            result = s_idx[q];
            res_pos = q;
            res_tau = tq;
            return true;
        };
        if (!full && seed >= 0) {
            int ff = -1;
            seeded = try_seed(seed, &ff);
            if (!seeded && ff >= 0) seeded = try_seed(ff, nullptr);
        }

        if (!full && !seeded) {
            // 1. a candidate: the approximate argmin of tau = nrm / (2 dot) in key order
            //    (quotients compared by cross-multiplication), stopping once key exceeds
            //    the best quotient with a margin.  Any candidate serves: steps 2-3 decide
            //    exactly whatever it is; the exact argmin only keeps step 3 idle.
            double bn = 0.0, bd = 0.0;  // best quotient bn / bd, bd > 0
            int bi = -1;
            bool ended = true, stop = false;
            for (int e0 = 0; e0 < n && !stop; e0 += kBatch) {
                double kb[kBatch], nb[kBatch], db[kBatch];
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
                    const int e = min(e0 + j, n - 1);
                    kb[j] = s_key[e];
                    nb[j] = s_ns[e].x;
                    db[j] = 2.0 * adot(s_pos[e]);
                }
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
                    if (e0 + j >= n) break;
                    if (bi >= 0 && kb[j] * bd > bn * (1.0 + 1e-11)) {
                        ended = false;
                        stop = true;
                        break;
                    }
                    // every collider of the exact test (dot > 1e-10, nrm > 0) has den > 0 here,
                    // since the block's L1 norms keep 4.01 u L1 below 1e-10
                    if (db[j] > 0.0 && nb[j] > 0.0 && (bi < 0 || nb[j] * bd < bn * db[j])) {
                        bn = nb[j];
                        bd = db[j];
                        bi = e0 + j;
                    }
                }
            }
            double best = CUDART_INF, dotm = 0.0;
            if (bi >= 0) {
                // the candidate's tau with the reference's operations (compute_delta_tab)
                dotm = mdot(s_pos[bi], x);
                if (dotm > 1e-10) best = __ddiv_rn(s_ns[bi].x, dmul(2.0, dotm));
                if (!(dotm > 1e-10) || !(best > 0.0)) full = true;  // not a collider by the exact test
            }
            if (!full && ended && !(kmax > best * (1.0 + 1e-11))) full = !(bi < 0 && kmax == CUDART_INF);
            if (!full && bi >= 0) {
                // 2. verify the candidate
                const D4 dm = s_pos[bi];
                const double nm = s_ns[bi].x;
                const double th = theta_of(bi, best);
                if (!(th < kmax)) {
                    full = true;
                } else {
                    int fails[kMaxFail];
                    int nfail = 0;
                    if (verify(s_idx[bi], bi, dm, nm, th, fails, nfail)) {
                        result = s_idx[bi];
                        res_pos = bi;
                        res_tau = best;
                    } else if (nfail > kMaxFail) {
                        full = true;
                    } else {
                        // 3. the passer, if any, is among the failures
                        for (int f = 0; f < nfail && result < 0 && !full; ++f) {
                            const int e = fails[f];
                            const D4 dc = s_pos[e];
                            const double dot = mdot(dc, x);
                            if (!(dot > 1e-10)) continue;
                            const double nc = s_ns[e].x;
                            const double tau = __ddiv_rn(nc, dmul(2.0, dot));
                            if (!(tau > 0.0)) continue;
                            const double thf = theta_of(e, tau);
                            if (!(thf < kmax)) {
                                full = true;
                                break;
                            }
                            int dummy = 0;
                            if (verify(s_idx[e], e, dc, nc, thf, nullptr, dummy)) {
                                result = s_idx[e];
                                res_pos = e;
                                res_tau = tau;
                            }
                        }
                    }
                }
            }
        }
        // directions that left the list are decided by the whole warp, one at a time
        unsigned fm = __ballot_sync(0xffffffffu, full && live);
        n_full += (full && live) ? 1 : 0;
        while (fm) {
            const int src = __ffs(fm) - 1;
            fm &= fm - 1;
            D4 xs;
            xs.t = __shfl_sync(0xffffffffu, x.t, src);
            xs.x = __shfl_sync(0xffffffffu, x.x, src);
            xs.y = __shfl_sync(0xffffffffu, x.y, src);
            xs.z = __shfl_sync(0xffffffffu, x.z, src);
            const long r = exhaustive_warp(B, n_tot, a, xa, xs);
            if (lane == src) result = r;
        }
        if (full && result >= 0) {
            // compute_delta_tab (GBF:457-466)
            const D4 dba = dsub4(B[result], xa);
            const double dot = mdot(dba, x);
            res_tau = fabs(dot) < 1e-10 ? 0.0 : __ddiv_rn(mdot(dba, dba), dmul(2.0, dot));
        }
        // compute_delta_tab (GBF:457-466): a listed result has dot > 1e-10, and its
        // tau above was formed with the same operations from the same Delta.
        if (live) {
            tau_row[d] = result >= 0 ? res_tau : 0.0;
            if (code_row)
                code_row[d] =
                    result < 0 ? -1 : ((size_t)result < n_int ? (int32_t)result : -((int32_t)(result - n_int) + 2));
        }
        seed = full ? -1 : res_pos;
      }
    }
    if (n_full) atomicAdd(counters, n_full);
}

// Blocks per radiating bubble and frame: whole rows of about eight thousand
// directions per block amortise the list gather and keep the seed chains long;
// ranges shrink (to one row at least) when there are too few blocks to fill the
// GPU.
static unsigned mask_split(size_t nd, size_t row_len, size_t n_pairs) {
    const size_t n_rows = nd / row_len;
    size_t rpb = std::max<size_t>(1, 8192 / row_len);
    size_t split = (n_rows + rpb - 1) / rpb;
    const size_t want = 148 * 16;  // blocks for about four waves of resident blocks
    while (split * n_pairs < want && split * 2 <= n_rows) split *= 2;
    if (split > n_rows) split = n_rows;
    return (unsigned)(split < 1 ? 1 : split);
}

// ------------------------------------------------------------------ host
void launch_masks_with_lists(cudaStream_t stream, const D4* bub, size_t n_int, size_t n_tot, const uint32_t* sel,
                             size_t n_sel, const D4* dirs, size_t nd, NbList* lists, double* tau, int32_t* codes,
                             unsigned long long* counters) {
    if (n_tot < 2) {
        CUDA_OK(cudaMemsetAsync(tau, 0, n_sel * nd * sizeof(double), stream));
        if (codes) CUDA_OK(cudaMemsetAsync(codes, 0xff, n_sel * nd * sizeof(int32_t), stream));
        return;
    }
    if (n_sel > 0x7fffffffULL) throw Error{"too many radiating bubbles"};
    k_neighbors<<<(unsigned)n_sel, kNbThreads, 0, stream>>>(bub, n_int, n_tot, sel, nullptr, lists);
    CUDA_OK(cudaGetLastError());
    // the directions' row structure is not known here: one row of nd directions
    const unsigned n_split = mask_split(nd, nd, n_sel);
    const size_t gx = (size_t)n_split * n_sel;
    if (gx > 0x7fffffffULL) throw Error{"too many (bubble, patch) pairs for one launch"};
    k_masks_list<<<dim3((unsigned)gx, 1), kMaskListThreads, 0, stream>>>(bub, n_int, n_tot, sel, nullptr, n_sel, lists,
                                                                        dirs, nd, nd, n_split, tau, codes, counters);
    CUDA_OK(cudaGetLastError());
}

void launch_mask_pipeline(Device* dev, const D4* bub_unrot, const D4* bub_frames, size_t n_int, size_t n_tot,
                          const uint32_t* sel, const uint2* ranges, size_t n_sel, const D4* dirs, size_t nd,
                          size_t row_len, size_t kn, double* tau, int32_t* codes, unsigned long long* counters,
                          bool build_lists, uint64_t* launches, int chunking) {
    if (row_len == 0 || nd % row_len != 0) row_len = nd;
    if (n_tot < 2) {
        // a lone bubble has no collider: every direction is None
        CUDA_OK(cudaMemsetAsync(tau, 0, kn * n_sel * nd * sizeof(double), dev->stream));
        if (codes) CUDA_OK(cudaMemsetAsync(codes, 0xff, kn * n_sel * nd * sizeof(int32_t), dev->stream));
        return;
    }
    dev->nblists.ensure(n_sel * sizeof(NbList));
    if (build_lists) {
        if (n_sel > 0x7fffffffULL) throw Error{"too many radiating bubbles"};
        k_neighbors<<<(unsigned)n_sel, kNbThreads, 0, dev->stream>>>(bub_unrot, n_int, n_tot, sel, ranges,
                                                                      (NbList*)dev->nblists.p);
        CUDA_OK(cudaGetLastError());
        if (launches) ++*launches;
    }
    // the launch shape may ask for 2 or 4 times the automatic number of blocks (at most one row each)
    const unsigned n_split = (unsigned)std::min<size_t>(
        nd / row_len, (size_t)mask_split(nd, row_len, n_sel * kn) * (size_t)std::max(1, std::min(chunking, 4)));
    const size_t gx = (size_t)n_split * n_sel;
    if (gx > 0x7fffffffULL || kn > 65535) throw Error{"too many (bubble, patch) pairs for one launch"};
    dim3 grid((unsigned)gx, (unsigned)kn);
    k_masks_list<<<grid, kMaskListThreads, 0, dev->stream>>>(bub_frames, n_int, n_tot, sel, ranges, n_sel,
                                                             (const NbList*)dev->nblists.p, dirs, nd, row_len, n_split, tau,
                                                             codes, counters);
    CUDA_OK(cudaGetLastError());
    if (launches) ++*launches;
}

}  // namespace bgw
