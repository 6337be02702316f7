// Device-side nucleation Monte Carlo for ensembles: every realization's
// bubbles are drawn on the GPU, one block per realization.
//
// Exponential-rate nucleation in a periodic box of side L: candidates arrive
// as a Poisson process with rate Gamma0 V e^{beta t}; a candidate is rejected
// when it lies inside an accepted bubble's wall (nearest periodic copy, the
// rejection against bubbles and images of
// rust/bubble-gw/src/many_bubbles/bubbles_nucleation/fixed_rate_nucleation.rs);
// when max_rejections candidates have been rejected before n bubbles are
// placed, the prefactor doubles and the draw restarts.  Random numbers:
// Philox4x32-10 (Salmon et al., SC'11), candidate q of attempt a from the
// block at counter (q, a, 0, 0) under key (seed mod 2^32, seed div 2^32),
// u_i = (x_i + 0.5) 2^-32, so the draws do not depend on the launch shape.
// The candidate loop is sequential per realization; the test against the
// accepted bubbles is spread over the block's threads.  Arithmetic is unfused
// (__dmul_rn / __dadd_rn) in a fixed order.

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "bgw_internal.h"
#include "device_common.cuh"

namespace bgw {

namespace {

constexpr int kNucThreads = 128;

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

struct NucArgs {
    const int64_t* n;         // (R) bubbles per realization
    const double* beta;       // (R)
    const uint64_t* seed;     // (R)
    const size_t* offset;     // (R + 1) first row of each realization
    double L, gamma_scale;
    int64_t max_rejections;
    int max_attempts;
    double* interior;         // (offset[R], 4)
    double* exterior;         // (6 offset[R], 4)
    int32_t* attempts;        // (R): attempts used, -1 when none placed every bubble
};

__global__ void __launch_bounds__(kNucThreads) k_nucleate(NucArgs A) {
    const int r = blockIdx.x;
    const int64_t n = A.n[r];
    const double beta = A.beta[r], L = A.L;
    const uint64_t seed = A.seed[r];
    double* out = A.interior + A.offset[r] * 4;  // accepted bubbles, times not yet shifted
    const double V = __dmul_rn(__dmul_rn(L, L), L);
    double g0 = __ddiv_rn(__dmul_rn(__dmul_rn(A.gamma_scale, (double)n), beta), V);
    int placed_attempt = -1;
    for (int attempt = 0; attempt < A.max_attempts && placed_attempt < 0; ++attempt) {
        int64_t k = 0, rej = 0;
        uint32_t q = 0;
        double t = 0.0;
        while (k < n && rej < A.max_rejections) {
            uint32_t c[4] = {q, (uint32_t)attempt, 0u, 0u};
            philox4x32_10(c, (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
            ++q;
            const double u0 = ((double)c[0] + 0.5) * 0x1p-32, u1 = ((double)c[1] + 0.5) * 0x1p-32;
            const double u2 = ((double)c[2] + 0.5) * 0x1p-32, u3 = ((double)c[3] + 0.5) * 0x1p-32;
            // next arrival: e^{beta t'} = e^{beta t} - beta log(u0) / (Gamma0 V)
            t = __ddiv_rn(log(__dsub_rn(exp(__dmul_rn(beta, t)), __ddiv_rn(__dmul_rn(beta, log(u0)),
                                                                              __dmul_rn(g0, V)))),
                          beta);
            const double x = __dmul_rn(L, u1), y = __dmul_rn(L, u2), z = __dmul_rn(L, u3);
            int hit = 0;
            for (int64_t j = threadIdx.x; j < k && !hit; j += kNucThreads) {
                const double* p = out + j * 4;
                double dx = fabs(__dsub_rn(x, p[1])), dy = fabs(__dsub_rn(y, p[2])), dz = fabs(__dsub_rn(z, p[3]));
                dx = fmin(dx, __dsub_rn(L, dx));
                dy = fmin(dy, __dsub_rn(L, dy));
                dz = fmin(dz, __dsub_rn(L, dz));
                const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                const double rad = __dsub_rn(t, p[0]);
                hit = r2 < __dmul_rn(rad, rad);
            }
            if (__syncthreads_or(hit)) {
                ++rej;
                continue;
            }
            if (threadIdx.x == 0) {
                double* p = out + k * 4;
                p[0] = t;
                p[1] = x;
                p[2] = y;
                p[3] = z;
            }
            __syncthreads();  // the new bubble is visible to every thread before the next test
            ++k;
        }
        if (k == n) placed_attempt = attempt;
        else g0 = __dmul_rn(g0, 2.0);
    }
    if (threadIdx.x == 0) A.attempts[r] = placed_attempt < 0 ? -1 : placed_attempt + 1;
    if (placed_attempt < 0 || n == 0) return;
    // times relative to the first bubble; six periodic images per bubble (+x, -x, +y, -y, +z, -z)
    const double t0 = out[0];
    __syncthreads();
    double* ext = A.exterior + A.offset[r] * 24;
    for (int64_t j = threadIdx.x; j < n; j += kNucThreads) {
        double* p = out + j * 4;
        const double tj = __dsub_rn(p[0], t0);
        const double px = p[1], py = p[2], pz = p[3];
        const double sh[6][3] = {{L, 0, 0}, {-L, 0, 0}, {0, L, 0}, {0, -L, 0}, {0, 0, L}, {0, 0, -L}};
        for (int m = 0; m < 6; ++m) {
            double* e = ext + (j * 6 + m) * 4;
            e[0] = tj;
            e[1] = __dadd_rn(px, sh[m][0]);
            e[2] = __dadd_rn(py, sh[m][1]);
            e[3] = __dadd_rn(pz, sh[m][2]);
        }
    }
    __syncthreads();
    for (int64_t j = threadIdx.x; j < n; j += kNucThreads) out[j * 4] = __dsub_rn(out[j * 4], t0);
}

}  // namespace

void run_nucleation(const int64_t* n, const double* beta, const uint64_t* seed, size_t R, double L,
                    double gamma_scale, int64_t max_rejections, int max_attempts, double* interior,
                    double* exterior, int32_t* attempts) {
    int dev_count = device_count();
    if (dev_count <= 0)
        throw Error{"no CUDA device is available: the nucleation sampler runs only on the GPU (no CPU fallback)"};
    std::vector<size_t> off(R + 1, 0);
    for (size_t r = 0; r < R; ++r) off[r + 1] = off[r] + (size_t)n[r];
    const size_t rows = off[R];
    if (R == 0) return;
    if (R > 0x7fffffffULL) throw Error{"too many realizations"};
    cudaStream_t st;
    CUDA_OK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    void* buf = nullptr;
    const size_t bytes = R * (sizeof(int64_t) + sizeof(double) + sizeof(uint64_t) + sizeof(int32_t)) +
                         (R + 1) * sizeof(size_t) + rows * 4 * sizeof(double) * 7 + 256;
    cudaError_t e = cudaMalloc(&buf, bytes);
    if (e != cudaSuccess) {
        cudaStreamDestroy(st);
        throw Error{std::string("cudaMalloc failed for the nucleation sampler: ") + cudaGetErrorString(e)};
    }
    try {
        unsigned char* p = static_cast<unsigned char*>(buf);
        auto take = [&](size_t b) {
            unsigned char* q = p;
            p += (b + 15) & ~size_t(15);
            return q;
        };
        NucArgs A;
        A.n = reinterpret_cast<int64_t*>(take(R * sizeof(int64_t)));
        A.beta = reinterpret_cast<double*>(take(R * sizeof(double)));
        A.seed = reinterpret_cast<uint64_t*>(take(R * sizeof(uint64_t)));
        A.offset = reinterpret_cast<size_t*>(take((R + 1) * sizeof(size_t)));
        A.attempts = reinterpret_cast<int32_t*>(take(R * sizeof(int32_t)));
        A.interior = reinterpret_cast<double*>(take(rows * 4 * sizeof(double)));
        A.exterior = reinterpret_cast<double*>(take(rows * 24 * sizeof(double)));
        A.L = L;
        A.gamma_scale = gamma_scale;
        A.max_rejections = max_rejections;
        A.max_attempts = max_attempts;
        CUDA_OK(cudaMemcpyAsync((void*)A.n, n, R * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync((void*)A.beta, beta, R * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync((void*)A.seed, seed, R * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync((void*)A.offset, off.data(), (R + 1) * sizeof(size_t), cudaMemcpyHostToDevice, st));
        k_nucleate<<<(unsigned)R, kNucThreads, 0, st>>>(A);
        CUDA_OK(cudaGetLastError());
        CUDA_OK(cudaMemcpyAsync(attempts, A.attempts, R * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        if (rows) {
            CUDA_OK(cudaMemcpyAsync(interior, A.interior, rows * 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
            CUDA_OK(cudaMemcpyAsync(exterior, A.exterior, rows * 24 * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        CUDA_OK(cudaStreamSynchronize(st));
    } catch (...) {
        cudaStreamSynchronize(st);
        cudaFree(buf);
        cudaStreamDestroy(st);
        throw;
    }
    cudaFree(buf);
    cudaStreamDestroy(st);
}

}  // namespace bgw
