// Measured launch shape of the factored spectrum kernels.
//
// Three knobs set how a spectrum call is cut into launches: the number of k-hat
// frames per launch (each launch runs masks, beta and the GEMM over that many
// frames; the memory budget gives the largest) and, for the tensor-core GEMM,
// the number of cos-theta row parts each (frequency tile, column tile) is
// split into (the wave-fill model picks one) and its pipeline stages (3 to 5
// stages of 32 steps).  The tuner times a few candidates around the automatic
// choice on a sample of the job's own frames, keeps the fastest shape, then
// times the stage counts at that shape.  Every candidate computes the same
// spectrum: frames are independent, the row parts only regroup FP64 partial
// sums and the stages only change the overlap of copies and MMAs.
//
// Choices are keyed by the device (name, multiprocessor count) and every size
// the launch shapes depend on; they live for the process and, when
// BGWX_AUTOTUNE_CACHE names a file, are read from and appended to that file
// (one "key frames row_parts stages mask_chunking" line per shape).  The mask
// search's chunking (blocks per bubble and frame: 1, 2 or 4 times the automatic
// number) is timed last, at the chosen shape.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "bgw_internal.h"
#include "device_common.cuh"

namespace bgw {

namespace {

std::mutex g_mu;
std::map<std::string, LaunchShape> g_cache;
bool g_loaded = false;

const char* cache_file() {
    const char* p = std::getenv("BGWX_AUTOTUNE_CACHE");
    return (p && *p) ? p : nullptr;
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const char* path = cache_file();
    if (!path) return;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string key;
        long long f = 0, r = 0, st = 0, mc = 0;
        if (!(ls >> key >> f >> r) || f < 1 || r < 1 || r > 16) continue;  // malformed lines are skipped
        if (!(ls >> st) || st < 3 || st > 5) st = 0;                       // older lines: automatic stages
        if (!(ls >> mc) || mc < 1 || mc > 4) mc = 0;                       // older lines: automatic chunking
        g_cache[key] = LaunchShape{(size_t)f, (int)r, (int)st, (int)mc};
    }
}

void append_locked(const std::string& key, const LaunchShape& s) {
    const char* path = cache_file();
    if (!path) return;
    std::ofstream out(path, std::ios::app);
    if (out)
        out << key << ' ' << s.frames_per_launch << ' ' << s.row_parts << ' ' << s.gemm_stages << ' '
            << s.mask_chunking << '\n';
}

std::string shape_key(const Device* dev, const SpectrumJob& job) {
    cudaDeviceProp prop{};
    CUDA_OK(cudaGetDeviceProperties(&prop, dev->id));
    std::string name = prop.name;
    for (auto& ch : name)
        if (ch == ' ' || ch == '\t') ch = '_';
    std::ostringstream k;
    k << name << ':' << dev->n_sm << ":k" << (int)job.kernel << ":int" << job.n_int << ":tot" << job.n_tot << ":sel"
      << job.n_sel << ":c" << job.n_cos << ":p" << job.n_phi << ":t" << job.n_t << ":w" << job.n_w << ":s"
      << job.n_sets << ":m" << job.n_terms << ":d" << (job.has_damping ? 1 : 0) << ":K" << job.n_k << ":R" << job.n_real;
    return k.str();
}

// Device time of one spectrum run of `job` into the device array `out`
// (run_spectrum's own events around its launches).  Throws Error when a
// kernel of the run reported a failed wait.
float time_run(Device* dev, const SpectrumJob& job, double* out) {
    run_spectrum(dev, job, out, true, nullptr);  // waits for the run and checks its error counters
    float ms = 0.0f;
    CUDA_OK(cudaEventElapsedTime(&ms, dev->ev[4], dev->ev[5]));
    return ms;
}

}  // namespace

LaunchShape autotune_launch_shape(Device* dev, const SpectrumJob& job) {
    LaunchShape automatic;
    if (job.kernel == BGWX_KERNEL_FP64_DIRECT || job.n_sel == 0 || job.n_k == 0 || job.n_w == 0 || job.n_sets == 0)
        return automatic;
    CUDA_OK(cudaSetDevice(dev->id));
    const std::string key = shape_key(dev, job);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_locked();
        auto it = g_cache.find(key);
        if (it != g_cache.end()) return it->second;
    }
    const size_t kc_max = std::min(job.n_k, spectrum_max_frames_per_launch(job));
    // the sample: one launch of the largest frame count (all frames if fewer)
    const size_t n_s = kc_max;
    std::vector<size_t> frames;
    for (size_t f = kc_max; f >= 1 && frames.size() < 3; f /= 2) {
        frames.push_back(f);
        if (f == 1) break;
    }
    struct Cand {
        size_t f;
        int r;
    };
    std::vector<Cand> cands;
    const int r_max = std::max(1, std::min(16, (int)job.n_cos / 8));
    for (size_t f : frames) {
        const int r0 = factored_auto_row_parts(dev, job, f);
        if (job.kernel != BGWX_KERNEL_MIXED) {
            cands.push_back({f, 1});
            continue;
        }
        for (int r : {r0, r0 - 1, r0 + 1})
            if (r >= 1 && r <= r_max) {
                bool dup = false;
                for (const Cand& c : cands) dup |= (c.f == f && c.r == r);
                if (!dup) cands.push_back({f, r});
            }
    }
    SpectrumJob sub = job;
    sub.n_k = n_s;  // the first n_s frames (rot rows are frame-major)
    if (!job.rot) sub.n_k = 1;
    const size_t out_bytes = std::max<size_t>(1, job.n_real) * sub.n_k * 2 * job.n_sets * job.n_w * sizeof(double2);
    double* out = nullptr;
    CUDA_OK(cudaMalloc(&out, out_bytes));
    LaunchShape best;
    float best_ms = 0.0f;
    try {
        // untimed first run: work arrays grow to the largest candidate, tables are built
        sub.frames_per_launch = cands.front().f;
        sub.row_parts = cands.front().r;
        run_spectrum(dev, sub, out, true, nullptr);
        std::string last_err;
        for (const Cand& c : cands) {
            sub.frames_per_launch = c.f;
            sub.row_parts = c.r;
            float ms = 0.0f;
            try {
                ms = time_run(dev, sub, out);
            } catch (const Error& e) {  // a shape whose run failed is never chosen
                last_err = e.msg;
                continue;
            }
            if (best.frames_per_launch == 0 || ms < best_ms) {
                best_ms = ms;
                best.frames_per_launch = c.f;
                best.row_parts = c.r;
            }
        }
        if (best.frames_per_launch == 0) throw Error{"autotune: every candidate launch shape failed: " + last_err};
        if (job.kernel == BGWX_KERNEL_MIXED) {
            // the GEMM's pipeline stages at the chosen shape (4 was among the timed runs)
            best.gemm_stages = 4;
            sub.frames_per_launch = best.frames_per_launch;
            sub.row_parts = best.row_parts;
            for (int stg : {3, 5}) {
                sub.gemm_stages = stg;
                float ms = 0.0f;
                try {
                    ms = time_run(dev, sub, out);
                } catch (const Error&) {
                    continue;
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best.gemm_stages = stg;
                }
            }
        }
        // the mask search's chunking at the chosen shape (1 was among the timed runs)
        best.mask_chunking = 1;
        sub.frames_per_launch = best.frames_per_launch;
        sub.row_parts = best.row_parts;
        sub.gemm_stages = best.gemm_stages;
        for (int mc : {2, 4}) {
            sub.mask_chunking = mc;
            float ms = 0.0f;
            try {
                ms = time_run(dev, sub, out);
            } catch (const Error&) {
                continue;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best.mask_chunking = mc;
            }
        }
    } catch (...) {
        cudaStreamSynchronize(dev->stream);
        cudaFree(out);
        throw;
    }
    CUDA_OK(cudaStreamSynchronize(dev->stream));
    CUDA_OK(cudaFree(out));
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_cache.find(key) == g_cache.end()) {
        g_cache[key] = best;
        append_locked(key, best);
    }
    return g_cache[key];
}

}  // namespace bgw
