// First-collider search with per-bubble candidate lists (masks.cu).
#pragma once

#include "device_common.cuh"

namespace bgw {

constexpr int kList = 512;           // candidate colliders per radiating bubble
constexpr int kMaxOutliers = 8;      // always-checked near-lightlike colliders
constexpr int kMaxFail = 8;          // failures of the argmin resolved without the reference loop
constexpr int kNbThreads = 256;
constexpr int kMaskListThreads = 128;

// Candidate list of one radiating bubble (frame independent).
struct NbList {
    double key[kList];   // lower bounds (|dx| + dt) / 2 of tau, ascending
    int idx[kList];      // collider indices (interior then exterior numbering)
    int outlier[kMaxOutliers];
    double kmax;         // every collider outside the list has key >= kmax (inf: list complete)
    double rho1, rho2;   // max (dt^2+|dx|^2)/D and (|dt|+|dx|)/D over the colliders
    int count;           // entries in the list
    int n_outliers;      // -1: too many near-lightlike colliders, use the exhaustive scan
};

// Builds candidate lists into `lists` (n_sel entries) and runs the exact
// search for one frame on `stream`; tau/codes: (n_sel, nd).  Allocates nothing.
void launch_masks_with_lists(cudaStream_t stream, const D4* bub, size_t n_int, size_t n_tot, const uint32_t* sel,
                             size_t n_sel, const D4* dirs, size_t nd, NbList* lists, double* tau, int32_t* codes,
                             unsigned long long* counters);

// Builds the lists (when build_lists) from the unrotated bubbles and runs the
// list-based exact search for kn frames.  tau/codes: (kn, n_sel, nd); the
// directions are rows of row_len (n_phi) consecutive patches.  ranges (device,
// n_sel, may be null): several realizations in one bubble array, slot s's
// colliders are rows [ranges[s].x, ranges[s].x + ranges[s].y) of each frame of
// n_tot rows and sel holds indices into the whole array.
void launch_mask_pipeline(Device* dev, const D4* bub_unrot, const D4* bub_frames, size_t n_int, size_t n_tot,
                          const uint32_t* sel, const uint2* ranges, size_t n_sel, const D4* dirs, size_t nd,
                          size_t row_len, size_t kn, double* tau, int32_t* codes, unsigned long long* counters,
                          bool build_lists, uint64_t* launches, int chunking = 1);

}  // namespace bgw
