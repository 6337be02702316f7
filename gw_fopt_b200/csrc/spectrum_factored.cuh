// Factored spectrum kernels (FP64 and mixed precision).
#pragma once

#include "device_common.cuh"

namespace bgw {

// Launches the factored spectrum for kn frames whose masks are in `tau`;
// writes (kn, 2, S, W) complex sums into out.  Returns the number of kernel
// launches.
inline uint64_t launch_factored(Device*, const SpectrumJob& job, const D4*, const uint32_t*, const double*,
                                const double*, const double*, const double*, const double*, const double*,
                                const double*, const double*, const double*, size_t, double2*) {
    throw Error{"spectrum kernel " + std::to_string((int)job.kernel) + " is not built in this library"};
}

}  // namespace bgw
