// The drop-in CSR pair kernel (dropin.cu), shared with the entry point in
// noalloc.cu that runs the same kernel on statically allocated scratch.
#pragma once

#include "internal.cuh"

namespace vext {

constexpr int kCsrChunk = 256;   // neighbours staged per shared-memory chunk

// Per-image record on the device: x, y, z, c12, c6, shift, floor2, pad.
struct CsrArgs {
    int n_centers, n_axes;
    double cutoff2;
    const double *centers;   // [n][3]
    const double *axes;      // [n_axes][3]
    const double *images8;   // [n_images][8]
    double off0, off1;
    const long long *starts; // rebased to 0, [n + 1]
    const int *indices;      // [nnz]
    double *out;             // [n][n_axes]
};

// One CTA per center; defined in dropin.cu.
__global__ void csr_kernel(CsrArgs a);

}  // namespace vext
