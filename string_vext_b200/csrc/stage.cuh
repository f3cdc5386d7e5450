// Chunked staging of one region's list into shared memory with 1-D bulk
// copies (TMA), STAGES-deep, one mbarrier per stage.  Near chunks bring
// hi + lo (FP64-exact positions), far chunks bring hi only.
//
// Chunk c of a region: near chunks first (entries [0, n_near) in kCH steps),
// then far chunks (entries [n_near, n_total)).  The barrier of a stage
// completes once per use; `seq` counts chunks over the CTA's lifetime so the
// phase parity stays right when one CTA processes several regions.
#pragma once

#include "internal.cuh"

namespace vext {

constexpr int kCH = 128;      // entries per chunk
constexpr int kStages = 4;    // pipeline depth (3: 1 % slower forward + adjoint)

struct ChunkPlan {
    long long off;
    int n_near, n_total, kn, n_chunks;

    __device__ __forceinline__ void init(const RegionInfo &r) {
        init_range(r.off, r.n_near, r.n_total);
    }
    // Entries [offset, offset + total) of which the first `near` are near.
    __device__ __forceinline__ void init_range(long long offset, int near, int total) {
        off = offset;
        n_near = near;
        n_total = total;
        kn = (n_near + kCH - 1) / kCH;
        n_chunks = kn + (n_total - n_near + kCH - 1) / kCH;
    }
    __device__ __forceinline__ void chunk(int c, int &start, int &len, bool &near) const {
        if (c < kn) {
            start = c * kCH;
            len = min(kCH, n_near - start);
            near = true;
        } else {
            start = n_near + (c - kn) * kCH;
            len = min(kCH, n_total - start);
            near = false;
        }
    }
};

struct Stager {
    uint64_t *bar;   // [kStages]
    float4 *hib;     // [kStages][kCH]
    float4 *lob;     // [kStages][kCH]

    // Single thread: arm stage (seq % kStages) and launch the copies of chunk c.
    __device__ __forceinline__ void issue(const ChunkPlan &p, const float4 *hi, const float4 *lo,
                                          int c, unsigned seq) const {
        int start, len;
        bool near;
        p.chunk(c, start, len, near);
        const int s = seq % kStages;
        const uint32_t bytes = (uint32_t)len * 16u;
        mbar_arrive_expect_tx(&bar[s], near ? 2 * bytes : bytes);
        bulk_g2s(hib + s * kCH, hi + p.off + start, bytes, &bar[s]);
        if (near) bulk_g2s(lob + s * kCH, lo + p.off + start, bytes, &bar[s]);
    }
};

// Shared-memory bytes of the staging buffers + barriers.
constexpr size_t kStageBytes = 64 + 2 * (size_t)kStages * kCH * sizeof(float4);

}  // namespace vext
