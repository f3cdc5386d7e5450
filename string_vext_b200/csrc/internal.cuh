// Internal structures shared by the vext_b200 translation units.
//
// Data layout in HBM (per system = framework + guest):
//   frac   double [n_atoms][3]   wrapped fractional coordinates
//   type   int    [n_atoms]      index into the pair-parameter tables
//   tf     float4 [n_types]      (c12, c6, shift, floor2) in FP32
//   td     double [n_types][4]   the same in FP64 (reference arithmetic)
// Per region set (one grid size + block shape, or the pose bins):
//   info   RegionInfo [n_regions]
//   hi     float4 [entries]  (x, y, z) of an image relative to the region
//                            origin rounded to FP32; w = type id (int bits)
//   lo     float4 [entries]  residual (x - hi.x, ...) so hi + lo is the FP64
//                            relative position to ~1e-14 A
// Each region's entries are contiguous (info.off), "near" entries first:
// entries closer to the origin than r_split + max|offset| + rho are near,
// so every (site, image) pair nearer than r_split has a near entry.  Then
// the far inner entries, then the shell, whose last n_outer entries lie
// beyond rc + rho + 1e-3 A of the origin.
#pragma once

#include <mutex>
#include <vector>

#include "common.cuh"

namespace vext {

constexpr int kMaxTypes = 1024;     // distinct framework (sigma, epsilon) pairs
constexpr double kDefaultRSplit = 5.0;

struct alignas(16) RegionInfo {
    double of[3];       // origin, fractional
    double rho;         // max distance (A) from the origin to any pose center
    long long off;      // first entry
    int n_near;         // near entries
    int n_total;        // all entries
    int i0, j0, k0;     // first grid center (field regions)
    int ni, nj, nk;     // grid centers per axis (field regions)
    int n_inner;        // far entries within the cutoff of every site of every pose of the
                        // region (they follow the near entries; the shell ones come last)
    int n_outer;        // the last shell entries: beyond rc + rho + 1e-3 A of the origin,
                        // hence beyond rc of every pose center of the region
};
static_assert(sizeof(RegionInfo) % 16 == 0, "RegionInfo must stay 16-byte aligned");

struct RegionSet {
    // key
    int size = 0, bi = 0, bj = 0, bk = 0;   // field regions (size > 0) or bins (size == 0)
    int nb[3] = {0, 0, 0};                  // bins per axis (pose regions)
    double bin_width = 0;                   // target bin width (A, pose regions)
    double r_split = 0;
    // data
    int n_regions = 0;
    int n_ri = 0, n_rj = 0, n_rk = 0;       // regions per axis
    long long n_entries = 0, n_near = 0, n_outer = 0;
    RegionInfo *d_info = nullptr;
    float4 *d_hi = nullptr, *d_lo = nullptr;
    std::vector<RegionInfo> h_info;
    long long capacity = 0;                 // allocated entries (hi and lo)
    bool stale = false;                     // rebuild before the next use
    float build_ms = 0;
    ~RegionSet();
};

// One system's view for the warp-per-pose kernel (posebatch.cu).
struct PoseBatchSys {
    Mat3 H, Hinv;
    double rc2;
    float rc2f;
    double off0, off1;
    int nb0, nb1, nb2;
    const RegionInfo *regs;
    const float4 *hi, *lo;
    const double *td;   // (c12, c6, shift, floor2) per type
    const float4 *tf;
};

struct System {
    int device = 0;
    Mat3 H, Hinv;
    double einv[3];        // |column k of Hinv| = 1 / lattice-plane spacing
    int n_atoms = 0, n_types = 0;
    double guest_sigma = 0, guest_epsilon = 0, offsets[2] = {0, 0}, cutoff = 0, temperature = 0;
    double max_offset = 0;
    // FNV-1a hash of the framework as the region lists see it (cell, cutoff,
    // wrapped fractional coordinates, type ids and the framework (sigma,
    // epsilon) of every type): systems with equal hashes differ only in the
    // guest, so one region-list set serves them all when it is built for the
    // largest site offset among them
    uint64_t frame_hash = 0;
    double *d_frac = nullptr;
    int *d_type = nullptr;
    float4 *d_tf = nullptr;
    double *d_td = nullptr;
    std::vector<double> h_td;  // n_types x 4
    std::vector<RegionSet *> sets;
    int *d_status = nullptr;   // device status word
    // scratch of the field path
    double *d_e64 = nullptr;
    size_t e64_cap = 0;
    int *d_refine = nullptr;   // [0] = count, then pose indices
    size_t refine_cap = 0;
    double *d_axes = nullptr;
    size_t axes_cap = 0;
    float *d_f32 = nullptr;        // host-output staging of the float32 field
    size_t f32_cap = 0;
    float *d_small = nullptr;      // marginal, 2 x site, grid
    size_t small_cap = 0;
    double *d_e64T = nullptr;      // [S^3][O] FP64 output staging
    size_t e64T_cap = 0;
    int *d_flags = nullptr;        // [0] non-finite count
    size_t flags_cap = 0;
    // scratch of the pose path
    void *d_pose_scratch = nullptr;
    size_t pose_scratch_cap = 0;
    double *d_pose_io = nullptr;     // host-pointer entry staging
    size_t pose_io_cap = 0;
    PoseBatchSys *d_pose_desc = nullptr;   // warp-per-pose path: device copy of h_pose_desc
    PoseBatchSys h_pose_desc;
    long long *d_pose_offsets = nullptr;
    cudaStream_t stream = nullptr;   // private stream for host-pointer entries
    cudaStream_t aux = nullptr;      // second stream: copy-back beside pair work
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    bool timed = false;              // ev[0..2] hold the last field call's kernel/epilogue
    bool list_timed = false;         // ev[3..4] hold the last list build
    bool split_timed = false;        // ev[5] separates the near and far kernels
    // cached one-system forward + adjoint batch (vext_field_adjoint_device and
    // vext_field_adjoint into page-locked buffers), keyed by grid size,
    // directors, options and the FP64 energy output; its float32 outputs are
    // retargeted per call
    vext_batch adj_batch = nullptr;
    int adj_size = 0;
    std::vector<double> adj_axes;
    double adj_key[4] = {0, 0, 0, 0};   // r_split, band_lo, band_hi, variant
    double *adj_energy64 = nullptr;
    float *d_g32 = nullptr;          // host-output staging of the float32 gradient
    size_t g32_cap = 0;
    // the host entry's batches (vext_field_adjoint): one per 32-director
    // block, each writing its contiguous slice of d_f32 / d_g32, so the copy
    // of one block overlaps the next block's pair work
    std::vector<vext_batch> host_parts;
    std::vector<cudaEvent_t> host_part_done;
    int host_size = 0;
    std::vector<double> host_axes;
    double host_key[4] = {0, 0, 0, 0};
    float *host_e = nullptr, *host_g = nullptr;
    std::mutex lock;
    void drop_adjoint_batch();   // both caches (they point into the region sets)
    void drop_host_parts();
    ~System();
};

// Batches (batch.cu); lock_systems = false when the caller holds the locks.
int batch_build(int n_systems, const vext_system *systems, int size, int n_axes,
                const double *axes, const vext_options *opt, float *const *outputs,
                float *const *gradients, double *const *outputs_f64, bool lock_systems,
                vext_batch *out);
int batch_replay(vext_batch b, cudaStream_t stream);
int batch_retarget(vext_batch b, int k, float *out, float *grad, cudaStream_t stream);

// Region sets (system.cu)
int get_field_regions(System *sys, int size, int cb, double r_split, RegionSet **out,
                      cudaStream_t stream);
constexpr double kBinWidth = 0.75;  // pose-bin width between lattice planes (A)
int get_bin_regions(System *sys, double r_split, RegionSet **out, cudaStream_t stream,
                    double bin_width = kBinWidth);
void choose_block_shape(const Mat3 &H, int size, int cb, int &bi, int &bj, int &bk);
double block_radius(const Mat3 &H, int size, int ni, int nj, int nk);

// Device buffer growth helper
template <typename T>
int ensure_capacity(T *&ptr, size_t &cap, size_t need) {
    if (need <= cap && ptr) return 0;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t n = need < 1 ? 1 : need;
    cudaError_t err = cudaMalloc((void **)&ptr, n * sizeof(T));
    if (err != cudaSuccess)
        return fail(VEXT_ERR_MEMORY, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T),
                    cudaGetErrorString(err));
    cap = n;
    return 0;
}

int check_status(System *sys, cudaStream_t stream);  // reads and clears the status word


struct Options {
    int mode;
    double r_split;
    double band_lo, band_hi;
    int cb;
    int variant;
    int batch_shape;   // 0 = autotune, else 1 + kernel-table index
};
Options resolve_options(const vext_options *opt);

// |d0|^2 (entry - grid center) beyond which no site of a pose lies inside any
// type's contact floor: a site is at least |d0| - max|o| from the entry, so
// beyond sqrt(max floor2) + max|o| (with a relative margin far above FP64
// rounding) every pair skips the floor test without changing a bit.
inline double floor_clear_radius2(const System &sys) {
    double fl = 0.0;
    for (int t = 0; t < sys.n_types; ++t) fl = std::max(fl, sys.h_td[4 * t + 3]);
    const double rf =
        (std::sqrt(fl) + std::max(std::fabs(sys.offsets[0]), std::fabs(sys.offsets[1]))) *
            (1.0 + 1e-9) + 1e-9;
    return rf * rf;
}

// Directors per work item of a batch with these options (32 or 64; its
// regions hold 512 / that many grid centers).
int batch_item_directors(const Options &o, bool adjoint);

// Pose pipeline (pose.cu): enqueue without host synchronisation, then check.
int pose_enqueue(System *sys, int n, const double *centers, const double *quats,
                 const Options &o, double *energy, double *gc, double *gq, double *gu,
                 cudaStream_t st);
int pose_status(System *sys, cudaStream_t st);

// Warp-per-pose evaluation of n poses of one system on its bin lists `rs`
// (small batches, where the binned pipeline's per-bin CTAs would idle).
int pose_warp_enqueue(System *sys, const RegionSet *rs, int n, const double *centers,
                      const double *quats, const Options &o, double *energy, double *gc,
                      double *gq, double *gu, cudaStream_t st);

// Field kernel launcher (field.cu): computes E64 [O][S^3] for all regions.
int launch_field(System *sys, const RegionSet *rs, int n_axes, const double *d_axes,
                 double *d_e64, int cb, int variant, cudaStream_t stream);

}  // namespace vext

struct vext_system_s {
    vext::System sys;
};
