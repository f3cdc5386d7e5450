/*
 * vext_b200 -- B200 (sm_100a) engine for the exact two-identical-site
 * Lennard-Jones guest energy in a full triclinic periodic cell.
 *
 * C ABI only: plain pointers and sizes, no C++ or torch types.  Every entry
 * returns 0 on success or a nonzero status; vext_last_error() gives a
 * message for the calling thread's last failure.
 *
 * Units: Angstrom, Kelvin.  Cells are row-vector matrices (Cartesian =
 * fractional @ cell, row k = lattice vector k), exactly the `cell` array of
 * the reference's case dictionary (src/string_vext/cell.py:7-29).
 */
#ifndef VEXT_B200_H
#define VEXT_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define VEXT_API __attribute__((visibility("default")))
#else
#define VEXT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1-4 are the reference kernel's own codes
 * (native/vext/kernel.cpp:11-41); 16 and above are new. */
enum {
    VEXT_OK = 0,
    VEXT_ERR_SIZES = 1,          /* bad sizes / cutoff                          */
    VEXT_ERR_STARTS = 2,         /* CSR starts decreasing (or negative)         */
    VEXT_ERR_INDEX = 3,          /* CSR neighbour index outside [0, n_images)   */
    VEXT_ERR_NONFINITE = 4,      /* non-finite energy                           */
    VEXT_ERR_CUDA = 16,          /* CUDA runtime error (message has details)    */
    VEXT_ERR_TIMEOUT = 17,       /* a bounded device wait gave up               */
    VEXT_ERR_ARGUMENT = 18,      /* invalid argument to a new entry point       */
    VEXT_ERR_CAPACITY = 19,      /* a documented size limit was exceeded        */
    VEXT_ERR_MEMORY = 20         /* device or host allocation failed            */
};

/* ------------------------------------------------------------------------ */
/* Drop-in replacement of the reference CPU kernel.
 *
 * Replaces `evaluate_reused_neighbors` of native/vext/kernel.cpp:5-10, bound
 * by ctypes in src/string_vext/native.py:18-22 (argtypes 3 x c_int, c_double,
 * 11 x c_void_p; restype c_int) and called per 512-center batch at
 * native.py:60-64.  Same arguments, same meaning (all HOST buffers, the
 * output written in place as [center][axis] FP64), same return codes 0-4.
 * The sum runs on the current CUDA device in FP64 with the reference's
 * operation order and no contraction, so outputs are bit-identical to the
 * reference kernel's.  Codes 2 and 3 are checked on the host before any
 * device work, in the reference's order; a negative starts[0] is reported as
 * code 2.  Images and per-image coefficients are cached on the device
 * between calls and re-uploaded whenever their contents change. */
VEXT_API int evaluate_reused_neighbors(int n_centers, int n_axes, int n_images, double cutoff2,
                              const double *centers, const double *axes, const double *images,
                              const double *offsets, const double *coeff12, const double *coeff6,
                              const double *shift, const double *floor2, const int64_t *starts,
                              const int32_t *indices, double *output);

/* The same pair sum for callers that cannot allocate device memory:
 * plug-ins whose host runtime owns the GPU memory budget and allows no
 * allocations of their own (fixed-pool servers, MPS clients with hard memory
 * limits), real-time loops that cannot afford an allocation's implicit
 * synchronisation.  It has no counterpart in the reference.  Same arguments,
 * host buffers, codes and bit-identical output as evaluate_reused_neighbors,
 * but it calls no cudaMalloc/cudaFree/cudaMallocHost and uses no host heap:
 * its scratch is one 64 MiB device array compiled into the library (held by
 * every GPU that loads it until exit).  Batches needing more than 64 MiB of
 * scratch (about 120 B per image + 4 B per neighbour index + 8 B per output
 * pose) return VEXT_ERR_CAPACITY before anything is copied to the device.
 * The first call on each device loads the library's module there; every
 * call looks the array's device address up with cudaGetSymbolAddress.  Work
 * runs eagerly on the calling thread's per-thread default stream and is
 * finished when the call returns (it synchronises that stream, so it is not
 * to be called while that stream is being captured); calls are serialised
 * inside the process.  The array
 * keeps the last call's contents, and calls that overlapped on the GPU would
 * race on it. */
VEXT_API int evaluate_reused_neighbors_noalloc(int n_centers, int n_axes, int n_images,
                                               double cutoff2, const double *centers,
                                               const double *axes, const double *images,
                                               const double *offsets, const double *coeff12,
                                               const double *coeff6, const double *shift,
                                               const double *floor2, const int64_t *starts,
                                               const int32_t *indices, double *output);

/* Message describing the calling thread's last nonzero status. */
VEXT_API const char *vext_last_error(void);

/* ------------------------------------------------------------------------ */
/* Systems: one framework + one symmetric two-site guest, resident on the
 * current device.  Replaces the per-call set-up of ReusePotential /
 * TriclinicSitePotential (src/string_vext/neighbor.py:10-30,
 * physics.py:43-57): Lorentz-Berthelot mixing, coefficients
 * c12 = 4 eps sigma^12, c6 = 4 eps sigma^6, shift = -4 eps ((sigma/rc)^12 -
 * (sigma/rc)^6), floor2 = (0.1 sigma)^2, every lattice image within the
 * cutoff (never minimum image). */
typedef struct vext_system_s *vext_system;

typedef struct {
    double cell[9];          /* row-vector cell                              */
    int n_atoms;             /* framework atoms (>= 1)                        */
    const double *frac;      /* n_atoms x 3 fractional (wrapped mod 1 inside) */
    const double *sigma;     /* n_atoms framework sigma (A)                   */
    const double *epsilon;   /* n_atoms framework epsilon/kB (K)              */
    double guest_sigma;      /* both guest sites (identical)                  */
    double guest_epsilon;
    double offsets[2];       /* signed site offsets along the director (A)    */
    double cutoff;           /* LJ cutoff rc (A)                              */
    double temperature;      /* K, for the marginal field                     */
} vext_system_desc;

VEXT_API int vext_system_create(const vext_system_desc *desc, vext_system *out);
VEXT_API int vext_system_destroy(vext_system sys);

/* Mark every cached region list of the system stale: the next call rebuilds
 * it (into the same device allocation when it still fits). */
VEXT_API int vext_system_invalidate(vext_system sys);

/* Device times (CUDA events on the launching stream), in ms, of the
 * system's most recent list build and of the most recent field call's near
 * (FP64) pair kernel, far (FP32) pair kernel and epilogue; waits for those
 * events.  list_ms is 0 if no list was built since the previous query; in
 * the FP64 modes near_ms is the whole pair kernel and far_ms 0. */
VEXT_API int vext_last_timings(vext_system sys, double *list_ms, double *near_ms,
                               double *far_ms, double *epilogue_ms);

/* Precision modes. */
enum {
    VEXT_MODE_MIXED = 0,     /* FP64 for pairs nearer than r_split, FP32 beyond,
                                FP64 re-evaluation of poses whose energy lies in
                                the refinement band                           */
    VEXT_MODE_FP64 = 1,      /* every pair in FP64 (the GPU oracle kernel)     */
    VEXT_MODE_FP64_PLAIN = 2,/* fields only: the plain FP64 baseline kernel
                                (one thread per pose, no staging)            */
    VEXT_MODE_FP32_NAIVE = 3 /* fields only, precision study: the same plain
                                loop in FP32 (FP32 positions, IEEE FP32
                                division, one FP32 sum per pose)             */
};

typedef struct {
    int mode;                /* VEXT_MODE_*                                   */
    double r_split;          /* A; <= 0 selects the default (5 A)             */
    double band_lo, band_hi; /* refinement band for E (K); band_hi <= band_lo
                                disables refinement; defaults via
                                vext_default_options                          */
    int centers_per_region;  /* 16 or 32; 0 = default (16)                    */
    int variant;             /* 0 = default.  Forward + adjoint batches
                                (studies and checks): bit 32 / 64 the
                                reciprocal of q^3 with / without a Newton
                                step, 128 / 512 FP32 gradient partials over
                                16 / 64 entries, 1024 no cutoff-border test,
                                4096 re-evaluates poses with a shell pair
                                within 1.25e-4 A^2 of the cutoff wholly in
                                FP64 instead of re-testing only their shell
                                pairs; 8192 evaluates both sites of the
                                outer shell entries (beyond rc + the region
                                radius, where only one site of a director
                                can be inside; the sums then differ only
                                in FP32 rounding);
                                2048 see batch_shape.
                                Forward field:
                                9 runs the earlier far kernel (reciprocal of
                                q^3, every far entry masked)                  */
    int batch_shape;         /* batches: 1 + index of the CTA shape to run at
                                full occupancy instead of autotuning; 0 =
                                autotune (vext_batch_tuning lists the shapes);
                                the autotuner keeps its pick per size class
                                for the process, and variant bit 2048 makes a
                                batch time its candidates afresh             */
    int reserved[2];
} vext_options;

VEXT_API void vext_default_options(vext_options *opt);

/* Statistics of the last field call. */
typedef struct {
    int64_t poses;
    int64_t regions;
    int64_t list_entries;    /* sum of per-region list lengths                */
    int64_t near_entries;
    int64_t refined_poses;
    double list_build_ms, kernel_ms, epilogue_ms;  /* device time (events)   */
    int64_t outer_entries;   /* shell entries beyond rc + the region radius of
                                their region's origin (at most one site of a
                                director inside the cutoff)                   */
} vext_field_stats;

/* Full Vext field on a size^3 fractional grid (centers ((i+.5)/S, ...),
 * i slowest) x n_axes unit directors (HOST, n_axes x 3, as the reference
 * normalises them, src/string_vext/native.py:33-35).  Replaces
 * calculate_vext (src/string_vext/vext.py:21-43).  HOST outputs (any may be
 * NULL):
 *   orientation_K  float32 [n_axes][S][S][S]   (= E.T.reshape(O,S,S,S))
 *   energy_f64     double  [S^3][n_axes]       (the reference's FP64 array)
 *   marginal_K     float32 [S][S][S]  -T (logsumexp(-E/T) - log O)
 *   site_K         float32 [2][S][S][S]  site-0 single-site field, twice
 *   grid           float32 [S][S][S]  asinh(marginal_K / 1000)              */
VEXT_API int vext_field(vext_system sys, int size, int n_axes, const double *axes,
               const vext_options *opt, float *orientation_K, double *energy_f64,
               float *marginal_K, float *site_K, float *grid, vext_field_stats *stats);

/* Same, with DEVICE output pointers on the caller's stream (cudaStream_t
 * passed as void*; NULL = legacy default stream).  The call returns once the
 * work is enqueued and the region lists for (size, shape) exist. */
VEXT_API int vext_field_device(vext_system sys, int size, int n_axes, const double *axes_host,
                      const vext_options *opt, float *orientation_K, double *energy_f64,
                      float *marginal_K, float *site_K, float *grid, void *stream);

/* Forward + adjoint over the field poses: energy and gradient of every
 * (grid center, director) pose of the size^3 x n_axes field (same centers,
 * directors and [n_axes][S^3] pose order as vext_field).  DEVICE outputs on
 * `stream` (cudaStream_t as void*):
 *   energy        float32 [n_axes][S^3]     E, K
 *   gradient      float32 [n_axes][S^3][6]  dE/d(center) (K/A, Cartesian),
 *                                          then dE/du projected on the plane
 *                                          normal to u (K per unit director)
 *   energy_f64    double [n_axes][S^3]     the energies before float32 rounding
 *                                          (NULL to skip)
 *   gradient_f64  double [n_axes][S^3][6]  FP64 modes only (NULL to skip)
 * VEXT_MODE_MIXED runs the persistent batched kernel (FP64 near pairs, packed
 * FP32 far pairs with FP64-flushed partial sums, FP64 energy refinement band)
 * on a one-system batch that is built, autotuned and graph-captured on the
 * first call and replayed while (size, directors, options, outputs) stay the
 * same; VEXT_MODE_FP64 and VEXT_MODE_FP64_PLAIN run the plain one-thread-per-
 * pose FP64 kernel (IEEE division), the FP64 reference of the adjoint.  No
 * reference counterpart: the reference has no field gradient; its String
 * solver differentiates by forward differences
 * (native/string/source_code/global.h:1141-1325). */
VEXT_API int vext_field_adjoint_device(vext_system sys, int size, int n_axes,
                                       const double *axes_host, const vext_options *opt,
                                       float *energy, float *gradient, double *energy_f64,
                                       double *gradient_f64, void *stream);
/* Same with HOST float32 outputs (staged on the device, copied back before
 * the call returns).  In the mixed mode with more than 32 directors the poses
 * run as one batch per 32-director block and each block's outputs are copied
 * back while the next block computes. */
VEXT_API int vext_field_adjoint(vext_system sys, int size, int n_axes, const double *axes,
                                const vext_options *opt, float *energy, float *gradient);

/* ------------------------------------------------------------------------ */
/* Pose energies and the analytic adjoint for arbitrary poses.  A pose is a
 * Cartesian center (A) and a quaternion q = (w, x, y, z), used normalised;
 * the guest director is u = R(q) e_x and site s sits at center + o_s u.
 * Replaces the String energy kernels Vext_cal_s0 / Vext_s0_deri_cal and the
 * forward-difference gradient (native/string/source_code/global.h:1071-1128,
 * 1141-1325).  Pair terms are recomputed in the adjoint, never stored.
 * Outputs (any gradient pointer may be NULL):
 *   energy         double [n]
 *   grad_center    double [n][3]   dE/d(center), K/A
 *   grad_quat      double [n][4]   dE/dq of E(q/|q|): the gradient projected
 *                                  to the tangent space of the unit sphere
 *   grad_director  double [n][3]   dE/du, K/A (u held free of the unit constraint)
 * The *_device variant takes device pointers and a stream; the plain variant
 * host pointers. */
VEXT_API int vext_pose_energy_grad(vext_system sys, int n, const double *centers, const double *quats,
                          const vext_options *opt, double *energy, double *grad_center,
                          double *grad_quat, double *grad_director);
VEXT_API int vext_pose_energy_grad_device(vext_system sys, int n, const double *centers,
                                 const double *quats, const vext_options *opt, double *energy,
                                 double *grad_center, double *grad_quat, double *grad_director,
                                 void *stream);

/* ------------------------------------------------------------------------ */
/* GPU String path update.  Replaces the iteration loop of the reference
 * String solver (native/string/source_code/RC_main.cu:1914-2420 with the
 * kernels of global.h:1281-2244): per-block normalised steepest-descent step,
 * end fixing along the transport axis, equal-arc-length reparametrisation of
 * the positions, energy check of the new angles, angle smoothing, movement-
 * based convergence test every check_every iterations -- the same rules and
 * constants -- with the finite-difference forces replaced by h x the analytic
 * gradient (or, with params->gradient = VEXT_STRING_REFERENCE_FD, the
 * reference's own differences, which reproduce its path files).  path is HOST [n][6] (fractional a, b, c; Euler alpha, beta,
 * gamma in radians, R = Rz(gamma) Ry(beta) Rx(alpha)), updated in place;
 * energy (may be NULL) receives the final energies [n]. */
typedef struct {
    int direction;             /* transport axis 1 = a, 2 = b, 3 = c            */
    double delta_frac;         /* step / difference size in fractional units    */
    double delta_angle_rad;    /* angular step (reference: 1 degree)            */
    double smooth;             /* angle smoothing coefficient (1e-4)            */
    double rounding;           /* truncation quantum (1e-15)                    */
    double conv_trans_percent; /* convergence thresholds (30 %)                 */
    double conv_rot_percent;
    int max_iterations;        /* Running_steps                                 */
    int check_every;           /* convergence test period (200)                 */
    int gradient;              /* VEXT_STRING_ANALYTIC (default): h x the
                                  analytic gradient; VEXT_STRING_REFERENCE_FD:
                                  the reference's own one-sided differences
                                  E(x + h e_k) - E(x) (global.h:1141-1325),
                                  seven pose energies per image per iteration */
} vext_string_params;

enum { VEXT_STRING_ANALYTIC = 0, VEXT_STRING_REFERENCE_FD = 1 };

typedef struct {
    int iterations;            /* iterations run (the reference's i_time)       */
    int converged;             /* both blocks below threshold at a test         */
    int converged_translation, converged_rotation;
    double movement_translation, movement_rotation;   /* last iteration        */
    double threshold_translation, threshold_rotation;
} vext_string_result;

VEXT_API void vext_string_default_params(vext_string_params *params);
VEXT_API int vext_string_run(vext_system sys, int n_images, double *path, double *energy,
                             const vext_string_params *params, const vext_options *opt,
                             vext_string_result *result);

/* ------------------------------------------------------------------------ */
/* Transition-state-theory post-processing of a String path (host only).
 * frac [n][3] fractional image positions, energy [n] in K, cell the
 * row-vector cell matrix (3 x 3), hop_A the hopping length (the cell length
 * along the transport axis), temperature in K, mass in g/mol.
 *   vext_tst_diffusivity: the hopping diffusivity D0 (m^2/s) the String
 *     program prints: 0.5 L^2 sqrt(kT/(2 pi m)) exp(-Vmax/T) / trapz over
 *     the Cartesian arc length of exp(-V/T) (capped at exp(-600))
 *     (native/string/source_code/RC_main.cu:2485-2527; the standalone
 *     diffusivity.c:117-172 computes the same without the cap).
 *   vext_tst_log_score: log D with the shifted-energy trapezoid in log
 *     space; *valid = 0 for invalid inputs or a non-finite result
 *     (legacy_policy.h:21-49).  The reference keeps the initial path when its
 *     score is valid and higher than the final one's (legacy_policy.h:50-52). */
VEXT_API int vext_tst_diffusivity(int n, const double *frac, const double *energy,
                                  const double *cell, double hop_A, double temperature,
                                  double mass_g_mol, double *d0);
VEXT_API int vext_tst_log_score(int n, const double *frac, const double *energy,
                                const double *cell, double temperature, double mass_g_mol,
                                double hop_A, int *valid, double *log_d);

/* ------------------------------------------------------------------------ */
/* Batched fields: many systems (frameworks x guests of uneven sizes and cell
 * shapes) in one persistent launch over a work queue of (system, region,
 * 32-director block) items, longest first, captured in a CUDA graph.  The
 * CTA shape and resident-CTA count are autotuned at creation on a sample of
 * the queue.  outputs[k] is a DEVICE float32 field [n_axes][S^3] for
 * systems[k] (mixed precision, with FP64 re-evaluation of the refinement
 * band).  The systems must outlive the batch and must not be invalidated
 * while it exists.  No reference counterpart: the reference runs one field
 * per process (tests/cof/reference_project/graph_vext/cof8948_oldff_vext_exact.py). */
typedef struct vext_batch_s *vext_batch;

VEXT_API int vext_batch_create(int n_systems, const vext_system *systems, int size, int n_axes,
                               const double *axes, const vext_options *opt,
                               float *const *outputs, vext_batch *out);
/* Forward + adjoint batch: energies[k] as outputs above, gradients[k] a
 * DEVICE float32 [n_axes][S^3][6] array (dE/d(center), tangent dE/du; layout
 * of vext_field_adjoint_device).  Same queue, autotuning and graph. */
VEXT_API int vext_batch_create_adjoint(int n_systems, const vext_system *systems, int size,
                                       int n_axes, const double *axes, const vext_options *opt,
                                       float *const *energies, float *const *gradients,
                                       vext_batch *out);
/* Replay the captured graph on `stream` (NULL: the batch's own stream). */
VEXT_API int vext_batch_run(vext_batch batch, void *stream);
/* Wait for the device and report a timeout or a refinement-list overflow. */
VEXT_API int vext_batch_status(vext_batch batch);
VEXT_API int vext_batch_destroy(vext_batch batch);
VEXT_API int vext_batch_info(vext_batch batch, int64_t *work_items, int64_t *poses,
                             int64_t *list_bytes, int *shape, int *grid);
/* Poses the last replay re-evaluated in FP64 (energies in the refinement
 * band; for forward + adjoint batches also poses with a shell pair within
 * 1.25e-4 A^2 of the cutoff), after waiting for the device. */
VEXT_API int vext_batch_refined(vext_batch batch, int64_t *poses);
/* The autotuner's candidates (kernel shape index, resident CTAs, sample time
 * in ms, shape name: threads x directors per thread[/CTAs-per-SM bound]),
 * at most max_candidates of them; any output may be NULL. */
VEXT_API int vext_batch_tuning(vext_batch batch, int max_candidates, int *n_candidates,
                               int *shapes, int *grids, float *ms, const char **names);

/* ------------------------------------------------------------------------ */
/* Batched poses of many systems in ONE launch: the String paths of a batch of
 * frameworks x guests, forward + adjoint every iteration.  The poses of
 * systems[k] are rows [pose_offsets[k], pose_offsets[k+1]) (host array of
 * n_systems + 1 entries, pose_offsets[0] = 0) of the DEVICE arrays given to
 * vext_pose_batch_run: centers [n][3] Cartesian A, quats [n][4] (w, x, y, z);
 * outputs as vext_pose_energy_grad (energy [n], grad_center [n][3], tangent
 * grad_quat [n][4], grad_director [n][3], any may be NULL).  One warp per
 * pose over its bin list: FP64 near pairs, FP32 far pairs with FP64-flushed
 * partial sums, poses in the refinement band recomputed in FP64 (mixed mode;
 * VEXT_MODE_FP64 evaluates every pair in FP64).  Replaces the per-image
 * String energy kernels run once per path (global.h:1071-1128, 1141-1325);
 * no reference counterpart for the batching.  The systems must outlive the
 * batch and must not be invalidated while it exists. */
typedef struct vext_pose_batch_s *vext_pose_batch;

VEXT_API int vext_pose_batch_create(int n_systems, const vext_system *systems,
                                    const int64_t *pose_offsets, const vext_options *opt,
                                    vext_pose_batch *out);
VEXT_API int vext_pose_batch_run(vext_pose_batch batch, const double *centers,
                                 const double *quats, double *energy, double *grad_center,
                                 double *grad_quat, double *grad_director, void *stream);
/* Wait for the device; report a non-finite input or a device error. */
VEXT_API int vext_pose_batch_status(vext_pose_batch batch);
VEXT_API int vext_pose_batch_destroy(vext_pose_batch batch);

/* ------------------------------------------------------------------------ */
/* Diagnostics. */

/* Non-tensor FP32 FMA throughput of the current device (FLOP/s, FMA = 2),
 * measured by a register-resident FFMA chain kernel; iterations controls
 * the run length. */
VEXT_API int vext_measure_fp32_peak(int iterations, double *flops_per_second);

/* Measured throughput of the SIMT pipes the pair kernels use: scalar FFMA
 * (FMA/s), packed FFMA2 (FMA/s, two per lane per instruction) and the
 * hardware reciprocal (results/s); any pointer may be NULL. */
VEXT_API int vext_measure_pipes(int iterations, double *ffma_per_s, double *ffma2_fma_per_s,
                                double *rcp_per_s);

/* Exact FP64 number of (site, image) pairs closer than the cutoff over the
 * size^3 x n_axes field (the algorithmic unit of work); far_pairs (may be
 * NULL) receives those whose image is a far entry of the default 16-center
 * regions for the given r_split (<= 0: the default), i.e. the pairs the FP32
 * far kernel of the mixed field evaluates. */
VEXT_API int vext_count_pairs(vext_system sys, int size, int n_axes, const double *axes,
                              double r_split, int64_t *pairs, int64_t *far_pairs);

/* Exercises the device-wait timeout path: a kernel arms an mbarrier for a
 * copy that is never issued and waits on it through the same bounded wait
 * the staged pair kernels use, with `polls` (1 .. 2^22) as the limit.  Returns
 * VEXT_ERR_TIMEOUT with a message when the wait gives up (the expected
 * outcome); nothing is left in flight, so the device stays usable.  No
 * reference counterpart: the reference kernels have no device waits
 * (native/vext/kernel.cpp returns codes 1-4 only). */
VEXT_API int vext_check_wait_timeout(int polls);

/* Library version string. */
VEXT_API const char *vext_version(void);

#ifdef __cplusplus
}
#endif
#endif
