// GPU String path update: the reference String method (native/string/
// source_code/RC_main.cu:1914-2420, kernels global.h:1281-2244) with the
// finite-difference "forces" replaced by the analytic adjoint.
//
// A path is N images (fractional a, b, c; Euler alpha, beta, gamma in
// radians, R = Rz(gamma) Ry(beta) Rx(alpha), device_fxn.h:34-63).  One
// iteration:
//   1. energies E0 and the analytic gradient of s0 (pose pipeline, pose.cu);
//      the reference's one-sided difference g_k = E(x + h_k e_k) - E(x) is
//      replaced by its first-order value g_k = h_k dE/dx_k (h = delta_frac for
//      a, b, c and delta_angle for the angles; dE/dalpha = 0 exactly for a
//      two-site guest), truncated as floor(g / 1e-15) 1e-15 (global.h:1281-1325);
//      in the reference-difference mode the seven poses x, x + h_k e_k of
//      every image are evaluated instead (one pose launch of 7 n poses, in the
//      reference's variable order, remap_string_var, global.h:1141-1200) and
//      g_k = E_k - E_0 is truncated the same way;
//   2. step: per block (translation / rotation) L = |g| (truncated); if
//      L < h: s1 = s0 - h g, else s1 = s0 - h trunc(g / L) (global.h:1347-1450);
//   3. end fixing along the transport axis (global.h:1452-1620): image 0
//      keeps its axis coordinate, the last image keeps its axis coordinate and
//      copies the other five from image 0, interior images that left [0, 1]
//      along the axis copy the nearest image inside (read from the values
//      before fixing);
//   4. equal-arc-length reparametrisation of the positions in Cartesian
//      space; angles are carried over (global.h:1640-1790);
//   5. E2 = E(s2); where E2 > E0 the image keeps its old angles (check_s2);
//   6. angle smoothing with coefficient 1e-4 and the reference's 2 pi
//      branch rules (smooth_angle);
//   7. movement totals sum_i |s0_i - s2_i| (positions in fractional units,
//      angles), and every 200 iterations from iteration 200 on the
//      convergence test movement < 30 % x h x N x sqrt(3) for both blocks
//      (legacy_policy.h:9-12, RC_main.cu:1853-1854); on convergence the loop
//      stops before the copy;
//   8. s0 = (s2 positions, smoothed angles wrapped into [0, 2 pi]) (copy2s0).
// Steps 2-8 run in two single-CTA kernels (one thread per image); the two
// pose evaluations are the only heavy work.  One iteration is captured in a
// CUDA graph and replayed; the host reads the stop flag only at check
// iterations.
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace vext {

constexpr double kPi = 3.141592653589793;

struct StringArgs {
    Mat3 H;
    int n;
    int axis;             // transport axis 0, 1, 2 (direction - 1)
    double hf, ha;        // delta_frac, delta_angle (rad)
    double rounding;      // 1e-15
    double smooth;        // 1e-4
    double conv_t, conv_r;
    double *s0, *s1, *s2; // [n][6]
    double *e0, *e2;      // [n]
    double *gc, *gu;      // [n][3]
    double *centers, *quats, *centers2, *quats2;
    double *lengths;      // [n] segment lengths, then cumulative
    int *flags;           // [0] stop, [1] conv_t, [2] conv_r, [3] iterations done
    double *totals;       // [0] translation movement, [1] rotation movement
    int fd;               // reference one-sided differences instead of the adjoint
    double *centers7, *quats7, *e7;   // [7n] poses x, x + h_k e_k and their energies
};

__device__ __forceinline__ double trunc_r(double x, double r) { return floor(x / r) * r; }

__device__ __forceinline__ void pose_of(const StringArgs &a, const double *s, double *c,
                                        double *q) {
    frac_to_cart(a.H, s[0], s[1], s[2], c[0], c[1], c[2]);
    const double ca = cos(s[3] / 2), sa = sin(s[3] / 2), cb = cos(s[4] / 2), sb = sin(s[4] / 2),
                 cg = cos(s[5] / 2), sg = sin(s[5] / 2);
    q[0] = cg * cb * ca + sg * sb * sa;
    q[1] = cg * cb * sa - sg * sb * ca;
    q[2] = cg * sb * ca + sg * cb * sa;
    q[3] = sg * cb * ca - cg * sb * sa;
}

__global__ void string_to_pose_kernel(StringArgs a) {
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < a.n; i += blockDim.x * gridDim.x)
        pose_of(a, a.s0 + 6 * i, a.centers + 3 * i, a.quats + 4 * i);
}

// The seven poses of image i for the reference's differences: variable 0 is
// s0 itself, variable k = 1..6 adds h to coordinate k - 1 (delta_frac for
// a, b, c; delta_angle for alpha, beta, gamma).  The director of a two-site
// guest, R e_x = (cos g cos b, sin g cos b, -sin b), does not depend on
// alpha, so the poses are built with alpha = 0: E(x + h e_alpha) - E(x) is
// then exactly 0, as in the reference's own rotation.
__global__ void string_fd_pose_kernel(StringArgs a) {
    for (int v = threadIdx.x + blockIdx.x * blockDim.x; v < 7 * a.n;
         v += blockDim.x * gridDim.x) {
        const int i = v / 7, k = v % 7;
        double s[6];
        for (int c = 0; c < 6; ++c) s[c] = a.s0[6 * i + c];
        if (k >= 1) s[k - 1] += k <= 3 ? a.hf : a.ha;
        s[3] = 0.0;
        pose_of(a, s, a.centers7 + 3 * v, a.quats7 + 4 * v);
    }
}

// Steps 2-4 (and the pose of s2).  One CTA, thread i = image i (n <= 1024 =
// blockDim): the step in registers, end fixing and segment lengths through
// shared memory, the running sum of the lengths by one thread in image order.
__global__ void __launch_bounds__(1024) string_step_kernel(StringArgs a) {
    __shared__ double ax[1024];       // axis coordinate of every stepped image (before fixing)
    __shared__ double cum[1024];      // segment lengths, then their running sums
    __shared__ double cart[3][1024];  // Cartesian positions of the fixed images
    __shared__ double pre0[6];        // image 0 before fixing
    if (a.flags[0]) return;   // converged earlier (uniform over the CTA)
    const int n = a.n, d = a.axis, i = threadIdx.x;
    double o[6];
    if (i < n) {
        const double *s = a.s0 + 6 * i;
        double g[6];
        if (a.fd) {
            // s0_grad_cal, global.h:1281-1300: E(var k) - E(var 0)
            const double *e7 = a.e7 + 7 * i;
            for (int k = 0; k < 6; ++k) g[k] = e7[k + 1] - e7[0];
            a.e0[i] = e7[0];
        } else {
            // dE/dfrac_k = sum_j H[k][j] dE/dcart_j
            for (int k = 0; k < 3; ++k)
                g[k] = a.hf * (a.H.m[3 * k] * a.gc[3 * i] + a.H.m[3 * k + 1] * a.gc[3 * i + 1] +
                               a.H.m[3 * k + 2] * a.gc[3 * i + 2]);
            // director u = (cg cb, sg cb, -sb); dE/dalpha = 0 for a linear guest
            const double cb = cos(s[4]), sb = sin(s[4]), cg = cos(s[5]), sg = sin(s[5]);
            const double *gu = a.gu + 3 * i;
            g[3] = 0.0;
            g[4] = a.ha * (gu[0] * (-cg * sb) + gu[1] * (-sg * sb) + gu[2] * (-cb));
            g[5] = a.ha * (gu[0] * (-sg * cb) + gu[1] * (cg * cb));
        }
        for (int k = 0; k < 6; ++k) g[k] = trunc_r(g[k], a.rounding);
        const double lt = trunc_r(sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]), a.rounding);
        const double lr = trunc_r(sqrt(g[3] * g[3] + g[4] * g[4] + g[5] * g[5]), a.rounding);
        for (int k = 0; k < 3; ++k)
            o[k] = lt < a.hf ? s[k] - a.hf * g[k] : s[k] - a.hf * trunc_r(g[k] / lt, a.rounding);
        for (int k = 3; k < 6; ++k)
            o[k] = lr < a.ha ? s[k] - a.ha * g[k] : s[k] - a.ha * trunc_r(g[k] / lr, a.rounding);
        // the values before fixing (s2), read by the images that copy them
        for (int k = 0; k < 6; ++k) a.s2[6 * i + k] = o[k];
        ax[i] = o[d];
        if (i == 0)
            for (int k = 0; k < 6; ++k) pre0[k] = o[k];
    }
    __syncthreads();
    if (i < n) {
        // end fixing: image 0 keeps its axis coordinate; the last image keeps
        // its axis coordinate and takes the other five from image 0; an
        // interior image outside [0, 1] along the axis copies the nearest
        // image inside (values before fixing)
        if (i == 0) {
            o[d] = a.s0[d];
        } else if (i == n - 1) {
            for (int k = 0; k < 6; ++k) o[k] = k == d ? a.s0[6 * (n - 1) + d] : pre0[k];
        } else {
            const double v = ax[i];
            int src = -1;
            if (v < 0) {
                for (int ii = i + 1; ii < n; ++ii)
                    if (ax[ii] > 0) {
                        src = ii;
                        break;
                    }
            } else if (v > 1) {
                for (int ii = i - 1; ii >= 0; --ii)
                    if (ax[ii] < 1) {
                        src = ii;
                        break;
                    }
            }
            if (src >= 0)
                for (int k = 0; k < 6; ++k) o[k] = a.s2[6 * src + k];
        }
        for (int k = 0; k < 6; ++k) a.s1[6 * i + k] = o[k];
        frac_to_cart(a.H, o[0], o[1], o[2], cart[0][i], cart[1][i], cart[2][i]);
    }
    __syncthreads();
    if (i < n && i > 0) {
        const double dx = cart[0][i] - cart[0][i - 1], dy = cart[1][i] - cart[1][i - 1],
                     dz = cart[2][i] - cart[2][i - 1];
        cum[i] = sqrt(dx * dx + dy * dy + dz * dz);
    }
    __syncthreads();
    if (i == 0) {   // running sum in image order
        double c = 0;
        cum[0] = 0;
        for (int k = 1; k < n; ++k) {
            c += cum[k];
            cum[k] = c;
        }
    }
    __syncthreads();
    if (i < n) {   // (s2 is read above only, three barriers back: rewrite it now)
        const double L = cum[n - 1];
        const double t = (double)i / (n - 1);
        // segment ii with cum[ii]/L <= t <= cum[ii+1]/L (binary search)
        int lo = 0, hi = n - 2;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (cum[mid] / L <= t) lo = mid;
            else hi = mid - 1;
        }
        const int ii = lo;
        const double l0 = cum[ii] / L, l1 = cum[ii + 1] / L;
        double *out = a.s2 + 6 * i;
        const double *p0 = a.s1 + 6 * ii, *p1 = a.s1 + 6 * (ii + 1);
        for (int k = 0; k < 3; ++k)
            out[k] = l1 > l0 ? p0[k] + (t - l0) * ((p1[k] - p0[k]) / (l1 - l0)) : p0[k];
        for (int k = 3; k < 6; ++k) out[k] = o[k];
        pose_of(a, out, a.centers2 + 3 * i, a.quats2 + 4 * i);
    }
}

__device__ __forceinline__ double smooth_one(double prev, double cur, double next, double k) {
    const double dp = prev - cur, dn = next - cur;
    double wrap = 0.0;   // the branch table of smooth_angle, global.h:1835-1905
    if (dp > kPi) wrap = dn > kPi ? -2 * 2 * kPi : -1 * 2 * kPi;
    else if (dp < -kPi) wrap = dn < -kPi ? 2 * 2 * kPi : 0.0;
    else if (dn > kPi) wrap = -1 * 2 * kPi;
    else if (dn < -kPi) wrap = 1 * 2 * kPi;
    return (1 - k) * cur + 0.5 * k * (prev + next + wrap);
}

// Steps 5-8.  One CTA.  check != 0 on convergence-test iterations.
__global__ void string_finish_kernel(StringArgs a, int check) {
    if (a.flags[0]) return;
    const int n = a.n;
    __shared__ double red[2][1024];
    double mt = 0, mr = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double *s2 = a.s2 + 6 * i;
        const double *s0 = a.s0 + 6 * i;
        if (a.e2[i] > a.e0[i])
            for (int k = 3; k < 6; ++k) s2[k] = s0[k];
        double dt = 0, dr = 0;
        for (int k = 0; k < 3; ++k) dt += (s0[k] - s2[k]) * (s0[k] - s2[k]);
        for (int k = 3; k < 6; ++k) dr += (s0[k] - s2[k]) * (s0[k] - s2[k]);
        mt += sqrt(dt);
        mr += sqrt(dr);
    }
    red[0][threadIdx.x] = mt;
    red[1][threadIdx.x] = mr;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0, r = 0;
        for (int k = 0; k < min(n, (int)blockDim.x); ++k) {   // (the other threads hold 0)
            t += red[0][k];
            r += red[1][k];
        }
        a.totals[0] = t;
        a.totals[1] = r;
        const int ct = isfinite(t) && t >= 0 && a.conv_t > 0 && t < a.conv_t;
        const int cr = isfinite(r) && r >= 0 && a.conv_r > 0 && r < a.conv_r;
        a.flags[1] = ct;
        a.flags[2] = cr;
        if (check && ct && cr) a.flags[0] = 1;
        else a.flags[3] += 1;
    }
    __syncthreads();
    if (a.flags[0]) return;
    // smoothing reads s2 (checked angles) and writes the new s0
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double *s0 = a.s1 + 6 * i;   // s1 is free now: build the new path there
        const double *s2 = a.s2 + 6 * i;
        for (int k = 0; k < 3; ++k) s0[k] = s2[k];
        for (int k = 3; k < 6; ++k) {
            double v = (i == 0 || i == n - 1)
                           ? s2[k]
                           : smooth_one(a.s2[6 * (i - 1) + k], s2[k], a.s2[6 * (i + 1) + k],
                                        a.smooth);
            if (v > 2 * kPi) v -= 2 * kPi;
            else if (v < 0) v += 2 * kPi;
            s0[k] = v;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 6 * n; k += blockDim.x) a.s0[k] = a.s1[k];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        pose_of(a, a.s0 + 6 * i, a.centers + 3 * i, a.quats + 4 * i);
}

}  // namespace vext

using namespace vext;

extern "C" void vext_string_default_params(vext_string_params *p) {
    p->direction = 1;
    p->delta_frac = 1e-4;
    p->delta_angle_rad = kPi / 180;
    p->smooth = 1e-4;
    p->rounding = 1e-15;
    p->conv_trans_percent = 30;
    p->conv_rot_percent = 30;
    p->max_iterations = 10000;
    p->check_every = 200;
    p->gradient = VEXT_STRING_ANALYTIC;
}

extern "C" int vext_string_run(vext_system h, int n, double *path, double *energy,
                               const vext_string_params *params, const vext_options *opt,
                               vext_string_result *result) {
    if (!h || !path || n < 2 || n > 1024) return fail(VEXT_ERR_ARGUMENT, "2 <= images <= 1024 and a path required");
    vext_string_params p;
    vext_string_default_params(&p);
    if (params) p = *params;
    if (p.direction < 1 || p.direction > 3 || !(p.delta_frac > 0) || !(p.delta_angle_rad > 0) ||
        p.max_iterations < 0 || p.check_every < 1 ||
        (p.gradient != VEXT_STRING_ANALYTIC && p.gradient != VEXT_STRING_REFERENCE_FD))
        return fail(VEXT_ERR_ARGUMENT, "invalid String parameters");
    for (int k = 0; k < 6 * n; ++k)
        if (!std::isfinite(path[k])) return fail(VEXT_ERR_ARGUMENT, "non-finite path");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    Options o = resolve_options(opt);
    if (o.mode != VEXT_MODE_MIXED && o.mode != VEXT_MODE_FP64)
        return fail(VEXT_ERR_ARGUMENT, "unknown precision mode %d", o.mode);
    cudaStream_t st = sys->stream;
    double *buf = nullptr;
    const size_t nd = (size_t)n;
    // s0 s1 s2 (6n each), e0 e2 lengths totals (n each), gc gu centers
    // centers2 (3n each), quats quats2 (4n each), centers7 quats7 e7 (21n,
    // 28n, 7n)
    const size_t words = 3 * 6 * nd + 4 * nd + 4 * 3 * nd + 2 * 4 * nd + 56 * nd;
    VEXT_CUDA(cudaMalloc(&buf, sizeof(double) * words));
    int *flags = nullptr;
    cudaError_t e = cudaMalloc(&flags, sizeof(int) * 8);
    if (e != cudaSuccess) {
        cudaFree(buf);
        return fail(VEXT_ERR_MEMORY, "cudaMalloc failed");
    }
    StringArgs a;
    a.H = sys->H;
    a.n = n;
    a.axis = p.direction - 1;
    a.hf = p.delta_frac;
    a.ha = p.delta_angle_rad;
    a.rounding = p.rounding;
    a.smooth = p.smooth;
    a.conv_t = p.conv_trans_percent / 100 * p.delta_frac * n * std::sqrt(3.0);
    a.conv_r = p.conv_rot_percent / 100 * p.delta_angle_rad * n * std::sqrt(3.0);
    double *q = buf;
    a.s0 = q; q += 6 * nd;
    a.s1 = q; q += 6 * nd;
    a.s2 = q; q += 6 * nd;
    a.e0 = q; q += nd;
    a.e2 = q; q += nd;
    a.lengths = q; q += nd;
    a.totals = q; q += nd;   // (2 used)
    a.gc = q; q += 3 * nd;
    a.gu = q; q += 3 * nd;
    a.centers = q; q += 3 * nd;
    a.quats = q; q += 4 * nd;
    a.centers2 = q; q += 3 * nd;
    a.quats2 = q; q += 4 * nd;
    a.centers7 = q; q += 21 * nd;
    a.quats7 = q; q += 28 * nd;
    a.e7 = q; q += 7 * nd;
    a.fd = p.gradient == VEXT_STRING_REFERENCE_FD;
    if ((size_t)(q - buf) != words) {   // the carve-out must match the allocation exactly
        cudaFree(buf);
        cudaFree(flags);
        return fail(VEXT_ERR_CAPACITY, "String workspace layout mismatch");
    }
    a.flags = flags;
    int rc = 0;
    auto run = [&]() -> int {
        VEXT_CUDA(cudaMemcpyAsync(a.s0, path, sizeof(double) * 6 * nd, cudaMemcpyHostToDevice, st));
        VEXT_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 8, st));
        string_to_pose_kernel<<<1, 256, 0, st>>>(a);
        VEXT_CUDA(cudaGetLastError());
        // one iteration = two pose evaluations + two single-CTA kernels
        auto iteration = [&](int check) -> int {
            if (a.fd) {
                string_fd_pose_kernel<<<(7 * n + 255) / 256, 256, 0, st>>>(a);
                VEXT_CUDA(cudaGetLastError());
                VEXT_TRY(pose_enqueue(sys, 7 * n, a.centers7, a.quats7, o, a.e7, nullptr, nullptr,
                                      nullptr, st));
            } else {
                VEXT_TRY(pose_enqueue(sys, n, a.centers, a.quats, o, a.e0, a.gc, nullptr, a.gu,
                                      st));
            }
            string_step_kernel<<<1, 1024, 0, st>>>(a);
            VEXT_CUDA(cudaGetLastError());
            VEXT_TRY(pose_enqueue(sys, n, a.centers2, a.quats2, o, a.e2, nullptr, nullptr,
                                  nullptr, st));
            string_finish_kernel<<<1, 1024, 0, st>>>(a, check);
            VEXT_CUDA(cudaGetLastError());
            return 0;
        };
        // first iteration eagerly (builds lists and scratch), then graphs
        int it = 0;
        if (p.max_iterations > 0) {
            VEXT_TRY(iteration(0));
            VEXT_TRY(pose_status(sys, st));
            it = 1;
        }
        cudaGraphExec_t plain = nullptr, checked = nullptr;
        for (int variant = 0; variant < 2 && p.max_iterations > 1; ++variant) {
            cudaGraph_t g = nullptr;
            VEXT_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const int irc = iteration(variant);
            const cudaError_t end = cudaStreamEndCapture(st, &g);
            if (irc) {
                if (g) cudaGraphDestroy(g);
                return irc;
            }
            VEXT_CUDA(end);
            cudaGraphExec_t ex = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            VEXT_CUDA(ie);
            (variant ? checked : plain) = ex;
        }
        int stop = 0;
        for (; it < p.max_iterations && !stop; ++it) {
            const bool check = it % p.check_every == 0 && it >= p.check_every;
            VEXT_CUDA(cudaGraphLaunch(check ? checked : plain, st));
            if (check) {
                VEXT_CUDA(cudaMemcpyAsync(&stop, flags, sizeof(int), cudaMemcpyDeviceToHost, st));
                VEXT_CUDA(cudaStreamSynchronize(st));
            }
        }
        if (plain) cudaGraphExecDestroy(plain);
        if (checked) cudaGraphExecDestroy(checked);
        // final energies of the path in s0
        string_to_pose_kernel<<<1, 256, 0, st>>>(a);
        VEXT_CUDA(cudaGetLastError());
        VEXT_TRY(pose_enqueue(sys, n, a.centers, a.quats, o, a.e0, nullptr, nullptr, nullptr, st));
        VEXT_CUDA(cudaMemcpyAsync(path, a.s0, sizeof(double) * 6 * nd, cudaMemcpyDeviceToHost, st));
        if (energy) VEXT_CUDA(cudaMemcpyAsync(energy, a.e0, sizeof(double) * nd, cudaMemcpyDeviceToHost, st));
        int hf[4] = {0, 0, 0, 0};
        double ht[2] = {0, 0};
        VEXT_CUDA(cudaMemcpyAsync(hf, flags, sizeof hf, cudaMemcpyDeviceToHost, st));
        VEXT_CUDA(cudaMemcpyAsync(ht, a.totals, sizeof ht, cudaMemcpyDeviceToHost, st));
        VEXT_TRY(pose_status(sys, st));
        if (result) {
            result->iterations = hf[0] ? it - 1 : it;
            result->converged = hf[1] && hf[2] && result->iterations >= p.check_every;
            result->converged_translation = hf[1];
            result->converged_rotation = hf[2];
            result->movement_translation = ht[0];
            result->movement_rotation = ht[1];
            result->threshold_translation = a.conv_t;
            result->threshold_rotation = a.conv_r;
        }
        return 0;
    };
    rc = run();
    cudaStreamSynchronize(st);
    cudaFree(buf);
    cudaFree(flags);
    return rc;
}
