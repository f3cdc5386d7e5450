/*
 * CPU FP64 oracle for the two-site Lennard-Jones pose energy -- TEST
 * INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and
 * only as the checker.
 *
 * Each function restates, in plain C, the arithmetic of one reference routine
 * (paths relative to the String_Vext project):
 *
 *   oracle_reused_neighbors   native/vext/kernel.cpp:5-45 (CSR pair sum, codes 0-4)
 *   oracle_site_energy        src/string_vext/physics.py:43-85 (TriclinicSitePotential:
 *                             image reach, wrap-to-cell, floored shifted LJ)
 *   oracle_pose_energy        src/string_vext/physics.py:88-106 (direct_pose_energy)
 *   oracle_pair_lj            native/string/source_code/triclinic_pair.h:14-68
 *   oracle_euler_pose_energy  native/string/source_code/global.h:1071-1128 with the
 *                             rotation of device_fxn.h:34-63 (R = Rz(g) Ry(b) Rx(a))
 *   oracle_pose_energy_grad   analytic dE/d(site) summed to dE/d(center) and the
 *                             director gradient (no reference counterpart; checked by
 *                             central differences of oracle_pose_energy in tests)
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- small 3x3 helpers (row-vector convention: cart = frac @ cell) ---- */

static void inverse3(const double *h, double *inv) {
    /* numpy.linalg.inv equivalent via the adjugate (FP64). */
    const double a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5],
                 g = h[6], k = h[7], l = h[8];
    const double det = a * (e * l - f * k) - b * (d * l - f * g) + c * (d * k - e * g);
    inv[0] = (e * l - f * k) / det; inv[1] = (c * k - b * l) / det; inv[2] = (b * f - c * e) / det;
    inv[3] = (f * g - d * l) / det; inv[4] = (a * l - c * g) / det; inv[5] = (c * d - a * f) / det;
    inv[6] = (d * k - e * g) / det; inv[7] = (b * g - a * k) / det; inv[8] = (a * e - b * d) / det;
}

static void row_times(const double *v, const double *m, double *out) {
    for (int j = 0; j < 3; ++j)
        out[j] = v[0] * m[j] + v[1] * m[3 + j] + v[2] * m[6 + j];
}

/* ------------------------------------------------------------------------ */
/* native/vext/kernel.cpp:5-45 -- same argument meaning and return codes.   */
/* Compiled without FP contraction so the sum matches the reference's own   */
/* separate multiply/add sequence.                                          */
int oracle_reused_neighbors(int n_centers, int n_axes, int n_images, double cutoff2,
                            const double *centers, const double *axes, const double *images,
                            const double *offsets, const double *coeff12, const double *coeff6,
                            const double *shift, const double *floor2, const int64_t *starts,
                            const int32_t *indices, double *output) {
    if (n_centers < 0 || n_axes < 1 || n_images < 1 || !(cutoff2 > 0)) return 1;
    for (int c = 0; c < n_centers; ++c) {
        const int64_t lo = starts[c], hi = starts[c + 1];
        if (lo > hi) return 2;
        for (int a = 0; a < n_axes; ++a) {
            double total = 0.0;
            for (int s = 0; s < 2; ++s) {
                double p[3];
                for (int k = 0; k < 3; ++k) p[k] = centers[3 * c + k] + offsets[s] * axes[3 * a + k];
                for (int64_t n = lo; n < hi; ++n) {
                    const int32_t j = indices[n];
                    if (j < 0 || j >= n_images) return 3;
                    const double dx = p[0] - images[3 * j], dy = p[1] - images[3 * j + 1],
                                 dz = p[2] - images[3 * j + 2];
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 >= cutoff2) continue;
                    const double s2 = r2 < floor2[j] ? floor2[j] : r2;
                    const double i2 = 1.0 / s2;
                    const double i6 = i2 * i2 * i2;
                    total += coeff12[j] * i6 * i6 - coeff6[j] * i6 + shift[j];
                }
            }
            if (!isfinite(total)) return 4;
            output[(int64_t)c * n_axes + a] = total;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Image set of TriclinicSitePotential (physics.py:43-57): spacing_k =      */
/* 1/|inv[:,k]|, reach_k = ceil(cutoff/spacing_k)+1, every shift in         */
/* [-reach, reach]^3 applied to the wrapped atoms.                          */
typedef struct {
    int n;            /* number of images */
    double *xyz;      /* n x 3 Cartesian */
    int *atom;        /* framework atom of each image */
} image_set;

static int build_images(const double *cell, int n_atoms, const double *frac, double cutoff,
                        image_set *out) {
    double inv[9];
    inverse3(cell, inv);
    int reach[3];
    for (int k = 0; k < 3; ++k) {
        const double norm = sqrt(inv[k] * inv[k] + inv[3 + k] * inv[3 + k] + inv[6 + k] * inv[6 + k]);
        reach[k] = (int)ceil(cutoff * norm) + 1;
    }
    const int64_t shifts = (int64_t)(2 * reach[0] + 1) * (2 * reach[1] + 1) * (2 * reach[2] + 1);
    const int64_t n = shifts * n_atoms;
    if (n > 400000000) return -1;
    out->n = (int)n;
    out->xyz = (double *)malloc(sizeof(double) * 3 * n);
    out->atom = (int *)malloc(sizeof(int) * n);
    if (!out->xyz || !out->atom) return -1;
    int64_t m = 0;
    for (int i = -reach[0]; i <= reach[0]; ++i)
        for (int j = -reach[1]; j <= reach[1]; ++j)
            for (int k = -reach[2]; k <= reach[2]; ++k)
                for (int t = 0; t < n_atoms; ++t) {
                    double f[3] = {frac[3 * t] - floor(frac[3 * t]) + i,
                                   frac[3 * t + 1] - floor(frac[3 * t + 1]) + j,
                                   frac[3 * t + 2] - floor(frac[3 * t + 2]) + k};
                    row_times(f, cell, out->xyz + 3 * m);
                    out->atom[m] = t;
                    ++m;
                }
    return 0;
}

static void free_images(image_set *s) {
    free(s->xyz);
    free(s->atom);
}

/* One wrapped Cartesian site against every image (physics.py:59-82):       */
/* r = |q - image|, ratio = (sigma/max(r, 0.1 sigma))^6,                    */
/* e = 4 eps (ratio^2 - ratio) - 4 eps ((sigma/rc)^12 - (sigma/rc)^6),      */
/* e = 0 where r >= rc.                                                     */
static double site_sum(const image_set *im, const double *q, const double *msig,
                       const double *meps, const double *mshift, double cutoff) {
    double total = 0.0;
    for (int m = 0; m < im->n; ++m) {
        const double dx = q[0] - im->xyz[3 * m], dy = q[1] - im->xyz[3 * m + 1],
                     dz = q[2] - im->xyz[3 * m + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (r >= cutoff) continue;
        const int t = im->atom[m];
        const double sig = msig[t];
        const double rr = r > 0.1 * sig ? r : 0.1 * sig;
        const double ratio = pow(sig / rr, 6);
        total += 4.0 * meps[t] * (ratio * ratio - ratio) + mshift[t];
    }
    return total;
}

static void wrap_cart(const double *cell, const double *inv, const double *p, double *q) {
    double f[3];
    row_times(p, inv, f);
    for (int k = 0; k < 3; ++k) f[k] -= floor(f[k]);
    row_times(f, cell, q);
}

static void mixed_params(int n_atoms, const double *sigma, const double *epsilon,
                         double guest_sigma, double guest_epsilon, double cutoff,
                         double *msig, double *meps, double *mshift) {
    for (int t = 0; t < n_atoms; ++t) {
        msig[t] = (sigma[t] + guest_sigma) / 2;
        meps[t] = sqrt(epsilon[t] * guest_epsilon);
        const double rc6 = pow(msig[t] / cutoff, 6);
        mshift[t] = -4 * meps[t] * (rc6 * rc6 - rc6);
    }
}

/* TriclinicSitePotential(case).evaluate(xyz, guest_sigma, guest_epsilon). */
int oracle_site_energy(const double *cell, int n_atoms, const double *frac, const double *sigma,
                       const double *epsilon, double guest_sigma, double guest_epsilon,
                       double cutoff, int n_query, const double *xyz, double *out) {
    image_set im;
    if (build_images(cell, n_atoms, frac, cutoff, &im)) return 1;
    double inv[9];
    inverse3(cell, inv);
    double *msig = malloc(sizeof(double) * 3 * n_atoms);
    double *meps = msig + n_atoms, *mshift = msig + 2 * n_atoms;
    mixed_params(n_atoms, sigma, epsilon, guest_sigma, guest_epsilon, cutoff, msig, meps, mshift);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n_query; ++i) {
        double q[3];
        wrap_cart(cell, inv, xyz + 3 * i, q);
        out[i] = site_sum(&im, q, msig, meps, mshift, cutoff);
    }
    free(msig);
    free_images(&im);
    return 0;
}

/* direct_pose_energy (physics.py:93-106): sites = frac_center @ cell +     */
/* offset_s * director (directors already unit length); E[c, a] summed over */
/* both sites; output row-major (n_centers, n_axes).                        */
int oracle_pose_energy(const double *cell, int n_atoms, const double *frac, const double *sigma,
                       const double *epsilon, double guest_sigma, double guest_epsilon,
                       const double *offsets, double cutoff, int n_centers,
                       const double *centers_frac, int n_axes, const double *axes, double *out) {
    image_set im;
    if (build_images(cell, n_atoms, frac, cutoff, &im)) return 1;
    double inv[9];
    inverse3(cell, inv);
    double *msig = malloc(sizeof(double) * 3 * n_atoms);
    double *meps = msig + n_atoms, *mshift = msig + 2 * n_atoms;
    mixed_params(n_atoms, sigma, epsilon, guest_sigma, guest_epsilon, cutoff, msig, meps, mshift);
    const int64_t total = (int64_t)n_centers * n_axes;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < total; ++p) {
        const int c = (int)(p / n_axes), a = (int)(p % n_axes);
        double center[3];
        row_times(centers_frac + 3 * c, cell, center);
        double e = 0.0;
        for (int s = 0; s < 2; ++s) {
            double site[3], q[3];
            for (int k = 0; k < 3; ++k) site[k] = center[k] + offsets[s] * axes[3 * a + k];
            wrap_cart(cell, inv, site, q);
            e += site_sum(&im, q, msig, meps, mshift, cutoff);
        }
        out[p] = e;
    }
    free(msig);
    free_images(&im);
    return 0;
}

/* Number of in-cutoff (site, image) pairs per pose -- the algorithmic unit */
/* of work.  Same image set and cutoff test as oracle_pose_energy.          */
int oracle_pair_counts(const double *cell, int n_atoms, const double *frac, const double *offsets,
                       double cutoff, int n_centers, const double *centers_frac, int n_axes,
                       const double *axes, int64_t *out) {
    image_set im;
    if (build_images(cell, n_atoms, frac, cutoff, &im)) return 1;
    double inv[9];
    inverse3(cell, inv);
    const int64_t total = (int64_t)n_centers * n_axes;
    const double c2 = cutoff * cutoff;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < total; ++p) {
        const int c = (int)(p / n_axes), a = (int)(p % n_axes);
        double center[3];
        row_times(centers_frac + 3 * c, cell, center);
        int64_t count = 0;
        for (int s = 0; s < 2; ++s) {
            double site[3], q[3];
            for (int k = 0; k < 3; ++k) site[k] = center[k] + offsets[s] * axes[3 * a + k];
            wrap_cart(cell, inv, site, q);
            for (int m = 0; m < im.n; ++m) {
                const double dx = q[0] - im.xyz[3 * m], dy = q[1] - im.xyz[3 * m + 1],
                             dz = q[2] - im.xyz[3 * m + 2];
                count += (dx * dx + dy * dy + dz * dz) < c2;
            }
        }
        out[p] = count;
    }
    free_images(&im);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Analytic FP64 energy and gradient of poses given as a Cartesian center  */
/* and a unit director.  Per site s at r_s = c + o_s u:                     */
/*   dE/dr_s = sum over pairs with r < rc and r > 0.1 sigma of             */
/*             -(48 eps sigma^12 / r^14 - 24 eps sigma^6 / r^8) (r_s - x)   */
/* (zero inside the floor, where the energy is constant), dE/dc = sum_s     */
/* dE/dr_s, dE/du = sum_s o_s dE/dr_s.  Outputs: energy (n), grad_center   */
/* (n x 3), grad_director (n x 3).                                          */
int oracle_pose_energy_grad(const double *cell, int n_atoms, const double *frac,
                            const double *sigma, const double *epsilon, double guest_sigma,
                            double guest_epsilon, const double *offsets, double cutoff, int n,
                            const double *centers_cart, const double *directors, double *energy,
                            double *grad_center, double *grad_director) {
    image_set im;
    if (build_images(cell, n_atoms, frac, cutoff, &im)) return 1;
    double inv[9];
    inverse3(cell, inv);
    double *msig = malloc(sizeof(double) * 3 * n_atoms);
    double *meps = msig + n_atoms, *mshift = msig + 2 * n_atoms;
    mixed_params(n_atoms, sigma, epsilon, guest_sigma, guest_epsilon, cutoff, msig, meps, mshift);
#pragma omp parallel for schedule(dynamic, 4)
    for (int p = 0; p < n; ++p) {
        double e = 0.0, gc[3] = {0, 0, 0}, gu[3] = {0, 0, 0};
        for (int s = 0; s < 2; ++s) {
            double site[3], q[3], g[3] = {0, 0, 0};
            for (int k = 0; k < 3; ++k) site[k] = centers_cart[3 * p + k] + offsets[s] * directors[3 * p + k];
            wrap_cart(cell, inv, site, q);
            for (int m = 0; m < im.n; ++m) {
                const double dx = q[0] - im.xyz[3 * m], dy = q[1] - im.xyz[3 * m + 1],
                             dz = q[2] - im.xyz[3 * m + 2];
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double r = sqrt(r2);
                if (r >= cutoff) continue;
                const int t = im.atom[m];
                const double sig = msig[t];
                const double rr = r > 0.1 * sig ? r : 0.1 * sig;
                const double ratio = pow(sig / rr, 6);
                e += 4.0 * meps[t] * (ratio * ratio - ratio) + mshift[t];
                if (r > 0.1 * sig) {
                    /* dE/d(r^2) = 4 eps (-6 ratio^2 + 3 ratio) / r^2 */
                    const double de = 4.0 * meps[t] * (-6.0 * ratio * ratio + 3.0 * ratio) / r2;
                    g[0] += 2 * de * dx; g[1] += 2 * de * dy; g[2] += 2 * de * dz;
                }
            }
            for (int k = 0; k < 3; ++k) {
                gc[k] += g[k];
                gu[k] += offsets[s] * g[k];
            }
        }
        energy[p] = e;
        for (int k = 0; k < 3; ++k) {
            grad_center[3 * p + k] = gc[k];
            grad_director[3 * p + k] = gu[k];
        }
    }
    free(msig);
    free_images(&im);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* triclinic_pair.h:14-68: one Cartesian site against every lattice image   */
/* of one framework atom (fractional fa, fb, fc).  A, B, C are the rows of  */
/* the fractional-to-Cartesian matrix in that header's convention, i.e.     */
/* x = A . (u, v, w): A = column 0 of the row-vector cell.                  */
double oracle_pair_lj(double x, double y, double z, double fa, double fb, double fc,
                      const double *A, const double *B, const double *C, double epsilon_guest,
                      double sigma_guest, double epsilon_frame, double sigma_frame, double cutoff) {
    const double det = A[0] * (B[1] * C[2] - B[2] * C[1]) - A[1] * (B[0] * C[2] - B[2] * C[0])
                       + A[2] * (B[0] * C[1] - B[1] * C[0]);
    if (!isfinite(det) || fabs(det) < 1e-12 || cutoff <= 0.0) return NAN;
    /* rows of the inverse map Cartesian -> fractional */
    const double ia[3] = {(B[1] * C[2] - B[2] * C[1]) / det, (A[2] * C[1] - A[1] * C[2]) / det,
                          (A[1] * B[2] - A[2] * B[1]) / det};
    const double ib[3] = {(B[2] * C[0] - B[0] * C[2]) / det, (A[0] * C[2] - A[2] * C[0]) / det,
                          (A[2] * B[0] - A[0] * B[2]) / det};
    const double ic[3] = {(B[0] * C[1] - B[1] * C[0]) / det, (A[1] * C[0] - A[0] * C[1]) / det,
                          (A[0] * B[1] - A[1] * B[0]) / det};
    double du = ia[0] * x + ia[1] * y + ia[2] * z - fa;
    double dv = ib[0] * x + ib[1] * y + ib[2] * z - fb;
    double dw = ic[0] * x + ic[1] * y + ic[2] * z - fc;
    du -= floor(du); dv -= floor(dv); dw -= floor(dw);
    const double ru = cutoff * sqrt(ia[0] * ia[0] + ia[1] * ia[1] + ia[2] * ia[2]);
    const double rv = cutoff * sqrt(ib[0] * ib[0] + ib[1] * ib[1] + ib[2] * ib[2]);
    const double rw = cutoff * sqrt(ic[0] * ic[0] + ic[1] * ic[1] + ic[2] * ic[2]);
    const double tol = 1e-12;
    const int ulo = (int)ceil(du - ru - tol), uhi = (int)floor(du + ru + tol);
    const int vlo = (int)ceil(dv - rv - tol), vhi = (int)floor(dv + rv + tol);
    const int wlo = (int)ceil(dw - rw - tol), whi = (int)floor(dw + rw + tol);
    const double sig = (sigma_guest + sigma_frame) * 0.5;
    const double eps = sqrt(epsilon_guest * epsilon_frame);
    const double sig2 = sig * sig, rc2 = cutoff * cutoff;
    const double q2 = sig2 / rc2;
    const double q6 = q2 * q2 * q2;
    double total = 0.0;
    for (int i = ulo; i <= uhi; ++i)
        for (int j = vlo; j <= vhi; ++j)
            for (int k = wlo; k <= whi; ++k) {
                const double u = du - i, v = dv - j, w = dw - k;
                const double dx = A[0] * u + A[1] * v + A[2] * w;
                const double dy = B[0] * u + B[1] * v + B[2] * w;
                const double dz = C[0] * u + C[1] * v + C[2] * w;
                const double r2 = fmax(dx * dx + dy * dy + dz * dz, 0.01 * sig2);
                if (r2 < rc2) {
                    const double x2 = sig2 / r2;
                    const double x6 = x2 * x2 * x2;
                    total += 4.0 * eps * (x6 * x6 - x6 - q6 * q6 + q6);
                }
            }
    return total;
}

/* Body-frame rotation of device_fxn.h:34-63: R = Rz(g) Ry(b) Rx(a).        */
void oracle_euler_rotate(double a, double b, double g, const double *v, double *out) {
    const double ca = cos(a), sa = sin(a), cb = cos(b), sb = sin(b), cg = cos(g), sg = sin(g);
    out[0] = v[0] * cg * cb - v[1] * sg * ca + v[1] * sa * cg * sb + v[2] * sg * sa + v[2] * ca * cg * sb;
    out[1] = v[0] * sg * cb + v[1] * cg * ca + v[1] * sg * sb * sa - v[2] * cg * sa + v[2] * sg * sb * ca;
    out[2] = -v[0] * sb + v[1] * cb * sa + v[2] * ca * cb;
}

/* String pose energy (global.h:1071-1128 + the per-pose segmented sum):    */
/* pose = (fractional a, b, c, Euler alpha, beta, gamma in radians); site   */
/* s at frac @ cell + R body_s; energy = sum over sites and framework atoms */
/* of oracle_pair_lj.  body is (n_sites x 3) relative to the center of mass.*/
int oracle_euler_pose_energy(const double *cell, int n_atoms, const double *frac,
                             const double *sigma, const double *epsilon, int n_sites,
                             const double *body, const double *site_sigma,
                             const double *site_epsilon, double cutoff, int n,
                             const double *poses, double *out) {
    const double A[3] = {cell[0], cell[3], cell[6]};
    const double B[3] = {cell[1], cell[4], cell[7]};
    const double C[3] = {cell[2], cell[5], cell[8]};
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < n; ++p) {
        const double *x = poses + 6 * p;
        double com[3];
        row_times(x, cell, com);
        double e = 0.0;
        for (int s = 0; s < n_sites; ++s) {
            double r[3];
            oracle_euler_rotate(x[3], x[4], x[5], body + 3 * s, r);
            const double px = com[0] + r[0], py = com[1] + r[1], pz = com[2] + r[2];
            for (int t = 0; t < n_atoms; ++t)
                e += oracle_pair_lj(px, py, pz, frac[3 * t], frac[3 * t + 1], frac[3 * t + 2], A, B,
                                    C, site_epsilon[s], site_sigma[s], epsilon[t], sigma[t], cutoff);
        }
        out[p] = e;
    }
    return 0;
}
