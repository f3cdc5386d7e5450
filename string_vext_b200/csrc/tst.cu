// Transition-state-theory post-processing of a String path (host code, no
// device work): the hopping diffusivity the String program prints
// (native/string/source_code/RC_main.cu:2485-2527) and the log-domain score
// it uses to choose between the initial and the final path
// (native/string/source_code/legacy_policy.h:21-53, RC_main.cu:2533-2542).
//
// Cell convention: `cell` is the row-vector cell matrix (cart = frac @ cell),
// so the reference's x / y / z coefficient rows (frac2car_a/b/c) are its
// columns.  Energies in K, temperature in K, mass in g/mol, lengths in A.
#include <cmath>

#include "internal.cuh"

namespace vext {

constexpr double kBoltzmann = 1.38e-23;          // J/K, the reference's value
constexpr double kAvogadro = 6.02214076e23;
constexpr double kPi = 3.141592653589793;

static double log_add(double x, double y) {
    if (x == -INFINITY) return y;
    if (y == -INFINITY) return x;
    const double hi = std::fmax(x, y);
    return hi + std::log1p(std::exp(std::fmin(x, y) - hi));
}

}  // namespace vext

using namespace vext;

extern "C" int vext_tst_log_score(int n, const double *frac, const double *energy,
                                  const double *cell, double temperature, double mass_g_mol,
                                  double hop_A, int *valid, double *log_d) {
    if (!valid || !log_d) return fail(VEXT_ERR_ARGUMENT, "valid and log_d outputs required");
    *valid = 0;
    *log_d = 0.0;
    if (n >= 1 && (!frac || !energy || !cell))
        return fail(VEXT_ERR_ARGUMENT, "frac, energy and cell required");
    const double T = temperature, mass = mass_g_mol, hop = hop_A;
    if (n < 2 || !(T > 0) || !(mass > 0) || !(hop > 0) || !std::isfinite(T) ||
        !std::isfinite(mass) || !std::isfinite(hop))
        return 0;
    double emin = INFINITY, emax = -INFINITY;
    for (int i = 0; i < n; ++i) {
        if (!std::isfinite(frac[3 * i]) || !std::isfinite(frac[3 * i + 1]) ||
            !std::isfinite(frac[3 * i + 2]) || !std::isfinite(energy[i]))
            return 0;
        emin = std::fmin(emin, energy[i]);
        emax = std::fmax(emax, energy[i]);
    }
    // rows of the column-vector convention: x = A . dfrac, ...
    const double A[3] = {cell[0], cell[3], cell[6]}, B[3] = {cell[1], cell[4], cell[7]},
                 C[3] = {cell[2], cell[5], cell[8]};
    double log_integral = -INFINITY;
    for (int i = 1; i < n; ++i) {
        const double da = frac[3 * i] - frac[3 * i - 3], db = frac[3 * i + 1] - frac[3 * i - 2],
                     dc = frac[3 * i + 2] - frac[3 * i - 1];
        const double x = A[0] * da + A[1] * db + A[2] * dc;
        const double y = B[0] * da + B[1] * db + B[2] * dc;
        const double z = C[0] * da + C[1] * db + C[2] * dc;
        const double ds = std::hypot(std::hypot(x, y), z) * 1e-10;
        if (!std::isfinite(ds)) return 0;
        if (ds == 0) continue;
        // trapezoid of exp(-(E - Emin)/T) over the unwrapped arc, in log space
        const double term = std::log(ds) - std::log(2.) +
                            log_add(-(energy[i - 1] - emin) / T, -(energy[i] - emin) / T);
        log_integral = log_add(log_integral, term);
    }
    const double ld = std::log(.5) + 2 * std::log(hop * 1e-10) +
                      .5 * std::log(kBoltzmann * T / (2 * kPi * (mass / 1000 / kAvogadro))) -
                      (emax - emin) / T - log_integral;
    *valid = std::isfinite(ld) ? 1 : 0;
    *log_d = ld;
    return 0;
}

extern "C" int vext_tst_diffusivity(int n, const double *frac, const double *energy,
                                    const double *cell, double hop_A, double temperature,
                                    double mass_g_mol, double *d0) {
    if (!d0) return fail(VEXT_ERR_ARGUMENT, "d0 output required");
    if (n < 2 || !frac || !energy || !cell)
        return fail(VEXT_ERR_ARGUMENT, "at least two images, frac, energy and cell required");
    const double T = temperature;
    if (!(T > 0) || !(mass_g_mol > 0) || !(hop_A > 0))
        return fail(VEXT_ERR_ARGUMENT, "T, mass and hop length must be > 0");
    const double A[3] = {cell[0], cell[3], cell[6]}, B[3] = {cell[1], cell[4], cell[7]},
                 C[3] = {cell[2], cell[5], cell[8]};
    // arc length of the path in m, trapezoid of exp(-V/T) (capped at exp(-600))
    double s_prev = 0.0, x_prev = 0.0, y_prev = 0.0, z_prev = 0.0, integral = 0.0, w_prev = 0.0;
    double vmax = energy[0];
    for (int i = 0; i < n; ++i) {
        const double fa = frac[3 * i], fb = frac[3 * i + 1], fc = frac[3 * i + 2];
        const double x = (fa * A[0] + fb * A[1] + fc * A[2]) * 1e-10;
        const double y = (fa * B[0] + fb * B[1] + fc * B[2]) * 1e-10;
        const double z = (fa * C[0] + fb * C[1] + fc * C[2]) * 1e-10;
        const double w = energy[i] / T > 6e2 ? std::exp(-6e2) : std::exp(-energy[i] / T);
        double s = 0.0;
        if (i > 0) {
            s = s_prev + std::sqrt(std::pow(x - x_prev, 2) + std::pow(y - y_prev, 2) +
                                   std::pow(z - z_prev, 2));
            integral = integral + (s - s_prev) * (w + w_prev) / 2;
        }
        if (energy[i] > vmax) vmax = energy[i];
        s_prev = s;
        x_prev = x;
        y_prev = y;
        z_prev = z;
        w_prev = w;
    }
    *d0 = 0.5 * std::pow(hop_A * 1e-10, 2) *
          std::sqrt((kBoltzmann * T) / (2 * kPi * (mass_g_mol / 1e3 / kAvogadro))) *
          (std::exp(-vmax / T) / integral);
    if (!std::isfinite(*d0)) return fail(VEXT_ERR_NONFINITE, "non-finite diffusivity");
    return 0;
}
