// so_scene_tables.cpp -- the lookup tables a scene carries to the kernels, computed on the host from
// the published formulas (geometric units G = c = M = 1 unless a unit is named):
//
//   * circular equatorial orbits of the Kerr metric (Bardeen, Press & Teukolsky 1972, ApJ 178, 347,
//     eqs. 2.12-2.13 and 2.21): energy, angular momentum and angular velocity per unit mass, and the
//     prograde ISCO;
//   * the Novikov-Thorne disk temperature, T ~ F^(1/4), from the Page & Thorne (1974, ApJ 191, 499)
//     flux  F(r) = -Omega'(r) / (4 pi r (E - Omega L)^2) * Integral_{r_isco}^{r} (E - Omega L) L' dr'
//     for an accretion rate of unit Eddington ratio scaled to the shot's;
//   * ln K2(1 / Theta_e) of the thermal synchrotron emissivity (modified Bessel function, libstdc++);
//   * CIE 1931 XYZ of a blackbody: Planck's law (SI, CODATA 2018 constants) against the CIE 1931
//     2-degree colour-matching functions.
//
// Shots must give the reference's tables bit for bit (the images are compared with the reference's
// own code), so every table samples the reference's grids (blackholes/src/scene_build.cpp:116-170,
// colour.cpp:33-60) and evaluates each formula with the same floating-point operations in the same
// order; the Page-Thorne integral keeps the reference's quadrature (trapezoid rule on 200 000
// log-spaced radii, L' by a central difference of step 1e-6 r, linear interpolation in ln r).  This
// file is compiled with -ffp-contract=off, so no expression is fused behind that order.
#include "so_scene_tables.h"

#include <algorithm>
#include <cmath>

namespace so {
namespace tables {
namespace {

constexpr double kPi = 3.14159265358979323846;

// The k-th of n points spread uniformly in [lo, hi] (a log grid when exponentiated).
inline double uniform_point(double lo, double hi, int k, int n) { return lo + (hi - lo) * k / (n - 1); }

}  // namespace

CircularOrbit circular_orbit(double a, double r) {
    // E = (r^3/2 - 2 r^1/2 + a) / D,  L = (r^2 - 2 a r^1/2 + a^2) / D,
    // D = r^3/4 (r^3/2 - 3 r^1/2 + 2 a)^1/2,  Omega = 1 / (r^3/2 + a)
    const double sqrt_r = std::sqrt(r);
    const double denom = std::pow(r, 0.75) * std::sqrt(r * sqrt_r - 3.0 * sqrt_r + 2.0 * a);
    CircularOrbit o;
    o.E = (r * sqrt_r - 2.0 * sqrt_r + a) / denom;
    o.L = (r * r - 2.0 * a * sqrt_r + a * a) / denom;
    o.Omega = 1.0 / (r * std::sqrt(r) + a);
    return o;
}

double isco(double a) {
    // r_isco = 3 + Z2 - sqrt((3 - Z1)(3 + Z1 + 2 Z2)),  Z1 = 1 + (1 - a^2)^1/3 ((1 + a)^1/3 + (1 - a)^1/3),
    // Z2 = (3 a^2 + Z1^2)^1/2  (prograde orbits)
    const double z1 = 1.0 + std::cbrt(1.0 - a * a) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
    const double z2 = std::sqrt(3.0 * a * a + z1 * z1);
    return 3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
}

PageThorneFlux::PageThorneFlux(double a, double r_max) : a_(a), r_isco_(isco(a)) {
    ln_lo_ = std::log(r_isco_);
    ln_hi_ = std::log(r_max);
    radius_.resize(kNodes);
    cumulative_.assign(kNodes, 0.0);
    for (int k = 0; k < kNodes; ++k) radius_[k] = std::exp(uniform_point(ln_lo_, ln_hi_, k, kNodes));
    // (E - Omega L) dL/dr, the derivative by a central difference of step 1e-6 r
    auto torque_density = [a](double r) {
        const double step = 1e-6 * r;
        const double dL = (circular_orbit(a, r + step).L - circular_orbit(a, r - step).L) / (2 * step);
        const CircularOrbit o = circular_orbit(a, r);
        return (o.E - o.Omega * o.L) * dL;
    };
    // the first node sits a hair outside the ISCO, where the orbit formulas are still regular
    double left = torque_density(radius_[0] * (1 + 1e-9));
    for (int k = 1; k < kNodes; ++k) {
        const double right = torque_density(radius_[k]);
        cumulative_[k] = cumulative_[k - 1] + 0.5 * (left + right) * (radius_[k] - radius_[k - 1]);
        left = right;
    }
}

double PageThorneFlux::operator()(double r) const {
    if (r <= r_isco_) return 0.0;
    const double pos = (std::log(r) - ln_lo_) / (ln_hi_ - ln_lo_) * (kNodes - 1);
    const int k = std::min(std::max((int)pos, 0), kNodes - 2);
    const double integral = cumulative_[k] + (cumulative_[k + 1] - cumulative_[k]) * (pos - k);
    const double dOmega_dr = -1.5 * std::sqrt(r) / std::pow(r * std::sqrt(r) + a_, 2);
    const CircularOrbit o = circular_orbit(a_, r);
    const double e_minus_omega_l = o.E - o.Omega * o.L;
    return -dOmega_dr / (4.0 * kPi * r * e_minus_omega_l * e_minus_omega_l) * integral;
}

DiskProfile disk_profile(double a, double r_isco, double r_out, double mass_msun, double rg_cm, double eddington) {
    DiskProfile d;
    const int n = DiskProfile::kSize;
    d.ln_r0 = std::log(r_isco * 1.0001);
    const double ln_r1 = std::log(r_out * 1.05);
    d.dln_r = (ln_r1 - d.ln_r0) / (n - 1);
    std::vector<double> radius(n);
    for (int k = 0; k < n; ++k) radius[k] = std::exp(uniform_point(d.ln_r0, ln_r1, k, n));
    const PageThorneFlux flux(a, radius.back());
    d.flux.resize(n);
    for (int k = 0; k < n; ++k) d.flux[k] = flux(radius[k]);
    d.flux_max = *std::max_element(d.flux.begin(), d.flux.end());
    // Physical scale: flux * Mdot c^2 / r_g^2 with Mdot = f_Edd L_Edd / (eta c^2), the radiative
    // efficiency eta = 1 - E(r_isco) and L_Edd = 1.26e38 erg/s per solar mass (cgs)
    const double c_cgs = 2.99792458e10, stefan_boltzmann = 5.670374419e-5;
    const double efficiency = 1.0 - circular_orbit(a, r_isco).E;
    const double l_edd = 1.26e38 * mass_msun;
    const double mdot = eddington * l_edd / (efficiency * c_cgs * c_cgs);
    d.eddington = eddington;
    d.t_max_physical =
        std::pow(d.flux_max * mdot * c_cgs * c_cgs / (rg_cm * rg_cm) / stefan_boltzmann, 0.25);
    return d;
}

std::vector<float> DiskProfile::ln_temperature(double t_max) const {
    std::vector<float> out(flux.size());
    for (size_t k = 0; k < flux.size(); ++k) {
        const double t = t_max * std::pow(std::max(flux[k], 1e-300) / flux_max, 0.25);
        out[k] = (float)std::log(std::max(t, 1.0));
    }
    return out;
}

double DiskProfile::eddington_at(double t_max) const { return eddington * std::pow(t_max / t_max_physical, 4.0); }

std::vector<float> ln_bessel_k2_table(int n, double theta_lo, double theta_hi, float* ln_lo, float* dln) {
    const double lo = std::log(theta_lo), hi = std::log(theta_hi);
    std::vector<float> out(n);
    for (int k = 0; k < n; ++k) {
        const double theta_e = std::exp(uniform_point(lo, hi, k, n));
        out[k] = (float)std::log(std::cyl_bessel_k(2.0, 1.0 / theta_e));
    }
    *ln_lo = (float)lo;
    *dln = (float)((hi - lo) / (n - 1));
    return out;
}

namespace {

// CIE 1931 2-degree standard observer x-bar, y-bar, z-bar at 380, 390, ..., 780 nm (the published
// standard table at 10 nm resolution).
const double kCieX[41] = {0.001368, 0.004243, 0.014310, 0.043510, 0.134380, 0.283900, 0.348280, 0.336200,
                          0.290800, 0.195360, 0.095640, 0.032010, 0.004900, 0.009300, 0.063270, 0.165500,
                          0.290400, 0.433450, 0.594500, 0.762100, 0.916300, 1.026300, 1.062200, 1.002600,
                          0.854450, 0.642400, 0.447900, 0.283500, 0.164900, 0.087400, 0.046770, 0.022700,
                          0.011359, 0.005790, 0.002899, 0.001440, 0.000690, 0.000332, 0.000166, 0.000083,
                          0.000042};
const double kCieY[41] = {0.000039, 0.000120, 0.000396, 0.001210, 0.004000, 0.011600, 0.023000, 0.038000,
                          0.060000, 0.090980, 0.139020, 0.208020, 0.323000, 0.503000, 0.710000, 0.862000,
                          0.954000, 0.994950, 0.995000, 0.952000, 0.870000, 0.757000, 0.631000, 0.503000,
                          0.381000, 0.265000, 0.175000, 0.107000, 0.061000, 0.032000, 0.017000, 0.008210,
                          0.004102, 0.002091, 0.001047, 0.000520, 0.000249, 0.000120, 0.000060, 0.000030,
                          0.000015};
const double kCieZ[41] = {0.006450, 0.020050, 0.067850, 0.207400, 0.645600, 1.385600, 1.747060, 1.772110,
                          1.669200, 1.287640, 0.812950, 0.465180, 0.272000, 0.158200, 0.078250, 0.042160,
                          0.020300, 0.008750, 0.003900, 0.002100, 0.001650, 0.001100, 0.000800, 0.000340,
                          0.000190, 0.000050, 0.000020, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

// The tabulated function at `nm`, linear between the 10 nm samples, constant beyond the ends.
double cie_at(const double* table, double nm) {
    const double x = (nm - 380.0) / 10.0;
    if (x <= 0) return table[0];
    if (x >= 40) return table[40];
    const int k = (int)x;
    const double frac = x - k;
    return table[k] * (1 - frac) + table[k + 1] * frac;
}

// Planck's law per unit wavelength, W m^-2 sr^-1 nm^-1.
double planck_per_nm(double nm, double kelvin) {
    const double h = 6.62607015e-34, c = 299792458.0, k_b = 1.380649e-23;
    const double m = nm * 1e-9;
    return 2.0 * h * c * c / (m * m * m * m * m) / std::expm1(h * c / (m * k_b * kelvin)) * 1e-9;
}

}  // namespace

std::vector<float> blackbody_xyz_table(float* ln_t0, float* dln_t) {
    // Colour-matching weights at the centres of the 400 one-nanometre bins 380.5 .. 779.5 nm
    constexpr int kBins = 400;
    double wl[kBins], wx[kBins], wy[kBins], wz[kBins];
    for (int b = 0; b < kBins; ++b) {
        wl[b] = 380.5 + b;
        wx[b] = cie_at(kCieX, wl[b]);
        wy[b] = cie_at(kCieY, wl[b]);
        wz[b] = cie_at(kCieZ, wl[b]);
    }
    const double lo = std::log(kBlackbodyT0), hi = std::log(kBlackbodyT1), step = (hi - lo) / (kBlackbodyN - 1);
    std::vector<float> out(3 * kBlackbodyN);
    for (int k = 0; k < kBlackbodyN; ++k) {
        const double kelvin = std::exp(lo + k * step);
        double X = 0, Y = 0, Z = 0;
        for (int b = 0; b < kBins; ++b) {
            const double radiance = planck_per_nm(wl[b], kelvin);
            X += radiance * wx[b];
            Y += radiance * wy[b];
            Z += radiance * wz[b];
        }
        out[3 * k] = (float)X;
        out[3 * k + 1] = (float)Y;
        out[3 * k + 2] = (float)Z;
    }
    *ln_t0 = (float)lo;
    *dln_t = (float)step;
    return out;
}

}  // namespace tables
}  // namespace so
