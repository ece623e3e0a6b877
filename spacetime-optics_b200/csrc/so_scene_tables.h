// so_scene_tables.h -- host computation of a scene's lookup tables (so_scene_tables.cpp).
#pragma once
#include <vector>

namespace so {
namespace tables {

// Circular equatorial prograde orbit of radius r around a hole of spin a (M = 1).
struct CircularOrbit {
    double E, L, Omega;
};
CircularOrbit circular_orbit(double a, double r);
double isco(double a);

// Page-Thorne flux for unit accretion rate: the cumulative torque integral is tabulated once from the
// ISCO out to r_max, then F(r) is read off by linear interpolation in ln r.
class PageThorneFlux {
  public:
    static constexpr int kNodes = 200000;
    PageThorneFlux(double a, double r_max);
    double operator()(double r) const;  // 0 at and inside the ISCO

  private:
    double a_, r_isco_, ln_lo_ = 0, ln_hi_ = 0;
    std::vector<double> radius_, cumulative_;
};

// The disk's flux profile on the temperature table's grid (kSize radii log-spaced from 1.0001 r_isco
// to 1.05 r_out) and the peak temperature it implies at an Eddington ratio.
struct DiskProfile {
    static constexpr int kSize = 1024;
    double ln_r0 = 0, dln_r = 0;
    std::vector<double> flux;
    double flux_max = 0, t_max_physical = 0, eddington = 0;
    // ln T per node for a disk whose peak temperature is t_max (T ~ flux^1/4, at least 1 K)
    std::vector<float> ln_temperature(double t_max) const;
    // Eddington ratio that makes the physical peak temperature t_max
    double eddington_at(double t_max) const;
};
DiskProfile disk_profile(double a, double r_isco, double r_out, double mass_msun, double rg_cm, double eddington);

// ln K2(1 / theta_e) on n log-spaced theta_e in [theta_lo, theta_hi]; the grid's ln start and step.
std::vector<float> ln_bessel_k2_table(int n, double theta_lo, double theta_hi, float* ln_lo, float* dln);

// Blackbody CIE XYZ on kBlackbodyN log-spaced temperatures in [kBlackbodyT0, kBlackbodyT1] K,
// interleaved (X, Y, Z); the grid's ln T start and step.
constexpr int kBlackbodyN = 2048;
constexpr double kBlackbodyT0 = 300.0, kBlackbodyT1 = 3e7;
std::vector<float> blackbody_xyz_table(float* ln_t0, float* dln_t);

}  // namespace tables
}  // namespace so
