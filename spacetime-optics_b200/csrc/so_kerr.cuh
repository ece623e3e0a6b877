// so_kerr.cuh -- Kerr null geodesics in Mino time and the Dormand-Prince 5(4) stepper, shared by the
// CUDA kernels and the host-side shot set-up (critical-curve search).
//
// Follows the reference's blackholes/src/kerr.hpp: kerr_point (:27-42), camera_photon (:63-92),
// geodesic_rhs (:103-116), dp54_step (:118-157), project_radial (:159-173), initial_step (:175-178),
// vacuum_fate (:184-203), critical_curve_point (:210-220).
//
// Arithmetic contract: every multiply-add is an explicit fma() in a fixed order, device code is
// compiled with -fmad=false and host code with -ffp-contract=off, so host and device evaluate the
// same operations and round identically.  The step controller's err^-0.2 (trace.cuh:93, 146) is
// so_rpow5 below (own Newton iteration), not libm/libdevice pow, for the same reason.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/so_tracer.h"

#if defined(__CUDACC__)
#define SO_HD __host__ __device__ __forceinline__
#else
#define SO_HD inline
#endif

namespace so {

constexpr double PI = 3.14159265358979323846;

SO_HD uint64_t dbits(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return b;
#endif
}
SO_HD double bitsd(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double x;
    std::memcpy(&x, &b, 8);
    return x;
#endif
}

// x^(-1/5) for positive normal x (0 for +inf, NaN for NaN).  x = m 2^e with m in [1,2) and
// e = 5q + r (0 <= r < 5): x^(-1/5) = m^(-1/5) 2^(-r/5) 2^(-q).  m^(-1/5) starts from a quadratic
// seed (relative error 1.1e-3) and takes three Newton steps y += (y/5)(1 - m y^5), each squaring
// the error (eps -> 3 eps^2), so the result is within ~1.5 ulp.
SO_HD double rpow5(double x) {
    if (!(x == x)) return x;
    if (x > 1.7976931348623157e308) return 0.0;
    uint64_t b = dbits(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    double m = bitsd((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    int q = e >= 0 ? e / 5 : -((-e + 4) / 5);
    int r = e - 5 * q;
    double y = fma(fma(0.05174, m, -0.28294), m, 1.23011);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double y2 = y * y;
        double y5 = (y2 * y2) * y;
        double t = fma(-m, y5, 1.0);
        y = fma(y * 0.2, t, y);
    }
    const double c = r == 0 ? 1.0 : r == 1 ? 0.8705505632961241 : r == 2 ? 0.757858283255199
                   : r == 3 ? 0.6597539553864471 : 0.5743491774985175;
    y = y * c;
    return y * bitsd((uint64_t)(1023 - q) << 52);
}

// cos(2 pi t) of a phase t given in turns, for |t| < 2^50, branch-free.  t = q/2 + g with the
// nearest half-turn q/2 and |g| <= 1/4: q is read off 2t + 1.5 * 2^52 (rounding to the nearest
// integer, parity in the low mantissa bit), g = t - q/2 is exact, and cos(2 pi t) = (-1)^q cos(2 pi g)
// with cos(2 pi g) from a near-minimax polynomial of degree 8 in g^2 (Chebyshev fit of
// cos(2 pi sqrt(z)) on z in [0, 1/16], coefficients by fit_cos_turns.py; abs error of the fit with
// double coefficients 1e-16).  Sixteen FP64 operations and no branch, so a loop over independent
// phases keeps the FP64 pipe fed; the CPU oracle repeats it operation for operation.
SO_HD double cos_turns(double t) {
    const double magic = 6755399441055744.0;  // 1.5 * 2^52
    const double s = fma(t, 2.0, magic);      // magic + nearest integer to 2t (ties to even)
    const double q = s - magic;                // exact
    const double g = fma(q, -0.5, t);          // exact, |g| <= 1/4
    const double z = g * g;
    double p = 0x1.1678f9078a9b3p-2;
    p = fma(p, z, -0x1.b6957b54dd389p+0);
    p = fma(p, z, 0x1.f9d254582ac30p+2);
    p = fma(p, z, -0x1.a6d1efc8c38bep+4);
    p = fma(p, z, 0x1.e1f506813a321p+5);
    p = fma(p, z, -0x1.55d3c7e3bfbf5p+6);
    p = fma(p, z, 0x1.03c1f081b5992p+6);
    p = fma(p, z, -0x1.3bd3cc9be45dbp+4);
    p = fma(p, z, 1.0);
    return bitsd(dbits(p) ^ ((dbits(s) & 1ull) << 63));  // (-1)^q
}

SO_HD double dot3(const so_vec3& a, const so_vec3& b) { return fma(a.z, b.z, fma(a.y, b.y, a.x * b.x)); }

SO_HD double horizon_radius(double a) { return 1.0 + sqrt(1.0 - a * a); }

// kerr_point (kerr.hpp:27-42): metric functions at (r, theta).  Host set-up, plain libm.
inline void kerr_point(double a, double r, double th, so_kerr_point* k) {
    k->r = r;
    k->s = std::sin(th);
    k->c = std::cos(th);
    double a2 = a * a, r2 = r * r;
    k->Sigma = r2 + a2 * k->c * k->c;
    k->Delta = r2 - 2.0 * r + a2;
    k->A = (r2 + a2) * (r2 + a2) - a2 * k->Delta * k->s * k->s;
    k->omega = 2.0 * a * r / k->A;
    k->e_nu = std::sqrt(k->Sigma * k->Delta / k->A);
    k->e_psi = std::sqrt(k->A / k->Sigma) * k->s;
    k->sqrtSigma = std::sqrt(k->Sigma);
    k->sqrtSigmaDelta = std::sqrt(k->Sigma * k->Delta);
}

// Constants of motion of one photon and the per-ray combinations the right-hand side uses.
struct RayC {
    double a, lam, eta, E;
    double A2, CP, K, Q3;  // a^2, a^2 - a lam, eta + (lam - a)^2, eta + lam^2
};

SO_HD void ray_consts(RayC& c, double a, double lam, double eta, double E) {
    c.a = a;
    c.lam = lam;
    c.eta = eta;
    c.E = E;
    c.A2 = a * a;
    c.CP = fma(-a, lam, c.A2);
    double lma = lam - a;
    c.K = fma(lma, lma, eta);
    c.Q3 = fma(lam, lam, eta);
}

// geodesic_rhs (kerr.hpp:103-116): backward Mino-time derivatives of y = (r, r', u, u', phi, t).
SO_HD void rhs(const RayC& c, const double* y, double* d) {
    double r = y[0], u = y[2];
    double r2 = r * r;
    double Delta = fma(r, r - 2.0, c.A2);
    double P = fma(r, r, c.CP);
    d[0] = y[1];
    d[1] = fma(2.0 * r, P, -((r - 1.0) * c.K));
    d[2] = y[3];
    double u2 = u * u;
    d[3] = u * fma(c.A2, fma(-2.0, u2, 1.0), -c.Q3);
    double s2 = fmax(1.0 - u2, 1e-300);
    double iD = 1.0 / Delta;
    d[4] = c.a - fma(c.a * P, iD, c.lam / s2);
    d[5] = -fma((r2 + c.A2) * P, iD, c.a * fma(-c.a, s2, c.lam));
}

// Dormand-Prince 5(4) tableau (kerr.hpp:124-129).
constexpr double A21 = 1.0 / 5, A31 = 3.0 / 40, A32 = 9.0 / 40, A41 = 44.0 / 45, A42 = -56.0 / 15, A43 = 32.0 / 9;
constexpr double A51 = 19372.0 / 6561, A52 = -25360.0 / 2187, A53 = 64448.0 / 6561, A54 = -212.0 / 729;
constexpr double A61 = 9017.0 / 3168, A62 = -355.0 / 33, A63 = 46732.0 / 5247, A64 = 49.0 / 176,
                 A65 = -5103.0 / 18656;
constexpr double B1 = 35.0 / 384, B3 = 500.0 / 1113, B4 = 125.0 / 192, B5 = -2187.0 / 6784, B6 = 11.0 / 84;
constexpr double E1 = 71.0 / 57600, E3 = -71.0 / 16695, E4 = 71.0 / 1920, E5 = -17253.0 / 339200,
                 E6 = 22.0 / 525, E7 = -1.0 / 40;

// dp54_step (kerr.hpp:122-157).  One FSAL attempt from (y, k1) with step h; writes yo and k7 = f(yo)
// and returns the scaled max-norm error (<= 1 accepts).  Stage inputs are formed for the four
// components the RHS reads; phi and t enter only through the 5th-order sum and the error.
SO_HD double dp54(const RayC& c, const double* y, const double* k1, double h, double tol, double* yo,
                  double* k7) {
    double k2[6], k3[6], k4[6], k5[6], k6[6], t[6];
    t[4] = y[4];
    t[5] = y[5];
#pragma unroll
    for (int i = 0; i < 4; ++i) t[i] = fma(h, A21 * k1[i], y[i]);
    rhs(c, t, k2);
#pragma unroll
    for (int i = 0; i < 4; ++i) t[i] = fma(h, fma(A32, k2[i], A31 * k1[i]), y[i]);
    rhs(c, t, k3);
#pragma unroll
    for (int i = 0; i < 4; ++i) t[i] = fma(h, fma(A43, k3[i], fma(A42, k2[i], A41 * k1[i])), y[i]);
    rhs(c, t, k4);
#pragma unroll
    for (int i = 0; i < 4; ++i)
        t[i] = fma(h, fma(A54, k4[i], fma(A53, k3[i], fma(A52, k2[i], A51 * k1[i]))), y[i]);
    rhs(c, t, k5);
#pragma unroll
    for (int i = 0; i < 4; ++i)
        t[i] = fma(h, fma(A65, k5[i], fma(A64, k4[i], fma(A63, k3[i], fma(A62, k2[i], A61 * k1[i])))), y[i]);
    rhs(c, t, k6);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        yo[i] = fma(h, fma(B6, k6[i], fma(B5, k5[i], fma(B4, k4[i], fma(B3, k3[i], B1 * k1[i])))), y[i]);
    rhs(c, yo, k7);
    double sc[5];
    sc[0] = tol * (1e-6 + fmax(fabs(y[0]), fabs(yo[0])));
    sc[1] = tol * (1e-6 + fmax(fmax(fabs(y[1]), fabs(yo[1])), y[0] * y[0]));
    sc[2] = tol;
    sc[3] = tol * fmax(1.0, fmax(fabs(y[3]), fabs(yo[3])));
    sc[4] = tol * 4.0;
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        double e = h * fma(E7, k7[i], fma(E6, k6[i], fma(E5, k5[i], fma(E4, k4[i], fma(E3, k3[i], E1 * k1[i])))));
        m = fmax(m, fabs(e) / sc[i]);
    }
    return m;
}

// radial_potential (kerr.hpp:94-97) with this file's fma order.
SO_HD double radial_pot(const RayC& c, double r) {
    double P = fma(r, r, c.CP);
    double D = fma(r, r - 2.0, c.A2);
    return fma(P, P, -(D * c.K));
}

// project_radial (kerr.hpp:166-173).
SO_HD void project_radial(const RayC& c, double* y, double* k) {
    double r = y[0];
    double R = radial_pot(c, r);
    double r2 = r * r;
    if (R > 0.25 * (r2 * r2)) {
        double v = sqrt(R);
        y[1] = y[1] < 0.0 ? -v : v;
        k[0] = y[1];
    }
}

// initial_step (kerr.hpp:175-178).
SO_HD double initial_step(const double* y) {
    return 0.02 * fmin(y[0] / (fabs(y[1]) + 1e-12), 1.0 / (fabs(y[3]) + 1e-3));
}

// Unit viewing direction of tangent-plane point (x, y): normalize(F + R (cx + x) + U (cy + y))
// (trace.cuh:64).
SO_HD so_vec3 view_dir(const so_frame& f, double x, double yv) {
    double cxx = f.cx + x, cyy = f.cy + yv;
    so_vec3 v = {fma(f.U.x, cyy, fma(f.R.x, cxx, f.F.x)), fma(f.U.y, cyy, fma(f.R.y, cxx, f.F.y)),
                 fma(f.U.z, cyy, fma(f.R.z, cxx, f.F.z))};
    double il = 1.0 / sqrt(dot3(v, v));
    so_vec3 d = {v.x * il, v.y * il, v.z * il};
    return d;
}

// camera_photon (kerr.hpp:63-92): constants of motion and backward initial state of the photon
// reaching the camera along -d, with the optional Lorentz boost of the camera velocity beta.
SO_HD void camera_photon(double a, const so_kerr_point& kp, double phi0, double t0, so_vec3 d, so_vec3 beta,
                         RayC& c, double* y) {
    double k0 = 1.0;
    so_vec3 k = {-d.x, -d.y, -d.z};
    double b2 = dot3(beta, beta);
    if (b2 > 0.0) {
        double b = sqrt(b2), g = 1.0 / sqrt(1.0 - b2);
        double ib = 1.0 / b;
        so_vec3 bh = {beta.x * ib, beta.y * ib, beta.z * ib};
        double kpar = dot3(k, bh);
        double k0z = g * fma(b, kpar, k0);
        double coef = fma(g - 1.0, kpar, (g * b) * k0);
        k.x = fma(bh.x, coef, k.x);
        k.y = fma(bh.y, coef, k.y);
        k.z = fma(bh.z, coef, k.z);
        k0 = k0z;
    }
    double L = kp.e_psi * k.z;
    double E = fma(kp.omega, L, kp.e_nu * k0);
    double pth = kp.sqrtSigma * k.y;
    double inner = fma(-(a * a), E * E, (L * L) / (kp.s * kp.s));
    double Q = fma(pth, pth, (kp.c * kp.c) * inner);
    ray_consts(c, a, L / E, Q / (E * E), E);
    double dr = (kp.sqrtSigmaDelta * k.x) / E;
    double dth = pth / E;
    y[0] = kp.r;
    y[1] = -dr;
    y[2] = kp.c;
    y[3] = kp.s * dth;
    y[4] = phi0;
    y[5] = t0;
}

// Step-size controller of trace.cuh:92-96 and :146.
SO_HD double reject_step(double hc, double err) {
    double h = hc * fmax(0.2, 0.9 * rpow5(fmax(err, 1e-30)));
    if (!(err == err)) h = hc * 0.1;
    return h;
}
SO_HD double accept_step(double hc, double err) { return hc * fmin(5.0, fmax(0.2, 0.9 * rpow5(fmax(err, 1e-30)))); }

// vacuum_fate (kerr.hpp:184-203): +1 escaped, -1 captured, 0 undecided.
SO_HD int vacuum_fate(double a, const so_frame& f, so_vec3 d, double tol, double r_escape, int max_steps) {
    RayC c;
    double y[6], k1[6], yn[6], k7[6];
    camera_photon(a, f.kp, f.ph, f.t, d, f.beta, c, y);
    double rh = horizon_radius(a);
    rhs(c, y, k1);
    double h = initial_step(y);
    for (int it = 0; it < max_steps; ++it) {
        double err = dp54(c, y, k1, h, tol, yn, k7);
        if (err > 1.0) {
            h *= fmax(0.2, 0.9 * rpow5(err));
            continue;
        }
        for (int i = 0; i < 6; ++i) {
            y[i] = yn[i];
            k1[i] = k7[i];
        }
        project_radial(c, y, k1);
        h *= fmin(5.0, fmax(0.2, 0.9 * rpow5(fmax(err, 1e-30))));
        if (y[0] < rh * 1.0001 + 1e-3) return -1;
        if (y[0] > r_escape && y[1] > 0.0) return 1;
    }
    return 0;
}

// critical_curve_point (kerr.hpp:210-220), Bardeen (1973).
SO_HD bool critical_curve_point(double a, double theta_o, double rp, double* alpha, double* beta_plus) {
    double D = rp * rp - 2.0 * rp + a * a;
    double lam = a + rp / a * (rp - 2.0 * D / (rp - 1.0));
    double eta = rp * rp * rp / (a * a) * (4.0 * D / ((rp - 1.0) * (rp - 1.0)) - rp);
    double so_ = sin(theta_o), co = cos(theta_o);
    double b2 = eta + a * a * co * co - lam * lam * co * co / (so_ * so_);
    if (b2 < 0.0) return false;
    *alpha = -lam / so_;
    *beta_plus = sqrt(b2);
    return true;
}

// ---- far-field transport in the inverse radius -----------------------------------------------
// A backward ray from a distant camera has r' ~ -r^2 in Mino time: r(lambda) has a pole near the
// camera, so a Mino-time integrator at relative tolerance tol advances r by ~ tol^(1/6) per step
// (about 280 DP5 attempts from r = 1e7 M to 100 M at tol = 1e-8).  With x = 1/r as the independent
// variable the motion is smooth on an ingoing leg without a radial turning point:
//   d lambda / dx = 1 / sqrt(Rt(x)),   Rt(x) = x^4 R(1/x) = (1 + CP x^2)^2 - x^2 D(x) K,
//   D(x) = x^2 Delta = 1 - 2x + a^2 x^2,  CP = a^2 - a lam,  K = eta + (lam - a)^2,
// and the polar and azimuthal equations of rhs() times d lambda / dx.  The coordinate time has poles
// 1/x^2 + 2/x, integrated in closed form:  t(x) = t0 + (1/x - 1/x0) - 2 ln(x / x0) + tau(x), with
//   d tau / dx = -(q + v N/D) - w a (lam - a s^2),   w = 1/sqrt(Rt) = 1 + x^2 v,
//   N/D = (1 + a^2 x^2)(1 + CP x^2) / D = 1 + 2x + x^2 q,   q = (CP + 4 - 2 a^2 x + a^2 CP x^2) / D,
//   v = (D K - 2 CP - CP^2 x^2) / (sqrt(Rt) (1 + sqrt(Rt))),
// all free of cancellation at x -> 0.  z = (u, u', phi, tau), u' = du/dlambda as in rhs().  An
// outgoing leg (sg = -1, x decreasing) has d lambda / dx = -1/sqrt(Rt) and the pole terms with the
// opposite sign: t(x) = t0 - (1/x - 1/x0) + 2 ln(x / x0) + tau, d tau / dx = (q + v N/D) - w a (...).
SO_HD void far_rhs(const RayC& c, double x, const double* z, double* d, double sg = 1.0) {
    double x2 = x * x;
    double D = fma(x, fma(c.A2, x, -2.0), 1.0);
    double cpx = fma(c.CP, x2, 1.0);
    double Rt = fma(cpx, cpx, -(x2 * D * c.K));
    double sR = sqrt(Rt);
    double w = sg / sR;
    double u = z[0], u2 = u * u;
    double s2 = fmax(1.0 - u2, 1e-300);
    double iD = 1.0 / D;
    d[0] = z[1] * w;
    d[1] = u * fma(c.A2, fma(-2.0, u2, 1.0), -c.Q3) * w;
    d[2] = (c.a - fma(c.a * cpx, iD, c.lam / s2)) * w;
    double q = fma(x, fma(c.A2 * c.CP, x, -2.0 * c.A2), c.CP + 4.0) * iD;
    double v = fma(-(c.CP * c.CP), x2, fma(D, c.K, -2.0 * c.CP)) / (sR * (1.0 + sR));
    double nd = fma(c.A2, x2, 1.0) * cpx * iD;
    d[3] = -sg * fma(v, nd, q) - w * c.a * fma(-c.a, s2, c.lam);
}

// Whether far_approach() applies from radius r0 (state y0) to r1: an ingoing ray towards a smaller
// r1, or an outgoing one towards a larger r1, whose radial potential keeps Rt >= 1/2 between them
// (K x^2 <= 1/4 at the inner end bounds the only decreasing term).
SO_HD bool far_applies(const RayC& c, const double* y0, double r1) {
    const bool in = y0[0] > r1 && y0[1] < 0.0, out = y0[0] < r1 && y0[1] > 0.0;
    if (!in && !out) return false;
    double x1 = 1.0 / (in ? r1 : y0[0]), x2 = x1 * x1;
    // outwards the ray is already past its last turning point: only keep clear of its neighbourhood
    if (!(c.K * x2 <= (in ? 0.25 : 0.5))) return false;
    double cpx = fma(c.CP, x2, 1.0);
    double D = fma(x1, fma(c.A2, x1, -2.0), 1.0);
    return fma(cpx, cpx, -(x2 * D * c.K)) >= (in ? 0.5 : 0.25);
}

// DP5(4) in x from the state y (r, r', u, u', phi, t) at r = y[0] to r1, in place, inwards (from the
// camera) or outwards (to the escape radius) as far_applies() decided: on return y is the state at
// r1 with r' = -sqrt(R(r1)) inwards, +sqrt(R(r1)) outwards, from the radial constraint.  Error norm as dp54's for
// u, u', phi (tol, tol max(1,|u'|), 4 tol) plus tol max(1, |tau|) for tau.  psi and ncross are
// accumulated per accepted step as the reference's driver does (trace.cuh:97-106).  Returns the
// number of attempts, or -1 (y, psi, ncross untouched) if max_att attempts did not reach r1.
SO_HD int far_approach(const RayC& c, double* y, double r1, double tol, int max_att, double* psi_io, int* ncross_io,
                       bool want_psi) {
    double psi = *psi_io;
    int ncross = *ncross_io;
    const double r0 = y[0], x0 = 1.0 / r0, x1 = 1.0 / r1;
    const double sg = x1 > x0 ? 1.0 : -1.0;  // +1 inwards (x increasing), -1 outwards
    double z[4] = {y[2], y[3], y[4], 0.0}, k1[4], k2[4], k3[4], k4[4], k5[4], k6[4], k7[4], t[4], zn[4];
    far_rhs(c, x0, z, k1, sg);
    double x = x0;
    double h = sg * fmin(sg * (x1 - x0), 0.1 / sqrt(c.K + 1.0));
    double sp = sqrt(fmax(fma(-z[0], z[0], 1.0), 0.0));
    double pp0 = sp * cos(z[2]), pp1 = sp * sin(z[2]), pp2 = z[0];
    int att = 0;
    while (sg * (x1 - x) > 0.0) {
        if (att >= max_att) return -1;
        ++att;
        const bool last = sg * (x + h - x1) >= 0.0;
        const double hc = last ? x1 - x : h;
#pragma unroll
        for (int i = 0; i < 4; ++i) t[i] = fma(hc, A21 * k1[i], z[i]);
        far_rhs(c, fma(0.2, hc, x), t, k2, sg);
#pragma unroll
        for (int i = 0; i < 4; ++i) t[i] = fma(hc, fma(A32, k2[i], A31 * k1[i]), z[i]);
        far_rhs(c, fma(0.3, hc, x), t, k3, sg);
#pragma unroll
        for (int i = 0; i < 4; ++i) t[i] = fma(hc, fma(A43, k3[i], fma(A42, k2[i], A41 * k1[i])), z[i]);
        far_rhs(c, fma(0.8, hc, x), t, k4, sg);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            t[i] = fma(hc, fma(A54, k4[i], fma(A53, k3[i], fma(A52, k2[i], A51 * k1[i]))), z[i]);
        far_rhs(c, fma(8.0 / 9.0, hc, x), t, k5, sg);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            t[i] = fma(hc, fma(A65, k5[i], fma(A64, k4[i], fma(A63, k3[i], fma(A62, k2[i], A61 * k1[i])))), z[i]);
        const double xn = last ? x1 : x + hc;
        far_rhs(c, xn, t, k6, sg);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            zn[i] = fma(hc, fma(B6, k6[i], fma(B5, k5[i], fma(B4, k4[i], fma(B3, k3[i], B1 * k1[i])))), z[i]);
        far_rhs(c, xn, zn, k7, sg);
        double sc[4];
        sc[0] = tol;
        sc[1] = tol * fmax(1.0, fmax(fabs(z[1]), fabs(zn[1])));
        sc[2] = tol * 4.0;
        sc[3] = tol * fmax(1.0, fmax(fabs(z[3]), fabs(zn[3])));
        double err = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            double e = hc * fma(E7, k7[i], fma(E6, k6[i], fma(E5, k5[i], fma(E4, k4[i], fma(E3, k3[i], E1 * k1[i])))));
            err = fmax(err, fabs(e) / sc[i]);
        }
        if (!(err <= 1.0)) {
            h = reject_step(hc, err);
            continue;
        }
        if (want_psi) {
            double sn = sqrt(fmax(fma(-zn[0], zn[0], 1.0), 0.0));
            double pn0 = sn * cos(zn[2]), pn1 = sn * sin(zn[2]), pn2 = zn[0];
            double cx = fma(pp1, pn2, -(pp2 * pn1)), cy = fma(pp2, pn0, -(pp0 * pn2)), cz = fma(pp0, pn1, -(pp1 * pn0));
            psi += atan2(sqrt(fma(cz, cz, fma(cy, cy, cx * cx))), fma(pp2, pn2, fma(pp1, pn1, pp0 * pn0)));
            pp0 = pn0;
            pp1 = pn1;
            pp2 = pn2;
        }
        if ((z[0] > 0.0) != (zn[0] > 0.0)) ++ncross;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            z[i] = zn[i];
            k1[i] = k7[i];
        }
        x = xn;
        if (!last) h = accept_step(hc, err);
    }
    y[5] = y[5] + sg * (r1 - r0) - sg * 2.0 * log(r0 / r1) + z[3];
    y[0] = r1;
    y[1] = -sg * sqrt(fmax(radial_pot(c, r1), 0.0));
    y[2] = z[0];
    y[3] = z[1];
    y[4] = z[2];
    *psi_io = psi;
    *ncross_io = ncross;
    return att;
}

// hermite_d (trace.cuh:19-22), fixed fma order.
SO_HD double hermite(double p0, double p1, double m0, double m1, double s) {
    double s2 = s * s, s3 = s2 * s;
    double c00 = fma(2.0, s3, fma(-3.0, s2, 1.0));
    double c10 = fma(-2.0, s2, s3) + s;
    double c01 = fma(-2.0, s3, 3.0 * s2);
    double c11 = s3 - s2;
    return fma(c11, m1, fma(c01, p1, fma(c10, m0, c00 * p0)));
}

}  // namespace so
