/* so_oracle.c -- CPU oracle for the Kerr ray-tracer path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the product: only tests, the smoke check and the bench's CPU
 * baseline load it.  It restates, in plain C99, the reference tracer of orrnithogalum/spacetime-optics
 * (bhrt).  Each function cites the reference file:line it follows (paths relative to the reference
 * project root).
 *
 * Arithmetic contract.  Every multiply-add that the CUDA kernel fuses is written here as an explicit
 * fma(), the file is compiled with -ffp-contract=off, and the step controller uses the project's own
 * err^(-1/5) (so_rpow5 below) instead of libm pow.  With that, the CUDA FP64 kernel (compiled with
 * -fmad=false and the same explicit fma placement) reproduces this oracle's trajectories bit for
 * bit: fate, winding order and step counts are exact, and the outputs differ only where a libm
 * transcendental (acos, atan2, sin, cos, exp, log) of the host and of the device round differently
 * (a few ulp, output-only).  Against the reference's own code (trace.cuh compiled for the host, see
 * ref_shim.cpp) the same rays agree to ~1e-12 in direction; only rays on the critical curve, where
 * the Lyapunov growth amplifies ulp differences, may change fate.
 *
 * Parity pinned: tests/golden holds vectors produced by the reference's own trace_ray / vacuum_fate
 * / critical_curve_point / find_critical_point (compiled from the reference sources by
 * oracle/Makefile), and tests check this oracle against them.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/so_tracer.h"

#define PI_D 3.14159265358979323846
/* cgs constants, common.hpp:16-27 */
#define CGS_C 2.99792458e10
#define CGS_KB 1.380649e-16
#define CGS_H 6.62607015e-27
#define CGS_ME 9.1093837e-28
#define CGS_MP 1.67262192e-24
#define CGS_QE 4.80320471e-10

/* ------------------------------------------------------------------------------------------------
 * err^(-1/5), own implementation (replaces pow(err, -0.2) of trace.cuh:93/146, kerr.hpp:193/198).
 * x = m 2^e, m in [1,2), e = 5q + r:  x^(-1/5) = m^(-1/5) 2^(-r/5) 2^(-q).  m^(-1/5) from a quadratic
 * seed (rel. error 1.1e-3) and three Newton steps on m y^5 = 1 (error -> 3 eps^2 each).
 * Valid for positive normal x, +inf (returns 0) and NaN (returns NaN).
 * ---------------------------------------------------------------------------------------------- */
static const double RPOW5_C[5] = {1.0, 0.8705505632961241, 0.757858283255199, 0.6597539553864471,
                                  0.5743491774985175};
double so_rpow5(double x) {
    if (!(x == x)) return x;
    if (x > 1.7976931348623157e308) return 0.0;
    uint64_t b;
    memcpy(&b, &x, 8);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    uint64_t mb = (b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &mb, 8);
    int q = e >= 0 ? e / 5 : -((-e + 4) / 5);
    int r = e - 5 * q;
    double y = fma(fma(0.05174, m, -0.28294), m, 1.23011);
    for (int i = 0; i < 3; ++i) {
        double y2 = y * y;
        double y5 = (y2 * y2) * y;
        double t = fma(-m, y5, 1.0);
        y = fma(y * 0.2, t, y);
    }
    y = y * RPOW5_C[r];
    uint64_t sb = (uint64_t)(1023 - q) << 52;
    double s;
    memcpy(&s, &sb, 8);
    return y * s;
}

/* ---- small vector helpers with a fixed fma order (common.hpp:31-42) -------------------------- */
static double dot3(so_vec3 a, so_vec3 b) { return fma(a.z, b.z, fma(a.y, b.y, a.x * b.x)); }
static so_vec3 cross3(so_vec3 a, so_vec3 b) {
    so_vec3 c = {fma(a.y, b.z, -(a.z * b.y)), fma(a.z, b.x, -(a.x * b.z)), fma(a.x, b.y, -(a.y * b.x))};
    return c;
}

/* kerr_point, kerr.hpp:27-42 (host side of the frame set-up; plain libm, as the reference). */
void orc_kerr_point(double a, double r, double th, so_kerr_point* k) {
    k->r = r;
    k->s = sin(th);
    k->c = cos(th);
    double a2 = a * a, r2 = r * r;
    k->Sigma = r2 + a2 * k->c * k->c;
    k->Delta = r2 - 2.0 * r + a2;
    k->A = (r2 + a2) * (r2 + a2) - a2 * k->Delta * k->s * k->s;
    k->omega = 2.0 * a * r / k->A;
    k->e_nu = sqrt(k->Sigma * k->Delta / k->A);
    k->e_psi = sqrt(k->A / k->Sigma) * k->s;
    k->sqrtSigma = sqrt(k->Sigma);
    k->sqrtSigmaDelta = sqrt(k->Sigma * k->Delta);
}

double orc_horizon_radius(double a) { return 1.0 + sqrt(1.0 - a * a); } /* kerr.hpp:44 */

/* ---- per-ray constants of motion and the geodesic right-hand side ---------------------------- */
typedef struct {
    double a, lam, eta, E;
    double A2, CP, K, Q3; /* a^2, a^2 - a lam, eta + (lam - a)^2, eta + lam^2 */
} RayC;

static void ray_consts(RayC* c, double a, double lam, double eta, double E) {
    c->a = a;
    c->lam = lam;
    c->eta = eta;
    c->E = E;
    c->A2 = a * a;
    c->CP = fma(-a, lam, c->A2);
    double lma = lam - a;
    c->K = fma(lma, lma, eta);
    c->Q3 = fma(lam, lam, eta);
}

/* geodesic_rhs, kerr.hpp:103-116: backward Mino-time derivatives of (r, r', u, u', phi, t). */
static void rhs(const RayC* c, const double* y, double* d) {
    double r = y[0], u = y[2];
    double r2 = r * r;
    double Delta = fma(r, r - 2.0, c->A2);
    double P = fma(r, r, c->CP);
    d[0] = y[1];
    d[1] = fma(2.0 * r, P, -((r - 1.0) * c->K));
    d[2] = y[3];
    double u2 = u * u;
    d[3] = u * fma(c->A2, fma(-2.0, u2, 1.0), -c->Q3);
    double s2 = fmax(1.0 - u2, 1e-300);
    double iD = 1.0 / Delta;
    d[4] = c->a - fma(c->a * P, iD, c->lam / s2);
    d[5] = -fma((r2 + c->A2) * P, iD, c->a * fma(-c->a, s2, c->lam));
}

/* dp54_step, kerr.hpp:122-157: Dormand-Prince 5(4), FSAL, scaled max-norm error over (r, r', u, u',
 * phi).  Stage inputs are formed only for the four components the RHS reads (phi and t are
 * quadratures). */
static const double A21 = 1.0 / 5, A31 = 3.0 / 40, A32 = 9.0 / 40, A41 = 44.0 / 45, A42 = -56.0 / 15,
                    A43 = 32.0 / 9;
static const double A51 = 19372.0 / 6561, A52 = -25360.0 / 2187, A53 = 64448.0 / 6561, A54 = -212.0 / 729;
static const double A61 = 9017.0 / 3168, A62 = -355.0 / 33, A63 = 46732.0 / 5247, A64 = 49.0 / 176,
                    A65 = -5103.0 / 18656;
static const double B1 = 35.0 / 384, B3 = 500.0 / 1113, B4 = 125.0 / 192, B5 = -2187.0 / 6784, B6 = 11.0 / 84;
static const double E1 = 71.0 / 57600, E3 = -71.0 / 16695, E4 = 71.0 / 1920, E5 = -17253.0 / 339200,
                    E6 = 22.0 / 525, E7 = -1.0 / 40;

static double dp54(const RayC* c, const double* y, const double* k1, double h, double tol, double* yo,
                   double* k7) {
    double k2[6], k3[6], k4[6], k5[6], k6[6], t[6];
    t[4] = y[4];
    t[5] = y[5];
    for (int i = 0; i < 4; ++i) t[i] = fma(h, A21 * k1[i], y[i]);
    rhs(c, t, k2);
    for (int i = 0; i < 4; ++i) t[i] = fma(h, fma(A32, k2[i], A31 * k1[i]), y[i]);
    rhs(c, t, k3);
    for (int i = 0; i < 4; ++i) t[i] = fma(h, fma(A43, k3[i], fma(A42, k2[i], A41 * k1[i])), y[i]);
    rhs(c, t, k4);
    for (int i = 0; i < 4; ++i)
        t[i] = fma(h, fma(A54, k4[i], fma(A53, k3[i], fma(A52, k2[i], A51 * k1[i]))), y[i]);
    rhs(c, t, k5);
    for (int i = 0; i < 4; ++i)
        t[i] = fma(h, fma(A65, k5[i], fma(A64, k4[i], fma(A63, k3[i], fma(A62, k2[i], A61 * k1[i])))), y[i]);
    rhs(c, t, k6);
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
    for (int i = 0; i < 5; ++i) {
        double e = h * fma(E7, k7[i], fma(E6, k6[i], fma(E5, k5[i], fma(E4, k4[i], fma(E3, k3[i], E1 * k1[i])))));
        m = fmax(m, fabs(e) / sc[i]);
    }
    return m;
}

/* project_radial, kerr.hpp:166-173 (radial_potential kerr.hpp:94-97). */
static void project_radial(const RayC* c, double* y, double* k) {
    double r = y[0];
    double P = fma(r, r, c->CP);
    double D = fma(r, r - 2.0, c->A2);
    double R = fma(P, P, -(D * c->K));
    double r2 = r * r;
    if (R > 0.25 * (r2 * r2)) {
        double v = sqrt(R);
        y[1] = y[1] < 0.0 ? -v : v;
        k[0] = y[1];
    }
}

/* initial_step, kerr.hpp:175-178. */
static double initial_step(const double* y) {
    return 0.02 * fmin(y[0] / (fabs(y[1]) + 1e-12), 1.0 / (fabs(y[3]) + 1e-3));
}

/* camera_photon, kerr.hpp:63-92.  y receives the backward state. */
static void camera_photon(double a, const so_kerr_point* kp, double phi0, double t0, so_vec3 d, so_vec3 beta,
                          RayC* c, double* y) {
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
    double L = kp->e_psi * k.z;
    double E = fma(kp->omega, L, kp->e_nu * k0);
    double pth = kp->sqrtSigma * k.y;
    double inner = fma(-(a * a), E * E, (L * L) / (kp->s * kp->s));
    double Q = fma(pth, pth, (kp->c * kp->c) * inner);
    ray_consts(c, a, L / E, Q / (E * E), E);
    double dr = (kp->sqrtSigmaDelta * k.x) / E;
    double dth = pth / E;
    y[0] = kp->r;
    y[1] = -dr;
    y[2] = kp->c;
    y[3] = kp->s * dth;
    y[4] = phi0;
    y[5] = t0;
}

/* ---- device_util.cuh restated: hash, R2 jitter, gradient noise, tables ----------------------- */
static uint32_t pcg(uint32_t v) { /* device_util.cuh:15-19 */
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
static float rnd(uint32_t* s) { /* device_util.cuh:20-23 */
    *s = pcg(*s);
    return (float)(*s >> 8) * (1.0f / 16777216.0f);
}
static float frac1(float x) { return x - floorf(x); }
static void r2_sample(uint32_t n, float r0, float r1, float* x, float* y) { /* device_util.cuh:25-30 */
    const double a1 = 0.7548776662466927, a2 = 0.5698402909980532;
    *x = frac1(r0 + (float)fmod(n * a1, 1.0));
    *y = frac1(r1 + (float)fmod(n * a2, 1.0));
}
static float lerpf_(float a, float b, float t) { return a + (b - a) * t; }
static float grad3(int ix, int iy, int iz, uint32_t seed, float fx, float fy, float fz) { /* :32-41 */
    uint32_t h = pcg((uint32_t)ix * 73856093u ^ pcg((uint32_t)iy * 19349663u ^ pcg((uint32_t)iz * 83492791u ^ seed)));
    switch (h % 12u) {
        case 0: return fx + fy;   case 1: return -fx + fy;  case 2: return fx - fy;   case 3: return -fx - fy;
        case 4: return fx + fz;   case 5: return -fx + fz;  case 6: return fx - fz;   case 7: return -fx - fz;
        case 8: return fy + fz;   case 9: return -fy + fz;  case 10: return fy - fz;  default: return -fy - fz;
    }
}
static float gnoise(float x, float y, float z, uint32_t seed) { /* device_util.cuh:42-59 */
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    float ux = x - fx, uy = y - fy, uz = z - fz;
    float wx = ux * ux * ux * (ux * (ux * 6.f - 15.f) + 10.f);
    float wy = uy * uy * uy * (uy * (uy * 6.f - 15.f) + 10.f);
    float wz = uz * uz * uz * (uz * (uz * 6.f - 15.f) + 10.f);
    float n000 = grad3(ix, iy, iz, seed, ux, uy, uz);
    float n100 = grad3(ix + 1, iy, iz, seed, ux - 1, uy, uz);
    float n010 = grad3(ix, iy + 1, iz, seed, ux, uy - 1, uz);
    float n110 = grad3(ix + 1, iy + 1, iz, seed, ux - 1, uy - 1, uz);
    float n001 = grad3(ix, iy, iz + 1, seed, ux, uy, uz - 1);
    float n101 = grad3(ix + 1, iy, iz + 1, seed, ux - 1, uy, uz - 1);
    float n011 = grad3(ix, iy + 1, iz + 1, seed, ux, uy - 1, uz - 1);
    float n111 = grad3(ix + 1, iy + 1, iz + 1, seed, ux - 1, uy - 1, uz - 1);
    float x00 = lerpf_(n000, n100, wx), x10 = lerpf_(n010, n110, wx);
    float x01 = lerpf_(n001, n101, wx), x11 = lerpf_(n011, n111, wx);
    return lerpf_(lerpf_(x00, x10, wy), lerpf_(x01, x11, wy), wz);
}
static float fbm3(float x, float y, float z, int oct, uint32_t seed) { /* device_util.cuh:61-72 */
    float s = 0.f, amp = 1.f, norm = 0.f;
    for (int i = 0; i < oct; ++i) {
        s += amp * gnoise(x, y, z, seed + 1013u * (uint32_t)i);
        norm += amp * amp;
        float nx = 0.80f * x + 0.60f * z, nz = -0.60f * x + 0.80f * z;
        x = nx * 2.03f;
        y = y * 2.03f;
        z = nz * 2.03f;
        amp *= 0.55f;
    }
    return s * 2.2f / sqrtf(norm);
}
static float table_lerp(const float* t, int n, float x0, float dx, float x) { /* device_util.cuh:74-80 */
    float f = (x - x0) / dx;
    f = fminf(fmaxf(f, 0.f), (float)(n - 2) + 0.9999f);
    int i = (int)f;
    f -= (float)i;
    return t[i] + (t[i + 1] - t[i]) * f;
}
static void blackbody_xyz(const so_scene* S, float T, float* xyz) { /* device_util.cuh:82-90 */
    float f = (logf(fmaxf(T, 1.f)) - S->bb_l0) / S->bb_dl;
    f = fminf(fmaxf(f, 0.f), (float)(S->bb_n - 2) + 0.9999f);
    int i = (int)f;
    f -= (float)i;
    const float* p = S->bb_xyz + 3 * i;
    xyz[0] = p[0] + (p[3] - p[0]) * f;
    xyz[1] = p[1] + (p[4] - p[1]) * f;
    xyz[2] = p[2] + (p[5] - p[2]) * f;
}

/* ---- emission.cuh restated ----------------------------------------------------------------- */
static double keplerian_omega(const so_scene* S, double R) { return 1.0 / fma(R, sqrt(R), S->a); } /* :20 */
/* sheared_noise, emission.cuh:34-51 (rsqrtf restated as 1/sqrtf). */
static float sheared_noise(const so_scene* S, double R, double phi, double z, double t, float scale, float tcorr,
                           uint32_t seed) {
    double Om = keplerian_omega(S, fmax(R, S->r_isco));
    double P = 6.283185307179586 / Om * (double)tcorr;
    double s = t / P;
    double k = floor(s);
    float f = (float)(s - k);
    float acc = 0.f;
    for (int j = 0; j < 2; ++j) {
        double tb = (k + j) * P;
        double ph = phi - Om * (t - tb);
        float inv = 1.f / (scale * (float)R);
        float x = (float)(R * cos(ph)) * inv, y = (float)(R * sin(ph)) * inv, zz = (float)z * inv * 2.f;
        float n = fbm3(x, y, zz, 4, seed + 7919u * (uint32_t)(long long)(k + j));
        float w = j == 0 ? 1.f - f : f;
        acc += w * n;
    }
    return acc * (1.f / sqrtf((1.f - f) * (1.f - f) + f * f));
}
/* disk_temperature / disk_shade, emission.cuh:53-86 (__expf restated as expf). */
static float disk_temperature(const so_scene* S, double r) {
    return expf(table_lerp(S->disk_lnT, S->disk_n, (float)S->disk_lr0, (float)S->disk_dlr, (float)log(r)));
}
static double circ_ut(double a, double r) { /* u^t of a circular prograde equatorial orbit */
    double sr = sqrt(r);
    double q = sqrt(sr);
    return fma(r, sr, a) / (q * q * q * sqrt(fmax(fma(r, sr, -3.0 * sr) + 2.0 * a, 1e-12)));
}
static void disk_shade(const so_scene* S, double r, double phi, double t, double lam, double eta, double Ecam,
                       float* out) {
    out[0] = out[1] = out[2] = out[3] = 0.f;
    if (r < S->disk_rin || r > S->disk_rout) return;
    double ut = circ_ut(S->a, r);
    double Om = keplerian_omega(S, r);
    double kdotu = ut * fma(-Om, lam, 1.0);
    double g = 1.0 / (Ecam * kdotu);
    float T = disk_temperature(S, r);
    float m = 1.f;
    if (S->disk_turb_amp > 0.f) {
        float n = sheared_noise(S, r, phi, 0.0, t, S->disk_turb_scale, S->disk_tcorr, S->seed);
        m = expf(S->disk_turb_amp * n - 0.5f * S->disk_turb_amp * S->disk_turb_amp);
    }
    T *= sqrtf(sqrtf(m));
    float ld = 1.f;
    if (S->disk_ld > 0.f) {
        float mu = (float)fmin(sqrt(fmax(eta, 0.0)) / (r * kdotu), 1.0);
        ld = (1.f + 2.06f * mu) / (1.f + 2.06f * 2.f / 3.f);
    }
    float fc = S->disk_fcol;
    float xyz[3];
    blackbody_xyz(S, (float)g * T * fc, xyz);
    float s = ld / (fc * fc * fc * fc);
    float e0 = (float)(0.75 * S->disk_rout), e1 = (float)S->disk_rout, xr = (float)r;
    float tt = (xr - e0) / (e1 - e0);
    tt = tt < 0.f ? 0.f : (tt > 1.f ? 1.f : tt);
    float edge = 1.f - tt * tt * (3.f - 2.f * tt);
    out[0] = xyz[0] * s * edge;
    out[1] = xyz[1] * s * edge;
    out[2] = xyz[2] * s * edge;
    out[3] = edge;
}
/* redshift of a circular prograde equatorial emitter at r seen by this photon (the g of
 * emission.cuh:66-71), recorded at equatorial crossings for the surrogate's targets. */
static double crossing_g(const so_scene* S, double r, double lam, double Ecam) {
    if (r < S->r_isco) return 0.0;
    double ut = circ_ut(S->a, r);
    double kdotu = ut * fma(-keplerian_omega(S, r), lam, 1.0);
    return 1.0 / (Ecam * kdotu);
}

/* cos(2 pi t) of a phase in turns: the library's cos_turns (so_kerr.cuh), operation for operation.
 * 2t is rounded to the nearest integer q by adding 1.5 * 2^52 (its parity is the low mantissa bit),
 * g = t - q/2 is exact, and cos(2 pi g) comes from a polynomial of degree 8 in g^2 (a Chebyshev fit
 * of cos(2 pi sqrt(z)) on [0, 1/16]). */
static double cos_turns(double t) {
    const double magic = 6755399441055744.0;
    const double s = fma(t, 2.0, magic);
    const double q = s - magic;
    const double g = fma(q, -0.5, t);
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
    uint64_t bs, bp;
    memcpy(&bs, &s, 8);
    memcpy(&bp, &p, 8);
    bp ^= (bs & 1ull) << 63;
    memcpy(&p, &bp, 8);
    return p;
}
double orc_cos_turns(double t) { return cos_turns(t); }

/* Turbulence of the torus plasma: delta = sum amp cos(2 pi (k.X + p)) with the wave vector and phase
 * in turns (k / 2 pi, phase / 2 pi, each a correctly rounded product with 1 / 2 pi), summed in the
 * CUDA kernel's order: 32 partial sums, partial l over modes l, l + 32, l + 64, ... in turn, then a
 * butterfly that adds partials l and l ^ o for o = 16, 8, 4, 2, 1. */
#define INV_2PI 0x1.45f306dc9c883p-3
static double torus_delta(const so_mode* md, int n, double X, double Y, double Z) {
    double part[32], next[32];
    for (int l = 0; l < 32; ++l) {
        double acc = 0.0;
        for (int m = l; m < n; m += 32) {
            const double kx = md[m].kx * INV_2PI, ky = md[m].ky * INV_2PI, kz = md[m].kz * INV_2PI;
            const double ph = md[m].phase * INV_2PI;
            acc = fma(md[m].amp, cos_turns(fma(kz, Z, fma(ky, Y, fma(kx, X, ph)))), acc);
        }
        part[l] = acc;
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int l = 0; l < 32; ++l) next[l] = part[l] + part[l ^ o];
        memcpy(part, next, sizeof part);
    }
    return part[0];
}

typedef struct {
    const so_scene* S;
    const so_frame* F;
    const so_plasma* pl; /* may be NULL (reference model) */
    const so_mode* modes;
} Ctx;

/* flow_step, emission.cuh:99-175, with the torus model as an alternative density/temperature. */
/* Baked flow turbulence (render.cu:447-460 bake, 594-620 set-up, emission.cuh:112-124 sampling).
 * Texel values are computed on demand with the bake's formula at the texel centre (the same values
 * as a full bake of the slice); the interpolation is the library kernels' FP32 trilinear (x, then
 * y, then z, each an fmaf), which the reference does in the texture unit with 8-bit weights. */
enum { TNPHI = 512, TNLR = 192, TNZ = 48, TNT = 24 };
void orc_turb_setup(so_scene* S) { /* render.cu:614-619 */
    S->turb_nt = TNT;
    S->turb_lr0 = (float)log(0.8 * S->rh);
    S->turb_lr1 = (float)log(S->r_flow_max * 1.05);
    S->turb_zmax = (float)fmin(2.0, 5.0 * S->h_r);
    S->turb_d0 = -250.f;
    S->turb_dd = 260.f / (TNT - 1);
}
static float turb_texel(const Ctx* X, int k, int l, int j, int i) { /* render.cu:449-460 */
    const so_scene* S = X->S;
    const so_frame* F = X->F;
    const float delta = S->turb_d0 + k * S->turb_dd;
    const double phi = (i + 0.5) / TNPHI * 2.0 * PI_D;
    const double R = exp(S->turb_lr0 + (j + 0.5) / TNLR * (S->turb_lr1 - S->turb_lr0));
    const double z = (-1.0 + 2.0 * (l + 0.5) / TNZ) * S->turb_zmax * R;
    const double r = sqrt(fma(R, R, z * z));
    const double t = (F->t - (F->r - r + 2.0 * log(F->r / r))) + delta;
    const float n = sheared_noise(S, R, phi, z, t, S->flow_turb_scale, S->flow_tcorr, S->seed ^ 0x51f15eedu);
    const float a = S->flow_turb_amp;
    return expf(a * n - 0.5f * a * a);
}
/* Layer l of baked slice k, texel (j, i) at out[j * 512 + i]: the bake's values, for the tests. */
void orc_turb_layer(const so_scene* S, const so_frame* F, int k, int l, float* out) {
    const Ctx X = {S, F, NULL, NULL};
    for (int j = 0; j < TNLR; ++j)
        for (int i = 0; i < TNPHI; ++i) out[j * TNPHI + i] = turb_texel(&X, k, l, j, i);
}
static float turb_fetch(const Ctx* X, int k, float x, float y, float z) {
    const float xb = (x - floorf(x)) * (float)TNPHI - 0.5f;
    const float yb = fminf(fmaxf(y * (float)TNLR - 0.5f, -1.f), (float)TNLR);
    const float zb = fminf(fmaxf(z * (float)TNZ - 0.5f, -1.f), (float)TNZ);
    const float fi = floorf(xb), fj = floorf(yb), fl = floorf(zb);
    const float a = xb - fi, b = yb - fj, c = zb - fl;
    const int i = (int)fi, j = (int)fj, l = (int)fl;
    const int i0 = i < 0 ? i + TNPHI : i, i1 = i + 1 >= TNPHI ? i + 1 - TNPHI : i + 1;
    const int j0 = j < 0 ? 0 : j > TNLR - 1 ? TNLR - 1 : j, j1 = j + 1 < 0 ? 0 : j + 1 > TNLR - 1 ? TNLR - 1 : j + 1;
    const int l0 = l < 0 ? 0 : l > TNZ - 1 ? TNZ - 1 : l, l1 = l + 1 < 0 ? 0 : l + 1 > TNZ - 1 ? TNZ - 1 : l + 1;
    float p, q;
    p = turb_texel(X, k, l0, j0, i0); q = turb_texel(X, k, l0, j0, i1);
    const float v00 = fmaf(a, q - p, p);
    p = turb_texel(X, k, l0, j1, i0); q = turb_texel(X, k, l0, j1, i1);
    const float v01 = fmaf(a, q - p, p);
    p = turb_texel(X, k, l1, j0, i0); q = turb_texel(X, k, l1, j0, i1);
    const float v10 = fmaf(a, q - p, p);
    p = turb_texel(X, k, l1, j1, i0); q = turb_texel(X, k, l1, j1, i1);
    const float v11 = fmaf(a, q - p, p);
    const float w0 = fmaf(b, v01 - v00, v00), w1 = fmaf(b, v11 - v10, v10);
    return fmaf(c, w1 - w0, w0);
}

static void flow_step(const Ctx* X, double r, double u, double phi, double t, double lam, double Ecam, double h,
                      double* dI, double* dtau) {
    const so_scene* S = X->S;
    *dI = 0.0;
    *dtau = 0.0;
    const double a = S->a;
    double s2 = fmax(fma(-u, u, 1.0), 1e-12), s = sqrt(s2);
    double R = r * s, z = r * u;
    if (r > S->r_flow_max || R < 1e-3) return;
    double ne, Th;
    int torus = X->pl && X->pl->model == SO_PLASMA_TORUS;
    if (torus) {
        double zh = u / X->pl->h_sph;
        double vert = exp(-0.5 * zh * zh);
        if (vert < 1e-7) return;
        double lx = log(r / S->rh);
        ne = S->n0 * exp(-X->pl->ne_index * lx) * vert;
        if (X->pl->n_modes > 0) {
            double Omf = S->flow_kep * keplerian_omega(S, fmax(R, S->r_isco));
            double phc = phi - Omf * (t + (X->F->r - r + 2.0 * log(X->F->r / r)));
            double d = torus_delta(X->modes, X->pl->n_modes, R * cos(phc), R * sin(phc), z);
            ne *= exp(d - 0.5 * X->pl->turb_rms * X->pl->turb_rms);
        }
        Th = (CGS_KB * X->pl->te0_kelvin / (CGS_ME * CGS_C * CGS_C)) * exp(-X->pl->te_index * lx);
    } else {
        double zh = z / (S->h_r * R);
        double vert = exp(-0.5 * zh * zh);
        if (vert < 1e-7) return;
        ne = S->n0 * exp(-S->n_index * log(r)) * vert;
        if (S->flow_turb_amp > 0.f && S->turb_nt > 0) {
            /* emission.cuh:112-124 */
            const double tref = X->F->t - (X->F->r - r + 2.0 * log(X->F->r / r));
            const float y = (float)((log(R) - S->turb_lr0) / (S->turb_lr1 - S->turb_lr0));
            const float x = (float)(phi * (0.5 / PI_D));
            const float w = (float)(0.5 + 0.5 * (z / R) / S->turb_zmax);
            float sl = (float)((t - tref) - S->turb_d0) / S->turb_dd;
            sl = fminf(fmaxf(sl, 0.f), (float)(TNT - 1) - 1e-4f);
            const int k = (int)sl;
            const float f = sl - (float)k;
            const float A = turb_fetch(X, k, x, y, w), B = turb_fetch(X, k + 1, x, y, w);
            ne *= fmaf(B - A, f, A);
        } else if (S->flow_turb_amp > 0.f) {
            float n = sheared_noise(S, R, phi, z, t, S->flow_turb_scale, S->flow_tcorr, S->seed ^ 0x51f15eedu);
            ne *= exp((double)(S->flow_turb_amp * n - 0.5f * S->flow_turb_amp * S->flow_turb_amp));
        }
        Th = 0.0;
    }
    double dr = r - S->rh;
    ne *= 1.0 - exp(-(dr * dr) / 0.25);
    if (ne < 1e-30) return;
    if (!torus) Th = S->theta0 * exp(-S->theta_index * log(r));
    double B = sqrt(8.0 * PI_D * ne * CGS_MP * CGS_C * CGS_C / (6.0 * r * S->beta_p));
    double r2 = r * r, a2 = a * a;
    double Sigma = fma(a2, u * u, r2), Delta = fma(r, r - 2.0, a2);
    double rpa = r2 + a2;
    double A = fma(rpa, rpa, -(a2 * Delta * s2));
    double g_tt = -(1.0 - 2.0 * r / Sigma), g_tph = -2.0 * a * r * s2 / Sigma, g_phph = A * s2 / Sigma;
    double omz = 2.0 * a * r / A;
    double Om = S->flow_kep * keplerian_omega(S, fmax(R, S->r_isco));
    double vmax = sqrt(Sigma * Delta / A) / sqrt(g_phph) * 0.999;
    Om = omz + fmax(-vmax, fmin(vmax, Om - omz));
    double norm = -fma(g_phph * Om, Om, fma(2.0 * g_tph, Om, g_tt));
    if (norm <= 0.0) return;
    double ut = 1.0 / sqrt(norm);
    double kdotu = ut * fma(-Om, lam, 1.0);
    double nu_f = S->nu_obs * Ecam * kdotu;
    double g = S->nu_obs / nu_f;
    double u_ph = ut * fma(g_phph, Om, g_tph);
    double kb = fma(-kdotu, u_ph, lam);
    double bb = fma(u_ph, u_ph, g_phph);
    double cosb = kb / (kdotu * sqrt(bb));
    double sinb = sqrt(fmax(fma(-cosb, cosb, 1.0), 1e-6));
    double nuc = CGS_QE * B / (2.0 * PI_D * CGS_ME * CGS_C);
    double nus = 2.0 / 9.0 * nuc * Th * Th * sinb;
    double Xs = nu_f / nus;
    double x3 = cbrt(Xs);
    double k2 = exp((double)table_lerp(S->k2_lntab, S->k2_n, S->k2_l0, S->k2_dl, (float)log(Th)));
    double brk = fma(1.887748625363387, sqrt(x3), sqrt(Xs));
    double j = ne * 1.4142135623730951 * PI_D * CGS_QE * CGS_QE * nus / (3.0 * k2 * CGS_C) * brk * brk * exp(-x3);
    double Te = Th * CGS_ME * CGS_C * CGS_C / CGS_KB;
    double hnu = CGS_H * nu_f / (CGS_KB * Te);
    double Bnu = 2.0 * CGS_H * nu_f * nu_f * nu_f / (CGS_C * CGS_C) / expm1(hnu);
    double alpha = j / Bnu;
    double dl = kdotu * Sigma * h * S->rg_cm;
    double tau = alpha * dl;
    *dtau = tau;
    *dI = g * g * g * Bnu * (-expm1(-tau));
}

/* hermite_d, trace.cuh:19-22, fixed fma order. */
static double hermite_d(double p0, double p1, double m0, double m1, double s) {
    double s2 = s * s, s3 = s2 * s;
    double c00 = fma(2.0, s3, fma(-3.0, s2, 1.0));
    double c10 = fma(-2.0, s2, s3) + s;
    double c01 = fma(-2.0, s3, 3.0 * s2);
    double c11 = s3 - s2;
    return fma(c11, m1, fma(c01, p1, fma(c10, m0, c00 * p0)));
}

/* escape_angles, trace.cuh:49-55. */
static void escape_angles(const double* y, const double* k, double* th, double* ph) {
    double s = sqrt(fmax(fma(-y[2], y[2], 1.0), 1e-30));
    double t0 = acos(fmax(-1.0, fmin(1.0, y[2])));
    double dthdr = (-y[3] / s) / y[1], dphdr = k[4] / y[1];
    *th = fma(y[0], dthdr, t0);
    *ph = fma(y[0], dphdr, y[4]);
}

typedef struct {
    float acc[4];
    int fate, ncross, n_acc, n_att;
    double th, ph;
    double cr[3], cg[3];
} RayOut;

/* trace_ray, trace.cuh:62-165 (sky lookups excluded: the sky texture is outside this path). */
/* Sky of the visible mode (trace.cuh:24-43, 149-161) for an analytic star map: brightness
 * s(u, v) = c0 + cu u + cv v at a fixed temperature T (the texture unit's filtering of a sampled map
 * has no CPU form; a constant map, which every filter returns unchanged, checks the rest exactly). */
static double g_sky[4] = {0.0, 0.0, 0.0, 0.0}; /* c0, cu, cv, T; c0 = cu = cv = 0: no sky */
void orc_set_sky(double c0, double cu, double cv, double T) {
    g_sky[0] = c0;
    g_sky[1] = cu;
    g_sky[2] = cv;
    g_sky[3] = T;
}
static void sky_uv(const so_scene* S, double th, double ph, float* u, float* v) { /* trace.cuh:24-33 */
    const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
    const double dx = st * cp, dy = st * sp, dz = ct;
    const so_mat3* m = &S->sky_rot;
    const double gx = fma(m->r0.z, dz, fma(m->r0.y, dy, m->r0.x * dx));
    const double gy = fma(m->r1.z, dz, fma(m->r1.y, dy, m->r1.x * dx));
    const double gz = fma(m->r2.z, dz, fma(m->r2.y, dy, m->r2.x * dx));
    const double l = atan2(gy, gx), b = asin(fmax(-1.0, fmin(1.0, gz)));
    float uu = (float)(0.5 - l * (0.5 / PI_D));
    uu -= floorf(uu);
    *u = uu;
    *v = (float)(0.5 - b / PI_D);
}

static void trace_ray(const Ctx* X, double x, double yv, RayOut* o) {
    const so_scene* S = X->S;
    const so_frame* F = X->F;
    const double a = S->a;
    memset(o, 0, sizeof *o);
    double cxx = F->cx + x, cyy = F->cy + yv;
    so_vec3 v = {fma(F->U.x, cyy, fma(F->R.x, cxx, F->F.x)), fma(F->U.y, cyy, fma(F->R.y, cxx, F->F.y)),
                 fma(F->U.z, cyy, fma(F->R.z, cxx, F->F.z))};
    double il = 1.0 / sqrt(dot3(v, v));
    so_vec3 d = {v.x * il, v.y * il, v.z * il};
    RayC c;
    double y[6], k1[6], yn[6], k7[6];
    camera_photon(a, &F->kp, F->ph, F->t, d, F->beta, &c, y);
    const double lam = c.lam, eta = c.eta, Ecam = c.E;
    rhs(&c, y, k1);
    double h = initial_step(y);
    double trans = 1.0;
    int ncross = 0;
    double psi = 0.0;
    double sp = sqrt(fmax(fma(-y[2], y[2], 1.0), 0.0));
    so_vec3 pprev = {sp * cos(y[4]), sp * sin(y[4]), y[2]};
    o->fate = 0;
    const int radio = S->mode == SO_MODE_RADIO;
    for (int it = 0; it < S->max_steps; ++it) {
        double hc = h;
        if (radio && S->flow_on && y[0] < S->r_flow_max) {
            double s = sqrt(fmax(fma(-y[2], y[2], 1.0), 0.0));
            double cap = S->step_frac * fmin(y[0] / (fabs(y[1]) + 1e-30), fmax(s, 0.05) / (fabs(y[3]) + 1e-30));
            hc = fmin(hc, cap);
        } else if (S->disk_on) {
            hc = fmin(hc, 0.3 / (fabs(y[3]) + 1e-30));
        }
        ++o->n_att;
        double err = dp54(&c, y, k1, hc, S->tol, yn, k7);
        if (!(err <= 1.0)) {
            h = hc * fmax(0.2, 0.9 * so_rpow5(fmax(err, 1e-30)));
            if (!(err == err)) h = hc * 0.1;
            continue;
        }
        ++o->n_acc;
        if (radio) {
            double sn = sqrt(fmax(fma(-yn[2], yn[2], 1.0), 0.0));
            so_vec3 pn = {sn * cos(yn[4]), sn * sin(yn[4]), yn[2]};
            so_vec3 cr = cross3(pprev, pn);
            psi += atan2(sqrt(dot3(cr, cr)), dot3(pprev, pn));
            pprev = pn;
        }
        if ((y[2] > 0.0) != (yn[2] > 0.0)) {
            ++ncross;
            int rec = ncross <= 3;
            if (S->disk_on || rec) {
                double lo = 0.0, hi = 1.0, u0 = y[2], u1 = yn[2], m0 = y[3] * hc, m1 = yn[3] * hc;
                for (int b = 0; b < 40; ++b) {
                    double mid = 0.5 * (lo + hi);
                    double um = hermite_d(u0, u1, m0, m1, mid);
                    if ((um > 0.0) == (u0 > 0.0)) lo = mid;
                    else hi = mid;
                }
                double sc = 0.5 * (lo + hi);
                double rc = hermite_d(y[0], yn[0], y[1] * hc, yn[1] * hc, sc);
                if (rec) {
                    o->cr[ncross - 1] = rc;
                    o->cg[ncross - 1] = crossing_g(S, rc, lam, Ecam);
                }
                if (S->disk_on) {
                    double pc = hermite_d(y[4], yn[4], k1[4] * hc, k7[4] * hc, sc);
                    double tc = hermite_d(y[5], yn[5], k1[5] * hc, k7[5] * hc, sc);
                    float cs[4];
                    disk_shade(S, rc, pc, tc, lam, eta, Ecam, cs);
                    if (cs[3] > 0.f) {
                        float tf = (float)trans;
                        o->acc[0] += tf * cs[0];
                        o->acc[1] += tf * cs[1];
                        o->acc[2] += tf * cs[2];
                        o->acc[3] += tf * cs[1] * (float)(ncross - 1);
                        trans *= 1.0 - cs[3];
                        if (trans < 1e-4) {
                            o->fate = -1;
                            break;
                        }
                    }
                }
            }
        }
        if (radio && S->flow_on && yn[0] < S->r_flow_max) {
            double dI, dtau;
            flow_step(X, yn[0], yn[2], yn[4], yn[5], lam, Ecam, hc, &dI, &dtau);
            float cc = (float)(trans * dI);
            int n = (int)(psi * (1.0 / PI_D));
            o->acc[0] += cc;
            if (n == 1) o->acc[1] += cc;
            else if (n == 2) o->acc[2] += cc;
            else if (n >= 3) o->acc[3] += cc;
            trans *= exp(-dtau);
            if (trans < 1e-5) {
                o->fate = -1;
                break;
            }
        }
        for (int i = 0; i < 6; ++i) {
            y[i] = yn[i];
            k1[i] = k7[i];
        }
        project_radial(&c, y, k1);
        h = hc * fmin(5.0, fmax(0.2, 0.9 * so_rpow5(fmax(err, 1e-30))));
        if (y[0] < S->r_stop) {
            o->fate = -1;
            break;
        }
        if (y[0] > S->r_escape && y[1] > 0.0) {
            o->fate = 1;
            escape_angles(y, k1, &o->th, &o->ph);
            if (!radio && S->sky_on && (g_sky[0] != 0.0 || g_sky[1] != 0.0 || g_sky[2] != 0.0)) {
                float u, v;
                sky_uv(S, o->th, o->ph, &u, &v);
                const float s = (float)(g_sky[0] + g_sky[1] * u + g_sky[2] * v);
                if (s > 0.f) {
                    const float T = (float)g_sky[3];
                    const float g = (float)(1.0 / c.E);
                    float xyz[3];
                    blackbody_xyz(S, g * T, xyz);
                    const float sc = s * S->sky_scale, tf = (float)trans;
                    o->acc[0] += tf * (xyz[0] * sc);
                    o->acc[1] += tf * (xyz[1] * sc);
                    o->acc[2] += tf * (xyz[2] * sc);
                }
            }
            break;
        }
    }
    o->ncross = ncross;
}

/* ---- exported entry points ------------------------------------------------------------------ */
typedef struct {
    const Ctx* X;
    int n;
    const double* x;
    const double* y;
    const so_rays_out* out;
    int t0, stride;
} Job;

static void store(const so_rays_out* out, int i, const RayOut* o) {
    if (out->fate) out->fate[i] = (int8_t)o->fate;
    if (out->ncross) out->ncross[i] = (int8_t)(o->ncross > 127 ? 127 : o->ncross);
    if (out->theta) out->theta[i] = o->fate == 1 ? o->th : 0.0;
    if (out->phi) out->phi[i] = o->fate == 1 ? o->ph : 0.0;
    if (out->I) memcpy(out->I + 4 * (size_t)i, o->acc, 16);
    if (out->n_accepted) out->n_accepted[i] = o->n_acc;
    if (out->n_attempts) out->n_attempts[i] = o->n_att;
    if (out->cross_r) memcpy(out->cross_r + 3 * (size_t)i, o->cr, 24);
    if (out->cross_g) memcpy(out->cross_g + 3 * (size_t)i, o->cg, 24);
}

static void* job_run(void* p) {
    Job* j = (Job*)p;
    for (int i = j->t0; i < j->n; i += j->stride) {
        RayOut o;
        trace_ray(j->X, j->x[i], j->y[i], &o);
        store(j->out, i, &o);
    }
    return NULL;
}

/* The oracle's noise at n points (fbm3, device_util.cuh:61-72; sheared_noise, emission.cuh:34-51),
   for the function-level pins against the reference's own code. */
void orc_fbm3(int n, const float* x, const float* y, const float* z, int oct, uint32_t seed, float* out) {
    for (int i = 0; i < n; ++i) out[i] = fbm3(x[i], y[i], z[i], oct, seed);
}
void orc_sheared_noise(const so_scene* S, int n, const double* R, const double* phi, const double* z, const double* t,
                       float scale, float tcorr, uint32_t seed, float* out) {
    for (int i = 0; i < n; ++i) out[i] = sheared_noise(S, R[i], phi[i], z[i], t[i], scale, tcorr, seed);
}

/* trace_ray over n explicit tangent-plane points (x[i], y[i]) with nthreads host threads. */
int orc_trace_rays(const so_scene* S, const so_plasma* pl, const so_mode* modes, const so_frame* F, int n,
                   const double* x, const double* y, const so_rays_out* out, int nthreads) {
    if (!S || !F || !out || n < 0 || (n > 0 && (!x || !y))) return SO_ERR_ARG;
    Ctx X = {S, F, pl, modes};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    Job jobs[256];
    for (int t = 0; t < nthreads; ++t) {
        Job j = {&X, n, x, y, out, t, nthreads};
        jobs[t] = j;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, job_run, &jobs[t]);
    job_run(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
    return SO_OK;
}

/* One camera sample of pixel (px, py), render.cu:70-85 (pixel_seed + R2 jitter + trace_ray).
 * spp samples per pixel are summed in float in sample order, as k_pass1 (render.cu:89-128). */
typedef struct {
    const Ctx* X;
    float* accum;
    float* ystat;
    long long* lim;
    long long* att;
    int t0, stride;
    int jitter;
} PixJob;

static void* pix_run(void* p) {
    PixJob* j = (PixJob*)p;
    const so_frame* F = j->X->F;
    const int radio = j->X->S->mode == SO_MODE_RADIO;
    long long lim = 0, att = 0;
    for (int pix = j->t0; pix < F->W * F->H; pix += j->stride) {
        int px = pix % F->W, py = pix / F->W;
        uint32_t hs = pcg((uint32_t)pix * 0x9E3779B9u ^ F->seed);
        float r0 = rnd(&hs), r1 = rnd(&hs);
        float a[4] = {0, 0, 0, 0};
        float ys = 0.f, yq = 0.f;
        for (int s = 0; s < F->spp; ++s) {
            float jx = 0.5f, jy = 0.5f;
            if (j->jitter) r2_sample((uint32_t)s, r0, r1, &jx, &jy);
            double tx = (px + jx - 0.5 * F->W) * F->pix;
            double ty = (0.5 * F->H - (py + jy)) * F->pix;
            RayOut o;
            trace_ray(j->X, tx, ty, &o);
            if (o.fate == 0) ++lim;
            att += o.n_att;
            for (int c = 0; c < 4; ++c) a[c] += o.acc[c];
            float Y = radio ? o.acc[0] : o.acc[1];
            ys += Y;
            yq += Y * Y;
        }
        memcpy(j->accum + 4 * (size_t)pix, a, 16);
        if (j->ystat) {
            j->ystat[2 * (size_t)pix] = ys;
            j->ystat[2 * (size_t)pix + 1] = yq;
        }
    }
    j->lim[0] = lim;
    j->att[0] = att;
    return NULL;
}

/* Pass 1 of a frame: W x H pixels of F, spp samples each (jitter = 1: R2 jitter as the reference;
 * jitter = 0: pixel centres).  accum: W*H*4 sums, ystat: W*H*2 (sum Y, sum Y^2) or NULL. */
int orc_render_pass1(const so_scene* S, const so_plasma* pl, const so_mode* modes, const so_frame* F, int jitter,
                     float* accum, float* ystat, long long* step_limited, long long* attempts, int nthreads) {
    if (!S || !F || !accum || F->W <= 0 || F->H <= 0 || F->spp <= 0) return SO_ERR_ARG;
    Ctx X = {S, F, pl, modes};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    PixJob jobs[256];
    long long lim[256], att[256];
    for (int t = 0; t < nthreads; ++t) {
        PixJob j = {&X, accum, ystat, &lim[t], &att[t], t, nthreads, jitter};
        jobs[t] = j;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, pix_run, &jobs[t]);
    pix_run(&jobs[0]);
    long long L = lim[0], A = att[0];
    for (int t = 1; t < nthreads; ++t) {
        pthread_join(th[t], NULL);
        L += lim[t];
        A += att[t];
    }
    if (step_limited) *step_limited = L;
    if (attempts) *attempts = A;
    return SO_OK;
}

/* Pass-2 chunks (render.cu:196-224): entry e is `count` consecutive R2-jittered samples s0[e] ..
 * s0[e] + count - 1 of pixel pix[e], summed in float in sample order into out[4 e .. 4 e + 3].  The
 * reference adds such chunk sums to their pixels with float atomics; the CUDA path adds them in
 * chunk order, which the caller repeats. */
typedef struct {
    const Ctx* X;
    long long n;
    const long long* pix;
    const int* s0;
    int count;
    float* out;
    long long* lim;
    int t0, stride;
} ChunkJob;

static void* chunk_run(void* p) {
    ChunkJob* j = (ChunkJob*)p;
    const so_frame* F = j->X->F;
    long long lim = 0;
    for (long long e = j->t0; e < j->n; e += j->stride) {
        const int pix = (int)j->pix[e];
        const int px = pix % F->W, py = pix / F->W;
        uint32_t hs = pcg((uint32_t)pix * 0x9E3779B9u ^ F->seed);
        float r0 = rnd(&hs), r1 = rnd(&hs);
        float a[4] = {0, 0, 0, 0};
        for (int i = 0; i < j->count; ++i) {
            float jx, jy;
            r2_sample((uint32_t)(j->s0[e] + i), r0, r1, &jx, &jy);
            double tx = (px + jx - 0.5 * F->W) * F->pix;
            double ty = (0.5 * F->H - (py + jy)) * F->pix;
            RayOut o;
            trace_ray(j->X, tx, ty, &o);
            if (o.fate == 0) ++lim;
            for (int c = 0; c < 4; ++c) a[c] += o.acc[c];
        }
        memcpy(j->out + 4 * (size_t)e, a, 16);
    }
    j->lim[0] = lim;
    return NULL;
}

int orc_render_chunks(const so_scene* S, const so_plasma* pl, const so_mode* modes, const so_frame* F, long long n,
                      const long long* pix, const int* s0, int count, float* out, long long* step_limited,
                      int nthreads) {
    if (!S || !F || n < 0 || (n > 0 && (!pix || !s0 || !out)) || count <= 0 || F->W <= 0 || F->H <= 0)
        return SO_ERR_ARG;
    for (long long e = 0; e < n; ++e)
        if (pix[e] < 0 || pix[e] >= (long long)F->W * F->H || s0[e] < 0) return SO_ERR_ARG;
    Ctx X = {S, F, pl, modes};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    ChunkJob jobs[256];
    long long lim[256];
    for (int t = 0; t < nthreads; ++t) {
        ChunkJob j = {&X, n, pix, s0, count, out, &lim[t], t, nthreads};
        jobs[t] = j;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, chunk_run, &jobs[t]);
    chunk_run(&jobs[0]);
    long long L = lim[0];
    for (int t = 1; t < nthreads; ++t) {
        pthread_join(th[t], NULL);
        L += lim[t];
    }
    if (step_limited) *step_limited = L;
    return SO_OK;
}

/* vacuum_fate, kerr.hpp:184-203 (the controller with so_rpow5, the same fma placement as above). */
int orc_vacuum_fate(double a, const so_frame* F, so_vec3 d, double tol, double r_escape, int max_steps) {
    RayC c;
    double y[6], k1[6], yn[6], k7[6];
    camera_photon(a, &F->kp, F->ph, F->t, d, F->beta, &c, y);
    double rh = orc_horizon_radius(a);
    rhs(&c, y, k1);
    double h = initial_step(y);
    for (int it = 0; it < max_steps; ++it) {
        double err = dp54(&c, y, k1, h, tol, yn, k7);
        if (err > 1.0) {
            h *= fmax(0.2, 0.9 * so_rpow5(err));
            continue;
        }
        for (int i = 0; i < 6; ++i) {
            y[i] = yn[i];
            k1[i] = k7[i];
        }
        project_radial(&c, y, k1);
        h *= fmin(5.0, fmax(0.2, 0.9 * so_rpow5(fmax(err, 1e-30))));
        if (y[0] < rh * 1.0001 + 1e-3) return -1;
        if (y[0] > r_escape && y[1] > 0.0) return 1;
    }
    return 0;
}

/* find_critical_point, shot.cpp:148-164: bisection on the vacuum fate along image direction psi. */
double orc_find_critical_point(const so_frame* F, double a, double psi, double cam_r) {
    double lo = 0.5, hi = 15.0;
    so_vec3 d;
    for (int pass = 0; pass < 2; ++pass) {
        double rho = pass == 0 ? lo : hi;
        double x = rho * cos(psi) / cam_r, yv = rho * sin(psi) / cam_r;
        so_vec3 v = {fma(F->U.x, yv, fma(F->R.x, x, F->F.x)), fma(F->U.y, yv, fma(F->R.y, x, F->F.y)),
                     fma(F->U.z, yv, fma(F->R.z, x, F->F.z))};
        double il = 1.0 / sqrt(dot3(v, v));
        d.x = v.x * il; d.y = v.y * il; d.z = v.z * il;
        int f = orc_vacuum_fate(a, F, d, 1e-12, 200.0, 2000000);
        if ((pass == 0 && f != -1) || (pass == 1 && f != 1)) return 0.0;
    }
    for (int it = 0; it < 64; ++it) {
        double mid = 0.5 * (lo + hi);
        double x = mid * cos(psi) / cam_r, yv = mid * sin(psi) / cam_r;
        so_vec3 v = {fma(F->U.x, yv, fma(F->R.x, x, F->F.x)), fma(F->U.y, yv, fma(F->R.y, x, F->F.y)),
                     fma(F->U.z, yv, fma(F->R.z, x, F->F.z))};
        double il = 1.0 / sqrt(dot3(v, v));
        d.x = v.x * il; d.y = v.y * il; d.z = v.z * il;
        if (orc_vacuum_fate(a, F, d, 1e-12, 200.0, 2000000) == 1) hi = mid;
        else lo = mid;
    }
    return 0.5 * (lo + hi);
}

/* critical_curve_point, kerr.hpp:210-220 (Bardeen 1973). */
int orc_critical_curve_point(double a, double theta_o, double rp, double* alpha, double* beta_plus) {
    double D = rp * rp - 2.0 * rp + a * a;
    double lam = a + rp / a * (rp - 2.0 * D / (rp - 1.0));
    double eta = rp * rp * rp / (a * a) * (4.0 * D / ((rp - 1.0) * (rp - 1.0)) - rp);
    double so = sin(theta_o), co = cos(theta_o);
    double b2 = eta + a * a * co * co - lam * lam * co * co / (so * so);
    if (b2 < 0.0) return 0;
    *alpha = -lam / so;
    *beta_plus = sqrt(b2);
    return 1;
}

/* Radial-constraint drift of the self-test (main.cpp:352-371): worst |R - r'^2| / r^4 over up to
 * max_acc accepted steps without projection. */
double orc_radial_drift(double a, double r0, double th0, so_vec3 dir, double tol, int max_acc, int* steps) {
    so_frame F;
    memset(&F, 0, sizeof F);
    orc_kerr_point(a, r0, th0, &F.kp);
    RayC c;
    double y[6], k1[6], yn[6], k7[6];
    double il = 1.0 / sqrt(dot3(dir, dir));
    so_vec3 d = {dir.x * il, dir.y * il, dir.z * il};
    so_vec3 zero = {0, 0, 0};
    camera_photon(a, &F.kp, 0.0, 0.0, d, zero, &c, y);
    rhs(&c, y, k1);
    double h = initial_step(y), worst = 0.0;
    int n = 0;
    double rh = orc_horizon_radius(a);
    for (int it = 0; it < 200000 && n < max_acc; ++it) {
        double err = dp54(&c, y, k1, h, tol, yn, k7);
        if (err > 1) {
            h *= fmax(0.2, 0.9 * so_rpow5(err));
            continue;
        }
        for (int i = 0; i < 6; ++i) {
            y[i] = yn[i];
            k1[i] = k7[i];
        }
        h *= fmin(5.0, fmax(0.2, 0.9 * so_rpow5(fmax(err, 1e-30))));
        ++n;
        double r = y[0];
        double P = fma(r, r, c.CP), D = fma(r, r - 2.0, c.A2);
        double R = fma(P, P, -(D * c.K));
        double r2 = r * r;
        double w = fabs(R - y[1] * y[1]) / (r2 * r2);
        if (w > worst) worst = w;
        if (y[0] < rh + 0.01 || y[0] > 1e4) break;
    }
    if (steps) *steps = n;
    return worst;
}
