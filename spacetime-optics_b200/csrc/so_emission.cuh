// so_emission.cuh -- emitting matter along the ray (device code): the reference's hot-flow
// synchrotron transfer and thin disk, the torus plasma with Fourier-mode turbulence, and the noise /
// hash / table helpers they use.
//
// Follows blackholes/src/emission.cuh (keplerian_omega :20, sheared_noise :34-51, disk_temperature
// :53-56, disk_shade :59-86, bessel_k2_inv :89-91, flow_step :99-175) and
// blackholes/src/device_util.cuh (pcg :15-19, rnd :20-23, r2_sample :25-30, grad3 / gnoise / fbm3
// :32-72, table_lerp :74-80, blackbody_xyz :82-90).  Float stages stay float, as in the reference;
// rsqrtf of sheared_noise is written 1/sqrtf and __expf is expf so that the CPU oracle can follow the
// same operations.
#pragma once
#include "so_kerr.cuh"
#include "so_launch.h"

namespace so {

namespace cgs {
constexpr double C = 2.99792458e10;
constexpr double KB = 1.380649e-16;
constexpr double H = 6.62607015e-27;
constexpr double ME = 9.1093837e-28;
constexpr double MP = 1.67262192e-24;
constexpr double QE = 4.80320471e-10;
}  // namespace cgs

__device__ __forceinline__ uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
__device__ __forceinline__ float rnd(uint32_t& s) {
    s = pcg(s);
    return (float)(s >> 8) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ float frac1(float x) { return x - floorf(x); }
__device__ __forceinline__ void r2_sample(uint32_t n, float r0, float r1, float* x, float* y) {
    const double a1 = 0.7548776662466927, a2 = 0.5698402909980532;
    *x = frac1(r0 + (float)fmod(n * a1, 1.0));
    *y = frac1(r1 + (float)fmod(n * a2, 1.0));
}
__device__ __forceinline__ float lerpf_(float a, float b, float t) { return a + (b - a) * t; }

// Tangent-plane point of sample s of pixel q in a W x H frame: pixel_seed + R2 jitter + sample_pixel
// (render.cu:70-85), or the pixel centre when jitter == 0.
__device__ __forceinline__ void sample_point(int W, int H, int jitter, const so_frame& F, long long q, int s,
                                             double* x, double* yv) {
    int px = (int)(q % W), py = (int)(q / W);
    float jx = 0.5f, jy = 0.5f;
    if (jitter) {
        uint32_t h = pcg((uint32_t)q * 0x9E3779B9u ^ F.seed);
        float r0 = rnd(h), r1 = rnd(h);
        r2_sample((uint32_t)s, r0, r1, &jx, &jy);
    }
    *x = (px + jx - 0.5 * W) * F.pix;
    *yv = (0.5 * H - (py + jy)) * F.pix;
}

// The twelve edge gradients of grad3's switch (device_util.cuh:32-41), selected without a branch (a 12-way
// switch on a hash diverges in every warp): case g < 8 takes fx first, else fy; g < 4 takes fy
// second, else fz; bit 0 of g negates the first term, bit 1 the second.  Same sums, bit for bit
// (a - b is a + (-b) in IEEE arithmetic).
__device__ __forceinline__ float grad3(int ix, int iy, int iz, uint32_t seed, float fx, float fy, float fz) {
    uint32_t h = pcg((uint32_t)ix * 73856093u ^ pcg((uint32_t)iy * 19349663u ^ pcg((uint32_t)iz * 83492791u ^ seed)));
    const uint32_t g = h % 12u;
    const float u = g < 8u ? fx : fy;
    const float v = g < 4u ? fy : fz;
    return ((g & 1u) ? -u : u) + ((g & 2u) ? -v : v);
}
static __device__ float gnoise(float x, float y, float z, uint32_t seed) {
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
static __device__ float fbm3(float x, float y, float z, int oct, uint32_t seed) {
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
__device__ __forceinline__ float table_lerp(const float* t, int n, float x0, float dx, float x) {
    float f = (x - x0) / dx;
    f = fminf(fmaxf(f, 0.f), (float)(n - 2) + 0.9999f);
    int i = (int)f;
    f -= (float)i;
    float t0 = __ldg(t + i), t1 = __ldg(t + i + 1);
    return t0 + (t1 - t0) * f;
}
__device__ __forceinline__ void blackbody_xyz(const so_scene& S, float T, float* xyz) {
    float f = (logf(fmaxf(T, 1.f)) - S.bb_l0) / S.bb_dl;
    f = fminf(fmaxf(f, 0.f), (float)(S.bb_n - 2) + 0.9999f);
    int i = (int)f;
    f -= (float)i;
    const float* p = S.bb_xyz + 3 * i;
    float p0 = __ldg(p), p1 = __ldg(p + 1), p2 = __ldg(p + 2), p3 = __ldg(p + 3), p4 = __ldg(p + 4), p5 = __ldg(p + 5);
    xyz[0] = p0 + (p3 - p0) * f;
    xyz[1] = p1 + (p4 - p1) * f;
    xyz[2] = p2 + (p5 - p2) * f;
}

__device__ __forceinline__ double keplerian_omega(double a, double R) { return 1.0 / fma(R, sqrt(R), a); }

static __device__ float sheared_noise(const so_scene& S, double R, double phi, double z, double t, float scale, float tcorr,
                               uint32_t seed) {
    double Om = keplerian_omega(S.a, fmax(R, S.r_isco));
    double P = 6.283185307179586 / Om * (double)tcorr;
    double s = t / P;
    double k = floor(s);
    float f = (float)(s - k);
    float acc = 0.f;
    for (int j = 0; j < 2; ++j) {
        double tb = (k + j) * P;
        double ph = phi - Om * (t - tb);
        float inv = 1.f / (scale * (float)R);
        double sp, cp;
        sincos(ph, &sp, &cp);
        float x = (float)(R * cp) * inv, y = (float)(R * sp) * inv, zz = (float)z * inv * 2.f;
        float n = fbm3(x, y, zz, 4, seed + 7919u * (uint32_t)(long long)(k + j));
        float w = j == 0 ? 1.f - f : f;
        acc += w * n;
    }
    return acc * (1.f / sqrtf((1.f - f) * (1.f - f) + f * f));
}

// u^t of a circular prograde equatorial orbit (emission.cuh:65-68).
__device__ __forceinline__ double circ_ut(double a, double r) {
    double sr = sqrt(r);
    double q = sqrt(sr);
    return fma(r, sr, a) / (q * q * q * sqrt(fmax(fma(r, sr, -3.0 * sr) + 2.0 * a, 1e-12)));
}

static __device__ void disk_shade(const so_scene& S, double r, double phi, double t, double lam, double eta, double Ecam,
                           float* out) {
    out[0] = out[1] = out[2] = out[3] = 0.f;
    if (r < S.disk_rin || r > S.disk_rout) return;
    double ut = circ_ut(S.a, r);
    double Om = keplerian_omega(S.a, r);
    double kdotu = ut * fma(-Om, lam, 1.0);
    double g = 1.0 / (Ecam * kdotu);
    float T = expf(table_lerp(S.disk_lnT, S.disk_n, (float)S.disk_lr0, (float)S.disk_dlr, (float)log(r)));
    float m = 1.f;
    if (S.disk_turb_amp > 0.f) {
        float n = sheared_noise(S, r, phi, 0.0, t, S.disk_turb_scale, S.disk_tcorr, S.seed);
        m = expf(S.disk_turb_amp * n - 0.5f * S.disk_turb_amp * S.disk_turb_amp);
    }
    T *= sqrtf(sqrtf(m));
    float ld = 1.f;
    if (S.disk_ld > 0.f) {
        float mu = (float)fmin(sqrt(fmax(eta, 0.0)) / (r * kdotu), 1.0);
        ld = (1.f + 2.06f * mu) / (1.f + 2.06f * 2.f / 3.f);
    }
    float fc = S.disk_fcol;
    float xyz[3];
    blackbody_xyz(S, (float)g * T * fc, xyz);
    float s = ld / (fc * fc * fc * fc);
    float e0 = (float)(0.75 * S.disk_rout), e1 = (float)S.disk_rout, xr = (float)r;
    float tt = (xr - e0) / (e1 - e0);
    tt = tt < 0.f ? 0.f : (tt > 1.f ? 1.f : tt);
    float edge = 1.f - tt * tt * (3.f - 2.f * tt);
    out[0] = xyz[0] * s * edge;
    out[1] = xyz[1] * s * edge;
    out[2] = xyz[2] * s * edge;
    out[3] = edge;
}

// Redshift factor of a circular prograde equatorial emitter at r for this photon (0 inside the ISCO).
__device__ __forceinline__ double crossing_g(const so_scene& S, double r, double lam, double Ecam) {
    if (r < S.r_isco) return 0.0;
    double ut = circ_ut(S.a, r);
    double kdotu = ut * fma(-keplerian_omega(S.a, r), lam, 1.0);
    return 1.0 / (Ecam * kdotu);
}

// Torus plasma parameters resolved for the kernel.
struct TorusParams {
    int on;          // SO_PLASMA_TORUS
    int n_modes;
    double ne_index, te_index, h_sph, theta_e0, half_var;
};

// Fourier-mode turbulence delta(X) = sum amp cos(k.X + phase), modes in shared memory (SoA, double),
// wave vector and phase stored in turns (multiplied by kInvTwoPi) for cos_turns.
constexpr double kInvTwoPi = 0x1.45f306dc9c883p-3;  // 1 / (2 pi), correctly rounded
struct ModesSmem {
    const double* kx;
    const double* ky;
    const double* kz;
    const double* ph;
    const double* amp;
};

// flow_step (emission.cuh:99-175): source term g^3 S (1 - e^-dtau) and optical depth of a Mino
// step h at (r, u, phi, t).  The torus model replaces the density / temperature / turbulence
// lines; the rest of the physics is the reference's.  The torus pattern is advected by the flow to
// the emission time counted from the radial light-travel time to the camera at rcam,
// t + (rcam - r + 2 ln(rcam / r)) (the retarded time of emission.cuh:26-28 plus the frame time):
// the raw coordinate time is ~ -rcam at the hole, which would put a factor rcam on every rounding
// error of the advected phase.
//
// Where the torus turbulence is needed for a flow step at (r, u, phi, t): false when flow_step
// returns before using it (only those flow steps can change the transfer); else the advected
// azimuth phc of the sum's position.
__device__ __forceinline__ bool torus_phase(const so_scene& S, const TorusParams& tp, double rcam, double r, double u,
                                            double phi, double t, double* phc) {
    if (!tp.on || tp.n_modes <= 0) return false;
    double s2 = fmax(fma(-u, u, 1.0), 1e-12), s = sqrt(s2);
    double R = r * s;
    if (r > S.r_flow_max || R < 1e-3) return false;
    double zh = u / tp.h_sph;
    if (exp(-0.5 * zh * zh) < 1e-7) return false;
    double Omf = S.flow_kep * keplerian_omega(S.a, fmax(R, S.r_isco));
    *phc = phi - Omf * (t + (rcam - r + 2.0 * log(rcam / r)));
    return true;
}
// The Cartesian position (X, Y, Z) of the sum at (r, u) and advected azimuth phc.
__device__ __forceinline__ void torus_xyz(double r, double u, double phc, double* X, double* Y, double* Z) {
    double s2 = fmax(fma(-u, u, 1.0), 1e-12), s = sqrt(s2);
    double R = r * s;
    double sp, cp;
    sincos(phc, &sp, &cp);
    *X = R * cp;
    *Y = R * sp;
    *Z = r * u;
}
__device__ __forceinline__ bool torus_position(const so_scene& S, const TorusParams& tp, double rcam, double r,
                                               double u, double phi, double t, double* X, double* Y, double* Z) {
    double phc;
    if (!torus_phase(S, tp, rcam, r, u, phi, t, &phc)) return false;
    torus_xyz(r, u, phc, X, Y, Z);
    return true;
}

// Trilinear sample of one baked turbulence slice at normalised coordinates (x = phi / 2 pi, wrapped;
// y = ln R, z = z / R, clamped to the edge texels), texel centres at (i + 1/2) / N as for linear
// texture filtering with normalised coordinates.  The reference fetches through the texture unit
// (emission.cuh:121-122), whose weights have 8 fractional bits; here the weights are FP32 and the
// three interpolations are explicit fmaf in a fixed order (x, then y, then z), which the CPU oracle
// repeats.
__device__ __forceinline__ float turb_fetch(const float* __restrict__ slice, float x, float y, float z) {
    const float xb = (x - floorf(x)) * (float)TURB_NPHI - 0.5f;
    const float yb = fminf(fmaxf(y * (float)TURB_NLR - 0.5f, -1.f), (float)TURB_NLR);
    const float zb = fminf(fmaxf(z * (float)TURB_NZ - 0.5f, -1.f), (float)TURB_NZ);
    const float fi = floorf(xb), fj = floorf(yb), fl = floorf(zb);
    const float a = xb - fi, b = yb - fj, c = zb - fl;
    const int i = (int)fi, j = (int)fj, l = (int)fl;
    const int i0 = i < 0 ? i + TURB_NPHI : i, i1 = i + 1 >= TURB_NPHI ? i + 1 - TURB_NPHI : i + 1;
    const int j0 = min(max(j, 0), TURB_NLR - 1), j1 = min(max(j + 1, 0), TURB_NLR - 1);
    const int l0 = min(max(l, 0), TURB_NZ - 1), l1 = min(max(l + 1, 0), TURB_NZ - 1);
    const float* p00 = slice + ((size_t)l0 * TURB_NLR + j0) * TURB_NPHI;
    const float* p01 = slice + ((size_t)l0 * TURB_NLR + j1) * TURB_NPHI;
    const float* p10 = slice + ((size_t)l1 * TURB_NLR + j0) * TURB_NPHI;
    const float* p11 = slice + ((size_t)l1 * TURB_NLR + j1) * TURB_NPHI;
    const float v00 = fmaf(a, __ldg(p00 + i1) - __ldg(p00 + i0), __ldg(p00 + i0));
    const float v01 = fmaf(a, __ldg(p01 + i1) - __ldg(p01 + i0), __ldg(p01 + i0));
    const float v10 = fmaf(a, __ldg(p10 + i1) - __ldg(p10 + i0), __ldg(p10 + i0));
    const float v11 = fmaf(a, __ldg(p11 + i1) - __ldg(p11 + i0), __ldg(p11 + i0));
    const float w0 = fmaf(b, v01 - v00, v00), w1 = fmaf(b, v11 - v10, v10);
    return fmaf(c, w1 - w0, w0);
}

// The baked turbulence's slices: in plain memory (`field`, FP32 trilinear by turb_fetch, which the CPU
// oracle repeats) or, when the scene carries their texture handles, through the texture unit with
// the reference's sampler (emission.cuh:121-122; its trilinear weights have 8 fractional bits).
__device__ __forceinline__ bool baked_on(const so_scene& S, const float* field) {
    return field != nullptr || (S.turb_nt > 0 && S.turb_tex[0] != 0);
}
__device__ __forceinline__ float baked_sample(const so_scene& S, const float* field, int k, float x, float y,
                                              float z) {
    if (field) return turb_fetch(field + (size_t)k * TURB_NPHI * TURB_NLR * TURB_NZ, x, y, z);
    return tex3D<float>((cudaTextureObject_t)S.turb_tex[k], x, y, z);
}

// Whether flow_step on the reference flow model (no torus) can change the transfer at (r, u): its
// first two returns, in its own arithmetic.  A step for which this is false emits nothing and
// transmits exactly 1.
__device__ __forceinline__ bool flow_wants(const so_scene& S, double r, double u) {
    double s2 = fmax(fma(-u, u, 1.0), 1e-12), s = sqrt(s2);
    double R = r * s, z = r * u;
    if (r > S.r_flow_max || R < 1e-3) return false;
    double zh = z / (S.h_r * R);
    return !(exp(-0.5 * zh * zh) < 1e-7);
}

// The same for the torus plasma (flow_step's torus branch: outside the flow region, or the vertical
// profile exp(-(u / h_sph)^2 / 2) below 1e-7).
__device__ __forceinline__ bool torus_wants(const so_scene& S, const TorusParams& tp, double r, double u) {
    double s2 = fmax(fma(-u, u, 1.0), 1e-12), s = sqrt(s2);
    double R = r * s;
    if (r > S.r_flow_max || R < 1e-3) return false;
    double zh = u / tp.h_sph;
    return !(exp(-0.5 * zh * zh) < 1e-7);
}

// flow_step with the torus turbulence sum `delta` at this point already evaluated (torus_position).
// With `field` (the frame's baked slices) the reference model's turbulence is sampled as
// emission.cuh:112-124 does, else its sheared noise is evaluated in place (the turb_nt = 0 path).
static __device__ void flow_step(const so_scene& S, const so_frame& F, const float* field, const TorusParams& tp,
                                 double delta, double r, double u, double phi, double t, double lam, double Ecam,
                                 double h, double* dI, double* dtau) {
    *dI = 0.0;
    *dtau = 0.0;
    const double a = S.a;
    double s2 = fmax(fma(-u, u, 1.0), 1e-12), s = sqrt(s2);
    double R = r * s, z = r * u;
    if (r > S.r_flow_max || R < 1e-3) return;
    double ne, Th;
    if (tp.on) {
        double zh = u / tp.h_sph;
        double vert = exp(-0.5 * zh * zh);
        if (vert < 1e-7) return;
        double lx = log(r / S.rh);
        ne = S.n0 * exp(-tp.ne_index * lx) * vert;
        if (tp.n_modes > 0) ne *= exp(delta - tp.half_var);
        Th = tp.theta_e0 * exp(-tp.te_index * lx);
    } else {
        double zh = z / (S.h_r * R);
        double vert = exp(-0.5 * zh * zh);
        if (vert < 1e-7) return;
        ne = S.n0 * exp(-S.n_index * log(r)) * vert;
        if (S.flow_turb_amp > 0.f) {
            if (baked_on(S, field)) {
                // two slices around the retarded time t - t_ref(r), interpolated (emission.cuh:112-124)
                const double tref = F.t - (F.r - r + 2.0 * log(F.r / r));
                const float y = (float)((log(R) - S.turb_lr0) / (S.turb_lr1 - S.turb_lr0));
                const float x = (float)(phi * (0.5 / PI));
                const float w = (float)(0.5 + 0.5 * (z / R) / S.turb_zmax);
                float sl = (float)((t - tref) - S.turb_d0) / S.turb_dd;
                sl = fminf(fmaxf(sl, 0.f), (float)(TURB_NT - 1) - 1e-4f);
                const int k = (int)sl;
                const float f = sl - (float)k;
                const float A = baked_sample(S, field, k, x, y, w);
                const float B = baked_sample(S, field, k + 1, x, y, w);
                ne *= fmaf(B - A, f, A);
            } else {
                float n = sheared_noise(S, R, phi, z, t, S.flow_turb_scale, S.flow_tcorr, S.seed ^ 0x51f15eedu);
                ne *= exp((double)(S.flow_turb_amp * n - 0.5f * S.flow_turb_amp * S.flow_turb_amp));
            }
        }
        Th = 0.0;
    }
    double dr = r - S.rh;
    ne *= 1.0 - exp(-(dr * dr) / 0.25);
    if (ne < 1e-30) return;
    if (!tp.on) Th = S.theta0 * exp(-S.theta_index * log(r));
    double B = sqrt(8.0 * PI * ne * cgs::MP * cgs::C * cgs::C / (6.0 * r * S.beta_p));
    double r2 = r * r, a2 = a * a;
    double Sigma = fma(a2, u * u, r2), Delta = fma(r, r - 2.0, a2);
    double rpa = r2 + a2;
    double A = fma(rpa, rpa, -(a2 * Delta * s2));
    double g_tt = -(1.0 - 2.0 * r / Sigma), g_tph = -2.0 * a * r * s2 / Sigma, g_phph = A * s2 / Sigma;
    double omz = 2.0 * a * r / A;
    double Om = S.flow_kep * keplerian_omega(a, fmax(R, S.r_isco));
    double vmax = sqrt(Sigma * Delta / A) / sqrt(g_phph) * 0.999;
    Om = omz + fmax(-vmax, fmin(vmax, Om - omz));
    double norm = -fma(g_phph * Om, Om, fma(2.0 * g_tph, Om, g_tt));
    if (norm <= 0.0) return;
    double ut = 1.0 / sqrt(norm);
    double kdotu = ut * fma(-Om, lam, 1.0);
    double nu_f = S.nu_obs * Ecam * kdotu;
    double g = S.nu_obs / nu_f;
    double u_ph = ut * fma(g_phph, Om, g_tph);
    double kb = fma(-kdotu, u_ph, lam);
    double bb = fma(u_ph, u_ph, g_phph);
    double cosb = kb / (kdotu * sqrt(bb));
    double sinb = sqrt(fmax(fma(-cosb, cosb, 1.0), 1e-6));
    double nuc = cgs::QE * B / (2.0 * PI * cgs::ME * cgs::C);
    double nus = 2.0 / 9.0 * nuc * Th * Th * sinb;
    double Xs = nu_f / nus;
    double x3 = cbrt(Xs);
    double k2 = exp((double)table_lerp(S.k2_lntab, S.k2_n, S.k2_l0, S.k2_dl, (float)log(Th)));
    double brk = fma(1.887748625363387, sqrt(x3), sqrt(Xs));
    double j = ne * 1.4142135623730951 * PI * cgs::QE * cgs::QE * nus / (3.0 * k2 * cgs::C) * brk * brk * exp(-x3);
    double Te = Th * cgs::ME * cgs::C * cgs::C / cgs::KB;
    double hnu = cgs::H * nu_f / (cgs::KB * Te);
    double Bnu = 2.0 * cgs::H * nu_f * nu_f * nu_f / (cgs::C * cgs::C) / expm1(hnu);
    double alpha = j / Bnu;
    double dl = kdotu * Sigma * h * S.rg_cm;
    double tau = alpha * dl;
    *dtau = tau;
    *dI = g * g * g * Bnu * (-expm1(-tau));
}

// escape_angles (trace.cuh:49-55).
__device__ __forceinline__ void escape_angles(const double* y, const double* k, double* th, double* ph) {
    double s = sqrt(fmax(fma(-y[2], y[2], 1.0), 1e-30));
    double t0 = acos(fmax(-1.0, fmin(1.0, y[2])));
    double dthdr = (-y[3] / s) / y[1], dphdr = k[4] / y[1];
    *th = fma(y[0], dthdr, t0);
    *ph = fma(y[0], dphdr, y[4]);
}

// sky_uv (trace.cuh:24-33): galactic texture coordinates of an escape direction, u wrapped into [0, 1).
__device__ __forceinline__ float2 sky_uv(const so_scene& S, double th, double ph) {
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(ph, &sp, &cp);
    const double dx = st * cp, dy = st * sp, dz = ct;
    const so_mat3& m = S.sky_rot;
    const double gx = fma(m.r0.z, dz, fma(m.r0.y, dy, m.r0.x * dx));
    const double gy = fma(m.r1.z, dz, fma(m.r1.y, dy, m.r1.x * dx));
    const double gz = fma(m.r2.z, dz, fma(m.r2.y, dy, m.r2.x * dx));
    const double l = atan2(gy, gx), b = asin(fmax(-1.0, fmin(1.0, gz)));
    float u = (float)(0.5 - l * (0.5 / PI));
    u -= floorf(u);
    return make_float2(u, (float)(0.5 - b / PI));
}

// pixel_grad (render.cu:56-72): the pixel's footprint on the sky from the escape coordinates of its
// four corners (uv grid of (W + 1) x (H + 1), (-1, -1) where a corner ray did not escape), u
// differences wrapped; a footprint that touches a non-escaping corner gets a fixed 0.02 box.
struct SkyGrad {
    float2 dx, dy;
};
__device__ __forceinline__ float wrapd(float d) { return d > 0.5f ? d - 1.f : (d < -0.5f ? d + 1.f : d); }
__device__ __forceinline__ SkyGrad pixel_grad(const float2* __restrict__ uv, int W, int px, int py, float scale) {
    const int W1 = W + 1;
    const float2 a = uv[(long long)py * W1 + px], b = uv[(long long)py * W1 + px + 1];
    const float2 c = uv[(long long)(py + 1) * W1 + px], d = uv[(long long)(py + 1) * W1 + px + 1];
    SkyGrad g;
    if (a.x < 0.f || b.x < 0.f || c.x < 0.f || d.x < 0.f) {
        g.dx = make_float2(0.02f, 0.f);
        g.dy = make_float2(0.f, 0.02f);
        return g;
    }
    const float dux = 0.5f * (wrapd(b.x - a.x) + wrapd(d.x - c.x)), dvx = 0.5f * ((b.y - a.y) + (d.y - c.y));
    const float duy = 0.5f * (wrapd(c.x - a.x) + wrapd(d.x - b.x)), dvy = 0.5f * ((c.y - a.y) + (d.y - b.y));
    g.dx = make_float2(dux * scale, dvx * scale);
    g.dy = make_float2(duy * scale, dvy * scale);
    return g;
}

// sky_radiance (trace.cuh:35-43): star-map texel (s, s T / 1e4) by the texture unit's anisotropic
// mip filtering over the pixel footprint, shifted by the photon's energy at the camera.
__device__ __forceinline__ void sky_radiance(const so_scene& S, float2 uv, const SkyGrad& gr, double Ecam,
                                             float* xyz) {
    const float2 v = tex2DGrad<float2>((cudaTextureObject_t)S.sky_tex, uv.x, uv.y, gr.dx, gr.dy);
    xyz[0] = xyz[1] = xyz[2] = 0.f;
    if (v.x <= 0.f) return;
    const float T = 1e4f * v.y / v.x;
    const float g = (float)(1.0 / Ecam);
    blackbody_xyz(S, g * T, xyz);
    const float s = v.x * S.sky_scale;
    xyz[0] *= s;
    xyz[1] *= s;
    xyz[2] *= s;
}

}  // namespace so
