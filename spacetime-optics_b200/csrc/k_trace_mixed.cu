// k_trace_mixed.cu -- mixed-precision tracer: FP32 far from the critical curve, FP64 where it matters.
//
// Same physics as the plain FP64 tracer (trace_ray, blackholes/src/trace.cuh:62-165; flow_step,
// emission.cuh:99-175), re-arranged for throughput:
//   k_route       per sample: distance of its image point from the analytic critical curve
//                 (critical_curve_point, kerr.hpp:210-220, tabulated per frame on the host).  Inside
//                 the band -> FP64 list; outside -> FP32 list.
//   k_approach64  FP64 from the camera to r_switch (the far field, where the coordinate time and
//                 radius are too large for FP32 increments): DP5(4) in the inverse radius
//                 (far_approach, so_kerr.cuh: a few steps where Mino time needs hundreds) on ingoing
//                 legs without a radial turning point, the reference's Mino-time DP5(4) otherwise;
//                 then parks the state in HBM as five float4 SoA planes (two-float hi/lo pairs for
//                 r, r', u, u', phi, t).
//   k_trace32     persistent FP32 tracer over the parked rays: compensated (two-sum) state update,
//                 FP32 stages and error estimate with the reference's error norm at tol32, err^-0.2
//                 on the SFU, torus turbulence with the mode table in shared memory, its 512-mode sum
//                 split across the 32 lanes of the warp for every lane that needs one (SFU cosines of
//                 phases reduced in turns).  At the end the Carter-constant and radial constraints are
//                 checked in FP64; a ray that fails, or whose radial turning point falls inside turn_r,
//                 goes to the FP64 re-trace list.
// The band and re-trace lists are then traced by the plain FP64 kernel (k_trace64, RAYS_SAMPLES).
// Scenes whose emission depends on the raw coordinate time at a generation boundary (the reference's
// sheared fBm turbulence of the flow or the disk: noise phase ~ t / P with t ~ -r_cam) are
// ill-conditioned for any integrator that differs from the FP64 one, so the router sends all of
// their rays to FP64.
// Compiled with -ftz=true -prec-div=false -prec-sqrt=false -fmad=false: FP32 fusions are the explicit
// fmaf calls; the FP64 approach keeps the fma placement of so_kerr.cuh.
#include <cuda_runtime.h>

#include "so_emission.cuh"
#include "so_launch.h"

namespace so {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void push(uint32_t* list, unsigned long long* count, uint32_t v, bool want) {
    const unsigned m = __ballot_sync(FULL, want);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(m));
    base = __shfl_sync(FULL, base, leader);
    if (want) list[base + __popc(m & ((1u << lane) - 1u))] = v;
}

// Bardeen coordinates (alpha, beta) of a viewing direction d in the camera's ZAMO frame
// (e_r, e_theta, e_phi): image +x is +alpha (main.cpp:345), beta along -e_theta.
__device__ __forceinline__ bool in_band(const TraceLaunch& L, const so_frame& F, double x, double yv) {
    so_vec3 d = view_dir(F, x, yv);
    if (!(d.x < 0.0)) return true;  // looking away from the hole: no critical curve to compare with
    double al = F.r * d.z / (-d.x), be = F.r * (-d.y) / (-d.x);
    double rho = sqrt(al * al + be * be);
    double psi = atan2(be, al);
    double u = (psi + PI) * (L.band_n / (2.0 * PI));
    int i = (int)floor(u);
    double f = u - i;
    i = ((i % L.band_n) + L.band_n) % L.band_n;
    int j = (i + 1) % L.band_n;
    double rc = L.band_rho[i] + (L.band_rho[j] - L.band_rho[i]) * f;
    return fabs(rho - rc) < L.band_m;
}

}  // namespace

// ---- router ------------------------------------------------------------------------------------
__global__ void k_route(const TraceLaunch L, int all64) {
    const so_frame& F = L.frames[0];
    const long long n = L.nsamples;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const long long sid = base + threadIdx.x;
        const bool valid = sid < n;
        bool band = all64 != 0;
        if (valid && !band) {
            double x, yv;
            sample_point(L.W, L.H, L.jitter, F, sid / L.spp, (int)(sid % L.spp), &x, &yv);
            band = in_band(L, F, x, yv);
        }
        push(L.list64, &L.nlists[1], (uint32_t)sid, valid && band);
        push(L.list32, &L.nlists[0], (uint32_t)sid, valid && !band);
    }
}

// ---- FP64 approach -----------------------------------------------------------------------------
// State planes (nsamples each): P0 = (r_hi, r_lo, pr_hi, pr_lo), P1 = (u_hi, u_lo, pu_hi, pu_lo),
// P2 = (phi_hi, phi_lo, t_hi, t_lo), P3 = (lam, eta, E, h), P4 = (psi, attempts, accepted, ncross).
__device__ __forceinline__ float2 split(double v) {
    float hi = (float)v;
    return make_float2(hi, (float)(v - (double)hi));
}

__global__ void __launch_bounds__(128) k_approach64(const TraceLaunch L) {
    const so_frame& F = L.frames[0];
    const so_scene& S = L.scenes[0];
    const long long n = (long long)L.nlists[0];
    const long long ns = L.nsamples;
    unsigned long long n_att = 0, n_acc = 0;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const long long j = base + threadIdx.x;
        bool park = false;
        uint32_t sid = 0;
        if (j < n) {
            sid = L.list32[j];
            double x, yv;
            sample_point(L.W, L.H, L.jitter, F, sid / L.spp, (int)(sid % L.spp), &x, &yv);
            RayC c;
            double y[6], k1[6], yn[6], k7[6];
            camera_photon(S.a, F.kp, F.ph, F.t, view_dir(F, x, yv), F.beta, c, y);
            rhs(c, y, k1);
            double h = initial_step(y);
            int fate = 0, it = 0, nacc = 0, ncross = 0;
            double psi = 0.0;
            const bool radio = S.mode == SO_MODE_RADIO;
            bool done = false, far = false;
            if (L.far_field && far_applies(c, y, L.r_switch)) {
                const int att = far_approach(c, y, L.r_switch, fmin(S.tol, L.tol_approach), 256, &psi, &ncross, radio);
                if (att >= 0) {
                    far = true;
                    n_att += (unsigned long long)att;
                    it = nacc = L.approach_it;
                    h = initial_step(y);
                }
            }
            double sp = sqrt(fmax(fma(-y[2], y[2], 1.0), 0.0));
            double s4, c4;
            sincos(y[4], &s4, &c4);
            double pp0 = sp * c4, pp1 = sp * s4, pp2 = y[2];
            for (; !far && it < S.max_steps;) {
                ++it;
                double err = dp54(c, y, k1, h, L.tol_approach, yn, k7);
                if (!(err <= 1.0)) {
                    h = reject_step(h, err);
                    continue;
                }
                ++nacc;
                if (radio) {
                    double sn = sqrt(fmax(fma(-yn[2], yn[2], 1.0), 0.0));
                    sincos(yn[4], &s4, &c4);
                    double pn0 = sn * c4, pn1 = sn * s4, pn2 = yn[2];
                    double cx = fma(pp1, pn2, -(pp2 * pn1)), cy = fma(pp2, pn0, -(pp0 * pn2)),
                           cz = fma(pp0, pn1, -(pp1 * pn0));
                    psi += atan2(sqrt(fma(cz, cz, fma(cy, cy, cx * cx))), fma(pp2, pn2, fma(pp1, pn1, pp0 * pn0)));
                    pp0 = pn0;
                    pp1 = pn1;
                    pp2 = pn2;
                }
                if ((y[2] > 0.0) != (yn[2] > 0.0)) ++ncross;
                double hc = h;
                for (int i = 0; i < 6; ++i) {
                    y[i] = yn[i];
                    k1[i] = k7[i];
                }
                project_radial(c, y, k1);
                h = accept_step(hc, err);
                if (y[0] < S.r_stop) {
                    fate = -1;
                    done = true;
                    break;
                }
                if (y[0] > S.r_escape && y[1] > 0.0) {
                    fate = 1;
                    done = true;
                    break;
                }
                if (y[0] < L.r_switch) break;
            }
            if (!far) {
                n_att += (unsigned long long)it;
                n_acc += (unsigned long long)nacc;
            }
            if (!done && it >= S.max_steps) done = true;  // step limit: fate 0
            if (done) {
                L.sample_out[sid] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (L.sample_fate) L.sample_fate[sid] = (int8_t)fate;
                if (fate == 1 && L.esc_list) {
                    // escaped in the far field of a star-map frame: the sky is added by k_sky_escape
                    float2 r = split(y[0]), pr = split(y[1]), u = split(y[2]), pu = split(y[3]), ph = split(y[4]),
                           t = split(y[5]);
                    L.state[0 * ns + sid] = make_float4(r.x, r.y, pr.x, pr.y);
                    L.state[1 * ns + sid] = make_float4(u.x, u.y, pu.x, pu.y);
                    L.state[2 * ns + sid] = make_float4(ph.x, ph.y, t.x, t.y);
                    L.state[3 * ns + sid] = make_float4((float)c.lam, (float)c.eta, (float)c.E, (float)h);
                    L.state[4 * ns + sid] = make_float4(1.f, 0.f, 0.f, 0.f);
                    L.esc_list[atomicAdd(&L.nlists[9], 1ull)] = sid;
                }
            } else {
                park = true;
                float2 r = split(y[0]), pr = split(y[1]), u = split(y[2]), pu = split(y[3]), ph = split(y[4]),
                       t = split(y[5]);
                L.state[0 * ns + sid] = make_float4(r.x, r.y, pr.x, pr.y);
                L.state[1 * ns + sid] = make_float4(u.x, u.y, pu.x, pu.y);
                L.state[2 * ns + sid] = make_float4(ph.x, ph.y, t.x, t.y);
                L.state[3 * ns + sid] = make_float4((float)c.lam, (float)c.eta, (float)c.E, (float)h);
                L.state[4 * ns + sid] = make_float4((float)psi, __int_as_float(it), __int_as_float(nacc),
                                                    __int_as_float(ncross));
            }
        }
        push(L.parked, &L.nlists[3], sid, park);
    }
    for (int o = 16; o > 0; o >>= 1) {
        n_att += __shfl_down_sync(FULL, n_att, o);
        n_acc += __shfl_down_sync(FULL, n_acc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&L.counters->pad[0], n_att);  // FP64 attempts of the approach
        atomicAdd(&L.counters->accepted, n_acc);
    }
}

// ---- FP32 tracer -----------------------------------------------------------------------------------
namespace {

struct C32 {
    float a, lam, eta, E, A2, CP, K, Q3;
};

// geodesic_rhs in FP32 (kerr.hpp:103-116); s2 = (1-u)(1+u) keeps its relative precision at the poles.
__device__ __forceinline__ void rhs32(const C32& c, float r, float pr, float u, float pu, float* d) {
    float Delta = fmaf(r, r - 2.f, c.A2);
    float P = fmaf(r, r, c.CP);
    d[0] = pr;
    d[1] = fmaf(2.f * r, P, -((r - 1.f) * c.K));
    d[2] = pu;
    float u2 = u * u;
    d[3] = u * fmaf(c.A2, fmaf(-2.f, u2, 1.f), -c.Q3);
    float s2 = fmaxf((1.f - u) * (1.f + u), 1e-30f);
    float iD = __frcp_rn(Delta);
    d[4] = c.a - fmaf(c.a * P, iD, __fdividef(c.lam, s2));
    d[5] = -fmaf(fmaf(r, r, c.A2) * P, iD, c.a * fmaf(-c.a, s2, c.lam));
}

// Two-sum: hi + lo + d renormalised (Knuth), the compensated state update.
__device__ __forceinline__ void acc2(float& hi, float& lo, float d) {
    float s = hi + d;
    float bp = s - hi;
    float e = (hi - (s - bp)) + (d - bp);
    lo += e;
    float s2 = s + lo;
    lo = lo - (s2 - s);
    hi = s2;
}

struct Ray32 {
    float rh, rl, prh, prl, uh, ul, puh, pul, phh, phl, th, tl;
    float k1[6];
    float h, trans, psi, pp0, pp1, pp2;
    float acc[4];
    int ncross, natt, nacc, nflow, it;
    int seg, cnt, head, nrec;  // deferred turbulence: current record segment, slots used in it, first, total
    uint32_t sid;
};

struct Torus32 {
    int on, n_modes;
    float ne_index, te_index, h_sph, theta_e0, half_var;
};

// Turbulence sums of the lanes in `want` (positions X, Y, Z per lane), each split across the warp:
// lane l takes modes l, l+32, ...; a butterfly shuffle reduction gives every lane the total, which
// the owning lane keeps.  Positions are served two at a time, so each mode read from shared memory
// feeds two cosines, with two independent accumulators per position.  All 32 lanes must call this.
// Modes in shared memory in radians (k, phase) and amplitude; the SFU cosine reduces the phase in
// turns itself, so the argument's FP32 rounding (|phase| <~ 1e3 rad: ~5e-5 rad) is the only error.
__device__ __forceinline__ float warp_turbulence(const float4* __restrict__ km, const float* __restrict__ amp, int n,
                                                 bool want, float X, float Y, float Z) {
    const int lane = threadIdx.x & 31;
    unsigned m = __ballot_sync(FULL, want);
    float mine = 0.f;
    while (m) {
        const int s0 = __ffs(m) - 1;
        m &= m - 1;
        const int s1 = m ? __ffs(m) - 1 : s0;
        if (m) m &= m - 1;
        const float x0 = __shfl_sync(FULL, X, s0), y0 = __shfl_sync(FULL, Y, s0), z0 = __shfl_sync(FULL, Z, s0);
        const float x1 = __shfl_sync(FULL, X, s1), y1 = __shfl_sync(FULL, Y, s1), z1 = __shfl_sync(FULL, Z, s1);
        float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
        int i = lane;
        for (; i + 32 < n; i += 64) {
            const float4 k = km[i], q = km[i + 32];
            const float w = amp[i], v = amp[i + 32];
            a0 = fmaf(w, __cosf(fmaf(k.z, z0, fmaf(k.y, y0, fmaf(k.x, x0, k.w)))), a0);
            b0 = fmaf(w, __cosf(fmaf(k.z, z1, fmaf(k.y, y1, fmaf(k.x, x1, k.w)))), b0);
            a1 = fmaf(v, __cosf(fmaf(q.z, z0, fmaf(q.y, y0, fmaf(q.x, x0, q.w)))), a1);
            b1 = fmaf(v, __cosf(fmaf(q.z, z1, fmaf(q.y, y1, fmaf(q.x, x1, q.w)))), b1);
        }
        if (i < n) {
            const float4 k = km[i];
            const float w = amp[i];
            a0 = fmaf(w, __cosf(fmaf(k.z, z0, fmaf(k.y, y0, fmaf(k.x, x0, k.w)))), a0);
            b0 = fmaf(w, __cosf(fmaf(k.z, z1, fmaf(k.y, y1, fmaf(k.x, x1, k.w)))), b0);
        }
        float a = a0 + a1, b = b0 + b1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(FULL, a, o);
            b += __shfl_xor_sync(FULL, b, o);
        }
        if (lane == s0) mine = a;
        if (lane == s1) mine = b;
    }
    return mine;
}

// flow_step (emission.cuh:99-175) in FP32, given the turbulence sum delta at this point (torus
// model).  The reference plasma enters only without its fBm turbulence (see the router).
// bfac: the reference model's baked turbulence factor at this point (1 without turbulence).
__device__ __forceinline__ void flow_step32(const so_scene& S, const Torus32& tp, float delta, float r, float u,
                                            float lam, float Ecam, float h, float* dI, float* dtau,
                                            float bfac = 1.f) {
    *dI = 0.f;
    *dtau = 0.f;
    const float a = (float)S.a;
    float s2 = fmaxf((1.f - u) * (1.f + u), 1e-12f), s = sqrtf(s2);
    float R = r * s, z = r * u;
    if (r > (float)S.r_flow_max || R < 1e-3f) return;
    const float risco = (float)S.r_isco, rh = (float)S.rh;
    float ne, Th;
    if (tp.on) {
        float zh = __fdividef(u, tp.h_sph);
        float vert = __expf(-0.5f * zh * zh);
        if (vert < 1e-7f) return;
        float lx = __logf(__fdividef(r, rh));
        ne = (float)S.n0 * __expf(-tp.ne_index * lx) * vert;
        if (tp.n_modes > 0) ne *= __expf(delta - tp.half_var);
        Th = tp.theta_e0 * __expf(-tp.te_index * lx);
    } else {
        float zh = __fdividef(z, (float)S.h_r * R);
        float vert = __expf(-0.5f * zh * zh);
        if (vert < 1e-7f) return;
        ne = (float)S.n0 * __expf(-(float)S.n_index * __logf(r)) * vert * bfac;
        Th = (float)S.theta0 * __expf(-(float)S.theta_index * __logf(r));
    }
    float dr = r - rh;
    ne *= 1.f - __expf(-(dr * dr) * 4.f);
    if (ne < 1e-30f) return;
    // B^2 / 8 pi = ne m_p c^2 / (6 r beta)
    const float kB = (float)(8.0 * PI * cgs::MP * cgs::C * cgs::C / 6.0);
    float B = sqrtf(kB * ne / (r * (float)S.beta_p));
    float r2 = r * r, a2 = a * a;
    float Sigma = fmaf(a2, u * u, r2), Delta = fmaf(r, r - 2.f, a2);
    float rpa = r2 + a2;
    float A = fmaf(rpa, rpa, -(a2 * Delta * s2));
    float iS = __frcp_rn(Sigma);
    float g_tt = -(1.f - 2.f * r * iS), g_tph = -2.f * a * r * s2 * iS, g_phph = A * s2 * iS;
    float omz = __fdividef(2.f * a * r, A);
    float Rk = fmaxf(R, risco);
    float Om = (float)S.flow_kep * __frcp_rn(fmaf(Rk, sqrtf(Rk), a));
    float vmax = sqrtf(__fdividef(Sigma * Delta, A)) * rsqrtf(g_phph) * 0.999f;
    Om = omz + fmaxf(-vmax, fminf(vmax, Om - omz));
    float norm = -fmaf(g_phph * Om, Om, fmaf(2.f * g_tph, Om, g_tt));
    if (norm <= 0.f) return;
    float ut = rsqrtf(norm);
    float kdotu = ut * fmaf(-Om, lam, 1.f);
    float nu_f = (float)S.nu_obs * Ecam * kdotu;
    float g = __fdividef((float)S.nu_obs, nu_f);
    float u_ph = ut * fmaf(g_phph, Om, g_tph);
    float kb = fmaf(-kdotu, u_ph, lam);
    float bb = fmaf(u_ph, u_ph, g_phph);
    float cosb = __fdividef(kb, kdotu * sqrtf(bb));
    float sinb = sqrtf(fmaxf(fmaf(-cosb, cosb, 1.f), 1e-6f));
    const float knuc = (float)(cgs::QE / (2.0 * PI * cgs::ME * cgs::C));
    float nus = (2.f / 9.f) * knuc * B * Th * Th * sinb;
    float Xs = __fdividef(nu_f, nus);
    float x3 = cbrtf(Xs);
    float k2 = __expf(table_lerp(S.k2_lntab, S.k2_n, S.k2_l0, S.k2_dl, __logf(Th)));
    float brk = fmaf(1.887748625363387f, sqrtf(x3), sqrtf(Xs));
    const float kj = (float)(1.4142135623730951 * PI * cgs::QE * cgs::QE / (3.0 * cgs::C));
    float j = __fdividef(ne * kj * nus, k2) * brk * brk * __expf(-x3);
    const float kte = (float)(cgs::H / (cgs::ME * cgs::C * cgs::C));  // h nu / (k Te) = kte nu / Th
    float hnu = __fdividef(kte * nu_f, Th);
    // 2 h nu^3 / c^2 with nu in GHz (2 h / c^2 itself is below the FP32 range)
    const float kbn = (float)(2.0 * cgs::H / (cgs::C * cgs::C) * 1e27);
    const float nu_g = nu_f * 1e-9f;
    float Bnu = __fdividef(kbn * nu_g * nu_g * nu_g, expm1f(hnu));
    float alpha = __fdividef(j, Bnu);
    float dl = kdotu * Sigma * h * (float)S.rg_cm;
    float tau = alpha * dl;
    *dtau = tau;
    *dI = g * g * g * Bnu * (-expm1f(-tau));
}

}  // namespace

// FP32 tracer.  One loop iteration = one DP5(4) attempt for every active lane.  The loop body is
// split in two around the warp-cooperative turbulence sum, so every lane reaches the shuffles.
// DEFER (radio torus with Fourier modes, or the reference flow model): instead of the turbulence
// sum and the transfer, every emitting flow step is recorded (r, u, advected azimuth, step; for the
// reference flow the baked turbulence factor, fetched here as the in-line form fetches it, goes to
// the record's sum slot) in the ray's chain of record segments; k_turb_records (torus) and
// k_flow_records finish the emission.  The geodesic does not depend on
// the emission; only the opacity cut (trans < 1e-5) does, and k_flow_records applies it at the
// record where it happens, so the result is the one of the in-line form to FP32 rounding.
template <int VAR, int MINB, bool DEFER>
__global__ void __launch_bounds__(128, MINB) k_trace32(const TraceLaunch L) {
    extern __shared__ float4 sm4[];
    const so_scene& S = L.scenes[0];
    const so_frame& F = L.frames[0];
    Torus32 tp;
    tp.on = VAR == VAR_RADIO && L.torus;
    tp.n_modes = tp.on ? L.n_modes : 0;
    tp.ne_index = (float)L.ne_index;
    tp.te_index = (float)L.te_index;
    tp.h_sph = (float)L.h_sph;
    tp.theta_e0 = (float)L.theta_e0;
    tp.half_var = (float)L.half_var;
    float4* km = sm4;
    float* amp = reinterpret_cast<float*>(sm4 + tp.n_modes);
    if (!DEFER && tp.n_modes > 0) {
        for (int i = threadIdx.x; i < tp.n_modes; i += blockDim.x) {
            so_mode m = L.modes[i];
            // phase folded into (-pi, pi]: its FP32 rounding then stays small
            double ph = m.phase - 2.0 * PI * floor(m.phase / (2.0 * PI) + 0.5);
            km[i] = make_float4((float)m.kx, (float)m.ky, (float)m.kz, (float)ph);
            amp[i] = (float)m.amp;
        }
        __syncthreads();
    }
    const long long ns = L.nsamples;
    const long long parked = (long long)L.nlists[3];
    const long long lo = L.wave_end > 0 ? min(L.wave_begin, parked) : 0;
    const long long total = L.wave_end > 0 ? min(L.wave_end, parked) : parked;
    const uint32_t* work = L.parked;
    const int lane = threadIdx.x & 31;
    const float tol = (float)L.tol32;
    const float rstop = (float)S.r_stop, resc = (float)S.r_escape, rflow = (float)S.r_flow_max;
    const float step_frac = (float)S.step_frac;
    const float rcam_hi = (float)F.r, rcam_lo = (float)(F.r - (double)(float)F.r);
    const float risco = (float)S.r_isco, flow_kep = (float)S.flow_kep;
    const float tcam = (float)F.t;
    const bool baked = VAR == VAR_RADIO && !tp.on && baked_on(S, L.turb_field) && S.flow_turb_amp > 0.f;
    const float r_out = (float)L.r_emit;
    const bool radio = VAR == VAR_RADIO;
    C32 c;
    c.a = (float)S.a;
    c.A2 = c.a * c.a;
    Ray32 R;
    bool active = false, exhausted = false;
    unsigned long long n_att = 0, n_acc = 0, n_flow = 0, n_lim = 0, n_turn = 0, n_drift = 0;
    for (;;) {
        const bool need = !active && !exhausted;
        const unsigned m = __ballot_sync(FULL, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&L.counters->next, (unsigned long long)__popc(m));
            base = __shfl_sync(FULL, base, leader);
            if (need) {
                const unsigned long long j = (unsigned long long)lo + base + __popc(m & ((1u << lane) - 1u));
                if (j >= (unsigned long long)total) {
                    exhausted = true;
                } else {
                    active = true;
                    const uint32_t sid = work[j];
                    R.sid = sid;
                    float4 p0 = L.state[0 * ns + sid], p1 = L.state[1 * ns + sid], p2 = L.state[2 * ns + sid],
                           p3 = L.state[3 * ns + sid], p4 = L.state[4 * ns + sid];
                    R.rh = p0.x; R.rl = p0.y; R.prh = p0.z; R.prl = p0.w;
                    R.uh = p1.x; R.ul = p1.y; R.puh = p1.z; R.pul = p1.w;
                    R.phh = p2.x; R.phl = p2.y; R.th = p2.z; R.tl = p2.w;
                    c.lam = p3.x;
                    c.eta = p3.y;
                    c.E = p3.z;
                    R.h = p3.w;
                    R.psi = p4.x;
                    R.it = __float_as_int(p4.y);  // attempts so far (max_steps covers the whole ray)
                    R.natt = 0;                   // FP32 attempts / accepted steps of this kernel
                    R.nacc = 0;
                    R.ncross = __float_as_int(p4.w);
                    R.nflow = 0;
                    c.CP = fmaf(-c.a, c.lam, c.A2);
                    float lma = c.lam - c.a;
                    c.K = fmaf(lma, lma, c.eta);
                    c.Q3 = fmaf(c.lam, c.lam, c.eta);
                    R.trans = 1.f;
                    R.acc[0] = R.acc[1] = R.acc[2] = R.acc[3] = 0.f;
                    R.seg = R.head = -1;
                    R.cnt = REC_SEG;
                    R.nrec = 0;
                    rhs32(c, R.rh + R.rl, R.prh + R.prl, R.uh + R.ul, R.puh + R.pul, R.k1);
                    float u = R.uh + R.ul, sp = sqrtf(fmaxf((1.f - u) * (1.f + u), 0.f)), s4, c4;
                    __sincosf(R.phh + R.phl, &s4, &c4);
                    R.pp0 = sp * c4;
                    R.pp1 = sp * s4;
                    R.pp2 = u;
                }
            }
        }
        if (__all_sync(FULL, !active)) break;
        // ---- part 1 (active lanes): one DP5(4) attempt in FP32 ----------------------------------
        int fate = 2;  // 2 = running, 3 = re-trace: radial turning point, 4 = re-trace: drift
        bool accepted = false, want_flow = false, want_turb = false;
        float nrh = 0.f, nrl = 0.f, nprh = 0.f, nprl = 0.f, nuh = 0.f, nul = 0.f, npuh = 0.f, npul = 0.f;
        float n0 = 0.f, n1 = 0.f, n2 = 0.f, hc = 0.f, err = 0.f, TX = 0.f, TY = 0.f, TZ = 0.f;
        float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
        float rec_bf = 1.f;  // reference flow model: the record's baked turbulence factor
        float bfac = 1.f;
        float k7[6], dy[6];
        if (active) {
            if (R.it >= S.max_steps || R.natt >= L.t32_max_att) {
                fate = 0;  // the FP64 re-trace decides (step limit, or an FP32 controller that stalls)
            } else {
                ++R.it;
                ++R.natt;
                const float y0 = R.rh + R.rl, y1 = R.prh + R.prl, y2 = R.uh + R.ul, y3 = R.puh + R.pul;
                hc = R.h;
                if (radio && S.flow_on && y0 < rflow) {
                    float s = sqrtf(fmaxf((1.f - y2) * (1.f + y2), 0.f));
                    float cap = step_frac * fminf(__fdividef(y0, fabsf(y1) + 1e-30f),
                                                  __fdividef(fmaxf(s, 0.05f), fabsf(y3) + 1e-30f));
                    hc = fminf(hc, cap);
                } else if (VAR == VAR_DISK && S.disk_on) {
                    hc = fminf(hc, __fdividef(0.3f, fabsf(y3) + 1e-30f));
                }
                const float* k1 = R.k1;
                float k2[6], k3[6], k4[6], k5[6], k6[6];
                const float yy[4] = {y0, y1, y2, y3};
                float t[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) t[i] = fmaf(hc, (float)A21 * k1[i], yy[i]);
                rhs32(c, t[0], t[1], t[2], t[3], k2);
#pragma unroll
                for (int i = 0; i < 4; ++i) t[i] = fmaf(hc, fmaf((float)A32, k2[i], (float)A31 * k1[i]), yy[i]);
                rhs32(c, t[0], t[1], t[2], t[3], k3);
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    t[i] = fmaf(hc, fmaf((float)A43, k3[i], fmaf((float)A42, k2[i], (float)A41 * k1[i])), yy[i]);
                rhs32(c, t[0], t[1], t[2], t[3], k4);
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    t[i] = fmaf(hc, fmaf((float)A54, k4[i], fmaf((float)A53, k3[i], fmaf((float)A52, k2[i],
                                                                                        (float)A51 * k1[i]))), yy[i]);
                rhs32(c, t[0], t[1], t[2], t[3], k5);
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    t[i] = fmaf(hc, fmaf((float)A65, k5[i], fmaf((float)A64, k4[i], fmaf((float)A63, k3[i],
                                   fmaf((float)A62, k2[i], (float)A61 * k1[i])))), yy[i]);
                rhs32(c, t[0], t[1], t[2], t[3], k6);
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    dy[i] = hc * fmaf((float)B6, k6[i], fmaf((float)B5, k5[i], fmaf((float)B4, k4[i],
                                      fmaf((float)B3, k3[i], (float)B1 * k1[i]))));
                nrh = R.rh; nrl = R.rl; nprh = R.prh; nprl = R.prl; nuh = R.uh; nul = R.ul; npuh = R.puh; npul = R.pul;
                acc2(nrh, nrl, dy[0]);
                acc2(nprh, nprl, dy[1]);
                acc2(nuh, nul, dy[2]);
                acc2(npuh, npul, dy[3]);
                n0 = nrh + nrl;
                n1 = nprh + nprl;
                n2 = nuh + nul;
                const float n3 = npuh + npul;
                rhs32(c, n0, n1, n2, n3, k7);
                // error norm of kerr.hpp:143-155 at tol32
                float sc[5];
                sc[0] = tol * (1e-6f + fmaxf(fabsf(y0), fabsf(n0)));
                sc[1] = tol * (1e-6f + fmaxf(fmaxf(fabsf(y1), fabsf(n1)), y0 * y0));
                sc[2] = tol;
                sc[3] = tol * fmaxf(1.f, fmaxf(fabsf(y3), fabsf(n3)));
                sc[4] = tol * 4.f;
#pragma unroll
                for (int i = 0; i < 5; ++i) {
                    float e = hc * fmaf((float)E7, k7[i], fmaf((float)E6, k6[i], fmaf((float)E5, k5[i],
                                        fmaf((float)E4, k4[i], fmaf((float)E3, k3[i], (float)E1 * k1[i])))));
                    err = fmaxf(err, __fdividef(fabsf(e), sc[i]));
                }
                if (!(err <= 1.f)) {
                    R.h = hc * fmaxf(0.2f, 0.9f * __powf(fmaxf(err, 1e-30f), -0.2f));
                    if (!(err == err)) R.h = hc * 0.1f;
                } else {
                    accepted = true;
                    ++R.nacc;
                    if (radio) {
                        float sn = sqrtf(fmaxf((1.f - n2) * (1.f + n2), 0.f)), s4, c4;
                        float phn = (R.phh + R.phl) + dy[4];
                        __sincosf(phn, &s4, &c4);
                        float pn0 = sn * c4, pn1 = sn * s4, pn2 = n2;
                        float cx = fmaf(R.pp1, pn2, -(R.pp2 * pn1)), cy = fmaf(R.pp2, pn0, -(R.pp0 * pn2)),
                              cz = fmaf(R.pp0, pn1, -(R.pp1 * pn0));
                        R.psi += atan2f(sqrtf(fmaf(cz, cz, fmaf(cy, cy, cx * cx))),
                                        fmaf(R.pp2, pn2, fmaf(R.pp1, pn1, R.pp0 * pn0)));
                        R.pp0 = pn0;
                        R.pp1 = pn1;
                        R.pp2 = pn2;
                    }
                    if ((y2 > 0.f) != (n2 > 0.f)) ++R.ncross;
                    if ((y1 < 0.f) && (n1 >= 0.f) && n0 < (float)L.turn_r) fate = 3;
                    want_flow = radio && S.flow_on && n0 < rflow && fate == 2;
                    if (want_flow && tp.n_modes > 0) {
                        // torus turbulence position: the flow-advected azimuth at the emission time
                        // counted from the radial light-travel time to the camera (so_emission.cuh)
                        float s2 = fmaxf((1.f - n2) * (1.f + n2), 1e-12f), s = sqrtf(s2);
                        float Rc = n0 * s, zh = __fdividef(n2, tp.h_sph);
                        if (Rc >= 1e-3f && __expf(-0.5f * zh * zh) >= 1e-7f) {
                            float ph_h = R.phh, ph_l = R.phl, t_h = R.th, t_l = R.tl;
                            acc2(ph_h, ph_l, dy[4]);
                            acc2(t_h, t_l, dy[5]);
                            float t_rel = ((t_h + rcam_hi) + (t_l + rcam_lo)) - n0 +
                                          2.f * __logf(__fdividef(rcam_hi, n0));
                            float Rk = fmaxf(Rc, risco);
                            float Omf = flow_kep * __frcp_rn(fmaf(Rk, sqrtf(Rk), c.a));
                            float phc = (ph_h + ph_l) - Omf * t_rel;
                            if (DEFER) {
                                // order n = floor(psi / pi) (>= 3 as 3) in the sign bits of r and h
                                const int nb = min((int)(R.psi * (float)(1.0 / PI)), 3);
                                rec = make_float4((nb & 1) ? -n0 : n0, n2, phc, (nb & 2) ? -hc : hc);
                            } else {
                                float sp, cp;
                                __sincosf(phc, &sp, &cp);
                                TX = Rc * cp;
                                TY = Rc * sp;
                                TZ = n0 * n2;
                            }
                            want_turb = true;
                        }
                    }
                    if (want_flow && baked) {
                        // the reference flow's baked turbulence (emission.cuh:112-124) at the end of
                        // the step, its retarded time t - t_ref(r) from the two-float t
                        float s2 = fmaxf((1.f - n2) * (1.f + n2), 1e-12f);
                        float Rc = n0 * sqrtf(s2);
                        if (Rc >= 1e-3f) {
                            float ph_h = R.phh, ph_l = R.phl, t_h = R.th, t_l = R.tl;
                            acc2(ph_h, ph_l, dy[4]);
                            acc2(t_h, t_l, dy[5]);
                            float tr = (((t_h + rcam_hi) + (t_l + rcam_lo)) - n0 + 2.f * __logf(__fdividef(rcam_hi, n0))) - tcam;
                            float y = __fdividef(__logf(Rc) - S.turb_lr0, S.turb_lr1 - S.turb_lr0);
                            float x = (ph_h + ph_l) * (float)(0.5 / PI);
                            float w = 0.5f + 0.5f * __fdividef(__fdividef(n0 * n2, Rc), S.turb_zmax);
                            float sl = __fdividef(tr - S.turb_d0, S.turb_dd);
                            sl = fminf(fmaxf(sl, 0.f), (float)(TURB_NT - 1) - 1e-4f);
                            const int k = (int)sl;
                            const float f = sl - (float)k;
                            const float A = baked_sample(S, L.turb_field, k, x, y, w);
                            const float B = baked_sample(S, L.turb_field, k + 1, x, y, w);
                            bfac = fmaf(B - A, f, A);
                        }
                    }
                    if (DEFER && want_flow && !tp.on) {
                        // reference flow model: record the steps flow_step32 does not return at once
                        // from (its first tests, in its own arithmetic) with their turbulence factor,
                        // fetched above exactly as the in-line form fetches it
                        float s2 = fmaxf((1.f - n2) * (1.f + n2), 1e-12f);
                        float Rc = n0 * sqrtf(s2);
                        if (Rc >= 1e-3f) {
                            float zh = __fdividef(n0 * n2, (float)S.h_r * Rc);
                            if (!(__expf(-0.5f * zh * zh) < 1e-7f)) {
                                const int nb = min((int)(R.psi * (float)(1.0 / PI)), 3);
                                rec = make_float4((nb & 1) ? -n0 : n0, n2, 0.f, (nb & 2) ? -hc : hc);
                                rec_bf = bfac;
                                want_turb = true;
                            }
                        }
                    }
                }
            }
        }
        // ---- all lanes: turbulence sums of the lanes that need one ------------------------------
        float delta = 0.f;
        if (DEFER) {
            // record slot: lanes whose segment is full take the next ones (one atomic per warp)
            const bool need_seg = want_turb && R.cnt == REC_SEG;
            const unsigned ms = __ballot_sync(FULL, need_seg);
            if (ms) {
                const int leader = __ffs(ms) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(&L.nlists[5], (unsigned long long)__popc(ms));
                base = __shfl_sync(FULL, base, leader);
                if (need_seg) {
                    const unsigned long long idx = base + __popc(ms & ((1u << lane) - 1u));
                    if (idx >= (unsigned long long)L.seg_cap) {
                        fate = 5;  // out of record segments: the FP64 tracer takes the ray
                        want_turb = false;
                    } else {
                        if (R.seg >= 0) L.seg_next[R.seg] = (uint32_t)idx;
                        else R.head = (int)idx;
                        R.seg = (int)idx;
                        R.cnt = 0;
                    }
                }
            }
            if (want_turb) {
                L.rec[(long long)R.seg * REC_SEG + R.cnt] = rec;
                if (!tp.on) L.rec_delta[(long long)R.seg * REC_SEG + R.cnt] = rec_bf;
                ++R.cnt;
                ++R.nrec;
            }
        } else if (VAR == VAR_RADIO && tp.n_modes > 0) {
            delta = warp_turbulence(km, amp, tp.n_modes, want_turb, TX, TY, TZ);
        }
        // ---- part 2 (active lanes): emission, commit, termination ------------------------------
        if (!active) continue;
        if (accepted) {
            if (VAR == VAR_DISK && S.disk_on && fate == 2 && ((R.uh + R.ul > 0.f) != (n2 > 0.f))) {
                // rare: the disk shading of the FP64 tracer on the crossing found in FP64
                const float y0 = R.rh + R.rl, y1 = R.prh + R.prl, y2 = R.uh + R.ul, y3 = R.puh + R.pul;
                double lo = 0.0, hi = 1.0, u0 = y2, u1 = n2, m0 = (double)y3 * hc, m1 = (double)(npuh + npul) * hc;
                for (int b = 0; b < 40; ++b) {
                    double mid = 0.5 * (lo + hi);
                    double um = hermite(u0, u1, m0, m1, mid);
                    if ((um > 0.0) == (u0 > 0.0)) lo = mid;
                    else hi = mid;
                }
                double scr = 0.5 * (lo + hi);
                double rc = hermite(y0, n0, (double)y1 * hc, (double)n1 * hc, scr);
                double ph0 = (double)R.phh + R.phl, t0 = (double)R.th + R.tl;
                double pc = hermite(ph0, ph0 + dy[4], (double)R.k1[4] * hc, (double)k7[4] * hc, scr);
                double tcv = hermite(t0, t0 + dy[5], (double)R.k1[5] * hc, (double)k7[5] * hc, scr);
                float cs[4];
                disk_shade(S, rc, pc, tcv, c.lam, c.eta, c.E, cs);
                if (cs[3] > 0.f) {
                    float tf = R.trans;
                    R.acc[0] += tf * cs[0];
                    R.acc[1] += tf * cs[1];
                    R.acc[2] += tf * cs[2];
                    R.acc[3] += tf * cs[1] * (float)(R.ncross - 1);
                    R.trans *= 1.f - cs[3];
                    if (R.trans < 1e-4f) fate = -1;
                }
            }
            if (DEFER && want_flow) ++R.nflow;
            if (!DEFER && want_flow) {
                float dI, dtau;
                flow_step32(S, tp, delta, n0, n2, c.lam, c.E, hc, &dI, &dtau, bfac);
                ++R.nflow;
                float cc = R.trans * dI;
                int nb = (int)(R.psi * (float)(1.0 / PI));
                R.acc[0] += cc;
                if (nb == 1) R.acc[1] += cc;
                else if (nb == 2) R.acc[2] += cc;
                else if (nb >= 3) R.acc[3] += cc;
                R.trans *= __expf(-dtau);
                if (R.trans < 1e-5f) fate = -1;
            }
            // commit the step
            R.rh = nrh; R.rl = nrl; R.prh = nprh; R.prl = nprl;
            R.uh = nuh; R.ul = nul; R.puh = npuh; R.pul = npul;
            acc2(R.phh, R.phl, dy[4]);
            acc2(R.th, R.tl, dy[5]);
#pragma unroll
            for (int i = 0; i < 6; ++i) R.k1[i] = k7[i];
            // project_radial (kerr.hpp:166-173) in FP32
            {
                float r = n0, P = fmaf(r, r, c.CP), D = fmaf(r, r - 2.f, c.A2);
                float Rr = fmaf(P, P, -(D * c.K)), r2 = r * r;
                if (Rr > 0.25f * (r2 * r2)) {
                    float v = sqrtf(Rr);
                    float pr = n1 < 0.f ? -v : v;
                    R.prh = pr;
                    R.prl = 0.f;
                    R.k1[0] = pr;
                }
            }
            R.h = hc * fminf(5.f, fmaxf(0.2f, 0.9f * __powf(fmaxf(err, 1e-30f), -0.2f)));
            if (fate == 2) {
                if (n0 < rstop) fate = -1;
                else if (n0 > resc && R.prh > 0.f) fate = 1;
                // outgoing beyond every emitter and beyond the largest radial turning point the
                // constants of motion allow (R(r) ~ r^4 - (eta + lam^2) r^2 + ...): no more emission,
                // the ray escapes; its escape direction is not part of the FP32 outputs
                else if (r_out > 0.f && R.prh > 0.f && n0 > r_out && n0 * n0 > 4.f * (c.eta + c.lam * c.lam + c.A2) + 16.f)
                    fate = 1;
            }
        }
        if (fate == 2) continue;
        // ---- ray finished: FP64 Carter-constant / radial constraint check ------------------------
        if (fate == -1 || fate == 1) {
            double r = (double)R.rh + R.rl, pr = (double)R.prh + R.prl, u = (double)R.uh + R.ul,
                   pu = (double)R.puh + R.pul;
            double lam = c.lam, eta = c.eta, a = S.a;
            double U = (1.0 - u * u) * (eta + a * a * u * u) - lam * lam * u * u;
            double scaleU = eta + a * a + lam * lam + 1e-12;
            double P = r * r + a * a - a * lam, D = r * r - 2.0 * r + a * a;
            double Rr = P * P - D * (eta + (lam - a) * (lam - a));
            double dU = fabs(pu * pu - U) / scaleU, dR = fabs(pr * pr - Rr) / (r * r * r * r);
            if (dU > L.drift_tol || dR > L.drift_tol) fate = 4;
        }
        n_att += (unsigned long long)R.natt;
        n_acc += (unsigned long long)R.nacc;
        n_flow += (unsigned long long)R.nflow;
        // a ray that used up max_steps in FP32 (the FP32 controller can stall where FP64 does not)
        // is decided by the FP64 tracer, like the constraint and turning-point failures
        const bool redo = fate >= 3 || fate == 0;
        n_turn += fate == 3 ? 1 : 0;
        n_drift += fate == 4 ? 1 : 0;
        n_lim += fate == 0 ? 1 : 0;
        if (fate == 5) atomicAdd(&L.nlists[6], 1ull);
        if (!redo && fate == 1 && L.esc_list) {
            // star-map frame: park the end state for the FP64 transport to the escape radius
            L.state[0 * ns + R.sid] = make_float4(R.rh, R.rl, R.prh, R.prl);
            L.state[1 * ns + R.sid] = make_float4(R.uh, R.ul, R.puh, R.pul);
            L.state[2 * ns + R.sid] = make_float4(R.phh, R.phl, R.th, R.tl);
            L.state[3 * ns + R.sid] = make_float4(c.lam, c.eta, c.E, R.h);
            L.state[4 * ns + R.sid] = make_float4(R.trans, 0.f, 0.f, 0.f);
            L.esc_list[atomicAdd(&L.nlists[9], 1ull)] = R.sid;
        }
        if (!redo) {
            if (DEFER && R.nrec > 0) {
                // emission by k_flow_records (which may still end the ray on its opacity)
                L.ray_meta[R.sid] = make_int2(R.head, R.nrec);
                L.acc_list[atomicAdd(&L.nlists[4], 1ull)] = R.sid;
            } else {
                L.sample_out[R.sid] = make_float4(R.acc[0], R.acc[1], R.acc[2], R.acc[3]);
            }
            if (L.sample_fate) L.sample_fate[R.sid] = (int8_t)fate;
        }
        active = false;
        // re-trace list: lanes finish at different iterations, so append without a warp vote
        if (redo) L.redo[atomicAdd(&L.nlists[2], 1ull)] = R.sid;
    }
    for (int o = 16; o > 0; o >>= 1) {
        n_att += __shfl_down_sync(FULL, n_att, o);
        n_acc += __shfl_down_sync(FULL, n_acc, o);
        n_flow += __shfl_down_sync(FULL, n_flow, o);
        n_lim += __shfl_down_sync(FULL, n_lim, o);
        n_turn += __shfl_down_sync(FULL, n_turn, o);
        n_drift += __shfl_down_sync(FULL, n_drift, o);
    }
    if (lane == 0) {
        atomicAdd(&L.counters->attempts, n_att);
        atomicAdd(&L.counters->pad[1], n_acc);  // FP32 accepted steps
        atomicAdd(&L.counters->flow_steps, n_flow);
        atomicAdd(&L.counters->redo_limit, n_lim);
        atomicAdd(&L.counters->redo_turn, n_turn);
        atomicAdd(&L.counters->redo_drift, n_drift);
    }
}

// ---- deferred turbulence: batched mode sums, ordered transfer ------------------------------------
// Torus parameters of the launch in FP32 (as the tracer sets them up).
__device__ __forceinline__ Torus32 torus32_of(const TraceLaunch& L) {
    Torus32 tp;
    tp.on = L.torus;
    tp.n_modes = L.torus ? L.n_modes : 0;
    tp.ne_index = (float)L.ne_index;
    tp.te_index = (float)L.te_index;
    tp.h_sph = (float)L.h_sph;
    tp.theta_e0 = (float)L.theta_e0;
    tp.half_var = (float)L.half_var;
    return tp;
}

// Turbulence sum at every record slot in use: the records' positions (the tracer's in-line form:
// R = r sqrt(max((1-u)(1+u), 1e-12)), x = R cos phi_c, y = R sin phi_c, z = r u), TURB_P positions
// per thread, the modes read from constant memory (the kernel parameter M, the same address for the
// whole warp: no shared-memory loads in the MIO queue that feeds the SFU), so every lane does the
// same work and the SFU cosine is the bound (three FMAs, the cosine's scaling multiply, the cosine
// and one FMA per mode and position).  Each mode's constant loads serve TURB_P positions: measured
// on the 2048^2 frame, 8 positions (64 registers, 4 CTAs / SM) 142.6 ms at 0.85 of the SFU rate, 12
// (80 registers, 3 CTAs) 134.0 ms at 0.90, 16 (126 registers, 2 CTAs) 142.3 ms.  Blocks take chunks
// of TURB_P x 256 slots from a work counter, so SMs that also host the FP64 re-trace (on the other
// stream) do less of it instead of finishing last.  Slots of a segment past its ray's last record
// hold stale data; their sums are never read.
constexpr int TURB_P = 12;
constexpr int TURB_CHUNK = TURB_P * 256;
__global__ void __launch_bounds__(256) k_turb_records(const TraceLaunch L, const __grid_constant__ TurbModes M) {
    const int nm = M.n;
    __shared__ long long chunk;
    unsigned long long used = L.nlists[5];
    if (used > (unsigned long long)L.seg_cap) used = (unsigned long long)L.seg_cap;
    const long long nslots = (long long)used * REC_SEG;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&L.nlists[10], used);
    for (;;) {
        __syncthreads();  // modes loaded; the previous chunk index read by every thread
        if (threadIdx.x == 0) chunk = (long long)atomicAdd(&L.nlists[7], 1ull) * TURB_CHUNK;
        __syncthreads();
        const long long c0 = chunk;
        if (c0 >= nslots) break;
        const long long i = c0 + threadIdx.x;  // slots i + 256 q, q < TURB_P
        float x[TURB_P], y[TURB_P], z[TURB_P], acc[TURB_P];
#pragma unroll
        for (int q = 0; q < TURB_P; ++q) {
            const long long j = min(i + q * 256, nslots - 1);
            const float4 v = L.rec[j];
            const float r = fabsf(v.x), u = v.y;
            const float s2 = fmaxf((1.f - u) * (1.f + u), 1e-12f), Rc = r * sqrtf(s2);
            float sp, cp;
            __sincosf(v.z, &sp, &cp);
            x[q] = Rc * cp;
            y[q] = Rc * sp;
            z[q] = r * u;
            acc[q] = 0.f;
        }
#pragma unroll 2
        for (int m = 0; m < nm; ++m) {
            const float4 k = M.k[m];
            const float am = M.a[m];
#pragma unroll
            for (int q = 0; q < TURB_P; ++q)
                acc[q] = fmaf(am, __cosf(fmaf(k.z, z[q], fmaf(k.y, y[q], fmaf(k.x, x[q], k.w)))), acc[q]);
        }
#pragma unroll
        for (int q = 0; q < TURB_P; ++q)
            if (i + q * 256 < nslots) L.rec_delta[i + q * 256] = acc[q];
    }
}

// Ordered transfer per ray (trace.cuh:130-143 in the tracer's FP32 form), one warp per ray: the
// warp takes 32 records (two segments) at a time, each lane runs flow_step32 on one with its
// turbulence sum, an inclusive warp scan of dtau gives every record the transmittance in front of
// it, T exp(-sum of the dtau before it) (the in-line form multiplies the factors one by one: the
// same to FP32 rounding), and the ray ends (class captured) after the first record behind which
// the transmittance is below 1e-5, that record's light included.  Sums by photon-ring order.  Warps
// take rays from a work counter (record counts per ray range from one to thousands).
__global__ void __launch_bounds__(256) k_flow_records(const TraceLaunch L) {
    const so_scene& S = L.scenes[0];
    const Torus32 tp = torus32_of(L);
    const long long n = (long long)L.nlists[4];
    const long long ns = L.nsamples;
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long ii = 0;
        if (lane == 0) ii = atomicAdd(&L.nlists[8], 1ull);
        const long long i = (long long)__shfl_sync(FULL, ii, 0);
        if (i >= n) break;
        const uint32_t sid = L.acc_list[i];
        const int2 meta = L.ray_meta[sid];
        const float4 p3 = L.state[3 * ns + sid];
        const float lam = p3.x, E = p3.z;
        const int nrec = meta.y;
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, T = 1.f;
        bool opaque = false;
        long long sa = meta.x;
        for (int k0 = 0; k0 < nrec && !opaque; k0 += 32) {
            const long long sb = k0 + 16 < nrec ? (long long)L.seg_next[sa] : sa;
            const int k = k0 + lane;
            float dI = 0.f, dtau = 0.f;
            int nb = 0;
            if (k < nrec) {
                const long long j = (lane < 16 ? sa : sb) * REC_SEG + (lane & 15);
                const float4 v = L.rec[j];
                // torus: the turbulence sum; reference flow: the baked turbulence factor
                const float delta = L.rec_delta[j];
                nb = (int)(__float_as_uint(v.x) >> 31) | (int)((__float_as_uint(v.w) >> 31) << 1);
                flow_step32(S, tp, tp.on ? delta : 0.f, fabsf(v.x), v.y, lam, E, fabsf(v.w), &dI, &dtau,
                            tp.on ? 1.f : delta);
            }
            float incl = dtau;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float t = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += t;
            }
            const float Tb = T * __expf(-(incl - dtau)), Ta = T * __expf(-incl);
            const unsigned cut = __ballot_sync(FULL, k < nrec && Ta < 1e-5f);
            bool use = k < nrec;
            if (cut) {
                use = use && lane <= __ffs(cut) - 1;
                opaque = true;
            }
            const float cc = use ? Tb * dI : 0.f;
            a0 += cc;
            a1 += nb == 1 ? cc : 0.f;
            a2 += nb == 2 ? cc : 0.f;
            a3 += nb == 3 ? cc : 0.f;
            T = __shfl_sync(FULL, Ta, 31);
            if (k0 + 32 < nrec) sa = (long long)L.seg_next[sb];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(FULL, a0, o);
            a1 += __shfl_xor_sync(FULL, a1, o);
            a2 += __shfl_xor_sync(FULL, a2, o);
            a3 += __shfl_xor_sync(FULL, a3, o);
        }
        if (lane == 0) {
            L.sample_out[sid] = make_float4(a0, a1, a2, a3);
            if (opaque && L.sample_fate) L.sample_fate[sid] = -1;
        }
    }
}

// ---- star map behind FP32 rays -----------------------------------------------------------------
// An FP32 ray of a star-map frame that escaped (beyond every emitter and radial turning point, or
// past r_escape) is carried to r_escape in FP64 by the inverse-radius transport (a few DP5 steps
// where Mino time takes hundreds; the Mino-time DP5(4) where that does not apply), its escape
// direction is taken there as the reference takes it
// (escape_angles, trace.cuh:45-55), and the star map's radiance through the pixel's footprint,
// weighted by the transmittance in front, is added to the sample (trace.cuh:149-161).
__global__ void __launch_bounds__(128) k_sky_escape(const TraceLaunch L) {
    const so_scene& S = L.scenes[0];
    const long long n = (long long)L.nlists[9];
    const long long ns = L.nsamples;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t sid = L.esc_list[i];
        const float4 p0 = L.state[0 * ns + sid], p1 = L.state[1 * ns + sid], p2 = L.state[2 * ns + sid];
        const float4 p3 = L.state[3 * ns + sid], p4 = L.state[4 * ns + sid];
        double y[6] = {(double)p0.x + p0.y, (double)p0.z + p0.w, (double)p1.x + p1.y,
                       (double)p1.z + p1.w, (double)p2.x + p2.y, (double)p2.z + p2.w};
        RayC c;
        ray_consts(c, S.a, (double)p3.x, (double)p3.y, (double)p3.z);
        double psi = 0.0;
        int nc = 0;
        double k[6];
        bool there = !(y[0] < S.r_escape);
        if (!there && far_applies(c, y, S.r_escape))
            there = far_approach(c, y, S.r_escape, S.tol, 256, &psi, &nc, false) >= 0;
        rhs(c, y, k);
        if (!there) {
            // the reference's Mino-time DP5(4) out to r_escape (trace.cuh:80-96, 150)
            double yn[6], k7[6];
            double h = initial_step(y);
            for (int it = 0; it < S.max_steps && !(y[0] > S.r_escape && y[1] > 0.0); ++it) {
                const double hc = h;
                const double err = dp54(c, y, k, hc, S.tol, yn, k7);
                if (!(err <= 1.0)) {
                    h = reject_step(hc, err);
                    continue;
                }
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    y[q] = yn[q];
                    k[q] = k7[q];
                }
                project_radial(c, y, k);
                h = accept_step(hc, err);
            }
        }
        double th, ph;
        escape_angles(y, k, &th, &ph);
        const long long pix = sid / L.spp;
        const SkyGrad g = pixel_grad(L.sky_uv, L.W, (int)(pix % L.W), (int)(pix / L.W), L.sky_grad_scale);
        float xyz[3];
        sky_radiance(S, sky_uv(S, th, ph), g, c.E, xyz);
        const float tf = p4.x;
        float4 o = L.sample_out[sid];
        o.x += tf * xyz[0];
        o.y += tf * xyz[1];
        o.z += tf * xyz[2];
        L.sample_out[sid] = o;
    }
}

// ---- launchers -----------------------------------------------------------------------------------
cudaError_t launch_sky_escape(const TraceLaunch& L, int num_sms, cudaStream_t st) {
    k_sky_escape<<<num_sms * 4, 128, 0, st>>>(L);
    return cudaGetLastError();
}

void turb_modes_fold(const so_mode* modes, int n, TurbModes* out) {
    out->n = n;
    for (int i = 0; i < n; ++i) {
        const so_mode& m = modes[i];
        const double ph = m.phase - 2.0 * PI * floor(m.phase / (2.0 * PI) + 0.5);
        out->k[i] = make_float4((float)m.kx, (float)m.ky, (float)m.kz, (float)ph);
        out->a[i] = (float)m.amp;
    }
}

cudaError_t launch_turb_records(const TraceLaunch& L, const TurbModes& M, int num_sms, cudaStream_t st) {
    int per_sm = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_turb_records, 256, 0);
    if (e != cudaSuccess) return e;
    k_turb_records<<<num_sms * (per_sm > 0 ? per_sm : 1), 256, 0, st>>>(L, M);
    return cudaGetLastError();
}

cudaError_t launch_flow_records(const TraceLaunch& L, int num_sms, cudaStream_t st) {
    int per_sm = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flow_records, 256, 0);
    if (e != cudaSuccess) return e;
    k_flow_records<<<num_sms * (per_sm > 0 ? per_sm : 1), 256, 0, st>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_route(const TraceLaunch& L, int all64, cudaStream_t st) {
    long long blocks = (L.nsamples + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_route<<<(int)(blocks > 0 ? blocks : 1), 256, 0, st>>>(L, all64);
    return cudaGetLastError();
}

cudaError_t launch_approach64(const TraceLaunch& L, long long n, int num_sms, cudaStream_t st) {
    int per_sm = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_approach64, 128, 0);
    if (e != cudaSuccess) return e;
    long long grid = (long long)num_sms * (per_sm > 0 ? per_sm : 1);
    long long want = (n + 127) / 128;
    if (grid > want) grid = want > 0 ? want : 1;
    k_approach64<<<(int)grid, 128, 0, st>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_trace32(const TraceLaunch& L, long long n, int variant, int num_sms, cudaStream_t st) {
    const bool torus = variant == VAR_RADIO && L.torus && L.n_modes > 0;
    const bool defer = variant == VAR_RADIO && L.defer;
    size_t smem = torus && !defer ? (size_t)L.n_modes * (sizeof(float4) + sizeof(float)) : 0;
    int per_sm = 1;
    cudaError_t e;
    auto go = [&](auto kern) -> cudaError_t {
        if (smem > 48 * 1024) {
            cudaError_t e2 = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e2 != cudaSuccess) return e2;
        }
        cudaError_t e2 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem);
        if (e2 != cudaSuccess) return e2;
        long long grid = (long long)num_sms * (per_sm > 0 ? per_sm : 1);
        long long want = (n + 127) / 128;
        if (grid > want) grid = want > 0 ? want : 1;
        kern<<<(int)grid, 128, smem, st>>>(L);
        return cudaGetLastError();
    };
    // register budget: 4 CTAs of 128 per SM (128 registers, no spills) or 5 / 6 (96 / 80 registers,
    // a few spills to L1); chosen by the caller or the autotuner
    switch (variant) {
        case VAR_VACUUM: e = go(k_trace32<VAR_VACUUM, 4, false>); break;
        case VAR_DISK: e = go(k_trace32<VAR_DISK, 4, false>); break;
        default:
            if (defer)
                e = L.t32_min_blocks >= 6 ? go(k_trace32<VAR_RADIO, 6, true>)
                    : L.t32_min_blocks == 5 ? go(k_trace32<VAR_RADIO, 5, true>) : go(k_trace32<VAR_RADIO, 4, true>);
            else
                e = L.t32_min_blocks >= 6 ? go(k_trace32<VAR_RADIO, 6, false>)
                    : L.t32_min_blocks == 5 ? go(k_trace32<VAR_RADIO, 5, false>) : go(k_trace32<VAR_RADIO, 4, false>);
            break;
    }
    return e;
}

}  // namespace so
