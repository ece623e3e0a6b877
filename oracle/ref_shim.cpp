// ref_shim.cpp -- host build of the REFERENCE's own tracer code.  TEST INFRASTRUCTURE ONLY.
//
// This translation unit includes the reference's blackholes/src/trace.cuh (which pulls in
// emission.cuh, device_util.cuh, scene.hpp, kerr.hpp, common.hpp) where it lies and compiles it as
// host C++.  The device-only builtins it uses are mapped to host equivalents below:
//   __ldg(p)   -> *p                       (device_util.cuh:79, 428)
//   __expf(x)  -> expf(x)                  (emission.cuh:55, 71)
//   rsqrtf(x)  -> 1.0f / sqrtf(x)          (emission.cuh:50)
//   tex3D / tex2DGrad -> zero stubs        (baked turbulence and sky: not used by the configs here)
// render.cu's turbulence bake k_bake_turb (render.cu:448-461) is cut out by line range into
// _ref/bake_kernel.inc by oracle/Makefile and compiled at the end of this file with its launch grid
// walked on the host and surf3Dwrite writing one z layer into a host array.
// The reference's own host builders (scene_build.cpp, shot.cpp, config.cpp, colour.cpp) are
// compiled unchanged by oracle/Makefile and linked in.  sample_pixel / pixel_seed of render.cu:70-85
// are restated here (render.cu itself needs the CUDA toolchain and the font atlas), calling the
// reference's pcg / rnd / r2_sample / trace_ray.
//
// Output: oracle/_ref/libbhref.so, loaded by tests/golden/make_golden.py (fixtures), by tests that
// pin the oracle and by bench.py --impl reference (the reference's CPU integrator, timed).
#include <cuda_runtime.h>

#include <cmath>
#define __ldg(p) (*(p))
#define __expf(x) expf(x)
static inline float so_ref_rsqrtf(float x) { return 1.0f / sqrtf(x); }
#define rsqrtf so_ref_rsqrtf
template <class T>
T tex3D(unsigned long long, float, float, float) { return T(); }
template <class T>
T tex2DGrad(unsigned long long, float, float, float2, float2) { return T(); }

#include "trace.cuh"
#include "scene_build.hpp"
#include "shot.hpp"

#include <cstddef>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {
struct RefShot {
    Config cfg;
    SceneGPU S;
    SceneTables T;
    SceneInfo info;
    Shot shot;
};

// render.cu:70-74
void pixel_seed_h(int p, uint32_t* h, float* r0, float* r1) {
    *h = pcg((uint32_t)p * 0x9E3779B9u ^ c_F.seed);
    *r0 = rnd(*h);
    *r1 = rnd(*h);
}
}  // namespace

extern "C" {

// Layout of SceneGPU / FrameGPU, to check the C ABI mirror field by field.
int ref_layout(long long* out, int cap) {
    const long long v[] = {
        (long long)sizeof(SceneGPU), (long long)sizeof(FrameGPU), (long long)offsetof(SceneGPU, tol),
        (long long)offsetof(SceneGPU, max_steps), (long long)offsetof(SceneGPU, r_escape),
        (long long)offsetof(SceneGPU, mode), (long long)offsetof(SceneGPU, disk_on),
        (long long)offsetof(SceneGPU, disk_lnT), (long long)offsetof(SceneGPU, disk_turb_amp),
        (long long)offsetof(SceneGPU, disk_plunge), (long long)offsetof(SceneGPU, flow_on),
        (long long)offsetof(SceneGPU, n0), (long long)offsetof(SceneGPU, flow_kep),
        (long long)offsetof(SceneGPU, flow_turb_amp), (long long)offsetof(SceneGPU, turb_tex),
        (long long)offsetof(SceneGPU, turb_nt), (long long)offsetof(SceneGPU, turb_dd),
        (long long)offsetof(SceneGPU, k2_lntab), (long long)offsetof(SceneGPU, k2_n),
        (long long)offsetof(SceneGPU, k2_dl), (long long)offsetof(SceneGPU, sky_on),
        (long long)offsetof(SceneGPU, sky_tex), (long long)offsetof(SceneGPU, sky_rot),
        (long long)offsetof(SceneGPU, bb_xyz), (long long)offsetof(SceneGPU, bb_dl),
        (long long)offsetof(SceneGPU, seed), (long long)offsetof(FrameGPU, kp),
        (long long)offsetof(FrameGPU, F), (long long)offsetof(FrameGPU, beta), (long long)offsetof(FrameGPU, cx),
        (long long)offsetof(FrameGPU, pix), (long long)offsetof(FrameGPU, W), (long long)offsetof(FrameGPU, spp),
        (long long)offsetof(FrameGPU, seed)};
    int n = (int)(sizeof v / sizeof v[0]);
    for (int i = 0; i < n && i < cap; ++i) out[i] = v[i];
    return n;
}

// Config::load + --set overrides (main.cpp:384-399) + build_scene + build_shot.
void* ref_shot_load(const char* path, const char* const* kv, int nkv) {
    RefShot* s = new RefShot;
    std::string err;
    if (!s->cfg.load(path, &err)) {
        delete s;
        return nullptr;
    }
    for (int i = 0; i < nkv; ++i) {
        std::string a = kv[i];
        size_t eq = a.find('=');
        if (eq != std::string::npos) s->cfg.set(trim(a.substr(0, eq)), trim(a.substr(eq + 1)));
    }
    if (!build_scene(s->cfg, &s->S, &s->T, &s->info, &err) || !build_shot(s->cfg, &s->shot, &err)) {
        delete s;
        return nullptr;
    }
    // Zoom target on the critical curve (main.cpp:421-428)
    if (s->shot.type == "render" && s->cfg.has("camera.target_psi_deg")) {
        double psi = s->cfg.num("camera.target_psi_deg", 0) * PI / 180;
        double rho = find_critical_point(s->shot, s->shot.frames[0], s->S.a, psi) + s->cfg.num("camera.target_offset_m", 0.0);
        s->shot.target_x = rho * std::cos(psi);
        s->shot.target_y = rho * std::sin(psi);
    }
    s->S.disk_lnT = s->T.disk_lnT.data();
    s->S.k2_lntab = s->T.k2_ln.data();
    s->S.bb_xyz = s->T.bb_xyz.data();
    return s;
}
void ref_shot_free(void* h) { delete (RefShot*)h; }
int ref_shot_nframes(void* h) { return (int)((RefShot*)h)->shot.frames.size(); }
// SceneGPU with the table pointers pointing at the shot's host tables.
void ref_shot_scene(void* h, void* scene_out) { std::memcpy(scene_out, &((RefShot*)h)->S, sizeof(SceneGPU)); }
void ref_shot_tables(void* h, const float** disk, int* nd, const float** k2, int* nk, const float** bb, int* nb) {
    RefShot* s = (RefShot*)h;
    *disk = s->T.disk_lnT.data();
    *nd = (int)s->T.disk_lnT.size();
    *k2 = s->T.k2_ln.data();
    *nk = (int)s->T.k2_ln.size();
    *bb = s->T.bb_xyz.data();
    *nb = (int)s->T.bb_xyz.size() / 3;
}
void ref_shot_info(void* h, double* out8) {
    const SceneInfo& i = ((RefShot*)h)->info;
    const double v[8] = {i.mass_msun, i.distance_cm, i.rg_cm, i.tg_s, i.uas_per_m, i.disk_tmax, i.disk_mdot_edd,
                         i.radio_flux_target_jy};
    std::memcpy(out8, v, sizeof v);
}
void ref_shot_settings(void* h, int* out4, float* target_err) {
    const Config& c = ((RefShot*)h)->cfg;
    out4[0] = c.integer("camera.width", 1920);
    out4[1] = c.integer("camera.height", 1080);
    out4[2] = c.integer("render.spp", 8);
    out4[3] = c.integer("render.spp_max", 128);
    *target_err = (float)c.num("render.target_error", 0.03);
}
// make_frame (shot.cpp:116-146).
void ref_shot_frame(void* h, int i, int W, uint32_t seed, void* frame_out) {
    RefShot* s = (RefShot*)h;
    FrameGPU F = make_frame(s->shot, s->shot.frames[i], s->S.a, W, seed);
    std::memcpy(frame_out, &F, sizeof F);
}
// find_critical_point (shot.cpp:148-164) for frame i's camera.
double ref_find_critical_point(void* h, int i, double a, double psi) {
    RefShot* s = (RefShot*)h;
    return find_critical_point(s->shot, s->shot.frames[i], a, psi);
}
// find_critical_point for a bare camera (the self-test's set-up, main.cpp:327-346).
double ref_find_critical_point_cam(double a, double r, double incl, double psi) {
    Shot sh;
    sh.motion = "static";
    ShotFrame f;
    f.r = r;
    f.incl = incl;
    f.fov_in_m = true;
    f.fov = 30;
    return find_critical_point(sh, f, a, psi);
}
int ref_critical_curve_point(double a, double th, double rp, double* al, double* be) {
    return critical_curve_point(a, th, rp, al, be) ? 1 : 0;
}
void ref_kerr_point(double a, double r, double th, void* kp_out) {
    KerrPoint k = kerr_point(a, r, th);
    std::memcpy(kp_out, &k, sizeof k);
}
// The self-test's radial drift (main.cpp:352-371), verbatim loop.
double ref_radial_drift(int* steps_out) {
    double a = 0.94;
    KerrPoint kp = kerr_point(a, 50.0, 1.2);
    Photon p = camera_photon(a, kp, 0, 0, normalize(dvec3{-1, 0.13, 0.11}), dvec3{0, 0, 0});
    double *y = p.y, k1[6], yn[6], k7[6];
    geodesic_rhs(a, p.lam, p.eta, y, k1);
    double h = initial_step(y), worst = 0;
    int steps = 0;
    for (int it = 0; it < 200000 && steps < 3000; ++it) {
        double err = dp54_step(a, p.lam, p.eta, y, k1, h, 1e-10, yn, k7);
        if (err > 1) { h *= std::max(0.2, 0.9 * std::pow(err, -0.2)); continue; }
        for (int i = 0; i < 6; ++i) { y[i] = yn[i]; k1[i] = k7[i]; }
        h *= std::min(5.0, std::max(0.2, 0.9 * std::pow(std::max(err, 1e-30), -0.2)));
        ++steps;
        double R = radial_potential(a, p.lam, p.eta, y[0]);
        worst = std::max(worst, std::fabs(R - y[1] * y[1]) / std::pow(y[0], 4.0));
        if (y[0] < horizon_radius(a) + 0.01 || y[0] > 1e4) break;
    }
    *steps_out = steps;
    return worst;
}

// The reference's noise at n points, for function-level pins of the oracle's noise (whole rays
// through turbulence are ill-conditioned in the noise phase): fbm3 (device_util.cuh:61-72) and
// sheared_noise (emission.cuh:34-51, which reads the scene's spin and ISCO radius).
void ref_fbm3(int n, const float* x, const float* y, const float* z, int oct, uint32_t seed, float* out) {
    for (int i = 0; i < n; ++i) out[i] = fbm3(x[i], y[i], z[i], oct, seed);
}
void ref_sheared_noise(const void* scene, int n, const double* R, const double* phi, const double* z, const double* t,
                       float scale, float tcorr, uint32_t seed, float* out) {
    std::memcpy(&c_S, scene, sizeof(SceneGPU));
    for (int i = 0; i < n; ++i) out[i] = sheared_noise(R[i], phi[i], z[i], t[i], scale, tcorr, seed);
}

// trace_ray (trace.cuh:62) for n tangent-plane points, nthreads host threads.  Outputs: fate (int8),
// theta/phi from escape_angles (recomputed from the uv path is not possible, so the shim exposes
// the reference's own escape_angles through a copy of the final state: see ref_trace_state).
int ref_trace_rays(const void* scene, const void* frame, int n, const double* x, const double* y, int8_t* fate,
                   float* I, int nthreads) {
    std::memcpy(&c_S, scene, sizeof(SceneGPU));
    std::memcpy(&c_F, frame, sizeof(FrameGPU));
    if (nthreads < 1) nthreads = 1;
    auto work = [&](int t0) {
        for (int i = t0; i < n; i += nthreads) {
            int f = 0;
            float2 uv;
            SkyGrad g = {make_float2(0, 0), make_float2(0, 0)};
            float4 v = trace_ray(x[i], y[i], g, false, &f, &uv);
            fate[i] = (int8_t)f;
            if (I) { I[4 * i] = v.x; I[4 * i + 1] = v.y; I[4 * i + 2] = v.z; I[4 * i + 3] = v.w; }
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
    return 0;
}

// Vacuum geometry of trace_ray with the reference's own kerr.hpp pieces, returning the outputs the
// tracer does not return by value: equatorial crossings (trace.cuh:104-105) and escape direction
// (escape_angles, trace.cuh:49-55).  The loop is trace_ray's (trace.cuh:81-163) for a scene with no
// emission (mode visible, disk off, sky off).
int ref_trace_vacuum(const void* scene, const void* frame, int n, const double* x, const double* y, int8_t* fate,
                     int8_t* ncross, double* th, double* ph, int32_t* nacc, int32_t* natt, int nthreads) {
    std::memcpy(&c_S, scene, sizeof(SceneGPU));
    std::memcpy(&c_F, frame, sizeof(FrameGPU));
    if (nthreads < 1) nthreads = 1;
    auto work = [&](int t0) {
        for (int i = t0; i < n; i += nthreads) {
            const double a = c_S.a;
            dvec3 d = normalize(c_F.F + c_F.R * (c_F.cx + x[i]) + c_F.U * (c_F.cy + y[i]));
            Photon p = camera_photon(a, c_F.kp, c_F.ph, c_F.t, d, c_F.beta);
            double* yy = p.y;
            double k1[6], yn[6], k7[6];
            geodesic_rhs(a, p.lam, p.eta, yy, k1);
            double h = initial_step(yy);
            int nc = 0, f = 0, acc = 0, att = 0;
            double t_ = 0, p_ = 0;
            for (int it = 0; it < c_S.max_steps; ++it) {
                double hc = h;
                ++att;
                double err = dp54_step(a, p.lam, p.eta, yy, k1, hc, c_S.tol, yn, k7);
                if (!(err <= 1.0)) {
                    h = hc * fmax(0.2, 0.9 * pow(fmax(err, 1e-30), -0.2));
                    if (!(err == err)) h = hc * 0.1;
                    continue;
                }
                ++acc;
                if ((yy[2] > 0.0) != (yn[2] > 0.0)) ++nc;
                for (int k = 0; k < 6; ++k) { yy[k] = yn[k]; k1[k] = k7[k]; }
                project_radial(a, p.lam, p.eta, yy, k1);
                h = hc * fmin(5.0, fmax(0.2, 0.9 * pow(fmax(err, 1e-30), -0.2)));
                if (yy[0] < c_S.r_stop) { f = -1; break; }
                if (yy[0] > c_S.r_escape && yy[1] > 0.0) {
                    f = 1;
                    escape_angles(yy, k1, &t_, &p_);
                    break;
                }
            }
            fate[i] = (int8_t)f;
            ncross[i] = (int8_t)(nc > 127 ? 127 : nc);
            th[i] = t_;
            ph[i] = p_;
            nacc[i] = acc;
            natt[i] = att;
        }
    };
    std::vector<std::thread> th_;
    for (int t = 1; t < nthreads; ++t) th_.emplace_back(work, t);
    work(0);
    for (auto& t : th_) t.join();
    return 0;
}

// k_pass1's per-pixel work (render.cu:89-115) on the host: spp R2-jittered samples per pixel.
int ref_render_pass1(const void* scene, const void* frame, float* accum, long long* nlim, int nthreads) {
    std::memcpy(&c_S, scene, sizeof(SceneGPU));
    std::memcpy(&c_F, frame, sizeof(FrameGPU));
    const int W = c_F.W, H = c_F.H;
    if (nthreads < 1) nthreads = 1;
    std::vector<long long> lim(nthreads, 0);
    auto work = [&](int t0) {
        for (int p = t0; p < W * H; p += nthreads) {
            int px = p % W, py = p / W;
            uint32_t h;
            float r0, r1;
            pixel_seed_h(p, &h, &r0, &r1);
            SkyGrad g = {make_float2(0, 0), make_float2(0, 0)};
            float4 a = make_float4(0, 0, 0, 0);
            for (int s = 0; s < c_F.spp; ++s) {
                float jx, jy;
                r2_sample((uint32_t)s, r0, r1, &jx, &jy);
                double tx = (px + jx - 0.5 * c_F.W) * c_F.pix;
                double ty = (0.5 * c_F.H - (py + jy)) * c_F.pix;
                int fate;
                float4 v = trace_ray(tx, ty, g, true, &fate, nullptr);
                if (fate == 0) ++lim[t0];
                a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
            }
            accum[4 * p] = a.x; accum[4 * p + 1] = a.y; accum[4 * p + 2] = a.z; accum[4 * p + 3] = a.w;
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
    long long L = 0;
    for (long long v : lim) L += v;
    if (nlim) *nlim = L;
    return 0;
}

// k_pass2's per-chunk work (render.cu:196-224) on the host: entry e is `count` samples s0[e] ..
// s0[e] + count - 1 of pixel pix[e] through sample_pixel's jitter, summed in float in sample order
// (the reference then adds each chunk sum to its pixel with float atomics).
int ref_render_chunks(const void* scene, const void* frame, long long n, const long long* pix, const int* s0,
                      int count, float* out, int nthreads) {
    std::memcpy(&c_S, scene, sizeof(SceneGPU));
    std::memcpy(&c_F, frame, sizeof(FrameGPU));
    const int W = c_F.W;
    if (nthreads < 1) nthreads = 1;
    auto work = [&](int t0) {
        for (long long e = t0; e < n; e += nthreads) {
            int p = (int)pix[e], px = p % W, py = p / W;
            uint32_t h;
            float r0, r1;
            pixel_seed_h(p, &h, &r0, &r1);
            SkyGrad g = {make_float2(0, 0), make_float2(0, 0)};
            float4 a = make_float4(0, 0, 0, 0);
            for (int i = 0; i < count; ++i) {
                float jx, jy;
                r2_sample((uint32_t)(s0[e] + i), r0, r1, &jx, &jy);
                double tx = (px + jx - 0.5 * c_F.W) * c_F.pix;
                double ty = (0.5 * c_F.H - (py + jy)) * c_F.pix;
                int fate;
                float4 v = trace_ray(tx, ty, g, true, &fate, nullptr);
                a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
            }
            out[4 * e] = a.x; out[4 * e + 1] = a.y; out[4 * e + 2] = a.z; out[4 * e + 3] = a.w;
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
    return 0;
}

}  // extern "C"

// k_bake_turb (render.cu:448-461) on the host.  The bake's surface is stood in for by a Layer: the
// texel row x (bytes / 4), y of z layer l go to out[y * TURB_NPHI + x]; other layers are dropped.
namespace refbake {
struct Idx3 {
    unsigned x, y, z;
};
thread_local Idx3 blockIdx, threadIdx, blockDim;
struct Layer {
    float* out;
    int l;
};
inline void surf3Dwrite(float v, cudaSurfaceObject_t s, int xbytes, int y, int z) {
    Layer* L = reinterpret_cast<Layer*>(s);
    if (z == L->l) L->out[(size_t)y * 512 + xbytes / 4] = v;
}
#include "bake_kernel.inc"
}  // namespace refbake

extern "C" {
// Layer l of the baked slice with time offset delta (render.cu:680: turb_d0 + k * turb_dd), through
// the reference's launch shape (16 x 16 blocks, render.cu:679-680): out[j * 512 + i], 192 x 512.
void ref_bake_turb_layer(const void* scene, const void* frame, float delta, int l, float* out) {
    using namespace refbake;
    std::memcpy(&c_S, scene, sizeof(SceneGPU));
    std::memcpy(&c_F, frame, sizeof(FrameGPU));
    static_assert(TURB_NPHI == 512, "layer row length");
    Layer L = {out, l};
    blockDim = {16u, 16u, 1u};
    for (unsigned by = 0; by < (TURB_NLR + 15) / 16; ++by)
        for (unsigned bx = 0; bx < (TURB_NPHI + 15) / 16; ++bx)
            for (unsigned ty = 0; ty < 16; ++ty)
                for (unsigned tx = 0; tx < 16; ++tx) {
                    blockIdx = {bx, by, (unsigned)l};
                    threadIdx = {tx, ty, 0u};
                    k_bake_turb(reinterpret_cast<cudaSurfaceObject_t>(&L), delta);
                }
}
}
