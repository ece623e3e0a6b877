// Surrogate training set and surrogate thin-disk frame: kernel parameter blocks and launchers
// (k_mlp.cu), and the renderer services the host side of the surrogate uses (so_renderer.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/so_tracer.h"

namespace so {
namespace sur {

// Routing of the pixel centres of one frame (k_route).
struct Route {
    const so_frame* F;  // device
    int W, H;
    const float* band;  // analytic critical-curve radius on band_n image angles (device)
    int band_n;
    double band_m, xy_max;
    uint32_t audit_thr, audit_key;  // audit when pcg(pixel ^ key) < thr
    float spin, incl_deg;
    unsigned long long* counts;  // [0] surrogate, [1] band, [2] audit
    uint32_t* list_s;            // pixel of each surrogate ray
    so_sur_ray* rays_s;          // its network input
    uint32_t* list_b;            // pixels of the band
    uint32_t* list_a;            // audited pixels
    uint32_t* audit_j;           // their index in the surrogate list
};

// Audit of the surrogate against the integrator (k_audit).  acc[11]: class mismatches, direction
// error sum and count, |du| sum and count, relative radius error sum, |dg| sum, their count,
// |dY| sum, surrogate Y sum, integrator Y sum.
struct Audit {
    int na, nb;
    const uint32_t* list_a;
    const uint32_t* audit_j;
    const float* out;  // network outputs of the surrogate list
    const float4* px;  // frame shaded by the surrogate (before the integrator's pixels go in)
    const float4* I;   // integrator pixels: band rays, then audit rays
    const int8_t* fate;
    const double* theta;
    const double* phi;
    const double* cross_r;
    const double* cross_g;
    double* acc;
};

// Training rays: ray i belongs to group g = i % groups (spin spin[g], inclination incl[g] degrees,
// camera at r_cam); alpha, beta uniform in [-xy_max, xy_max] from the seed.
void launch_sample(long long n, int groups, uint32_t seed, double xy_max, const float* spin, const float* incl,
                   double r_cam, double* x, double* y, so_sur_ray* rays, cudaStream_t st);
// Targets from the integrator's records of those rays (r_stop[g]: the group's stopping radius).
void launch_targets(long long n, int groups, const double* r_stop, const int8_t* fate, const double* th,
                    const double* ph, const double* cr, const double* cg, so_sur_target* tgt, cudaStream_t st);
void launch_route(const Route& R, int num_sms, cudaStream_t st);
void launch_xy(const so_frame* F, int W, int H, const uint32_t* list_b, int nb, const uint32_t* list_a, int na, double* x,
               double* y, cudaStream_t st);
void launch_shade(const so_scene* S, const so_frame* F, int W, int H, const uint32_t* list_s, int ns, const float* out,
                  float4* px, cudaStream_t st);
void launch_audit(const Audit& A, cudaStream_t st);
void launch_scatter(const uint32_t* list_b, int nb, const uint32_t* list_a, int na, const float4* I, float4* px,
                    cudaStream_t st);

}  // namespace sur

// Spin-dependent scalars of a scene (so_shot.cpp).
void scene_set_spin(so_scene* S, double a);

// Renderer services (so_renderer.cpp).
int rend_device(so_renderer* r);
int rend_num_sms(so_renderer* r);
cudaStream_t rend_stream(so_renderer* r);
const so_scene& rend_scene(so_renderer* r);
const so_settings& rend_settings(so_renderer* r);
const so_scene* rend_scene_dev(so_renderer* r);
int rend_fail(so_renderer* r, int code, const char* msg);
// Critical-curve radius table of the renderer's spin seen from inclination th (device, cached).
int rend_band_table(so_renderer* r, double th, const float** d_band, int* n);
// Frame f into the renderer's device frame slot; returns its device address.
int rend_upload_frame(so_renderer* r, const so_frame& f, const so_frame** d_frame);
// trace_ray over n device rays (x, y) of the frame already uploaded, with the tracer variant
// `vacuum` = 1 (no emission, crossing records) or 0 (the scene's own variant), on the renderer's
// stream, or with side = 1 on its second stream (ordered after the work queued on the first so far,
// own queue head).  Does not synchronise.
int rend_trace_list(so_renderer* r, int n, const double* d_x, const double* d_y, const so_rays_out& d_out, int vacuum,
                    int side = 0);
// The same over many frames in one launch: ray i uses frame i % nframes of the device arrays
// d_frames / d_scenes (through d_frame_scene).
int rend_trace_list_frames(so_renderer* r, int n, const double* d_x, const double* d_y, const so_rays_out& d_out,
                           int vacuum, const so_scene* d_scenes, const so_frame* d_frames, const int* d_frame_scene,
                           int nframes);
// Orders the renderer's stream after everything queued on its second stream.
int rend_join_side(so_renderer* r);

}  // namespace so
