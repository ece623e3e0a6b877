// so_launch.h -- launch descriptors shared by the host renderer and the CUDA kernels.
#pragma once
#include <cstdint>

#include "../../include/so_tracer.h"

namespace so {

// What a tracer launch computes.
enum RayKind : int {
    RAYS_LIST = 0,   // explicit tangent-plane points x[i], y[i] of frame 0, one sample each
    RAYS_PIXELS = 1, // every pixel of every frame, spp samples per pixel (frames share W, H, spp)
    RAYS_CHUNKS = 2  // adaptive pass 2: job j = `chunk` more samples of the pixel owning chunk j
};

// Scene features a kernel instantiation supports (uniform over the frames of one launch).
enum Variant : int {
    VAR_VACUUM = 0,  // no emission: geometry, fate, winding order, escape direction
    VAR_RADIO = 1,   // hot-flow synchrotron transfer (reference or torus plasma)
    VAR_DISK = 2     // thin disk at equatorial crossings
};

// Device counters of one launch (zeroed before the launch).
struct Counters {
    unsigned long long next;          // ray-queue head
    unsigned long long step_limited;  // samples that hit max_steps
    unsigned long long attempts;      // DP5(4) attempts
    unsigned long long accepted;      // accepted steps
    unsigned long long fp64_rays;     // mixed precision: rays (or restarts) integrated in FP64
    unsigned long long flow_steps;    // accepted steps that evaluated the hot-flow transfer
    unsigned long long pad[2];
};

struct TraceLaunch {
    const so_scene* scenes;   // device array, indexed by frame_scene[f]
    const so_frame* frames;   // device array
    const int* frame_scene;   // device array
    int nframes;
    int kind;                 // RayKind
    int record_cross;         // RAYS_LIST: record the first 3 equatorial crossings
    long long nrays;          // RAYS_LIST: number of points; RAYS_PIXELS: W*H*nframes
    int W, H, spp;            // RAYS_PIXELS geometry (shared by the frames)
    int jitter;               // RAYS_PIXELS: 1 = R2 jitter per sample (reference), 0 = pixel centres
    int sample0;              // first sample index (pass 2 continues the sequence)
    // plasma
    int torus, n_modes;
    double ne_index, te_index, h_sph, theta_e0, half_var;
    const so_mode* modes;     // device array (n_modes)
    // inputs / outputs (device pointers)
    const double* x;
    const double* y;
    so_rays_out out;          // RAYS_LIST outputs (device pointers, NULL = skip)
    float* accum;             // RAYS_PIXELS: W*H*nframes*4 sums
    float* ystat;             // RAYS_PIXELS: W*H*nframes*2 (sum Y, sum Y^2), or NULL
    Counters* counters;
    // RAYS_CHUNKS
    const uint32_t* offsets;  // exclusive scan of chunks per pixel (W*H)
    float* chunk_acc;         // per chunk: 4 float sums
    int chunk;                // samples per chunk
    // mixed precision
    double band_m, tol32, turn_frac, drift_tol;
    const uint8_t* band_mask; // per ray: 1 = integrate in FP64 (critical band), or NULL
};

}  // namespace so
