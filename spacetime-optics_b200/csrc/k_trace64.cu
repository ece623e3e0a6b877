// k_trace64.cu -- plain FP64 tracer: the drop-in path, bit-reproducible against the CPU oracle.
//
// Reference: trace_ray (blackholes/src/trace.cuh:62-165) run per sample by k_pass1 / k_pass2
// (blackholes/src/render.cu:89-128, 196-224), which give one CUDA thread one pixel for all its
// samples.  Step counts differ by 100x between neighbouring pixels near the critical curve, so a
// fixed thread-to-pixel map leaves most lanes of a warp idle behind the slowest ray.
//
// Here the kernel is persistent: a grid sized to fill the SMs once, each lane owning one ray (or one
// pixel and its samples) at a time.  A lane whose ray retires takes the next one from a global
// queue head; lanes needing work are found with a warp vote (__ballot_sync) and served by a single
// warp-aggregated atomicAdd.  One loop iteration is one DP5(4) attempt for every active lane, so
// lanes stay converged through the stepper and diverge only in the short accept / emission code.
// The loop ends when the queue is empty and every lane has retired; each ray is bounded by
// max_steps attempts, so there is no unbounded wait anywhere.
//
// The torus turbulence (a 512-mode Fourier sum per flow step) is evaluated cooperatively: the
// iteration is split around it, every lane that needs a sum has its modes spread over the 32 lanes
// of the warp, and a shuffle reduction returns it.  The geometry and the rest of the emission are
// per lane.  EMIT32 evaluates that sum with FP32 SFU cosines (the geometry stays FP64): used where
// the geometry must be FP64 (critical band, photon-ring batches) but the emission needs no more
// than FP32.
//
// Large frames, batches and ray lists take the emission out of the tracer altogether (DEFER): a
// recording pass integrates the geodesics and records each flow step that can emit;
// k_turb64_records / k_turb32_rec64 sum the turbulence at the records, k_emit64_records evaluates
// flow_step at each, and k_transfer64 applies them in each sample's order.  Every one of those
// kernels runs with all its lanes on the same kind of work, where inside the tracer the emission
// ran on the lanes that happened to take a flow step.
//
// Compiled with -fmad=false: every fusion is an explicit fma() (so_kerr.cuh), matching the oracle.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "so_emission.cuh"
#include "so_launch.h"

namespace so {

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct Ray64 {
    RayC c;
    double y[6], k1[6];
    double h, trans, psi;
    double pp0, pp1, pp2;
    float acc[4];
    int ncross, nacc, natt, it, nflow;
};

__device__ __forceinline__ void pixel_point(const TraceLaunch& L, const so_frame& F, long long q, int s, double* x,
                                            double* yv) {  // s: absolute sample index
    sample_point(L.W, L.H, L.jitter, F, q, s, x, yv);
}

// Where a job of the launch lands: its frame, pixel, first sample and number of samples.
struct JobPlace {
    long long pix;
    int fidx, sbase, jobs_n;
};
__device__ __forceinline__ JobPlace job_place(const TraceLaunch& L, long long job) {
    JobPlace q;
    q.pix = 0;
    q.fidx = 0;
    q.sbase = 0;
    q.jobs_n = 1;
    if (L.kind == RAYS_LIST) {
        q.fidx = L.list_frames > 0 ? (int)(job % L.list_frames) : 0;
    } else if (L.kind == RAYS_SAMPLES) {
        const long long sid = (long long)__ldg(L.list + job);
        q.pix = sid / L.spp;
        q.sbase = (int)(sid % L.spp);
    } else if (L.kind == RAYS_PIXELS) {
        const long long npix = (long long)L.W * L.H;
        if (L.interleave && L.nframes > 1) {
            // consecutive tiles of `tile` pixels cycle through the frames: cheap and expensive frames
            // (different spins, zooms) mix in every warp instead of queueing up (the host keeps tile
            // a divisor of W * H)
            const long long T = L.tile > 1 ? L.tile : 1;
            const long long t = job / T;
            q.fidx = (int)(t % L.nframes);
            q.pix = (t / L.nframes) * T + job % T;
        } else {
            q.fidx = (int)(job / npix);
            q.pix = job % npix;
        }
        q.sbase = L.sample0;
        q.jobs_n = L.spp;
    } else {
        // upper bound of job in the exclusive scan: the pixel owning chunk `job`
        long long lo = 0, hi = (long long)L.W * L.H;
        while (lo < hi) {
            long long mid = (lo + hi) >> 1;
            if ((long long)__ldg(L.offsets + mid) <= job) lo = mid + 1;
            else hi = mid;
        }
        q.pix = lo - 1;
        q.sbase = L.sample0 + (int)(job - (long long)__ldg(L.offsets + q.pix)) * L.chunk;
        q.jobs_n = L.chunk;
    }
    return q;
}

template <int VAR>
__device__ __forceinline__ void ray_init(Ray64& R, const so_scene& S, const so_frame& F, double x, double yv) {
    so_vec3 d = view_dir(F, x, yv);
    camera_photon(S.a, F.kp, F.ph, F.t, d, F.beta, R.c, R.y);
    rhs(R.c, R.y, R.k1);
    R.h = initial_step(R.y);
    R.trans = 1.0;
    R.psi = 0.0;
    R.ncross = R.nacc = R.natt = R.it = R.nflow = 0;
    R.acc[0] = R.acc[1] = R.acc[2] = R.acc[3] = 0.f;
    if (VAR == VAR_RADIO) {
        double sp = sqrt(fmax(fma(-R.y[2], R.y[2], 1.0), 0.0));
        double s4, c4;
        sincos(R.y[4], &s4, &c4);
        R.pp0 = sp * c4;
        R.pp1 = sp * s4;
        R.pp2 = R.y[2];
    }
}

enum Stage : int { ST_REJECTED = 0, ST_ACCEPTED = 1, ST_DONE = 2 };

// A ray list's per-ray outputs but the intensity (trace_ray's results, trace.cuh:57-61, 149-163):
// fate, crossings (saturated at 127), escape direction of an escaped ray, step counts, and the first
// three crossings' radius and redshift (cr, cg: 0 past the ray's crossings).
__device__ __forceinline__ void list_out(const so_rays_out& o, long long job, int fate, int ncross, double th,
                                         double ph, int nacc, int natt, const double* cr, const double* cg) {
    if (o.fate) o.fate[job] = (int8_t)fate;
    if (o.ncross) o.ncross[job] = (int8_t)(ncross > 127 ? 127 : ncross);
    if (o.theta) o.theta[job] = fate == 1 ? th : 0.0;
    if (o.phi) o.phi[job] = fate == 1 ? ph : 0.0;
    if (o.n_accepted) o.n_accepted[job] = nacc;
    if (o.n_attempts) o.n_attempts[job] = natt;
    if (o.cross_r) {
        for (int c = 0; c < 3; ++c) {
            o.cross_r[3 * job + c] = cr[c];
            o.cross_g[3 * job + c] = cg[c];
        }
    }
}

// First half of one loop iteration of trace_ray (trace.cuh:81-129): step cap, DP5(4) attempt,
// controller on rejection, swept angle, equatorial crossing (with the disk).  On acceptance the new
// state is in yn / k7 and the ray continues in ray_commit.  Without `emit` (the recording pass of the
// deferred turbulence) the disk is not shaded, so no ray ends on its opacity.
template <int VAR>
__device__ __forceinline__ int ray_attempt(Ray64& R, const so_scene& S, bool emit, double* yn, double* k7,
                                           double* hc_out, double* err_out, int* fate, double* cross_r,
                                           double* cross_g) {
    if (R.it >= S.max_steps) {
        *fate = 0;
        return ST_DONE;
    }
    ++R.it;
    double hc = R.h;
    if (VAR == VAR_RADIO && S.flow_on && R.y[0] < S.r_flow_max) {
        double s = sqrt(fmax(fma(-R.y[2], R.y[2], 1.0), 0.0));
        double cap = S.step_frac * fmin(R.y[0] / (fabs(R.y[1]) + 1e-30), fmax(s, 0.05) / (fabs(R.y[3]) + 1e-30));
        hc = fmin(hc, cap);
    } else if (VAR != VAR_VACUUM && S.disk_on) {
        hc = fmin(hc, 0.3 / (fabs(R.y[3]) + 1e-30));
    }
    ++R.natt;
    double err = dp54(R.c, R.y, R.k1, hc, S.tol, yn, k7);
    *hc_out = hc;
    *err_out = err;
    if (!(err <= 1.0)) {
        R.h = reject_step(hc, err);
        return ST_REJECTED;
    }
    ++R.nacc;
    if (VAR == VAR_RADIO) {
        double sn = sqrt(fmax(fma(-yn[2], yn[2], 1.0), 0.0));
        double s4, c4;
        sincos(yn[4], &s4, &c4);
        double pn0 = sn * c4, pn1 = sn * s4, pn2 = yn[2];
        double cx = fma(R.pp1, pn2, -(R.pp2 * pn1));
        double cy = fma(R.pp2, pn0, -(R.pp0 * pn2));
        double cz = fma(R.pp0, pn1, -(R.pp1 * pn0));
        double cc = fma(cz, cz, fma(cy, cy, cx * cx));
        double dd = fma(R.pp2, pn2, fma(R.pp1, pn1, R.pp0 * pn0));
        R.psi += atan2(sqrt(cc), dd);
        R.pp0 = pn0;
        R.pp1 = pn1;
        R.pp2 = pn2;
    }
    if ((R.y[2] > 0.0) != (yn[2] > 0.0)) {
        ++R.ncross;
        const bool rec = cross_r != nullptr && R.ncross <= 3;
        const bool disk = VAR != VAR_VACUUM && S.disk_on && emit;
        if (disk || rec) {
            double lo = 0.0, hi = 1.0, u0 = R.y[2], u1 = yn[2], m0 = R.y[3] * hc, m1 = yn[3] * hc;
            for (int b = 0; b < 40; ++b) {
                double mid = 0.5 * (lo + hi);
                double um = hermite(u0, u1, m0, m1, mid);
                if ((um > 0.0) == (u0 > 0.0)) lo = mid;
                else hi = mid;
            }
            double sc = 0.5 * (lo + hi);
            double rc = hermite(R.y[0], yn[0], R.y[1] * hc, yn[1] * hc, sc);
            if (rec) {
                cross_r[R.ncross - 1] = rc;
                cross_g[R.ncross - 1] = crossing_g(S, rc, R.c.lam, R.c.E);
            }
            if (disk) {
                double pc = hermite(R.y[4], yn[4], R.k1[4] * hc, k7[4] * hc, sc);
                double tc = hermite(R.y[5], yn[5], R.k1[5] * hc, k7[5] * hc, sc);
                float cs[4];
                disk_shade(S, rc, pc, tc, R.c.lam, R.c.eta, R.c.E, cs);
                if (cs[3] > 0.f) {
                    float tf = (float)R.trans;
                    R.acc[0] += tf * cs[0];
                    R.acc[1] += tf * cs[1];
                    R.acc[2] += tf * cs[2];
                    R.acc[3] += tf * cs[1] * (float)(R.ncross - 1);
                    R.trans *= 1.0 - cs[3];
                    if (R.trans < 1e-4) {
                        *fate = -1;
                        return ST_DONE;
                    }
                }
            }
        }
    }
    return ST_ACCEPTED;
}

// Second half (trace.cuh:130-163): hot-flow transfer with the turbulence sum delta, commit,
// projection, controller, termination.  Returns 1 when the ray is finished.  Without `emit` only the
// geometry advances (the ray's transmittance stays 1, so it ends only by capture, escape or the step
// limit, never earlier than with emission).
template <int VAR>
__device__ __forceinline__ int ray_commit(Ray64& R, const so_scene& S, const so_frame& F, const float* field,
                                          const TorusParams& tp, double delta, bool emit,
                                          const double* yn, const double* k7, double hc, double err, int* fate,
                                          double* th, double* ph) {
    if (VAR == VAR_RADIO && S.flow_on && yn[0] < S.r_flow_max) {
        ++R.nflow;
        if (emit) {
            double dI, dtau;
            flow_step(S, F, field, tp, delta, yn[0], yn[2], yn[4], yn[5], R.c.lam, R.c.E, hc, &dI, &dtau);
            float cc = (float)(R.trans * dI);
            int n = (int)(R.psi * (1.0 / PI));
            R.acc[0] += cc;
            if (n == 1) R.acc[1] += cc;
            else if (n == 2) R.acc[2] += cc;
            else if (n >= 3) R.acc[3] += cc;
            R.trans *= exp(-dtau);
            if (R.trans < 1e-5) {
                *fate = -1;
                return 1;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        R.y[i] = yn[i];
        R.k1[i] = k7[i];
    }
    project_radial(R.c, R.y, R.k1);
    R.h = accept_step(hc, err);
    if (R.y[0] < S.r_stop) {
        *fate = -1;
        return 1;
    }
    if (R.y[0] > S.r_escape && R.y[1] > 0.0) {
        *fate = 1;
        escape_angles(R.y, R.k1, th, ph);
        return 1;
    }
    return 0;
}

// Turbulence sums delta = sum_m amp_m cos(2 pi (k_m . X + p_m)) (k and p in turns) at four positions
// (px, py, pz)[j], split over the warp: lane l takes modes l, l + 32, l + 64, ... in that order into
// one accumulator per position, then the 32 partial sums are added by butterfly shuffles (xor 16,
// 8, 4, 2, 1), which leaves every lane with the same four sums.  The CPU oracle adds in exactly this
// order.  Every mode read from shared memory feeds four independent branch-free cosines (cos_turns),
// so the FP64 pipe has independent work while each chain waits on its previous operation.  All 32
// lanes must call this.
template <int P>
__device__ __forceinline__ void warp_sums(const ModesSmem& md, int n, const double* px, const double* py,
                                          const double* pz, double* acc) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < P; ++j) acc[j] = 0.0;
#pragma unroll 1
    for (int i = lane; i < n; i += 32) {
        const double kx = md.kx[i], ky = md.ky[i], kz = md.kz[i], p0 = md.ph[i], w = md.amp[i];
#pragma unroll
        for (int j = 0; j < P; ++j)
            acc[j] = fma(w, cos_turns(fma(kz, pz[j], fma(ky, py[j], fma(kx, px[j], p0)))), acc[j]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int j = 0; j < P; ++j) acc[j] += __shfl_xor_sync(FULL, acc[j], o);
    }
}

// The sums of the lanes in `want` (at their own X, Y, Z), four lanes' positions per warp_sums pass.
// All 32 lanes must call this; it returns at once when no lane wants a sum.
__device__ __forceinline__ double warp_turbulence64(const ModesSmem& md, int n, bool want, double X, double Y,
                                                    double Z) {
    const int lane = threadIdx.x & 31;
    unsigned m = __ballot_sync(FULL, want);
    double mine = 0.0;
    while (m) {
        int src[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            src[j] = m ? __ffs(m) - 1 : src[0];  // fewer than four left: repeat the first
            if (m) m &= m - 1;
        }
        double px[4], py[4], pz[4], acc[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            px[j] = __shfl_sync(FULL, X, src[j]);
            py[j] = __shfl_sync(FULL, Y, src[j]);
            pz[j] = __shfl_sync(FULL, Z, src[j]);
        }
        warp_sums<4>(md, n, px, py, pz, acc);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (lane == src[j]) mine = acc[j];
    }
    return mine;
}

// The mode table in shared memory as SoA doubles, wave vector and phase in turns (k / 2 pi,
// phase / 2 pi: each a correctly rounded product with 1 / 2 pi) for cos_turns.  Block-wide.
__device__ __forceinline__ ModesSmem stage_modes64(double* smem, const so_mode* modes, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const so_mode m = modes[i];
        smem[i] = m.kx * kInvTwoPi;
        smem[n + i] = m.ky * kInvTwoPi;
        smem[2 * n + i] = m.kz * kInvTwoPi;
        smem[3 * n + i] = m.phase * kInvTwoPi;
        smem[4 * n + i] = m.amp;
    }
    return ModesSmem{smem, smem + n, smem + 2 * n, smem + 3 * n, smem + 4 * n};
}

// Same with FP32 SFU cosines (modes as float4 (k, phase) and float amplitude in shared memory),
// kTurb32PerPass positions per pass: each lane then has that many independent cosines in flight
// per mode it reads.  Every position's sum is formed in the same order whatever the number of
// positions per pass (lane-strided modes, then the butterfly), so the number changes no bit.
// Measured on the photon-ring batch (64 x 512^2): 2 per pass 1.12 Mrays/s, 4 1.23, 8 1.11.
constexpr int kTurb32PerPass = 4;
__device__ __forceinline__ double warp_turbulence32(const float4* __restrict__ km, const float* __restrict__ amp, int n,
                                                    bool want, double X, double Y, double Z) {
    constexpr int P = kTurb32PerPass;
    const int lane = threadIdx.x & 31;
    unsigned m = __ballot_sync(FULL, want);
    float mine = 0.f;
    const float Xf = (float)X, Yf = (float)Y, Zf = (float)Z;
    while (m) {
        int src[P];
#pragma unroll
        for (int j = 0; j < P; ++j) {
            src[j] = m ? __ffs(m) - 1 : src[0];  // fewer than P left: repeat the first
            if (m) m &= m - 1;
        }
        float px[P], py[P], pz[P], acc[P];
#pragma unroll
        for (int j = 0; j < P; ++j) {
            px[j] = __shfl_sync(FULL, Xf, src[j]);
            py[j] = __shfl_sync(FULL, Yf, src[j]);
            pz[j] = __shfl_sync(FULL, Zf, src[j]);
            acc[j] = 0.f;
        }
        for (int i = lane; i < n; i += 32) {
            const float4 k = km[i];
            const float w = amp[i];
#pragma unroll
            for (int j = 0; j < P; ++j)
                acc[j] = fmaf(w, __cosf(fmaf(k.z, pz[j], fmaf(k.y, py[j], fmaf(k.x, px[j], k.w)))), acc[j]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int j = 0; j < P; ++j) acc[j] += __shfl_xor_sync(FULL, acc[j], o);
        }
#pragma unroll
        for (int j = 0; j < P; ++j)
            if (lane == src[j]) mine = acc[j];
    }
    return (double)mine;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    return v;
}

}  // namespace

// Register budget: three 128-thread CTAs per SM (at most 170 registers).  Measured on the B200
// against the compiler's free choice (194 registers, two CTAs): the plain FP64 synchrotron frame
// runs 1.29x faster with a few spilled registers and 50 % more warps.
// DEFER (deferred FP64 passes, radio only): 0 = emission in the tracer, 1 = recording pass (geometry
// only: no emission code), 2 = replay pass, 3 = recording pass of a ray list (also records each
// step's crossings and writes the rays' outputs without emission).  Both passes run four CTAs per
// SM (128 registers): measured on the 1024^2 synchrotron frame, the replay pass takes 178 ms there against 205 ms at
// three CTAs (168 registers, fewer spills); the recording pass 78 ms, against 84 ms at five CTAs
// (96 registers) and 88 ms at six (80), whose spills cost more than the warps gain (the reference
// flow frame: 80, 89 and 100 ms).
template <int VAR, bool EMIT32, int DEFER>
__global__ void __launch_bounds__(128, DEFER >= 1 ? 4 : 3) k_trace64(const TraceLaunch L) {
    extern __shared__ double smem[];
    constexpr int defer = (VAR == VAR_RADIO && !EMIT32) ? (DEFER == 3 ? 1 : DEFER) : 0;
    constexpr bool emit = defer != 1;
    constexpr bool list_rec = defer == 1 && DEFER == 3;  // the recording pass of a ray list
    // the replay pass behind the deferred emission runs only when the recording pass left samples
    // without records (the same value for every thread: the whole grid returns)
    if (defer == 2 && L.replay_if_short && *(volatile unsigned long long*)&L.rec64_ctl[1] == 0ull) return;
    TorusParams tp;
    tp.on = VAR == VAR_RADIO && L.torus;
    tp.n_modes = tp.on ? L.n_modes : 0;
    tp.ne_index = L.ne_index;
    tp.te_index = L.te_index;
    tp.h_sph = L.h_sph;
    tp.theta_e0 = L.theta_e0;
    tp.half_var = L.half_var;
    ModesSmem md = {smem, smem, smem, smem, smem};
    float4* km = reinterpret_cast<float4*>(smem);
    float* kamp = reinterpret_cast<float*>(km + tp.n_modes);
    // The recording pass of the deferred turbulence sums nothing; the others stage the mode table
    // once per CTA and every lane then reads the modes of its share
    if (tp.n_modes > 0 && defer != 1) {
        if (EMIT32) {
            for (int i = threadIdx.x; i < tp.n_modes; i += blockDim.x) {
                so_mode m = L.modes[i];
                double p = m.phase - 2.0 * PI * floor(m.phase / (2.0 * PI) + 0.5);
                km[i] = make_float4((float)m.kx, (float)m.ky, (float)m.kz, (float)p);
                kamp[i] = (float)m.amp;
            }
        } else {
            md = stage_modes64(smem, L.modes, tp.n_modes);
        }
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const long long total = L.nrays_dev ? (long long)*L.nrays_dev : L.nrays;
    // Short lists (re-trace lists, small ray lists) leave most lanes of the grid without a ray; then
    // only every stride-th lane takes rays, so the rays spread over more warps and each warp's
    // cooperative turbulence sums serve fewer lanes.  The same for every lane of the grid.
    int stride = 1;
    {
        const long long lanes = (long long)gridDim.x * blockDim.x;
        while (stride < 32 && total > 0 && (long long)(stride * 2) * total <= lanes) stride *= 2;
    }
    bool active = false, exhausted = false;
    Ray64 R;
    float pa[4] = {0.f, 0.f, 0.f, 0.f};
    float ys = 0.f, yq = 0.f;
    double cr[3], cg[3];
    unsigned long long n_att = 0, n_acc = 0, n_lim = 0, n_flow = 0, n_rec = 0;
    const so_scene* S = nullptr;
    const so_frame* F = nullptr;
    const bool radio_lum = VAR == VAR_RADIO;  // sample_lum, render.cu:87
    const bool rec = L.kind == RAYS_LIST && L.record_cross;
    // deferred FP64 turbulence: the lane's place in its sample's record chain (segment, slots used in
    // it, first segment, records so far) and whether the sample's sums are in place (pass 1: the pool
    // ran out; pass 2: the sample's records are incomplete)
    int rseg = -1, rcnt = REC_SEG, rhead = -1, rtot = 0;
    bool rinline = false;
    long long job = 0, pix = 0;
    int sample = 0, fidx = 0, sbase = 0, jobs_n = 1;
    // Each sample of a job has its own chain, head at job_head64[job * jobs_n + s]: the replay pass can
    // end a sample on its opacity before the recording pass did, so the chains must not run on.
    auto chain_start = [&](int s) {
        if (defer == 1) {
            rseg = rhead = -1;
            rcnt = REC_SEG;  // the first record opens a segment
            rtot = 0;
            rinline = false;
        } else {
            rhead = L.job_head64[(job - L.job0) * jobs_n + s];
            rseg = rhead;
            rcnt = 0;
            rinline = rhead == -2;
        }
    };

    // Queue grabs: a lane takes `qchunk` consecutive jobs per grab (one atomic per warp for all its
    // grabbing lanes) and works through them before grabbing again.
    const int qchunk = L.queue_chunk > 1 ? L.queue_chunk : 1;
    int chunk_left = 0;
    for (;;) {
        const bool need = !active && !exhausted && (lane & (stride - 1)) == 0;
        const bool grab = need && chunk_left == 0;
        const unsigned m = __ballot_sync(FULL, grab);
        unsigned long long j = (unsigned long long)(job - L.job0) + 1;  // the next job of the lane's grab
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&L.counters->next, (unsigned long long)qchunk * __popc(m));
            base = __shfl_sync(FULL, base, leader);
            if (grab) {
                j = base + (unsigned long long)qchunk * __popc(m & ((1u << lane) - 1u));
                chunk_left = qchunk;
            }
        }
        if (need) {
            --chunk_left;
            {
                if (j >= (unsigned long long)total) {
                    exhausted = true;
                } else {
                    job = L.job0 + (long long)j;
                    active = true;
                    sample = 0;
                    const JobPlace q = job_place(L, job);
                    fidx = q.fidx;
                    pix = q.pix;
                    sbase = q.sbase;
                    jobs_n = q.jobs_n;
                    double x, yv;
                    if (L.kind == RAYS_LIST) {
                        x = L.x[job];
                        yv = L.y[job];
                    } else {
                        pixel_point(L, L.frames[fidx], pix, sbase, &x, &yv);
                    }
                    S = &L.scenes[L.frame_scene[fidx]];
                    F = &L.frames[fidx];
                    if (defer) chain_start(0);
                    pa[0] = pa[1] = pa[2] = pa[3] = 0.f;
                    ys = yq = 0.f;
                    cr[0] = cr[1] = cr[2] = 0.0;
                    cg[0] = cg[1] = cg[2] = 0.0;
                    ray_init<VAR>(R, *S, *F, x, yv);
                }
            }
        }
        if (__all_sync(FULL, !active)) break;
        // ---- first half: the attempt (active lanes) ------------------------------------------
        int fate = 0, stage = ST_REJECTED;
        double yn[6], k7[6], hc = 0.0, err = 0.0;
        bool want = false;
        double TX = 0.0, TY = 0.0, TZ = 0.0;  // the sum's position (recording / replay pass: TX = azimuth)
        if (active) {
            stage = ray_attempt<VAR>(R, *S, emit, yn, k7, &hc, &err, &fate, rec ? cr : nullptr, cg);
            if (VAR == VAR_RADIO && stage == ST_ACCEPTED && S->flow_on && yn[0] < S->r_flow_max) {
                if (tp.n_modes > 0) {
                    if (defer == 1 || (defer == 2 && !rinline))
                        want = torus_phase(*S, tp, F->r, yn[0], yn[2], yn[4], yn[5], &TX);
                    else
                        want = torus_position(*S, tp, F->r, yn[0], yn[2], yn[4], yn[5], &TX, &TY, &TZ);
                } else if (defer == 1) {
                    // no turbulence sums: the torus without modes or the reference flow model
                    want = tp.on ? torus_wants(*S, tp, yn[0], yn[2]) : flow_wants(*S, yn[0], yn[2]);
                }
            }
        }
        // ---- all lanes: turbulence sums --------------------------------------------------------
        double delta = 0.0;
        if (VAR == VAR_RADIO && defer == 1) {
            {
                // recording pass: append the step (r, u, azimuth or phi, h, tag[, t]) to the sample's
                // chain; a lane whose segment is full closes it and takes the next one (one atomic per
                // warp); a sample the pool cannot hold is left to the replay pass
                const bool need_seg = want && !rinline && rcnt == REC_SEG;
                const unsigned ms = __ballot_sync(FULL, need_seg);
                if (ms) {
                    const int leader = __ffs(ms) - 1;
                    unsigned long long base = 0;
                    if (lane == leader) base = atomicAdd(&L.rec64_ctl[0], (unsigned long long)__popc(ms));
                    base = __shfl_sync(FULL, base, leader);
                    if (need_seg) {
                        const unsigned long long idx = base + __popc(ms & ((1u << lane) - 1u));
                        if (rseg >= 0)
                            L.seg_meta64[rseg] =
                                make_uint2((uint32_t)((job - L.job0) * jobs_n + sample), (uint32_t)REC_SEG);
                        if (idx >= (unsigned long long)L.seg_cap64) {
                            rinline = true;
                        } else {
                            if (rseg >= 0) L.seg_next64[rseg] = (uint32_t)idx;
                            else rhead = (int)idx;
                            rseg = (int)idx;
                            rcnt = 0;
                        }
                    }
                }
                if (want && !rinline) {
                    // image-order bucket as ray_commit forms it, counts after this step
                    const int b = (int)(R.psi * (1.0 / PI));
                    const unsigned long long tag =
                        (unsigned long long)(b >= 3 ? 3 : (b < 0 ? 0 : b)) | ((unsigned long long)R.natt << 2) |
                        ((unsigned long long)R.nacc << (2 + REC64_COUNT_BITS)) |
                        ((unsigned long long)(R.nflow + 1) << (2 + 2 * REC64_COUNT_BITS));
                    double* slot = L.rec64 + (long long)L.rec64_w * ((long long)rseg * REC_SEG + rcnt);
                    slot[0] = yn[0];
                    slot[1] = yn[2];
                    slot[2] = tp.n_modes > 0 ? TX : yn[4];
                    slot[3] = hc;
                    slot[4] = __longlong_as_double((long long)tag);
                    if (tp.n_modes <= 0) slot[5] = yn[5];
                    if (list_rec) slot[L.rec64_w - 1] = (double)R.ncross;
                    ++rcnt;
                    ++rtot;
                    ++n_rec;
                }
            }
        } else if (VAR == VAR_RADIO && tp.n_modes > 0) {
            if (EMIT32) {
                delta = warp_turbulence32(km, kamp, tp.n_modes, want, TX, TY, TZ);
            } else {
                // in the tracer (defer 0), or in place for the replay pass's incomplete jobs
                delta = warp_turbulence64(md, tp.n_modes, want && (defer == 0 || rinline), TX, TY, TZ);
                if (defer == 2 && want && !rinline) {
                    if (rcnt == REC_SEG && rseg >= 0) {  // the job's next segment, in recording order
                        const uint32_t nx = L.seg_next64[rseg];
                        rseg = nx < (uint32_t)L.seg_cap64 ? (int)nx : -1;
                        rcnt = 0;
                    }
                    // both passes take the same flow steps, so the chain always holds the record;
                    // were it ever short, the sum would be NaN (visible), never a read out of bounds
                    delta = rseg >= 0 ? L.rec64[(long long)L.rec64_w * ((long long)rseg * REC_SEG + rcnt) + 2]
                                      : __longlong_as_double(-1ll);
                    ++rcnt;
                }
            }
        }
        // ---- second half: emission and commit (active lanes) ----------------------------------
        if (!active || stage == ST_REJECTED) continue;
        double th = 0.0, ph = 0.0;
        if (stage == ST_ACCEPTED &&
            !ray_commit<VAR>(R, *S, *F, L.turb_field, tp, delta, emit, yn, k7, hc, err, &fate, &th, &ph))
            continue;
        // sample finished
        if (defer == 1) {
            // recording pass: the sample's chain is closed with its end state, and the job's next
            // sample, if any, opens its own
            const long long sid = (job - L.job0) * jobs_n + sample;
            L.job_head64[sid] = rinline ? -2 : rhead;
            if (rinline) atomicAdd(&L.rec64_ctl[1], 1ull);
            else if (rseg >= 0) L.seg_meta64[rseg] = make_uint2((uint32_t)sid, (uint32_t)rcnt);
            Sample64 e;
            e.lam = R.c.lam;
            e.E = R.c.E;
            e.nrec = rtot;
            e.natt = R.natt;
            e.nacc = R.nacc;
            e.nflow = R.nflow;
            e.fate = fate;
            e.fidx = fidx;
            L.samp64[sid] = e;
            // a ray list's outputs of the ray without emission; the transfer writes its intensity and,
            // where the opacity cut ends it earlier, what the tracer reports for it there
            if (list_rec) list_out(L.out, job, fate, R.ncross, th, ph, R.nacc, R.natt, cr, cg);
            if ((L.kind == RAYS_PIXELS || L.kind == RAYS_CHUNKS) && ++sample < jobs_n) {
                double x, yv;
                pixel_point(L, *F, pix, sbase + sample, &x, &yv);
                ray_init<VAR>(R, *S, *F, x, yv);
                chain_start(sample);
                continue;
            }
            active = false;
            continue;
        }
        n_att += (unsigned long long)R.natt;
        n_acc += (unsigned long long)R.nacc;
        n_flow += (unsigned long long)R.nflow;
        if (fate == 0) ++n_lim;
        if (VAR != VAR_RADIO && fate == 1 && L.sky_uv && L.kind != RAYS_LIST) {
            // escaped in visible mode: the star map through the pixel's footprint (trace.cuh:149-161)
            const int px = (int)(pix % L.W), py = (int)(pix / L.W);
            const SkyGrad g = pixel_grad(L.sky_uv, L.W, px, py, L.sky_grad_scale);
            float xyz[3];
            sky_radiance(*S, sky_uv(*S, th, ph), g, R.c.E, xyz);
            const float tf = (float)R.trans;
            R.acc[0] += tf * xyz[0];
            R.acc[1] += tf * xyz[1];
            R.acc[2] += tf * xyz[2];
        }
        if (L.kind == RAYS_LIST) {
            list_out(L.out, job, fate, R.ncross, th, ph, R.nacc, R.natt, cr, cg);
            if (L.out.I)
                reinterpret_cast<float4*>(L.out.I)[job] = make_float4(R.acc[0], R.acc[1], R.acc[2], R.acc[3]);
            active = false;
        } else {
            pa[0] += R.acc[0];
            pa[1] += R.acc[1];
            pa[2] += R.acc[2];
            pa[3] += R.acc[3];
            const float Y = radio_lum ? R.acc[0] : R.acc[1];
            ys += Y;
            yq += Y * Y;
            if (L.kind == RAYS_SAMPLES) {
                const long long sid = pix * L.spp + sbase;
                L.sample_out[sid] = make_float4(R.acc[0], R.acc[1], R.acc[2], R.acc[3]);
                if (L.sample_fate) L.sample_fate[sid] = (int8_t)fate;
                active = false;
            } else if (++sample < jobs_n) {
                double x, yv;
                pixel_point(L, *F, pix, sbase + sample, &x, &yv);
                ray_init<VAR>(R, *S, *F, x, yv);
                if (defer) chain_start(sample);
            } else if (L.kind == RAYS_PIXELS) {
                const long long o = (long long)fidx * L.W * L.H + pix;
                reinterpret_cast<float4*>(L.accum)[o] = make_float4(pa[0], pa[1], pa[2], pa[3]);
                if (L.ystat) reinterpret_cast<float2*>(L.ystat)[o] = make_float2(ys, yq);
                active = false;
            } else {
                reinterpret_cast<float4*>(L.chunk_acc)[job] = make_float4(pa[0], pa[1], pa[2], pa[3]);
                active = false;
            }
        }
    }
    n_att = warp_sum(n_att);
    n_acc = warp_sum(n_acc);
    n_lim = warp_sum(n_lim);
    n_flow = warp_sum(n_flow);
    if (defer == 1) {
        n_rec = warp_sum(n_rec);
        if (lane == 0) atomicAdd(&L.rec64_ctl[2], n_rec);
    }
    if (lane == 0) {
        atomicAdd(&L.counters->attempts, n_att);
        atomicAdd(&L.counters->accepted, n_acc);
        atomicAdd(&L.counters->step_limited, n_lim);
        atomicAdd(&L.counters->flow_steps, n_flow);
    }
}

// Deferred FP64 turbulence: the sum at every record written by a recording pass of k_trace64, by the
// same warp_sums arithmetic as the tracer's own sums (so the emission reads exactly the value the
// tracer would have computed).  Each warp takes kTurb64PerPass consecutive slots at a time, the grid
// strides over all slots of the segments taken; lane j turns slot j's (r, u, azimuth) into its
// position and the warp shares it, and the slots past a chain's last record (the segment's count)
// are summed at the origin and left unwritten.  The whole SM runs this kernel, without the tracer's
// register load, so many more warps hide the FP64 latency of the cosine chains.
// Records per warp pass: their cosines interleave.  Measured on the 1024^2 synchrotron frame: 2 per
// pass (42 registers) 212 ms, 4 (62) 201 ms, 8 (118 registers, two 256-thread CTAs per SM) 167 ms.
constexpr int kTurb64PerPass = 8;
__global__ void __launch_bounds__(256) k_turb64_records(const TraceLaunch L) {
    extern __shared__ double smem64[];
    const int n = L.n_modes;
    const ModesSmem md = stage_modes64(smem64, L.modes, n);
    __syncthreads();
    unsigned long long used = *(volatile unsigned long long*)&L.rec64_ctl[0];
    if (used > (unsigned long long)L.seg_cap64) used = (unsigned long long)L.seg_cap64;
    const long long nslots = (long long)used * REC_SEG;
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    constexpr int P = kTurb64PerPass;
    for (long long s0 = P * warp; s0 < nslots; s0 += P * nwarps) {
        const long long mine_slot = s0 + lane;
        const bool live = lane < P && mine_slot < nslots &&
                          (int)(mine_slot % REC_SEG) < (int)L.seg_meta64[mine_slot / REC_SEG].y;
        double X = 0.0, Y = 0.0, Z = 0.0;
        double* rec = L.rec64 + (long long)L.rec64_w * (live ? mine_slot : 0);
        if (live) torus_xyz(rec[0], rec[1], rec[2], &X, &Y, &Z);
        double px[P], py[P], pz[P], acc[P];
#pragma unroll
        for (int j = 0; j < P; ++j) {
            px[j] = __shfl_sync(FULL, X, j);
            py[j] = __shfl_sync(FULL, Y, j);
            pz[j] = __shfl_sync(FULL, Z, j);
        }
        warp_sums<P>(md, n, px, py, pz, acc);
        double mine = acc[0];
#pragma unroll
        for (int j = 1; j < P; ++j)
            if (lane == j) mine = acc[j];
        if (live) rec[2] = mine;
    }
}

cudaError_t launch_turb64_records(const TraceLaunch& L, int num_sms, cudaStream_t st) {
    const size_t smem = (size_t)L.n_modes * 5 * sizeof(double);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_turb64_records, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int per_sm = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_turb64_records, 256, smem);
    if (e != cudaSuccess) return e;
    k_turb64_records<<<num_sms * (per_sm > 0 ? per_sm : 1), 256, smem, st>>>(L);
    return cudaGetLastError();
}

// The mixed form of the deferred sums (FP64 geometry, FP32 turbulence sums, as the tracer's EMIT32):
// FP32 SFU cosines at every record of a recording pass, the modes folded to FP32 in constant memory
// (the kernel parameter), kTurb32RecP positions per thread at slots c0 + t + 256 q of a block's
// chunk, each position formed in FP64 from (r, u, azimuth) as the tracer forms it and rounded to
// FP32.  The sum (in mode order) goes to the record's slot [2] as the FP64 sums do.  Twelve
// positions per mode load (80 registers): the photon-ring batch at 2.15 Mrays/s against 2.09 with
// eight (74 registers).
constexpr int kTurb32RecP = 12;
__global__ void __launch_bounds__(256) k_turb32_rec64(const TraceLaunch L, const __grid_constant__ TurbModes M) {
    unsigned long long used = *(volatile unsigned long long*)&L.rec64_ctl[0];
    if (used > (unsigned long long)L.seg_cap64) used = (unsigned long long)L.seg_cap64;
    const long long nslots = (long long)used * REC_SEG;
    const int nm = M.n;
    constexpr int P = kTurb32RecP;
    const long long chunk = 256LL * P;
    for (long long c0 = (long long)blockIdx.x * chunk; c0 < nslots; c0 += (long long)gridDim.x * chunk) {
        float x[P], y[P], z[P], acc[P];
        bool live[P];
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const long long slot = c0 + threadIdx.x + 256LL * q;
            live[q] = slot < nslots && (int)(slot % REC_SEG) < (int)L.seg_meta64[slot / REC_SEG].y;
            double X = 0.0, Y = 0.0, Z = 0.0;
            if (live[q]) {
                const double* rec = L.rec64 + (long long)L.rec64_w * slot;
                torus_xyz(rec[0], rec[1], rec[2], &X, &Y, &Z);
            }
            x[q] = (float)X;
            y[q] = (float)Y;
            z[q] = (float)Z;
            acc[q] = 0.f;
        }
#pragma unroll 2
        for (int m = 0; m < nm; ++m) {
            const float4 k = M.k[m];
            const float am = M.a[m];
#pragma unroll
            for (int q = 0; q < P; ++q)
                acc[q] = fmaf(am, __cosf(fmaf(k.z, z[q], fmaf(k.y, y[q], fmaf(k.x, x[q], k.w)))), acc[q]);
        }
#pragma unroll
        for (int q = 0; q < P; ++q)
            if (live[q]) L.rec64[(long long)L.rec64_w * (c0 + threadIdx.x + 256LL * q) + 2] = (double)acc[q];
    }
}

cudaError_t launch_turb32_rec64(const TraceLaunch& L, const TurbModes& M, int num_sms, cudaStream_t st) {
    int per_sm = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_turb32_rec64, 256, 0);
    if (e != cudaSuccess) return e;
    k_turb32_rec64<<<num_sms * (per_sm > 0 ? per_sm : 1), 256, 0, st>>>(L, M);
    return cudaGetLastError();
}

// Deferred emission: flow_step at every record (after its sum, on the torus plasma), one thread per
// slot over the slots of the segments taken (a slot past its chain's last record is skipped).
// Writes the step's emission dI over r and its transmission exp(-dtau) over u.  The torus model with
// turbulence reads the sum, and neither the azimuth nor the time of the step; without modes it takes
// the flow records' form (phi, t) and reads neither; the reference flow model reads its phi and t
// and fetches the frame's turbulence as the tracer does.  Left to the replay pass when a sample ran
// out of segments.
__global__ void __launch_bounds__(256) k_emit64_records(const TraceLaunch L) {
    if (*(volatile unsigned long long*)&L.rec64_ctl[1] != 0ull) return;
    unsigned long long used = *(volatile unsigned long long*)&L.rec64_ctl[0];
    if (used > (unsigned long long)L.seg_cap64) used = (unsigned long long)L.seg_cap64;
    const long long nslots = (long long)used * REC_SEG;
    TorusParams tp;
    tp.on = L.torus;
    tp.n_modes = tp.on ? L.n_modes : 0;
    tp.ne_index = L.ne_index;
    tp.te_index = L.te_index;
    tp.h_sph = L.h_sph;
    tp.theta_e0 = L.theta_e0;
    tp.half_var = L.half_var;
    for (long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x; slot < nslots;
         slot += (long long)gridDim.x * blockDim.x) {
        const uint2 m = L.seg_meta64[slot / REC_SEG];
        if ((int)(slot % REC_SEG) >= (int)m.y) continue;
        const Sample64& smp = L.samp64[m.x];
        const int fidx = smp.fidx;
        double* rec = L.rec64 + (long long)L.rec64_w * slot;
        double dI, dtau;
        if (tp.n_modes > 0)
            flow_step(L.scenes[L.frame_scene[fidx]], L.frames[fidx], nullptr, tp, rec[2], rec[0], rec[1], 0.0, 0.0,
                      smp.lam, smp.E, rec[3], &dI, &dtau);
        else  // the reference flow model, or the torus without turbulence (flow_step's tp.on branch)
            flow_step(L.scenes[L.frame_scene[fidx]], L.frames[fidx], L.turb_field, tp, 0.0, rec[0], rec[1], rec[2],
                      rec[5], smp.lam, smp.E, rec[3], &dI, &dtau);
        rec[0] = dI;
        rec[1] = exp(-dtau);
    }
}

cudaError_t launch_emit64_records(const TraceLaunch& L, int num_sms, cudaStream_t st) {
    int per_sm = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_emit64_records, 256, 0);
    if (e != cudaSuccess) return e;
    k_emit64_records<<<num_sms * (per_sm > 0 ? per_sm : 1), 256, 0, st>>>(L);
    return cudaGetLastError();
}

// Deferred emission, ordered transfer: one thread per job walks each sample's chain in recording
// order with ray_commit's arithmetic (intensity into the image-order bucket, transmission, the
// 1e-5 opacity cut, after which the counts of the cut step stand), then writes the job's outputs
// and counts as the tracer does (a ray list's cut ray: also its crossings at the cut step).  Flow
// steps without a record emit nothing and transmit 1, so skipping them changes no bit.  Left to the
// replay pass when a sample ran out of segments.
__global__ void __launch_bounds__(128) k_transfer64(const TraceLaunch L) {
    const bool skip = *(volatile unsigned long long*)&L.rec64_ctl[1] != 0ull;
    const unsigned long long cmask = (1ull << REC64_COUNT_BITS) - 1ull;
    unsigned long long n_att = 0, n_acc = 0, n_lim = 0, n_flow = 0;
    const long long total = skip ? 0 : L.nrays;
    for (long long jrel = (long long)blockIdx.x * blockDim.x + threadIdx.x; jrel < total;
         jrel += (long long)gridDim.x * blockDim.x) {
        const long long job = L.job0 + jrel;
        const JobPlace q = job_place(L, job);
        float pa[4] = {0.f, 0.f, 0.f, 0.f};
        float ys = 0.f, yq = 0.f;
        for (int s = 0; s < q.jobs_n; ++s) {
            const long long sid = jrel * q.jobs_n + s;
            const Sample64 e = L.samp64[sid];
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            double trans = 1.0;
            int fate = e.fate, natt = e.natt, nacc = e.nacc, nflow = e.nflow, ncut = -1;
            long long seg = L.job_head64[sid];
            for (int i = 0; i < e.nrec; ++i) {
                const int k = i % REC_SEG;
                if (k == 0 && i > 0) seg = (long long)L.seg_next64[seg];
                if (seg < 0 || seg >= L.seg_cap64) {  // never with a complete chain; visible, not a stray read
                    acc[0] = __int_as_float(0x7fc00000);
                    break;
                }
                const double* rec = L.rec64 + (long long)L.rec64_w * (seg * REC_SEG + k);
                const double dI = rec[0], ex = rec[1];
                const unsigned long long tag = (unsigned long long)__double_as_longlong(rec[4]);
                const float cc = (float)(trans * dI);
                const int b = (int)(tag & 3ull);
                acc[0] += cc;
                if (b == 1) acc[1] += cc;
                else if (b == 2) acc[2] += cc;
                else if (b == 3) acc[3] += cc;
                trans *= ex;
                if (trans < 1e-5) {
                    fate = -1;
                    natt = (int)((tag >> 2) & cmask);
                    nacc = (int)((tag >> (2 + REC64_COUNT_BITS)) & cmask);
                    nflow = (int)((tag >> (2 + 2 * REC64_COUNT_BITS)) & cmask);
                    if (L.kind == RAYS_LIST) ncut = (int)rec[L.rec64_w - 1];
                    break;
                }
            }
            n_att += (unsigned long long)natt;
            n_acc += (unsigned long long)nacc;
            n_flow += (unsigned long long)nflow;
            if (fate == 0) ++n_lim;
            pa[0] += acc[0];
            pa[1] += acc[1];
            pa[2] += acc[2];
            pa[3] += acc[3];
            const float Y = acc[0];  // radio: sample_lum is the total intensity
            ys += Y;
            yq += Y * Y;
            if (L.kind == RAYS_SAMPLES) {
                const long long o = q.pix * L.spp + q.sbase;
                L.sample_out[o] = make_float4(acc[0], acc[1], acc[2], acc[3]);
                if (L.sample_fate) L.sample_fate[o] = (int8_t)fate;
            } else if (L.kind == RAYS_LIST) {
                // the recording pass wrote the uncut ray's outputs; a ray cut on its opacity reports
                // the tracer's values at the cut: captured, no escape direction, the counts and
                // crossings of that step (later crossings were never reached)
                const so_rays_out& o = L.out;
                if (o.I) reinterpret_cast<float4*>(o.I)[job] = make_float4(acc[0], acc[1], acc[2], acc[3]);
                if (ncut >= 0) {
                    double cr[3] = {0.0, 0.0, 0.0}, cg[3] = {0.0, 0.0, 0.0};
                    if (o.cross_r) {
                        for (int c = 0; c < 3 && c < ncut; ++c) {
                            cr[c] = o.cross_r[3 * job + c];
                            cg[c] = o.cross_g[3 * job + c];
                        }
                    }
                    list_out(o, job, -1, ncut, 0.0, 0.0, nacc, natt, cr, cg);
                }
            }
        }
        if (L.kind == RAYS_PIXELS) {
            const long long o = (long long)q.fidx * L.W * L.H + q.pix;
            reinterpret_cast<float4*>(L.accum)[o] = make_float4(pa[0], pa[1], pa[2], pa[3]);
            if (L.ystat) reinterpret_cast<float2*>(L.ystat)[o] = make_float2(ys, yq);
        } else if (L.kind == RAYS_CHUNKS) {
            reinterpret_cast<float4*>(L.chunk_acc)[job] = make_float4(pa[0], pa[1], pa[2], pa[3]);
        }
    }
    n_att = warp_sum(n_att);
    n_acc = warp_sum(n_acc);
    n_lim = warp_sum(n_lim);
    n_flow = warp_sum(n_flow);
    if ((threadIdx.x & 31) == 0 && n_att + n_acc + n_lim + n_flow > 0) {
        atomicAdd(&L.counters->attempts, n_att);
        atomicAdd(&L.counters->accepted, n_acc);
        atomicAdd(&L.counters->step_limited, n_lim);
        atomicAdd(&L.counters->flow_steps, n_flow);
    }
}

cudaError_t launch_transfer64(const TraceLaunch& L, int num_sms, cudaStream_t st) {
    const long long blocks = (L.nrays + 127) / 128;
    const long long cap = (long long)num_sms * 16;
    k_transfer64<<<(int)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap), 128, 0, st>>>(L);
    return cudaGetLastError();
}

// Host launcher: grid = SMs x resident CTAs per SM (persistent; capped by L.ctas_per_sm), dynamic
// shared memory for the mode table.  Returns the CUDA error of the launch.
// Bake of the flow turbulence for the frame in d_frame (k_bake_turb, render.cu:449-460): slice k
// holds exp(a n - a^2 / 2) of the sheared noise n at the retarded time t_ref(r) + delta_k, on cell
// centres phi = 2 pi (i + 1/2) / 512, ln R uniform over [lr0, lr1] (192 cells), z / R uniform over
// [-zmax, zmax] (48 cells).  One thread per cell, phi fastest (coalesced stores).
__device__ __forceinline__ float bake_texel(const so_scene& S, const so_frame& F, const TurbBake& b, int i, int j,
                                             int l, int k) {
    const double phi = (i + 0.5) / TURB_NPHI * 2.0 * PI;
    const double R = exp(S.turb_lr0 + (j + 0.5) / TURB_NLR * (S.turb_lr1 - S.turb_lr0));
    const double z = (-1.0 + 2.0 * (l + 0.5) / TURB_NZ) * S.turb_zmax * R;
    const double r = sqrt(fma(R, R, z * z));
    const double t = (F.t - (F.r - r + 2.0 * log(F.r / r))) + b.delta[k];
    const float n = sheared_noise(S, R, phi, z, t, S.flow_turb_scale, S.flow_tcorr, S.seed ^ 0x51f15eedu);
    const float a = S.flow_turb_amp;
    return __expf(a * n - 0.5f * a * a);
}

__global__ void __launch_bounds__(256) k_bake_turb(const so_scene* __restrict__ Sp, const so_frame* __restrict__ Fp,
                                                   const TurbBake b, float* __restrict__ field) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = blockIdx.z % TURB_NZ, k = blockIdx.z / TURB_NZ;
    if (i >= TURB_NPHI || j >= TURB_NLR) return;
    field[(((size_t)k * TURB_NZ + l) * TURB_NLR + j) * TURB_NPHI + i] = bake_texel(*Sp, *Fp, b, i, j, l, k);
}

// The same texels into slice k's 3-D array through its surface (x = phi, y = ln R, z = z / R), for
// the texture-unit fetch (render.cu:449-460 writes its slices the same way).
__global__ void __launch_bounds__(256) k_bake_turb_surf(const so_scene* __restrict__ Sp,
                                                        const so_frame* __restrict__ Fp, const TurbBake b,
                                                        const SurfaceSet surf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = blockIdx.z % TURB_NZ, k = blockIdx.z / TURB_NZ;
    if (i >= TURB_NPHI || j >= TURB_NLR) return;
    surf3Dwrite(bake_texel(*Sp, *Fp, b, i, j, l, k), surf.s[k], i * (int)sizeof(float), j, l);
}

// Pixel corners (k_corners, render.cu:40-52): corner (x, y) of a W x H frame at tangent-plane point
// ((x - W/2) pix, (H/2 - y) pix), x in [0, W], y in [0, H].
__global__ void k_corner_points(const so_frame* __restrict__ Fp, int W, int H, double* __restrict__ xs,
                                double* __restrict__ ys) {
    const long long n = (long long)(W + 1) * (H + 1);
    const double pix = Fp->pix;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % (W + 1)), y = (int)(i / (W + 1));
        xs[i] = (x - 0.5 * W) * pix;
        ys[i] = (0.5 * H - y) * pix;
    }
}

__global__ void k_corner_uv(const so_scene* __restrict__ Sp, long long n, const int8_t* __restrict__ fate,
                            const double* __restrict__ th, const double* __restrict__ ph, float2* __restrict__ uv) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        uv[i] = fate[i] == 1 ? sky_uv(*Sp, th[i], ph[i]) : make_float2(-1.f, -1.f);
}

// One mip level of the star map (k_mip_half2, render.cu:462-475): mean of the 2 x 2 texels below
// (indices clamped to the level above), rounded to half.
__global__ void k_mip_half2(cudaSurfaceObject_t src, int sw, int sh, cudaSurfaceObject_t dst, int dw, int dh) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dw || y >= dh) return;
    float a = 0.f, b = 0.f;
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            ushort2 v;
            surf2Dread(&v, src, min(2 * x + i, sw - 1) * 4, min(2 * y + j, sh - 1));
            a += __half2float(__ushort_as_half(v.x));
            b += __half2float(__ushort_as_half(v.y));
        }
    surf2Dwrite(make_ushort2(__half_as_ushort(__float2half(0.25f * a)), __half_as_ushort(__float2half(0.25f * b))), dst,
                x * 4, y);
}

cudaError_t launch_corner_points(const so_frame* d_frame, int W, int H, double* x, double* y, cudaStream_t st) {
    k_corner_points<<<592, 256, 0, st>>>(d_frame, W, H, x, y);
    return cudaGetLastError();
}

cudaError_t launch_corner_uv(const so_scene* d_scene, long long n, const int8_t* fate, const double* th,
                             const double* ph, float2* uv, cudaStream_t st) {
    k_corner_uv<<<592, 256, 0, st>>>(d_scene, n, fate, th, ph, uv);
    return cudaGetLastError();
}

cudaError_t launch_mip_half2(cudaSurfaceObject_t src, int sw, int sh, cudaSurfaceObject_t dst, int dw, int dh,
                             cudaStream_t st) {
    k_mip_half2<<<dim3((dw + 15) / 16, (dh + 15) / 16), dim3(16, 16), 0, st>>>(src, sw, sh, dst, dw, dh);
    return cudaGetLastError();
}

cudaError_t launch_bake_turb(const so_scene* d_scene, const so_frame* d_frame, const TurbBake& b, float* field,
                             cudaStream_t st) {
    const dim3 block(32, 8), grid(TURB_NPHI / 32, TURB_NLR / 8, TURB_NZ * TURB_NT);
    k_bake_turb<<<grid, block, 0, st>>>(d_scene, d_frame, b, field);
    return cudaGetLastError();
}

cudaError_t launch_bake_turb_surf(const so_scene* d_scene, const so_frame* d_frame, const TurbBake& b,
                                  const SurfaceSet& surf, cudaStream_t st) {
    const dim3 block(32, 8), grid(TURB_NPHI / 32, TURB_NLR / 8, TURB_NZ * TURB_NT);
    k_bake_turb_surf<<<grid, block, 0, st>>>(d_scene, d_frame, b, surf);
    return cudaGetLastError();
}

cudaError_t launch_trace64(const TraceLaunch& L, int variant, int num_sms, cudaStream_t st) {
    const int tpb = 128;
    const bool torus = variant == VAR_RADIO && L.torus && L.n_modes > 0;
    const bool emit32 = torus && L.emit32;
    size_t smem = torus && !(L.defer64 == 1 && !emit32)
                      ? (size_t)L.n_modes * (emit32 ? sizeof(float4) + sizeof(float) : 5 * sizeof(double)) : 0;
    int per_sm = 1;
    auto go = [&](auto kern) -> cudaError_t {
        cudaError_t e;
        if (smem > 48 * 1024) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, tpb, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        if (L.ctas_per_sm > 0 && L.ctas_per_sm < per_sm) per_sm = L.ctas_per_sm;
        long long want = (L.nrays * 32 + tpb - 1) / tpb;  // up to a warp per ray for short lists
        long long grid = (long long)num_sms * per_sm;
        if (grid > want) grid = want;
        if (grid < 1) grid = 1;
        kern<<<(int)grid, tpb, smem, st>>>(L);
        return cudaGetLastError();
    };
    switch (variant) {
        case VAR_VACUUM: return go(k_trace64<VAR_VACUUM, false, 0>);
        case VAR_DISK: return go(k_trace64<VAR_DISK, false, 0>);
        default:
            if (emit32) return go(k_trace64<VAR_RADIO, true, 0>);
            if (L.defer64 == 1)
                return L.kind == RAYS_LIST ? go(k_trace64<VAR_RADIO, false, 3>) : go(k_trace64<VAR_RADIO, false, 1>);
            if (L.defer64 == 2) return go(k_trace64<VAR_RADIO, false, 2>);
            return go(k_trace64<VAR_RADIO, false, 0>);
    }
}

}  // namespace so
