// Ray surrogate: the element-wise and reduction kernels around the tensor-core GEMMs of k_umma.cu
// (Fourier features, loss and its gradient, bias gradients, deterministic split sums, AdamW), and
// the kernels of the training set and of the surrogate thin-disk frame (routing, shading from the
// predicted crossings, audit against the integrator).
#include <cuda_runtime.h>

#include "so_emission.cuh"
#include "so_mlp.h"
#include "so_sur.h"

namespace so {
namespace mlp {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr float TWO_PI = 6.283185307179586f;

__device__ __forceinline__ void scaled_input(const so_sur_ray& r, float* x) {
    x[0] = r.alpha * (1.f / XY_SCALE);
    x[1] = r.beta * (1.f / XY_SCALE);
    x[2] = (r.spin - A_MID) * (1.f / A_MID);
    x[3] = (r.incl_deg - I_MID) * (1.f / I_HALF);
}

// One thread per ray: X[i, j] = sin(2 pi f_j . x), X[i, 64 + j] = cos(2 pi f_j . x).
__global__ void __launch_bounds__(128) k_features(const so_sur_ray* __restrict__ rays, long off, long n, int rows,
                                                  int wrap, const float* __restrict__ freq, bf16* __restrict__ X,
                                                  bf16* __restrict__ XT, long ldxt) {
    __shared__ float f[NFREQ * 4];
    for (int i = threadIdx.x; i < NFREQ * 4; i += blockDim.x) f[i] = freq[i];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    float x[4] = {0.f, 0.f, 0.f, 0.f};
    const long src = wrap ? (off + i) % n : off + i;
    if (src < n) scaled_input(rays[src], x);
    __align__(16) bf16 sv[8], cv[8];
    for (int j0 = 0; j0 < NFREQ; j0 += 8) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float* fj = f + (j0 + q) * 4;
            const float z = TWO_PI * fmaf(fj[3], x[3], fmaf(fj[2], x[2], fmaf(fj[1], x[1], fj[0] * x[0])));
            float s, c;
            sincosf(z, &s, &c);
            sv[q] = __float2bfloat16_rn(s);
            cv[q] = __float2bfloat16_rn(c);
            if (XT) {
                XT[(long)(j0 + q) * ldxt + i] = sv[q];
                XT[(long)(NFREQ + j0 + q) * ldxt + i] = cv[q];
            }
        }
        *reinterpret_cast<uint4*>(X + (long)i * NFEAT + j0) = *reinterpret_cast<const uint4*>(sv);
        *reinterpret_cast<uint4*>(X + (long)i * NFEAT + NFREQ + j0) = *reinterpret_cast<const uint4*>(cv);
    }
}

// Loss per ray and dL/dO (mean over the rows).  Block partials of the head-bias gradient and of the
// loss terms go to part_gb / part_acc and are summed in block order by k_loss_reduce.
__global__ void __launch_bounds__(128) k_loss(const float* __restrict__ O, const so_sur_target* __restrict__ tgt,
                                              long off, long n, int rows, LossWeights w, bf16* __restrict__ dO,
                                              bf16* __restrict__ dOT, float* __restrict__ part_gb,
                                              double* __restrict__ part_acc) {
    __shared__ float s_gb[4][LDO];
    __shared__ double s_acc[4][8];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    float dl[LDO];
    double st[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < LDO; ++k) dl[k] = 0.f;
    if (i < rows) {
        const so_sur_target t = tgt[(off + i) % n];
        const float* o = O + (long)i * LDO;
        const int c = (int)t.cls;
        const float m = fmaxf(o[0], fmaxf(o[1], o[2]));
        const float e0 = expf(o[0] - m), e1 = expf(o[1] - m), e2 = expf(o[2] - m);
        const float s = e0 + e1 + e2, is = 1.f / s;
        const float oc = c == 0 ? o[0] : c == 1 ? o[1] : o[2];
        const float ce = logf(s) + m - oc;
        dl[0] = e0 * is - (c == 0 ? 1.f : 0.f);
        dl[1] = e1 * is - (c == 1 ? 1.f : 0.f);
        dl[2] = e2 * is - (c == 2 ? 1.f : 0.f);
        const int am = (o[1] > o[0] && o[1] >= o[2]) ? 1 : (o[2] > o[0] && o[2] > o[1]) ? 2 : 0;
        float ld = 0.f, lu = 0.f, lg = 0.f;
        const bool esc = c == 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float dd = o[3 + k] - t.dir[k];
            if (esc) {
                ld += dd * dd;
                dl[3 + k] = 2.f * w.dir * dd;
            }
            const float du = o[6 + k] - t.u[k];
            lu += du * du;
            dl[6 + k] = 2.f * w.u * du;
            if (t.g[k] >= 0.f) {
                const float dg = o[9 + k] - t.g[k];
                lg += dg * dg;
                dl[9 + k] = 2.f * w.g * dg;
            }
        }
        const float inv = 1.f / (float)rows;
#pragma unroll
        for (int k = 0; k < NOUT; ++k) dl[k] *= inv;
        __align__(16) bf16 h[LDO];
#pragma unroll
        for (int k = 0; k < LDO; ++k) h[k] = __float2bfloat16_rn(dl[k]);
        uint4* dst = reinterpret_cast<uint4*>(dO + (long)i * LDO);
        dst[0] = reinterpret_cast<const uint4*>(h)[0];
        dst[1] = reinterpret_cast<const uint4*>(h)[1];
#pragma unroll
        for (int k = 0; k < LDO; ++k) dOT[(long)k * rows + i] = h[k];
        st[0] = ce;
        st[1] = ld;
        st[2] = lu;
        st[3] = lg;
        st[4] = am == c ? 1.0 : 0.0;
        st[5] = ce + w.dir * ld + w.u * lu + w.g * lg;
    }
#pragma unroll
    for (int k = 0; k < LDO; ++k) {
        float v = dl[k];
        for (int sh = 16; sh > 0; sh >>= 1) v += __shfl_xor_sync(FULL, v, sh);
        if (lane == 0) s_gb[wp][k] = v;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        double v = st[k];
        for (int sh = 16; sh > 0; sh >>= 1) v += __shfl_xor_sync(FULL, v, sh);
        if (lane == 0) s_acc[wp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < LDO)
        part_gb[(long)blockIdx.x * LDO + threadIdx.x] =
            ((s_gb[0][threadIdx.x] + s_gb[1][threadIdx.x]) + s_gb[2][threadIdx.x]) + s_gb[3][threadIdx.x];
    if (threadIdx.x < 6)
        part_acc[(long)blockIdx.x * 8 + threadIdx.x] =
            ((s_acc[0][threadIdx.x] + s_acc[1][threadIdx.x]) + s_acc[2][threadIdx.x]) + s_acc[3][threadIdx.x];
}

// Sum of the block partials in a fixed order and a fixed tree (deterministic): one block, each
// output summed by 256 threads over strided partials, then a shared-memory tree.
__global__ void __launch_bounds__(256) k_loss_reduce(const float* __restrict__ part_gb,
                                                     const double* __restrict__ part_acc, int nblk,
                                                     float* __restrict__ gb, double* __restrict__ acc) {
    __shared__ double red[256];
    for (int k = 0; k < LDO + 6; ++k) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x)
            v += k < LDO ? (double)part_gb[(long)b * LDO + k] : part_acc[(long)b * 8 + (k - LDO)];
        red[threadIdx.x] = v;
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            if (k < LDO) gb[k] = (float)red[0];
            else acc[k - LDO] += red[0];
        }
        __syncthreads();
    }
}

// One block of 512 threads per row, 16-byte loads (8 values), fixed per-thread order and a fixed
// tree: deterministic.  cols is a multiple of 8 and rows are 16-byte aligned.
__global__ void __launch_bounds__(512) k_rowsum(const bf16* __restrict__ dT, int cols, float* __restrict__ gb) {
    __shared__ float s[16];
    const uint4* row = reinterpret_cast<const uint4*>(dT + (long)blockIdx.x * cols);
    float v = 0.f;
    for (int c = threadIdx.x; c < cols / 8; c += blockDim.x) {
        const uint4 q = __ldg(row + c);
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f = __bfloat1622float2(h[i]);
            v += f.x + f.y;
        }
    }
    for (int sh = 16; sh > 0; sh >>= 1) v += __shfl_xor_sync(FULL, v, sh);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += s[i];
        gb[blockIdx.x] = t;
    }
}

__global__ void k_sum_splits(const float* __restrict__ part, int splits, long count, float* __restrict__ out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < splits; ++z) s += part[(long)z * count + i];
        out[i] = s;
    }
}

__device__ __forceinline__ void store_bf16_copies(long i, float p, const Layout& L, bf16* W, bf16* WT) {
    const bf16 h = __float2bfloat16_rn(p);
    W[i] = h;
#pragma unroll
    for (int l = 0; l < NLAYER; ++l) {
        if (i >= L.w[l] && i < L.b[l]) {
            const long e = i - L.w[l];
            const int row = (int)(e / L.k[l]), col = (int)(e % L.k[l]);
            WT[L.w[l] + (long)col * L.n[l] + row] = h;
        }
    }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long n, float lr, float b1, float b2, float eps, float wd, float bc1, float bc2,
                       bf16* __restrict__ W, bf16* __restrict__ WT) {
    const Layout L = param_layout();
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = fmaf(b1, m[i], (1.f - b1) * gi);
        const float vi = fmaf(b2, v[i], (1.f - b2) * gi * gi);
        m[i] = mi;
        v[i] = vi;
        const float mh = mi / bc1, vh = vi / bc2;
        float pi = p[i];
        pi -= lr * (mh / (sqrtf(vh) + eps) + wd * pi);
        p[i] = pi;
        store_bf16_copies(i, pi, L, W, WT);
    }
}

__global__ void k_pack(const float* __restrict__ p, long n, bf16* __restrict__ W, bf16* __restrict__ WT) {
    const Layout L = param_layout();
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        store_bf16_copies(i, p[i], L, W, WT);
}

}  // namespace

void launch_features(const so_sur_ray* rays, long off, long n, int rows, int wrap, const float* freq, bf16* X,
                     bf16* XT, long ldxt, cudaStream_t st) {
    k_features<<<(rows + 127) / 128, 128, 0, st>>>(rays, off, n, rows, wrap, freq, X, XT, ldxt);
}

void launch_loss(const float* O, const so_sur_target* tgt, long off, long n, int rows, LossWeights w, bf16* dO,
                 bf16* dOT, float* part_gb, double* part_acc, float* gb, double* acc, cudaStream_t st) {
    const int nblk = (rows + 127) / 128;
    k_loss<<<nblk, 128, 0, st>>>(O, tgt, off, n, rows, w, dO, dOT, part_gb, part_acc);
    k_loss_reduce<<<1, 256, 0, st>>>(part_gb, part_acc, nblk, gb, acc);
}

void launch_rowsum(const bf16* dT, int rows, int cols, float* gb, cudaStream_t st) {
    k_rowsum<<<rows, 512, 0, st>>>(dT, cols, gb);
}

void launch_sum_splits(const float* part, int splits, long count, float* out, cudaStream_t st) {
    const int blocks = (int)((count + 255) / 256 < 1184 ? (count + 255) / 256 : 1184);
    k_sum_splits<<<blocks, 256, 0, st>>>(part, splits, count, out);
}

void launch_adam(float* p, const float* g, float* m, float* v, long n, float lr, float b1, float b2, float eps,
                 float wd, int t, bf16* W, bf16* WT, cudaStream_t st) {
    const float bc1 = 1.f - powf(b1, (float)t), bc2 = 1.f - powf(b2, (float)t);
    k_adam<<<296, 256, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, wd, bc1, bc2, W, WT);
}

void launch_pack(const float* p, long n, bf16* W, bf16* WT, cudaStream_t st) { k_pack<<<296, 256, 0, st>>>(p, n, W, WT); }

}  // namespace mlp

// ---- training set ------------------------------------------------------------------------------
namespace sur {

namespace {

using mlp::FULL;

__device__ __forceinline__ float unit_rand(uint32_t seed, uint32_t a, uint32_t b) {
    uint32_t h = pcg(seed ^ pcg(a * 0x9E3779B9u ^ pcg(b + 0x632BE5ABu)));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

__global__ void k_sample(long long n, int groups, uint32_t seed, double xy_max, const float* __restrict__ spin,
                         const float* __restrict__ incl, double r_cam, double* __restrict__ x,
                         double* __restrict__ y, so_sur_ray* __restrict__ rays) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(i % groups);
        const uint32_t j = (uint32_t)(i / groups);
        const double al = (2.0 * unit_rand(seed, (uint32_t)g, 2 * j) - 1.0) * xy_max;
        const double be = (2.0 * unit_rand(seed, (uint32_t)g, 2 * j + 1) - 1.0) * xy_max;
        x[i] = al / r_cam;
        y[i] = be / r_cam;
        so_sur_ray r;
        r.alpha = (float)al;
        r.beta = (float)be;
        r.spin = spin[g];
        r.incl_deg = incl[g];
        rays[i] = r;
    }
}

__global__ void k_targets(long long n, int groups, const double* __restrict__ r_stop, const int8_t* __restrict__ fate,
                          const double* __restrict__ th, const double* __restrict__ ph, const double* __restrict__ cr,
                          const double* __restrict__ cg, so_sur_target* __restrict__ tgt) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        so_sur_target t;
        const int f = fate[i];
        t.cls = f == SO_FATE_ESCAPED ? 0.f : f == SO_FATE_CAPTURED ? 1.f : 2.f;
        if (f == SO_FATE_ESCAPED) {
            double s, c, sp, cp;
            sincos(th[i], &s, &c);
            sincos(ph[i], &sp, &cp);
            t.dir[0] = (float)(s * cp);
            t.dir[1] = (float)(s * sp);
            t.dir[2] = (float)c;
        } else {
            t.dir[0] = t.dir[1] = t.dir[2] = 0.f;
        }
        // A crossing that does not happen lies at infinity for a ray that escapes and at the stopping
        // radius for one that is captured: the target then moves continuously as a crossing appears.
        const float u_none = f == SO_FATE_CAPTURED ? (float)(1.0 / r_stop[i % groups]) : 0.f;
        for (int k = 0; k < 3; ++k) {
            const double r = cr[3 * i + k];
            t.u[k] = r > 0.0 ? (float)(1.0 / r) : u_none;
            t.g[k] = r > 0.0 ? (float)cg[3 * i + k] : -1.f;
        }
        t.pad[0] = t.pad[1] = 0.f;
        tgt[i] = t;
    }
}

// ---- surrogate frame ---------------------------------------------------------------------------
__device__ __forceinline__ long long push_idx(unsigned long long* count, bool want) {
    const unsigned m = __ballot_sync(FULL, want);
    if (!m) return -1;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(m));
    base = __shfl_sync(FULL, base, leader);
    return want ? (long long)(base + __popc(m & ((1u << lane) - 1u))) : -1;
}

__device__ __forceinline__ void pixel_centre(const so_frame& F, int W, int H, long long p, double* x, double* y) {
    const int px = (int)(p % W), py = (int)(p / W);
    *x = (px + 0.5 - 0.5 * W) * F.pix;
    *y = (0.5 * H - (py + 0.5)) * F.pix;
}

__global__ void k_route(const Route R) {
    const so_frame& F = *R.F;
    const long long n = (long long)R.W * R.H;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const long long p = base + threadIdx.x;
        const bool valid = p < n;
        bool band = true, audit = false;
        float al = 0.f, be = 0.f;
        if (valid) {
            double x, y;
            pixel_centre(F, R.W, R.H, p, &x, &y);
            so_vec3 d = view_dir(F, x, y);
            if (d.x < 0.0) {
                const double a = F.r * d.z / (-d.x), b = F.r * (-d.y) / (-d.x);
                const double rho = sqrt(a * a + b * b), psi = atan2(b, a);
                const double u = (psi + PI) * (R.band_n / (2.0 * PI));
                int i = (int)floor(u);
                const double f = u - i;
                i = ((i % R.band_n) + R.band_n) % R.band_n;
                const int j = (i + 1) % R.band_n;
                const double rc = R.band[i] + (R.band[j] - R.band[i]) * f;
                band = fabs(rho - rc) < R.band_m || fabs(a) > R.xy_max || fabs(b) > R.xy_max;
                al = (float)a;
                be = (float)b;
            }
            audit = !band && (pcg((uint32_t)p ^ R.audit_key) < R.audit_thr);
        }
        const long long js = push_idx(&R.counts[0], valid && !band);
        if (js >= 0) {
            R.list_s[js] = (uint32_t)p;
            so_sur_ray r;
            r.alpha = al;
            r.beta = be;
            r.spin = R.spin;
            r.incl_deg = R.incl_deg;
            R.rays_s[js] = r;
        }
        const long long jb = push_idx(&R.counts[1], valid && band);
        if (jb >= 0) R.list_b[jb] = (uint32_t)p;
        const long long ja = push_idx(&R.counts[2], audit);
        if (ja >= 0) {
            R.list_a[ja] = (uint32_t)p;
            R.audit_j[ja] = (uint32_t)js;
        }
    }
}

__global__ void k_xy(const so_frame* Fp, int W, int H, const uint32_t* __restrict__ list_b, int nb,
                     const uint32_t* __restrict__ list_a, int na, double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb + na) return;
    const long long p = i < nb ? list_b[i] : list_a[i - nb];
    pixel_centre(*Fp, W, H, p, x + i, y + i);
}

// Disk emission along the predicted crossings, in the integrator's order and with its transmission
// rule (k_trace64.cu, VAR_DISK): crossing k adds trans * disk_shade and dims trans by the disk's
// opacity; below 1e-4 the ray ends.
__device__ float4 shade_crossings(const so_scene& S, const so_frame& F, double x, double y, const float* o) {
    so_vec3 d = view_dir(F, x, y);
    RayC c;
    double ys[6];
    camera_photon(S.a, F.kp, F.ph, F.t, d, F.beta, c, ys);
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    double trans = 1.0;
    for (int k = 0; k < 3; ++k) {
        const float u = o[6 + k];
        if (!(u > 1e-4f)) continue;
        const double r = 1.0 / (double)u;
        float cs[4];
        disk_shade(S, r, 0.0, 0.0, c.lam, c.eta, c.E, cs);
        if (cs[3] > 0.f) {
            const float tf = (float)trans;
            acc[0] += tf * cs[0];
            acc[1] += tf * cs[1];
            acc[2] += tf * cs[2];
            acc[3] += tf * cs[1] * (float)k;
            trans *= 1.0 - cs[3];
            if (trans < 1e-4) break;
        }
    }
    return make_float4(acc[0], acc[1], acc[2], acc[3]);
}

__global__ void k_shade(const so_scene* Sp, const so_frame* Fp, int W, int H, const uint32_t* __restrict__ list_s,
                        int ns, const float* __restrict__ out, float4* __restrict__ px) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    const long long p = list_s[j];
    double x, y;
    pixel_centre(*Fp, W, H, p, &x, &y);
    px[p] = shade_crossings(*Sp, *Fp, x, y, out + (long)j * mlp::LDO);
}

__global__ void k_audit(const Audit A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < A.na) {
        const float* o = A.out + (long)A.audit_j[i] * mlp::LDO;
        const long long p = A.list_a[i];
        const int f = A.fate[i];
        const int cls = f == SO_FATE_ESCAPED ? 0 : f == SO_FATE_CAPTURED ? 1 : 2;
        const int am = (o[1] > o[0] && o[1] >= o[2]) ? 1 : (o[2] > o[0] && o[2] > o[1]) ? 2 : 0;
        v[0] = am != cls ? 1.0 : 0.0;
        if (cls == 0 && am == 0) {
            double s, c, sp, cp;
            sincos(A.theta[i], &s, &c);
            sincos(A.phi[i], &sp, &cp);
            const double tx = s * cp, ty = s * sp, tz = c;
            const double nn = sqrt((double)o[3] * o[3] + (double)o[4] * o[4] + (double)o[5] * o[5]);
            const double dot = nn > 0.0 ? (o[3] * tx + o[4] * ty + o[5] * tz) / nn : -1.0;
            v[1] = acos(fmax(-1.0, fmin(1.0, dot)));
            v[2] = 1.0;
        }
        for (int k = 0; k < 3; ++k) {
            const double rt = A.cross_r[3 * (long)i + k];
            if (rt > 0.0) {
                v[3] += fabs((double)o[6 + k] - 1.0 / rt);
                v[4] += 1.0;
                if (rt < 50.0) {
                    const double rp = 1.0 / fmax((double)o[6 + k], 1e-6);
                    v[5] += fabs(rp - rt) / rt;
                    v[6] += fabs((double)o[9 + k] - A.cross_g[3 * (long)i + k]);
                    v[7] += 1.0;
                }
            }
        }
        const float ys = A.px[p].y, yt = A.I[A.nb + i].y;
        v[8] = fabs((double)ys - (double)yt);
        v[9] = (double)ys;
    }
    double yt = 0.0;
    if (i < A.na) yt = A.I[A.nb + i].y;
    for (int k = 0; k < 10; ++k) {
        double t = v[k];
        for (int sh = 16; sh > 0; sh >>= 1) t += __shfl_xor_sync(FULL, t, sh);
        if (lane == 0 && t != 0.0) atomicAdd(&A.acc[k], t);
    }
    for (int sh = 16; sh > 0; sh >>= 1) yt += __shfl_xor_sync(FULL, yt, sh);
    if (lane == 0 && yt != 0.0) atomicAdd(&A.acc[10], yt);
}

__global__ void k_scatter(const uint32_t* __restrict__ list_b, int nb, const uint32_t* __restrict__ list_a, int na,
                          const float4* __restrict__ I, float4* __restrict__ px) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb + na) return;
    const long long p = i < nb ? list_b[i] : list_a[i - nb];
    px[p] = I[i];
}

}  // namespace

void launch_sample(long long n, int groups, uint32_t seed, double xy_max, const float* spin, const float* incl,
                   double r_cam, double* x, double* y, so_sur_ray* rays, cudaStream_t st) {
    k_sample<<<1184, 256, 0, st>>>(n, groups, seed, xy_max, spin, incl, r_cam, x, y, rays);
}

void launch_targets(long long n, int groups, const double* r_stop, const int8_t* fate, const double* th,
                    const double* ph, const double* cr, const double* cg, so_sur_target* tgt, cudaStream_t st) {
    k_targets<<<1184, 256, 0, st>>>(n, groups, r_stop, fate, th, ph, cr, cg, tgt);
}

void launch_route(const Route& R, int num_sms, cudaStream_t st) { k_route<<<num_sms * 8, 256, 0, st>>>(R); }

void launch_xy(const so_frame* F, int W, int H, const uint32_t* list_b, int nb, const uint32_t* list_a, int na, double* x,
               double* y, cudaStream_t st) {
    if (nb + na > 0) k_xy<<<(nb + na + 255) / 256, 256, 0, st>>>(F, W, H, list_b, nb, list_a, na, x, y);
}

void launch_shade(const so_scene* S, const so_frame* F, int W, int H, const uint32_t* list_s, int ns, const float* out,
                  float4* px, cudaStream_t st) {
    if (ns > 0) k_shade<<<(ns + 127) / 128, 128, 0, st>>>(S, F, W, H, list_s, ns, out, px);
}

void launch_audit(const Audit& A, cudaStream_t st) {
    if (A.na > 0) k_audit<<<(A.na + 127) / 128, 128, 0, st>>>(A);
}

void launch_scatter(const uint32_t* list_b, int nb, const uint32_t* list_a, int na, const float4* I, float4* px,
                    cudaStream_t st) {
    if (nb + na > 0) k_scatter<<<(nb + na + 255) / 256, 256, 0, st>>>(list_b, nb, list_a, na, I, px);
}

}  // namespace sur
}  // namespace so
