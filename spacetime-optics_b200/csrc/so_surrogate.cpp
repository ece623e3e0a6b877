// Ray surrogate, host side: parameters and optimiser state, the training step (features, four
// GELU layers and the head on the tensor cores, loss, backward GEMMs, deterministic split sums,
// AdamW), batched inference, the training set drawn from the FP64 integrator, and the surrogate
// thin-disk frame with band / audit routing to the integrator.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/so_tracer.h"
#include "so_kerr.cuh"
#include "so_mlp.h"
#include "so_sur.h"

using namespace so;
using mlp::bf16;

namespace so {
void set_global_error(const std::string& msg);
}

namespace {

constexpr double PI_D = 3.14159265358979323846;

// PCG-XSH-RR 32-bit generator (O'Neill 2014), for the initial weights, frequencies and the
// (spin, inclination) pairs of the training set.
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(0) {
        next();
        s += seed;
        next();
    }
    uint32_t next() {
        uint64_t old = s;
        s = old * 6364136223846793005ull + 1442695040888963407ull;
        uint32_t x = (uint32_t)(((old >> 18u) ^ old) >> 27u), rot = (uint32_t)(old >> 59u);
        return (x >> rot) | (x << ((32u - rot) & 31u));
    }
    double uniform() { return (next() + 0.5) * (1.0 / 4294967296.0); }
    double normal() {  // Box-Muller
        double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * PI_D * u2);
    }
};

template <class T>
cudaError_t dalloc(T** p, size_t n) {
    return cudaMalloc((void**)p, n * sizeof(T));
}

}  // namespace

struct so_surrogate {
    int device = 0;
    cudaStream_t st = nullptr;
    so_sur_opts o{};
    mlp::Layout L{};
    float *d_p = nullptr, *d_g = nullptr, *d_m = nullptr, *d_v = nullptr, *d_freq = nullptr;
    bf16 *d_W = nullptr, *d_WT = nullptr;
    int* d_err = nullptr;
    double* d_acc = nullptr;  // loss sums (8)
    int t = 0;                // AdamW steps taken
    long long cursor = 0;     // next training ray
    // training buffers for tb rows
    int tb = 0;
    bf16 *X = nullptr, *XT = nullptr, *dO = nullptr, *dOT = nullptr;
    bf16 *A[mlp::NHID] = {}, *AT[mlp::NHID] = {}, *dZ[2] = {}, *dZT[2] = {};
    bf16* D[mlp::NHID] = {};  // GELU derivatives of the hidden layers
    float *O = nullptr, *part = nullptr, *part_gb = nullptr;
    double* part_acc = nullptr;
    // fused inference: packed weight chunks of the 2-SM form (and of the 1-SM form, used where a
    // cluster launch is refused), rebuilt when the parameters change
    bf16 *d_wpack = nullptr, *d_wpack1 = nullptr;
    long pack_elems = 0, pack_elems1 = 0;
    mlp::FusedChunk chunks[mlp::FUSED_MAX_CHUNKS], chunks1[mlp::FUSED_MAX_CHUNKS];
    int nchunks = 0, nchunks1 = 0, num_sms = 148;
    bool use2 = false;  // 2-SM (cta_group::2) form on request: measured slower than the 1-SM form
    long long version = 1, packed_version = 0, packed_version1 = 0;
    // frame buffers for fcap pixels
    long long fcap = 0;
    uint32_t *list_s = nullptr, *list_b = nullptr, *list_a = nullptr, *audit_j = nullptr;
    so_sur_ray* rays_s = nullptr;
    unsigned long long* counts = nullptr;
    float* out = nullptr;
    double *fx = nullptr, *fy = nullptr, *fth = nullptr, *fph = nullptr, *fcr = nullptr, *fcg = nullptr;
    float4* fI = nullptr;
    int8_t* ffate = nullptr;
    double* facc = nullptr;
    cudaEvent_t ev[5] = {};
    std::string err;
};

namespace {

int fail(so_surrogate* s, int code, const std::string& msg) {
    if (s) s->err = msg;
    so::set_global_error(msg);
    return code;
}

#define SUR_CK(s, x)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) return fail(s, SO_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_train(so_surrogate* s) {
    void* ps[] = {s->X, s->XT, s->dO, s->dOT, s->O, s->part, s->part_gb, s->part_acc};
    for (void* p : ps)
        if (p) cudaFree(p);
    for (int l = 0; l < mlp::NHID; ++l) {
        if (s->A[l]) cudaFree(s->A[l]);
        if (s->AT[l]) cudaFree(s->AT[l]);
        if (s->D[l]) cudaFree(s->D[l]);
        s->A[l] = s->AT[l] = s->D[l] = nullptr;
    }
    for (int i = 0; i < 2; ++i) {
        if (s->dZ[i]) cudaFree(s->dZ[i]);
        if (s->dZT[i]) cudaFree(s->dZT[i]);
        s->dZ[i] = s->dZT[i] = nullptr;
    }
    s->X = s->XT = s->dO = s->dOT = nullptr;
    s->O = s->part = s->part_gb = nullptr;
    s->part_acc = nullptr;
    s->tb = 0;
}

void free_frame(so_surrogate* s) {
    void* ps[] = {s->list_s, s->list_b, s->list_a, s->audit_j, s->rays_s, s->counts, s->out, s->fx, s->fy,
                  s->fth, s->fph, s->fcr, s->fcg, s->fI, s->ffate, s->facc};
    for (void* p : ps)
        if (p) cudaFree(p);
    s->list_s = s->list_b = s->list_a = s->audit_j = nullptr;
    s->rays_s = nullptr;
    s->counts = nullptr;
    s->out = nullptr;
    s->fx = s->fy = s->fth = s->fph = s->fcr = s->fcg = nullptr;
    s->fI = nullptr;
    s->ffate = nullptr;
    s->facc = nullptr;
    s->fcap = 0;
}

// Split count of a reduction over `rows` rays: about 1024 rays per slice, a multiple of 64 each.
int splits_for(int rows) {
    int S = std::max(1, rows / 1024);
    while (S > 1 && (rows % S != 0 || (rows / S) % 64 != 0)) --S;
    return S;
}

int ensure_train(so_surrogate* s, int rows) {
    if (rows <= s->tb) return SO_OK;
    free_train(s);
    const size_t R = (size_t)rows;
    bool ok = dalloc(&s->X, R * mlp::NFEAT) == cudaSuccess && dalloc(&s->XT, R * mlp::NFEAT) == cudaSuccess &&
              dalloc(&s->dO, R * mlp::LDO) == cudaSuccess && dalloc(&s->dOT, R * mlp::LDO) == cudaSuccess &&
              dalloc(&s->O, R * mlp::LDO) == cudaSuccess &&
              dalloc(&s->part, (size_t)splits_for(rows) * mlp::HID * mlp::HID) == cudaSuccess &&
              dalloc(&s->part_gb, (R / 128 + 1) * mlp::LDO) == cudaSuccess &&
              dalloc(&s->part_acc, (R / 128 + 1) * 8) == cudaSuccess;
    for (int l = 0; ok && l < mlp::NHID; ++l)
        ok = dalloc(&s->A[l], R * mlp::HID) == cudaSuccess && dalloc(&s->AT[l], R * mlp::HID) == cudaSuccess &&
             dalloc(&s->D[l], R * mlp::HID) == cudaSuccess;
    for (int i = 0; ok && i < 2; ++i)
        ok = dalloc(&s->dZ[i], R * mlp::HID) == cudaSuccess && dalloc(&s->dZT[i], R * mlp::HID) == cudaSuccess;
    if (!ok) {
        free_train(s);
        return fail(s, SO_ERR_ALLOC, "surrogate: training buffers");
    }
    s->tb = rows;
    return SO_OK;
}

int gemm(so_surrogate* s, const mlp::GemmArgs& g0, cudaStream_t st) {
    mlp::GemmArgs g = g0;
    g.err = s->d_err;
    const char* why = nullptr;
    int rc = mlp::launch_gemm(g, st, &why);
    if (rc) return fail(s, rc, why ? why : "surrogate: gemm launch");
    return SO_OK;
}

mlp::GemmArgs args(const bf16* A, long lda, const bf16* B, long ldb, int M, int N, int K, int epi) {
    mlp::GemmArgs g;
    std::memset(&g, 0, sizeof g);
    g.A = A;
    g.lda = lda;
    g.B = B;
    g.ldb = ldb;
    g.M = M;
    g.N = N;
    g.K = K;
    g.splits = 1;
    g.epi = epi;
    return g;
}

// Training forward pass of `rows` rays starting at `off` (layer by layer, keeping the GELU
// derivatives D, the activations and their transposes for the backward pass).  The head's FP32
// outputs go to O (16 floats per row).
int forward(so_surrogate* s, const so_sur_ray* rays, long long n, long long off, int rows, int wrap, float* O,
            cudaStream_t st) {
    const mlp::Layout& L = s->L;
    mlp::launch_features(rays, off, n, rows, wrap, s->d_freq, s->X, s->XT, rows, st);
    const bf16* in = s->X;
    for (int l = 0; l < mlp::NHID; ++l) {
        mlp::GemmArgs g = args(in, L.k[l], s->d_W + L.w[l], L.k[l], rows, L.n[l], L.k[l], mlp::EPI_GELU);
        g.bias = s->d_p + L.b[l];
        g.out_b = s->A[l];
        g.ldob = mlp::HID;
        g.out_t = s->AT[l];
        g.ldot = rows;
        g.d_out = s->D[l];
        g.ldd = mlp::HID;
        int rc = gemm(s, g, st);
        if (rc) return rc;
        in = s->A[l];
    }
    mlp::GemmArgs g = args(in, mlp::HID, s->d_W + L.w[mlp::NHID], mlp::HID, rows, mlp::LDO, mlp::HID, mlp::EPI_F32);
    g.bias = s->d_p + L.b[mlp::NHID];
    g.out_f = O;
    g.ldf = mlp::LDO;
    return gemm(s, g, st);
}

// Loss and backward pass of the rows of the last training forward: gradients into d_g.
int backward(so_surrogate* s, const so_sur_target* tgt, long long n, long long off, int rows, cudaStream_t st) {
    const mlp::Layout& L = s->L;
    const int H = mlp::HID, S = splits_for(rows);
    mlp::LossWeights w{s->o.w_dir, s->o.w_u, s->o.w_g};
    mlp::launch_loss(s->O, tgt, off, n, rows, w, s->dO, s->dOT, s->part_gb, s->part_acc, s->d_g + L.b[mlp::NHID],
                     s->d_acc, st);
    // head weights: dWh^T [256 x 16] = A3^T . dO
    {
        mlp::GemmArgs g = args(s->AT[mlp::NHID - 1], rows, s->dOT, rows, H, mlp::LDO, rows, mlp::EPI_SPLIT_T);
        g.splits = S;
        g.out_f = s->part;
        g.ldf = H;
        g.split_stride = (long)H * mlp::LDO;
        int rc = gemm(s, g, st);
        if (rc) return rc;
        mlp::launch_sum_splits(s->part, S, (long)H * mlp::LDO, s->d_g + L.w[mlp::NHID], st);
    }
    // dZ3 = (dO . Wh) * gelu'(Z3)
    int cur = 0;
    {
        mlp::GemmArgs g = args(s->dO, mlp::LDO, s->d_WT + L.w[mlp::NHID], mlp::LDO, rows, H, mlp::LDO, mlp::EPI_GELU_BWD);
        g.d_in = s->D[mlp::NHID - 1];
        g.ldd = H;
        g.out_b = s->dZ[cur];
        g.ldob = H;
        g.out_t = s->dZT[cur];
        g.ldot = rows;
        int rc = gemm(s, g, st);
        if (rc) return rc;
    }
    for (int l = mlp::NHID - 1; l >= 0; --l) {
        const int K = L.k[l];
        const bf16* inT = l == 0 ? s->XT : s->AT[l - 1];
        mlp::GemmArgs g = args(s->dZT[cur], rows, inT, rows, H, K, rows, mlp::EPI_SPLIT);
        g.splits = S;
        g.out_f = s->part;
        g.ldf = K;
        g.split_stride = (long)H * K;
        int rc = gemm(s, g, st);
        if (rc) return rc;
        mlp::launch_sum_splits(s->part, S, (long)H * K, s->d_g + L.w[l], st);
        mlp::launch_rowsum(s->dZT[cur], H, rows, s->d_g + L.b[l], st);
        if (l > 0) {
            mlp::GemmArgs d = args(s->dZ[cur], H, s->d_WT + L.w[l], H, rows, K, H, mlp::EPI_GELU_BWD);
            d.d_in = s->D[l - 1];
            d.ldd = H;
            d.out_b = s->dZ[cur ^ 1];
            d.ldob = H;
            d.out_t = s->dZT[cur ^ 1];
            d.ldot = rows;
            rc = gemm(s, d, st);
            if (rc) return rc;
            cur ^= 1;
        }
    }
    return SO_OK;
}

int read_loss(so_surrogate* s, long long rays, so_sur_loss* out) {
    double acc[8];
    SUR_CK(s, cudaMemcpyAsync(acc, s->d_acc, sizeof acc, cudaMemcpyDeviceToHost, s->st));
    SUR_CK(s, cudaStreamSynchronize(s->st));
    int e = 0;
    SUR_CK(s, cudaMemcpy(&e, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(s, SO_ERR_WATCHDOG, "surrogate: a tensor-core wait gave up");
    if (out) {
        const double k = rays > 0 ? 1.0 / (double)rays : 0.0;
        out->ce = acc[0] * k;
        out->dir = acc[1] * k;
        out->u = acc[2] * k;
        out->g = acc[3] * k;
        out->accuracy = acc[4] * k;
        out->total = acc[5] * k;
        out->rays = rays;
    }
    return SO_OK;
}

float schedule(const so_sur_opts& o, int step, int steps) {
    if (o.warmup > 0 && step < o.warmup) return o.lr * (float)(step + 1) / (float)o.warmup;
    const int span = std::max(1, steps - o.warmup);
    const double q = std::min(1.0, (double)(step - o.warmup) / span);
    return (float)(o.lr_final + 0.5 * (o.lr - o.lr_final) * (1.0 + std::cos(PI_D * q)));
}

int set_device(so_surrogate* s) {
    SUR_CK(s, cudaSetDevice(s->device));
    return SO_OK;
}

}  // namespace

extern "C" {

void so_sur_default_opts(so_sur_opts* o) {
    if (!o) return;
    o->fourier_sigma = 0.35f;
    o->seed = 1;
    o->batch = 65536;
    o->lr = 2e-3f;
    o->lr_final = 5e-5f;
    o->warmup = 100;
    o->beta1 = 0.9f;
    o->beta2 = 0.999f;
    o->eps = 1e-8f;
    o->weight_decay = 0.0f;
    o->w_dir = 1.0f;
    o->w_u = 30.0f;
    o->w_g = 1.0f;
}

int so_sur_create(int device, const so_sur_opts* opts, so_surrogate** out) {
    if (!out) return SO_ERR_ARG;
    *out = nullptr;
    so_sur_opts o;
    so_sur_default_opts(&o);
    if (opts) o = *opts;
    if (o.batch <= 0 || o.batch % 128) return fail(nullptr, SO_ERR_ARG, "so_sur_create: batch must be a positive multiple of 128");
    if (!(o.fourier_sigma > 0.f)) return fail(nullptr, SO_ERR_ARG, "so_sur_create: fourier_sigma must be positive");
    so_surrogate* s = new so_surrogate;
    s->device = device;
    s->o = o;
    s->L = mlp::param_layout();
    if (s->L.total != SO_SUR_NPARAMS) {
        delete s;
        return fail(nullptr, SO_ERR_ARG, "so_sur_create: parameter layout mismatch");
    }
    auto bad = [&](int code, const char* m) {
        so_sur_destroy(s);
        return fail(nullptr, code, m);
    };
    if (cudaSetDevice(device) != cudaSuccess) return bad(SO_ERR_CUDA, "so_sur_create: cudaSetDevice");
    // a blocking stream: work on it is ordered after the legacy default stream's, where callers
    // such as torch put the rays and targets they pass in
    if (cudaStreamCreate(&s->st) != cudaSuccess) return bad(SO_ERR_CUDA, "so_sur_create: stream");
    const size_t P = SO_SUR_NPARAMS;
    if (dalloc(&s->d_p, P) || dalloc(&s->d_g, P) || dalloc(&s->d_m, P) || dalloc(&s->d_v, P) ||
        dalloc(&s->d_freq, (size_t)mlp::NFREQ * 4) || dalloc(&s->d_W, P) || dalloc(&s->d_WT, P) || dalloc(&s->d_err, 1) ||
        dalloc(&s->d_acc, 8))
        return bad(SO_ERR_ALLOC, "so_sur_create: device allocation");
    for (auto& e : s->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return bad(SO_ERR_CUDA, "so_sur_create: events");
    s->nchunks = mlp::fused2_chunks(s->chunks, &s->pack_elems);
    s->nchunks1 = mlp::fused_chunks(s->chunks1, &s->pack_elems1);
    if (s->nchunks <= 0 || s->nchunks1 <= 0) return bad(SO_ERR_ARG, "so_sur_create: weight chunk table overflow");
    if (dalloc(&s->d_wpack, (size_t)s->pack_elems) || dalloc(&s->d_wpack1, (size_t)s->pack_elems1))
        return bad(SO_ERR_ALLOC, "so_sur_create: device allocation");
    if (cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return bad(SO_ERR_CUDA, "so_sur_create: device attributes");
    // initial parameters: U(-1/sqrt(K), 1/sqrt(K)) for weights and biases; head rows 12-15 zero
    std::vector<float> p(P, 0.f), f((size_t)mlp::NFREQ * 4);
    Rng rng(((uint64_t)o.seed << 1) | 1u);
    for (int l = 0; l < mlp::NLAYER; ++l) {
        const double bound = 1.0 / std::sqrt((double)s->L.k[l]);
        const int rows = l < mlp::NHID ? s->L.n[l] : mlp::NOUT;
        for (int i = 0; i < rows; ++i)
            for (int k = 0; k < s->L.k[l]; ++k)
                p[s->L.w[l] + (size_t)i * s->L.k[l] + k] = (float)((2.0 * rng.uniform() - 1.0) * bound);
        for (int i = 0; i < rows; ++i) p[s->L.b[l] + i] = (float)((2.0 * rng.uniform() - 1.0) * bound);
    }
    for (auto& v : f) v = (float)(rng.normal() * o.fourier_sigma);
    int rc = so_sur_set_params(s, p.data(), f.data());
    if (rc) {
        so_sur_destroy(s);
        return rc;
    }
    *out = s;
    return SO_OK;
}

void so_sur_destroy(so_surrogate* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->st) cudaStreamSynchronize(s->st);
    free_train(s);
    free_frame(s);
    void* ps[] = {s->d_p, s->d_g, s->d_m, s->d_v, s->d_freq, s->d_W, s->d_WT, s->d_err, s->d_acc, s->d_wpack, s->d_wpack1};
    for (void* p : ps)
        if (p) cudaFree(p);
    for (auto e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
}

int so_sur_get_params(so_surrogate* s, float* params, float* freqs) {
    if (!s) return SO_ERR_ARG;
    if (int rc = set_device(s)) return rc;
    SUR_CK(s, cudaStreamSynchronize(s->st));
    if (params) SUR_CK(s, cudaMemcpy(params, s->d_p, SO_SUR_NPARAMS * sizeof(float), cudaMemcpyDeviceToHost));
    if (freqs) SUR_CK(s, cudaMemcpy(freqs, s->d_freq, mlp::NFREQ * 4 * sizeof(float), cudaMemcpyDeviceToHost));
    return SO_OK;
}

int so_sur_set_params(so_surrogate* s, const float* params, const float* freqs) {
    if (!s) return SO_ERR_ARG;
    if (int rc = set_device(s)) return rc;
    SUR_CK(s, cudaStreamSynchronize(s->st));
    if (params) {
        SUR_CK(s, cudaMemcpy(s->d_p, params, SO_SUR_NPARAMS * sizeof(float), cudaMemcpyHostToDevice));
        SUR_CK(s, cudaMemsetAsync(s->d_m, 0, SO_SUR_NPARAMS * sizeof(float), s->st));
        SUR_CK(s, cudaMemsetAsync(s->d_v, 0, SO_SUR_NPARAMS * sizeof(float), s->st));
        SUR_CK(s, cudaMemsetAsync(s->d_WT, 0, SO_SUR_NPARAMS * sizeof(bf16), s->st));
        mlp::launch_pack(s->d_p, SO_SUR_NPARAMS, s->d_W, s->d_WT, s->st);
        SUR_CK(s, cudaGetLastError());
        s->t = 0;
        ++s->version;
    }
    if (freqs) SUR_CK(s, cudaMemcpy(s->d_freq, freqs, mlp::NFREQ * 4 * sizeof(float), cudaMemcpyHostToDevice));
    SUR_CK(s, cudaMemsetAsync(s->d_err, 0, sizeof(int), s->st));
    SUR_CK(s, cudaStreamSynchronize(s->st));
    return SO_OK;
}

int so_sur_train(so_surrogate* s, const so_sur_ray* d_rays, const so_sur_target* d_tgt, long long n, int steps,
                 so_sur_loss* last) {
    if (!s || !d_rays || !d_tgt || n <= 0 || steps < 0) return fail(s, SO_ERR_ARG, "so_sur_train: bad arguments");
    if (int rc = set_device(s)) return rc;
    const int B = s->o.batch;
    if (int rc = ensure_train(s, B)) return rc;
    for (int k = 0; k < steps; ++k) {
        const long long off = s->cursor % n;
        SUR_CK(s, cudaMemsetAsync(s->d_acc, 0, 8 * sizeof(double), s->st));
        int rc = forward(s, d_rays, n, off, B, 1, s->O, s->st);
        if (!rc) rc = backward(s, d_tgt, n, off, B, s->st);
        if (rc) return rc;
        ++s->t;
        mlp::launch_adam(s->d_p, s->d_g, s->d_m, s->d_v, SO_SUR_NPARAMS, schedule(s->o, k, steps), s->o.beta1,
                         s->o.beta2, s->o.eps, s->o.weight_decay, s->t, s->d_W, s->d_WT, s->st);
        SUR_CK(s, cudaGetLastError());
        ++s->version;
        s->cursor = (off + B) % n;
    }
    return read_loss(s, steps > 0 ? B : 0, last);
}

int so_sur_evaluate(so_surrogate* s, const so_sur_ray* d_rays, const so_sur_target* d_tgt, long long n,
                    so_sur_loss* loss) {
    if (!s || !d_rays || !d_tgt || n < 128) return fail(s, SO_ERR_ARG, "so_sur_evaluate: bad arguments");
    if (int rc = set_device(s)) return rc;
    const int B = s->o.batch;
    if (int rc = ensure_train(s, B)) return rc;
    const long long m = n - n % 128;
    SUR_CK(s, cudaMemsetAsync(s->d_acc, 0, 8 * sizeof(double), s->st));
    for (long long off = 0; off < m; off += B) {
        const int rows = (int)std::min<long long>(B, m - off);
        int rc = forward(s, d_rays, n, off, rows, 0, s->O, s->st);
        if (rc) return rc;
        mlp::LossWeights w{s->o.w_dir, s->o.w_u, s->o.w_g};
        // the loss kernel scales gradients by 1/rows; the loss sums themselves are unscaled
        mlp::launch_loss(s->O, d_tgt, off, n, rows, w, s->dO, s->dOT, s->part_gb, s->part_acc, s->d_g + s->L.b[mlp::NHID],
                         s->d_acc, s->st);
    }
    return read_loss(s, m, loss);
}

int so_sur_gradients(so_surrogate* s, const so_sur_ray* d_rays, const so_sur_target* d_tgt, int n, float* grads,
                     so_sur_loss* loss) {
    if (!s || !d_rays || !d_tgt || n <= 0 || n % 128 || !grads) return fail(s, SO_ERR_ARG, "so_sur_gradients: bad arguments");
    if (int rc = set_device(s)) return rc;
    if (int rc = ensure_train(s, n)) return rc;
    SUR_CK(s, cudaMemsetAsync(s->d_acc, 0, 8 * sizeof(double), s->st));
    int rc = forward(s, d_rays, n, 0, n, 0, s->O, s->st);
    if (!rc) rc = backward(s, d_tgt, n, 0, n, s->st);
    if (rc) return rc;
    rc = read_loss(s, n, loss);
    if (rc) return rc;
    SUR_CK(s, cudaMemcpy(grads, s->d_g, SO_SUR_NPARAMS * sizeof(float), cudaMemcpyDeviceToHost));
    return SO_OK;
}

int so_sur_infer(so_surrogate* s, const so_sur_ray* d_rays, long long n, float* d_out, void* stream) {
    if (!s || n < 0 || (n > 0 && (!d_rays || !d_out))) return fail(s, SO_ERR_ARG, "so_sur_infer: bad arguments");
    if (n == 0) return SO_OK;
    if (((uintptr_t)d_out & 15u) != 0) return fail(s, SO_ERR_ARG, "so_sur_infer: d_out must be 16-byte aligned");
    if (int rc = set_device(s)) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->st;
    mlp::FusedArgs a;
    std::memset(&a, 0, sizeof a);
    a.rays = d_rays;
    a.n = n;
    a.out = d_out;
    a.params = s->d_p;
    for (int l = 0; l < mlp::NLAYER; ++l) a.bias_off[l] = s->L.b[l];
    a.freq = s->d_freq;
    a.err = s->d_err;
    if (s->use2) {  // 2-SM form
        a.wpack = reinterpret_cast<const uint8_t*>(s->d_wpack);
        for (int q = 0; q < s->nchunks; ++q) a.chunks[q] = s->chunks[q];
        a.nchunks = s->nchunks;
        if (s->packed_version != s->version) {
            mlp::launch_pack_chunks(s->d_W, a, s->d_wpack, st);
            SUR_CK(s, cudaGetLastError());
            s->packed_version = s->version;
        }
        if (mlp::launch_mlp_fused2(a, s->num_sms, st) == SO_OK) return SO_OK;
        cudaGetLastError();  // a refused cluster launch: use the 1-SM form from now on
        s->use2 = false;
    }
    a.wpack = reinterpret_cast<const uint8_t*>(s->d_wpack1);
    for (int q = 0; q < s->nchunks1; ++q) a.chunks[q] = s->chunks1[q];
    a.nchunks = s->nchunks1;
    if (s->packed_version1 != s->version) {
        mlp::launch_pack_chunks(s->d_W, a, s->d_wpack1, st);
        SUR_CK(s, cudaGetLastError());
        s->packed_version1 = s->version;
    }
    if (mlp::launch_mlp_fused(a, s->num_sms, st)) return fail(s, SO_ERR_CUDA, "so_sur_infer: launch");
    return SO_OK;
}

int so_sur_set_infer_ctas(so_surrogate* s, int ctas) {
    if (!s || (ctas != 1 && ctas != 2)) return s ? fail(s, SO_ERR_ARG, "so_sur_set_infer_ctas: 1 or 2") : SO_ERR_ARG;
    s->use2 = ctas == 2;
    return SO_OK;
}

int so_sur_dataset(so_renderer* r, const so_frame* f, long long n, int groups, uint32_t seed, const so_sur_ranges* rg,
                   so_sur_ray* d_rays, so_sur_target* d_tgt, so_stats* stats) {
    if (!r || !f || !rg || !d_rays || !d_tgt || groups <= 0 || n <= 0 || n % groups)
        return r ? rend_fail(r, SO_ERR_ARG, "so_sur_dataset: bad arguments (n must be a multiple of groups)") : SO_ERR_ARG;
    if (n > 0x7fffffffll) return rend_fail(r, SO_ERR_SIZE, "so_sur_dataset: more than 2^31 rays");
    if (cudaSetDevice(rend_device(r)) != cudaSuccess) return rend_fail(r, SO_ERR_CUDA, "cudaSetDevice");
    cudaStream_t st = rend_stream(r);
    const so_scene S0 = rend_scene(r);  // host copy; its table pointers are the renderer's device tables
    // one scene and one camera frame per (spin, inclination) group
    std::vector<so_scene> scenes((size_t)groups);
    std::vector<so_frame> frames((size_t)groups);
    std::vector<int> fscene((size_t)groups);
    std::vector<float> spin((size_t)groups), incl((size_t)groups);
    std::vector<double> r_stop((size_t)groups);
    Rng rng(((uint64_t)seed << 1) | 1u);
    for (int g = 0; g < groups; ++g) {
        const double a = rg->a_min + (rg->a_max - rg->a_min) * rng.uniform();
        const double i_deg = rg->incl_min + (rg->incl_max - rg->incl_min) * rng.uniform();
        so_scene S = S0;
        scene_set_spin(&S, a);
        so_frame F = *f;
        F.th = i_deg * PI_D / 180.0;
        F.ph = 0.0;
        F.t = 0.0;
        kerr_point(S.a, F.r, F.th, &F.kp);
        F.F = so_vec3{-1, 0, 0};
        F.U = so_vec3{0, -1, 0};
        F.R = so_vec3{0, 0, 1};
        F.beta = so_vec3{0, 0, 0};
        F.cx = F.cy = 0.0;
        scenes[g] = S;
        frames[g] = F;
        fscene[g] = g;
        spin[g] = (float)S.a;
        incl[g] = (float)i_deg;
        r_stop[g] = S.r_stop;
    }
    double *x = nullptr, *y = nullptr, *th = nullptr, *ph = nullptr, *cr = nullptr, *cg = nullptr, *d_rstop = nullptr;
    int8_t* fate = nullptr;
    so_scene* d_scenes = nullptr;
    so_frame* d_frames = nullptr;
    int* d_fscene = nullptr;
    float *d_spin = nullptr, *d_incl = nullptr;
    auto cleanup = [&]() {
        void* ps[] = {x, y, th, ph, cr, cg, d_rstop, fate, d_scenes, d_frames, d_fscene, d_spin, d_incl};
        for (void* p : ps)
            if (p) cudaFree(p);
    };
    const size_t N = (size_t)n, G = (size_t)groups;
    if (dalloc(&x, N) || dalloc(&y, N) || dalloc(&th, N) || dalloc(&ph, N) || dalloc(&cr, 3 * N) || dalloc(&cg, 3 * N) ||
        dalloc(&fate, N) || dalloc(&d_scenes, G) || dalloc(&d_frames, G) || dalloc(&d_fscene, G) || dalloc(&d_spin, G) ||
        dalloc(&d_incl, G) || dalloc(&d_rstop, G)) {
        cleanup();
        return rend_fail(r, SO_ERR_ALLOC, "so_sur_dataset: device allocation");
    }
    int rc = SO_OK;
    auto up = [&](void* d, const void* h, size_t bytes) {
        if (!rc && cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
            rc = rend_fail(r, SO_ERR_CUDA, "so_sur_dataset: upload");
    };
    up(d_scenes, scenes.data(), G * sizeof(so_scene));
    up(d_frames, frames.data(), G * sizeof(so_frame));
    up(d_fscene, fscene.data(), G * sizeof(int));
    up(d_spin, spin.data(), G * sizeof(float));
    up(d_incl, incl.data(), G * sizeof(float));
    up(d_rstop, r_stop.data(), G * sizeof(double));
    so_rays_out o;
    std::memset(&o, 0, sizeof o);
    o.fate = fate;
    o.theta = th;
    o.phi = ph;
    o.cross_r = cr;
    o.cross_g = cg;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    if (!rc) sur::launch_sample(n, groups, seed, rg->xy_max, d_spin, d_incl, f->r, x, y, d_rays, st);
    // every group in one persistent launch: ray i uses frame / scene i % groups
    if (!rc) rc = rend_trace_list_frames(r, (int)n, x, y, o, 1, d_scenes, d_frames, d_fscene, groups);
    if (!rc) sur::launch_targets(n, groups, d_rstop, fate, th, ph, cr, cg, d_tgt, st);
    if (!rc && cudaGetLastError() != cudaSuccess) rc = rend_fail(r, SO_ERR_CUDA, "so_sur_dataset: kernel launch");
    cudaEventRecord(e1, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = rend_fail(r, SO_ERR_CUDA, "so_sur_dataset: trace");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cleanup();
    if (!rc && stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->ms_trace = ms;
        stats->samples = n;
    }
    return rc;
}

int so_sur_render(so_surrogate* s, so_renderer* r, const so_frame* f, const so_sur_frame_opts* opt, float* d_px,
                  so_sur_report* rep) {
    if (!s || !r || !f || !opt || !d_px) return fail(s, SO_ERR_ARG, "so_sur_render: bad arguments");
    if (rend_device(r) != s->device) return fail(s, SO_ERR_ARG, "so_sur_render: renderer and surrogate on different devices");
    const so_scene& S = rend_scene(r);
    if (S.mode != SO_MODE_VISIBLE || !S.disk_on) return fail(s, SO_ERR_UNSUPPORTED, "so_sur_render: needs a visible-mode disk scene");
    if (S.disk_turb_amp > 0.f) return fail(s, SO_ERR_UNSUPPORTED, "so_sur_render: disk turbulence depends on the crossing phase");
    if (!(opt->band_m >= 0.0) || !(opt->audit_frac >= 0.0 && opt->audit_frac <= 1.0))
        return fail(s, SO_ERR_ARG, "so_sur_render: band_m >= 0 and audit_frac in [0, 1]");
    if (int rc = set_device(s)) return rc;
    const so_settings& rs = rend_settings(r);
    const long long npix = (long long)rs.W * rs.H;
    if (npix <= 0 || npix > 0x7fffffffll) return fail(s, SO_ERR_SIZE, "so_sur_render: frame size");
    if (npix > s->fcap) {
        free_frame(s);
        const size_t P = (size_t)npix;
        if (dalloc(&s->list_s, P) || dalloc(&s->list_b, P) || dalloc(&s->list_a, P) || dalloc(&s->audit_j, P) ||
            dalloc(&s->rays_s, P) || dalloc(&s->counts, 4) || dalloc(&s->out, P * mlp::LDO) || dalloc(&s->fx, P) ||
            dalloc(&s->fy, P) || dalloc(&s->fth, P) || dalloc(&s->fph, P) || dalloc(&s->fcr, 3 * P) ||
            dalloc(&s->fcg, 3 * P) || dalloc(&s->fI, P) || dalloc(&s->ffate, P) || dalloc(&s->facc, 16)) {
            free_frame(s);
            return fail(s, SO_ERR_ALLOC, "so_sur_render: device allocation");
        }
        s->fcap = npix;
    }
    cudaStream_t st = rend_stream(r);
    so_frame F = *f;
    F.W = rs.W;
    F.H = rs.H;
    F.spp = 1;
    const so_frame* dF = nullptr;
    int rc = rend_upload_frame(r, F, &dF);
    if (rc) return fail(s, rc, "so_sur_render: frame upload");
    const float* band = nullptr;
    int band_n = 0;
    rc = rend_band_table(r, F.th, &band, &band_n);
    if (rc) return fail(s, rc, "so_sur_render: critical-curve table");
    SUR_CK(s, cudaEventRecord(s->ev[0], st));
    SUR_CK(s, cudaMemsetAsync(s->counts, 0, 4 * sizeof(unsigned long long), st));
    SUR_CK(s, cudaMemsetAsync(s->facc, 0, 16 * sizeof(double), st));
    sur::Route R;
    R.F = dF;
    R.W = rs.W;
    R.H = rs.H;
    R.band = band;
    R.band_n = band_n;
    R.band_m = opt->band_m;
    R.xy_max = 12.0;
    R.audit_thr = (uint32_t)std::min(4294967295.0, opt->audit_frac * 4294967296.0);
    R.audit_key = (uint32_t)(opt->audit_seed * 2654435761u + 0x5bd1e995u);
    R.spin = (float)S.a;
    R.incl_deg = (float)(F.th * 180.0 / PI_D);
    R.counts = s->counts;
    R.list_s = s->list_s;
    R.rays_s = s->rays_s;
    R.list_b = s->list_b;
    R.list_a = s->list_a;
    R.audit_j = s->audit_j;
    sur::launch_route(R, rend_num_sms(r), st);
    SUR_CK(s, cudaGetLastError());
    SUR_CK(s, cudaEventRecord(s->ev[1], st));
    unsigned long long cnt[4];
    SUR_CK(s, cudaMemcpyAsync(cnt, s->counts, sizeof cnt, cudaMemcpyDeviceToHost, st));
    SUR_CK(s, cudaStreamSynchronize(st));
    const int ns = (int)cnt[0], nb = (int)cnt[1], na = (int)cnt[2];
    rc = so_sur_infer(s, s->rays_s, ns, s->out, st);
    if (rc) return rc;
    SUR_CK(s, cudaEventRecord(s->ev[2], st));
    float4* px = reinterpret_cast<float4*>(d_px);
    sur::launch_shade(rend_scene_dev(r), dF, rs.W, rs.H, s->list_s, ns, s->out, px, st);
    SUR_CK(s, cudaGetLastError());
    SUR_CK(s, cudaEventRecord(s->ev[3], st));
    // integrator: band and audit rays with the scene's own (disk) tracer, then the audit rays again
    // in vacuum for their crossing records
    sur::launch_xy(dF, rs.W, rs.H, s->list_b, nb, s->list_a, na, s->fx, s->fy, st);
    if (na > 0) {  // the audit rays' vacuum records, on the renderer's second stream meanwhile
        so_rays_out v;
        std::memset(&v, 0, sizeof v);
        v.fate = s->ffate;
        v.theta = s->fth;
        v.phi = s->fph;
        v.cross_r = s->fcr;
        v.cross_g = s->fcg;
        rc = rend_trace_list(r, na, s->fx + nb, s->fy + nb, v, 1, 1);
        if (rc) return fail(s, rc, "so_sur_render: audit integrator");
    }
    so_rays_out o;
    std::memset(&o, 0, sizeof o);
    o.I = reinterpret_cast<float*>(s->fI);
    rc = rend_trace_list(r, nb + na, s->fx, s->fy, o, 0);
    if (rc) return fail(s, rc, "so_sur_render: integrator");
    if (na > 0) {
        rc = rend_join_side(r);
        if (rc) return fail(s, rc, "so_sur_render: stream join");
        sur::Audit A;
        A.na = na;
        A.nb = nb;
        A.list_a = s->list_a;
        A.audit_j = s->audit_j;
        A.out = s->out;
        A.px = px;
        A.I = s->fI;
        A.fate = s->ffate;
        A.theta = s->fth;
        A.phi = s->fph;
        A.cross_r = s->fcr;
        A.cross_g = s->fcg;
        A.acc = s->facc;
        sur::launch_audit(A, st);
    }
    sur::launch_scatter(s->list_b, nb, s->list_a, na, s->fI, px, st);
    SUR_CK(s, cudaGetLastError());
    SUR_CK(s, cudaEventRecord(s->ev[4], st));
    double acc[16];
    SUR_CK(s, cudaMemcpyAsync(acc, s->facc, sizeof acc, cudaMemcpyDeviceToHost, st));
    SUR_CK(s, cudaStreamSynchronize(st));
    int e = 0;
    SUR_CK(s, cudaMemcpy(&e, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(s, SO_ERR_WATCHDOG, "surrogate: a tensor-core wait gave up");
    if (rep) {
        std::memset(rep, 0, sizeof *rep);
        rep->rays = npix;
        rep->surrogate_rays = ns - na;
        rep->band_rays = nb;
        rep->audit_rays = na;
        float t[4];
        for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&t[i], s->ev[i], s->ev[i + 1]);
        rep->ms_route = t[0];
        rep->ms_mlp = t[1];
        rep->ms_shade = t[2];
        rep->ms_integrator = t[3];
        rep->ms_total = (double)t[0] + t[1] + t[2] + t[3];
        rep->audit_class_mismatch = (long long)acc[0];
        rep->audit_dir_err = acc[2] > 0 ? acc[1] / acc[2] : 0.0;
        rep->audit_u_err = acc[4] > 0 ? acc[3] / acc[4] : 0.0;
        rep->audit_r_err = acc[7] > 0 ? acc[5] / acc[7] : 0.0;
        rep->audit_g_err = acc[7] > 0 ? acc[6] / acc[7] : 0.0;
        rep->audit_l1 = acc[10] > 0 ? acc[8] / acc[10] : 0.0;
        rep->audit_flux = acc[10] > 0 ? acc[9] / acc[10] - 1.0 : 0.0;
    }
    return SO_OK;
}

int so_sur_gemm(const void* d_a, const void* d_b, const float* d_bias, float* d_c, int M, int N, int K, int splits,
                int layout) {
    if (!d_a || !d_b || !d_c || layout < 0 || layout > 2 || splits < 1 || (layout == 0 && splits != 1))
        return SO_ERR_ARG;
    mlp::GemmArgs g = args((const bf16*)d_a, K, (const bf16*)d_b, K, M, N, K,
                           layout == 0 ? mlp::EPI_F32 : layout == 1 ? mlp::EPI_SPLIT : mlp::EPI_SPLIT_T);
    g.splits = splits;
    g.bias = layout == 0 ? d_bias : nullptr;
    g.out_f = d_c;
    g.ldf = layout == 2 ? M : N;
    g.split_stride = (long)M * N;
    int* d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) return SO_ERR_ALLOC;
    cudaMemset(d_err, 0, sizeof(int));
    g.err = d_err;
    const char* why = nullptr;
    int rc = mlp::launch_gemm(g, nullptr, &why);
    if (rc) {
        cudaFree(d_err);
        so::set_global_error(why ? why : "so_sur_gemm");
        return rc;
    }
    int e = 0;
    cudaError_t ce = cudaStreamSynchronize(nullptr);
    if (ce == cudaSuccess) ce = cudaMemcpy(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (ce != cudaSuccess) {
        so::set_global_error(std::string("so_sur_gemm: ") + cudaGetErrorString(ce));
        return SO_ERR_CUDA;
    }
    if (e) {
        so::set_global_error("so_sur_gemm: a tensor-core wait gave up");
        return SO_ERR_WATCHDOG;
    }
    return SO_OK;
}

}  // extern "C"
