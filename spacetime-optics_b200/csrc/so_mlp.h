// Ray surrogate: BF16 tcgen05 GEMM tiles and the MLP kernels built on them (sm_100a).
//
// Every GEMM here is C[M x N] = A[M x K] . B[N x K]^T with BOTH operands K-major (row-major with the
// reduction index contiguous), BF16 in, FP32 accumulated in tensor memory.  The network's three
// products map onto that one form:
//   forward        Z_l   = A_{l-1} . W_l^T          A = activations [rays x K], B = W_l [N_l x K_l]
//   input gradient dA    = dZ_l . W_l               B = W_l^T, kept as its own BF16 copy [K_l x N_l]
//   weight grad.   dW_l  = dZ_l^T . A_{l-1}         A = dZ_l^T [N_l x rays], B = A_{l-1}^T [K_l x rays]
// so the epilogues that produce activations and gradients also write their transposes.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/so_tracer.h"

namespace so {
namespace mlp {

typedef __nv_bfloat16 bf16;

enum Epilogue {
    EPI_F32 = 0,       // out_f[m, n] = acc + bias[n]
    EPI_GELU = 1,      // z = acc + bias[n]; d_out[m, n] = gelu'(z); out_b[m, n] = out_t[n, m] = gelu(z)
    EPI_GELU_BWD = 2,  // y = acc * d_in[m, n]; out_b[m, n] = out_t[n, m] = y   (all BF16)
    EPI_SPLIT = 3,     // out_f[z][m, n] = acc   (partial sums of split reductions, z = slice)
    EPI_SPLIT_T = 4,   // out_f[z][n, m] = acc
};

struct GemmArgs {
    const bf16* A;
    long lda;
    const bf16* B;
    long ldb;
    int M, N, K;
    int splits;  // the reduction is cut into `splits` slices, one CTA each (EPI_SPLIT*)
    int epi;
    const float* bias;
    float* out_f;
    long ldf;
    long split_stride;  // floats between the partial-sum planes of EPI_SPLIT*
    bf16* out_b;
    long ldob;
    bf16* out_t;
    long ldot;
    bf16* d_out;       // GELU derivative at the pre-activation, for the backward pass
    const bf16* d_in;
    long ldd;
    int* err;  // device status word: set to a nonzero code when a wait gives up
};

// Checks shapes, strides and alignment (returns a nonzero status and a message when they are not
// supported) and launches on st.  Requirements: M % 128 == 0; N <= 256 with N % 16 == 0, or
// N % 256 == 0; (K / splits) % 16 == 0; lda, ldb multiples of 8 elements; A, B 16-byte aligned.
int launch_gemm(const GemmArgs& g, cudaStream_t st, const char** why);

// tanh-form GELU and its derivative (float) from one tanh, for the training epilogue.
__host__ __device__ inline void gelu_and_grad_f(float z, float* y, float* d) {
    const float c = 0.7978845608028654f, k = 0.044715f;
    const float t = tanhf(c * (z + k * z * z * z));
    *y = 0.5f * z * (1.f + t);
    *d = 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * c * (1.f + 3.f * k * z * z);
}

// ---- network shape and parameter layout ------------------------------------------------------
constexpr int NFREQ = SO_SUR_NFREQ;     // 64 random frequencies
constexpr int NFEAT = 2 * NFREQ;        // sin and cos of each
constexpr int HID = SO_SUR_HIDDEN;      // 256
constexpr int NHID = SO_SUR_LAYERS;     // 4 hidden layers
constexpr int NOUT = SO_SUR_NOUT;       // 12 outputs
constexpr int LDO = SO_SUR_LDOUT;       // head padded to 16 rows (tensor-core N granularity)
constexpr int NLAYER = NHID + 1;        // GEMM layers including the head

// FP32 master parameters, one flat array: for each layer its weight [N x K] row-major, then its
// bias [N].  Layer 0: 256 x 128, layers 1-3: 256 x 256, head: 16 x 256 (rows 12-15 stay zero).
// Every weight starts at a multiple of 8 elements, so its BF16 copy has 16-byte aligned rows.
struct Layout {
    long w[NLAYER], b[NLAYER];
    int n[NLAYER], k[NLAYER];
    long total;
};
__host__ __device__ inline Layout param_layout() {
    Layout L{};
    long off = 0;
    for (int l = 0; l < NLAYER; ++l) {
        L.n[l] = l < NHID ? HID : LDO;
        L.k[l] = l == 0 ? NFEAT : HID;
        L.w[l] = off;
        off += (long)L.n[l] * L.k[l];
        L.b[l] = off;
        off += L.n[l];
    }
    L.total = off;
    return L;
}

// Input scaling of (alpha, beta, spin, inclination) to [-1, 1] over the training ranges.
constexpr float XY_SCALE = 12.f;   // alpha, beta in [-12, 12] M
constexpr float A_MID = 0.495f;    // spin in [0, 0.99]
constexpr float I_MID = 90.f;      // inclination in [5, 175] deg
constexpr float I_HALF = 85.f;

struct LossWeights {
    float dir, u, g;
};

// ---- kernel launchers (k_mlp.cu) ------------------------------------------------------------
// Features of rays off + i, i < rows (taken mod n when wrap, else zero inputs past n):
// X [rows x 128] row-major and, optionally, XT [128 x ldxt].
void launch_features(const so_sur_ray* rays, long off, long n, int rows, int wrap, const float* freq, bf16* X,
                     bf16* XT, long ldxt, cudaStream_t st);
// Loss of the head outputs O [rows x 16] against targets (off + i) mod n; writes dO = dL/dO (BF16,
// row-major and transposed [16 x rows]), the head-bias gradient gb[16] (FP32, before rounding) and
// adds the loss terms into acc[6] (sums of ce, dir, u, g, correct and the total).
// part_gb (rows/128 x 16 floats) and part_acc (rows/128 x 8 doubles) are scratch.
void launch_loss(const float* O, const so_sur_target* tgt, long off, long n, int rows, LossWeights w, bf16* dO,
                 bf16* dOT, float* part_gb, double* part_acc, float* gb, double* acc, cudaStream_t st);
// gb[r] = sum over c < cols of dT[r * cols + c]   (bias gradient from a transposed BF16 gradient)
void launch_rowsum(const bf16* dT, int rows, int cols, float* gb, cudaStream_t st);
// out[i] = sum_{s < splits} part[s * count + i], in slice order (deterministic split reduction)
void launch_sum_splits(const float* part, int splits, long count, float* out, cudaStream_t st);
// AdamW over the flat parameters; refreshes the BF16 weights W (same layout) and transposes WT
// (layer l at w[l], [K x N]).
void launch_adam(float* p, const float* g, float* m, float* v, long n, float lr, float b1, float b2, float eps,
                 float wd, int t, bf16* W, bf16* WT, cudaStream_t st);
// BF16 weights and transposes from the master parameters (no update).
void launch_pack(const float* p, long n, bf16* W, bf16* WT, cudaStream_t st);

// ---- fused inference (k_mlp_fused.cu) --------------------------------------------------------
// The weights of every layer cut into 64-wide K chunks, each stored as one contiguous tile in the
// tensor cores' shared-memory layout, so that one bulk copy brings a chunk in.
struct FusedChunk {
    long offset;  // bytes from the start of the packed weights
    int bytes;
    int layer, row0, rows, k0;  // the weight rows [row0, row0 + rows) x columns [k0, k0 + 64) of layer
};
constexpr int FUSED_MAX_CHUNKS = 64;
struct FusedArgs {
    const so_sur_ray* rays;
    long long n;
    float* out;            // n x LDO floats
    const float* params;   // FP32 master parameters (biases)
    long bias_off[NLAYER];
    const float* freq;     // NFREQ x 4
    const uint8_t* wpack;  // packed BF16 weights
    FusedChunk chunks[FUSED_MAX_CHUNKS];
    int nchunks;
    int* err;
};
// Fills the chunk table (in the order the kernel consumes it, at most FUSED_MAX_CHUNKS entries)
// and the packed size in elements; returns the number of chunks, or -1 if the table is too small.
int fused_chunks(FusedChunk* chunks, long* pack_elems);
// Packs the BF16 weights into the chunks of a.chunks.
void launch_pack_chunks(const bf16* W, const FusedArgs& a, bf16* wpack, cudaStream_t st);
// Persistent launch, one CTA per SM (at most one per 256-ray tile).
int launch_mlp_fused(const FusedArgs& a, int num_sms, cudaStream_t st);
// The 2-SM form (clusters of two CTAs, tcgen05.mma.cta_group::2): its chunk table has the two
// CTAs' halves of every chunk as consecutive entries.
int fused2_chunks(FusedChunk* chunks, long* pack_elems);
int launch_mlp_fused2(const FusedArgs& a, int num_sms, cudaStream_t st);

}  // namespace mlp
}  // namespace so
