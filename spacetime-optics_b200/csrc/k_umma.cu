// BF16 GEMM tile on the fifth-generation tensor cores: tcgen05.mma with both operands in shared
// memory and the FP32 accumulator in tensor memory (TMEM), read back with tcgen05.ld for the
// epilogue.  One CTA of 128 threads owns a 128 x BN output tile (BN <= 256 TMEM columns):
//   * all threads stage A and B K-slices into shared memory (a ring of four, cp.async), in the K-major
//     no-swizzle canonical layout: an 8-row x 16-byte "core matrix" is 128 contiguous bytes, the
//     K-neighbouring core matrices of one 8-row group sit 128 B apart (leading byte offset) and the
//     8-row groups BK*16 B apart (stride byte offset);
//   * thread 0 issues BK/16 tcgen05.mma (M=128, N=BN, K=16) per slice and commits them to the
//     slice's mbarrier, so three slices load while the tensor core works on one;
//   * after the last commit every warp reads its 32 TMEM lanes (= 32 output rows) with tcgen05.ld
//     and applies the epilogue.
// Every mbarrier wait is bounded (about one second of %globaltimer); a wait that gives up writes
// SO_ERR_WATCHDOG into *err, skips the epilogue and still frees the TMEM columns.
#include "so_mlp.h"

namespace so {
namespace mlp {

namespace {

constexpr int BM = 128;
constexpr int NT = 128;  // threads per CTA
constexpr int NS = 4;    // K-slices in the shared-memory ring
constexpr unsigned long long WAIT_NS = 1000000000ull;
// shared tiles of the epilogue: bf16 [128][40] x 2 + bf16 [32][136] (or fp32 [128][36]), after the
// [128][BN + 8] derivative tile of the backward epilogue
constexpr int EPI_SMEM = BM * 40 * 2 * 2 + 32 * 136 * 2;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Shared-memory matrix descriptor (sm_100 format: version 1, no swizzle, base offset 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16 (bits 7-9, 10-12 = 1),
// both K-major (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool bar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of phase `parity`; false after about a second.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
    if (bar_try(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (;;) {
        if (bar_try(bar, parity)) return true;
        if (now_ns() - t0 > WAIT_NS) return false;
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* f) {
    uint32_t v[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = __uint_as_float(v[i]);
}

// Stage rows [0, rows) x K-slice [k0, k0 + BK) of a K-major global matrix into the canonical
// layout with asynchronous 16-byte copies (cp.async, L2 only).  One item moves 32 bytes (two
// core-matrix rows along K); a warp's 32 items cover 8 rows x 4 K-pairs, so the shared-memory
// side touches every bank once per 128 bytes.
__device__ __forceinline__ void stage_async(uint8_t* sm, const bf16* g, long ld, int rows, int k0, int BK, int tid) {
    const int nkq = BK >> 4;
    const int items = rows * nkq;
    for (int w = tid; w < items; w += NT) {
        const int rr = w & 7, kq = (w >> 3) % nkq, rg = (w >> 3) / nkq;
        const bf16* src = g + (long)(rg * 8 + rr) * ld + k0 + kq * 16;
        const uint32_t dst = smem_u32(sm + rg * (BK * 16) + kq * 256 + rr * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 128), "l"(src + 8) : "memory");
    }
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int EPI>
__global__ void __launch_bounds__(NT) k_gemm_bf16(GemmArgs g, int BN, int BK, int tmem_cols) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bars[NS];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int kps = g.K / g.splits, kbeg = blockIdx.z * kps;
    const int nk = kps / BK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int b = 0; b < NS; ++b) bar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(BM, BN);
    bool ok = true;

    // NS-slice ring: slices s+1 .. s+NS-1 are in flight while the tensor core works on slice s.
    const int slice = (BM + BN) * BK * 2;
    auto load = [&](int sl) {
        uint8_t* sa = smem + (sl % NS) * slice;
        const int k0 = kbeg + sl * BK;
        stage_async(sa, g.A + (long)m0 * g.lda, g.lda, BM, k0, BK, tid);
        stage_async(sa + BM * BK * 2, g.B + (long)n0 * g.ldb, g.ldb, BN, k0, BK, tid);
    };
    for (int sl = 0; sl < NS - 1; ++sl) {
        if (sl < nk) load(sl);
        cp_commit();
    }
    for (int s = 0; s < nk; ++s) {
        cp_wait<NS - 2>();  // this thread's copies of slice s have landed
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            fence_after();
            const uint32_t a0 = smem_u32(smem + (s % NS) * slice), b0 = a0 + BM * BK * 2;
            for (int j = 0; j < (BK >> 4); ++j) {
                const uint64_t da = smem_desc(a0 + j * 256, 128, BK * 16);
                const uint64_t db = smem_desc(b0 + j * 256, 128, BK * 16);
                mma_bf16(tmem, da, db, idesc, (s > 0 || j > 0) ? 1u : 0u);
            }
            mma_commit(&bars[s % NS]);
        }
        // slice s + NS - 1 goes into the buffer of slice s - 1 once that slice's MMAs are done; the
        // verdict is block-uniform so that no thread leaves the loop alone
        const int sn = s + NS - 1;
        const bool freed = sn >= nk || s < 1 || bar_wait(&bars[(s - 1) % NS], ((s - 1) / NS) & 1);
        if (!__syncthreads_and(freed)) {
            ok = false;
            break;
        }
        if (sn < nk) load(sn);
        cp_commit();
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // The last commit tracks every MMA issued before it.
    if (ok && nk > 0) ok = bar_wait(&bars[(nk - 1) % NS], ((nk - 1) / NS) & 1);
    ok = __syncthreads_and(ok);
    fence_after();

    if (ok) {
        // Epilogue in column blocks of cb = 32 (16 for a 16-wide tile), staged through shared memory
        // (the K-slice buffers are free now): each thread takes its row's accumulators from TMEM
        // (its TMEM lane), the values go to small shared tiles, and the block then stores whole
        // 16-byte row segments -- or, for the transposed outputs, whole column segments -- so every
        // global store instruction of a warp writes contiguous 128-byte lines.
        const int r = warp * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        uint8_t* ep = smem;
        bf16* TD = nullptr;  // GELU_BWD: the tile's derivatives, [128][BN + 8]
        if (EPI == EPI_GELU_BWD) {
            TD = reinterpret_cast<bf16*>(ep);
            const int segs = BN / 8;
            for (int w = tid; w < BM * segs; w += NT) {
                const int rr = w / segs, sg = w % segs;
                const uint32_t dst = smem_u32(TD + rr * (BN + 8) + 8 * sg);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst),
                             "l"(g.d_in + (long)(m0 + rr) * g.ldd + n0 + 8 * sg)
                             : "memory");
            }
            cp_commit();
            ep += BM * (BN + 8) * 2;
        }
        float* T32 = reinterpret_cast<float*>(ep);                // [128][36] fp32 (F32, SPLIT)
        bf16* T16 = reinterpret_cast<bf16*>(ep);                  // [128][40] bf16, row-major
        bf16* TG = T16 + BM * 40;                                 // [128][40] bf16, derivatives
        bf16* TT = TG + BM * 40;                                  // [32][136] bf16, transposed
        if (EPI == EPI_GELU_BWD) {
            cp_wait<0>();
            __syncthreads();
        }
        const int cb = BN < 32 ? BN : 32;
        for (int c = 0; c < BN; c += cb) {
            const int n = n0 + c;
            for (int h = 0; h < cb; h += 16) {
                float f[16];
                tmem_ld16(lane_addr + c + h, f);
                if (EPI == EPI_F32 || EPI == EPI_SPLIT) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) f[i] += (EPI == EPI_F32 && g.bias) ? g.bias[n + h + i] : 0.f;
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        *reinterpret_cast<float4*>(T32 + r * 36 + h + 4 * i) =
                            make_float4(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
                } else if (EPI == EPI_SPLIT_T) {  // column-major target: rows of a warp are contiguous
                    float* o = g.out_f + blockIdx.z * g.split_stride;
#pragma unroll
                    for (int i = 0; i < 16; ++i) o[(long)(n + h + i) * g.ldf + m0 + r] = f[i];
                } else {
                    __align__(16) bf16 o16[16], d16[16];
                    if (EPI == EPI_GELU_BWD) {
                        const uint4* src = reinterpret_cast<const uint4*>(TD + r * (BN + 8) + c + h);
                        *reinterpret_cast<uint4*>(d16) = src[0];
                        *reinterpret_cast<uint4*>(d16 + 8) = src[1];
                    }
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        float y;
                        if (EPI == EPI_GELU) {
                            float d;
                            gelu_and_grad_f(f[i] + (g.bias ? g.bias[n + h + i] : 0.f), &y, &d);
                            d16[i] = __float2bfloat16_rn(d);
                        } else {
                            y = f[i] * __bfloat162float(d16[i]);
                        }
                        o16[i] = __float2bfloat16_rn(y);
                        TT[(h + i) * 136 + r] = o16[i];
                    }
                    *reinterpret_cast<uint4*>(T16 + r * 40 + h) = reinterpret_cast<const uint4*>(o16)[0];
                    *reinterpret_cast<uint4*>(T16 + r * 40 + h + 8) = reinterpret_cast<const uint4*>(o16)[1];
                    if (EPI == EPI_GELU) {
                        *reinterpret_cast<uint4*>(TG + r * 40 + h) = reinterpret_cast<const uint4*>(d16)[0];
                        *reinterpret_cast<uint4*>(TG + r * 40 + h + 8) = reinterpret_cast<const uint4*>(d16)[1];
                    }
                }
            }
            __syncthreads();
            if (EPI == EPI_F32 || EPI == EPI_SPLIT) {
                float* base = g.out_f + (EPI == EPI_SPLIT ? blockIdx.z * g.split_stride : 0);
                const int segs = cb / 4;
                for (int w = tid; w < BM * segs; w += NT) {
                    const int rr = w / segs, sg = w % segs;
                    *reinterpret_cast<float4*>(base + (long)(m0 + rr) * g.ldf + n + 4 * sg) =
                        *reinterpret_cast<const float4*>(T32 + rr * 36 + 4 * sg);
                }
            }
            if (EPI == EPI_GELU || EPI == EPI_GELU_BWD) {
                const int segs = cb / 8;
                for (int w = tid; w < BM * segs; w += NT) {
                    const int rr = w / segs, sg = w % segs;
                    if (g.out_b)
                        *reinterpret_cast<uint4*>(g.out_b + (long)(m0 + rr) * g.ldob + n + 8 * sg) =
                            *reinterpret_cast<const uint4*>(T16 + rr * 40 + 8 * sg);
                    if (EPI == EPI_GELU && g.d_out)
                        *reinterpret_cast<uint4*>(g.d_out + (long)(m0 + rr) * g.ldd + n + 8 * sg) =
                            *reinterpret_cast<const uint4*>(TG + rr * 40 + 8 * sg);
                }
                if (g.out_t) {
                    for (int w = tid; w < cb * (BM / 8); w += NT) {
                        const int j = w / (BM / 8), sg = w % (BM / 8);
                        *reinterpret_cast<uint4*>(g.out_t + (long)(n + j) * g.ldot + m0 + 8 * sg) =
                            *reinterpret_cast<const uint4*>(TT + j * 136 + 8 * sg);
                    }
                }
            }
            __syncthreads();
        }
    } else if (tid == 0 && g.err) {
        atomicExch(g.err, SO_ERR_WATCHDOG);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
    }
}

template <int EPI>
int launch_epi(const GemmArgs& g, int BN, int BK, cudaStream_t st) {
    const int stage_bytes = NS * (BM + BN) * BK * 2;
    const int epi_bytes = EPI_SMEM + (EPI == EPI_GELU_BWD ? BM * (BN + 8) * 2 : 0);
    const int smem = stage_bytes > epi_bytes ? stage_bytes : epi_bytes;
    const int cols = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
    if (cudaFuncSetAttribute(k_gemm_bf16<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return SO_ERR_CUDA;
    dim3 grid(g.M / BM, g.N / BN, g.splits);
    k_gemm_bf16<EPI><<<grid, NT, smem, st>>>(g, BN, BK, cols);
    return cudaGetLastError() == cudaSuccess ? SO_OK : SO_ERR_CUDA;
}

bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

int launch_gemm(const GemmArgs& g, cudaStream_t st, const char** why) {
    auto bad = [&](const char* m) {
        if (why) *why = m;
        return SO_ERR_ARG;
    };
    if (!g.A || !g.B) return bad("gemm: null operand");
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.splits <= 0) return bad("gemm: empty shape");
    if (g.M % BM) return bad("gemm: M must be a multiple of 128");
    int BN;
    if (g.N <= 256) {
        if (g.N % 16) return bad("gemm: N <= 256 must be a multiple of 16");
        BN = g.N;
    } else {
        if (g.N % 256) return bad("gemm: N > 256 must be a multiple of 256");
        BN = 256;
    }
    // small grids (the split weight-gradient products): 128-wide tiles for twice the CTAs
    if (BN == 256 && (long)(g.M / BM) * (g.N / BN) * g.splits < 148) BN = 128;
    if (g.K % g.splits) return bad("gemm: K must divide into the splits");
    const int kps = g.K / g.splits;
    if (kps % 16) return bad("gemm: K per split must be a multiple of 16");
    const int BK = (kps % 32 == 0) ? 32 : 16;  // four 32-wide slices: 96 KB, two CTAs per SM
    if (g.lda % 8 || g.ldb % 8 || g.lda < g.K || g.ldb < g.K || !al16(g.A) || !al16(g.B))
        return bad("gemm: operands need 16-byte aligned rows");
    if (g.splits > 1 && g.epi != EPI_SPLIT && g.epi != EPI_SPLIT_T) return bad("gemm: split reductions need a split epilogue");
    switch (g.epi) {
        case EPI_F32:
            if (!g.out_f || g.ldf < g.N || g.ldf % 4 || !al16(g.out_f))
                return bad("gemm: EPI_F32 needs out_f with 16-byte aligned rows");
            return launch_epi<EPI_F32>(g, BN, BK, st);
        case EPI_GELU:
            if ((!g.out_b && !g.out_t) || (g.out_b && (g.ldob % 8 || g.ldob < g.N || !al16(g.out_b))) ||
                (g.out_t && (g.ldot < g.M || g.ldot % 8 || !al16(g.out_t))) ||
                (g.d_out && (g.ldd < g.N || g.ldd % 8 || !al16(g.d_out))))
                return bad("gemm: EPI_GELU outputs need 16-byte aligned rows");
            return launch_epi<EPI_GELU>(g, BN, BK, st);
        case EPI_GELU_BWD:
            if (!g.d_in || g.ldd < g.N || g.ldd % 8 || !al16(g.d_in) || (!g.out_b && !g.out_t) ||
                (g.out_b && (g.ldob % 8 || g.ldob < g.N || !al16(g.out_b))) ||
                (g.out_t && (g.ldot < g.M || g.ldot % 8 || !al16(g.out_t))))
                return bad("gemm: EPI_GELU_BWD operands need 16-byte aligned rows");
            return launch_epi<EPI_GELU_BWD>(g, BN, BK, st);
        case EPI_SPLIT:
            if (!g.out_f || g.ldf < g.N || g.ldf % 4 || !al16(g.out_f) ||
                (g.splits > 1 && g.split_stride < (long)g.M * g.ldf) || g.split_stride % 4)
                return bad("gemm: EPI_SPLIT needs out_f with 16-byte aligned rows and disjoint planes");
            return launch_epi<EPI_SPLIT>(g, BN, BK, st);
        case EPI_SPLIT_T:
            if (!g.out_f || g.ldf < g.M || (g.splits > 1 && g.split_stride < (long)g.N * g.ldf))
                return bad("gemm: EPI_SPLIT_T needs out_f with disjoint planes");
            return launch_epi<EPI_SPLIT_T>(g, BN, BK, st);
        default:
            return bad("gemm: unknown epilogue");
    }
}

}  // namespace mlp
}  // namespace so
