// Fused surrogate inference: one persistent kernel runs the whole network for tiles of 256 rays
// with the activations resident in shared memory.
//
//   warps 0-15 (512 threads, two per ray): Fourier features of the tile into shared memory (sine
//              and cosine on the SFU after an exact reduction of the phase to one turn); after each
//              half of a layer, read the accumulators from tensor memory (tcgen05.ld), add the bias,
//              tanh-form GELU in half precision, round to BF16 and write the next layer's input in
//              place; after the head, write the 16 FP32 outputs to global memory.
//   warp 16    (one elected thread): streams the packed BF16 weights through a ring of six 16 KB
//              shared-memory buffers with bulk copies (cp.async.bulk, mbarrier transaction counts,
//              no multicast) and issues the tensor-core MMAs (tcgen05.mma, M=128, K=16, N=128 or
//              16 for the head), each weight chunk serving both 128-ray halves of the tile.
//
// Each layer is cut into output halves n0, n1 (128 columns, TMEM columns [0,128) and [128,256) of
// each ray half) and input halves k0, k1, and its four blocks run in the order (n0,k0), (n1,k0),
// (n0,k1), (n1,k1).  Then input half k0 is no longer read once n0 is complete, so the epilogue of
// n0 (which writes the next layer's k0 in place) runs while the tensor core does (n1,k1); and the
// next layer's (n0,k0) needs only that epilogue, so it runs while the epilogue of n1 does.  The
// weights are read from L2 once per tile (456 KB per 256 rays).
//
// Shared memory: 2 x 64 KB activations (K-major no-swizzle canonical layout, 128 B core matrices,
// row groups K*16 B apart) + 6 x 16 KB weight chunks = 224 KB; one CTA per SM.
//
// Every mbarrier wait is bounded (about a second); a wait that gives up sets the CTA's abort flag
// and *err = SO_ERR_WATCHDOG, every role leaves its loop, the bulk copies still in flight are waited
// for (bounded), and the TMEM columns are freed.
#include <cuda_fp16.h>

#include "so_mlp.h"

namespace so {
namespace mlp {

namespace {

constexpr int TILE = 256;      // rays per tile (two MMA halves of 128)
constexpr int NEPI = 512;      // epilogue threads (16 warps)
constexpr int NTHR = NEPI + 32;
#ifndef SO_FUSED_NBUF
#define SO_FUSED_NBUF 6
#define SO_FUSED_CHUNK_K 64
#endif
constexpr int NBUF = SO_FUSED_NBUF;        // weight ring: NBUF chunks of 128 rows x CHUNK_K
constexpr int CHUNK_K = SO_FUSED_CHUNK_K;
constexpr int CHUNK_ROWS = 128;
constexpr int CHUNK_BYTES = CHUNK_ROWS * CHUNK_K * 2;  // 16 KB
constexpr int ACT_HALF = 128 * HID * 2;          // 64 KB
constexpr int SMEM_BYTES = 2 * ACT_HALF + NBUF * CHUNK_BYTES;
constexpr unsigned long long WAIT_NS = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

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

__device__ __forceinline__ void bar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
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

// Bounded wait; false after about a second or as soon as another role has aborted.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
    if (bar_try(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (;;) {
        if (bar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (now_ns() - t0 > WAIT_NS) {
            *abort_flag = 1;
            return false;
        }
    }
}

// Bulk copy global -> shared (no multicast), completing on the mbarrier's transaction count.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
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

// Byte offset of element (row, k) in a K-major canonical tile whose rows hold K elements.
__device__ __forceinline__ uint32_t canon(int row, int k, int K) {
    return (uint32_t)((row >> 3) * (K * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// 32 accumulator columns of this warp's TMEM lanes, issued without waiting: the registers belong
// to the load until tmem_wait32 on the same array (whose "+r" operands keep the compiler from using
// them earlier).
#define SO_R32(v)                                                                                          \
    "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),        \
        "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),          \
        "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]),        \
        "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]),        \
        "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
__device__ __forceinline__ void tmem_ld32_async(uint32_t addr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : SO_R32(v)
        : "r"(addr));
}
__device__ __forceinline__ void tmem_wait32(uint32_t (&v)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : SO_R32(v)::"memory");
}
#undef SO_R32

// tanh-form GELU of a pair of pre-activations in half precision, z (c + k z^2) on the FMA pipe and
// tanh.approx.f16x2 on the SFU (one instruction per pair), returned as two packed BF16 values.
// Half precision carries 11 bits, more than the BF16 result keeps; |z| > 256 saturates the tanh
// argument to +-inf, where GELU(z) is z or 0 as it should be.
__device__ __forceinline__ uint32_t gelu2_bf16(__half2 z) {
    const __half2 p = __hfma2(__hmul2(z, z), __float2half2_rn(0.044715f * 0.7978845608028654f),
                              __float2half2_rn(0.7978845608028654f));
    const __half2 u = __hmul2(z, p);
    __half2 t;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(*reinterpret_cast<uint32_t*>(&t)) : "r"(*reinterpret_cast<const uint32_t*>(&u)));
    const __half2 half = __float2half2_rn(0.5f);
    const float2 g = __half22float2(__hmul2(z, __hfma2(t, half, half)));
    const __nv_bfloat162 b = __floats2bfloat162_rn(g.x, g.y);
    return *reinterpret_cast<const uint32_t*>(&b);
}

// Bias + GELU of 32 accumulator columns (starting at column c0) of one row, into the next layer's
// input in shared memory.
__device__ __forceinline__ void epilogue32(const uint32_t (&v)[32], const __half2* bias2, int c0, uint8_t* act_row_base,
                                           int row) {
    __align__(16) uint32_t o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const __half2 z = __hadd2(__floats2half2_rn(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1])),
                                  bias2[c0 / 2 + i]);
        o[i] = gelu2_bf16(z);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        *reinterpret_cast<uint4*>(act_row_base + canon(row, c0 + 8 * i, HID)) = reinterpret_cast<const uint4*>(o)[i];
}


__global__ void __launch_bounds__(NTHR, 1) k_mlp_fused(const FusedArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t full[NBUF], empty[NBUF], acc_ready[2], epi_done[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ __half2 bias2[NHID][HID / 2];  // hidden-layer biases in half precision
    uint8_t* act = smem;                   // two ray halves of ACT_HALF
    uint8_t* wbuf = smem + 2 * ACT_HALF;   // NBUF chunks
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long ntiles = (a.n + TILE - 1) / TILE;
    const int my_tiles = blockIdx.x < ntiles ? (int)((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) {
            bar_init(&full[b], 1);
            bar_init(&empty[b], 1);
        }
        for (int n = 0; n < 2; ++n) {
            bar_init(&acc_ready[n], 1);
            bar_init(&epi_done[n], NEPI);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < NHID * HID / 2; i += NTHR) {
        const int l = i / (HID / 2), c = i % (HID / 2);
        const float* b = a.params + a.bias_off[l] + 2 * c;
        bias2[l][c] = __floats2half2_rn(b[0], b[1]);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == NEPI / 32) {
        // ---- weight stream and MMA issue (one thread) ----
        if (lane == 0) {
            const long long total = (long long)my_tiles * a.nchunks;
            long long issued = 0, consumed = 0;
            auto load = [&](long long q) {
                const int b = (int)(q % NBUF);
                const FusedChunk& c = a.chunks[q % a.nchunks];
                bar_expect_tx(&full[b], (uint32_t)c.bytes);
                bulk_g2s(wbuf + b * CHUNK_BYTES, a.wpack + c.offset, (uint32_t)c.bytes, &full[b]);
            };
            for (; issued < total && issued < NBUF - 1; ++issued) load(issued);
            uint32_t ph_epi[2] = {0, 0};
            bool ok = true;
            // Descriptors are linear in the address (the start field holds address >> 4), so each
            // MMA's pair is a base plus a constant.
            const uint64_t wdesc = smem_desc(smem_u32(wbuf), 128, CHUNK_K * 16);
            const uint64_t adesc128 = smem_desc(smem_u32(act), 128, NFEAT * 16);
            const uint64_t adesc256 = smem_desc(smem_u32(act), 128, HID * 16);
            // block (n, kh) of a layer: its chunks in stream order, into TMEM columns n * 128
            auto block = [&](int n, int kh, int K, uint32_t idesc) -> bool {
                const int kcp = K / 2 / CHUNK_K;
                const uint64_t abase = K == NFEAT ? adesc128 : adesc256;
                for (int c = 0; c < kcp; ++c) {
                    const long long q = consumed;
                    const int b = (int)(q % NBUF);
                    if (!bar_wait(&full[b], (uint32_t)((q / NBUF) & 1), &abort_flag)) return false;
                    fence_after();
                    const uint64_t bd = wdesc + (uint64_t)(b * (CHUNK_BYTES >> 4));
                    const uint64_t ad = abase + (uint64_t)(kh * (K / 2) + c * CHUNK_K);  // (k * 16 B) >> 4
                    const uint32_t d = tmem + n * 128;
                    const uint32_t acc0 = (kh > 0 || c > 0) ? 1u : 0u;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
#pragma unroll
                        for (int j = 0; j < CHUNK_K / 16; ++j)
                            mma_bf16(d + h * 256, ad + h * (ACT_HALF >> 4) + j * 16, bd + j * 16, idesc,
                                     j > 0 ? 1u : acc0);
                    }
                    mma_commit(&empty[b]);
                    ++consumed;
                    // refill: chunk `issued` goes into the buffer of chunk issued - NBUF, the one
                    // issued just before chunk q (the tensor core still has q queued meanwhile)
                    if (issued < total) {
                        const long long prev = issued - NBUF;
                        if (prev >= 0 &&
                            !bar_wait(&empty[issued % NBUF], (uint32_t)((prev / NBUF) & 1), &abort_flag))
                            return false;
                        load(issued);
                        ++issued;
                    }
                }
                return true;
            };
            auto wait_epi = [&](int n) -> bool {
                if (!bar_wait(&epi_done[n], ph_epi[n] & 1, &abort_flag)) return false;
                ++ph_epi[n];
                fence_after();
                return true;
            };
            for (int t = 0; t < my_tiles && ok; ++t) {
                for (int l = 0; l < NLAYER && ok; ++l) {
                    const bool head = l == NHID;
                    const int K = l == 0 ? NFEAT : HID;
                    const uint32_t idesc = idesc_bf16(128, head ? LDO : 128);
                    ok = wait_epi(0) && block(0, 0, K, idesc) && wait_epi(1);
                    if (ok && !head) ok = block(1, 0, K, idesc);
                    if (ok) ok = block(0, 1, K, idesc);
                    if (ok) mma_commit(&acc_ready[0]);
                    if (ok && !head) ok = block(1, 1, K, idesc);
                    if (ok && !head) mma_commit(&acc_ready[1]);
                }
            }
            // copies still in flight land before the CTA exits
            for (long long q = consumed; q < issued; ++q) {
                volatile int never = 0;
                bar_wait(&full[q % NBUF], (uint32_t)((q / NBUF) & 1), &never);
            }
            if (!ok && a.err) atomicExch(a.err, SO_ERR_WATCHDOG);
        }
    } else {
        // ---- features and epilogues: 16 warps.  Warp w serves TMEM lanes 32 (w % 4) .. + 31 (the
        // rows it may read) of ray half w / 8, and 64 of the 128 columns of each output half
        // (group (w / 4) % 2).
        const int h = warp >> 3;
        const int cg = (warp >> 2) & 1;
        const int row = (warp & 3) * 32 + lane;  // row within the half = TMEM lane
        uint8_t* my_act = act + h * ACT_HALF;
        const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + h * 256;
        uint32_t ph_acc[2] = {0, 0};
        bool ok = true;
        auto wait_acc = [&](int n) -> bool {
            if (!bar_wait(&acc_ready[n], ph_acc[n] & 1, &abort_flag)) return false;
            ++ph_acc[n];
            fence_after();
            return true;
        };
        for (int t = 0; t < my_tiles && ok; ++t) {
            const long long tile = blockIdx.x + (long long)t * gridDim.x;
            const long long ray = tile * TILE + h * 128 + row;
            float x[4] = {0.f, 0.f, 0.f, 0.f};
            if (ray < a.n) {
                const so_sur_ray r = a.rays[ray];
                x[0] = r.alpha * (1.f / XY_SCALE);
                x[1] = r.beta * (1.f / XY_SCALE);
                x[2] = (r.spin - A_MID) * (1.f / A_MID);
                x[3] = (r.incl_deg - I_MID) * (1.f / I_HALF);
            }
            // this thread's 32 frequencies: sin into columns j, cos into 64 + j
            for (int j0 = cg * 32; j0 < cg * 32 + 32; j0 += 8) {
                __align__(16) bf16 sv[8], cv[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float4 fj = __ldg(reinterpret_cast<const float4*>(a.freq) + j0 + q);
                    const float turns = fmaf(fj.w, x[3], fmaf(fj.z, x[2], fmaf(fj.y, x[1], fj.x * x[0])));
                    const float rr = 6.283185307179586f * (turns - rintf(turns));  // in [-pi, pi]
                    sv[q] = __float2bfloat16_rn(__sinf(rr));
                    cv[q] = __float2bfloat16_rn(__cosf(rr));
                }
                *reinterpret_cast<uint4*>(my_act + canon(row, j0, NFEAT)) = *reinterpret_cast<const uint4*>(sv);
                *reinterpret_cast<uint4*>(my_act + canon(row, NFREQ + j0, NFEAT)) = *reinterpret_cast<const uint4*>(cv);
            }
            fence_async_smem();
            bar_arrive(&epi_done[0]);
            bar_arrive(&epi_done[1]);
            for (int l = 0; l < NHID && ok; ++l) {
                for (int n = 0; n < 2 && ok; ++n) {
                    if (!wait_acc(n)) {
                        ok = false;
                        break;
                    }
                    // 64 columns: the second load is in flight while the first 32 are processed
                    const int c0 = n * 128 + cg * 64;
                    uint32_t va[32], vb[32];
                    tmem_ld32_async(lane_addr + c0, va);
                    tmem_wait32(va);
                    tmem_ld32_async(lane_addr + c0 + 32, vb);
                    epilogue32(va, bias2[l], c0, my_act, row);
                    tmem_wait32(vb);
                    epilogue32(vb, bias2[l], c0 + 32, my_act, row);
                    fence_before();
                    fence_async_smem();
                    bar_arrive(&epi_done[n]);
                }
            }
            if (!ok || !wait_acc(0)) {
                ok = false;
                break;
            }
            float f[16];
            tmem_ld16(lane_addr, f);
            fence_before();
            if (cg == 0 && ray < a.n) {
                const float* bias = a.params + a.bias_off[NHID];
                float4* o = reinterpret_cast<float4*>(a.out + ray * LDO);
                const float4* b4 = reinterpret_cast<const float4*>(bias);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float4 b = __ldg(b4 + i);
                    o[i] = make_float4(f[4 * i] + b.x, f[4 * i + 1] + b.y, f[4 * i + 2] + b.z, f[4 * i + 3] + b.w);
                }
            }
        }
        if (!ok && a.err && tid == 0) atomicExch(a.err, SO_ERR_WATCHDOG);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// ==== 2-SM form (cta_group::2) ==================================================================
// A cluster of two CTAs on two SMs runs pairs of 256-ray tiles T0, T1; each CTA holds its 128 rays
// of both tiles (activations 2 x 64 KB) and its half of every weight chunk (N/2 weight rows).  One
// tcgen05.mma.cta_group::2 (M = 256, N = 256, K = 16), issued by the leader CTA, multiplies both
// CTAs' rows by both halves of the weights; each CTA's TMEM receives its own rows (all 256
// columns).  Per SM that is 8 KB of shared-memory operands per 128 tensor cycles, half of the 1-SM
// form's share.  The tiles alternate on the tensor core, layer by layer (T0 layer l, T1 layer l,
// T0 layer l+1, ...), so each tile's epilogue runs while the other tile's MMAs do, and each weight
// chunk serves both tiles before its buffer is refilled.
//
// Cross-CTA hand-offs (bounded polls everywhere):
//   weights   each CTA bulk-copies its half-chunk into its own ring slot; the leader's `full`
//             barrier counts its own transaction bytes plus one arrival that the second CTA's
//             control thread forwards (remote mbarrier arrive) once its half has landed;
//   buffers   the leader's commit after a chunk's last use (tile T1) arrives on `empty` in both CTAs;
//   MMA done  the commit after a tile's last chunk arrives on `acc` in both CTAs;
//   epilogue  each CTA's 512 epilogue threads arrive on its local `epi_done`; the second CTA's
//             control thread forwards each completion to the leader's `epi_pair`.
constexpr int F2_RAYS = 512;   // rays per pair iteration (2 tiles x 256, 128 per CTA per tile)
constexpr int F2_NBUF = 6;     // weight ring slots of 16 KB
constexpr int F2_SLOT = 128 * CHUNK_K * 2;
constexpr int F2_SMEM = 2 * ACT_HALF + F2_NBUF * F2_SLOT;
constexpr int F2_CHUNKS = 2 + 3 * 4 + 4;  // weight chunks per iteration (K = 64 slices)

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void remote_arrive(uint64_t* bar, uint32_t rank) {
    asm volatile(
        "{\n\t.reg .b32 ra;\n\t"
        "mapa.shared::cluster.u32 ra, %0, %1;\n\t"
        "mbarrier.arrive.release.cluster.shared::cluster.b64 _, [ra];\n\t}\n" ::"r"(smem_u32(bar)),
        "r"(rank)
        : "memory");
}
// Non-blocking phase tests for the control threads' polling loops (try_wait may suspend the thread
// for a while, which would hold up the other events it serves).
__device__ __forceinline__ bool bar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.test_wait.parity.acquire.cta.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool bar_test_cluster(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void mma2_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z),
          "r"(z));
}
__device__ __forceinline__ void commit2_both(uint64_t* bar) {
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(mask)
        : "memory");
}
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
}

// Chunk c (K slice of 64) of layer l within an iteration: its index in the iteration's stream.
__device__ __forceinline__ int f2_chunk_index(int l, int c) { return l == 0 ? c : 2 + (l - 1) * 4 + c; }

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NTHR, 1) k_mlp_fused2(const FusedArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t full[F2_NBUF], empty[F2_NBUF], acc[2], epi_done[2], epi_pair[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ __half2 bias2[NHID][HID / 2];
    uint8_t* act = smem;                   // tiles T0, T1: this CTA's 128 rows each
    uint8_t* wbuf = smem + 2 * ACT_HALF;   // F2_NBUF half-chunks
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_rank();
    const int cluster = blockIdx.x >> 1, nclusters = gridDim.x >> 1;
    const long long iters = (a.n + F2_RAYS - 1) / F2_RAYS;
    const int my_iters = cluster < iters ? (int)((iters - 1 - cluster) / nclusters + 1) : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int b = 0; b < F2_NBUF; ++b) {
            bar_init(&full[b], rank == 0 ? 2 : 1);
            bar_init(&empty[b], 1);
        }
        for (int t = 0; t < 2; ++t) {
            bar_init(&acc[t], 1);
            bar_init(&epi_done[t], NEPI);
            bar_init(&epi_pair[t], 1);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < NHID * HID / 2; i += NTHR) {
        const int l = i / (HID / 2), c = i % (HID / 2);
        const float* b = a.params + a.bias_off[l] + 2 * c;
        bias2[l][c] = __floats2half2_rn(b[0], b[1]);
    }
    fence_before();
    __syncthreads();
    cluster_sync();  // both CTAs' barriers exist before any remote arrive
    fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == NEPI / 32) {
        if (lane == 0) {
            // ---- control thread: weight loads of this CTA's halves; MMAs (leader) or forwarding ----
            const long long total = (long long)my_iters * F2_CHUNKS;
            const long long total_steps = (long long)my_iters * 2 * F2_CHUNKS;  // each chunk serves T0 and T1
            long long issued = 0, step = 0, fwd = 0;
            long long efwd[2] = {0, 0}, ecnt[2] = {0, 0};
            const long long total_epi = (long long)my_iters * NLAYER;
            bool ok = true;
            const uint64_t wdesc = smem_desc(smem_u32(wbuf), 128, CHUNK_K * 16);
            const uint64_t adesc128 = smem_desc(smem_u32(act), 128, NFEAT * 16);
            const uint64_t adesc256 = smem_desc(smem_u32(act), 128, HID * 16);
            // deadline on the SM clock (cheap to read, unlike %globaltimer): ~2 s without progress
            long long t_last = clock64();
            for (;;) {
                bool progress = false;
                // 1. next weight load into its ring slot once the slot's previous chunk is released
                if (issued < total) {
                    const int b = (int)(issued % F2_NBUF);
                    if (issued < F2_NBUF || bar_test(&empty[b], (uint32_t)(((issued / F2_NBUF) - 1) & 1))) {
                        const FusedChunk& c = a.chunks[2 * (issued % F2_CHUNKS) + rank];
                        bar_expect_tx(&full[b], (uint32_t)c.bytes);
                        bulk_g2s(wbuf + b * F2_SLOT, a.wpack + c.offset, (uint32_t)c.bytes, &full[b]);
                        ++issued;
                        progress = true;
                    }
                }
                if (rank == 0) {
                    // 2. next MMA step: iteration, layer, tile, chunk in the schedule's order
                    if (step < total_steps) {
                        const long long it = step / (2 * F2_CHUNKS);
                        int r = (int)(step % (2 * F2_CHUNKS));
                        int l = 0, c = 0, T = 0;
                        for (l = 0; l < NLAYER; ++l) {  // per layer: T0's chunks, then T1's
                            const int kc = (l == 0 ? NFEAT : HID) / CHUNK_K;
                            if (r < 2 * kc) {
                                T = r / kc;
                                c = r % kc;
                                break;
                            }
                            r -= 2 * kc;
                        }
                        const long long q = it * F2_CHUNKS + f2_chunk_index(l, c);
                        const int b = (int)(q % F2_NBUF);
                        bool ready = true;
                        if (c == 0)  // the tile's input (features or the previous epilogue) in both CTAs
                            ready = bar_test(&epi_done[T], (uint32_t)(ecnt[T] & 1)) &&
                                    bar_test_cluster(&epi_pair[T], (uint32_t)(ecnt[T] & 1));
                        ready = ready && bar_test_cluster(&full[b], (uint32_t)((q / F2_NBUF) & 1));
                        if (ready) {
                            if (c == 0) ++ecnt[T];
                            fence_after();
                            const bool head = l == NHID;
                            const int K = l == 0 ? NFEAT : HID;
                            const uint32_t idesc = idesc_bf16(256, head ? LDO : HID);
                            const uint64_t ad = (K == NFEAT ? adesc128 : adesc256) + (uint64_t)(T * (ACT_HALF >> 4)) +
                                                (uint64_t)(c * CHUNK_K);
                            const uint64_t bd = wdesc + (uint64_t)(b * (F2_SLOT >> 4));
#pragma unroll
                            for (int j = 0; j < CHUNK_K / 16; ++j)
                                mma2_bf16(tmem + T * 256, ad + j * 16, bd + j * 16, idesc, (c > 0 || j > 0) ? 1u : 0u);
                            if (T == 1) commit2_both(&empty[b]);        // chunk done with: release its slot
                            if (c == K / CHUNK_K - 1) commit2_both(&acc[T]);  // the tile's layer is done
                            ++step;
                            progress = true;
                        }
                    }
                } else {
                    // 2'. forward this CTA's landed weight halves and finished epilogues to the leader
                    if (fwd < issued && bar_test(&full[fwd % F2_NBUF], (uint32_t)((fwd / F2_NBUF) & 1))) {
                        remote_arrive(&full[fwd % F2_NBUF], 0);
                        ++fwd;
                        progress = true;
                    }
                    for (int T = 0; T < 2; ++T)
                        if (efwd[T] < total_epi && bar_test(&epi_done[T], (uint32_t)(efwd[T] & 1))) {
                            remote_arrive(&epi_pair[T], 0);
                            ++efwd[T];
                            progress = true;
                        }
                }
                const bool done = issued == total &&
                                  (rank == 0 ? step == total_steps : (fwd == total && efwd[0] == total_epi && efwd[1] == total_epi));
                if (done) break;
                const long long t = clock64();
                if (progress) t_last = t;
                else if (abort_flag || t - t_last > 4000000000ll) {
                    abort_flag = 1;
                    ok = false;
                    break;
                }
            }
            if (!ok) {  // let copies in flight land before the CTA can exit
                const unsigned long long t0 = now_ns();
                while (now_ns() - t0 < 20000ull) {
                }
                if (a.err) atomicExch(a.err, SO_ERR_WATCHDOG);
            }
        }
    } else {
        // ---- features and epilogues: 16 warps.  Warp w serves TMEM lanes 32 (w % 4) .. + 31 of
        // this CTA's 128 rows; for features it takes tile w / 8 and half the frequencies
        // ((w / 4) % 2), for epilogues 64 of the 256 columns (w / 4) of the current tile.
        const int q4 = warp & 3, cg = warp >> 2;
        const int row = q4 * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(q4 * 32) << 16);
        uint32_t acnt[2] = {0, 0};
        bool ok = true;
        auto wait_acc = [&](int T) -> bool {
            if (!bar_wait(&acc[T], acnt[T] & 1, &abort_flag)) return false;
            ++acnt[T];
            fence_after();
            return true;
        };
        for (int t = 0; t < my_iters && ok; ++t) {
            const long long it = cluster + (long long)t * nclusters;
            {   // features of both tiles
                const int T = warp >> 3, half = (warp >> 2) & 1;
                const long long ray = it * F2_RAYS + T * 256 + rank * 128 + row;
                float x[4] = {0.f, 0.f, 0.f, 0.f};
                if (ray < a.n) {
                    const so_sur_ray r = a.rays[ray];
                    x[0] = r.alpha * (1.f / XY_SCALE);
                    x[1] = r.beta * (1.f / XY_SCALE);
                    x[2] = (r.spin - A_MID) * (1.f / A_MID);
                    x[3] = (r.incl_deg - I_MID) * (1.f / I_HALF);
                }
                uint8_t* my_act = act + T * ACT_HALF;
                for (int j0 = half * 32; j0 < half * 32 + 32; j0 += 8) {
                    __align__(16) bf16 sv[8], cv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const float4 fj = __ldg(reinterpret_cast<const float4*>(a.freq) + j0 + q);
                        const float turns = fmaf(fj.w, x[3], fmaf(fj.z, x[2], fmaf(fj.y, x[1], fj.x * x[0])));
                        const float rr = 6.283185307179586f * (turns - rintf(turns));
                        sv[q] = __float2bfloat16_rn(__sinf(rr));
                        cv[q] = __float2bfloat16_rn(__cosf(rr));
                    }
                    *reinterpret_cast<uint4*>(my_act + canon(row, j0, NFEAT)) = *reinterpret_cast<const uint4*>(sv);
                    *reinterpret_cast<uint4*>(my_act + canon(row, NFREQ + j0, NFEAT)) = *reinterpret_cast<const uint4*>(cv);
                }
            }
            fence_async_smem();
            bar_arrive(&epi_done[0]);
            bar_arrive(&epi_done[1]);
            for (int l = 0; l < NHID && ok; ++l) {
                for (int T = 0; T < 2 && ok; ++T) {
                    if (!wait_acc(T)) {
                        ok = false;
                        break;
                    }
                    uint8_t* my_act = act + T * ACT_HALF;
                    const int c0 = cg * 64;
                    uint32_t va[32], vb[32];
                    tmem_ld32_async(lane_base + T * 256 + c0, va);
                    tmem_wait32(va);
                    tmem_ld32_async(lane_base + T * 256 + c0 + 32, vb);
                    epilogue32(va, bias2[l], c0, my_act, row);
                    tmem_wait32(vb);
                    epilogue32(vb, bias2[l], c0 + 32, my_act, row);
                    fence_before();
                    fence_async_smem();
                    bar_arrive(&epi_done[T]);
                }
            }
            for (int T = 0; T < 2 && ok; ++T) {  // head
                if (!wait_acc(T)) {
                    ok = false;
                    break;
                }
                float f[16];
                tmem_ld16(lane_base + T * 256, f);
                fence_before();
                const long long ray = it * F2_RAYS + T * 256 + rank * 128 + row;
                if (cg == 0 && ray < a.n) {
                    float4* o = reinterpret_cast<float4*>(a.out + ray * LDO);
                    const float4* b4 = reinterpret_cast<const float4*>(a.params + a.bias_off[NHID]);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const float4 b = __ldg(b4 + i);
                        o[i] = make_float4(f[4 * i] + b.x, f[4 * i + 1] + b.y, f[4 * i + 2] + b.z, f[4 * i + 3] + b.w);
                    }
                }
            }
        }
        if (!ok && a.err && tid == 0) atomicExch(a.err, SO_ERR_WATCHDOG);
    }
    fence_before();
    __syncthreads();
    cluster_sync();  // the leader's last MMAs read this CTA's shared memory and write its TMEM
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// Pack the BF16 weights (row-major [N x K] per layer, flat layout) into the chunks of the table,
// each a [rows x 64] tile in the canonical layout (row groups 1024 B apart, K core matrices 128 B
// apart), in the order the kernel consumes them.
__global__ void k_pack_chunks(const bf16* __restrict__ W, const FusedArgs a, bf16* __restrict__ wpack) {
    const Layout L = param_layout();
    for (int q = 0; q < a.nchunks; ++q) {
        const FusedChunk& c = a.chunks[q];
        const int K = L.k[c.layer];
        const int count = c.rows * CHUNK_K;
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
            const int rr = e / CHUNK_K, kk = e % CHUNK_K;
            const bf16 v = W[L.w[c.layer] + (long)(c.row0 + rr) * K + c.k0 + kk];
            wpack[c.offset / 2 + canon(rr, kk, CHUNK_K) / 2] = v;
        }
    }
}

}  // namespace

int fused_chunks(FusedChunk* chunks, long* pack_elems) {
    const Layout L = param_layout();
    int q = 0;
    long off = 0;
    auto add = [&](int l, int row0, int rows, int k0) {
        if (q >= FUSED_MAX_CHUNKS) {
            q = FUSED_MAX_CHUNKS + 1;
            return;
        }
        chunks[q].offset = off;
        chunks[q].bytes = rows * CHUNK_K * 2;
        chunks[q].layer = l;
        chunks[q].row0 = row0;
        chunks[q].rows = rows;
        chunks[q].k0 = k0;
        off += chunks[q].bytes;
        ++q;
    };
    for (int l = 0; l < NLAYER; ++l) {
        const int K = L.k[l], kcp = K / 2 / CHUNK_K;
        const bool head = l == NHID;
        const int rows = head ? LDO : CHUNK_ROWS;
        // blocks (n0,k0), (n1,k0), (n0,k1), (n1,k1); the head has n0 only
        const int order[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
        for (int bi = 0; bi < 4; ++bi) {
            const int n = order[bi][0], kh = order[bi][1];
            if (head && n == 1) continue;
            for (int c = 0; c < kcp; ++c) add(l, n * CHUNK_ROWS, rows, kh * (K / 2) + c * CHUNK_K);
        }
    }
    *pack_elems = off / 2;
    return q > FUSED_MAX_CHUNKS ? -1 : q;
}

int fused2_chunks(FusedChunk* chunks, long* pack_elems) {
    const Layout L = param_layout();
    int q = 0;
    long off = 0;
    for (int l = 0; l < NLAYER; ++l) {
        const int K = L.k[l], N = L.n[l];
        for (int c = 0; c < K / CHUNK_K; ++c)
            for (int h = 0; h < 2; ++h) {  // the two CTAs' halves of the weight rows
                if (q >= FUSED_MAX_CHUNKS) return -1;
                chunks[q].offset = off;
                chunks[q].bytes = (N / 2) * CHUNK_K * 2;
                chunks[q].layer = l;
                chunks[q].row0 = h * (N / 2);
                chunks[q].rows = N / 2;
                chunks[q].k0 = c * CHUNK_K;
                off += chunks[q].bytes;
                ++q;
            }
    }
    *pack_elems = off / 2;
    return q;
}

int launch_mlp_fused2(const FusedArgs& a, int num_sms, cudaStream_t st) {
    if (a.n <= 0) return SO_OK;
    if (cudaFuncSetAttribute(k_mlp_fused2, cudaFuncAttributeMaxDynamicSharedMemorySize, F2_SMEM) != cudaSuccess)
        return SO_ERR_CUDA;
    const long long iters = (a.n + F2_RAYS - 1) / F2_RAYS;
    const int clusters = (int)(iters < num_sms / 2 ? iters : num_sms / 2);
    k_mlp_fused2<<<2 * clusters, NTHR, F2_SMEM, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? SO_OK : SO_ERR_CUDA;
}

void launch_pack_chunks(const bf16* W, const FusedArgs& a, bf16* wpack, cudaStream_t st) {
    k_pack_chunks<<<64, 256, 0, st>>>(W, a, wpack);
}
int launch_mlp_fused(const FusedArgs& a, int num_sms, cudaStream_t st) {
    if (a.n <= 0) return SO_OK;
    if (cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) != cudaSuccess)
        return SO_ERR_CUDA;
    const long long ntiles = (a.n + TILE - 1) / TILE;
    const int grid = (int)(ntiles < num_sms ? ntiles : num_sms);
    k_mlp_fused<<<grid, NTHR, SMEM_BYTES, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? SO_OK : SO_ERR_CUDA;
}

}  // namespace mlp
}  // namespace so
