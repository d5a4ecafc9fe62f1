// umma_gemm.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05) for sm_100a.
//
//   C[m][n] = sum_k A[m][k] B[n][k]        (A, B row-major bf16, both K-major)
//
// followed by a fused epilogue (bias, GELU, GELU backward, FP32 store).  One CTA of
// 128 threads computes one 128 x 256 tile:
//   thread 0    TMA producer: 128B-swizzled 128x64 (A) and 256x64 (B) tiles into a
//               4-stage shared-memory ring (cp.async.bulk.tensor + mbarrier tx counts)
//   thread 32   MMA issuer: 4 x tcgen05.mma (M=128, N=256, K=16) per stage into a
//               128-lane x 256-column FP32 accumulator in tensor memory; each stage
//               is released by tcgen05.commit on its "empty" barrier
//   all warps   epilogue: tcgen05.ld 32x32b (warp w reads TMEM lanes 32w..32w+31 =
//               tile rows), fused math, guarded stores.
// Ragged M, N, K are handled by TMA zero fill on loads and bounds checks on stores.
// Every mbarrier wait is bounded; on a timeout the kernel records an error in *err,
// skips the remaining work, frees its tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace irs {
namespace umma {

// Tile shapes: BM x TBN x BK with TBN = 256 (4 stages, one CTA per SM) or TBN = 128
// (3 stages, 97 KB of shared memory and 128 TMEM columns, two CTAs per SM so that one
// CTA's epilogue overlaps the other's main loop).
constexpr int BM = 128, BK = 64;
constexpr int kThreads = 128;
constexpr uint32_t kTileA = BM * BK * 2;  // 16 KB
template <int TBN> struct TileCfg {
    static constexpr int STAGES = TBN == 256 ? 4 : 3;
    static constexpr uint32_t kTileB = TBN * BK * 2;
    static constexpr size_t kSmemBytes = STAGES * (kTileA + kTileB) + 1024 + 256;
    static constexpr int kMinBlocks = TBN == 256 ? 1 : 2;
};
constexpr uint32_t kMaxSpin = 1u << 22;

enum Epilogue : int {
    EPI_F32 = 0,        // Cf[m][n] = acc
    EPI_BIAS_F32 = 1,   // Cf[m][n] = acc + bias[n]
    EPI_GELU_FWD = 2,   // Z[m][n] = acc + bias[n] (bf16), Cb[m][n] = gelu(Z) (bf16)
    EPI_GELU_BWD = 3,   // Cb[m][n] = acc * gelu'(Zin[m][n]) (bf16)
    EPI_SUMSQ = 4,      // Cf[m] += sum_n acc^2 / N (Cf zeroed by the caller)
};

struct EpiArgs {
    float* Cf;                 // FP32 output
    __nv_bfloat16* Cb;         // BF16 output
    __nv_bfloat16* Z;          // BF16 pre-activation output (GELU_FWD)
    const __nv_bfloat16* Zin;  // BF16 pre-activation input (GELU_BWD)
    const float* bias;
    const float* scale;        // EPI_BIAS_F32, nullable: Cf = (acc + bias) * scale[n] + shift[n]
    const float* shift;
    int ldc;                   // leading dimension of every output / Zin (elements)
    int M, N;
    int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
    const uint32_t a = smem_u32(b);
    for (uint32_t it = 0; it < kMaxSpin; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}
// K-major operand tile, 128-byte swizzle: rows of 64 bf16 (128 B), 8-row atoms 1024 B apart.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset: next 8-row atom
    d |= (uint64_t)1 << 46;              // descriptor version for sm_100
    d |= (uint64_t)2 << 61;              // SWIZZLE_128B
    return d;
}
// kind::f16 instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = TBN
template <int TBN>
struct IdescBf16 {
    static constexpr uint32_t value =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TBN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

template <int EPI, int TBN>
__global__ void __launch_bounds__(kThreads, TileCfg<TBN>::kMinBlocks)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int K,
                     EpiArgs ep) {
    constexpr int BN = TBN;
    constexpr int STAGES = TileCfg<TBN>::STAGES;
    constexpr uint32_t kTileB = TileCfg<TBN>::kTileB;
    constexpr uint32_t kIdesc = IdescBf16<TBN>::value;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * kTileA;
    uint64_t* full = (uint64_t*)(sB + STAGES * kTileB);
    uint64_t* empty = full + STAGES;
    uint64_t* done = empty + STAGES;
    uint32_t* tmem_slot = (uint32_t*)(done + 1);
    int* s_fail = (int*)(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int KT = (K + BK - 1) / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {  // TMA producer
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % STAGES;
            const uint32_t ph = (uint32_t)(kt / STAGES) & 1u;
            if (kt >= STAGES && !mbar_wait(&empty[s], ph ^ 1u)) {
                atomicExch(s_fail, 1);
                break;
            }
            if (*(volatile int*)s_fail) break;
            mbar_expect_tx(&full[s], kTileA + kTileB);
            tma_load_2d(sA + s * kTileA, &tmA, &full[s], kt * BK, m0);
            tma_load_2d(sB + s * kTileB, &tmB, &full[s], kt * BK, n0);
        }
    } else if (threadIdx.x == 32) {  // MMA issuer
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % STAGES;
            const uint32_t ph = (uint32_t)(kt / STAGES) & 1u;
            if (!mbar_wait(&full[s], ph)) {
                atomicExch(s_fail, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sA + s * kTileA), b0 = smem_u32(sB + s * kTileB);
#pragma unroll
            for (int k = 0; k < BK / 16; ++k)
                umma_bf16(tmem, sdesc_sw128(a0 + 32u * k), sdesc_sw128(b0 + 32u * k), kIdesc, (kt | k) != 0 ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        umma_commit(done);  // arrives once every MMA issued above has completed
    }
    __syncwarp();

    // epilogue: thread (warp w, lane l) owns tile row 32 w + l
    const bool ok = mbar_wait(done, 0) && !*(volatile int*)s_fail;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (__all_sync(0xffffffffu, ok)) {
        const int m = m0 + warp * 32 + lane;
        const bool row_ok = m < ep.M;
        for (int c0 = 0; c0 < BN; c0 += 16) {
            if (n0 + c0 >= ep.N) break;  // warp-uniform
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            const int nb = n0 + c0;
            if (EPI == EPI_SUMSQ) {
                float ss = 0.f;
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (nb + i < ep.N) ss = fmaf(v[i], v[i], ss);
                if (row_ok) atomicAdd(ep.Cf + m, ss / (float)ep.N);
                continue;
            }
            if ((EPI == EPI_F32 || EPI == EPI_BIAS_F32) && (ep.ldc & 3) != 0) {
                // rows not 16-byte aligned: stage the warp's 32 x 16 chunk in shared memory
                // (the operand ring is idle now) and write each row's 64 bytes contiguously,
                // two rows per store instruction
                float* stg = (float*)smem + warp * (32 * 17);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float x = v[i];
                    if (EPI == EPI_BIAS_F32 && nb + i < ep.N) {
                        x += ep.bias[nb + i];
                        if (ep.scale) x = fmaf(x, ep.scale[nb + i], ep.shift[nb + i]);
                    }
                    stg[lane * 17 + i] = x;
                }
                __syncwarp();
                const int col = lane & 15, half = lane >> 4;
#pragma unroll 4
                for (int rr = 0; rr < 32; rr += 2) {
                    const int r = rr + half, mr = m0 + warp * 32 + r;
                    if (mr < ep.M && nb + col < ep.N) ep.Cf[(size_t)mr * ep.ldc + nb + col] = stg[r * 17 + col];
                }
                __syncwarp();
                continue;
            }
            if (!row_ok) continue;
            const size_t rowoff = (size_t)m * ep.ldc;
            const bool full16 = nb + 16 <= ep.N;
            if (EPI == EPI_F32 || EPI == EPI_BIAS_F32) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float x = v[i];
                    if (EPI == EPI_BIAS_F32 && (full16 || nb + i < ep.N)) {
                        x += ep.bias[nb + i];
                        if (ep.scale) x = fmaf(x, ep.scale[nb + i], ep.shift[nb + i]);
                    }
                    v[i] = x;
                }
                if (full16 && (ep.ldc & 3) == 0) {
                    float4* dst = (float4*)(ep.Cf + rowoff + nb);
#pragma unroll
                    for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                } else {
                    for (int i = 0; i < 16 && nb + i < ep.N; ++i) ep.Cf[rowoff + nb + i] = v[i];
                }
            } else {
                __align__(16) __nv_bfloat16 out[16];
                __align__(16) __nv_bfloat16 zo[16];
                if (EPI == EPI_GELU_FWD) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const float z = v[i] + ((full16 || nb + i < ep.N) ? ep.bias[nb + i] : 0.f);
                        const __nv_bfloat16 zb = __float2bfloat16_rn(z);
                        zo[i] = zb;
                        out[i] = __float2bfloat16_rn(gelu(__bfloat162float(zb)));
                    }
                } else {  // GELU_BWD
                    __align__(16) __nv_bfloat16 zi[16];
                    if (full16) {
                        const uint4* src = (const uint4*)(ep.Zin + rowoff + nb);
                        ((uint4*)zi)[0] = src[0];
                        ((uint4*)zi)[1] = src[1];
                    } else {
                        for (int i = 0; i < 16; ++i)
                            zi[i] = nb + i < ep.N ? ep.Zin[rowoff + nb + i] : __float2bfloat16_rn(0.f);
                    }
#pragma unroll
                    for (int i = 0; i < 16; ++i) out[i] = __float2bfloat16_rn(v[i] * gelu_grad(__bfloat162float(zi[i])));
                }
                if (full16) {
                    uint4* dst = (uint4*)(ep.Cb + rowoff + nb);
                    dst[0] = ((const uint4*)out)[0];
                    dst[1] = ((const uint4*)out)[1];
                    if (EPI == EPI_GELU_FWD) {
                        uint4* dz = (uint4*)(ep.Z + rowoff + nb);
                        dz[0] = ((const uint4*)zo)[0];
                        dz[1] = ((const uint4*)zo)[1];
                    }
                } else {
                    for (int i = 0; i < 16 && nb + i < ep.N; ++i) {
                        ep.Cb[rowoff + nb + i] = out[i];
                        if (EPI == EPI_GELU_FWD) ep.Z[rowoff + nb + i] = zo[i];
                    }
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicExch(ep.err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

}  // namespace umma
}  // namespace irs
