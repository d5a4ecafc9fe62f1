// umma_gemm.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05) for sm_100a.
//
//   C[m][n] = sum_k A[m][k] B[n][k]        (A, B row-major bf16, both K-major)
//
// followed by a fused epilogue (bias, GELU, GELU backward, FP32 store).  The kernel is
// persistent: one CTA of 320 threads per SM walks the 128 x TBN output tiles
// t = blockIdx.x, blockIdx.x + gridDim.x, ... with three warp roles:
//   warp 0 (lane 0)  TMA producer: 128B-swizzled 128x64 (A) and TBNx64 (B) tiles into a
//                    STAGES-deep shared-memory ring (cp.async.bulk.tensor + mbarrier
//                    tx counts), running ahead across tile boundaries
//   warp 1 (lane 0)  MMA issuer: 4 x tcgen05.mma (M=128, N=TBN, K=16) per stage into one
//                    of two TBN-column FP32 accumulators in tensor memory; each stage is
//                    released by tcgen05.commit on its "empty" barrier, each finished
//                    accumulator by a commit on its "tfull" barrier
//   warps 2..9       epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (= tile rows)
//                    and one half of the columns with tcgen05.ld 32x32b, applies the
//                    fused math, stores, and hands the accumulator back ("tempty")
// so the epilogue of tile i runs under the main loop of tile i + 1.
// Ragged M, N, K are handled by TMA zero fill on loads and bounds checks on stores.
// Every mbarrier wait is bounded; on a timeout the kernel records an error in *err,
// skips the remaining work, waits (bounded) for its own copies and MMAs in flight,
// frees its tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace irs {
namespace umma {

// Tile shapes: BM x TBN x BK with TBN = 256 (4 stages of 48 KB) or TBN = 128 (6 stages of
// 32 KB); either way 192 KB of operand ring, 33 KB (17 KB) of FP32 epilogue staging and
// 2 x TBN tensor-memory columns; one CTA per SM.
constexpr int BM = 128, BK = 64;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr uint32_t kTileA = BM * BK * 2;  // 16 KB
template <int TBN> struct TileCfg {
    static constexpr int STAGES = TBN == 256 ? 4 : 6;
    static constexpr uint32_t kTileB = TBN * BK * 2;
    // FP32 epilogue staging per warp: 8 rows of its TBN / 2 columns, rows padded by 4
    // floats so that 8 rows' float4 writes fall in distinct banks
    static constexpr int kStgStride = TBN / 2 + 4;
    static constexpr uint32_t kStgBytes = kEpiWarps * 8 * kStgStride * 4;
    static constexpr size_t kSmemBytes = STAGES * (kTileA + kTileB) + kStgBytes + 1024 + 256;
    static constexpr uint32_t kTmemCols = 2 * TBN;
    static_assert(kSmemBytes <= 232448, "dynamic shared memory per CTA (227 KB)");
    static_assert(kTmemCols <= 512, "tensor memory columns per SM");
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
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
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

// 32 consecutive accumulator columns of the warp's 32 lanes (one row per lane)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}


// Column constants of one epilogue warp's HALF columns of an FP32-output tile, starting
// at column cfirst: lane l holds column cfirst + 32 j + l in element j.  Loaded before
// the tile's accumulator is ready, so their latency hides under its main loop.
template <int EPI, int J>
__device__ __forceinline__ void load_cols(const EpiArgs& ep, int cfirst, int lane, float (&cb)[J], float (&cs)[J],
                                          float (&ch)[J]) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const int n = cfirst + 32 * j + lane;
        cb[j] = 0.f;
        cs[j] = 1.f;
        ch[j] = 0.f;
        if (EPI == EPI_BIAS_F32 && n < ep.N) {
            cb[j] = __ldg(ep.bias + n);
            if (ep.scale) {
                cs[j] = __ldg(ep.scale + n);
                ch[j] = __ldg(ep.shift + n);
            }
        }
    }
}

// The same constants for the per-row chunk epilogue, staged in the warp's shared-memory
// area as [bias | scale | shift] (HALF floats each) so that every lane reads a chunk's 16
// columns as broadcast float4 loads.
template <int EPI, int HALF>
__device__ __forceinline__ void stage_cols(const EpiArgs& ep, int cfirst, float* cst, int lane) {
    if constexpr (EPI == EPI_BIAS_F32 || EPI == EPI_GELU_FWD) {
#pragma unroll
        for (int j = lane; j < HALF; j += 32) {
            const int n = cfirst + j;
            float b = 0.f, sc = 1.f, sh = 0.f;
            if (n < ep.N) {
                b = __ldg(ep.bias + n);
                if (EPI == EPI_BIAS_F32 && ep.scale) {
                    sc = __ldg(ep.scale + n);
                    sh = __ldg(ep.shift + n);
                }
            }
            cst[j] = b;
            cst[HALF + j] = sc;
            cst[2 * HALF + j] = sh;
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void lds16(const float* p, float (&x)[16]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 t = ((const float4*)p)[i];
        x[4 * i] = t.x;
        x[4 * i + 1] = t.y;
        x[4 * i + 2] = t.z;
        x[4 * i + 3] = t.w;
    }
}

// FP32-output epilogue of one warp's 32 rows (r0 ..) x HALF columns (cfirst ..) of a
// tile whose accumulator columns start at TMEM address tb.  Short row pieces from many
// rows per store instruction leave the SM slowly (and FP32 rows need not be 16-byte
// aligned: ldc = 8461 for the IASI channels); writing 512-byte row runs instead of
// 2 x 64-byte pieces per instruction took a 4096 x 8461 store from 63 to 34 us.  So each
// of four passes stages 8 rows x HALF raw accumulators in shared memory (the pass's 8
// lanes write their rows), and the warp then writes each row as one run, 128 bytes per
// store instruction, applying the epilogue per column on the way out:
//   EPI_F32       Cf[m][n] = acc
//   EPI_BIAS_F32  Cf[m][n] = acc + bias[n], or (acc + bias[n]) * scale[n] + shift[n]
template <int EPI, int HALF>
__device__ __forceinline__ void epilogue_tile(uint32_t tb, int r0, int cfirst, const EpiArgs& ep,
                                              const float (&cb)[HALF / 32], const float (&cs)[HALF / 32],
                                              const float (&ch)[HALF / 32], float* stg, int lane) {
    static_assert(EPI == EPI_F32 || EPI == EPI_BIAS_F32, "bf16 outputs: epilogue_chunk");
    constexpr int S = HALF + 4, J = HALF / 32;
    const int ncols = min(HALF, ep.N - cfirst);  // valid columns (>= 1)
    const int nld = (ncols + 31) / 32;          // 32-column accumulator loads
    const bool scaled = EPI == EPI_BIAS_F32 && ep.scale != nullptr;
#pragma unroll 1
    for (int p = 0; p < 4; ++p) {
        if (r0 + 8 * p >= ep.M) break;  // warp-uniform
        const bool mine = (lane >> 3) == p;
        float* srow = stg + (lane & 7) * S;
#pragma unroll 1
        for (int c = 0; c < nld; ++c) {
            float v[32];
            __syncwarp();  // tcgen05.ld is .sync.aligned
            tmem_ld32(tb + (uint32_t)(32 * c), v);
            if (mine) {
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    ((float4*)(srow + 32 * c))[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
        }
        __syncwarp();
#pragma unroll 2
        for (int r = 0; r < 8; ++r) {
            const int m = r0 + 8 * p + r;
            if (m >= ep.M) break;  // warp-uniform
            const float* src = stg + r * S;
            const size_t row = (size_t)m * ep.ldc + cfirst;
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int col = 32 * j + lane;
                float x = src[col];
                if (EPI == EPI_BIAS_F32) {
                    x += cb[j];
                    if (scaled) x = fmaf(x, cs[j], ch[j]);
                }
                if (col < ncols) ep.Cf[row + col] = x;
            }
        }
        __syncwarp();
    }
}

// One 32-row x 16-column accumulator chunk: lane l holds row r0 + l, columns nb..nb+15;
// cc points at the chunk's staged column constants (bias, then scale and shift HALF and
// 2 HALF floats further).  Each lane works on its own row, so all 32 lanes share the
// arithmetic (the GELU dominates these epilogues), and each row piece is written whole
// (FP32 rows here are 16-byte aligned; unaligned ones go through epilogue_tile).  Every
// array is indexed by compile-time constants only (ragged chunks use predicated
// stores), so all of them stay in registers.
//   EPI_F32       Cf[m][n] = acc
//   EPI_BIAS_F32  Cf[m][n] = acc + bias[n], or (acc + bias[n]) * scale[n] + shift[n]
//   EPI_SUMSQ     Cf[m] += sum_n acc^2 / N
//   EPI_GELU_FWD  Z[m][n] = bf16(acc + bias[n]) (if Z), Cb[m][n] = bf16(gelu(Z[m][n]))
//   EPI_GELU_BWD  Cb[m][n] = bf16(acc * gelu'(Zin[m][n]))
template <int EPI, int HALF>
__device__ __forceinline__ void epilogue_chunk(const float (&v)[16], const float* cc, int r0, int nb,
                                               const EpiArgs& ep, int lane) {
    const int m = r0 + lane;
    const int nv = ep.N - nb;  // valid columns in this chunk (>= 1)
    if (m >= ep.M) return;
    if (EPI == EPI_SUMSQ) {
        float ss = 0.f;
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (i < nv) ss = fmaf(v[i], v[i], ss);
        atomicAdd(ep.Cf + m, ss / (float)ep.N);
        return;
    }
    if (EPI == EPI_F32 || EPI == EPI_BIAS_F32) {
        float x[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = v[i];
        if (EPI == EPI_BIAS_F32) {
            float b[16];
            lds16(cc, b);
            if (ep.scale) {
                float sc[16], sh[16];
                lds16(cc + HALF, sc);
                lds16(cc + 2 * HALF, sh);
#pragma unroll
                for (int i = 0; i < 16; ++i) x[i] = fmaf(x[i] + b[i], sc[i], sh[i]);
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) x[i] += b[i];
            }
        }
        float* dst = ep.Cf + (size_t)m * ep.ldc + nb;
        if (nv >= 16) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
                ((float4*)dst)[i] = make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (i < nv) dst[i] = x[i];
        }
        return;
    }
    const size_t rowoff = (size_t)m * ep.ldc + nb;
    uint32_t out[8], zo[8];  // bf16 pairs
    if (EPI == EPI_GELU_FWD) {
        float b[16];
        lds16(cc, b);
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
            const __nv_bfloat162 zb = __floats2bfloat162_rn(v[i] + b[i], v[i + 1] + b[i + 1]);
            const float2 zf = __bfloat1622float2(zb);
            const __nv_bfloat162 ob = __floats2bfloat162_rn(gelu(zf.x), gelu(zf.y));
            zo[i / 2] = *(const uint32_t*)&zb;
            out[i / 2] = *(const uint32_t*)&ob;
        }
    } else {  // GELU_BWD
        uint32_t zi[8];
        if (nv >= 16) {
            const uint4 a = ((const uint4*)(ep.Zin + rowoff))[0], c = ((const uint4*)(ep.Zin + rowoff))[1];
            zi[0] = a.x; zi[1] = a.y; zi[2] = a.z; zi[3] = a.w;
            zi[4] = c.x; zi[5] = c.y; zi[6] = c.z; zi[7] = c.w;
        } else {
            const unsigned short* zs = (const unsigned short*)(ep.Zin + rowoff);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint32_t lo = 2 * i < nv ? zs[2 * i] : 0u, hi = 2 * i + 1 < nv ? zs[2 * i + 1] : 0u;
                zi[i] = lo | (hi << 16);
            }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float2 zf = __bfloat1622float2(*(const __nv_bfloat162*)&zi[i]);
            const __nv_bfloat162 ob =
                __floats2bfloat162_rn(v[2 * i] * gelu_grad(zf.x), v[2 * i + 1] * gelu_grad(zf.y));
            out[i] = *(const uint32_t*)&ob;
        }
    }
    const bool keep_z = EPI == EPI_GELU_FWD && ep.Z != nullptr;  // inference keeps no pre-activations
    if (nv >= 16) {
        uint4* dst = (uint4*)(ep.Cb + rowoff);
        dst[0] = make_uint4(out[0], out[1], out[2], out[3]);
        dst[1] = make_uint4(out[4], out[5], out[6], out[7]);
        if (keep_z) {
            uint4* dz = (uint4*)(ep.Z + rowoff);
            dz[0] = make_uint4(zo[0], zo[1], zo[2], zo[3]);
            dz[1] = make_uint4(zo[4], zo[5], zo[6], zo[7]);
        }
    } else {
        unsigned short* cbo = (unsigned short*)(ep.Cb + rowoff);
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (i < nv) {
                cbo[i] = (unsigned short)(out[i / 2] >> (16 * (i & 1)));
                if (keep_z) ((unsigned short*)(ep.Z + rowoff))[i] = (unsigned short)(zo[i / 2] >> (16 * (i & 1)));
            }
    }
}

template <int EPI, int TBN>
__global__ void __launch_bounds__(kThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int K,
                     EpiArgs ep) {
    constexpr int BN = TBN;
    constexpr int STAGES = TileCfg<TBN>::STAGES;
    constexpr uint32_t kTileB = TileCfg<TBN>::kTileB;
    constexpr uint32_t kCols = TileCfg<TBN>::kTmemCols;
    constexpr uint32_t kIdesc = IdescBf16<TBN>::value;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * kTileA;
    float* stg_all = (float*)(sB + STAGES * kTileB);
    uint64_t* full = (uint64_t*)((uint8_t*)stg_all + TileCfg<TBN>::kStgBytes);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;  // [2] accumulator ready for the epilogue
    uint64_t* tempty = tfull + 2;      // [2] accumulator drained by the epilogue
    uint64_t* drain = tempty + 2;
    uint32_t* tmem_slot = (uint32_t*)(drain + 1);
    int* s_fail = (int*)(tmem_slot + 1);
    volatile int* fail = s_fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = (K + BK - 1) / BK;
    const int mblocks = (ep.M + BM - 1) / BM;
    const int ntiles = mblocks * ((ep.N + BN - 1) / BN);

    if (threadIdx.x == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmB) : "memory");
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kEpiWarps);
        }
        mbar_init(drain, 1);
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    // Launched with programmatic stream serialization: the next kernel in the stream may
    // start its own prologue on idle SMs now, and this grid's reads and writes of global
    // memory wait until the previous grid has completed (its outputs are our operands).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            uint32_t it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const int m0 = (t % mblocks) * BM, n0 = (t / mblocks) * BN;
                for (int kt = 0; kt < KT; ++kt) {
                    const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
                    if ((it >= (uint32_t)STAGES && !mbar_wait(&empty[s], ph ^ 1u)) || *fail) {
                        atomicExch(s_fail, 1);
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full[s], kTileA + kTileB);
                    tma_load_2d(sA + s * kTileA, &tmA, &full[s], kt * BK, m0);
                    tma_load_2d(sB + s * kTileB, &tmB, &full[s], kt * BK, n0);
                    ++it;
                }
            }
            // every copy issued has landed before the CTA may exit (the last use of
            // each stage s was load number s + (n_s - 1) STAGES, phase parity n_s - 1)
            for (uint32_t s = 0; s < (uint32_t)STAGES; ++s) {
                if (it <= s) break;
                const uint32_t n_s = (it - 1u - s) / STAGES + 1u;
                if (!mbar_wait(&full[s], (n_s - 1u) & 1u)) atomicExch(s_fail, 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            uint32_t it = 0;
            int li = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++li) {
                const int buf = li & 1;
                const uint32_t acc_ph = (uint32_t)(li >> 1) & 1u;
                if ((li >= 2 && !mbar_wait(&tempty[buf], acc_ph ^ 1u)) || *fail) {
                    atomicExch(s_fail, 1);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(buf * BN);
                for (int kt = 0; kt < KT; ++kt, ++it) {
                    const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
                    if (!mbar_wait(&full[s], ph)) {
                        atomicExch(s_fail, 1);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t a0 = smem_u32(sA + s * kTileA), b0 = smem_u32(sB + s * kTileB);
#pragma unroll
                    for (int k = 0; k < BK / 16; ++k)
                        umma_bf16(d, sdesc_sw128(a0 + 32u * k), sdesc_sw128(b0 + 32u * k), kIdesc,
                                  (kt | k) != 0 ? 1u : 0u);
                    umma_commit(&empty[s]);
                }
                if (ok) umma_commit(&tfull[buf]);
            }
            // arrives once every MMA issued above has completed
            umma_commit(drain);
            if (!mbar_wait(drain, 0)) atomicExch(s_fail, 1);
        }
    } else {  // epilogue warps
        constexpr int HALF = BN / 2, J = HALF / 32;
        // unaligned FP32 rows: staged row runs; everything else: per-row chunks
        const bool rowrun = (EPI == EPI_F32 || EPI == EPI_BIAS_F32) && (ep.ldc & 3) != 0;
        const int q = warp & 3, h = (warp - 2) >> 2;
        float* stg = stg_all + (warp - 2) * (8 * TileCfg<TBN>::kStgStride);
        int li = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++li) {
            const int buf = li & 1;
            const uint32_t acc_ph = (uint32_t)(li >> 1) & 1u;
            const int m0 = (t % mblocks) * BM, n0 = (t / mblocks) * BN;
            const int cfirst = n0 + h * HALF;
            // column constants, fetched under the tile's main loop
            float cb[J], cs[J], ch[J];
            if (rowrun)
                load_cols<EPI, J>(ep, cfirst, lane, cb, cs, ch);
            else
                stage_cols<EPI, HALF>(ep, cfirst, stg, lane);
            const bool ok = mbar_wait(&tfull[buf], acc_ph) && !*fail;
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) atomicExch(s_fail, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * BN + h * HALF);
            if (cfirst < ep.N) {  // warp-uniform
                if (rowrun) {
                    if constexpr (EPI == EPI_F32 || EPI == EPI_BIAS_F32)
                        epilogue_tile<EPI, HALF>(tb, m0 + q * 32, cfirst, ep, cb, cs, ch, stg, lane);
                } else {
#pragma unroll 1
                    for (int c = 0; c < HALF && cfirst + c < ep.N; c += 16) {  // warp-uniform bound
                        float v[16];
                        __syncwarp();  // tcgen05.ld is .sync.aligned
                        tmem_ld16(tb + (uint32_t)c, v);
                        epilogue_chunk<EPI, HALF>(v, stg + c, m0 + q * 32, cfirst + c, ep, lane);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0 && *fail) atomicExch(ep.err, 1);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

}  // namespace umma
}  // namespace irs
