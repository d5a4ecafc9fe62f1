// surrogate.cu -- the MLP surrogate of forward_model (profile + scan angle -> channel
// BTs) on the tcgen05 tensor cores: BF16 weights and activations, FP32 accumulation,
// FP32 master weights with Adam.  The GEMMs are umma_gemm.cuh; everything around them
// (input scaling, loss, transposes, bias gradients, optimiser, OOD score) is here.
// No counterpart in the reference: it is the learned fast path that the LBL kernels
// train and judge.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <vector>

#include "irs_internal.h"
#include "umma_gemm.cuh"

using irs::Error;
using bf16 = __nv_bfloat16;

namespace irs {
namespace sg {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    if (!fn) throw Error{IRS_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver"};
    return fn;
}

// [rows][cols] bf16 with leading dimension ld: box of 64 columns x box_rows rows, 128B swizzle
static CUtensorMap make_map(const void* ptr, int64_t rows, int64_t cols, int64_t ld, int box_rows) {
    IRS_REQUIRE(((uintptr_t)ptr & 15) == 0 && ld % 8 == 0 && rows >= 1 && cols >= 1, "GEMM operand layout");
    CUtensorMap m;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
                                   es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error{IRS_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")"};
    return m;
}

// SM count and "max dynamic shared memory" attribute per device (a process may drive
// several devices, one host thread each)
static int sm_count(int dev) {
    static std::mutex mu;
    static int cached[64] = {};
    IRS_REQUIRE(dev >= 0 && dev < 64, "device index");
    std::lock_guard<std::mutex> lk(mu);
    if (!cached[dev]) IRS_CUDA(cudaDeviceGetAttribute(&cached[dev], cudaDevAttrMultiProcessorCount, dev));
    return cached[dev];
}

template <int EPI, int TBN>
static void gemm_tbn(cudaStream_t st, int dev, int nsm, const bf16* A, int64_t lda, const bf16* B, int64_t ldb, int M,
                     int N, int K, umma::EpiArgs ep) {
    using Cfg = umma::TileCfg<TBN>;
    static std::mutex mu;
    static uint64_t attr_set = 0;  // bit d: attribute set on device d
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!(attr_set >> dev & 1u)) {
            IRS_CUDA(cudaFuncSetAttribute(umma::umma_gemm_kernel<EPI, TBN>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmemBytes));
            attr_set |= (uint64_t)1 << dev;
        }
    }
    const CUtensorMap ta = make_map(A, M, K, lda, umma::BM);
    const CUtensorMap tb = make_map(B, N, K, ldb, TBN);
    ep.M = M;
    ep.N = N;
    const int64_t tiles = (int64_t)((M + umma::BM - 1) / umma::BM) * ((N + TBN - 1) / TBN);
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, nsm);  // persistent: one CTA per SM at most
    // programmatic dependent launch: the kernel waits (griddepcontrol.wait) for the
    // previous grid before touching global memory, so only its prologue overlaps
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(umma::kThreads);
    cfg.dynamicSmemBytes = Cfg::kSmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    IRS_CUDA(cudaLaunchKernelEx(&cfg, umma::umma_gemm_kernel<EPI, TBN>, ta, tb, K, ep));
}

// Tile width: 128 x 256 tiles halve the B-operand traffic per FLOP; 128 x 128 tiles are
// taken when they spread a small problem over clearly more SMs (the makespan in units
// of a 128 x 128 tile, rounds x tile cost, at least 25 % shorter).
template <int EPI>
static void gemm(cudaStream_t st, const bf16* A, int64_t lda, const bf16* B, int64_t ldb, int M, int N, int K,
                 umma::EpiArgs ep) {
    const bool f32_out = EPI == umma::EPI_F32 || EPI == umma::EPI_BIAS_F32;
    IRS_REQUIRE(M >= 1 && N >= 1 && K >= 1 && ep.ldc >= N && (f32_out || ep.ldc % 8 == 0), "GEMM sizes");
    int dev = 0;
    IRS_CUDA(cudaGetDevice(&dev));
    const int nsm = sm_count(dev);
    const int64_t mb = (M + umma::BM - 1) / umma::BM;
    const int64_t t128 = mb * ((N + 127) / 128), t256 = mb * ((N + 255) / 256);
    const int64_t cost128 = (t128 + nsm - 1) / nsm, cost256 = 2 * ((t256 + nsm - 1) / nsm);
    if (4 * cost128 <= 3 * cost256)
        gemm_tbn<EPI, 128>(st, dev, nsm, A, lda, B, ldb, M, N, K, ep);
    else
        gemm_tbn<EPI, 256>(st, dev, nsm, A, lda, B, ldb, M, N, K, ep);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error{IRS_E_CUDA, std::string("GEMM launch: ") + cudaGetErrorString(e)};
}

// ------------------------------------------------------------ helper kernels
// dst[c][r] = src[r][c] for r < rows, c < cols (32 x 32 tiles through shared memory)
__global__ void transpose_kernel(const bf16* __restrict__ src, int rows, int cols, int64_t lds, bf16* __restrict__ dst,
                                 int64_t ldd) {
    __shared__ bf16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int r = r0 + j, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[j][threadIdx.x] = src[(size_t)r * lds + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int c = c0 + j, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(size_t)c * ldd + r] = t[threadIdx.x][j];
    }
}
static void transpose(cudaStream_t st, const bf16* src, int rows, int cols, int64_t lds, bf16* dst, int64_t ldd) {
    transpose_kernel<<<dim3((cols + 31) / 32, (rows + 31) / 32), dim3(32, 8), 0, st>>>(src, rows, cols, lds, dst, ldd);
}

// X0[b][k] = bf16((x[idx[b]][k] - mean[k]) / std[k]) for k < n_in, 0 up to ld
__global__ void prep_input_kernel(const float* __restrict__ x, const int* __restrict__ idx, int n_in, int ld, int B,
                                  const float* __restrict__ mean, const float* __restrict__ sd, bf16* __restrict__ X0) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const int64_t row = idx ? idx[b] : b;
    for (int k = threadIdx.x; k < ld; k += blockDim.x) {
        const float v = k < n_in ? (x[row * n_in + k] - mean[k]) / sd[k] : 0.f;
        X0[(size_t)b * ld + k] = __float2bfloat16_rn(v);
    }
}

// scaled targets and the loss gradient of 0.5 mean((y - t)^2) over the valid outputs:
// dY = (y - t) / (B n_out) (bf16, 0 in the padding); loss accumulated in FP64
__global__ void loss_kernel(const float* __restrict__ Y, int ldy, const float* __restrict__ t, const int* __restrict__ idx,
                            int n_out, int B, const float* __restrict__ ymean, const float* __restrict__ ysd,
                            bf16* __restrict__ dY, double* __restrict__ loss) {
    const int b = blockIdx.x;
    const int64_t row = idx ? idx[b] : b;
    const float scale = 1.f / ((float)B * (float)n_out);
    double acc = 0.0;
    for (int k = threadIdx.x; k < ldy; k += blockDim.x) {
        float g = 0.f;
        if (k < n_out) {
            const float tt = (t[row * n_out + k] - ymean[k]) / ysd[k];
            const float d = Y[(size_t)b * ldy + k] - tt;
            acc += 0.5 * (double)d * (double)d;
            g = d * scale;
        }
        dY[(size_t)b * ldy + k] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        atomicAdd(loss, s / ((double)B * (double)n_out));
    }
}

// db[n] = sum_b dZ[b][n]
__global__ void colsum_kernel(const bf16* __restrict__ dZ, int B, int N, int64_t ld, float* __restrict__ db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f, c = 0.f;
    for (int b = 0; b < B; ++b) {  // compensated: B is up to a few thousand
        const float y = __bfloat162float(dZ[(size_t)b * ld + n]) - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    db[n] = s;
}

// Adam (bias-corrected) on the FP32 master copy; refreshes the BF16 weights
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}
__global__ void to_bf16_kernel(const float* __restrict__ w, int64_t n, bf16* __restrict__ o) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = __float2bfloat16_rn(w[i]);
}

inline int64_t pad64(int64_t n) { return (n + 63) / 64 * 64; }

}  // namespace sg
}  // namespace irs

using namespace irs;
using namespace irs::sg;

struct irs_surrogate {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_in = 0, n_hidden = 0, n_layers = 0, n_out = 0;
    int nl = 0;                    // linear maps = n_layers + 1
    std::vector<int> din, dout;    // true sizes per map
    std::vector<int> pin, pout;    // padded sizes (multiples of 64)
    std::vector<int64_t> woff, boff;  // offsets in the padded parameter vector
    int64_t n_par = 0;
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    bf16 *wb = nullptr, *wt = nullptr;  // BF16 weights [pout][pin] and transposes [pin][pout] (same offsets)
    float *xmean = nullptr, *xsd = nullptr, *ymean = nullptr, *ysd = nullptr;
    bf16* white_b = nullptr;  // whitening matrix, BF16 [n_in][pin0], for the tensor-core OOD score
    int* err = nullptr;
    double* loss = nullptr;
    int64_t t_step = 0;
    // batch workspace
    int cap = 0;
    std::vector<bf16*> act, z;     // act[0] = scaled input, act[l] l >= 1 hidden outputs; z[l] pre-activations
    float* Y = nullptr;
    bf16 *dY = nullptr, *dZa = nullptr, *dZb = nullptr, *T1 = nullptr, *T2 = nullptr;
    // device data (training set, inference input)
    float *dx = nullptr, *dt = nullptr;
    int64_t dx_cap = 0, dt_cap = 0;
    int* didx = nullptr;
    int64_t didx_cap = 0;
    float *dout_buf = nullptr, *dood = nullptr;
    int64_t dout_cap = 0, dood_cap = 0;
};

static void* dmalloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
        cudaGetLastError();
        throw Error{IRS_E_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed (surrogate)"};
    }
    return p;
}
template <typename T>
static void grow(T*& p, int64_t& cap, int64_t n) {
    if (n <= cap && p) return;
    if (p) cudaFree(p);
    p = (T*)dmalloc((size_t)n * sizeof(T));
    cap = n;
}

static void ensure_batch(irs_surrogate* s, int B) {
    if (B <= s->cap) return;
    for (auto p : s->act) cudaFree(p);
    for (auto p : s->z) cudaFree(p);
    cudaFree(s->Y); cudaFree(s->dY); cudaFree(s->dZa); cudaFree(s->dZb); cudaFree(s->T1); cudaFree(s->T2);
    const int Bp = (int)pad64(B);
    s->act.assign(s->nl, nullptr);
    s->z.assign(s->nl, nullptr);
    int widest = 0;
    for (int l = 0; l < s->nl; ++l) widest = std::max({widest, s->pin[l], s->pout[l]});
    for (int l = 0; l < s->nl; ++l) {
        s->act[l] = (bf16*)dmalloc((size_t)Bp * s->pin[l] * sizeof(bf16));
        if (l < s->nl - 1) s->z[l] = (bf16*)dmalloc((size_t)Bp * s->pout[l] * sizeof(bf16));
    }
    s->Y = (float*)dmalloc((size_t)Bp * s->pout[s->nl - 1] * sizeof(float));
    s->dY = (bf16*)dmalloc((size_t)Bp * widest * sizeof(bf16));
    s->dZa = (bf16*)dmalloc((size_t)Bp * widest * sizeof(bf16));
    s->dZb = (bf16*)dmalloc((size_t)Bp * widest * sizeof(bf16));
    s->T1 = (bf16*)dmalloc((size_t)Bp * widest * sizeof(bf16));
    s->T2 = (bf16*)dmalloc((size_t)Bp * widest * sizeof(bf16));
    s->cap = B;
}

static void check_err(irs_surrogate* s) {
    int e = 0;
    IRS_CUDA(cudaMemcpyAsync(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    IRS_CUDA(cudaStreamSynchronize(s->stream));
    if (e) throw Error{IRS_E_CUDA, "tensor-core GEMM: a pipeline wait timed out"};
}

static void refresh_bf16(irs_surrogate* s) {
    const cudaStream_t st = s->stream;
    to_bf16_kernel<<<(unsigned)((s->n_par + 255) / 256), 256, 0, st>>>(s->w, s->n_par, s->wb);
    for (int l = 0; l < s->nl; ++l)
        transpose(st, s->wb + s->woff[l], s->pout[l], s->pin[l], s->pin[l], s->wt + s->woff[l], s->pout[l]);
    IRS_CUDA(cudaGetLastError());
}

// forward pass of B rows already in act[0]; Y = scaled outputs, or with yout the
// unscaled outputs y' y_sd + y_mean written straight to yout [B][ldy] (n_out columns)
static void forward(irs_surrogate* s, int B, float* yout = nullptr, int ldy = 0) {
    const cudaStream_t st = s->stream;
    for (int l = 0; l < s->nl; ++l) {
        umma::EpiArgs ep{};
        ep.bias = s->w + s->boff[l];
        ep.err = s->err;
        if (l < s->nl - 1) {
            ep.Cb = s->act[l + 1];
            ep.Z = yout ? nullptr : s->z[l];  // inference keeps no pre-activations
            ep.ldc = s->pout[l];
            gemm<umma::EPI_GELU_FWD>(st, s->act[l], s->pin[l], s->wb + s->woff[l], s->pin[l], B, s->pout[l], s->pin[l], ep);
        } else if (yout) {
            ep.Cf = yout;
            ep.ldc = ldy;
            ep.scale = s->ysd;
            ep.shift = s->ymean;
            gemm<umma::EPI_BIAS_F32>(st, s->act[l], s->pin[l], s->wb + s->woff[l], s->pin[l], B, s->n_out, s->pin[l], ep);
        } else {
            ep.Cf = s->Y;
            ep.ldc = s->pout[l];
            gemm<umma::EPI_BIAS_F32>(st, s->act[l], s->pin[l], s->wb + s->woff[l], s->pin[l], B, s->pout[l], s->pin[l], ep);
        }
    }
}

// loss and gradients of B rows (targets t[idx[b]]); gradients into s->g
static void backward(irs_surrogate* s, int B, const float* t, const int* idx) {
    const cudaStream_t st = s->stream;
    const int Bp = (int)pad64(B);
    const int last = s->nl - 1;
    loss_kernel<<<B, 256, 0, st>>>(s->Y, s->pout[last], t, idx, s->n_out, B, s->ymean, s->ysd, s->dY, s->loss);
    IRS_CUDA(cudaMemsetAsync(s->g, 0, (size_t)s->n_par * sizeof(float), st));
    bf16* dcur = s->dY;  // dZ of map l, [B][pout[l]]
    for (int l = last; l >= 0; --l) {
        // dW[l] = dZ^T act[l]: M = pout, N = pin, K = B
        transpose(st, dcur, B, s->pout[l], s->pout[l], s->T1, Bp);
        transpose(st, s->act[l], B, s->pin[l], s->pin[l], s->T2, Bp);
        umma::EpiArgs ep{};
        ep.Cf = s->g + s->woff[l];
        ep.ldc = s->pin[l];
        ep.err = s->err;
        gemm<umma::EPI_F32>(st, s->T1, Bp, s->T2, Bp, s->pout[l], s->pin[l], B, ep);
        colsum_kernel<<<(s->pout[l] + 255) / 256, 256, 0, st>>>(dcur, B, s->pout[l], s->pout[l], s->g + s->boff[l]);
        if (l > 0) {
            // dZ[l-1] = (dZ[l] W[l]) * gelu'(z[l-1]): M = B, N = pin[l], K = pout[l]
            bf16* dnext = dcur == s->dZa ? s->dZb : s->dZa;
            umma::EpiArgs eb{};
            eb.Cb = dnext;
            eb.Zin = s->z[l - 1];
            eb.ldc = s->pin[l];
            eb.err = s->err;
            gemm<umma::EPI_GELU_BWD>(st, dcur, s->pout[l], s->wt + s->woff[l], s->pout[l], B, s->pin[l], s->pout[l], eb);
            dcur = dnext;
        }
    }
    IRS_CUDA(cudaGetLastError());
}

#define SG_BEGIN try {
#define SG_END                                       \
    }                                                \
    catch (const Error& e) {                         \
        irs::set_error(e.msg);                       \
        return e.code;                               \
    }                                                \
    catch (const std::exception& e) {                \
        irs::set_error(e.what());                    \
        return IRS_E_STATE;                          \
    }                                                \
    return IRS_OK;

static void upload_white_bf16(irs_surrogate* s, const float* W) {
    const int ld = s->pin[0];
    std::vector<uint16_t> h((size_t)s->n_in * ld, 0);
    for (int i = 0; i < s->n_in; ++i)
        for (int j = 0; j < s->n_in; ++j) {
            uint32_t u;
            std::memcpy(&u, &W[(size_t)i * s->n_in + j], 4);
            h[(size_t)i * ld + j] = (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);  // round to nearest even
        }
    if (!s->white_b) s->white_b = (bf16*)dmalloc(h.size() * sizeof(bf16));
    IRS_CUDA(cudaMemcpy(s->white_b, h.data(), h.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
}

extern "C" {

int irs_surrogate_create(irs_ctx* ctx, int n_in, int n_hidden, int n_layers, int n_out, uint64_t seed,
                         irs_surrogate** out) {
    SG_BEGIN
    IRS_REQUIRE(ctx && out && n_in >= 1 && n_hidden >= 8 && n_layers >= 1 && n_out >= 1, "invalid surrogate sizes");
    IRS_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<irs_surrogate> s(new irs_surrogate());
    s->device = ctx->device;
    IRS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));  // owned: outlives the context
    s->n_in = n_in, s->n_hidden = n_hidden, s->n_layers = n_layers, s->n_out = n_out;
    s->nl = n_layers + 1;
    for (int l = 0; l < s->nl; ++l) {
        s->din.push_back(l == 0 ? n_in : n_hidden);
        s->dout.push_back(l == s->nl - 1 ? n_out : n_hidden);
        s->pin.push_back((int)pad64(s->din[l]));
        s->pout.push_back((int)pad64(s->dout[l]));
        s->woff.push_back(s->n_par);
        s->n_par += (int64_t)s->pin[l] * s->pout[l];
        s->boff.push_back(s->n_par);
        s->n_par += pad64(s->pout[l]);
    }
    // Glorot-uniform weights, zero biases, zero padding (host RNG, seeded)
    std::vector<float> h((size_t)s->n_par, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < s->nl; ++l) {
        const float a = std::sqrt(6.f / (float)(s->din[l] + s->dout[l]));
        std::uniform_real_distribution<float> U(-a, a);
        for (int o = 0; o < s->dout[l]; ++o)
            for (int i = 0; i < s->din[l]; ++i) h[s->woff[l] + (size_t)o * s->pin[l] + i] = U(rng);
    }
    s->w = (float*)dmalloc(s->n_par * sizeof(float));
    s->m = (float*)dmalloc(s->n_par * sizeof(float));
    s->v = (float*)dmalloc(s->n_par * sizeof(float));
    s->g = (float*)dmalloc(s->n_par * sizeof(float));
    s->wb = (bf16*)dmalloc(s->n_par * sizeof(bf16));
    s->wt = (bf16*)dmalloc(s->n_par * sizeof(bf16));
    s->err = (int*)dmalloc(sizeof(int));
    s->loss = (double*)dmalloc(sizeof(double));
    IRS_CUDA(cudaMemcpy(s->w, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
    IRS_CUDA(cudaMemset(s->m, 0, s->n_par * sizeof(float)));
    IRS_CUDA(cudaMemset(s->v, 0, s->n_par * sizeof(float)));
    IRS_CUDA(cudaMemset(s->err, 0, sizeof(int)));
    std::vector<float> ones(std::max(n_in, n_out), 1.f), zeros(std::max(n_in, n_out), 0.f);
    s->xmean = (float*)dmalloc(n_in * sizeof(float));
    s->xsd = (float*)dmalloc(n_in * sizeof(float));
    s->ymean = (float*)dmalloc(n_out * sizeof(float));
    s->ysd = (float*)dmalloc(n_out * sizeof(float));
    IRS_CUDA(cudaMemcpy(s->xmean, zeros.data(), n_in * sizeof(float), cudaMemcpyHostToDevice));
    IRS_CUDA(cudaMemcpy(s->xsd, ones.data(), n_in * sizeof(float), cudaMemcpyHostToDevice));
    IRS_CUDA(cudaMemcpy(s->ymean, zeros.data(), n_out * sizeof(float), cudaMemcpyHostToDevice));
    IRS_CUDA(cudaMemcpy(s->ysd, ones.data(), n_out * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<float> eye((size_t)n_in * n_in, 0.f);
    for (int i = 0; i < n_in; ++i) eye[(size_t)i * n_in + i] = 1.f;
    upload_white_bf16(s.get(), eye.data());
    refresh_bf16(s.get());
    IRS_CUDA(cudaStreamSynchronize(s->stream));
    *out = s.release();
    SG_END
}

int irs_surrogate_destroy(irs_surrogate* s) {
    SG_BEGIN
    if (!s) return IRS_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    for (auto p : s->act) cudaFree(p);
    for (auto p : s->z) cudaFree(p);
    void* bufs[] = {s->w, s->m, s->v, s->g, s->wb, s->wt, s->xmean, s->xsd, s->ymean, s->ysd, s->white_b, s->err,
                    s->loss, s->Y, s->dY, s->dZa, s->dZb, s->T1, s->T2, s->dx, s->dt, s->didx, s->dout_buf, s->dood};
    for (void* p : bufs)
        if (p) cudaFree(p);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    SG_END
}

int irs_surrogate_param_count(irs_surrogate* s, int64_t* n) {
    SG_BEGIN
    IRS_REQUIRE(s && n, "invalid arguments");
    int64_t c = 0;
    for (int l = 0; l < s->nl; ++l) c += (int64_t)s->din[l] * s->dout[l] + s->dout[l];
    *n = c;
    SG_END
}

// flat FP32 parameters: per map W [dout][din] row-major, then b [dout]
static void pack_params(irs_surrogate* s, const float* dev, float* host) {
    std::vector<float> h((size_t)s->n_par);
    IRS_CUDA(cudaMemcpyAsync(h.data(), dev, h.size() * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    IRS_CUDA(cudaStreamSynchronize(s->stream));
    size_t k = 0;
    for (int l = 0; l < s->nl; ++l) {
        for (int o = 0; o < s->dout[l]; ++o)
            for (int i = 0; i < s->din[l]; ++i) host[k++] = h[s->woff[l] + (size_t)o * s->pin[l] + i];
        for (int o = 0; o < s->dout[l]; ++o) host[k++] = h[s->boff[l] + o];
    }
}

int irs_surrogate_get_params(irs_surrogate* s, float* params) {
    SG_BEGIN
    IRS_REQUIRE(s && params, "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    pack_params(s, s->w, params);
    SG_END
}

int irs_surrogate_set_params(irs_surrogate* s, const float* params) {
    SG_BEGIN
    IRS_REQUIRE(s && params, "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    std::vector<float> h((size_t)s->n_par, 0.f);
    size_t k = 0;
    for (int l = 0; l < s->nl; ++l) {
        for (int o = 0; o < s->dout[l]; ++o)
            for (int i = 0; i < s->din[l]; ++i) h[s->woff[l] + (size_t)o * s->pin[l] + i] = params[k++];
        for (int o = 0; o < s->dout[l]; ++o) h[s->boff[l] + o] = params[k++];
    }
    IRS_CUDA(cudaMemcpyAsync(s->w, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    IRS_CUDA(cudaMemsetAsync(s->m, 0, s->n_par * sizeof(float), s->stream));
    IRS_CUDA(cudaMemsetAsync(s->v, 0, s->n_par * sizeof(float), s->stream));
    s->t_step = 0;
    refresh_bf16(s);
    IRS_CUDA(cudaStreamSynchronize(s->stream));
    SG_END
}

int irs_surrogate_set_scaling(irs_surrogate* s, const float* x_mean, const float* x_sd, const float* y_mean,
                              const float* y_sd) {
    SG_BEGIN
    IRS_REQUIRE(s && x_mean && x_sd && y_mean && y_sd, "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    for (int i = 0; i < s->n_in; ++i) IRS_REQUIRE(x_sd[i] > 0.f, "input scales must be positive");
    for (int i = 0; i < s->n_out; ++i) IRS_REQUIRE(y_sd[i] > 0.f, "output scales must be positive");
    IRS_CUDA(cudaMemcpy(s->xmean, x_mean, s->n_in * sizeof(float), cudaMemcpyHostToDevice));
    IRS_CUDA(cudaMemcpy(s->xsd, x_sd, s->n_in * sizeof(float), cudaMemcpyHostToDevice));
    IRS_CUDA(cudaMemcpy(s->ymean, y_mean, s->n_out * sizeof(float), cudaMemcpyHostToDevice));
    IRS_CUDA(cudaMemcpy(s->ysd, y_sd, s->n_out * sizeof(float), cudaMemcpyHostToDevice));
    SG_END
}

int irs_surrogate_set_whitening(irs_surrogate* s, const float* W) {
    SG_BEGIN
    IRS_REQUIRE(s && W, "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    upload_white_bf16(s, W);
    SG_END
}

int irs_surrogate_train(irs_surrogate* s, const float* X, const float* Yt, int64_t n, int batch, int epochs, float lr,
                        uint64_t seed, double* loss_per_epoch) {
    SG_BEGIN
    IRS_REQUIRE(s && X && Yt && n >= 1 && batch >= 1 && epochs >= 1 && lr > 0.f && loss_per_epoch,
                "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    grow(s->dx, s->dx_cap, n * s->n_in);
    grow(s->dt, s->dt_cap, n * s->n_out);
    grow(s->didx, s->didx_cap, n);
    IRS_CUDA(cudaMemcpyAsync(s->dx, X, (size_t)n * s->n_in * sizeof(float), cudaMemcpyHostToDevice, st));
    IRS_CUDA(cudaMemcpyAsync(s->dt, Yt, (size_t)n * s->n_out * sizeof(float), cudaMemcpyHostToDevice, st));
    const int B = (int)std::min<int64_t>(batch, n);
    ensure_batch(s, B);
    std::vector<int> perm((size_t)n);
    std::mt19937_64 rng(seed);
    for (int ep = 0; ep < epochs; ++ep) {
        // cosine learning-rate schedule from lr down to lr / 100 over the epochs
        const float lr_min = 0.01f * lr;
        const float lr_ep = epochs > 1 ? lr_min + 0.5f * (lr - lr_min) *
                                                      (1.f + std::cos(3.14159265f * (float)ep / (float)(epochs - 1)))
                                       : lr;
        std::iota(perm.begin(), perm.end(), 0);
        std::shuffle(perm.begin(), perm.end(), rng);
        IRS_CUDA(cudaMemcpyAsync(s->didx, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        IRS_CUDA(cudaMemsetAsync(s->loss, 0, sizeof(double), st));
        int n_batches = 0;
        for (int64_t b0 = 0; b0 + B <= n; b0 += B, ++n_batches) {  // full batches only
            const int* idx = s->didx + b0;
            prep_input_kernel<<<B, 256, 0, st>>>(s->dx, idx, s->n_in, s->pin[0], B, s->xmean, s->xsd, s->act[0]);
            forward(s, B);
            backward(s, B, s->dt, idx);
            s->t_step += 1;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)s->t_step), c2 = 1.f - std::pow(b2, (float)s->t_step);
            adam_kernel<<<(unsigned)((s->n_par + 255) / 256), 256, 0, st>>>(s->w, s->m, s->v, s->g, s->n_par, lr_ep,
                                                                             b1, b2, 1e-8f, c1, c2);
            refresh_bf16(s);
        }
        double l = 0.0;
        IRS_CUDA(cudaMemcpyAsync(&l, s->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
        check_err(s);
        loss_per_epoch[ep] = n_batches ? l / n_batches : 0.0;
    }
    SG_END
}

int irs_surrogate_gradients(irs_surrogate* s, const float* X, const float* Yt, int64_t n, float* grads, double* loss) {
    SG_BEGIN
    IRS_REQUIRE(s && X && Yt && grads && loss && n >= 1 && n <= (1 << 20), "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    grow(s->dx, s->dx_cap, n * s->n_in);
    grow(s->dt, s->dt_cap, n * s->n_out);
    IRS_CUDA(cudaMemcpyAsync(s->dx, X, (size_t)n * s->n_in * sizeof(float), cudaMemcpyHostToDevice, st));
    IRS_CUDA(cudaMemcpyAsync(s->dt, Yt, (size_t)n * s->n_out * sizeof(float), cudaMemcpyHostToDevice, st));
    ensure_batch(s, (int)n);
    IRS_CUDA(cudaMemsetAsync(s->loss, 0, sizeof(double), st));
    prep_input_kernel<<<(int)n, 256, 0, st>>>(s->dx, nullptr, s->n_in, s->pin[0], (int)n, s->xmean, s->xsd, s->act[0]);
    forward(s, (int)n);
    backward(s, (int)n, s->dt, nullptr);
    IRS_CUDA(cudaMemcpyAsync(loss, s->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    check_err(s);
    pack_params(s, s->g, grads);
    SG_END
}

// ---------------------------------------------------- data-parallel training steps
// A training step split so that the gradient can cross devices between its halves:
// irs_surrogate_grad_device leaves the flat gradient (the padded layout of
// irs_surrogate_grad_size) in the caller's device buffer, the caller reduces it over its
// ranks (an NCCL all-reduce), and irs_surrogate_apply_device takes one Adam step from it.
// Both order the library's stream after `stream` on entry and `stream` after their work.
struct StreamJoin {
    cudaEvent_t ev = nullptr;
    cudaStream_t caller = nullptr, own = nullptr;
    StreamJoin(cudaStream_t c, cudaStream_t o) : caller(c), own(o) {
        if (!caller) return;
        IRS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        IRS_CUDA(cudaEventRecord(ev, caller));
        IRS_CUDA(cudaStreamWaitEvent(own, ev, 0));
    }
    void done() {
        if (!caller) return;
        IRS_CUDA(cudaEventRecord(ev, own));
        IRS_CUDA(cudaStreamWaitEvent(caller, ev, 0));
    }
    ~StreamJoin() {
        if (ev) cudaEventDestroy(ev);
    }
};

int irs_surrogate_grad_size(irs_surrogate* s, int64_t* n) {
    SG_BEGIN
    IRS_REQUIRE(s && n, "invalid arguments");
    *n = s->n_par;
    SG_END
}

int irs_surrogate_grad_device(irs_surrogate* s, const float* X_dev, const float* Y_dev, const int32_t* idx_dev,
                              int64_t n, float* g_dev, double* loss, void* stream) {
    SG_BEGIN
    IRS_REQUIRE(s && X_dev && Y_dev && g_dev && n >= 1 && n <= (1 << 20), "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    StreamJoin j((cudaStream_t)stream, st);
    ensure_batch(s, (int)n);
    IRS_CUDA(cudaMemsetAsync(s->loss, 0, sizeof(double), st));
    prep_input_kernel<<<(int)n, 256, 0, st>>>(X_dev, idx_dev, s->n_in, s->pin[0], (int)n, s->xmean, s->xsd,
                                               s->act[0]);
    forward(s, (int)n);
    backward(s, (int)n, Y_dev, idx_dev);
    IRS_CUDA(cudaMemcpyAsync(g_dev, s->g, (size_t)s->n_par * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (loss) {
        IRS_CUDA(cudaMemcpyAsync(loss, s->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
        check_err(s);
    }
    j.done();
    SG_END
}

int irs_surrogate_apply_device(irs_surrogate* s, const float* g_dev, float lr, void* stream) {
    SG_BEGIN
    IRS_REQUIRE(s && g_dev && lr > 0.f, "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    StreamJoin j((cudaStream_t)stream, st);
    s->t_step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)s->t_step), c2 = 1.f - std::pow(b2, (float)s->t_step);
    adam_kernel<<<(unsigned)((s->n_par + 255) / 256), 256, 0, st>>>(s->w, s->m, s->v, g_dev, s->n_par, lr, b1, b2,
                                                                     1e-8f, c1, c2);
    refresh_bf16(s);
    j.done();
    SG_END
}

// inference of n samples already on the device; out [n][n_out] BTs, ood [n] (nullable)
static void infer_device(irs_surrogate* s, const float* dX, int64_t n, float* dOut, float* dOod) {
    const cudaStream_t st = s->stream;
    const int B = (int)std::min<int64_t>(n, 4096);
    ensure_batch(s, B);
    for (int64_t b0 = 0; b0 < n; b0 += B) {
        const int nb = (int)std::min<int64_t>(B, n - b0);
        prep_input_kernel<<<nb, 256, 0, st>>>(dX + b0 * s->n_in, nullptr, s->n_in, s->pin[0], nb, s->xmean, s->xsd,
                                              s->act[0]);
        if (dOod) {  // |W x'|^2 / n_in on the tensor cores from the BF16 scaled inputs
            IRS_CUDA(cudaMemsetAsync(dOod + b0, 0, (size_t)nb * sizeof(float), st));
            umma::EpiArgs eo{};
            eo.Cf = dOod + b0;
            eo.ldc = s->n_in;
            eo.err = s->err;
            gemm<umma::EPI_SUMSQ>(st, s->act[0], s->pin[0], s->white_b, s->pin[0], nb, s->n_in, s->pin[0], eo);
        }
        forward(s, nb, dOut + b0 * s->n_out, s->n_out);
    }
    IRS_CUDA(cudaGetLastError());
}

int irs_surrogate_infer_device(irs_surrogate* s, const float* X_dev, int64_t n, float* out_dev, float* ood_dev,
                               void* stream) {
    SG_BEGIN
    IRS_REQUIRE(s && X_dev && out_dev && n >= 1, "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    cudaEvent_t ev = nullptr;
    if (stream) {
        IRS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        IRS_CUDA(cudaEventRecord(ev, (cudaStream_t)stream));
        IRS_CUDA(cudaStreamWaitEvent(s->stream, ev, 0));
    }
    infer_device(s, X_dev, n, out_dev, ood_dev);
    if (stream) {
        IRS_CUDA(cudaEventRecord(ev, s->stream));
        IRS_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, ev, 0));
        IRS_CUDA(cudaEventDestroy(ev));
    }
    SG_END
}

int irs_surrogate_infer(irs_surrogate* s, const float* X, int64_t n, float* out, float* ood) {
    SG_BEGIN
    IRS_REQUIRE(s && X && out && n >= 1, "invalid arguments");
    IRS_CUDA(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    grow(s->dx, s->dx_cap, n * s->n_in);
    grow(s->dout_buf, s->dout_cap, n * s->n_out);
    grow(s->dood, s->dood_cap, n);
    IRS_CUDA(cudaMemcpyAsync(s->dx, X, (size_t)n * s->n_in * sizeof(float), cudaMemcpyHostToDevice, st));
    infer_device(s, s->dx, n, s->dout_buf, s->dood);
    IRS_CUDA(cudaMemcpyAsync(out, s->dout_buf, (size_t)n * s->n_out * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (ood) IRS_CUDA(cudaMemcpyAsync(ood, s->dood, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st));
    check_err(s);
    SG_END
}

// C[M][N] = A[M][K] B[N][K]^T in BF16 with FP32 output (tests of the tensor-core GEMM)
int irs_gemm_bf16(irs_ctx* ctx, const uint16_t* A, const uint16_t* B, int M, int N, int K, float* C) {
    SG_BEGIN
    IRS_REQUIRE(ctx && A && B && C && M >= 1 && N >= 1 && K >= 1, "invalid arguments");
    IRS_CUDA(cudaSetDevice(ctx->device));
    const cudaStream_t st = ctx->stream;
    const int64_t lk = pad64(K), ln = pad64(N);
    bf16* dA = (bf16*)dmalloc((size_t)M * lk * 2);
    bf16* dB = (bf16*)dmalloc((size_t)N * lk * 2);
    float* dC = (float*)dmalloc((size_t)M * ln * 4);
    int* err = (int*)dmalloc(sizeof(int));
    try {
        IRS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        IRS_CUDA(cudaMemcpy2DAsync(dA, lk * 2, A, (size_t)K * 2, (size_t)K * 2, M, cudaMemcpyHostToDevice, st));
        IRS_CUDA(cudaMemcpy2DAsync(dB, lk * 2, B, (size_t)K * 2, (size_t)K * 2, N, cudaMemcpyHostToDevice, st));
        umma::EpiArgs ep{};
        ep.Cf = dC;
        ep.ldc = (int)ln;
        ep.err = err;
        gemm<umma::EPI_F32>(st, dA, lk, dB, lk, M, N, K, ep);
        IRS_CUDA(cudaMemcpy2DAsync(C, (size_t)N * 4, dC, ln * 4, (size_t)N * 4, M, cudaMemcpyDeviceToHost, st));
        int e = 0;
        IRS_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        IRS_CUDA(cudaStreamSynchronize(st));
        if (e) throw Error{IRS_E_CUDA, "tensor-core GEMM: a pipeline wait timed out"};
    } catch (...) {
        cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(err);
        throw;
    }
    cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(err);
    SG_END
}

}  // extern "C"
