// oe.cuh -- batched optimal estimation (optimal_estimation.jl:142-291) on the GPU, FP64.
//
//   oe_normal_kernel   M = K^T Se^-1 K and b = K^T Se^-1 r for every active scene
//                      (diagonal Se; K is the FP32 Jacobian [scene][state][channel])
//   oe_solve_kernel    H = (1 + gamma) Sa^-1 + M, Cholesky H = L L^T in shared memory,
//                      dx = H^-1 (b - Sa^-1 (x - xa)), d^2 = dx^T (Sa^-1 dx + M dx)
// Both are persistent launches over an index list of scenes (grid-stride), so scenes
// with uneven iteration counts share one launch per LM stage.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace irs {

constexpr int kOeThreads = 256;   // oe_solve_kernel; oe_normal_kernel takes 256 or 512
constexpr int kOeMaxState = 160;  // the Cholesky's n x n FP64 matrix in shared memory (200 KB)
constexpr int kOePairsPerThread = 32;  // n (n + 1) / 2 pairs <= 32 per thread of oe_normal_kernel
constexpr int kOeTile = 32;       // channels per shared-memory tile

// shared memory: tile [kOeTile][n] of K and of K * w, plus w r per channel.  THREADS
// x 32 pairs cover the upper triangle: 256 threads up to n = 127, 512 up to n = 180.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) oe_normal_kernel(const int* __restrict__ list, int n_list, int n,
                                                            int n_ch, const float* __restrict__ K,
                                                            const double* __restrict__ w,
                                                            const double* __restrict__ r, double* __restrict__ M,
                                                            double* __restrict__ b) {
    extern __shared__ double sh[];
    double* tk = sh;                       // [kOeTile][n]
    double* tw = sh + kOeTile * n;         // [kOeTile][n] (K w)
    double* wr = tw + kOeTile * n;         // [kOeTile]
    const int P = n * (n + 1) / 2;
    int pij[kOePairsPerThread];            // (i << 8) | j, or -1
#pragma unroll
    for (int k = 0; k < kOePairsPerThread; ++k) {
        int p = threadIdx.x + k * THREADS, i = 0;
        if (p < P) {  // row-major upper triangle: row i holds n - i pairs
            while (p >= n - i) {
                p -= n - i;
                ++i;
            }
            pij[k] = (i << 8) | (i + p);
        } else {
            pij[k] = -1;
        }
    }
    for (int a = blockIdx.x; a < n_list; a += gridDim.x) {
        const int s = list[a];
        const float* Ks = K + (size_t)s * n * n_ch;
        const double* ws = w + (size_t)s * n_ch;
        const double* rs = r + (size_t)s * n_ch;
        double acc[kOePairsPerThread];
#pragma unroll
        for (int k = 0; k < kOePairsPerThread; ++k) acc[k] = 0.0;
        double bacc = 0.0;
        for (int c0 = 0; c0 < n_ch; c0 += kOeTile) {
            __syncthreads();
            for (int idx = threadIdx.x; idx < n * kOeTile; idx += THREADS) {
                const int i = idx / kOeTile, c = idx % kOeTile;
                const bool in = c0 + c < n_ch;
                const double kv = in ? (double)Ks[(size_t)i * n_ch + c0 + c] : 0.0;
                tk[c * n + i] = kv;
                tw[c * n + i] = in ? kv * ws[c0 + c] : 0.0;
            }
            for (int c = threadIdx.x; c < kOeTile; c += THREADS)
                wr[c] = c0 + c < n_ch ? ws[c0 + c] * rs[c0 + c] : 0.0;
            __syncthreads();
#pragma unroll 4
            for (int c = 0; c < kOeTile; ++c) {
                const double* rowk = tk + c * n;
                const double* roww = tw + c * n;
#pragma unroll
                for (int k = 0; k < kOePairsPerThread; ++k)
                    if (pij[k] >= 0) acc[k] = fma(rowk[pij[k] >> 8], roww[pij[k] & 255], acc[k]);
                if (threadIdx.x < n) bacc = fma(rowk[threadIdx.x], wr[c], bacc);
            }
        }
        double* Ms = M + (size_t)s * n * n;
#pragma unroll
        for (int k = 0; k < kOePairsPerThread; ++k)
            if (pij[k] >= 0) {
                const int i = pij[k] >> 8, j = pij[k] & 255;
                Ms[(size_t)i * n + j] = acc[k];
                Ms[(size_t)j * n + i] = acc[k];
            }
        if (threadIdx.x < n) b[(size_t)s * n + threadIdx.x] = bacc;
    }
}

// shared memory: H [n][n], g [n], g0 [n], y [n], t [n], and a status word
__global__ void __launch_bounds__(kOeThreads) oe_solve_kernel(const int* __restrict__ list, int n_list, int n,
                                                              const double* __restrict__ M,
                                                              const double* __restrict__ b,
                                                              const double* __restrict__ Sa_inv,
                                                              const double* __restrict__ x,
                                                              const double* __restrict__ xa,
                                                              const double* __restrict__ gamma,
                                                              double* __restrict__ dx, double* __restrict__ d2,
                                                              int* __restrict__ ok) {
    extern __shared__ double sh[];
    double* H = sh;
    double* g = H + (size_t)n * n;
    double* g0 = g + n;
    double* y = g0 + n;
    double* t = y + n;
    __shared__ int fail;
    for (int a = blockIdx.x; a < n_list; a += gridDim.x) {
        const int s = list[a];
        const double gm = gamma[s];
        const double* Ms = M + (size_t)s * n * n;
        const double* xs = x + (size_t)s * n;
        const double* xas = xa + (size_t)s * n;
        __syncthreads();
        if (threadIdx.x == 0) fail = 0;
        for (int idx = threadIdx.x; idx < n * n; idx += kOeThreads) H[idx] = (1.0 + gm) * Sa_inv[idx] + Ms[idx];
        for (int i = threadIdx.x; i < n; i += kOeThreads) t[i] = xs[i] - xas[i];
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kOeThreads) {  // g = b - Sa^-1 (x - xa)
            double v = b[(size_t)s * n + i];
            for (int j = 0; j < n; ++j) v -= Sa_inv[(size_t)i * n + j] * t[j];
            g[i] = v;
            g0[i] = v;
        }
        __syncthreads();
        // right-looking Cholesky, lower triangle in place
        for (int k = 0; k < n; ++k) {
            if (threadIdx.x == 0) {
                const double d = H[(size_t)k * n + k];
                if (!(d > 0.0)) fail = 1;
                H[(size_t)k * n + k] = d > 0.0 ? sqrt(d) : 1.0;
            }
            __syncthreads();
            const double dk = H[(size_t)k * n + k];
            for (int i = k + 1 + threadIdx.x; i < n; i += kOeThreads) H[(size_t)i * n + k] /= dk;
            __syncthreads();
            const int m = n - k - 1;
            for (int idx = threadIdx.x; idx < m * m; idx += kOeThreads) {
                const int i = k + 1 + idx / m, j = k + 1 + idx % m;
                if (j <= i) H[(size_t)i * n + j] -= H[(size_t)i * n + k] * H[(size_t)j * n + k];
            }
            __syncthreads();
        }
        // L y = g
        for (int k = 0; k < n; ++k) {
            if (threadIdx.x == 0) y[k] = g[k] / H[(size_t)k * n + k];
            __syncthreads();
            for (int i = k + 1 + threadIdx.x; i < n; i += kOeThreads) g[i] -= H[(size_t)i * n + k] * y[k];
            __syncthreads();
        }
        // L^T dx = y (dx kept in t)
        for (int k = n - 1; k >= 0; --k) {
            if (threadIdx.x == 0) t[k] = y[k] / H[(size_t)k * n + k];
            __syncthreads();
            for (int i = threadIdx.x; i < k; i += kOeThreads) y[i] -= H[(size_t)k * n + i] * t[k];
            __syncthreads();
        }
        // d^2 = dx^T (Sa^-1 dx + M dx) = dx^T (H dx - gamma Sa^-1 dx) = dx^T g0 - gamma dx^T Sa^-1 dx
        double part = 0.0;
        for (int i = threadIdx.x; i < n; i += kOeThreads) {
            double v = 0.0;
            for (int j = 0; j < n; ++j) v += Sa_inv[(size_t)i * n + j] * t[j];
            part += t[i] * (g0[i] - gm * v);
        }
        for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        __shared__ double red[kOeThreads / 32];
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
        __syncthreads();
        if (threadIdx.x == 0) {
            double v = 0.0;
            for (int w = 0; w < kOeThreads / 32; ++w) v += red[w];
            d2[s] = fail ? 0.0 : v;
            ok[s] = fail ? 0 : 1;
        }
        for (int i = threadIdx.x; i < n; i += kOeThreads) dx[(size_t)s * n + i] = fail ? 0.0 : t[i];
    }
}

// Whitening by a banded Cholesky factor of Se (apodised covariance, covariance.jl:62-81):
// every row x of K for the scenes in `list` (over the kept channels kidx, in order)
// becomes L^-1 x by forward substitution, L[i][k] = L(i, i-k) for k = 0..bw.  Then
// K^T K = K^T Se^-1 K.  One thread per (scene, state row); the recurrence runs in FP64.
constexpr int kOeMaxBand = 32;
__global__ void __launch_bounds__(128) oe_whiten_kernel(const int* __restrict__ list, int n_list, int n,
                                                        int n_ch, float* __restrict__ K, const int* __restrict__ kidx,
                                                        int n_kept, const double* __restrict__ Lb, int bw) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_list * n) return;
    const int s = list[t / n], row = t % n;
    float* x = K + ((size_t)s * n + row) * n_ch;
    const double* L = Lb + (size_t)s * n_kept * (bw + 1);
    double z[kOeMaxBand + 1];  // the last bw values, ring-indexed
    for (int i = 0; i < n_kept; ++i) {
        const double* Li = L + (size_t)i * (bw + 1);
        double v = (double)x[kidx[i]];
        for (int k = 1; k <= bw && k <= i; ++k) v -= Li[k] * z[(i - k) % (kOeMaxBand + 1)];
        v /= Li[0];
        z[i % (kOeMaxBand + 1)] = v;
        x[kidx[i]] = (float)v;
    }
}

}  // namespace irs
