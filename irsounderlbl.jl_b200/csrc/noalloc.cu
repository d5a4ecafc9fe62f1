// noalloc.cu -- cross sections for callers that cannot allocate device memory.
//
// irs_cross_sections_noalloc is compute_voigt_cross_sections (FP64) for callers that
// must not call cudaMalloc themselves or through this library: hosts whose device
// memory is reserved up front by their own allocator (for example a Julia process
// whose CUDA.jl memory pool owns the device and hands this library only the input and
// output buffers), real-time or embedded hosts that forbid allocation after start-up,
// and plug-ins that may not grow a process's device footprint.  The caller passes the
// line list, the TIPS tables, the grid and the output as device pointers; the per-line
// parameters go to the file-scope array below instead of a context workspace.
//
// TIPS: the caller passes up to kNoAllocMaxTips tables packed one after another on the
// device (all on the same 1 K temperature grid) and, on the host, the (mol, iso) of
// each.  Every line takes the table of its own (mol, iso), as Q_ratio does
// (partition.jl:41-47); a line whose (mol, iso) has no table takes Q proportional to T,
// the reference's fallback.
//
// The array is sized for kNoAllocMaxLines lines (5 doubles each, about 5.2 MB) and
// every GPU that loads this library holds it until the process exits.  Every call
// shares it, so calls that overlap on the GPU (concurrent streams, or host threads
// using different streams) race on it: serialise them.  Its contents persist between
// calls; each call rewrites all the entries it reads.  The first call in each CUDA
// context performs a one-time set-up (it looks up the array's device address with
// cudaGetSymbolAddress and uploads the Faddeeva constants); make that first call
// before any stream capture.  The set-up is remembered per context: after
// cudaDeviceReset (which destroys the context and the array's contents with it) the
// process must reload this library before calling it again.
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "faddeeva.cuh"
#include "irs_internal.h"

namespace irs {

constexpr long long kNoAllocMaxLines = 1LL << 17;  // 131,072 lines
constexpr int kNoAllocMaxTips = 64;                // TIPS tables per call

// the (mol, iso) of each packed TIPS table, by value in the kernel's parameters
struct NoAllocTips {
    int mol[kNoAllocMaxTips], iso[kNoAllocMaxTips];
    int n_tab, tmin, n;
};

struct NoAllocScratch {
    double nu0[kNoAllocMaxLines];
    double f[kNoAllocMaxLines];
    double y[kNoAllocMaxLines];
    double Sn[kNoAllocMaxLines];
    double Hc[kNoAllocMaxLines];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

namespace {

__device__ double na_tips(const double* q, int tmin, int n, double T) {  // partition.jl:10-18
    int lo = (int)floor(T) - tmin + 1, hi = lo + 1;
    lo = min(max(lo, 1), n);
    hi = min(max(hi, 1), n);
    const double fr = T - floor(T);
    return q[lo - 1] * (1.0 - fr) + q[hi - 1] * fr;
}

__device__ double na_mass(int mol) {  // broadening.jl:131-148
    const double m[11] = {18.010, 44.010, 47.998, 44.013, 28.010, 16.043, 31.999, 34.015, 64.065, 36.461, 17.031};
    return (mol < 1 || mol > 11) ? 30.0 : m[mol - 1];
}

// per-line parameters (voigt.jl:402-454) from the caller's 56-byte line records
__global__ void na_params_kernel(const irs_line* __restrict__ lines, long long n, const double* __restrict__ q,
                                 NoAllocTips tt, double T, double p, double vs, double cutoff, int method,
                                 double x_far, NoAllocScratch* __restrict__ s) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const irs_line l = lines[j];
    const int mol = l.mol_id;
    const double n_air = (double)l.temp_depend;
    const double n_self = mol == 1 ? 0.95 : (mol == 2 ? 0.75 : n_air);
    const double d_self = mol == 1 ? 0.002 : (mol == 2 ? -0.003 : 0.0);
    const double tr = 296.0 / T;
    const double gl = pow(tr, n_air) * (double)l.air_broad * (1.0 - vs) * p +
                      pow(tr, n_self) * (double)l.self_broad * vs * p;
    const double gd = fmax(l.wavenumber * 3.58126e-7 * sqrt(T / na_mass(mol)), 1e-10);
    int tab = -1;  // this line's (mol, iso) table, partition.jl:41-47
    for (int k = 0; q && k < tt.n_tab; ++k)
        if (tt.mol[k] == mol && tt.iso[k] == (int)l.iso_id) { tab = k; break; }
    const double* qt = tab >= 0 ? q + (size_t)tab * tt.n : nullptr;
    const double Qr = qt ? na_tips(qt, tt.tmin, tt.n, 296.0) / na_tips(qt, tt.tmin, tt.n, T) : 296.0 / T;
    const double c2 = 1.4387752;
    const double S = l.intensity * Qr * exp(-c2 * l.lower_energy * (1.0 / T - 1.0 / 296.0)) *
                     (1.0 - exp(-c2 * l.wavenumber / T)) / (1.0 - exp(-c2 * l.wavenumber / 296.0));
    s->nu0[j] = l.wavenumber + ((double)l.pressure_shift * (1.0 - vs) + d_self * vs) * p;
    if (method == 2) {  // PseudoVoigt, voigt.jl:422-441
        const double fG = 2.0 * gd, fL = 2.0 * gl;
        const double fV = pow(pow(fG, 5.0) + 2.69269 * pow(fG, 4.0) * fL + 2.42843 * pow(fG, 3.0) * (fL * fL) +
                              4.47163 * (fG * fG) * pow(fL, 3.0) + 0.07842 * fG * pow(fL, 4.0) + pow(fL, 5.0), 0.2);
        const double rr = fL / fV, gV = 0.5 * fV;
        const double eta = 1.36603 * rr - 0.47719 * (rr * rr) + 0.11116 * (rr * rr * rr);
        const double Gc = 0.46971863934982566 / gV * exp(-0.69314718055994531 * (cutoff * cutoff) / (gV * gV));
        const double Lc = gV * 0.31830988618379067 / (cutoff * cutoff + gV * gV);
        s->f[j] = gV; s->y[j] = eta; s->Sn[j] = S; s->Hc[j] = S * (eta * Lc + (1.0 - eta) * Gc);
        return;
    }
    const double f = kSqrtLn2 / gd, y = gl * f;
    const double xc = cutoff * f;
    s->f[j] = f;
    s->y[j] = y;
    s->Sn[j] = S * f * kInvSqrtPi;
    s->Hc[j] = fabs(xc) > x_far ? y * kInvSqrtPi / (xc * xc + y * y)
                                : (method == 1 ? weideman24_64(xc, y) : faddeeva64(xc, y).x);
}

__device__ long long na_lower(const double* a, double v, long long n) {  // voigt.jl:220-227
    long long lo = 1, hi = n + 1;
    while (lo < hi) { const long long m = (lo + hi) >> 1; if (a[m - 1] < v) lo = m + 1; else hi = m; }
    return lo;
}
__device__ long long na_upper(const double* a, double v, long long n) {  // voigt.jl:229-236
    long long lo = 0, hi = n;
    while (lo < hi) { const long long m = (lo + hi + 1) >> 1; if (a[m - 1] > v) hi = m - 1; else lo = m; }
    return lo;
}

// voigt.jl:243-313, one thread per grid point
template <int METHOD>
__global__ void na_sum_kernel(const NoAllocScratch* __restrict__ s, long long n, const double* __restrict__ grid,
                              long long n_nu, double cutoff, double x_far, double* __restrict__ sigma) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nu) return;
    const double nu = grid[i];
    const long long jlo = na_lower(s->nu0, nu - cutoff, n), jhi = na_upper(s->nu0, nu + cutoff, n);
    const double rc = 1.0 / cutoff;
    double acc = 0.0;
    for (long long jj = jlo; jj <= jhi; ++jj) {
        const long long j = jj - 1;
        const double d = nu - s->nu0[j];
        const double zr = d * rc;
        if (METHOD == 2) {
            const double gV = s->f[j], eta = s->y[j];
            const double G = 0.46971863934982566 / gV * exp(-0.69314718055994531 * d * d / (gV * gV));
            const double Lz = gV * 0.31830988618379067 / (d * d + gV * gV);
            acc += s->Sn[j] * (eta * Lz + (1.0 - eta) * G) - (2.0 - zr * zr) * s->Hc[j];
        } else {
            const double x = d * s->f[j], y = s->y[j];
            const double H = fabs(x) > x_far ? y * kInvSqrtPi / (x * x + y * y) : hcore64<METHOD>(x, y);
            acc += s->Sn[j] * (H - (2.0 - zr * zr) * s->Hc[j]);
        }
    }
    sigma[i] = fmax(acc, 0.0);
}

// Device address of the scratch array and the Faddeeva constants, once per CUDA
// context (the current one, as the driver reports it).
std::mutex g_mu;
std::map<void*, NoAllocScratch*> g_addr;

void* current_context() {
    typedef int (*GetCtx)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)
    static GetCtx fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult r;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r) != cudaSuccess ||
            r != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (GetCtx)p;
    }();
    if (!fn) throw Error{IRS_E_CUDA, "cuCtxGetCurrent is not available from the driver"};
    int dev = 0;  // cudaSetDevice makes the device's primary context current
    IRS_CUDA(cudaGetDevice(&dev));
    IRS_CUDA(cudaSetDevice(dev));
    void* c = nullptr;
    if (fn(&c) != 0 || !c) throw Error{IRS_E_CUDA, "no current CUDA context"};
    return c;
}

NoAllocScratch* scratch_for_current_context() {
    void* cx = current_context();
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_addr.find(cx);
    if (it != g_addr.end()) return it->second;
    void* ptr = nullptr;
    IRS_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    FaddeevaConsts fc;
    compute_faddeeva_consts(&fc);
    IRS_CUDA(cudaMemcpyToSymbol(c_fad, &fc, sizeof fc));
    g_addr[cx] = (NoAllocScratch*)ptr;
    return (NoAllocScratch*)ptr;
}

}  // namespace
}  // namespace irs

extern "C" int irs_cross_sections_noalloc(const irs_line* d_lines, int64_t n_lines, const double* d_tips_q,
                                          const int32_t* tips_keys, int n_tips, int tips_t_min, int tips_n,
                                          const double* d_grid, int64_t n_nu, double T, double p_atm,
                                          double vmr_self, double cutoff, int method, double x_far,
                                          double* d_sigma, void* stream) {
    using namespace irs;
    try {
        IRS_REQUIRE(n_lines >= 0 && n_lines <= kNoAllocMaxLines,
                    "irs_cross_sections_noalloc: n_lines exceeds the scratch capacity of 131072 lines");
        IRS_REQUIRE(n_nu >= 1 && d_grid && d_sigma && (n_lines == 0 || d_lines), "invalid arguments");
        IRS_REQUIRE(method >= 1 && method <= 3, "method must be 1 (Weideman), 2 (PseudoVoigt) or 3 (FullFaddeeva)");
        IRS_REQUIRE(T > 0.0 && p_atm >= 0.0 && cutoff > 0.0, "T and cutoff must be positive, p_atm non-negative");
        IRS_REQUIRE(n_tips >= 0 && n_tips <= kNoAllocMaxTips,
                    "irs_cross_sections_noalloc: at most 64 TIPS tables per call");
        IRS_REQUIRE(!d_tips_q || n_tips == 0 || (tips_keys && tips_n >= 2),
                    "the TIPS tables need their (mol, iso) keys and at least two points each");
        NoAllocTips tt{};
        tt.n_tab = d_tips_q ? n_tips : 0;
        tt.tmin = tips_t_min;
        tt.n = tips_n;
        for (int k = 0; k < tt.n_tab; ++k) {
            tt.mol[k] = tips_keys[2 * k];
            tt.iso[k] = tips_keys[2 * k + 1];
        }
        NoAllocScratch* s = scratch_for_current_context();
        cudaStream_t st = (cudaStream_t)stream;
        if (n_lines > 0)
            na_params_kernel<<<(unsigned)((n_lines + 255) / 256), 256, 0, st>>>(
                d_lines, n_lines, d_tips_q, tt, T, p_atm, vmr_self, cutoff, method, x_far, s);
        const unsigned g = (unsigned)((n_nu + 255) / 256);
        if (method == 1) na_sum_kernel<1><<<g, 256, 0, st>>>(s, n_lines, d_grid, n_nu, cutoff, x_far, d_sigma);
        else if (method == 2) na_sum_kernel<2><<<g, 256, 0, st>>>(s, n_lines, d_grid, n_nu, cutoff, x_far, d_sigma);
        else na_sum_kernel<3><<<g, 256, 0, st>>>(s, n_lines, d_grid, n_nu, cutoff, x_far, d_sigma);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) throw Error{IRS_E_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e)};
        return IRS_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    }
}
