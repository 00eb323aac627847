// Phase response basis on the device: u = G e^{i phi}, the phase VJP
// Re(conj(G^H g) i e^{i phi}) and trilinear target rows
// (phase_response_basis.py:139-253). G is stored as M columns of N complex
// values (complex64 or complex128), column m = field of transducer m at its
// amplitude and zero phase. Accumulation is FP64.
#include <cmath>

#include "usv_internal.cuh"

namespace usv {

template <typename C2>
__global__ void __launch_bounds__(256) k_field(const C2* G, long long N, int M,
                                               const double* phases, double2* out) {
    extern __shared__ double2 w[];
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        double s, c;
        sincos(phases[m], &s, &c);
        w[m] = make_double2(c, s);
    }
    __syncthreads();
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N;
         n += (long long)gridDim.x * blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int m = 0; m < M; ++m) acc = cadd(acc, cmul(to_d(G[(long long)m * N + n]), w[m]));
        out[n] = acc;
    }
}

// partial[m][blk] = sum over the block's nodes of conj(G_m) g
template <typename C2>
__global__ void __launch_bounds__(256) k_basis_dots(const C2* G, long long N, int M, int chunk,
                                                    const double2* g, double2* partial) {
    const int m = blockIdx.y;
    __shared__ double sh[32];
    const long long n0 = (long long)blockIdx.x * chunk;
    const long long n1 = min(n0 + chunk, N);
    const C2* col = G + (long long)m * N;
    double re = 0.0, im = 0.0;
    for (long long n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
        const double2 a = to_d(col[n]), b = g[n];
        re = fma(a.x, b.x, fma(a.y, b.y, re));
        im = fma(a.x, b.y, fma(-a.y, b.x, im));
    }
    re = block_sum(re, sh);
    im = block_sum(im, sh);
    if (threadIdx.x == 0) partial[(long long)m * gridDim.x + blockIdx.x] = make_double2(re, im);
}

__global__ void k_basis_finish(const double2* partial, int nblk, int M, const double* phases,
                               double2* response, double* grad) {
    __shared__ double sh[32];
    const int m = blockIdx.x;
    double re = 0.0, im = 0.0;
    for (int q = threadIdx.x; q < nblk; q += blockDim.x) {
        re += partial[(long long)m * nblk + q].x;
        im += partial[(long long)m * nblk + q].y;
    }
    re = block_sum(re, sh);
    im = block_sum(im, sh);
    if (threadIdx.x == 0) {
        if (response) response[m] = make_double2(re, im);
        if (grad) {
            double s, c;
            sincos(phases[m], &s, &c);
            // Re(conj(r) * i e^{i phi}) = Re((re - i im)(-s + i c))
            grad[m] = -re * s + im * c;
        }
    }
}

template <typename C2>
__global__ void k_target(const C2* G, long long nx, long long ny, long long nz, int M,
                         const double* pts, int P, double dx, double2* out) {
    const long long total = (long long)P * M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int p = int(t / M), m = int(t % M);
        const long long dims[3] = {nx, ny, nz};
        long long lo[3];
        double fr[3];
        bool finite = true;
        for (int a = 0; a < 3; ++a) {
            const double pos = pts[3 * p + a] / dx;
            finite = finite && isfinite(pos);
            // the low corner stays in [0, dims-2] (clamped before the integer
            // conversion): a point outside the grid extrapolates from the edge
            // cell, a non-finite one gives NaN, and no load leaves G
            const double l = fmin(fmax(floor(pos), 0.0), double(dims[a] - 2));
            lo[a] = finite ? (long long)l : 0;
            fr[a] = pos - l;
        }
        if (!finite) {
            out[t] = make_double2(nan(""), nan(""));
            continue;
        }
        const long long N = nx * ny * nz;
        double2 acc = make_double2(0.0, 0.0);
        for (int corner = 0; corner < 8; ++corner) {
            const int ci = (corner >> 2) & 1, cj = (corner >> 1) & 1, ck = corner & 1;
            const double w = (ci ? fr[0] : 1 - fr[0]) * (cj ? fr[1] : 1 - fr[1]) *
                             (ck ? fr[2] : 1 - fr[2]);
            const long long row = (lo[0] + ci) + nx * ((lo[1] + cj) + ny * (lo[2] + ck));
            acc = cadd(acc, cscale(to_d(G[(long long)m * N + row]), w));
        }
        out[t] = acc;
    }
}

static unsigned grid1(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 32) b = 148LL * 32;
    return unsigned(b < 1 ? 1 : b);
}

static const int kBasisChunk = 8192;

}  // namespace usv

using namespace usv;

extern "C" {

int usv_basis_field(const void* basis, int64_t n, int m, int prec, const double* phases,
                    void* field, void* stream) {
    if (!basis || n < 1 || m < 1 || m > 3072 || !phases || !field) return USV_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t smem = sizeof(double2) * m;
    if (prec == USV_PREC_MIXED)
        k_field<float2><<<grid1(n), 256, smem, s>>>(static_cast<const float2*>(basis), n, m,
                                                    phases, static_cast<double2*>(field));
    else if (prec == USV_PREC_FP64)
        k_field<double2><<<grid1(n), 256, smem, s>>>(static_cast<const double2*>(basis), n, m,
                                                     phases, static_cast<double2*>(field));
    else
        return USV_ERR_ARG;
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

int usv_basis_adjoint_workspace_bytes(int64_t n, int m, size_t* bytes) {
    if (n < 1 || m < 1 || !bytes) return USV_ERR_ARG;
    const long long nblk = (n + kBasisChunk - 1) / kBasisChunk;
    *bytes = sizeof(double2) * size_t(nblk) * size_t(m);
    return USV_OK;
}

int usv_basis_adjoint(const void* basis, int64_t n, int m, int prec, const void* cotangent,
                      const double* phases, double* response, double* grad, void* workspace,
                      size_t workspace_bytes, void* stream) {
    if (!basis || n < 1 || m < 1 || m > 65535 || !cotangent || !phases || !workspace)
        return USV_ERR_ARG;
    size_t need = 0;
    usv_basis_adjoint_workspace_bytes(n, m, &need);
    if (workspace_bytes < need) return USV_ERR_WORKSPACE;
    const int nblk = int((n + kBasisChunk - 1) / kBasisChunk);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double2* part = static_cast<double2*>(workspace);
    dim3 grid(nblk, m);
    if (prec == USV_PREC_MIXED)
        k_basis_dots<float2><<<grid, 256, 0, s>>>(static_cast<const float2*>(basis), n, m,
                                                  kBasisChunk, static_cast<const double2*>(cotangent), part);
    else if (prec == USV_PREC_FP64)
        k_basis_dots<double2><<<grid, 256, 0, s>>>(static_cast<const double2*>(basis), n, m,
                                                   kBasisChunk, static_cast<const double2*>(cotangent), part);
    else
        return USV_ERR_ARG;
    USV_CUDA_TRY(cudaGetLastError());
    k_basis_finish<<<m, 256, 0, s>>>(part, nblk, m, phases, reinterpret_cast<double2*>(response), grad);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

int usv_basis_target_response(const void* basis, int64_t nx, int64_t ny, int64_t nz, int m,
                              int prec, const double* points, int p, double dx, void* out,
                              void* stream) {
    if (!basis || nx < 2 || ny < 2 || nz < 2 || m < 1 || !points || p < 1 || !(dx > 0) || !out)
        return USV_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long total = (long long)p * m;
    if (prec == USV_PREC_MIXED)
        k_target<float2><<<grid1(total), 256, 0, s>>>(static_cast<const float2*>(basis), nx, ny, nz,
                                                      m, points, p, dx, static_cast<double2*>(out));
    else if (prec == USV_PREC_FP64)
        k_target<double2><<<grid1(total), 256, 0, s>>>(static_cast<const double2*>(basis), nx, ny,
                                                       nz, m, points, p, dx, static_cast<double2*>(out));
    else
        return USV_ERR_ARG;
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// No-allocation variant of usv_basis_adjoint.
//
// Some callers cannot allocate device memory when they need the phase
// gradient: an application that hands all device memory to its own pool at
// start-up, a real-time control loop that must not pay cudaMalloc latency or
// risk an out-of-memory failure mid-run, or host code running while a CUDA
// graph is being captured (where cudaMalloc is not allowed). For them the
// per-chunk partial sums live in the file-scope array below instead of a
// caller workspace. It is 1 MiB and every GPU that loads this library keeps it
// until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace usv {

constexpr long long kNoAllocPartials = 1LL << 16;  // double2 entries = 1 MiB
constexpr int kNoAllocMaxEmitters = 4096;
static __device__ __align__(256) double2 g_noalloc_partials[kNoAllocPartials];

// Same partial sums as k_basis_dots, but each CTA walks chunk, chunk+nblk, ...
// so the partial count nblk*M stays inside the static array for any N.
template <typename C2>
__global__ void __launch_bounds__(256) k_basis_dots_strided(const C2* G, long long N, int chunk,
                                                            const double2* g, double2* partial) {
    const int m = blockIdx.y;
    __shared__ double sh[32];
    const C2* col = G + (long long)m * N;
    double re = 0.0, im = 0.0;
    for (long long n0 = (long long)blockIdx.x * chunk; n0 < N; n0 += (long long)gridDim.x * chunk) {
        const long long n1 = min(n0 + chunk, N);
        for (long long n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
            const double2 a = to_d(col[n]), b = g[n];
            re = fma(a.x, b.x, fma(a.y, b.y, re));
            im = fma(a.x, b.y, fma(-a.y, b.x, im));
        }
    }
    re = block_sum(re, sh);
    im = block_sum(im, sh);
    if (threadIdx.x == 0) partial[(long long)m * gridDim.x + blockIdx.x] = make_double2(re, im);
}

// Device address of g_noalloc_partials, resolved once per device and cached
// for the life of the process; a cudaDeviceReset invalidates the cached
// address, so this entry point must not be used on a device after a reset.
static int noalloc_scratch(double2** out) {
    static std::mutex lock;
    static void* addr[256] = {};
    int dev = 0;
    USV_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return USV_ERR_ARG;
    std::lock_guard<std::mutex> guard(lock);
    if (!addr[dev]) {
        void* p = nullptr;
        USV_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_partials));
        addr[dev] = p;
    }
    *out = static_cast<double2*>(addr[dev]);
    return USV_OK;
}

}  // namespace usv

extern "C" int usv_basis_adjoint_noalloc(const void* basis, int64_t n, int m, int prec,
                                         const void* cotangent, const double* phases,
                                         double* response, double* grad, void* stream) {
    using namespace usv;
    if (!basis || n < 1 || m < 1 || !cotangent || !phases) return USV_ERR_ARG;
    if (m > kNoAllocMaxEmitters) return USV_ERR_TOO_LARGE;
    if (prec != USV_PREC_MIXED && prec != USV_PREC_FP64) return USV_ERR_ARG;
    double2* part = nullptr;
    int st = noalloc_scratch(&part);
    if (st) return st;
    const long long chunks = (n + kBasisChunk - 1) / kBasisChunk;
    const long long cap = kNoAllocPartials / m;
    const int nblk = int(chunks < cap ? chunks : cap);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    dim3 grid(nblk, m);
    // every partial slot [m][0..nblk) is written before k_basis_finish reads it,
    // so stale contents of the shared array never reach the result
    if (prec == USV_PREC_MIXED)
        k_basis_dots_strided<float2><<<grid, 256, 0, s>>>(static_cast<const float2*>(basis), n,
                                                          kBasisChunk,
                                                          static_cast<const double2*>(cotangent), part);
    else
        k_basis_dots_strided<double2><<<grid, 256, 0, s>>>(static_cast<const double2*>(basis), n,
                                                           kBasisChunk,
                                                           static_cast<const double2*>(cotangent), part);
    USV_CUDA_TRY(cudaGetLastError());
    k_basis_finish<<<m, 256, 0, s>>>(part, nblk, m, phases, reinterpret_cast<double2*>(response),
                                     grad);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}
