// Focal losses and their field cotangents on the device (FP64), for
// dL = Re(g^H du) (the reference's convention, which is also torch's).
//
//   USV_LOSS_FOCAL_PRESSURE  FocalPressureLoss.evaluate
//        L = -w_t mean_targets |u_t| + 0.5 w_b mean |u|^2
//        (phase_adjoint_optimizer.py:210-270)
//   USV_LOSS_FOCAL_CONTRAST  FocalContrastLoss.evaluate
//        L = -w_t mean_targets |u_t| + w_s (max + T (log sum exp((|u|-max)/T)
//            - log n)) over the background mask (phase_adjoint_optimizer.py:283-364)
//   USV_LOSS_CONTRAST_RATIO  L = -|u_t|^2 / mean_mask |u|^2 (mean over targets
//        of |u_t|^2; the mask is the focal shell)
//
// Reductions use per-chunk partials and a fixed-order finish, so results are
// deterministic; repeated target indices accumulate like the reference.
#include <cmath>

#include "usv_internal.cuh"

namespace usv {

constexpr int kLossChunk = 4096;

// partial[blk] = {sum |u|^2, sum_mask |u|^2, max_mask |u|, count_mask}
__global__ void __launch_bounds__(256) k_loss_pass1(const double2* u, long long n,
                                                    const unsigned char* mask, double4* partial) {
    __shared__ double sh[32];
    const long long n0 = (long long)blockIdx.x * kLossChunk;
    const long long n1 = min(n0 + kLossChunk, n);
    double s_all = 0.0, s_m = 0.0, mx = 0.0, cnt = 0.0;
    for (long long i = n0 + threadIdx.x; i < n1; i += blockDim.x) {
        const double a2 = cabs2(u[i]);
        s_all += a2;
        if (!mask || mask[i]) {
            s_m += a2;
            mx = fmax(mx, sqrt(a2));
            cnt += 1.0;
        }
    }
    s_all = block_sum(s_all, sh);
    s_m = block_sum(s_m, sh);
    cnt = block_sum(cnt, sh);
    mx = block_max(mx, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double4(s_all, s_m, mx, cnt);
}

// partial2[blk] = sum_mask exp((|u| - max)/T)
__global__ void __launch_bounds__(256) k_loss_pass2(const double2* u, long long n,
                                                    const unsigned char* mask, const double* stat,
                                                    double temperature, double* partial2) {
    __shared__ double sh[32];
    const double mx = stat[2];
    const long long n0 = (long long)blockIdx.x * kLossChunk;
    const long long n1 = min(n0 + kLossChunk, n);
    double s = 0.0;
    for (long long i = n0 + threadIdx.x; i < n1; i += blockDim.x)
        if (!mask || mask[i]) s += exp((sqrt(cabs2(u[i])) - mx) / temperature);
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial2[blockIdx.x] = s;
}

// stat = {sum |u|^2, sum_mask |u|^2, max_mask |u|, count_mask, sum exp}
__global__ void k_loss_finish1(const double4* partial, int nblk, double* stat) {
    __shared__ double sh[32];
    double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
    for (int q = threadIdx.x; q < nblk; q += blockDim.x) {
        const double4 p = partial[q];
        a += p.x;
        b += p.y;
        c = fmax(c, p.z);
        d += p.w;
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    d = block_sum(d, sh);
    c = block_max(c, sh);
    if (threadIdx.x == 0) {
        stat[0] = a;
        stat[1] = b;
        stat[2] = c;
        stat[3] = d;
    }
}

__global__ void k_loss_finish2(const double* partial2, int nblk, double* stat) {
    __shared__ double sh[32];
    double a = 0.0;
    for (int q = threadIdx.x; q < nblk; q += blockDim.x) a += partial2[q];
    a = block_sum(a, sh);
    if (threadIdx.x == 0) stat[4] = a;
}

struct LossArgs {
    int mode;
    double target_weight, background_weight, temperature, eps;
    long long n;
    int n_targets;
};

// Loss value (single thread) from the statistics and the target samples.
__global__ void k_loss_value(LossArgs a, const double2* u, const long long* targets,
                             const double* stat, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mean_amp = 0.0, mean_pow = 0.0;
    for (int t = 0; t < a.n_targets; ++t) {
        const double2 v = u[targets[t]];
        mean_amp += sqrt(cabs2(v));
        mean_pow += cabs2(v);
    }
    mean_amp /= a.n_targets;
    mean_pow /= a.n_targets;
    double loss = 0.0;
    if (a.mode == USV_LOSS_FOCAL_PRESSURE) {
        loss = -a.target_weight * mean_amp;
        if (a.background_weight > 0) loss += 0.5 * a.background_weight * stat[0] / double(a.n);
    } else if (a.mode == USV_LOSS_FOCAL_CONTRAST) {
        loss = -a.target_weight * mean_amp;
        loss += a.background_weight *
                (stat[2] + a.temperature * (log(stat[4]) - log(stat[3])));
    } else {
        const double shell = stat[1] / stat[3];
        loss = -mean_pow / shell;
    }
    out[0] = loss;
    out[1] = mean_amp;
    out[2] = mean_pow;
}

// Field cotangent: background/mask terms elementwise.
__global__ void __launch_bounds__(256) k_loss_cot(LossArgs a, const double2* u,
                                                  const unsigned char* mask, const double* stat,
                                                  const double* val, double2* cot) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n;
         i += (long long)gridDim.x * blockDim.x) {
        const double2 v = u[i];
        double2 g = make_double2(0.0, 0.0);
        const bool in = !mask || mask[i];
        if (a.mode == USV_LOSS_FOCAL_PRESSURE) {
            if (a.background_weight > 0) g = cscale(v, a.background_weight / double(a.n));
        } else if (a.mode == USV_LOSS_FOCAL_CONTRAST) {
            if (in) {
                const double amp = sqrt(cabs2(v));
                const double p = exp((amp - stat[2]) / a.temperature) / stat[4];
                g = cscale(v, a.background_weight * p / (amp + a.eps));
            }
        } else if (in) {
            // d(-P/S)/du_i = P/S^2 dS,  S = sum_mask |u|^2 / count
            const double S = stat[1] / stat[3];
            g = cscale(v, 2.0 * val[2] / (S * S * stat[3]));
        }
        cot[i] = g;
    }
}

// Target terms, added in target order by one thread (repeated indices accumulate).
__global__ void k_loss_targets(LossArgs a, const double2* u, const long long* targets,
                               const double* stat, double2* cot) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int t = 0; t < a.n_targets; ++t) {
        const long long i = targets[t];
        const double2 v = u[i];
        double2 g;
        if (a.mode == USV_LOSS_CONTRAST_RATIO) {
            const double S = stat[1] / stat[3];
            g = cscale(v, -2.0 / (S * a.n_targets));
        } else {
            const double amp = sqrt(cabs2(v));
            g = cscale(v, -a.target_weight / a.n_targets / (amp + a.eps));
        }
        cot[i] = cadd(cot[i], g);
    }
}

static unsigned grid1(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 32) b = 148LL * 32;
    return unsigned(b < 1 ? 1 : b);
}

}  // namespace usv

using namespace usv;

extern "C" {

int usv_loss_workspace_bytes(int64_t n, size_t* bytes) {
    if (n < 1 || !bytes) return USV_ERR_ARG;
    const long long nblk = (n + kLossChunk - 1) / kLossChunk;
    *bytes = sizeof(double4) * nblk + sizeof(double) * nblk + sizeof(double) * 8;
    return USV_OK;
}

int usv_loss(int mode, const void* field, int64_t n, const unsigned char* mask,
             const int64_t* targets, int n_targets, double target_weight,
             double background_weight, double temperature, double eps, double* value,
             void* cotangent, void* workspace, size_t workspace_bytes, void* stream) {
    if (!field || n < 1 || !targets || n_targets < 1 || !value || !workspace) return USV_ERR_ARG;
    if (mode < USV_LOSS_FOCAL_PRESSURE || mode > USV_LOSS_CONTRAST_RATIO) return USV_ERR_ARG;
    if (mode == USV_LOSS_FOCAL_CONTRAST && !(temperature > 0)) return USV_ERR_ARG;
    size_t need = 0;
    usv_loss_workspace_bytes(n, &need);
    if (workspace_bytes < need) return USV_ERR_WORKSPACE;
    const int nblk = int((n + kLossChunk - 1) / kLossChunk);
    char* ws = static_cast<char*>(workspace);
    double4* p1 = reinterpret_cast<double4*>(ws);
    double* p2 = reinterpret_cast<double*>(ws + sizeof(double4) * nblk);
    double* stat = p2 + nblk;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double2* u = static_cast<const double2*>(field);
    const long long* tg = reinterpret_cast<const long long*>(targets);
    LossArgs a{mode, target_weight, background_weight, temperature, eps, n, n_targets};
    k_loss_pass1<<<nblk, 256, 0, s>>>(u, n, mask, p1);
    k_loss_finish1<<<1, 256, 0, s>>>(p1, nblk, stat);
    if (mode == USV_LOSS_FOCAL_CONTRAST) {
        k_loss_pass2<<<nblk, 256, 0, s>>>(u, n, mask, stat, temperature, p2);
        k_loss_finish2<<<1, 256, 0, s>>>(p2, nblk, stat);
    }
    k_loss_value<<<1, 32, 0, s>>>(a, u, tg, stat, value);
    if (cotangent) {
        double2* cot = static_cast<double2*>(cotangent);
        k_loss_cot<<<grid1(n), 256, 0, s>>>(a, u, mask, stat, value, cot);
        k_loss_targets<<<1, 32, 0, s>>>(a, u, tg, stat, cot);
    }
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

}  // extern "C"
