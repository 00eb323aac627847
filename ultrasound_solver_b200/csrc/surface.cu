// z recurrences of the homogeneous surface solver: for every (x, y) mode the
// backward continued fraction H[j] = u[j+1]/u[0] of the z axis operator,
// then the running products (homogeneous_surface.py:41-85, which launches
// one CUDA thread per mode the same way; the reference's CPU path at
// homogeneous_surface.py:144-155 runs the same recurrence in numpy).
#include "usv_internal.cuh"

namespace usv {

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    // a / b = a conj(b) / |b|^2 with b scaled by its larger component first
    const double s = fmax(fabs(b.x), fabs(b.y));
    const double2 bs = make_double2(b.x / s, b.y / s);
    const double d = bs.x * bs.x + bs.y * bs.y;
    return make_double2((a.x * bs.x + a.y * bs.y) / (d * s), (a.y * bs.x - a.x * bs.y) / (d * s));
}

__global__ void __launch_bounds__(128) k_z_transfer(const double2* shift, const double2* diag,
                                                    const double2* upper, const double2* lower,
                                                    double2* history, int modes, int nz) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= modes) return;
    const double2 sh = shift[q];
    double2 ratio = make_double2(0.0, 0.0);
    for (int j = nz - 1; j >= 1; --j) {
        double2 value = cadd(sh, diag[j]);
        if (j < nz - 1) value = cadd(value, cmul(upper[j], ratio));
        const double2 num = make_double2(-lower[j - 1].x, -lower[j - 1].y);
        ratio = cdiv(num, value);
        history[(long long)(j - 1) * modes + q] = ratio;
    }
    for (int j = 1; j < nz - 1; ++j)
        history[(long long)j * modes + q] =
            cmul(history[(long long)j * modes + q], history[(long long)(j - 1) * modes + q]);
}

}  // namespace usv

using namespace usv;

extern "C" {

int usv_z_transfer(const void* shift, const void* diag, const void* upper, const void* lower,
                   void* history, int modes, int nz, void* stream) {
    if (!shift || !diag || !upper || !lower || !history || modes < 1 || nz < 2) return USV_ERR_ARG;
    k_z_transfer<<<(modes + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double2*>(shift), static_cast<const double2*>(diag),
        static_cast<const double2*>(upper), static_cast<const double2*>(lower),
        static_cast<double2*>(history), modes, nz);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

}  // extern "C"
