// Scene set-up on the device: obstacle material blend, sinc_neumann aperture
// deposition, source right-hand sides, the phase gradient through the source
// columns and the material VJP.
//
// Parity:
//   usv_materials_blend   warp_utils.py:11-23 (blend), 57-73 (sphere SDF, h)
//   usv_source_masses     sinc_aperture.py:36-72 (bilinear unit-mass deposition)
//                         and the overlap checks of warp_utils.py:105-113
//   usv_source_rhs        sinc_aperture.py:75-85, warp_utils.py:118-120
//   usv_source_phase_grad phase_response_basis.py:208-253 with G = A^-1 B diag(a)
//   usv_material_vjp      conservative_helmholtz.py:151-175
#include <cmath>
#include <vector>

#include "usv_internal.cuh"

namespace usv {

__global__ void __launch_bounds__(256)
k_blend(int nx, int ny, int nz, double dx, const double* sdf, double cx, double cy, double cz,
        double radius, double width, double rho_o, double c_o, const double* rho_m,
        const double* c_m, double rho0, double c0, double* rho, double* c) {
    const long long N = (long long)nx * ny * nz;
    const double inv_rho_o = 1.0 / rho_o;
    const double comp_o = 1.0 / (rho_o * c_o * c_o);
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N;
         n += (long long)gridDim.x * blockDim.x) {
        double d;
        if (sdf) {
            d = sdf[n];
        } else {
            const Node p = decode(n, nx, ny);
            const double x = p.i * dx - cx, y = p.j * dx - cy, z = p.k * dx - cz;
            d = sqrt(x * x + y * y + z * z) - radius;
        }
        double h;
        if (width > 0) {
            double t = fmin(fmax(d / width, -1.0), 1.0);
            h = 0.5 * (1.0 + t + sin(M_PI * t) / M_PI);
        } else {
            h = d > 0 ? 1.0 : 0.0;
        }
        const double rm = rho_m ? rho_m[n] : rho0;
        const double cm = c_m ? c_m[n] : c0;
        const double inv_rho = inv_rho_o + (1.0 / rm - inv_rho_o) * h;
        const double comp = comp_o + (1.0 / (rm * cm * cm) - comp_o) * h;
        rho[n] = 1.0 / inv_rho;
        c[n] = sqrt(inv_rho / comp);
    }
}

// One CTA per emitter; each thread owns one node of the emitter's bounding
// box and gathers, in the reference's summation order (corner-major, then
// quadrature order), the bilinear masses that land on it. Deterministic, no
// atomics.
__global__ void __launch_bounds__(256)
k_deposit(int nx, int ny, double dx, const double* centers, const double* qx,
          const double* qy, const double* qw, int q, double diameter, double* masses) {
    const int m = blockIdx.x;
    const double cx = centers[3 * m], cy = centers[3 * m + 1];
    const int x0 = int(floor((cx - 0.5 * diameter) / dx)) - 1;
    const int y0 = int(floor((cy - 0.5 * diameter) / dx)) - 1;
    const int x1 = int(floor((cx + 0.5 * diameter) / dx)) + 2;
    const int y1 = int(floor((cy + 0.5 * diameter) / dx)) + 2;
    const int bw = x1 - x0 + 1, bh = y1 - y0 + 1;
    double* col = masses + (long long)m * nx * ny;
    for (int t = threadIdx.x; t < bw * bh; t += blockDim.x) {
        const int ix = x0 + t % bw, iy = y0 + t / bw;
        if (ix < 0 || iy < 0 || ix >= nx || iy >= ny) continue;
        double acc = 0.0;
        for (int corner = 0; corner < 4; ++corner) {
            const int a = corner >> 1, b = corner & 1;
            for (int k = 0; k < q; ++k) {
                const double px = (cx + qx[k]) / dx, py = (cy + qy[k]) / dx;
                const double fx0 = floor(px), fy0 = floor(py);
                if (int(fx0) + a != ix || int(fy0) + b != iy) continue;
                const double fx = px - fx0, fy = py - fy0;
                acc += qw[k] * (a ? fx : 1.0 - fx) * (b ? fy : 1.0 - fy);
            }
        }
        col[(long long)iy * nx + ix] = acc;
    }
}

// flags: bit0 a deposited node lies in the PML, bit1 on a soft face
__global__ void k_source_check(int nx, int ny, int m_emitters, const double* masses,
                               const double2* Tx, const double2* Ty, const double2* Tz,
                               unsigned soft, int nz, int* flag) {
    const long long nxy = (long long)nx * ny;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nxy;
         n += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int m = 0; m < m_emitters; ++m) s += fabs(masses[m * nxy + n]);
        if (s <= 0) continue;
        const int i = int(n % nx), j = int(n / nx);
        if (Tx[i].y + Ty[j].y + Tz[0].y > 0) atomicOr(flag, 1);
        if (node_fixed(soft, i, j, 0, nx, ny, nz)) atomicOr(flag, 2);
    }
}

__global__ void __launch_bounds__(256)
k_source_rhs(long long nxy, long long N, int m_emitters, const double* masses,
             const double2* coeff, double scale, double2* rhs, long long ld) {
    const int b = blockIdx.y;
    const double2* cb = coeff + (long long)b * m_emitters;
    double2* out = rhs + b * ld;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N;
         n += (long long)gridDim.x * blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        if (n < nxy) {
            for (int m = 0; m < m_emitters; ++m) {
                const double w = masses[m * nxy + n];
                if (w != 0.0) acc = cadd(acc, cscale(cb[m], scale * w));
            }
        }
        out[n] = acc;
    }
}

__global__ void __launch_bounds__(256)
k_source_grad(long long nxy, const double* masses, const double2* lam, const double* phases,
              const double* amps, double scale, double* grad) {
    __shared__ double sh[32];
    const int m = blockIdx.x;
    double re = 0.0, im = 0.0;
    for (long long n = threadIdx.x; n < nxy; n += blockDim.x) {
        const double w = masses[m * nxy + n];
        re += w * lam[n].x;
        im += w * lam[n].y;
    }
    re = block_sum(re, sh);
    im = block_sum(im, sh);
    if (threadIdx.x == 0) {
        // r = (B^H lam)_m ; grad = Re(conj(a r) * i e^{i phi})
        const double a = amps ? amps[m] : 1.0;
        const double rr = a * scale * re, ri = a * scale * im;
        double sp, cp;
        sincos(phases[m], &sp, &cp);
        // conj(r) * (i e^{i phi}) = (rr - i ri)(-sp + i cp); real part:
        grad[m] += -rr * sp + ri * cp;
    }
}

// dL = -Re(lambda^H dA u): mass, edge (density) and open-face terms.
__global__ void __launch_bounds__(256)
k_material_vjp(OpView<double> op, const double* rho, const double* c, double omega,
               double dx, int open_mask, const double2* u, const double2* lam_in,
               double* g_rho, double* g_c) {
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < op.n;
         n += (long long)gridDim.x * blockDim.x) {
        const Node p = decode(n, op.nx, op.ny);
        auto lam_at = [&](long long m, int i, int j, int k) {
            return node_fixed(op.soft, i, j, k, op.nx, op.ny, op.nz) ? make_double2(0.0, 0.0)
                                                                      : lam_in[m];
        };
        const double r = rho[n], cc = c[n];
        const double2 un = u[n];
        const double2 ln = lam_at(n, p.i, p.j, p.k);
        const double2 tx = op.T[0][p.i], ty = op.T[1][p.j], tz = op.T[2][p.k];
        const double2 mass = cscale(cmul(cmul(tx, ty), tz), omega * omega / (r * cc * cc));
        const double2 prod = cmul(cmulc(ln, un), mass);
        double gr = prod.x / r;
        double gc = 2.0 * prod.x / cc;
        const double2 fyz = cmul(ty, tz), fxz = cmul(tx, tz), fxy = cmul(tx, ty);
        auto edge = [&](long long m, int i, int j, int k, double2 F) {
            const double s = r + rho[m];
            const double2 dr = cscale(F, -2.0 / (s * s));
            const double2 lm = lam_at(m, i, j, k);
            // (conj(l_lo) - conj(l_hi)) (u_hi - u_lo) is symmetric in lo/hi
            const double2 dl = make_double2(ln.x - lm.x, -(ln.y - lm.y));
            const double2 du = csub(u[m], un);
            gr += -cmul(cmul(dl, du), dr).x;
        };
        const long long sy = op.nx, sz = (long long)op.nx * op.ny;
        if (p.i > 0) edge(n - 1, p.i - 1, p.j, p.k, cmul(fyz, op.Q[0][p.i - 1]));
        if (p.i < op.nx - 1) edge(n + 1, p.i + 1, p.j, p.k, cmul(fyz, op.Q[0][p.i]));
        if (p.j > 0) edge(n - sy, p.i, p.j - 1, p.k, cmul(fxz, op.Q[1][p.j - 1]));
        if (p.j < op.ny - 1) edge(n + sy, p.i, p.j + 1, p.k, cmul(fxz, op.Q[1][p.j]));
        if (p.k > 0) edge(n - sz, p.i, p.j, p.k - 1, cmul(fxy, op.Q[2][p.k - 1]));
        if (p.k < op.nz - 1) edge(n + sz, p.i, p.j, p.k + 1, cmul(fxy, op.Q[2][p.k]));
        const int coord[3] = {p.i, p.j, p.k};
        const int dims[3] = {op.nx, op.ny, op.nz};
        for (int f = 0; f < 6; ++f) {
            if (!(open_mask & (1 << f))) continue;
            const int axis = f >> 1;
            if (coord[axis] != ((f & 1) ? dims[axis] - 1 : 0)) continue;
            const double2 area = cscale(axis == 0 ? fyz : (axis == 1 ? fxz : fxy), 1.0 / dx);
            const double2 term = cmul(make_double2(0.0, omega), cscale(area, 1.0 / (r * cc)));
            const double contrib = cmul(cmulc(ln, un), term).x;
            gr += contrib / r;
            gc += contrib / cc;
        }
        g_rho[n] = gr;
        g_c[n] = gc;
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

int usv_materials_blend(const usv_scene* scene, const double* sdf, const double* center,
                        double radius, double width, double rho_obstacle, double c_obstacle,
                        const double* rho_medium, const double* c_medium, double rho0, double c0,
                        double* rho, double* c, void* stream) {
    if (!scene || !rho || !c) return USV_ERR_ARG;
    if (!sdf && (!center || !(radius >= 0))) return USV_ERR_ARG;
    if (!(width >= 0) || !std::isfinite(width) || !(rho_obstacle > 0) || !(c_obstacle > 0))
        return USV_ERR_ARG;
    const usv_scene& s = *scene;
    const long long N = (long long)s.nx * s.ny * s.nz;
    const double cx = center ? center[0] : 0, cy = center ? center[1] : 0,
                 cz = center ? center[2] : 0;
    k_blend<<<grid1(N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        s.nx, s.ny, s.nz, s.dx, sdf, cx, cy, cz, radius, width, rho_obstacle, c_obstacle,
        rho_medium, c_medium, rho0, c0, rho, c);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

// `masses` holds nx*ny*M doubles followed by one spare double used as the
// check-flag word; `op_buf` must be built for the same scene (PML tables).
int usv_source_masses(const usv_scene* scene, const void* op_buf,
                              const double* centers_host, const double* centers_dev,
                              int m_emitters, double diameter, const double* quad_x,
                              const double* quad_y, const double* quad_w, int q_points,
                              double* masses, void* stream) {
    if (!scene || !op_buf || !centers_host || !centers_dev || m_emitters < 1 || !quad_x ||
        !quad_y || !quad_w || q_points < 1 || !masses)
        return USV_ERR_ARG;
    const usv_scene& s = *scene;
    if (s.nx < 3 || s.ny < 3 || !(diameter > 0) || !std::isfinite(diameter)) return USV_ERR_ARG;
    const double ex = (s.nx - 1) * s.dx, ey = (s.ny - 1) * s.dx;
    for (int m = 0; m < m_emitters; ++m) {
        const double x = centers_host[3 * m], y = centers_host[3 * m + 1],
                     z = centers_host[3 * m + 2];
        if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z) || z != 0.0)
            return USV_ERR_ARG;
        if (x - diameter / 2 < s.dx || y - diameter / 2 < s.dx || x + diameter / 2 > ex - s.dx ||
            y + diameter / 2 > ey - s.dx)
            return USV_ERR_SOURCE_CLEARANCE;
    }
    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    const long long nxy = (long long)s.nx * s.ny;
    USV_CUDA_TRY(cudaMemsetAsync(masses, 0, sizeof(double) * (nxy * m_emitters + 1), strm));
    k_deposit<<<m_emitters, 256, 0, strm>>>(s.nx, s.ny, s.dx, centers_dev, quad_x, quad_y, quad_w,
                                            q_points, diameter, masses);
    USV_CUDA_TRY(cudaGetLastError());
    const OpView<double> op = make_view<double>(s, op_buf, false);
    int* flag = reinterpret_cast<int*>(masses + nxy * m_emitters);
    k_source_check<<<grid1(nxy), 256, 0, strm>>>(s.nx, s.ny, m_emitters, masses, op.T[0],
                                                 op.T[1], op.T[2], op.soft, s.nz, flag);
    USV_CUDA_TRY(cudaGetLastError());
    int h = 0;
    USV_CUDA_TRY(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, strm));
    USV_CUDA_TRY(cudaStreamSynchronize(strm));
    if (h & 1) return USV_ERR_SOURCE_PML;
    if (h & 2) return USV_ERR_SOURCE_SOFT;
    return USV_OK;
}

int usv_source_rhs(const usv_scene* scene, const double* masses, int m_emitters,
                   const double* coeff, double rho_ref, void* rhs, int nrhs, int64_t ld,
                   void* stream) {
    if (!scene || !masses || m_emitters < 1 || !coeff || !rhs || nrhs < 1 || nrhs > 65535 ||
        !(rho_ref > 0))
        return USV_ERR_ARG;
    const usv_scene& s = *scene;
    const long long N = (long long)s.nx * s.ny * s.nz, nxy = (long long)s.nx * s.ny;
    if (ld < N) return USV_ERR_ARG;
    const double scale = -2.0 * M_PI / (rho_ref * s.dx * s.dx * s.dx);
    dim3 grid(grid1(N), nrhs);
    k_source_rhs<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        nxy, N, m_emitters, masses, reinterpret_cast<const double2*>(coeff), scale,
        static_cast<double2*>(rhs), ld);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

int usv_source_phase_grad(const usv_scene* scene, const double* masses, int m_emitters,
                          const void* lam, const double* phases, const double* amplitudes,
                          double rho_ref, double* grad, void* stream) {
    if (!scene || !masses || m_emitters < 1 || !lam || !phases || !grad || !(rho_ref > 0))
        return USV_ERR_ARG;
    const usv_scene& s = *scene;
    const double scale = -2.0 * M_PI / (rho_ref * s.dx * s.dx * s.dx);
    k_source_grad<<<m_emitters, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        (long long)s.nx * s.ny, masses, static_cast<const double2*>(lam), phases, amplitudes,
        scale, grad);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

int usv_material_vjp(const usv_scene* scene, const void* op_buf, const double* rho,
                     const double* c, const void* field, const void* adjoint, double* grad_rho,
                     double* grad_c, void* stream) {
    if (!scene || !op_buf || !rho || !c || !field || !adjoint || !grad_rho || !grad_c)
        return USV_ERR_ARG;
    const usv_scene& s = *scene;
    int open_mask = 0;
    for (int f = 0; f < 6; ++f)
        if (s.face_kind[f] == USV_FACE_OPEN) open_mask |= 1 << f;
    const OpView<double> op = make_view<double>(s, op_buf, false);
    k_material_vjp<<<grid1(op.n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        op, rho, c, s.omega, s.dx, open_mask, static_cast<const double2*>(field),
        static_cast<const double2*>(adjoint), grad_rho, grad_c);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

}  // extern "C"
