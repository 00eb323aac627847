// Operator set-up and application: per-node coefficient records built on the
// device from rho and c, and the matrix-free 7-point apply kernels.
//
// Parity: the diagonal, edge coefficients and face terms follow
// ConservativeHelmholtz (src/algorithm/physics/conservative_helmholtz.py:36-149);
// R = 1/max|row| and s = 1/(R A_ii) follow GpuIterativeSolver.solve
// (src/algorithm/solvers/iterative_solver.py:37-56), for A and for A^H.
#include <cmath>
#include <cstring>
#include <vector>

#include "usv_internal.cuh"

namespace usv {

static thread_local cudaError_t g_last_cuda = cudaSuccess;
int set_last_cuda_error(cudaError_t e) {
    g_last_cuda = e;
    return USV_ERR_CUDA;
}

// ------------------------------------------------------------ 1-D tables
// Half-volume weights w and PML stretch s = 1 + i sigma per axis
// (conservative_helmholtz.py:48-64), folded into T = w s and
// Q = 1/(0.5 (s_i + s_{i+1}) dx^2).
struct AxisTables {
    std::vector<double2> T, Q;
};

static int validate_scene(const usv_scene& s) {
    if (s.nx < 2 || s.ny < 2 || s.nz < 2) return USV_ERR_ARG;
    if (!(std::isfinite(s.dx) && s.dx > 0 && std::isfinite(s.omega) && s.omega > 0))
        return USV_ERR_ARG;
    for (int f = 0; f < 6; ++f) {
        int k = s.face_kind[f];
        if (k < USV_FACE_REFLECTING || k > USV_FACE_IMPEDANCE) return USV_ERR_ARG;
        if (k == USV_FACE_IMPEDANCE) {
            double zr = s.impedance_re[f], zi = s.impedance_im[f];
            if (!std::isfinite(zr) || !std::isfinite(zi) || zr < 0 || (zr == 0 && zi == 0))
                return USV_ERR_ARG;
        }
    }
    if (s.pml_cells < 0 || s.pml_order < 1 || !(s.pml_strength >= 0) ||
        !std::isfinite(s.pml_strength))
        return USV_ERR_ARG;
    if (s.pml_faces & ~0x3f) return USV_ERR_ARG;
    const int dims[3] = {s.nx, s.ny, s.nz};
    for (int a = 0; a < 3; ++a) {
        int active = 0;
        for (int side = 0; side < 2; ++side)
            if (s.pml_faces & (1 << (2 * a + side))) ++active;
        if (s.pml_cells && active) {
            if ((long long)s.pml_cells * active >= dims[a] - 1) return USV_ERR_ARG;
            for (int side = 0; side < 2; ++side)
                if ((s.pml_faces & (1 << (2 * a + side))) &&
                    s.face_kind[2 * a + side] != USV_FACE_OPEN)
                    return USV_ERR_ARG;
        }
    }
    return USV_OK;
}

static AxisTables axis_tables(const usv_scene& s, int axis) {
    const int dims[3] = {s.nx, s.ny, s.nz};
    const int n = dims[axis];
    std::vector<double> w(n, 1.0), sigma(n, 0.0);
    w[0] = w[n - 1] = 0.5;
    if (s.pml_cells > 0) {
        for (int side = 0; side < 2; ++side) {
            if (!(s.pml_faces & (1 << (2 * axis + side)))) continue;
            for (int i = 0; i < n; ++i) {
                double dist = side == 0 ? double(i) : double(n - 1 - i);
                double t = 1.0 - dist / double(s.pml_cells);
                if (t > 0) sigma[i] += s.pml_strength * std::pow(t, double(s.pml_order));
            }
        }
    }
    AxisTables t;
    t.T.resize(n);
    t.Q.resize(n);
    const double dx2 = s.dx * s.dx;
    for (int i = 0; i < n; ++i) t.T[i] = make_double2(w[i], w[i] * sigma[i]);
    for (int i = 0; i < n; ++i) {
        if (i + 1 < n) {
            double2 mid = make_double2(1.0, 0.5 * (sigma[i] + sigma[i + 1]));
            t.Q[i] = cinv(make_double2(mid.x * dx2, mid.y * dx2));
        } else {
            t.Q[i] = make_double2(0.0, 0.0);
        }
    }
    return t;
}

// ------------------------------------------------------------ build kernel
struct BuildArgs {
    OpView<double> op;      // tables + output records (cast away const below)
    const double* rho;
    const double* c;
    double omega, dx;
    int face_kind[6];
    double2 face_adm[6];    // 1/Z for impedance faces
    double4* rec64f;
    double4* rec64a;
    double2* d64;
    float4* rec32f;
    float4* rec32a;
    int* flag;
};

__global__ void __launch_bounds__(256) k_build(BuildArgs a) {
    const OpView<double>& op = a.op;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < op.n;
         n += (long long)gridDim.x * blockDim.x) {
        const Node p = decode(n, op.nx, op.ny);
        const double rho = a.rho[n], c = a.c[n];
        if (!(rho > 0) || !(c > 0) || !isfinite(rho) || !isfinite(c)) atomicOr(a.flag, 1);
        const bool fixed = node_fixed(op.soft, p.i, p.j, p.k, op.nx, op.ny, op.nz);
        const double2 tx = op.T[0][p.i], ty = op.T[1][p.j], tz = op.T[2][p.k];
        // mass term: w_x w_y w_z s_x s_y s_z omega^2 / (rho c^2)
        double2 diag = cscale(cmul(cmul(tx, ty), tz), a.omega * a.omega / (rho * c * c));
        double emax_all = 0.0, emax_free = 0.0;
        const double2 fyz = cmul(ty, tz), fxz = cmul(tx, tz), fxy = cmul(tx, ty);
        auto edge = [&](long long m, double2 F, bool nb_fixed) {
            const double g = 2.0 / (rho + a.rho[m]);
            const double2 e = cscale(F, g);
            diag = csub(diag, e);
            const double ae = hypot(e.x, e.y);
            emax_all = fmax(emax_all, ae);
            if (!nb_fixed) emax_free = fmax(emax_free, ae);
        };
        const long long sy = op.nx, sz = (long long)op.nx * op.ny;
        if (p.i > 0)
            edge(n - 1, cmul(fyz, op.Q[0][p.i - 1]),
                 node_fixed(op.soft, p.i - 1, p.j, p.k, op.nx, op.ny, op.nz));
        if (p.i < op.nx - 1)
            edge(n + 1, cmul(fyz, op.Q[0][p.i]),
                 node_fixed(op.soft, p.i + 1, p.j, p.k, op.nx, op.ny, op.nz));
        if (p.j > 0)
            edge(n - sy, cmul(fxz, op.Q[1][p.j - 1]),
                 node_fixed(op.soft, p.i, p.j - 1, p.k, op.nx, op.ny, op.nz));
        if (p.j < op.ny - 1)
            edge(n + sy, cmul(fxz, op.Q[1][p.j]),
                 node_fixed(op.soft, p.i, p.j + 1, p.k, op.nx, op.ny, op.nz));
        if (p.k > 0)
            edge(n - sz, cmul(fxy, op.Q[2][p.k - 1]),
                 node_fixed(op.soft, p.i, p.j, p.k - 1, op.nx, op.ny, op.nz));
        if (p.k < op.nz - 1)
            edge(n + sz, cmul(fxy, op.Q[2][p.k]),
                 node_fixed(op.soft, p.i, p.j, p.k + 1, op.nx, op.ny, op.nz));
        // face terms i omega * area * admittance (conservative_helmholtz.py:89-103)
        const int coord[3] = {p.i, p.j, p.k};
        const int dims[3] = {op.nx, op.ny, op.nz};
        for (int f = 0; f < 6; ++f) {
            const int kind = a.face_kind[f];
            if (kind != USV_FACE_OPEN && kind != USV_FACE_IMPEDANCE) continue;
            const int axis = f >> 1;
            if (coord[axis] != ((f & 1) ? dims[axis] - 1 : 0)) continue;
            double2 area;
            if (axis == 0) area = fyz;
            else if (axis == 1) area = fxz;
            else area = fxy;
            area = cscale(area, 1.0 / a.dx);
            const double2 adm = kind == USV_FACE_OPEN ? make_double2(1.0 / (rho * c), 0.0)
                                                      : a.face_adm[f];
            const double2 term = cmul(make_double2(0.0, a.omega), cmul(area, adm));
            diag = cadd(diag, term);
        }
        if (fixed) diag = make_double2(1.0, 0.0);
        const double adiag = hypot(diag.x, diag.y);
        // forward: row maxima of |A| (fixed rows keep only the unit diagonal)
        const double rowmax = fixed ? 1.0 : fmax(adiag, emax_all);
        const double R = rowmax > 0 ? 1.0 / rowmax : 1.0;
        const double2 sd = cscale(diag, R);
        const double2 s = (sd.x != 0 || sd.y != 0) ? cinv(sd) : make_double2(1.0, 0.0);
        // adjoint: row maxima of |A^H| = column maxima of |A|
        const double colmax = fmax(adiag, emax_free);
        const double Ra = colmax > 0 ? 1.0 / colmax : 1.0;
        const double2 sda = cscale(cconj(diag), Ra);
        const double2 sa = (sda.x != 0 || sda.y != 0) ? cinv(sda) : make_double2(1.0, 0.0);
        a.rec64f[n] = make_double4(rho, R, s.x, s.y);
        a.rec64a[n] = make_double4(rho, Ra, sa.x, sa.y);
        a.d64[n] = diag;
        a.rec32f[n] = make_float4(float(rho), float(R), float(s.x), float(s.y));
        a.rec32a[n] = make_float4(float(rho), float(Ra), float(sa.x), float(sa.y));
        if (!isfinite(diag.x) || !isfinite(diag.y)) atomicOr(a.flag, 2);
    }
}

// FP64 edge coefficients of A for the FP64 rows (usv_internal.cuh: a_row):
// e_nd = F_d 2/(rho_n + rho_d), F_d the face product of the direction tables,
// by the same expressions a row used to evaluate on the fly (equal to the
// last bits: the on-the-fly form may fuse the face product into the row's
// FMAs); zero where the neighbour is missing.
__global__ void __launch_bounds__(256) k_edges(OpView<double> op, double2* e64) {
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < op.n;
         n += (long long)gridDim.x * blockDim.x) {
        const Node p = decode(n, op.nx, op.ny);
        const double rho = op.rec[n].x;
        const double2 tx = op.T[0][p.i], ty = op.T[1][p.j], tz = op.T[2][p.k];
        const double2 fyz = cmul(ty, tz), fxz = cmul(tx, tz), fxy = cmul(tx, ty);
        const long long sy = op.nx, sz = (long long)op.nx * op.ny;
        double2 e[6];
        for (int d = 0; d < 6; ++d) e[d] = make_double2(0.0, 0.0);
        auto edge = [&](int dir, long long m, double2 F) { e[dir] = cscale(F, 2.0 / (rho + op.rec[m].x)); };
        if (p.i > 0) edge(0, n - 1, cmul(fyz, op.Q[0][p.i - 1]));
        if (p.i < op.nx - 1) edge(1, n + 1, cmul(fyz, op.Q[0][p.i]));
        if (p.j > 0) edge(2, n - sy, cmul(fxz, op.Q[1][p.j - 1]));
        if (p.j < op.ny - 1) edge(3, n + sy, cmul(fxz, op.Q[1][p.j]));
        if (p.k > 0) edge(4, n - sz, cmul(fxy, op.Q[2][p.k - 1]));
        if (p.k < op.nz - 1) edge(5, n + sz, cmul(fxy, op.Q[2][p.k]));
        for (int d = 0; d < 6; ++d) e64[6 * n + d] = e[d];
    }
}

// Complex64 row coefficients c_nd = R_n e_nd s_d (conj(e_nd) and the adjoint
// scalings for K'), evaluated in FP64 by the same row code as the FP64
// operator with a unit value in direction d only, then rounded once to fp32
// (and, for the bfloat16 Arnoldi rows, to packed bfloat16 {re, im}). The
// complex64 rows (usv_internal.cuh: k_row_cf) then cost six complex
// multiply-adds per node.
template <bool ADJ>
__global__ void __launch_bounds__(256) k_coef(OpView<double> op, float4* cf, uint2* cb) {
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < op.n;
         n += (long long)gridDim.x * blockDim.x) {
        const Node p = decode(n, op.nx, op.ny);
        const long long sy = op.nx, sz = (long long)op.nx * op.ny;
        const long long off[6] = {-1, 1, -sy, sy, -sz, sz};
        const double4 me = op.rec[n];
        float2 c[6];
        for (int d = 0; d < 6; ++d) {
            const double2 v = k_row_from<double, ADJ>(
                op, p, me, make_double2(0.0, 0.0), [&](int dir, double4& r, double2& uv) {
                    r = op.rec[n + off[dir]];
                    uv = make_double2(dir == d ? 1.0 : 0.0, 0.0);
                });
            c[d] = make_float2(float(v.x), float(v.y));
        }
        unsigned pk[6];
        for (int d = 0; d < 6; ++d) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(c[d].x, c[d].y);
            pk[d] = *reinterpret_cast<const unsigned*>(&h);
        }
        cb[3 * n] = make_uint2(pk[0], pk[1]);
        cb[3 * n + 1] = make_uint2(pk[2], pk[3]);
        cb[3 * n + 2] = make_uint2(pk[4], pk[5]);
        cf[3 * n] = make_float4(c[0].x, c[0].y, c[1].x, c[1].y);
        cf[3 * n + 1] = make_float4(c[2].x, c[2].y, c[3].x, c[3].y);
        cf[3 * n + 2] = make_float4(c[4].x, c[4].y, c[5].x, c[5].y);
    }
}

static unsigned grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b > 148LL * 32) b = 148LL * 32;
    if (b < 1) b = 1;
    return unsigned(b);
}

// ------------------------------------------------------------ apply kernels
template <int VARIANT>
__global__ void __launch_bounds__(256) k_apply_fp64(OpView<double> op, const double2* x,
                                                    double2* y, long long ld, Step step) {
    const int b = blockIdx.y;
    const double2* xb = x + b * ld;
    double2* yb = y + b * ld;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    Node p = decode(n, op.nx, op.ny);
    for (; n < op.n; n += (long long)gridDim.x * blockDim.x) {
        yb[n] = a_row<VARIANT>(op, xb, n, p);
        advance(p, step, op.nx, op.ny);
    }
}

// y = K x for complex64 from the precomputed row coefficients: one thread per
// node reads the node's coefficients once and applies them to every
// right-hand side (nrhs vectors at stride ld), so a batch reads the operator
// data once.
__global__ void __launch_bounds__(256, 4) k_apply_kc(OpView<float> op, const float2* __restrict__ x,
                                                  float2* __restrict__ y, long long ld, Step step,
                                                  int nrhs) {
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    Node p = decode(n, op.nx, op.ny);
    const long long sy = op.nx, sz = (long long)op.nx * op.ny;
    for (; n < op.n; n += (long long)gridDim.x * blockDim.x) {
        const float4* cf = op.cf + 3 * n;
        const float4 c01 = __ldg(cf), c23 = __ldg(cf + 1), c45 = __ldg(cf + 2);
        const long long i0 = p.i > 0 ? n - 1 : n, i1 = p.i < op.nx - 1 ? n + 1 : n;
        const long long i2 = p.j > 0 ? n - sy : n, i3 = p.j < op.ny - 1 ? n + sy : n;
        const long long i4 = p.k > 0 ? n - sz : n, i5 = p.k < op.nz - 1 ? n + sz : n;
#pragma unroll 2
        for (int b = 0; b < nrhs; ++b) {
            const float2* xb = x + b * ld;
            float2 v = __ldg(xb + n);
            auto mac = [&](float cr, float ci, float2 u) {
                v.x = fmaf(cr, u.x, fmaf(-ci, u.y, v.x));
                v.y = fmaf(cr, u.y, fmaf(ci, u.x, v.y));
            };
            mac(c01.x, c01.y, __ldg(xb + i0));
            mac(c01.z, c01.w, __ldg(xb + i1));
            mac(c23.x, c23.y, __ldg(xb + i2));
            mac(c23.z, c23.w, __ldg(xb + i3));
            mac(c45.x, c45.y, __ldg(xb + i4));
            mac(c45.z, c45.w, __ldg(xb + i5));
            y[b * ld + n] = v;
        }
        advance(p, step, op.nx, op.ny);
    }
}

// The same for batches of up to 8 right-hand sides on a 3-D grid, so that no
// thread divides: a CTA of 32 x 8 threads covers 32 nodes along x of a few
// rows j of plane k. The R right-hand sides (nrhs rounded up to a power of
// two) are split into G = R / NB groups of NB; a thread applies its node's
// coefficients (loaded once) to the NB vectors b = g, g + G, ..., and each
// warp holds 32 consecutive nodes (coalesced loads and stores); the G warps
// of a row share its coefficient loads through L1.
template <int R, int NB>
__global__ void __launch_bounds__(256) k_apply_kc_rhs(OpView<float> op, const float2* __restrict__ x,
                                                      float2* __restrict__ y, long long ld, int nrhs) {
    constexpr int G = R / NB, kRows = 8 / G;
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int g = threadIdx.y % G;
    const int j = blockIdx.y * kRows + threadIdx.y / G;
    const int k = blockIdx.z;
    if (i >= op.nx || j >= op.ny || g >= nrhs) return;
    const long long sy = op.nx, sz = (long long)op.nx * op.ny;
    const long long n = i + sy * j + sz * k;
    const float4* cf = op.cf + 3 * n;
    const float4 c01 = __ldg(cf), c23 = __ldg(cf + 1), c45 = __ldg(cf + 2);
    const long long o0 = i > 0 ? -1 : 0, o1 = i < op.nx - 1 ? 1 : 0;
    const long long o2 = j > 0 ? -sy : 0, o3 = j < op.ny - 1 ? sy : 0;
    const long long o4 = k > 0 ? -sz : 0, o5 = k < op.nz - 1 ? sz : 0;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = g + G * q;
        if (b < nrhs) {
            const float2* xb = x + b * ld + n;
            float2 v = __ldg(xb);
            const float2 u0 = __ldg(xb + o0), u1 = __ldg(xb + o1), u2 = __ldg(xb + o2);
            const float2 u3 = __ldg(xb + o3), u4 = __ldg(xb + o4), u5 = __ldg(xb + o5);
            auto mac = [&](float cr, float ci, float2 u) {
                v.x = fmaf(cr, u.x, fmaf(-ci, u.y, v.x));
                v.y = fmaf(cr, u.y, fmaf(ci, u.x, v.y));
            };
            mac(c01.x, c01.y, u0);
            mac(c01.z, c01.w, u1);
            mac(c23.x, c23.y, u2);
            mac(c23.z, c23.w, u3);
            mac(c45.x, c45.y, u4);
            mac(c45.z, c45.w, u5);
            y[b * ld + n] = v;
        }
    }
}

// y = K x through the z-marching tile kernel (usv_internal.cuh: zmarch_rows):
// usv_operator_apply K / K^H in complex128 (74 us at 128^3 against 97 us for a
// row-per-thread kernel); complex64 uses the coefficient rows (k_apply_kc_rhs /
// k_apply_kc; its z-marching form measured 40 us against 35 us for the
// row-per-thread kernel of that time).
template <typename R, bool ADJ>
__global__ void __launch_bounds__(kZTX * kZTY) k_apply_k25(OpView<R> op, const typename Tr<R>::c2* x,
                                                           typename Tr<R>::c2* y, long long ld,
                                                           int zseg) {
    __shared__ ZTile<R> sm;
    const int b = blockIdx.z;
    auto* yb = y + b * ld;
    const int z0 = blockIdx.y * zseg, z1 = min(op.nz, z0 + zseg);
    zmarch_rows<R, ADJ>(op, x + b * ld, blockIdx.x, z0, z1, sm,
                        [&](long long n, typename Tr<R>::c2 v) { yb[n] = v; });
}

// y = K x (K' x) in complex64 for up to NB right-hand sides from the 16-byte
// node records {rho, R, s}: the operator data a batch reads is 16 B per node
// (the coefficients are formed in registers: harmonic densities, face
// products of the 1-D tables, row scale and neighbour Jacobi), plus 8 B of x
// and 8 B of y per node and right-hand side. z-marching tile (2.5-D
// blocking): a CTA owns a 32 x 8 tile of (i, j) columns and the planes
// [z0, z1); each thread keeps its column's record and values at z-1 .. z+2 in
// registers (two planes of prefetch) and the halo node of its tile edge one
// plane ahead; the x/y neighbours of plane z come from a double-buffered
// shared-memory tile with a one-node halo (one barrier per plane). Each
// thread forms its row's six coefficients once and applies them to every
// right-hand side.
template <int NB, bool ADJ>
__global__ void __launch_bounds__(kZTX * kZTY) k_apply_rec25(OpView<float> op,
                                                             const float2* __restrict__ x,
                                                             float2* __restrict__ y, long long ld,
                                                             int nrhs, int zseg) {
    __shared__ float4 srec[2][kZTY + 2][kZTX + 2];
    __shared__ float2 su[2][NB][kZTY + 2][kZTX + 2];
    const int tiles_x = (op.nx + kZTX - 1) / kZTX;
    const int bx = blockIdx.x % tiles_x, by = blockIdx.x / tiles_x;
    const int tx = threadIdx.x % kZTX, ty = threadIdx.x / kZTX;
    const int i = bx * kZTX + tx, j = by * kZTY + ty;
    const bool in = i < op.nx && j < op.ny;
    const int z0 = blockIdx.y * zseg, z1 = min(op.nz, z0 + zseg);
    const long long sz = (long long)op.nx * op.ny;
    auto load = [&](int ii, int jj, int z, float4& r, float2 (&v)[NB]) {
        if (ii >= 0 && ii < op.nx && jj >= 0 && jj < op.ny && z >= 0 && z < op.nz) {
            const long long n = ii + (long long)op.nx * jj + sz * z;
            r = __ldg(op.rec + n);
#pragma unroll
            for (int b = 0; b < NB; ++b)
                v[b] = b < nrhs ? __ldg(x + b * ld + n) : make_float2(0.f, 0.f);
        } else {
            r = make_float4(1.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int b = 0; b < NB; ++b) v[b] = make_float2(0.f, 0.f);
        }
    };
    const int hxi = tx == 0 ? i - 1 : (tx == kZTX - 1 ? i + 1 : -2);
    const int hyj = ty == 0 ? j - 1 : (ty == kZTY - 1 ? j + 1 : -2);
    const int hxs = tx == 0 ? 0 : kZTX + 1, hys = ty == 0 ? 0 : kZTY + 1;
    float4 rp, rc, r1, r2, hxr, hyr, hxr1, hyr1;
    float2 up[NB], uc[NB], u1[NB], u2[NB], hxu[NB], hyu[NB], hxu1[NB], hyu1[NB];
    load(i, j, z0 - 1, rp, up);
    load(i, j, z0, rc, uc);
    load(i, j, z0 + 1, r1, u1);
    if (hxi != -2) load(hxi, j, z0, hxr, hxu);
    if (hyj != -2) load(i, hyj, z0, hyr, hyu);
    for (int z = z0; z < z1; ++z) {
        load(i, j, z + 2, r2, u2);
        if (hxi != -2) load(hxi, j, z + 1, hxr1, hxu1);
        if (hyj != -2) load(i, hyj, z + 1, hyr1, hyu1);
        const int bf = (z - z0) & 1;
        srec[bf][ty + 1][tx + 1] = rc;
#pragma unroll
        for (int b = 0; b < NB; ++b) su[bf][b][ty + 1][tx + 1] = uc[b];
        if (hxi != -2) {
            srec[bf][ty + 1][hxs] = hxr;
#pragma unroll
            for (int b = 0; b < NB; ++b) su[bf][b][ty + 1][hxs] = hxu[b];
        }
        if (hyj != -2) {
            srec[bf][hys][tx + 1] = hyr;
#pragma unroll
            for (int b = 0; b < NB; ++b) su[bf][b][hys][tx + 1] = hyu[b];
        }
        __syncthreads();  // plane z visible; the other buffer was last read two planes ago
        if (in) {
            const Node p{i, j, z};
            float2 c[6];
            k_coefs_from<ADJ>(op, p, rc, [&](int dir) {
                switch (dir) {
                    case 0: return srec[bf][ty + 1][tx];
                    case 1: return srec[bf][ty + 1][tx + 2];
                    case 2: return srec[bf][ty][tx + 1];
                    case 3: return srec[bf][ty + 2][tx + 1];
                    case 4: return rp;
                    default: return r1;
                }
            }, c);
            const long long n = i + (long long)op.nx * j + sz * z;
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                if (b >= nrhs) break;
                float2 v = uc[b];
                auto mac = [&](float2 cd, float2 u) {
                    v.x = fmaf(cd.x, u.x, fmaf(-cd.y, u.y, v.x));
                    v.y = fmaf(cd.x, u.y, fmaf(cd.y, u.x, v.y));
                };
                mac(c[0], su[bf][b][ty + 1][tx]);
                mac(c[1], su[bf][b][ty + 1][tx + 2]);
                mac(c[2], su[bf][b][ty][tx + 1]);
                mac(c[3], su[bf][b][ty + 2][tx + 1]);
                mac(c[4], up[b]);
                mac(c[5], u1[b]);
                y[b * ld + n] = v;
            }
        }
        rp = rc; rc = r1; r1 = r2;
        hxr = hxr1; hyr = hyr1;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            up[b] = uc[b]; uc[b] = u1[b]; u1[b] = u2[b];
            hxu[b] = hxu1[b]; hyu[b] = hyu1[b];
        }
    }
}

__global__ void k_export(OpView<double> f, OpView<double> a, double* diag, double* rs,
                         double* jac, double* rsa, double* jaca) {
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < f.n;
         n += (long long)gridDim.x * blockDim.x) {
        if (diag) { diag[2 * n] = f.d[n].x; diag[2 * n + 1] = f.d[n].y; }
        if (rs) rs[n] = f.rec[n].y;
        if (jac) { jac[2 * n] = f.rec[n].z; jac[2 * n + 1] = f.rec[n].w; }
        if (rsa) rsa[n] = a.rec[n].y;
        if (jaca) { jaca[2 * n] = a.rec[n].z; jaca[2 * n + 1] = a.rec[n].w; }
    }
}

}  // namespace usv

using namespace usv;

extern "C" {

int usv_abi_version(void) { return USV_ABI_VERSION; }

const char* usv_status_string(int status) {
    switch (status) {
        case USV_OK: return "ok";
        case USV_ERR_ARG: return "invalid argument";
        case USV_ERR_CUDA: return cudaGetErrorString(g_last_cuda);
        case USV_ERR_WORKSPACE: return "workspace too small";
        case USV_ERR_NOT_CONVERGED: return "GMRES did not converge";
        case USV_ERR_NONFINITE: return "non-finite value";
        case USV_ERR_SOURCE_PML: return "PML overlaps the deposited sinc aperture";
        case USV_ERR_SOURCE_SOFT: return "Sinc flux conflicts with a pressure-release boundary";
        case USV_ERR_SOURCE_CLEARANCE:
            return "Sinc aperture needs one grid cell clearance from side boundaries";
        case USV_ERR_TOO_LARGE:
            return "size exceeds the fixed maximum of the no-allocation entry point";
        case USV_ERR_DEVICE_TIMEOUT: return "a bounded device-side wait ran out";
        default: return "unknown status";
    }
}

int usv_device_info(int* sm_count, int* cc_major, int* cc_minor) {
    int dev = 0;
    USV_CUDA_TRY(cudaGetDevice(&dev));
    if (sm_count) USV_CUDA_TRY(cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev));
    if (cc_major) USV_CUDA_TRY(cudaDeviceGetAttribute(cc_major, cudaDevAttrComputeCapabilityMajor, dev));
    if (cc_minor) USV_CUDA_TRY(cudaDeviceGetAttribute(cc_minor, cudaDevAttrComputeCapabilityMinor, dev));
    return USV_OK;
}

int usv_operator_bytes(const usv_scene* scene, size_t* bytes) {
    if (!scene || !bytes) return USV_ERR_ARG;
    int st = validate_scene(*scene);
    if (st) return st;
    *bytes = make_layout(*scene).total;
    return USV_OK;
}

int usv_operator_build(const usv_scene* scene, const double* rho, const double* c,
                       void* op_buf, size_t op_bytes, void* stream) {
    if (!scene || !rho || !c || !op_buf) return USV_ERR_ARG;
    const usv_scene& s = *scene;
    int st = validate_scene(s);
    if (st) return st;
    const Layout L = make_layout(s);
    if (op_bytes < L.total) return USV_ERR_WORKSPACE;
    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    char* buf = static_cast<char*>(op_buf);
    for (int a = 0; a < 3; ++a) {
        AxisTables t = axis_tables(s, a);
        const size_t n = t.T.size();
        std::vector<float2> T32(n), Q32(n);
        for (size_t i = 0; i < n; ++i) {
            T32[i] = make_float2(float(t.T[i].x), float(t.T[i].y));
            Q32[i] = make_float2(float(t.Q[i].x), float(t.Q[i].y));
        }
        USV_CUDA_TRY(cudaMemcpyAsync(buf + L.tab64[a], t.T.data(), n * sizeof(double2),
                                     cudaMemcpyHostToDevice, strm));
        USV_CUDA_TRY(cudaMemcpyAsync(buf + L.q64[a], t.Q.data(), n * sizeof(double2),
                                     cudaMemcpyHostToDevice, strm));
        USV_CUDA_TRY(cudaMemcpyAsync(buf + L.tab32[a], T32.data(), n * sizeof(float2),
                                     cudaMemcpyHostToDevice, strm));
        USV_CUDA_TRY(cudaMemcpyAsync(buf + L.q32[a], Q32.data(), n * sizeof(float2),
                                     cudaMemcpyHostToDevice, strm));
        // the host vectors die at scope end: finish the copies first
        USV_CUDA_TRY(cudaStreamSynchronize(strm));
    }
    USV_CUDA_TRY(cudaMemsetAsync(buf + L.flag, 0, 64, strm));
    BuildArgs a{};
    a.op = make_view<double>(s, op_buf, false);
    a.rho = rho;
    a.c = c;
    a.omega = s.omega;
    a.dx = s.dx;
    for (int f = 0; f < 6; ++f) {
        a.face_kind[f] = s.face_kind[f];
        a.face_adm[f] = s.face_kind[f] == USV_FACE_IMPEDANCE
                            ? cinv(make_double2(s.impedance_re[f], s.impedance_im[f]))
                            : make_double2(0.0, 0.0);
    }
    a.rec64f = reinterpret_cast<double4*>(buf + L.rec64f);
    a.rec64a = reinterpret_cast<double4*>(buf + L.rec64a);
    a.d64 = reinterpret_cast<double2*>(buf + L.d64);
    a.rec32f = reinterpret_cast<float4*>(buf + L.rec32f);
    a.rec32a = reinterpret_cast<float4*>(buf + L.rec32a);
    a.flag = reinterpret_cast<int*>(buf + L.flag);
    k_build<<<grid_for(a.op.n), 256, 0, strm>>>(a);
    USV_CUDA_TRY(cudaGetLastError());
    k_edges<<<grid_for(a.op.n), 256, 0, strm>>>(a.op, reinterpret_cast<double2*>(buf + L.e64));
    USV_CUDA_TRY(cudaGetLastError());
    k_coef<false><<<grid_for(a.op.n), 256, 0, strm>>>(
        make_view<double>(s, op_buf, false), reinterpret_cast<float4*>(buf + L.cf32f),
        reinterpret_cast<uint2*>(buf + L.cb16f));
    k_coef<true><<<grid_for(a.op.n), 256, 0, strm>>>(
        make_view<double>(s, op_buf, true), reinterpret_cast<float4*>(buf + L.cf32a),
        reinterpret_cast<uint2*>(buf + L.cb16a));
    USV_CUDA_TRY(cudaGetLastError());
    int flag = 0;
    USV_CUDA_TRY(cudaMemcpyAsync(&flag, a.flag, sizeof(int), cudaMemcpyDeviceToHost, strm));
    USV_CUDA_TRY(cudaStreamSynchronize(strm));
    if (flag & 1) return USV_ERR_ARG;
    if (flag & 2) return USV_ERR_NONFINITE;
    return USV_OK;
}

int usv_operator_apply(const usv_scene* scene, const void* op_buf, int variant, int precision,
                       const void* x, void* y, int nrhs, int64_t ld, void* stream) {
    return usv_operator_apply_kernel(scene, op_buf, variant, precision, USV_STENCIL_AUTO, x, y,
                                     nrhs, ld, stream);
}

int usv_operator_apply_kernel(const usv_scene* scene, const void* op_buf, int variant,
                              int precision, int kernel, const void* x, void* y, int nrhs,
                              int64_t ld, void* stream) {
    if (!scene || !op_buf || !x || !y || nrhs < 1 || nrhs > 65535) return USV_ERR_ARG;
    if (kernel < USV_STENCIL_AUTO || kernel > USV_STENCIL_RECORD_TILES) return USV_ERR_ARG;
    const usv_scene& s = *scene;
    const long long n = (long long)s.nx * s.ny * s.nz;
    if (ld < n) return USV_ERR_ARG;
    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    dim3 grid(grid_for(n), nrhs);
    const Step step = make_step((long long)grid.x * 256, s.nx, s.ny);
    switch (variant) {
        case USV_APPLY_A:
            k_apply_fp64<USV_APPLY_A><<<grid, 256, 0, strm>>>(
                make_view<double>(s, op_buf, false), (const double2*)x, (double2*)y, ld, step);
            break;
        case USV_APPLY_AH:
            k_apply_fp64<USV_APPLY_AH><<<grid, 256, 0, strm>>>(
                make_view<double>(s, op_buf, false), (const double2*)x, (double2*)y, ld, step);
            break;
        case USV_APPLY_ABS_A:
            k_apply_fp64<USV_APPLY_ABS_A><<<grid, 256, 0, strm>>>(
                make_view<double>(s, op_buf, false), (const double2*)x, (double2*)y, ld, step);
            break;
        case USV_APPLY_ABS_AH:
            k_apply_fp64<USV_APPLY_ABS_AH><<<grid, 256, 0, strm>>>(
                make_view<double>(s, op_buf, false), (const double2*)x, (double2*)y, ld, step);
            break;
        case USV_APPLY_K:
        case USV_APPLY_KH: {
            const bool adj = variant == USV_APPLY_KH;
            if (precision == USV_PREC_FP64) {
                // z-marching grid: tiles x runs of planes x right-hand sides
                int dev = 0, sms = 148, per_sm = 1;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &per_sm, adj ? (const void*)k_apply_k25<double, true> : (const void*)k_apply_k25<double, false>,
                    kZTX * kZTY, 0);
                const ZGrid zg = zmarch_grid(s.nx, s.ny, s.nz, (per_sm > 0 ? per_sm : 1) * sms / nrhs);
                const dim3 g25(zg.tiles, zg.runs, nrhs);
                auto v = make_view<double>(s, op_buf, adj);
                if (adj) k_apply_k25<double, true><<<g25, kZTX * kZTY, 0, strm>>>(v, (const double2*)x, (double2*)y, ld, zg.zseg);
                else k_apply_k25<double, false><<<g25, kZTX * kZTY, 0, strm>>>(v, (const double2*)x, (double2*)y, ld, zg.zseg);
            } else if (precision == USV_PREC_MIXED) {
                auto v = make_view<float>(s, op_buf, adj);
                if (kernel == USV_STENCIL_RECORD_TILES && nrhs > 4) return USV_ERR_ARG;
                if (kernel == USV_STENCIL_RECORD_TILES) {
                    const int r = nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : 4;
                    int dev = 0, sms = 148, per_sm = 1;
                    cudaGetDevice(&dev);
                    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                    const void* fn = nullptr;
                    if (r == 1) fn = adj ? (const void*)k_apply_rec25<1, true> : (const void*)k_apply_rec25<1, false>;
                    else if (r == 2) fn = adj ? (const void*)k_apply_rec25<2, true> : (const void*)k_apply_rec25<2, false>;
                    else fn = adj ? (const void*)k_apply_rec25<4, true> : (const void*)k_apply_rec25<4, false>;
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kZTX * kZTY, 0);
                    const ZGrid zg = zmarch_grid(s.nx, s.ny, s.nz, (per_sm > 0 ? per_sm : 1) * sms);
                    const float2* xf = (const float2*)x;
                    float2* yf = (float2*)y;
                    int zseg = zg.zseg;
                    void* args[] = {&v, &xf, &yf, &ld, &nrhs, &zseg};
                    USV_CUDA_TRY(cudaLaunchKernel(fn, dim3(zg.tiles, zg.runs), dim3(kZTX * kZTY), args, 0, strm));
                } else if (nrhs <= 8 && s.nz <= 65535) {
                    const float2* xf = (const float2*)x;
                    float2* yf = (float2*)y;
                    const int r = nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : nrhs <= 4 ? 4 : 8;
                    const int rows = 8 / (r == 1 ? 1 : r / 2);  // rows of a CTA: 8 / groups
                    const dim3 g3((s.nx + 31) / 32, (s.ny + rows - 1) / rows, s.nz);
                    const dim3 b3(32, 8);
                    if (r == 1) k_apply_kc_rhs<1, 1><<<g3, b3, 0, strm>>>(v, xf, yf, ld, nrhs);
                    else if (r == 2) k_apply_kc_rhs<2, 2><<<g3, b3, 0, strm>>>(v, xf, yf, ld, nrhs);
                    else if (r == 4) k_apply_kc_rhs<4, 2><<<g3, b3, 0, strm>>>(v, xf, yf, ld, nrhs);
                    else k_apply_kc_rhs<8, 2><<<g3, b3, 0, strm>>>(v, xf, yf, ld, nrhs);
                } else {
                    k_apply_kc<<<dim3(grid.x), 256, 0, strm>>>(v, (const float2*)x, (float2*)y, ld,
                                                               step, nrhs);
                }
            } else {
                return USV_ERR_ARG;
            }
            break;
        }
        default:
            return USV_ERR_ARG;
    }
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

int usv_operator_export(const usv_scene* scene, const void* op_buf, double* diag,
                        double* row_scale, double* jacobi, double* row_scale_adj,
                        double* jacobi_adj, void* stream) {
    if (!scene || !op_buf) return USV_ERR_ARG;
    const usv_scene& s = *scene;
    auto f = make_view<double>(s, op_buf, false);
    auto a = make_view<double>(s, op_buf, true);
    k_export<<<grid_for(f.n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        f, a, diag, row_scale, jacobi, row_scale_adj, jacobi_adj);
    USV_CUDA_TRY(cudaGetLastError());
    return USV_OK;
}

}  // extern "C"
