// Internal device/host helpers of the sm_100a Helmholtz backend.
//
// The operator is matrix-free. Instead of the reference's CSR matrix
// (conservative_helmholtz.py:119-149, ~7 nnz/row, ~176 B/row) each node keeps
// one record {rho, R, s.re, s.im}: the density (edge coefficients are formed
// on the fly as F * 2/(rho_i + rho_j), F from 1-D PML tables), the row scale
// R = 1/max|row| and the Jacobi factor s = 1/(R A_ii) of the reference's
// row-scaled Jacobi GMRES (iterative_solver.py:37-56). A second record holds
// the same for A^H (column maxima), and an fp64 array holds the diagonal A_ii
// for the unscaled residual. Fixed (soft-face) rows are recognised from the
// node coordinates, so no mask is stored.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "usv.h"

namespace usv {

// ---------------------------------------------------------------- types
template <typename R> struct Tr;
template <> struct Tr<float> {
    using c2 = float2;
    using c4 = float4;
};
template <> struct Tr<double> {
    using c2 = double2;
    using c4 = double4;
};

template <typename C> __host__ __device__ __forceinline__ C cmake(double re, double im);
template <> __host__ __device__ __forceinline__ float2 cmake<float2>(double re, double im) {
    return make_float2(float(re), float(im));
}
template <> __host__ __device__ __forceinline__ double2 cmake<double2>(double re, double im) {
    return make_double2(re, im);
}

template <typename C4> __host__ __device__ __forceinline__ C4 make_c4();
template <> __host__ __device__ __forceinline__ float4 make_c4<float4>() {
    return make_float4(0.f, 0.f, 0.f, 0.f);
}
template <> __host__ __device__ __forceinline__ double4 make_c4<double4>() {
    return make_double4(0.0, 0.0, 0.0, 0.0);
}

template <typename C, typename S> __host__ __device__ __forceinline__ C make_c2(S re, S im) {
    C r; r.x = re; r.y = im; return r;
}

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) {
    C r; r.x = a.x + b.x; r.y = a.y + b.y; return r;
}
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) {
    C r; r.x = a.x - b.x; r.y = a.y - b.y; return r;
}
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
template <typename C, typename S> __host__ __device__ __forceinline__ C cscale(C a, S s) {
    C r; r.x = a.x * s; r.y = a.y * s; return r;
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) {
    C r; r.x = a.x; r.y = -a.y; return r;
}
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double cabs(double2 a) { return hypot(a.x, a.y); }
__device__ __forceinline__ float cabs(float2 a) { return hypotf(a.x, a.y); }
__host__ __device__ __forceinline__ double2 cinv(double2 a) {
    double d = a.x * a.x + a.y * a.y;
    return make_double2(a.x / d, -a.y / d);
}
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
template <typename C> __device__ __forceinline__ C from_d(double2 a);
template <> __device__ __forceinline__ float2 from_d<float2>(double2 a) {
    return make_float2(float(a.x), float(a.y));
}
template <> __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }

// bfloat16 complex storage of Krylov vectors (USV_PREC_MIXED_BF16): 4 bytes per
// value, widened to float for the stencil and to double for the dots.
using bf2 = __nv_bfloat162;
// bfloat16 -> fp32 is exact: the 16 bits are the high half of the fp32 word,
// so the packed pair {lo, hi} widens with one shift and one mask (integer
// pipe) instead of two conversion instructions.
__device__ __forceinline__ float2 bf2_to_f2(bf2 a) {
    const unsigned u = *reinterpret_cast<const unsigned*>(&a);
    return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}
__device__ __forceinline__ double2 to_d(bf2 a) {
    const float2 f = bf2_to_f2(a);
    return make_double2(f.x, f.y);
}
template <> __device__ __forceinline__ bf2 from_d<bf2>(double2 a) {
    return __floats2bfloat162_rn(float(a.x), float(a.y));
}
// stored value S -> compute value C, and back
template <typename C> __device__ __forceinline__ C widen(float2 a) { return cmake<C>(a.x, a.y); }
template <typename C> __device__ __forceinline__ C widen(double2 a) { return cmake<C>(a.x, a.y); }
template <typename C> __device__ __forceinline__ C widen(bf2 a) {
    const float2 f = bf2_to_f2(a);
    return cmake<C>(f.x, f.y);
}
template <> __device__ __forceinline__ float2 widen<float2>(float2 a) { return a; }
template <> __device__ __forceinline__ double2 widen<double2>(double2 a) { return a; }
template <typename S> __device__ __forceinline__ S narrow(float2 a);
template <typename S> __device__ __forceinline__ S narrow(double2 a);
template <> __device__ __forceinline__ float2 narrow<float2>(float2 a) { return a; }
template <> __device__ __forceinline__ double2 narrow<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ bf2 narrow<bf2>(float2 a) { return __float22bfloat162_rn(a); }

// Mixed-precision multiply-adds on packed bfloat16 complex words {re, im}
// (PTX fma.rn.f32.bf16, sm_100: bf16 x bf16 products, exact in fp32, added to
// an fp32 sum with one rounding). bf_mac accumulates the four real products of
// conj(v) y: Re = rr + ii, Im = ri - ir.
__device__ __forceinline__ void bf_mac(float& rr, float& ii, float& ri, float& ir, unsigned v,
                                       unsigned y) {
    asm("{\n\t.reg .b16 vl, vh, yl, yh;\n\t"
        "mov.b32 {vl, vh}, %4;\n\t"
        "mov.b32 {yl, yh}, %5;\n\t"
        "fma.rn.f32.bf16 %0, vl, yl, %0;\n\t"
        "fma.rn.f32.bf16 %1, vh, yh, %1;\n\t"
        "fma.rn.f32.bf16 %2, vl, yh, %2;\n\t"
        "fma.rn.f32.bf16 %3, vh, yl, %3;\n\t}"
        : "+f"(rr), "+f"(ii), "+f"(ri), "+f"(ir)
        : "r"(v), "r"(y));
}
// |y|^2 of a packed word: rr += re^2, ii += im^2
__device__ __forceinline__ void bf_sq(float& rr, float& ii, unsigned y) {
    asm("{\n\t.reg .b16 yl, yh;\n\t"
        "mov.b32 {yl, yh}, %2;\n\t"
        "fma.rn.f32.bf16 %0, yl, yl, %0;\n\t"
        "fma.rn.f32.bf16 %1, yh, yh, %1;\n\t}"
        : "+f"(rr), "+f"(ii)
        : "r"(y));
}

// ---------------------------------------------------------------- layout
// Byte offsets of the operator buffer. Everything is derived from the scene,
// so host and device agree without storing the layout itself.
struct Layout {
    size_t tab64[3], q64[3], tab32[3], q32[3];
    size_t rec64f, rec64a, d64, e64, rec32f, rec32a, cf32f, cf32a, cb16f, cb16a, flag;
    size_t total;
};

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

inline Layout make_layout(const usv_scene& s) {
    Layout L{};
    const size_t n = size_t(s.nx) * size_t(s.ny) * size_t(s.nz);
    const int dims[3] = {s.nx, s.ny, s.nz};
    size_t off = 0;
    for (int a = 0; a < 3; ++a) {
        L.tab64[a] = off; off = align_up(off + sizeof(double2) * dims[a]);
        L.q64[a] = off;   off = align_up(off + sizeof(double2) * dims[a]);
        L.tab32[a] = off; off = align_up(off + sizeof(float2) * dims[a]);
        L.q32[a] = off;   off = align_up(off + sizeof(float2) * dims[a]);
    }
    L.rec64f = off; off = align_up(off + sizeof(double4) * n);
    L.rec64a = off; off = align_up(off + sizeof(double4) * n);
    L.d64 = off;    off = align_up(off + sizeof(double2) * n);
    // FP64 edge coefficients e_nd = F_d 2/(rho_n + rho_d) of A, six per node
    // (zero for a missing neighbour); A is symmetric off the diagonal, so the
    // same array gives the A^H rows (conj(e))
    L.e64 = off;    off = align_up(off + 6 * sizeof(double2) * n);
    L.rec32f = off; off = align_up(off + sizeof(float4) * n);
    L.rec32a = off; off = align_up(off + sizeof(float4) * n);
    // complex64 row coefficients c_nd = R_n e_nd s_d of the six neighbour
    // directions, three float4 per node (forward, adjoint)
    L.cf32f = off;  off = align_up(off + 3 * sizeof(float4) * n);
    L.cf32a = off;  off = align_up(off + 3 * sizeof(float4) * n);
    // the same coefficients in packed bfloat16 {re, im}, three uint2 per node
    // (the bfloat16 Arnoldi rows: bf16 x bf16 products)
    L.cb16f = off;  off = align_up(off + 3 * sizeof(uint2) * n);
    L.cb16a = off;  off = align_up(off + 3 * sizeof(uint2) * n);
    L.flag = off;   off = align_up(off + 64);
    L.total = off;
    return L;
}

// Kernel-side view of one operator in precision R (float: complex64 path,
// double: complex128 path).
template <typename R> struct OpView {
    using C2 = typename Tr<R>::c2;
    using C4 = typename Tr<R>::c4;
    int nx, ny, nz;
    long long n;
    unsigned soft;          // bit f: face f is a pressure-release face
    const C2* T[3];         // T_a[i] = w_a[i] * s_a[i]
    const C2* Q[3];         // Q_a[i] = 1 / (0.5 (s_a[i] + s_a[i+1]) dx^2)
    const C4* rec;          // {rho, R, s.re, s.im} (forward or adjoint)
    const double2* d;       // diagonal A_ii (fp64 path only)
    const float4* cf;       // complex64 path: row coefficients, 3 float4 per node
    const uint2* cb;        // the same in packed bfloat16, 3 uint2 per node
    const double2* e64;     // FP64 edge coefficients of A, 6 per node
};

inline unsigned soft_mask(const usv_scene& s) {
    unsigned m = 0;
    for (int f = 0; f < 6; ++f)
        if (s.face_kind[f] == USV_FACE_SOFT) m |= 1u << f;
    return m;
}

template <typename R>
inline OpView<R> make_view(const usv_scene& s, const void* buf, bool adjoint) {
    Layout L = make_layout(s);
    const char* b = static_cast<const char*>(buf);
    OpView<R> v{};
    v.nx = s.nx; v.ny = s.ny; v.nz = s.nz;
    v.n = (long long)s.nx * s.ny * s.nz;
    v.soft = soft_mask(s);
    const bool dbl = sizeof(R) == 8;
    for (int a = 0; a < 3; ++a) {
        v.T[a] = reinterpret_cast<const typename OpView<R>::C2*>(b + (dbl ? L.tab64[a] : L.tab32[a]));
        v.Q[a] = reinterpret_cast<const typename OpView<R>::C2*>(b + (dbl ? L.q64[a] : L.q32[a]));
    }
    size_t rec = dbl ? (adjoint ? L.rec64a : L.rec64f) : (adjoint ? L.rec32a : L.rec32f);
    v.rec = reinterpret_cast<const typename OpView<R>::C4*>(b + rec);
    v.d = reinterpret_cast<const double2*>(b + L.d64);
    v.cf = dbl ? nullptr : reinterpret_cast<const float4*>(b + (adjoint ? L.cf32a : L.cf32f));
    v.cb = dbl ? nullptr : reinterpret_cast<const uint2*>(b + (adjoint ? L.cb16a : L.cb16f));
    v.e64 = reinterpret_cast<const double2*>(b + L.e64);
    return v;
}

// ---------------------------------------------------------------- nodes
__device__ __forceinline__ bool node_fixed(unsigned soft, int i, int j, int k, int nx, int ny,
                                           int nz) {
    return ((soft & 1u) && i == 0) || ((soft & 2u) && i == nx - 1) ||
           ((soft & 4u) && j == 0) || ((soft & 8u) && j == ny - 1) ||
           ((soft & 16u) && k == 0) || ((soft & 32u) && k == nz - 1);
}

struct Node {
    int i, j, k;
};

// Node-index increment of a fixed flat stride, decomposed once on the host so
// kernels walk their nodes without integer division.
struct Step {
    int di, dj, dk;
};
inline Step make_step(long long stride, int nx, int ny) {
    Step s;
    s.di = int(stride % nx);
    s.dj = int((stride / nx) % ny);
    s.dk = int(stride / ((long long)nx * ny));
    return s;
}
__device__ __forceinline__ void advance(Node& p, const Step& s, int nx, int ny) {
    p.i += s.di;
    if (p.i >= nx) {
        p.i -= nx;
        p.j += 1;
    }
    p.j += s.dj;
    if (p.j >= ny) {
        p.j -= ny;
        p.k += 1;
    }
    p.k += s.dk;
}

__device__ __forceinline__ Node decode(long long n, int nx, int ny) {
    long long t = n / nx;
    Node p;
    p.i = int(n - t * nx);
    p.k = int(t / ny);
    p.j = int(t - (long long)p.k * ny);
    return p;
}

// 2 / (a + b): correctly rounded in fp64, fast reciprocal in the complex64
// inner operator (whose rounding the FP64 restart residual corrects).
template <typename R> __device__ __forceinline__ R harmonic2(R a, R b);
template <> __device__ __forceinline__ float harmonic2<float>(float a, float b) {
    return __fdividef(2.0f, a + b);
}
template <> __device__ __forceinline__ double harmonic2<double>(double a, double b) {
    return 2.0 / (a + b);
}

// Row of the row-scaled Jacobi operator K = R A S (forward) or
// K' = R' A^H S' (adjoint) at node n, applied to u (scaled by `scale`):
//   forward : y = u_n + R_n sum_j e_nj s_j u_j          (fixed row: y = u_n)
//   adjoint : y = u_n + R'_n sum_{j not fixed} conj(e_nj) s'_j u_j
// The unit diagonal follows from s = 1/(R A_ii) (iterative_solver.py:46-56).
// The same row from the node's own record `me` and value `un` and a fetch
// fetch(dir, r, u) of the neighbour record and value in direction
// dir = 0..5 (x-, x+, y-, y+, z-, z+); directions outside the grid are never
// fetched. Used with global-memory fetches (k_row) and with shared-memory /
// register tiles (the z-marching stencil); the arithmetic is the same.
template <typename R, bool ADJ, typename Fetch>
__device__ __forceinline__ typename Tr<R>::c2 k_row_from(const OpView<R>& op, Node p,
                                                        typename Tr<R>::c4 me,
                                                        typename Tr<R>::c2 un, Fetch&& fetch) {
    using C2 = typename Tr<R>::c2;
    using C4 = typename Tr<R>::c4;
    const bool fixed = node_fixed(op.soft, p.i, p.j, p.k, op.nx, op.ny, op.nz);
    if (!ADJ && fixed) return un;
    const C2 tx = op.T[0][p.i], ty = op.T[1][p.j], tz = op.T[2][p.k];
    const C2 fyz = cmul(ty, tz), fxz = cmul(tx, tz), fxy = cmul(tx, ty);
    C2 acc = cmake<C2>(0.0, 0.0);
    auto edge = [&](int dir, C2 F, bool nb_fixed) {
        if (ADJ && nb_fixed) return;
        C4 r;
        C2 uv;
        fetch(dir, r, uv);
        const R g = harmonic2<R>(me.x, r.x);
        C2 e = cscale(F, g);
        if (ADJ) e = cconj(e);
        C2 sv = cmul(make_c2<C2>(r.z, r.w), uv);
        acc = cadd(acc, cmul(e, sv));
    };
    if (p.i > 0)
        edge(0, cmul(fyz, op.Q[0][p.i - 1]),
             ADJ && node_fixed(op.soft, p.i - 1, p.j, p.k, op.nx, op.ny, op.nz));
    if (p.i < op.nx - 1)
        edge(1, cmul(fyz, op.Q[0][p.i]),
             ADJ && node_fixed(op.soft, p.i + 1, p.j, p.k, op.nx, op.ny, op.nz));
    if (p.j > 0)
        edge(2, cmul(fxz, op.Q[1][p.j - 1]),
             ADJ && node_fixed(op.soft, p.i, p.j - 1, p.k, op.nx, op.ny, op.nz));
    if (p.j < op.ny - 1)
        edge(3, cmul(fxz, op.Q[1][p.j]),
             ADJ && node_fixed(op.soft, p.i, p.j + 1, p.k, op.nx, op.ny, op.nz));
    if (p.k > 0)
        edge(4, cmul(fxy, op.Q[2][p.k - 1]),
             ADJ && node_fixed(op.soft, p.i, p.j, p.k - 1, op.nx, op.ny, op.nz));
    if (p.k < op.nz - 1)
        edge(5, cmul(fxy, op.Q[2][p.k]),
             ADJ && node_fixed(op.soft, p.i, p.j, p.k + 1, op.nx, op.ny, op.nz));
    return cadd(un, cscale(acc, me.y));
}

// The six coefficients c_d of the complex64 row of K (K') at node p from the
// 16-byte node records {rho, R, s.re, s.im}: c_d = R_n e_nd s_d with
// e_nd = F_d 2/(rho_n + rho_d) (conj(e_nd) for K'), zero for a missing
// neighbour, for a fixed neighbour of an adjoint row and for every edge of a
// fixed forward row, so that y = u_n + sum_d c_d u_d. rec(dir) returns the
// neighbour record in direction dir = 0..5 (x-, x+, y-, y+, z-, z+); it is
// never called for a direction outside the grid.
template <bool ADJ, typename Rec>
__device__ __forceinline__ void k_coefs_from(const OpView<float>& op, Node p, float4 me, Rec&& rec,
                                             float2 (&c)[6]) {
#pragma unroll
    for (int d = 0; d < 6; ++d) c[d] = make_float2(0.f, 0.f);
    const bool fixed = node_fixed(op.soft, p.i, p.j, p.k, op.nx, op.ny, op.nz);
    if (!ADJ && fixed) return;
    const float2 tx = op.T[0][p.i], ty = op.T[1][p.j], tz = op.T[2][p.k];
    const float2 fyz = cmul(ty, tz), fxz = cmul(tx, tz), fxy = cmul(tx, ty);
    auto edge = [&](int dir, float2 F, bool nb_fixed) {
        if (ADJ && nb_fixed) return;
        const float4 r = rec(dir);
        float2 e = cscale(F, harmonic2<float>(me.x, r.x) * me.y);
        if (ADJ) e = cconj(e);
        c[dir] = cmul(e, make_float2(r.z, r.w));
    };
    if (p.i > 0)
        edge(0, cmul(fyz, op.Q[0][p.i - 1]),
             ADJ && node_fixed(op.soft, p.i - 1, p.j, p.k, op.nx, op.ny, op.nz));
    if (p.i < op.nx - 1)
        edge(1, cmul(fyz, op.Q[0][p.i]),
             ADJ && node_fixed(op.soft, p.i + 1, p.j, p.k, op.nx, op.ny, op.nz));
    if (p.j > 0)
        edge(2, cmul(fxz, op.Q[1][p.j - 1]),
             ADJ && node_fixed(op.soft, p.i, p.j - 1, p.k, op.nx, op.ny, op.nz));
    if (p.j < op.ny - 1)
        edge(3, cmul(fxz, op.Q[1][p.j]),
             ADJ && node_fixed(op.soft, p.i, p.j + 1, p.k, op.nx, op.ny, op.nz));
    if (p.k > 0)
        edge(4, cmul(fxy, op.Q[2][p.k - 1]),
             ADJ && node_fixed(op.soft, p.i, p.j, p.k - 1, op.nx, op.ny, op.nz));
    if (p.k < op.nz - 1)
        edge(5, cmul(fxy, op.Q[2][p.k]),
             ADJ && node_fixed(op.soft, p.i, p.j, p.k + 1, op.nx, op.ny, op.nz));
}

// Complex64 row from the precomputed coefficients (operator.cu: k_coef):
// y = u_n + sum_d c_nd u_d over the six neighbour directions. A missing
// neighbour (grid edge) and every edge of a fixed forward row carry a zero
// coefficient, so their loads are redirected to u_n, which exists and is finite.
template <typename S>
__device__ __forceinline__ float2 k_row_cf(const OpView<float>& op, const S* __restrict__ u,
                                           long long n, Node p) {
    const float4* c = op.cf + 3 * n;
    const float4 c01 = __ldg(c), c23 = __ldg(c + 1), c45 = __ldg(c + 2);
    const long long sy = op.nx, sz = (long long)op.nx * op.ny;
    const float2 u0 = widen<float2>(u[p.i > 0 ? n - 1 : n]);
    const float2 u1 = widen<float2>(u[p.i < op.nx - 1 ? n + 1 : n]);
    const float2 u2 = widen<float2>(u[p.j > 0 ? n - sy : n]);
    const float2 u3 = widen<float2>(u[p.j < op.ny - 1 ? n + sy : n]);
    const float2 u4 = widen<float2>(u[p.k > 0 ? n - sz : n]);
    const float2 u5 = widen<float2>(u[p.k < op.nz - 1 ? n + sz : n]);
    float2 y = widen<float2>(u[n]);
    auto mac = [&](float cr, float ci, float2 v) {
        y.x = fmaf(cr, v.x, fmaf(-ci, v.y, y.x));
        y.y = fmaf(cr, v.y, fmaf(ci, v.x, y.y));
    };
    mac(c01.x, c01.y, u0);
    mac(c01.z, c01.w, u1);
    mac(c23.x, c23.y, u2);
    mac(c23.z, c23.w, u3);
    mac(c45.x, c45.y, u4);
    mac(c45.z, c45.w, u5);
    return y;
}

// The same row without grid coordinates: a missing neighbour (zero
// coefficient) is read at the neighbour index clamped into [0, N), a node of
// the same vector. Equal to k_row_cf wherever u is finite (a zero coefficient
// times a finite value adds zero).
template <typename S>
__device__ __forceinline__ float2 k_row_cf_clamped(const OpView<float>& op,
                                                   const S* __restrict__ u, long long n) {
    const float4* c = op.cf + 3 * n;
    const float4 c01 = __ldg(c), c23 = __ldg(c + 1), c45 = __ldg(c + 2);
    const long long sy = op.nx, sz = (long long)op.nx * op.ny, last = op.n - 1;
    const float2 u0 = widen<float2>(u[n > 0 ? n - 1 : 0]);
    const float2 u1 = widen<float2>(u[n < last ? n + 1 : last]);
    const float2 u2 = widen<float2>(u[n >= sy ? n - sy : 0]);
    const float2 u3 = widen<float2>(u[n + sy <= last ? n + sy : last]);
    const float2 u4 = widen<float2>(u[n >= sz ? n - sz : 0]);
    const float2 u5 = widen<float2>(u[n + sz <= last ? n + sz : last]);
    float2 y = widen<float2>(u[n]);
    auto mac = [&](float cr, float ci, float2 v) {
        y.x = fmaf(cr, v.x, fmaf(-ci, v.y, y.x));
        y.y = fmaf(cr, v.y, fmaf(ci, v.x, y.y));
    };
    mac(c01.x, c01.y, u0);
    mac(c01.z, c01.w, u1);
    mac(c23.x, c23.y, u2);
    mac(c23.z, c23.w, u3);
    mac(c45.x, c45.y, u4);
    mac(c45.z, c45.w, u5);
    return y;
}

// The bfloat16 row from the packed bfloat16 coefficients: every product
// c_d u_d is bf16 x bf16, exact in fp32 (fma.rn.f32.bf16), summed in fp32;
// clamped neighbour indices as above.
__device__ __forceinline__ float2 k_row_cb_clamped(const OpView<float>& op,
                                                   const bf2* __restrict__ u, long long n) {
    const uint2* c = op.cb + 3 * n;
    const uint2 c01 = __ldg(c), c23 = __ldg(c + 1), c45 = __ldg(c + 2);
    const long long sy = op.nx, sz = (long long)op.nx * op.ny, last = op.n - 1;
    const unsigned* w = reinterpret_cast<const unsigned*>(u);
    const unsigned u0 = w[n > 0 ? n - 1 : 0], u1 = w[n < last ? n + 1 : last];
    const unsigned u2 = w[n >= sy ? n - sy : 0], u3 = w[n + sy <= last ? n + sy : last];
    const unsigned u4 = w[n >= sz ? n - sz : 0], u5 = w[n + sz <= last ? n + sz : last];
    // bf_mac accumulates conj(c) u: Re(c u) = rr - ii, Im(c u) = ri + ir
    float rr = 0.f, ii = 0.f, ri = 0.f, ir = 0.f;
    bf_mac(rr, ii, ri, ir, c01.x, u0);
    bf_mac(rr, ii, ri, ir, c01.y, u1);
    bf_mac(rr, ii, ri, ir, c23.x, u2);
    bf_mac(rr, ii, ri, ir, c23.y, u3);
    bf_mac(rr, ii, ri, ir, c45.x, u4);
    bf_mac(rr, ii, ri, ir, c45.y, u5);
    const float2 un = widen<float2>(u[n]);
    return make_float2(un.x + (rr - ii), un.y + (ri + ir));
}

template <typename R, bool ADJ, typename S = typename Tr<R>::c2>
__device__ __forceinline__ typename Tr<R>::c2 k_row(const OpView<R>& op, const S* __restrict__ u,
                                                    long long n, Node p) {
    using C2 = typename Tr<R>::c2;
    using C4 = typename Tr<R>::c4;
    if constexpr (sizeof(R) == 4) {
        return k_row_cf(op, u, n, p);
    } else {
        const C2 un = widen<C2>(u[n]);
        if (!ADJ && node_fixed(op.soft, p.i, p.j, p.k, op.nx, op.ny, op.nz)) return un;
        const long long sy = op.nx, sz = (long long)op.nx * op.ny;
        const long long off[6] = {-1, 1, -sy, sy, -sz, sz};
        return k_row_from<R, ADJ>(op, p, op.rec[n], un, [&](int dir, C4& r, C2& uv) {
            const long long m = n + off[dir];
            r = op.rec[m];
            uv = widen<C2>(u[m]);
        });
    }
}

// z-marching application of the K rows (2.5-D blocking): a CTA owns a
// kZTX x kZTY tile of (i, j) columns and the planes [z0, z1). Each thread keeps
// the record and value of its own column at z-1 .. z+2 in registers (two
// planes of prefetch) and, on the tile edge, the halo node of the next plane;
// the x/y neighbours of plane z come from a double-buffered shared-memory
// tile with a one-node halo (one barrier per plane). Every node record and
// value is read from HBM about once (plus the tile halo and the run ends) and
// the neighbour accesses are register or shared-memory reads instead of
// dependent global loads. out(n, value) receives the row of every grid node
// of the tile column.
constexpr int kZTX = 32, kZTY = 8;
template <typename R> struct ZTile {
    typename Tr<R>::c4 rec[2][kZTY + 2][kZTX + 2];
    typename Tr<R>::c2 u[2][kZTY + 2][kZTX + 2];
};
template <typename R, bool ADJ, typename S, typename Out>
__device__ __forceinline__ void zmarch_rows(const OpView<R>& op, const S* __restrict__ u, int tile,
                                            int z0, int z1, ZTile<R>& sm, Out&& out) {
    using C2 = typename Tr<R>::c2;
    using C4 = typename Tr<R>::c4;
    const int tiles_x = (op.nx + kZTX - 1) / kZTX;
    const int bx = tile % tiles_x, by = tile / tiles_x;
    const int tx = threadIdx.x % kZTX, ty = threadIdx.x / kZTX;
    const int i = bx * kZTX + tx, j = by * kZTY + ty;
    const bool in = i < op.nx && j < op.ny;
    const long long sz = (long long)op.nx * op.ny;
    auto load = [&](int ii, int jj, int z, C4& r, C2& v) {
        if (ii >= 0 && ii < op.nx && jj >= 0 && jj < op.ny && z >= 0 && z < op.nz) {
            const long long n = ii + (long long)op.nx * jj + sz * z;
            r = op.rec[n];
            v = widen<C2>(u[n]);
        } else {
            r = make_c4<C4>();
            v = cmake<C2>(0.0, 0.0);
        }
    };
    // halo node of this thread (x edge, y edge), if any
    const int hxi = tx == 0 ? i - 1 : (tx == kZTX - 1 ? i + 1 : -2);
    const int hyj = ty == 0 ? j - 1 : (ty == kZTY - 1 ? j + 1 : -2);
    const int hxs = tx == 0 ? 0 : kZTX + 1, hys = ty == 0 ? 0 : kZTY + 1;
    C4 rp, rc, r1, r2, hxr, hyr, hxr1, hyr1;
    C2 up, uc, u1, u2, hxu, hyu, hxu1, hyu1;
    load(i, j, z0 - 1, rp, up);
    load(i, j, z0, rc, uc);
    load(i, j, z0 + 1, r1, u1);
    if (hxi != -2) load(hxi, j, z0, hxr, hxu);
    if (hyj != -2) load(i, hyj, z0, hyr, hyu);
    for (int z = z0; z < z1; ++z) {
        // prefetch: own column two planes ahead, halo one plane ahead
        load(i, j, z + 2, r2, u2);
        if (hxi != -2) load(hxi, j, z + 1, hxr1, hxu1);
        if (hyj != -2) load(i, hyj, z + 1, hyr1, hyu1);
        const int bf = (z - z0) & 1;
        sm.rec[bf][ty + 1][tx + 1] = rc;
        sm.u[bf][ty + 1][tx + 1] = uc;
        if (hxi != -2) {
            sm.rec[bf][ty + 1][hxs] = hxr;
            sm.u[bf][ty + 1][hxs] = hxu;
        }
        if (hyj != -2) {
            sm.rec[bf][hys][tx + 1] = hyr;
            sm.u[bf][hys][tx + 1] = hyu;
        }
        __syncthreads();  // plane z visible; the other buffer was last read two planes ago
        if (in) {
            const Node p{i, j, z};
            const C2 val = k_row_from<R, ADJ>(op, p, rc, uc, [&](int dir, C4& r, C2& v) {
                switch (dir) {
                    case 0: r = sm.rec[bf][ty + 1][tx]; v = sm.u[bf][ty + 1][tx]; break;
                    case 1: r = sm.rec[bf][ty + 1][tx + 2]; v = sm.u[bf][ty + 1][tx + 2]; break;
                    case 2: r = sm.rec[bf][ty][tx + 1]; v = sm.u[bf][ty][tx + 1]; break;
                    case 3: r = sm.rec[bf][ty + 2][tx + 1]; v = sm.u[bf][ty + 2][tx + 1]; break;
                    case 4: r = rp; v = up; break;
                    default: r = r1; v = u1; break;
                }
            });
            out(i + (long long)op.nx * j + sz * z, val);
        }
        rp = rc; up = uc;
        rc = r1; uc = u1;
        r1 = r2; u1 = u2;
        hxr = hxr1; hxu = hxu1;
        hyr = hyr1; hyu = hyu1;
    }
}

// Grid of the z-marching kernels: tiles x runs of zseg planes, at most
// `ctas` CTAs in total (one wave of resident CTAs).
struct ZGrid {
    int tiles, runs, zseg;
};
inline ZGrid zmarch_grid(int nx, int ny, int nz, int ctas) {
    ZGrid z;
    z.tiles = ((nx + kZTX - 1) / kZTX) * ((ny + kZTY - 1) / kZTY);
    int runs = ctas / z.tiles;
    runs = runs < 1 ? 1 : runs;
    z.zseg = (nz + runs - 1) / runs;
    z.zseg = z.zseg < 2 ? 2 : z.zseg;
    z.runs = (nz + z.zseg - 1) / z.zseg;
    return z;
}

// Row of the unscaled fp64 operator at node n applied to x (complex128).
//   A     : fixed -> x_n ; else A_nn x_n + sum_j e_nj x_j
//   A^H   : conj(A_nn) x_n + sum_{j not fixed} conj(e_nj) x_j
//   |A|   : fixed -> |x_n| ; else |A_nn||x_n| + sum_j |e_nj||x_j|
//   |A^H| : |A_nn||x_n| + sum_{j not fixed} |e_nj||x_j|
template <int VARIANT>
__device__ __forceinline__ double2 a_row(const OpView<double>& op,
                                         const double2* __restrict__ x, long long n, Node p) {
    constexpr bool H = (VARIANT == USV_APPLY_AH || VARIANT == USV_APPLY_ABS_AH);
    constexpr bool ABS = (VARIANT == USV_APPLY_ABS_A || VARIANT == USV_APPLY_ABS_AH);
    const double2 xn = x[n];
    const bool fixed = node_fixed(op.soft, p.i, p.j, p.k, op.nx, op.ny, op.nz);
    if (!H && fixed) return ABS ? make_double2(cabs(xn), 0.0) : xn;
    const double2 d = op.d[n];
    double2 acc = ABS ? make_double2(cabs(d) * cabs(xn), 0.0) : (H ? cmulc(d, xn) : cmul(d, xn));
    const double2* en = op.e64 + 6 * n;  // k_edges: F_d 2/(rho_n + rho_d)
    auto edge = [&](int dir, long long m, bool nb_fixed) {
        if (H && nb_fixed) return;
        const double2 e = en[dir];
        const double2 xm = x[m];
        if (ABS) acc.x += cabs(e) * cabs(xm);
        else acc = cadd(acc, H ? cmulc(e, xm) : cmul(e, xm));
    };
    const long long sy = op.nx, sz = (long long)op.nx * op.ny;
    if (p.i > 0) edge(0, n - 1, H && node_fixed(op.soft, p.i - 1, p.j, p.k, op.nx, op.ny, op.nz));
    if (p.i < op.nx - 1)
        edge(1, n + 1, H && node_fixed(op.soft, p.i + 1, p.j, p.k, op.nx, op.ny, op.nz));
    if (p.j > 0) edge(2, n - sy, H && node_fixed(op.soft, p.i, p.j - 1, p.k, op.nx, op.ny, op.nz));
    if (p.j < op.ny - 1)
        edge(3, n + sy, H && node_fixed(op.soft, p.i, p.j + 1, p.k, op.nx, op.ny, op.nz));
    if (p.k > 0) edge(4, n - sz, H && node_fixed(op.soft, p.i, p.j, p.k - 1, op.nx, op.ny, op.nz));
    if (p.k < op.nz - 1)
        edge(5, n + sz, H && node_fixed(op.soft, p.i, p.j, p.k + 1, op.nx, op.ny, op.nz));
    return acc;
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Warp sums of two values with one shuffle per step: after the first exchange
// the low half-warp carries a, the high half b; returns a's sum in lanes
// 0..15 and b's sum in lanes 16..31 (lane 0 and lane 16 hold the results).
__device__ __forceinline__ double warp_sum_pair(double a, double b) {
    const bool hi = (threadIdx.x & 16) != 0;
    double v = (hi ? b : a) + __shfl_xor_sync(0xffffffffu, hi ? a : b, 16);
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum over the block (blockDim.x a multiple of 32, <= 1024); result valid in
// every thread. `sh` needs 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = (lane < nw) ? sh[lane] : 0.0;
    return warp_sum(t);
}
__device__ __forceinline__ double block_max(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = (lane < nw) ? sh[lane] : 0.0;
    return warp_max(t);
}

// ---------------------------------------------------------------- bulk copies
// Global -> shared bulk copies (cp.async.bulk, the 1-D TMA path; no
// multicast) completed on an mbarrier, and the mbarrier operations of a
// producer / consumer tile ring. Addresses are 16-byte aligned and sizes
// multiples of 16 bytes (the callers round a ragged tail up into the zeroed
// padding of the vector).
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of `parity` to complete, at most ~2^31 SM cycles (about a
// second); false when the bound ran out (the caller records an error and
// leaves instead of waiting forever).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    if (mbar_test(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(bar, parity))
        if (clock64() - t0 > (1LL << 31)) return false;
    return true;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------------- tcgen05
// 5th-generation tensor-core operations (sm_100a): tensor-memory (TMEM)
// allocation, one-thread MMA issue with shared-memory operand descriptors,
// completion on an mbarrier, and TMEM -> register loads. The descriptor and
// instruction-descriptor bit layouts follow the PTX ISA's tcgen05 matrix
// descriptors (the same fields as CUTLASS's UMMA::SmemDescriptor and
// UMMA::InstrDescriptor).
//
// Shared-memory matrix descriptor, no swizzle: start address, leading-
// dimension byte offset (LBO) and stride-dimension byte offset (SBO), each
// >> 4 in 14 bits, version 1 (bits 46-47), layout type 0.
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, unsigned lbo,
                                                        unsigned sbo) {
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) |
           ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16 with bf16 A and B, fp32 accumulator:
// bit 4 D = f32, bits 7/10 A/B = bf16, bit 15 A MN-major (1) / K-major (0),
// bit 16 the same for B, bits 17-22 N >> 3, bits 24-28 M >> 4.
__host__ __device__ constexpr unsigned umma_idesc_bf16(int m, int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (unsigned(a_mn) << 15) | (unsigned(b_mn) << 16) |
           (unsigned(n >> 3) << 17) | (unsigned(m >> 4) << 24);
}
// D[tmem] (+)= A B; accumulate = 0 overwrites D. Issued by one thread.
__device__ __forceinline__ void umma_bf16(unsigned tmem_d, unsigned long long a,
                                          unsigned long long b, unsigned idesc, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive (once) on `bar` when every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar))
                 : "memory");
}
// One warp: allocate `ncols` TMEM columns (a power of two >= 32), address into *dst.
__device__ __forceinline__ void tmem_alloc(unsigned* dst, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes -> visible to the async proxy (MMA operands)
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 32 consecutive fp32 columns of this thread's TMEM lane (32x32b shape: warp
// w % 4 reads lanes 32 (w % 4) .. +31), then wait for the load.
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float (&v)[32]) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Status helpers shared by the translation units.
int set_last_cuda_error(cudaError_t e);
}  // namespace usv

#define USV_CUDA_TRY(expr)                                              \
    do {                                                                \
        cudaError_t _e = (expr);                                        \
        if (_e != cudaSuccess) return ::usv::set_last_cuda_error(_e);   \
    } while (0)
