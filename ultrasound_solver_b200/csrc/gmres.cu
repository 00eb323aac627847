// Restarted, right-preconditioned GMRES(m) on the row-scaled Jacobi operator
// K = R A S (or K' = R' A^H S' for the adjoint), batched over right-hand
// sides, with Krylov vectors in complex64 (USV_PREC_MIXED) or complex128
// (USV_PREC_FP64).
//
// Algorithm parity: iterative_solver.py:30-104 drives CuPy's gmres
// (cupyx.scipy.sparse.linalg.gmres, cupy>=14, not vendored by the
// reference): x0 = 0, residual r = Rb - K x tested against rtol*||Rb|| only
// at restarts, one-pass classical Gram-Schmidt, all m steps per cycle,
// least squares of the (m+1) x m Hessenberg, x += V y, solution S x.
// Here the restart residual r = R (b - A x_sol) and the solution update
// x_sol += S V y are always FP64; the Gram-Schmidt dots and the Hessenberg /
// Givens least squares are FP64 on the device; only the Krylov vectors and
// the in-cycle stencil use the vector precision. With complex64 vectors this
// is GMRES with FP64 iterative refinement at every restart.
//
// Per Arnoldi step two kernels run over (node chunk, RHS):
//   k_dots : w = sigma_j K u_j (stencil) stored as u_{j+1}; partial dots
//            <sigma_t u_t, w>, t<=j, and ||w||^2, reduced by the last CTA
//   k_orth : u_{j+1} = w - sum_t h_tj sigma_t u_t, ||u_{j+1}||^2; the last
//            CTA forms beta, applies the Givens rotations, and at the end of
//            the cycle back-substitutes y.
// Basis vectors are stored unnormalised with a scale sigma_t = 1/||u_t||.
#include <cmath>
#include <cstring>
#include <vector>

#include "usv_internal.cuh"

#define USV_MAX_RESTART 112  // keeps the m x (m+1) least-squares tile in shared memory

namespace usv {

enum { ST_ACTIVE = 0, ST_CONVERGED = 1, ST_MAXITER = 2, ST_NONFINITE = 3 };

struct GState {
    int m, nblk, chunk, full_cycles, maxiter;
    int nchunk;        // node chunks of `chunk` nodes; CTAs loop over them (grid <= nblk)
    long long n;
    long long nv;      // Krylov vector stride: n rounded up to 64 (512-B aligned pairs)
    double rtol;
    double2* partial;  // [B][nblk][m+2], one slot per CTA of the launch
    double2* H;        // [B][m][m+1]  column j, rows 0..m
    double* gc;        // [B][m]
    double2* gs;       // [B][m]
    double2* g;        // [B][m+1]
    double2* y;        // [B][m]   (y_t * sigma_t)
    double* sigma;     // [B][m+1]
    double* bnorm;     // [B]
    double* atol;      // [B]
    double* wnorm;     // [B]
    double* gates;     // [B][4]
    double* hist;      // [B][hcap] ||r||/||Rb|| at each restart test
    int hcap;
    int* status;       // [B]
    int* cycles;       // [B]
    int* iters;        // [B]
    int* len;          // [B]
    int* ended;        // [B]
    unsigned* counter; // [B]
};

struct WsLayout {
    size_t V, partial, H, gc, gs, g, y, sigma, bnorm, atol, wnorm, gates, hist, status, cycles,
        iters, len, ended, counter, state_begin, total;
};

static long long padded(long long n) { return (n + 63) / 64 * 64; }

static WsLayout ws_layout(long long n, int m, int B, int nblk, size_t vec_bytes, int hcap) {
    WsLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes);
        return o;
    };
    L.V = take(vec_bytes * size_t(padded(n)) * size_t(m + 1) * size_t(B));
    L.partial = take(sizeof(double2) * size_t(B) * nblk * (m + 2));
    L.state_begin = off;
    L.H = take(sizeof(double2) * size_t(B) * m * (m + 1));
    L.gc = take(sizeof(double) * size_t(B) * m);
    L.gs = take(sizeof(double2) * size_t(B) * m);
    L.g = take(sizeof(double2) * size_t(B) * (m + 1));
    L.y = take(sizeof(double2) * size_t(B) * m);
    L.sigma = take(sizeof(double) * size_t(B) * (m + 1));
    L.bnorm = take(sizeof(double) * B);
    L.atol = take(sizeof(double) * B);
    L.wnorm = take(sizeof(double) * B);
    L.gates = take(sizeof(double) * 4 * B);
    L.hist = take(sizeof(double) * size_t(B) * size_t(hcap > 0 ? hcap : 1));
    L.status = take(sizeof(int) * B);
    L.cycles = take(sizeof(int) * B);
    L.iters = take(sizeof(int) * B);
    L.len = take(sizeof(int) * B);
    L.ended = take(sizeof(int) * B);
    L.counter = take(sizeof(unsigned) * B);
    L.total = off;
    return L;
}

__device__ __forceinline__ bool last_block_done(unsigned* counter, int nblk) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(counter, 1u) == unsigned(nblk - 1);
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

__device__ __forceinline__ double2 ld_cg(const double2* p) { return __ldcg(p); }

// Sum of the gridDim.x norm partials (slot 0) by the last CTA, in a fixed
// order (thread-strided, then the block tree).
__device__ __forceinline__ double reduce_slot0(const GState& g, int b, double* sh) {
    double t = 0.0;
    const double2* p = g.partial + (long long)b * g.nblk * (g.m + 2);
    for (int q = threadIdx.x; q < int(gridDim.x); q += blockDim.x)
        t += ld_cg(p + (long long)q * (g.m + 2)).x;
    return block_sum(t, sh);
}

// ------------------------------------------------------------ residual
// r = Rs (rhs - OP x) in fp64 (OP = A or A^H); first=1: x = 0, r = Rs rhs.
template <bool ADJ, typename C2>
__global__ void __launch_bounds__(256) k_residual(OpView<double> op, const double2* rhs,
                                                  const double2* x, long long ld, C2* V,
                                                  GState g, int first, Step step) {
    const int b = blockIdx.y;
    if (!first && (g.status[b] != ST_ACTIVE)) return;
    __shared__ double sh[32];
    const double2* rb = rhs + b * ld;
    const double2* xb = x + b * ld;
    C2* v0 = V + (long long)b * (g.m + 1) * g.nv;
    double acc = 0.0;
    for (int ch = blockIdx.x; ch < g.nchunk; ch += gridDim.x) {
        const long long n0 = (long long)ch * g.chunk;
        const long long n1 = min(n0 + g.chunk, op.n);
        Node p = decode(n0 + threadIdx.x, op.nx, op.ny);
        for (long long n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
            double2 r = rb[n];
            if (!first) {
                const double2 ax = a_row<ADJ ? USV_APPLY_AH : USV_APPLY_A>(op, xb, n, p);
                r = csub(r, ax);
            }
            advance(p, step, op.nx, op.ny);
            r = cscale(r, op.rec[n].y);
            const C2 rv = from_d<C2>(r);
            v0[n] = rv;
            acc += cabs2(to_d(rv));
        }
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0)
        g.partial[((long long)b * g.nblk + blockIdx.x) * (g.m + 2)] = make_double2(acc, 0.0);
    if (!last_block_done(&g.counter[b], gridDim.x)) return;
    const double t = reduce_slot0(g, b, sh);
    if (threadIdx.x == 0) {
        const double beta = sqrt(t);
        if (first) {
            g.bnorm[b] = beta;
            g.atol[b] = g.rtol * beta;
            g.cycles[b] = 0;
            g.iters[b] = 0;
        } else {
            g.cycles[b] += 1;
            g.iters[b] += g.full_cycles ? g.m : g.len[b];
            const int c = g.cycles[b] - 1;
            if (c < g.hcap) g.hist[(long long)b * g.hcap + c] = g.bnorm[b] > 0 ? beta / g.bnorm[b] : 0.0;
        }
        int st = ST_ACTIVE;
        if (!isfinite(beta)) st = ST_NONFINITE;
        else if (beta <= g.atol[b]) st = ST_CONVERGED;
        else if (g.iters[b] >= g.maxiter) st = ST_MAXITER;
        g.status[b] = st;
        if (st == ST_ACTIVE) {
            g.sigma[b * (g.m + 1)] = 1.0 / beta;
            g.g[b * (g.m + 1)] = make_double2(beta, 0.0);
            for (int i = 1; i <= g.m; ++i) g.g[b * (g.m + 1) + i] = make_double2(0.0, 0.0);
            g.len[b] = g.m;
            g.ended[b] = 0;
        }
        g.counter[b] = 0;
    }
}

// ------------------------------------------------------------ Arnoldi: stencil + dots
// A CTA owns a chunk of kChunk consecutive nodes. Streaming passes over the
// Krylov basis work on node PAIRS: thread t owns the pairs at node offsets
// 2(t + kThreads k), k < kPairs, so a warp touches 512 B (complex64) or 1 KB
// (complex128) contiguous per vector. Basis vectors reach shared memory
// through a per-thread cp.async pipeline of kStages(R) stages: each thread
// copies, waits for and reads only its own 16-byte slots, so the pipeline
// needs no CTA barrier and holds no loads in registers.
constexpr int kThreads = 256;
constexpr int kPairs = 4;
constexpr int kChunk = 2 * kThreads * kPairs;  // 2048 nodes

// Per-thread node mapping and staging geometry by vector element size:
//   complex128 (16 B): pair k = nodes 2(t + kThreads k) + {0,1}, two 16-B units
//   complex64  (8 B) : same pairs, one 16-B unit per pair (cp.async staged)
//   bfloat16   (4 B) : a 16-B unit holds 4 nodes; thread t owns units at nodes
//                      4(t + kThreads u), u < kPairs/2, pair k = half k%2 of
//                      unit k/2 (cp.async staged)
template <typename C2> struct Pipe {
    static constexpr int ES = int(sizeof(C2));
    static constexpr bool STAGED = ES <= 8;                 // cp.async pipeline
    static constexpr int UNITS = kPairs * 2 * ES / 16;      // 16-B units per thread per vector
    static constexpr int S = ES == 4 ? 6 : (ES == 8 ? 4 : 3);  // stages
    static constexpr int STAGE_UNITS = UNITS * kThreads;
    static constexpr size_t BYTES = size_t(S) * STAGE_UNITS * 16;
};

// First node (chunk-relative) of this thread's pair k.
template <typename C2> __device__ __forceinline__ int pair_node(int k) {
    if constexpr (sizeof(C2) == 4) return 4 * (threadIdx.x + kThreads * (k >> 1)) + 2 * (k & 1);
    else return 2 * (threadIdx.x + kThreads * k);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gmem),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Stage basis vector t (chunk at `base`, `len` valid nodes) into stage t % S;
// slots of pairs outside the chunk (or t > last) are zero-filled, no read.
// A unit that starts inside the chunk is copied whole: a bfloat16 unit may
// run past the last node into the zeroed padding of the vector.
template <typename C2>
__device__ __forceinline__ void stage_vector(uint4* stg, const C2* base, int t, int last,
                                             int len) {
    using P = Pipe<C2>;
    static_assert(P::STAGED, "complex128 is not staged");
    const int s = t % P::S;
    const char* src0 = reinterpret_cast<const char*>(base);
#pragma unroll
    for (int u = 0; u < P::UNITS; ++u) {
        const int e = pair_node<C2>(P::ES == 4 ? 2 * u : u);
        const bool ok = t <= last && e < len;
        uint4* dst = stg + (s * P::UNITS + u) * kThreads + threadIdx.x;
        cp_async16(dst, ok ? src0 + size_t(e) * sizeof(C2) : src0, ok ? 16 : 0);
    }
    cp_async_commit();
}

// Complex value c (0/1) of pair k of stage t % S, widened to double.
template <typename C2>
__device__ __forceinline__ double2 staged(const uint4* stg, int t, int k, int c);
template <>
__device__ __forceinline__ double2 staged<float2>(const uint4* stg, int t, int k, int c) {
    using P = Pipe<float2>;
    const int s = t % P::S;
    const float4 v = reinterpret_cast<const float4*>(stg)[(s * P::UNITS + k) * kThreads + threadIdx.x];
    return c ? make_double2(v.z, v.w) : make_double2(v.x, v.y);
}
template <>
__device__ __forceinline__ double2 staged<bf2>(const uint4* stg, int t, int k, int c) {
    using P = Pipe<bf2>;
    const int s = t % P::S;
    const unsigned* v = reinterpret_cast<const unsigned*>(
        &stg[(s * P::UNITS + (k >> 1)) * kThreads + threadIdx.x]);
    const unsigned raw = v[2 * (k & 1) + c];
    return to_d(*reinterpret_cast<const bf2*>(&raw));
}

__device__ __forceinline__ void st_pair(float2* p, double2 a, double2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(float(a.x), float(a.y), float(b.x), float(b.y));
}
__device__ __forceinline__ void st_pair(double2* p, double2 a, double2 b) {
    p[0] = a;
    p[1] = b;
}
__device__ __forceinline__ void ld_pair(const float2* p, double2& a, double2& b) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    a = make_double2(v.x, v.y);
    b = make_double2(v.z, v.w);
}
__device__ __forceinline__ void ld_pair(const double2* p, double2& a, double2& b) {
    a = p[0];
    b = p[1];
}
__device__ __forceinline__ void st_pair(bf2* p, double2 a, double2 b) {
    bf2 v[2] = {from_d<bf2>(a), from_d<bf2>(b)};
    *reinterpret_cast<uint2*>(p) = *reinterpret_cast<const uint2*>(v);
}
__device__ __forceinline__ void ld_pair(const bf2* p, double2& a, double2& b) {
    const uint2 raw = *reinterpret_cast<const uint2*>(p);
    a = to_d(*reinterpret_cast<const bf2*>(&raw.x));
    b = to_d(*reinterpret_cast<const bf2*>(&raw.y));
}
__device__ __forceinline__ double2 rounded(const bf2*, double2 a) { return to_d(from_d<bf2>(a)); }
// value actually stored (rounded to the vector precision)
__device__ __forceinline__ double2 rounded(const float2*, double2 a) {
    return make_double2(double(float(a.x)), double(float(a.y)));
}
__device__ __forceinline__ double2 rounded(const double2*, double2 a) { return a; }

// Stream basis vectors t = first..last (t relative to `base`, stride nv) and
// call f(t, k, c, value) for every pair slot of this thread. complex64 goes
// through the cp.async pipeline (the caller has already issued the first
// kStages-1 vectors when `prefetched`); complex128 uses direct 16-byte loads
// unrolled over kUnroll vectors, which keeps enough bytes in flight with the
// wider elements.
template <typename C2> constexpr int kUnrollFor = 2;
template <typename C2, typename F>
__device__ __forceinline__ void stream_basis(uint4* stg, const C2* base, long long nv, int last,
                                             int len, bool prefetched, F&& f) {
    if constexpr (Pipe<C2>::STAGED) {
        using P = Pipe<C2>;
        auto issue = [&](int t) {
            stage_vector<C2>(stg, base + (long long)(t <= last ? t : 0) * nv, t, last, len);
        };
        if (!prefetched) {
#pragma unroll
            for (int t = 0; t < P::S - 1; ++t) issue(t);
        }
        for (int t = 0; t <= last; ++t) {
            issue(t + P::S - 1);
            cp_async_wait<P::S - 1>();
#pragma unroll
            for (int k = 0; k < kPairs; ++k)
#pragma unroll
                for (int c = 0; c < 2; ++c) f(t, k, c, staged<C2>(stg, t, k, c));
        }
        cp_async_wait<0>();
    } else {
        constexpr int kUnroll = kUnrollFor<C2>;
        for (int t0 = 0; t0 <= last; t0 += kUnroll) {
            double2 v[kUnroll][kPairs][2];
#pragma unroll
            for (int q = 0; q < kUnroll; ++q)
#pragma unroll
                for (int k = 0; k < kPairs; ++k) {
                    const int e = pair_node<C2>(k);
                    if (t0 + q <= last && e < len)
                        ld_pair(base + (long long)(t0 + q) * nv + e, v[q][k][0], v[q][k][1]);
                    else
                        v[q][k][0] = v[q][k][1] = make_double2(0.0, 0.0);
                }
#pragma unroll
            for (int q = 0; q < kUnroll; ++q)
                if (t0 + q <= last) {
#pragma unroll
                    for (int k = 0; k < kPairs; ++k)
#pragma unroll
                        for (int c = 0; c < 2; ++c) f(t0 + q, k, c, v[q][k][c]);
                }
        }
    }
}

// Dots of w with u_0..u_j: one warp per (basis vector, segment of the chunk),
// lanes over groups of NL nodes (one 16-byte load for complex64 / bfloat16,
// two for complex128) with kDotUnroll loads in flight, kept packed until use;
// one warp reduction per task; segments per vector grow when j is small so
// all warps work.
constexpr int kDotUnroll = 8;
constexpr int kDotsThreads = 512;

template <typename C2> struct LaneLoad;
template <> struct LaneLoad<bf2> {
    static constexpr int NL = 4;
    uint4 r;
    __device__ __forceinline__ void load(const bf2* p) { r = *reinterpret_cast<const uint4*>(p); }
    __device__ __forceinline__ void zero() { r = make_uint4(0u, 0u, 0u, 0u); }
    __device__ __forceinline__ double2 get(int i) const {
        const unsigned v = i == 0 ? r.x : i == 1 ? r.y : i == 2 ? r.z : r.w;
        return to_d(*reinterpret_cast<const bf2*>(&v));
    }
};
template <> struct LaneLoad<float2> {
    static constexpr int NL = 2;
    float4 r;
    __device__ __forceinline__ void load(const float2* p) { r = *reinterpret_cast<const float4*>(p); }
    __device__ __forceinline__ void zero() { r = make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ __forceinline__ double2 get(int i) const {
        return i ? make_double2(r.z, r.w) : make_double2(r.x, r.y);
    }
};
template <> struct LaneLoad<double2> {
    static constexpr int NL = 2;
    double2 a, b;
    __device__ __forceinline__ void load(const double2* p) { a = p[0]; b = p[1]; }
    __device__ __forceinline__ void zero() { a = b = make_double2(0.0, 0.0); }
    __device__ __forceinline__ double2 get(int i) const { return i ? b : a; }
};

// Arnoldi step j, part 1: each CTA computes its chunk of w = sigma_j K u_j
// (stencil) into shared and global memory, then the dots <sigma_t u_t, w>,
// t <= j, and ||w||^2. (A separate stencil kernel ahead of a streaming dots
// kernel measured 9% slower per iteration at 128^3: the extra launch and the
// re-read of w cost more than the overlap of the two phases gains.)
template <typename R, typename S, bool ADJ, int NT>
__global__ void __launch_bounds__(NT, 2) k_dots(OpView<R> op, S* V, GState g, int j, Step step) {
    using C2 = S;  // stored vector element
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || g.ended[b]) return;
    __shared__ __align__(16) C2 ys[kChunk];
    __shared__ double2 segsum[USV_MAX_RESTART + 2 > NT / 16 ? USV_MAX_RESTART + 2 : NT / 16];
    const long long N = op.n;
    C2* Vb = V + (long long)b * (g.m + 1) * g.nv;
    const C2* uj = Vb + (long long)j * g.nv;
    C2* w = Vb + (long long)(j + 1) * g.nv;
    const R sj = R(g.sigma[b * (g.m + 1) + j]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nw = NT / 32;
    const int tasks_t = j + 2;  // t = 0..j dots, t = j+1: ||w||^2
    int segs = 1;
    while (segs < nw && tasks_t * segs < nw) segs <<= 1;
    // each task belongs to one warp for every chunk: its sum accumulates in
    // segsum in chunk order
    for (int task = threadIdx.x; task < tasks_t * segs; task += NT)
        segsum[task] = make_double2(0.0, 0.0);
    for (int ch = blockIdx.x; ch < g.nchunk; ch += gridDim.x) {
        const long long n0 = (long long)ch * kChunk;
        const int len = int(min((long long)kChunk, N - n0));
        __syncthreads();  // the previous chunk's dots are done with ys
        Node p = decode(n0 + threadIdx.x, op.nx, op.ny);
        constexpr int kStencilUnroll = sizeof(R) == 4 ? 4 : 2;
#pragma unroll(kStencilUnroll)
        for (int e = threadIdx.x; e < kChunk; e += NT) {
            C2 y = from_d<C2>(make_double2(0.0, 0.0));
            if (e < len) {
                const long long n = n0 + e;
                y = narrow<C2>(cscale(k_row<R, ADJ, S>(op, uj, n, p), sj));
                w[n] = y;
            }
            ys[e] = y;
            advance(p, step, op.nx, op.ny);
        }
        __syncthreads();
        constexpr int NL = LaneLoad<C2>::NL;
        const int ngroups = (len + NL - 1) / NL;  // ys and the vector padding are zero past len
        const int per_seg = (ngroups + segs - 1) / segs;
        for (int task = warp; task < tasks_t * segs; task += nw) {
            const int t = task / segs, seg = task % segs;
            const int q0 = seg * per_seg, q1 = min(ngroups, q0 + per_seg);
            double re = 0.0, im = 0.0;
            if (t <= j) {
                const C2* ut = Vb + (long long)t * g.nv + n0;
                for (int qb = q0 + lane; qb < q1; qb += 32 * kDotUnroll) {
                    LaneLoad<C2> a[kDotUnroll];
#pragma unroll
                    for (int u = 0; u < kDotUnroll; ++u) {
                        const int q = qb + 32 * u;
                        if (q < q1) a[u].load(ut + NL * q);
                        else a[u].zero();
                    }
#pragma unroll
                    for (int u = 0; u < kDotUnroll; ++u) {
                        const int q = min(qb + 32 * u, ngroups - 1);
#pragma unroll
                        for (int c = 0; c < NL; ++c) {
                            const double2 y = to_d(ys[NL * q + c]);
                            const double2 av = a[u].get(c);
                            re = fma(av.x, y.x, fma(av.y, y.y, re));
                            im = fma(av.x, y.y, fma(-av.y, y.x, im));
                        }
                    }
                }
            } else {
                for (int q = q0 + lane; q < q1; q += 32)
#pragma unroll
                    for (int c = 0; c < NL; ++c) re += cabs2(to_d(ys[NL * q + c]));
            }
            re = warp_sum(re);
            im = warp_sum(im);
            if (lane == 0) segsum[task] = cadd(segsum[task], make_double2(re, im));
        }
    }
    __syncthreads();
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * (g.m + 2);
    for (int t = threadIdx.x; t < tasks_t; t += NT) {
        double re = 0.0, im = 0.0;
        for (int sg = 0; sg < segs; ++sg) {
            re += segsum[t * segs + sg].x;
            im += segsum[t * segs + sg].y;
        }
        if (t <= j) {
            const double st = g.sigma[b * (g.m + 1) + t];
            re *= st;
            im *= st;
        }
        part[t] = make_double2(re, im);
    }
    if (!last_block_done(&g.counter[b], gridDim.x)) return;
    const int nparts = int(gridDim.x);
    for (int t = warp; t <= j + 1; t += nw) {
        double re0 = 0.0, im0 = 0.0;
        const double2* pt = g.partial + (long long)b * g.nblk * (g.m + 2) + t;
        for (int q0 = 0; q0 < nparts; q0 += 32 * 4) {
            double2 pv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = q0 + 32 * u + lane;
                pv[u] = q < nparts ? ld_cg(pt + (long long)q * (g.m + 2)) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                re0 += pv[u].x;
                im0 += pv[u].y;
            }
        }
        re0 = warp_sum(re0);
        im0 = warp_sum(im0);
        if (lane == 0) {
            if (t <= j) g.H[((long long)b * g.m + j) * (g.m + 1) + t] = make_double2(re0, im0);
            else g.wnorm[b] = sqrt(re0);
        }
    }
    if (threadIdx.x == 0) g.counter[b] = 0;
}

// ------------------------------------------------------------ Arnoldi: orthogonalise + norm
template <typename S>
__global__ void __launch_bounds__(kThreads) k_orth(S* V, long long N, GState g, int j) {
    using C2 = S;
    using P = Pipe<C2>;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || g.ended[b]) return;
    extern __shared__ __align__(16) uint4 stg[];
    __shared__ double2 hs[USV_MAX_RESTART + 2];
    __shared__ double2 gsS[USV_MAX_RESTART + 1];
    __shared__ double gcS[USV_MAX_RESTART + 1];
    __shared__ double sh[32];
    const int m = g.m;
    for (int t = threadIdx.x; t <= j; t += kThreads)
        hs[t] = cscale(g.H[((long long)b * m + j) * (m + 1) + t], g.sigma[b * (m + 1) + t]);
    C2* Vb = V + (long long)b * (m + 1) * g.nv;
    __syncthreads();  // hs visible
    double acc = 0.0;
    for (int ch = blockIdx.x; ch < g.nchunk; ch += gridDim.x) {
        const long long n0 = (long long)ch * kChunk;
        const int len = int(min((long long)kChunk, N - n0));
        C2* w = Vb + (long long)(j + 1) * g.nv + n0;
        double2 u[kPairs][2];
#pragma unroll
        for (int k = 0; k < kPairs; ++k) {
            const int e = pair_node<C2>(k);
            if (e < len) ld_pair(w + e, u[k][0], u[k][1]);
            else u[k][0] = u[k][1] = make_double2(0.0, 0.0);
        }
        stream_basis<C2>(stg, Vb + n0, g.nv, j, len, false, [&](int t, int k, int c, double2 vv) {
            const double2 h = hs[t];
            u[k][c].x -= h.x * vv.x - h.y * vv.y;
            u[k][c].y -= h.x * vv.y + h.y * vv.x;
        });
#pragma unroll
        for (int k = 0; k < kPairs; ++k) {
            const int e = pair_node<C2>(k);
            if (e < len) {
                st_pair(w + e, u[k][0], u[k][1]);
                acc += cabs2(rounded(w, u[k][0]));
                if (e + 1 < len) acc += cabs2(rounded(w, u[k][1]));
            }
        }
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0)
        g.partial[((long long)b * g.nblk + blockIdx.x) * (m + 2)] = make_double2(acc, 0.0);
    if (!last_block_done(&g.counter[b], gridDim.x)) return;
    const double beta = sqrt(reduce_slot0(g, b, sh));
    // stage column j and the previous rotations in shared memory
    double2* col = g.H + ((long long)b * m + j) * (m + 1);
    for (int t = threadIdx.x; t <= j; t += kThreads) {
        hs[t] = col[t];
        if (t < j) {
            gcS[t] = g.gc[(long long)b * m + t];
            gsS[t] = g.gs[(long long)b * m + t];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        g.counter[b] = 0;
        hs[j + 1] = make_double2(beta, 0.0);
        for (int i = 0; i < j; ++i) {
            const double2 a = hs[i], c2 = hs[i + 1];
            const double c = gcS[i];
            const double2 sn = gsS[i];
            hs[i] = cadd(cscale(a, c), cmul(sn, c2));
            hs[i + 1] = csub(cscale(c2, c), cmulc(sn, a));
        }
        // rotation zeroing beta: c = |a|/r, s = (a/|a|) beta/r, rho = (a/|a|) r
        const double2 a = hs[j];
        const double aa = hypot(a.x, a.y);
        const double r = hypot(aa, beta);
        double c;
        double2 sn, rho;
        if (aa == 0.0) {
            c = 0.0;
            sn = make_double2(1.0, 0.0);
            rho = make_double2(beta, 0.0);
        } else {
            c = aa / r;
            const double2 ph = cscale(a, 1.0 / aa);
            sn = cscale(ph, beta / r);
            rho = cscale(ph, r);
        }
        hs[j] = rho;
        gcS[j] = c;
        gsS[j] = sn;
        double2* gg = g.g + (long long)b * (m + 1);
        const double2 gj = gg[j];
        const double2 gn = make_double2(-(sn.x * gj.x + sn.y * gj.y), -(sn.x * gj.y - sn.y * gj.x));
        gg[j + 1] = gn;
        gg[j] = cscale(gj, c);
        const bool nonfinite = !isfinite(beta);
        const bool breakdown = !(beta > 1e-30 * g.wnorm[b]);
        g.sigma[b * (m + 1) + j + 1] = (breakdown || nonfinite) ? 0.0 : 1.0 / beta;
        const double resid = hypot(gn.x, gn.y);
        const bool end = (j == m - 1) || breakdown || nonfinite ||
                         (!g.full_cycles && resid <= g.atol[b]);
        if (end) {
            g.len[b] = j + 1;
            g.ended[b] = 1;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t <= j; t += kThreads) col[t] = hs[t];
    if (threadIdx.x == 0) {
        g.gc[(long long)b * m + j] = gcS[j];
        g.gs[(long long)b * m + j] = gsS[j];
    }
}

// ------------------------------------------------------------ least squares (once per cycle)
// Back-substitution R y = g on the Givens-reduced Hessenberg, staged in
// shared memory; y is stored pre-multiplied by sigma (the basis scales).
__global__ void __launch_bounds__(128) k_lsq(GState g) {
    const int b = blockIdx.x;
    if (g.status[b] != ST_ACTIVE || !g.ended[b]) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int m = g.m, L = g.len[b];
    double2* Rs = reinterpret_cast<double2*>(smem_raw);  // L x L, column-major
    double2* gv = Rs + (size_t)L * L;
    for (int idx = threadIdx.x; idx < L * L; idx += blockDim.x) {
        const int k = idx / L, i = idx % L;
        Rs[idx] = i <= k ? g.H[((long long)b * m + k) * (m + 1) + i] : make_double2(0.0, 0.0);
    }
    for (int i = threadIdx.x; i < L; i += blockDim.x) gv[i] = g.g[(long long)b * (m + 1) + i];
    __syncthreads();
    for (int k = L - 1; k >= 0; --k) {
        // y_k = g_k / R_kk (every thread computes it from shared memory)
        const double2 yk = cmul(gv[k], cinv(Rs[(size_t)k * L + k]));
        __syncthreads();
        for (int i = threadIdx.x; i < k; i += blockDim.x)
            gv[i] = csub(gv[i], cmul(Rs[(size_t)k * L + i], yk));
        if (threadIdx.x == 0) gv[k] = yk;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < L; i += blockDim.x)
        g.y[(long long)b * m + i] = cscale(gv[i], g.sigma[b * (m + 1) + i]);
}

// ------------------------------------------------------------ solution update (fp64)
template <typename S>
__global__ void __launch_bounds__(kThreads) k_update(OpView<double> op, const S* V, double2* x,
                                                     long long ld, GState g) {
    using C2 = S;
    using P = Pipe<C2>;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || !g.ended[b]) return;
    extern __shared__ __align__(16) uint4 stg[];
    __shared__ double2 ys[USV_MAX_RESTART];
    const int L = g.len[b];
    for (int t = threadIdx.x; t < L; t += kThreads) ys[t] = g.y[(long long)b * g.m + t];
    const long long N = op.n;
    __syncthreads();  // ys visible
    for (int ch = blockIdx.x; ch < g.nchunk; ch += gridDim.x) {
        const long long n0 = (long long)ch * kChunk;
        const int len = int(min((long long)kChunk, N - n0));
        const C2* base = V + (long long)b * (g.m + 1) * g.nv + n0;
        double2 acc[kPairs][2];
#pragma unroll
        for (int k = 0; k < kPairs; ++k) acc[k][0] = acc[k][1] = make_double2(0.0, 0.0);
        stream_basis<C2>(stg, base, g.nv, L - 1, len, false, [&](int t, int k, int c, double2 vv) {
            acc[k][c] = cadd(acc[k][c], cmul(ys[t], vv));
        });
        double2* xb = x + b * ld + n0;
#pragma unroll
        for (int k = 0; k < kPairs; ++k)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int e = pair_node<C2>(k) + c;
                if (e < len) {
                    const double4 rc = op.rec[n0 + e];
                    xb[e] = cadd(xb[e], cmul(make_double2(rc.z, rc.w), acc[k][c]));
                }
            }
    }
}

// ------------------------------------------------------------ final gates (fp64)
// iterative_solver.py:70-79: ||R(OP x) - Rb|| / ||Rb|| and
// max |OP x - b| / max(|OP||x| + |b|, 1e-30), plus a finiteness check.
template <bool ADJ>
__global__ void __launch_bounds__(256) k_gates(OpView<double> op, const double2* rhs,
                                               const double2* x, long long ld, GState g) {
    const int b = blockIdx.y;
    __shared__ double sh[32];
    const double2* rb = rhs + b * ld;
    const double2* xb = x + b * ld;
    double s2 = 0.0, b2 = 0.0, bwd = 0.0, bad = 0.0;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < op.n;
         n += (long long)gridDim.x * blockDim.x) {
        const Node p = decode(n, op.nx, op.ny);
        const double2 ax = a_row<ADJ ? USV_APPLY_AH : USV_APPLY_A>(op, xb, n, p);
        const double2 den = a_row<ADJ ? USV_APPLY_ABS_AH : USV_APPLY_ABS_A>(op, xb, n, p);
        const double2 bv = rb[n];
        const double2 r = csub(ax, bv);
        const double Rs = op.rec[n].y;
        s2 += cabs2(cscale(r, Rs));
        b2 += cabs2(cscale(bv, Rs));
        const double e = hypot(r.x, r.y) / fmax(den.x + hypot(bv.x, bv.y), 1e-30);
        bwd = (e > bwd || isnan(e)) ? e : bwd;
        if (!isfinite(xb[n].x) || !isfinite(xb[n].y)) bad += 1.0;
    }
    s2 = block_sum(s2, sh);
    b2 = block_sum(b2, sh);
    bad = block_sum(bad, sh);
    bwd = block_max(isnan(bwd) ? INFINITY : bwd, sh);
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * (g.m + 2);
    if (threadIdx.x == 0) {
        part[0] = make_double2(s2, b2);
        part[1] = make_double2(bwd, bad);
    }
    if (!last_block_done(&g.counter[b], gridDim.x)) return;
    double ts = 0, tb = 0, tw = 0, tbad = 0;
    for (int q = threadIdx.x; q < int(gridDim.x); q += blockDim.x) {
        const double2* pq = g.partial + ((long long)b * g.nblk + q) * (g.m + 2);
        const double2 p0 = ld_cg(pq), p1 = ld_cg(pq + 1);
        ts += p0.x;
        tb += p0.y;
        tw = fmax(tw, p1.x);
        tbad += p1.y;
    }
    ts = block_sum(ts, sh);
    tb = block_sum(tb, sh);
    tbad = block_sum(tbad, sh);
    tw = block_max(tw, sh);
    if (threadIdx.x == 0) {
        double* out = g.gates + 4 * b;
        out[0] = tb > 0 ? sqrt(ts) / sqrt(tb) : 0.0;
        out[1] = tb > 0 ? tw : 0.0;
        out[2] = tbad;
        out[3] = sqrt(tb);
        g.counter[b] = 0;
    }
}

// ------------------------------------------------------------ host driver
static cudaStream_t capture_stream() {
    static thread_local cudaStream_t s = nullptr;
    static thread_local int dev = -1;
    int cur = 0;
    cudaGetDevice(&cur);
    if (s == nullptr || dev != cur) {
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        dev = cur;
    }
    return s;
}


template <typename R, typename S, bool ADJ>
static int run_gmres(const usv_scene& s, const void* op_buf, const usv_gmres_params& p,
                     const double2* rhs, double2* x, int B, long long ld, char* ws,
                     const WsLayout& L, GState& g, usv_gmres_stats* stats, cudaStream_t strm) {
    using C2 = S;  // stored Krylov vector element
    const OpView<double> op64 = make_view<double>(s, op_buf, ADJ);
    const OpView<R> opk = make_view<R>(s, op_buf, ADJ);
    C2* V = reinterpret_cast<C2*>(ws + L.V);
    const size_t lsq_smem = sizeof(double2) * size_t(g.m) * (g.m + 1);
    const size_t pipe_smem = Pipe<C2>::STAGED ? Pipe<C2>::BYTES : 16;
    const Step step = make_step(kThreads, s.nx, s.ny);
    const Step step_d = make_step(kDotsThreads, s.nx, s.ny);
    USV_CUDA_TRY(cudaFuncSetAttribute(k_orth<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(pipe_smem)));
    USV_CUDA_TRY(cudaFuncSetAttribute(k_update<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(pipe_smem)));
    // Grids fill the GPU once (resident CTAs per SM x SMs, shared by the B
    // right-hand sides); every CTA loops over node chunks, so there is no
    // partial last wave and the last CTA reduces one partial per CTA.
    int dev = 0, sms = 0;
    USV_CUDA_TRY(cudaGetDevice(&dev));
    USV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    auto grid_for = [&](const void* fn, int threads, size_t smem, dim3& grid) -> int {
        int per_sm = 0;
        USV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
        long long x = (long long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1) / B;
        x = x < 1 ? 1 : (x > g.nchunk ? g.nchunk : x);
        grid = dim3(unsigned(x), unsigned(B));
        return USV_OK;
    };
    dim3 grid_res, grid_dots, grid_orth, grid_upd, grid_gates;
    if (int e = grid_for((const void*)k_residual<ADJ, C2>, 256, 0, grid_res)) return e;
    if (int e = grid_for((const void*)k_dots<R, S, ADJ, kDotsThreads>, kDotsThreads, 0, grid_dots))
        return e;
    if (int e = grid_for((const void*)k_orth<S>, kThreads, pipe_smem, grid_orth)) return e;
    if (int e = grid_for((const void*)k_update<S>, kThreads, pipe_smem, grid_upd)) return e;
    if (int e = grid_for((const void*)k_gates<ADJ>, 256, 0, grid_gates)) return e;
    if (lsq_smem > 48 * 1024)
        USV_CUDA_TRY(cudaFuncSetAttribute(k_lsq, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(lsq_smem)));
    // zero the state and the solution
    USV_CUDA_TRY(cudaMemsetAsync(ws + L.state_begin, 0, L.total - L.state_begin, strm));
    // paired loads may touch the padding past node n-1 of each basis vector:
    // keep it zero so it contributes nothing to the dots
    if (g.nv > g.n)
        USV_CUDA_TRY(cudaMemset2DAsync(V + g.n, g.nv * sizeof(C2), 0, (g.nv - g.n) * sizeof(C2),
                                       size_t(g.m + 1) * B, strm));
    USV_CUDA_TRY(cudaMemset2DAsync(x, ld * sizeof(double2), 0, g.n * sizeof(double2), B, strm));
    k_residual<ADJ, C2><<<grid_res, 256, 0, strm>>>(op64, rhs, x, ld, V, g, 1, step);
    USV_CUDA_TRY(cudaGetLastError());

    // Event timing: one event before the first kernel of a cycle and one after
    // every kernel; consecutive pairs bracket single launches.
    usv_gmres_profile* prof = p.profile;
    const int kernels_per_cycle = 2 * g.m + 3;
    std::vector<cudaEvent_t> ev;
    std::vector<int> fam;
    if (prof) {
        ev.resize(kernels_per_cycle + 1);
        for (auto& e : ev) USV_CUDA_TRY(cudaEventCreate(&e));
    }
    const double vb = double(sizeof(C2)), nn = double(g.n);
    std::vector<double> fam_bytes;
    auto mark = [&](cudaStream_t st, int idx, bool capturing) {
        if (!prof) return cudaSuccess;
        return capturing ? cudaEventRecordWithFlags(ev[idx], st, cudaEventRecordExternal)
                         : cudaEventRecord(ev[idx], st);
    };
    auto launch_cycle = [&](cudaStream_t st, bool capturing) -> int {
        int k = 0;
        fam.clear();
        fam_bytes.clear();
        USV_CUDA_TRY(mark(st, k++, capturing));
        for (int j = 0; j < g.m; ++j) {
            k_dots<R, S, ADJ, kDotsThreads><<<grid_dots, kDotsThreads, 0, st>>>(opk, V, g, j, step_d);
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(0);
            // read u_0..u_j (u_j also feeds the stencil) + node record, write w
            fam_bytes.push_back(nn * (vb * (j + 2) + 4.0 * sizeof(R)));
            k_orth<S><<<grid_orth, kThreads, pipe_smem, st>>>(V, g.n, g, j);
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(1);
            fam_bytes.push_back(nn * vb * (j + 3));
        }
        k_lsq<<<B, 128, lsq_smem, st>>>(g);
        USV_CUDA_TRY(mark(st, k++, capturing));
        fam.push_back(2);
        fam_bytes.push_back(0.0);
        k_update<S><<<grid_upd, kThreads, pipe_smem, st>>>(op64, V, x, ld, g);
        USV_CUDA_TRY(mark(st, k++, capturing));
        fam.push_back(3);
        fam_bytes.push_back(nn * (vb * g.m + 2 * sizeof(double2) + sizeof(double4)));
        k_residual<ADJ, C2><<<grid_res, 256, 0, st>>>(op64, rhs, x, ld, V, g, 0, step);
        USV_CUDA_TRY(mark(st, k++, capturing));
        fam.push_back(4);
        fam_bytes.push_back(nn * (2 * sizeof(double2) + sizeof(double4) + sizeof(double2) + vb));
        USV_CUDA_TRY(cudaGetLastError());
        return USV_OK;
    };
    auto accumulate = [&](std::vector<int>& active_counts) -> int {
        if (!prof) return USV_OK;
        for (size_t i = 0; i < fam.size(); ++i) {
            float ms = 0.f;
            USV_CUDA_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            prof->milliseconds[fam[i]] += ms;
            prof->launches[fam[i]] += 1;
            prof->bytes[fam[i]] += fam_bytes[i] * active_counts[0];
        }
        return USV_OK;
    };

    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    if (p.use_graph) {
        cudaStream_t cap = capture_stream();
        USV_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int st = launch_cycle(cap, true);
        cudaError_t e = cudaStreamEndCapture(cap, &graph);
        if (st) return st;
        USV_CUDA_TRY(e);
        USV_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
    }
    std::vector<int> status(B);
    std::vector<int> active(1, 0);
    int rc = USV_OK;
    bool pending = false;
    const int max_cycles = p.maxiter + 2;  // safety bound; the device status ends the loop
    for (int cycle = 0; cycle <= max_cycles; ++cycle) {
        cudaError_t e = cudaMemcpyAsync(status.data(), ws + L.status, sizeof(int) * B,
                                        cudaMemcpyDeviceToHost, strm);
        if (e == cudaSuccess) e = cudaStreamSynchronize(strm);
        if (e != cudaSuccess) { rc = set_last_cuda_error(e); break; }
        if (pending) {
            rc = accumulate(active);
            if (rc) break;
            pending = false;
        }
        int any = 0;
        for (int b = 0; b < B; ++b) any += status[b] == ST_ACTIVE;
        if (!any) break;
        active[0] = any;
        if (exec) {
            e = cudaGraphLaunch(exec, strm);
            if (e != cudaSuccess) { rc = set_last_cuda_error(e); break; }
        } else {
            rc = launch_cycle(strm, false);
            if (rc) break;
        }
        pending = true;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (rc) {
        for (auto& e : ev) cudaEventDestroy(e);
        return rc;
    }
    if (prof) USV_CUDA_TRY(cudaEventRecord(ev[0], strm));
    k_gates<ADJ><<<grid_gates, 256, 0, strm>>>(op64, rhs, x, ld, g);
    USV_CUDA_TRY(cudaGetLastError());
    if (prof) {
        USV_CUDA_TRY(cudaEventRecord(ev[1], strm));
        USV_CUDA_TRY(cudaEventSynchronize(ev[1]));
        float ms = 0.f;
        USV_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        prof->milliseconds[5] += ms;
        prof->launches[5] += 1;
        prof->bytes[5] += nn * B * (2 * sizeof(double2) + sizeof(double4) + sizeof(double2));
        for (auto& e : ev) cudaEventDestroy(e);
    }
    std::vector<double> gates(4 * B);
    std::vector<int> cycles(B), iters(B);
    USV_CUDA_TRY(cudaMemcpyAsync(gates.data(), ws + L.gates, sizeof(double) * 4 * B,
                                 cudaMemcpyDeviceToHost, strm));
    USV_CUDA_TRY(cudaMemcpyAsync(cycles.data(), ws + L.cycles, sizeof(int) * B,
                                 cudaMemcpyDeviceToHost, strm));
    USV_CUDA_TRY(cudaMemcpyAsync(iters.data(), ws + L.iters, sizeof(int) * B,
                                 cudaMemcpyDeviceToHost, strm));
    USV_CUDA_TRY(cudaMemcpyAsync(status.data(), ws + L.status, sizeof(int) * B,
                                 cudaMemcpyDeviceToHost, strm));
    if (p.history && p.history_capacity > 0)
        USV_CUDA_TRY(cudaMemcpyAsync(p.history, ws + L.hist,
                                     sizeof(double) * size_t(B) * p.history_capacity,
                                     cudaMemcpyDeviceToHost, strm));
    USV_CUDA_TRY(cudaStreamSynchronize(strm));
    for (int b = 0; b < B; ++b) {
        usv_gmres_stats& st = stats[b];
        st.cycles = cycles[b];
        st.iterations = iters[b];
        st.scaled_residual = gates[4 * b];
        st.backward_error = gates[4 * b + 1];
        st.initial_residual = gates[4 * b + 3];
        // CuPy reports info = iterations only when the cap was hit exactly
        st.info = (status[b] != ST_CONVERGED && iters[b] == p.maxiter) ? iters[b] : 0;
        const bool finite = gates[4 * b + 2] == 0.0;
        if (!finite || status[b] == ST_NONFINITE) st.status = USV_ERR_NONFINITE;
        else if (st.info != 0 || status[b] != ST_CONVERGED || !(st.scaled_residual <= p.rtol) ||
                 !(st.backward_error <= p.backward_error_tol))
            st.status = USV_ERR_NOT_CONVERGED;
        else st.status = USV_OK;
    }
    return USV_OK;
}

static size_t vector_bytes(int precision) {
    return precision == USV_PREC_FP64 ? sizeof(double2)
                                      : precision == USV_PREC_MIXED_BF16 ? sizeof(bf2) : sizeof(float2);
}

static int check_params(const usv_scene* scene, const usv_gmres_params* p, int nrhs,
                        long long* n, int* m, int* chunk, int* nblk) {
    if (!scene || !p || nrhs < 1 || nrhs > 65535) return USV_ERR_ARG;
    *n = (long long)scene->nx * scene->ny * scene->nz;
    if (*n < 8) return USV_ERR_ARG;
    if (p->restart < 1 || p->restart > USV_MAX_RESTART || p->maxiter < 0) return USV_ERR_ARG;
    if (p->history_capacity < 0) return USV_ERR_ARG;
    if (!(p->rtol >= 0) || !(p->backward_error_tol >= 0)) return USV_ERR_ARG;
    if (p->precision != USV_PREC_FP64 && p->precision != USV_PREC_MIXED &&
        p->precision != USV_PREC_MIXED_BF16)
        return USV_ERR_ARG;
    *m = int(p->restart < *n ? p->restart : *n);
    *chunk = kChunk;  // node chunk per CTA (block_nodes is reserved)
    if (p->block_nodes != 0 && p->block_nodes != kChunk) return USV_ERR_ARG;
    *nblk = int((*n + *chunk - 1) / *chunk);
    return USV_OK;
}

}  // namespace usv

using namespace usv;

extern "C" {

int usv_gmres_workspace_bytes(const usv_scene* scene, const usv_gmres_params* params, int nrhs,
                              size_t* bytes) {
    long long n;
    int m, chunk, nblk;
    int st = check_params(scene, params, nrhs, &n, &m, &chunk, &nblk);
    if (st) return st;
    if (!bytes) return USV_ERR_ARG;
    const size_t vb = vector_bytes(params->precision);
    *bytes = ws_layout(n, m, nrhs, nblk, vb, params->history_capacity).total;
    return USV_OK;
}

int usv_gmres_solve(const usv_scene* scene, const void* op_buf, const usv_gmres_params* params,
                    const void* rhs, void* x, int nrhs, int64_t ld, void* workspace,
                    size_t workspace_bytes, usv_gmres_stats* stats, void* stream) {
    long long n;
    int m, chunk, nblk;
    int st = check_params(scene, params, nrhs, &n, &m, &chunk, &nblk);
    if (st) return st;
    if (!op_buf || !rhs || !x || !workspace || !stats || ld < n) return USV_ERR_ARG;
    const size_t vb = vector_bytes(params->precision);
    const WsLayout L = ws_layout(n, m, nrhs, nblk, vb, params->history_capacity);
    if (workspace_bytes < L.total) return USV_ERR_WORKSPACE;
    char* ws = static_cast<char*>(workspace);
    GState g{};
    g.m = m;
    g.nblk = nblk;
    g.nchunk = nblk;
    g.chunk = chunk;
    g.full_cycles = params->full_cycles ? 1 : 0;
    g.maxiter = params->maxiter;
    g.n = n;
    g.nv = padded(n);
    g.rtol = params->rtol;
    g.partial = reinterpret_cast<double2*>(ws + L.partial);
    g.H = reinterpret_cast<double2*>(ws + L.H);
    g.gc = reinterpret_cast<double*>(ws + L.gc);
    g.gs = reinterpret_cast<double2*>(ws + L.gs);
    g.g = reinterpret_cast<double2*>(ws + L.g);
    g.y = reinterpret_cast<double2*>(ws + L.y);
    g.sigma = reinterpret_cast<double*>(ws + L.sigma);
    g.bnorm = reinterpret_cast<double*>(ws + L.bnorm);
    g.atol = reinterpret_cast<double*>(ws + L.atol);
    g.wnorm = reinterpret_cast<double*>(ws + L.wnorm);
    g.gates = reinterpret_cast<double*>(ws + L.gates);
    g.hist = reinterpret_cast<double*>(ws + L.hist);
    g.hcap = params->history_capacity > 0 ? params->history_capacity : 0;
    g.status = reinterpret_cast<int*>(ws + L.status);
    g.cycles = reinterpret_cast<int*>(ws + L.cycles);
    g.iters = reinterpret_cast<int*>(ws + L.iters);
    g.len = reinterpret_cast<int*>(ws + L.len);
    g.ended = reinterpret_cast<int*>(ws + L.ended);
    g.counter = reinterpret_cast<unsigned*>(ws + L.counter);
    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    const double2* b = static_cast<const double2*>(rhs);
    double2* xx = static_cast<double2*>(x);
    const bool adj = params->adjoint != 0;
#define USV_RUN(R, S, A) run_gmres<R, S, A>(*scene, op_buf, *params, b, xx, nrhs, ld, ws, L, g, stats, strm)
    if (params->precision == USV_PREC_FP64)
        return adj ? USV_RUN(double, double2, true) : USV_RUN(double, double2, false);
    if (params->precision == USV_PREC_MIXED_BF16)
        return adj ? USV_RUN(float, bf2, true) : USV_RUN(float, bf2, false);
    return adj ? USV_RUN(float, float2, true) : USV_RUN(float, float2, false);
#undef USV_RUN
}

}  // extern "C"
