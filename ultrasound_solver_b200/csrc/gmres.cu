// Restarted, right-preconditioned GMRES(m) on the row-scaled Jacobi operator
// K = R A S (or K' = R' A^H S' for the adjoint), batched over right-hand
// sides, with Krylov vectors in complex64 (USV_PREC_MIXED), bfloat16
// (USV_PREC_MIXED_BF16) or complex128 (USV_PREC_FP64).
//
// Algorithm parity: iterative_solver.py:30-104 drives CuPy's gmres
// (cupyx.scipy.sparse.linalg.gmres, cupy>=14, not vendored by the
// reference): x0 = 0, residual r = Rb - K x tested against rtol*||Rb|| only
// at restarts, one-pass classical Gram-Schmidt, all m steps per cycle,
// least squares of the (m+1) x m Hessenberg, x += V y, solution S x.
// Here the restart residual r = R (b - A x_sol) and the solution x_sol are
// always FP64 (the correction V y is summed in FP64, in fp32 for bfloat16
// vectors); the Gram-Schmidt reductions and the Hessenberg / Givens least
// squares are FP64 on the device; the Krylov vectors and the in-cycle stencil
// use the vector precision. With complex64 or bfloat16 vectors this is GMRES
// with FP64 iterative refinement at every restart.
//
// Per Arnoldi step two kernels run over (node chunk, RHS):
//   k_dots : w = sigma_j K u_j (stencil) stored as u_{j+1}; partial dots
//            <sigma_t u_t, w>, t<=j, and ||w||^2, reduced by the last CTA
//   k_orth : u_{j+1} = w - sum_t h_tj sigma_t u_t, ||u_{j+1}||^2; the last
//            CTA forms beta, applies the Givens rotations, and at the end of
//            the cycle back-substitutes y.
// Basis vectors are stored unnormalised with a scale sigma_t = 1/||u_t||.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "dense.h"
#include "usv_internal.cuh"

#define USV_MAX_RESTART 112  // keeps the m x (m+1) least-squares tile in shared memory

static_assert(sizeof(usv_gmres_params) == 80, "usv_gmres_params layout (include/usv.h)");

namespace usv {

enum { ST_ACTIVE = 0, ST_CONVERGED = 1, ST_MAXITER = 2, ST_NONFINITE = 3,
       ST_DEVICE_TIMEOUT = 4 };  // a bounded device-side wait ran out

// Per-RHS control words of a recycled (GCRO-DR) cycle, written by the host
// before each cycle.
enum {
    CW_KC = 0,      // recycled vectors used by this cycle (0 or k)
    CW_PAIR,        // pair buffer (U, C) used by this cycle
    CW_VBUF,        // Krylov buffer of this cycle
    CW_COMBINE,     // 1: build pair CW_DST at the start of this cycle
    CW_SRC_PAIR,    // pair used by the cycle whose data builds the new pair
    CW_SRC_VBUF,    // its Krylov buffer
    CW_SRC_KC,      // its recycled count
    CW_DST,         // pair buffer written by the combine
    CW_HARVEST,     // 1: this cycle's data feeds a harmonic Ritz step
    kCtl
};
constexpr int kPairBufs = 3;   // pairs in use: this cycle's, the source cycle's, the new one
constexpr int kVBufs = 2;      // Krylov buffers: this cycle's and the previous cycle's

struct GState {
    int m, nblk, chunk, full_cycles, maxiter;
    int nchunk;        // node chunks of `chunk` nodes; CTAs loop over them (grid <= nblk)
    int ps;            // partial-sum slots per CTA
    long long n;
    long long nv;      // Krylov vector stride: n rounded up to 64 (512-B aligned pairs)
    double rtol;
    double2* partial;  // [B][nblk][ps], one row per CTA of the launch
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
    // recycling (GCRO-DR), kr > 0 only
    int kr;            // recycled vectors k
    int hb_len;        // doubles per RHS in the host-read block
    long long vstride; // elements between the Krylov buffers (B (m+1) nv)
    long long pstride; // elements between pair buffers (B k nv)
    void* Ubuf;        // [kPairBufs][B][k][nv] U, K U = C
    void* Cbuf;        // [kPairBufs][B][k][nv] C, orthonormal
    int* ctl;          // [B][kCtl]
    double2* coef;     // [B][k + m + 1][2k] combine coefficients
    double* hb;        // [B][hb_len] read by the host after each cycle:
                       //   raw G columns [m][m+1] complex, bd [m+1][k] complex,
                       //   sigma [m+1], d [k], then len, kc
    double* dU;        // [kPairBufs][B][k] 1/||U_i||
    double2* alpha;    // [B][k] projection C^H r of the cycle's first residual
    int* klast;        // [B] recycled count of the last finished cycle
    int* started;      // [B]
    const struct SceneSlot* slots;  // [B] multi-scene solves: the scene of each RHS
};

// Scene of one right-hand side of a multi-scene solve (usv_gmres_solve_scenes):
// the operator views, node count and chunk count of that scene and the node
// steps of the 256- and kDotsThreads-thread kernels. Kernels instantiated
// with MS = true read their scene from here (blockIdx.y = right-hand side);
// single-scene kernels take it from their arguments.
struct SceneSlot {
    OpView<double> op64;
    OpView<float> op32;
    long long n;
    int nchunk;
    Step step, step_d;
};
template <typename R> __device__ __forceinline__ const OpView<R>& slot_view(const SceneSlot& s);
template <> __device__ __forceinline__ const OpView<double>& slot_view<double>(const SceneSlot& s) {
    return s.op64;
}
template <> __device__ __forceinline__ const OpView<float>& slot_view<float>(const SceneSlot& s) {
    return s.op32;
}
// CTAs of the launch that work for right-hand side b: all of them for a
// single scene; for a multi-scene batch a share proportional to the RHS's
// scene size (the grid is sized for the largest scene), at least one.
template <bool MS> __device__ __forceinline__ int rhs_ctas(const GState& g, int b) {
    if constexpr (MS) {
        const long long c = ((long long)gridDim.x * g.slots[b].n + g.n - 1) / g.n;
        return int(c < 1 ? 1 : c);
    } else {
        return int(gridDim.x);
    }
}


// host-read block offsets (in doubles)
__host__ __device__ __forceinline__ int hb_graw(int) { return 0; }
__host__ __device__ __forceinline__ int hb_bd(int m) { return 2 * m * (m + 1); }
__host__ __device__ __forceinline__ int hb_sigma(int m, int k) { return hb_bd(m) + 2 * (m + 1) * k; }
__host__ __device__ __forceinline__ int hb_d(int m, int k) { return hb_sigma(m, k) + m + 1; }
__host__ __device__ __forceinline__ int hb_tail(int m, int k) { return hb_d(m, k) + k; }
__host__ __device__ __forceinline__ int hb_size(int m, int k) { return hb_tail(m, k) + 2; }

struct WsLayout {
    size_t V, partial, H, gc, gs, g, y, sigma, bnorm, atol, wnorm, gates, hist, status, cycles,
        iters, len, ended, counter, state_begin, total;
    size_t U, C, bpart, coef, hb, dU, alpha, klast, started, ctl;  // recycling
    size_t slots;  // multi-scene solves: SceneSlot per right-hand side
};

static long long padded(long long n) { return (n + 63) / 64 * 64; }

// Partial-sum slots per CTA: m+2 for the Arnoldi dots, (m+1) k for the
// recycled-space dots.
static int partial_slots(int m, int k) { return k > 0 && (m + 1) * k > m + 2 ? (m + 1) * k : m + 2; }

static WsLayout ws_layout(long long n, int m, int B, int nblk, size_t vec_bytes, int hcap, int k) {
    WsLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes);
        return o;
    };
    const size_t vecs = size_t(padded(n)) * vec_bytes;
    L.V = take(vecs * size_t(m + 1) * size_t(B) * (k > 0 ? kVBufs : 1));
    if (k > 0) {
        L.U = take(vecs * size_t(k) * B * kPairBufs);
        L.C = take(vecs * size_t(k) * B * kPairBufs);
        L.coef = take(sizeof(double2) * size_t(B) * (k + m + 1) * 2 * k);
        L.hb = take(sizeof(double) * size_t(B) * hb_size(m, k));
        L.ctl = take(sizeof(int) * size_t(B) * kCtl);
    }
    L.partial = take(sizeof(double2) * size_t(B) * nblk * partial_slots(m, k));
    // (before state_begin: the driver clears the state after uploading the slots)
    L.slots = take(sizeof(SceneSlot) * size_t(B));
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
    if (k > 0) {
        L.dU = take(sizeof(double) * size_t(kPairBufs) * B * k);
        L.alpha = take(sizeof(double2) * size_t(B) * k);
        L.klast = take(sizeof(int) * B);
        L.started = take(sizeof(int) * B);
    }
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

// Sum of the nparts norm partials (slot 0) by the last CTA, in a fixed
// order (thread-strided, then the block tree).
__device__ __forceinline__ double reduce_slot0(const GState& g, int b, double* sh, int nparts) {
    double t = 0.0;
    const double2* p = g.partial + (long long)b * g.nblk * g.ps;
    for (int q = threadIdx.x; q < nparts; q += blockDim.x)
        t += ld_cg(p + (long long)q * g.ps).x;
    return block_sum(t, sh);
}

// Vectors of RHS b's current cycle: t < kc are the recycled C_t (and U_t for
// the solution update), the others Krylov slots of the cycle's buffer.
template <typename S> struct CycleBasis {
    S* V;        // Krylov slot 0
    const S* C;  // C_0 of the cycle's pair (kc > 0)
    const S* U;  // U_0 of the cycle's pair (kc > 0)
    int kc;
    int pair;
};
template <typename S>
__device__ __forceinline__ CycleBasis<S> cycle_basis(S* V, const GState& g, int b) {
    CycleBasis<S> cb;
    cb.V = V + (long long)b * (g.m + 1) * g.nv;
    cb.C = cb.U = cb.V;
    cb.kc = 0;
    cb.pair = 0;
    if (g.kr > 0) {
        const int* cw = g.ctl + b * kCtl;
        cb.V += cw[CW_VBUF] * g.vstride;
        cb.kc = cw[CW_KC];
        cb.pair = cw[CW_PAIR] > 0 ? cw[CW_PAIR] : 0;
        const long long po = cb.pair * g.pstride + (long long)b * g.kr * g.nv;
        cb.C = static_cast<const S*>(g.Cbuf) + po;
        cb.U = static_cast<const S*>(g.Ubuf) + po;
    }
    return cb;
}

// ------------------------------------------------------------ residual
// r = Rs (rhs - OP x) in fp64 (OP = A or A^H) into Krylov slot kc of the
// cycle; first=1 (or, when recycling, the first call for this RHS): x = 0,
// r = Rs rhs. Recycled cycles (kc > 0) also set up the fixed leading block of
// G = [[D, B], [0, Hbar]]: columns t < kc are d_t e_t (identity rotations),
// C slots have unit scale; the projection kernels then form beta.
template <bool ADJ, typename C2, bool MS = false>
__global__ void __launch_bounds__(256) k_residual(OpView<double> op, const double2* rhs,
                                                  const double2* x, long long ld, C2* V,
                                                  GState g, int first, Step step) {
    const int b = blockIdx.y;
    if (g.kr > 0) first = !g.started[b];
    if (!first && (g.status[b] != ST_ACTIVE)) return;
    int nchunk = g.nchunk;
    if constexpr (MS) {
        const SceneSlot& sl = g.slots[b];
        op = sl.op64;
        step = sl.step;
        nchunk = sl.nchunk;
    }
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    __shared__ double sh[32];
    const double2* rb = rhs + b * ld;
    const double2* xb = x + b * ld;
    const CycleBasis<C2> cb = cycle_basis(V, g, b);
    C2* v0 = cb.V + (long long)cb.kc * g.nv;
    double acc = 0.0, acc_s = 0.0;
    for (int ch = blockIdx.x; ch < nchunk; ch += ncta) {
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
            acc += cabs2(r);
            acc_s += cabs2(to_d(rv));
        }
    }
    acc = block_sum(acc, sh);
    acc_s = block_sum(acc_s, sh);
    if (threadIdx.x == 0)
        g.partial[((long long)b * g.nblk + blockIdx.x) * g.ps] = make_double2(acc, acc_s);
    if (!last_block_done(&g.counter[b], ncta)) return;
    // FP64 norm of the residual (the convergence test, like the final gate)
    // and of its stored copy (the scale of the cycle's first basis vector)
    const double t = reduce_slot0(g, b, sh, ncta);
    double ts = 0.0;
    {
        const double2* pp = g.partial + (long long)b * g.nblk * g.ps;
        for (int q = threadIdx.x; q < ncta; q += blockDim.x) ts += ld_cg(pp + (long long)q * g.ps).y;
        ts = block_sum(ts, sh);
    }
    __shared__ int st_sh;
    const int m = g.m, kc = cb.kc;
    if (threadIdx.x == 0) {
        const double beta = sqrt(t), beta_s = sqrt(ts);
        if (first) {
            g.bnorm[b] = beta;
            g.atol[b] = g.rtol * beta;
            g.cycles[b] = 0;
            g.iters[b] = 0;
            if (g.kr > 0) g.started[b] = 1;
        } else {
            g.cycles[b] += 1;
            g.iters[b] += (g.full_cycles ? m : g.len[b]) - (g.kr > 0 ? g.klast[b] : 0);
            const int c = g.cycles[b] - 1;
            if (c < g.hcap) g.hist[(long long)b * g.hcap + c] = g.bnorm[b] > 0 ? beta / g.bnorm[b] : 0.0;
        }
        int st = ST_ACTIVE;
        if (!isfinite(beta)) st = ST_NONFINITE;
        // (a hair inside atol: the final gate recomputes this norm with another
        // summation order and must not miss rtol by a rounding)
        else if (beta <= g.atol[b] * (1.0 - 1e-12)) st = ST_CONVERGED;
        else if (g.iters[b] >= g.maxiter) st = ST_MAXITER;
        g.status[b] = st;
        st_sh = st;
        if (st == ST_ACTIVE) {
            g.sigma[b * (m + 1) + kc] = 1.0 / beta_s;
            for (int i = 0; i <= m; ++i) g.g[b * (m + 1) + i] = make_double2(i == kc ? beta_s : 0.0, 0.0);
            g.len[b] = m;
            g.ended[b] = 0;
        }
        g.counter[b] = 0;
    }
    if (kc > 0) {
        __syncthreads();
        if (st_sh != ST_ACTIVE) return;
        const double* d = g.dU + ((long long)cb.pair * gridDim.y + b) * g.kr;
        for (int idx = threadIdx.x; idx < kc * (m + 1); idx += blockDim.x) {
            const int col = idx / (m + 1), row = idx % (m + 1);
            g.H[((long long)b * m + col) * (m + 1) + row] = make_double2(row == col ? d[col] : 0.0, 0.0);
        }
        for (int t = threadIdx.x; t < kc; t += blockDim.x) {
            g.sigma[b * (m + 1) + t] = 1.0;
            g.gc[(long long)b * m + t] = 1.0;
            g.gs[(long long)b * m + t] = make_double2(0.0, 0.0);
        }
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

// Arithmetic of the basis passes per storage type. bfloat16 values (8-bit
// mantissa) are combined in fp32: their products, the orthogonalisation
// update and per-lane partial sums of at most a few dozen terms are far more
// precise than the stored values; every reduction across lanes, CTAs and
// chunks stays FP64. complex64 and complex128 bases use FP64 throughout.
// (Widening to FP64 costs conversion-unit throughput: with bfloat16 the FP64
// dots saturated that unit in the Arnoldi kernel.)
template <typename C2> struct MathT {
    using T = double;
    using T2 = double2;
};
template <> struct MathT<bf2> {
    using T = float;
    using T2 = float2;
};
__device__ __forceinline__ double2 to_d(double2 a);
__device__ __forceinline__ float2 to_f(bf2 a) { return bf2_to_f2(a); }

// Complex value c (0/1) of pair k of stage t % S (in the pass arithmetic).
template <typename C2>
__device__ __forceinline__ typename MathT<C2>::T2 staged(const uint4* stg, int t, int k, int c);
template <>
__device__ __forceinline__ double2 staged<float2>(const uint4* stg, int t, int k, int c) {
    using P = Pipe<float2>;
    const int s = t % P::S;
    const float4 v = reinterpret_cast<const float4*>(stg)[(s * P::UNITS + k) * kThreads + threadIdx.x];
    return c ? make_double2(v.z, v.w) : make_double2(v.x, v.y);
}
template <>
__device__ __forceinline__ float2 staged<bf2>(const uint4* stg, int t, int k, int c) {
    using P = Pipe<bf2>;
    const int s = t % P::S;
    const unsigned* v = reinterpret_cast<const unsigned*>(
        &stg[(s * P::UNITS + (k >> 1)) * kThreads + threadIdx.x]);
    const unsigned raw = v[2 * (k & 1) + c];
    return to_f(*reinterpret_cast<const bf2*>(&raw));
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
__device__ __forceinline__ void st_pair(bf2* p, float2 a, float2 b) {
    bf2 v[2] = {__float22bfloat162_rn(a), __float22bfloat162_rn(b)};
    *reinterpret_cast<uint2*>(p) = *reinterpret_cast<const uint2*>(v);
}
__device__ __forceinline__ void ld_pair(const bf2* p, float2& a, float2& b) {
    const uint2 raw = *reinterpret_cast<const uint2*>(p);
    a = to_f(*reinterpret_cast<const bf2*>(&raw.x));
    b = to_f(*reinterpret_cast<const bf2*>(&raw.y));
}
__device__ __forceinline__ float2 rounded(const bf2*, float2 a) { return to_f(__float22bfloat162_rn(a)); }
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
__device__ __forceinline__ void stream_basis(uint4* stg, const C2* base0, const C2* base1,
                                             int split, long long nv, int last, int len,
                                             bool prefetched, F&& f) {
    // vector t lives at (t < split ? base0 : base1) + t nv
    auto vec = [&](int t) { return (t < split ? base0 : base1) + (long long)t * nv; };
    if constexpr (Pipe<C2>::STAGED) {
        using P = Pipe<C2>;
        auto issue = [&](int t) { stage_vector<C2>(stg, vec(t <= last ? t : 0), t, last, len); };
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
                        ld_pair(vec(t0 + q) + e, v[q][k][0], v[q][k][1]);
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

template <typename Y, typename C2> __device__ __forceinline__ Y as_ys(C2 v) { return v; }
template <> __device__ __forceinline__ double2 as_ys<double2, float2>(float2 v) {
    return make_double2(v.x, v.y);
}

template <typename C2> struct LaneLoad;
template <> struct LaneLoad<bf2> {
    static constexpr int NL = 4;
    uint4 r;
    __device__ __forceinline__ void load(const bf2* p) { r = *reinterpret_cast<const uint4*>(p); }
    __device__ __forceinline__ void zero() { r = make_uint4(0u, 0u, 0u, 0u); }
    __device__ __forceinline__ float2 get(int i) const {
        const unsigned v = i == 0 ? r.x : i == 1 ? r.y : i == 2 ? r.z : r.w;
        return to_f(*reinterpret_cast<const bf2*>(&v));
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

// Last CTA of a dots launch: sum the per-CTA partials of t = 0..j (the dots)
// and t = j+1 (||w||^2) in a fixed order into Hessenberg column j (or the
// projection coefficients alpha) and wnorm.
__device__ __forceinline__ void dots_finish(GState& g, int b, int j, bool proj, int nparts) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = int(blockDim.x >> 5);
    for (int t = warp; t <= j + 1; t += nw) {
        double re0 = 0.0, im0 = 0.0;
        const double2* pt = g.partial + (long long)b * g.nblk * g.ps + t;
        for (int q0 = 0; q0 < nparts; q0 += 32 * 4) {
            double2 pv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = q0 + 32 * u + lane;
                pv[u] = q < nparts ? ld_cg(pt + (long long)q * g.ps) : make_double2(0.0, 0.0);
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
            if (t > j) g.wnorm[b] = sqrt(re0);
            else if (proj) g.alpha[(long long)b * g.kr + t] = make_double2(re0, im0);
            else g.H[((long long)b * g.m + j) * (g.m + 1) + t] = make_double2(re0, im0);
        }
    }
    if (threadIdx.x == 0) g.counter[b] = 0;
}

// Arnoldi step j, part 1: each CTA computes its chunk of w = sigma_j K u_j
// (stencil) into shared and global memory, then the dots <sigma_t u_t, w>,
// t <= j, and ||w||^2. (A separate stencil kernel ahead of a streaming dots
// kernel, plain or z-marching, measured 6-10% slower per iteration at 128^3:
// the extra launch and the re-read of w cost more than the overlap of the two
// phases gains. Streaming the dots per thread through the cp.async pipeline
// instead of warp tasks measured the same for bfloat16 and 8% slower for
// complex64. Two bulk-copy forms of the dots were measured at 128^3 and
// dropped: the chunk tiles of u_0 .. u_j through a cp.async.bulk ring with
// every warp owning 1/16 of the chunk, 15% slower (a warp reduction per tile
// and warp); each thread owning 8 nodes with its stencil in registers and
// shared-memory partial sums, 1.7x slower (the stencil loads of 8 nodes per
// thread at 25 warps per SM). Also measured at 128^3 (4 RHS) and dropped:
// one CTA per node chunk of all right-hand sides (row coefficients read once
// per batch: faster at small j, slower at large j, 9% more dots time); a
// bulk L2 prefetch of the next chunk's coefficient rows during the dots (5%
// slower); segment counts balancing the dot tasks' load batches over the
// warps (1% faster, but complex64 spilled).)
// mode 1 (recycled cycles): no stencil; the dots alpha_t = <C_t, r> of the
// cycle's first residual r (slot kc) with the recycled C_t, t < kc.
template <typename R, typename S, bool ADJ, int NT, bool MS = false>
__global__ void __launch_bounds__(NT, 2) k_dots(OpView<R> op, S* V, GState g, int j, Step step,
                                                int mode, int rows16) {
    using C2 = S;  // stored vector element
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || g.ended[b]) return;
    if constexpr (MS) {
        op = slot_view<R>(g.slots[b]);
        step = g.slots[b].step_d;
    }
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const CycleBasis<C2> cb = cycle_basis(V, g, b);
    const bool proj = mode == 1;
    if (proj) {
        if (cb.kc == 0) return;
        j = cb.kc - 1;
    } else if (j < cb.kc) {
        return;
    }
    // w of the chunk in shared memory, widened once for complex64 (FP64 dots)
    using YS = typename std::conditional<std::is_same<C2, float2>::value, double2, C2>::type;
    // bfloat16: two chunks per phase (half the barriers, twice the loads in
    // flight per phase)
    constexpr int DC = std::is_same<C2, bf2>::value ? 2 * kChunk : kChunk;
    // bfloat16: w of consecutive chunks alternates between two buffers, so a
    // warp done with the dots of chunk c starts the stencil of chunk c+1 while
    // others still read chunk c (one barrier per chunk, between the stencil
    // and the dots)
    constexpr int NBUF = std::is_same<C2, bf2>::value ? 2 : 1;
    __shared__ __align__(16) YS ys_buf[NBUF][DC];
    __shared__ double2 segsum[USV_MAX_RESTART + 2 > NT / 16 ? USV_MAX_RESTART + 2 : NT / 16];
    const long long N = op.n;
    const C2* uj = cb.V + (long long)j * g.nv;
    C2* w = cb.V + (long long)(j + 1) * g.nv;
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
    const int nphase = int((N + DC - 1) / DC);
    for (int ch = blockIdx.x, par = 0; ch < nphase; ch += ncta, par ^= NBUF - 1) {
        const long long n0 = (long long)ch * DC;
        const int len = int(min((long long)DC, N - n0));
        YS* ys = ys_buf[par];
        // single buffer: the previous chunk's dots are done with ys. Double
        // buffer: every warp passed the barrier below after its dots of the
        // chunk before the previous one, the last reader of this buffer.
        if (NBUF == 1) __syncthreads();
        if (mode == 0) {
            if constexpr (std::is_same<C2, bf2>::value) {
                (void)step;
                // bfloat16 vectors: rows without grid coordinates (the
                // coefficient of a missing neighbour is zero, so its load only
                // has to stay inside the vector: clamped index; 75 vs 84 us
                // per launch at j = 0, 128^3, 4 RHS), from the packed bfloat16
                // coefficients with bf16 x bf16 products (rows16: 24 B per node,
                // 4% less dots time and the same iteration count at 128^3) or
                // from the complex64 ones (48 B)
#pragma unroll 4
                for (int e = threadIdx.x; e < DC; e += NT) {
                    C2 y = from_d<C2>(make_double2(0.0, 0.0));
                    if (e < len) {
                        const long long n = n0 + e;
                        y = narrow<C2>(cscale(rows16 ? k_row_cb_clamped(op, uj, n)
                                                     : k_row_cf_clamped(op, uj, n), sj));
                        w[n] = y;
                    }
                    ys[e] = as_ys<YS>(y);
                }
            } else {
                Node p = decode(n0 + threadIdx.x, op.nx, op.ny);
                constexpr int kStencilUnroll = sizeof(R) == 4 ? 4 : 2;
#pragma unroll(kStencilUnroll)
                for (int e = threadIdx.x; e < DC; e += NT) {
                    C2 y = from_d<C2>(make_double2(0.0, 0.0));
                    if (e < len) {
                        const long long n = n0 + e;
                        y = narrow<C2>(cscale(k_row<R, ADJ, S>(op, uj, n, p), sj));
                        w[n] = y;
                    }
                    ys[e] = as_ys<YS>(y);
                    advance(p, step, op.nx, op.ny);
                }
            }
        } else {
            for (int e = threadIdx.x; e < DC; e += NT)
                ys[e] = as_ys<YS>(e < len ? w[n0 + e] : from_d<C2>(make_double2(0.0, 0.0)));
        }
        __syncthreads();
        constexpr int NL = LaneLoad<C2>::NL;
        const int ngroups = (len + NL - 1) / NL;  // ys and the vector padding are zero past len
        const int per_seg = (ngroups + segs - 1) / segs;
        for (int task = warp; task < tasks_t * segs; task += nw) {
            const int t = task / segs, seg = task % segs;
            const int q0 = seg * per_seg, q1 = min(ngroups, q0 + per_seg);
            // lane sums in the pass arithmetic (fp32 for bfloat16, <= 64 terms
            // per lane and chunk), FP64 from the warp reduction on
            using MT = typename MathT<C2>::T;
            using M2 = typename MathT<C2>::T2;
            MT lre = 0, lim = 0;
            if constexpr (std::is_same<C2, bf2>::value) {
                // bfloat16 x bfloat16 products straight from the packed words
                // (exact in fp32), four fp32 lane sums: Re = rr + ii, Im = ri - ir
                float rr = 0.f, ii = 0.f, ri = 0.f, ir = 0.f;
                const uint4* yw = reinterpret_cast<const uint4*>(ys);
                if (t <= j) {
                    const uint4* ut = reinterpret_cast<const uint4*>(
                        (t < cb.kc ? cb.C : cb.V) + (long long)t * g.nv + n0);
                    for (int qb = q0 + lane; qb < q1; qb += 32 * kDotUnroll) {
                        uint4 a[kDotUnroll];
#pragma unroll
                        for (int u = 0; u < kDotUnroll; ++u) {
                            const int q = qb + 32 * u;
                            a[u] = q < q1 ? ut[q] : make_uint4(0u, 0u, 0u, 0u);
                        }
#pragma unroll
                        for (int u = 0; u < kDotUnroll; ++u) {
                            const uint4 y = yw[min(qb + 32 * u, ngroups - 1)];
                            bf_mac(rr, ii, ri, ir, a[u].x, y.x);
                            bf_mac(rr, ii, ri, ir, a[u].y, y.y);
                            bf_mac(rr, ii, ri, ir, a[u].z, y.z);
                            bf_mac(rr, ii, ri, ir, a[u].w, y.w);
                        }
                    }
                } else {
                    for (int q = q0 + lane; q < q1; q += 32) {
                        const uint4 y = yw[q];
                        bf_sq(rr, ii, y.x);
                        bf_sq(rr, ii, y.y);
                        bf_sq(rr, ii, y.z);
                        bf_sq(rr, ii, y.w);
                    }
                }
                lre = rr + ii;
                lim = ri - ir;
            } else if (t <= j) {
                const C2* ut = (t < cb.kc ? cb.C : cb.V) + (long long)t * g.nv + n0;
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
                            const M2 y = widen<M2>(ys[NL * q + c]);
                            const M2 av = a[u].get(c);
                            lre = fma(av.x, y.x, fma(av.y, y.y, lre));
                            lim = fma(av.x, y.y, fma(-av.y, y.x, lim));
                        }
                    }
                }
            } else {
                for (int q = q0 + lane; q < q1; q += 32)
#pragma unroll
                    for (int c = 0; c < NL; ++c) lre += cabs2(widen<M2>(ys[NL * q + c]));
            }
            const double v = warp_sum_pair(double(lre), double(lim));
            if ((lane & 15) == 0) reinterpret_cast<double*>(&segsum[task])[lane >> 4] += v;
        }
    }
    __syncthreads();
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * g.ps;
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
    if (!last_block_done(&g.counter[b], ncta)) return;
    dots_finish(g, b, j, proj, ncta);
}

// d = a * b + c on two fp32 lanes at once (PTX fma.rn.f32x2, sm_100)
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;"
        : "=l"(d)
        : "l"(*reinterpret_cast<const unsigned long long*>(&a)),
          "l"(*reinterpret_cast<const unsigned long long*>(&b)),
          "l"(*reinterpret_cast<const unsigned long long*>(&c)));
    return *reinterpret_cast<const float2*>(&d);
}

// Last CTA of an orthogonalisation launch: beta = ||u_{j+1}|| from the
// per-CTA partials, then (proj) the start of the Krylov part of a recycled
// cycle, or the Givens update of Hessenberg column j, the raw column for the
// harmonic Ritz step and the end-of-cycle flag.
template <typename C2>
__device__ __forceinline__ void orth_finish(GState& g, int b, const CycleBasis<C2>& cb, int j, int proj,
                                         double* sh, double2* hs, double2* gsS, double* gcS, int nparts) {
    const int m = g.m;
    const double beta = sqrt(reduce_slot0(g, b, sh, nparts));
    if (proj) {
        if (threadIdx.x == 0) {
            g.counter[b] = 0;
            const int kc = cb.kc;
            if (beta > 1e-300 && isfinite(beta)) {
                g.g[b * (m + 1) + kc] = make_double2(beta, 0.0);
                g.sigma[b * (m + 1) + kc] = 1.0 / beta;
            } else {  // r lies in span(C): the projection alone solves this cycle
                g.g[b * (m + 1) + kc] = make_double2(0.0, 0.0);
                g.len[b] = kc;
                g.ended[b] = 1;
            }
        }
        return;
    }
    // stage column j and the previous rotations in shared memory
    double2* col = g.H + ((long long)b * m + j) * (m + 1);
    for (int t = threadIdx.x; t <= j; t += blockDim.x) {
        hs[t] = col[t];
        if (t < j) {
            gcS[t] = g.gc[(long long)b * m + t];
            gsS[t] = g.gs[(long long)b * m + t];
        }
    }
    __syncthreads();
    if (g.kr > 0) {  // raw column of G (before the rotations) for the harmonic Ritz step
        double* gr = g.hb + (long long)b * g.hb_len + hb_graw(m) + 2LL * j * (m + 1);
        for (int t = threadIdx.x; t <= j + 1; t += blockDim.x) {
            const double2 v = t <= j ? hs[t] : make_double2(beta, 0.0);
            gr[2 * t] = v.x;
            gr[2 * t + 1] = v.y;
        }
    }
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
    for (int t = threadIdx.x; t <= j; t += blockDim.x) col[t] = hs[t];
    if (threadIdx.x == 0) {
        g.gc[(long long)b * m + j] = gcS[j];
        g.gs[(long long)b * m + j] = gsS[j];
    }
}

// ------------------------------------------------------------ Arnoldi: orthogonalise + norm
// proj = 1 (recycled cycles): r -= sum_t alpha_t C_t on the cycle's first
// residual (slot kc), then beta = ||r|| starts the Krylov part of the cycle.
template <typename S, bool MS = false>
__global__ void __launch_bounds__(kThreads) k_orth(S* V, long long N, GState g, int j, int proj) {
    using C2 = S;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || g.ended[b]) return;
    int nchunk = g.nchunk;
    if constexpr (MS) {
        N = g.slots[b].n;
        nchunk = g.slots[b].nchunk;
    }
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const CycleBasis<C2> cb = cycle_basis(V, g, b);
    if (proj) {
        if (cb.kc == 0) return;
        j = cb.kc - 1;
    } else if (j < cb.kc) {
        return;
    }
    extern __shared__ __align__(16) uint4 stg[];
    __shared__ double2 hs[USV_MAX_RESTART + 2];
    __shared__ double2 gsS[USV_MAX_RESTART + 1];
    __shared__ double gcS[USV_MAX_RESTART + 1];
    __shared__ double sh[32];
    using M2 = typename MathT<C2>::T2;
    __shared__ M2 hm[USV_MAX_RESTART + 2];
    const int m = g.m;
    for (int t = threadIdx.x; t <= j; t += kThreads) {
        hs[t] = proj ? g.alpha[(long long)b * g.kr + t]
                     : cscale(g.H[((long long)b * m + j) * (m + 1) + t], g.sigma[b * (m + 1) + t]);
        hm[t] = cmake<M2>(hs[t].x, hs[t].y);
    }
    __syncthreads();  // hs, hm visible
    double acc = 0.0;
    for (int ch = blockIdx.x; ch < nchunk; ch += ncta) {
        const long long n0 = (long long)ch * kChunk;
        const int len = int(min((long long)kChunk, N - n0));
        C2* w = cb.V + (long long)(j + 1) * g.nv + n0;
        M2 u[kPairs][2];
#pragma unroll
        for (int k = 0; k < kPairs; ++k) {
            const int e = pair_node<C2>(k);
            if (e < len) ld_pair(w + e, u[k][0], u[k][1]);
            else u[k][0] = u[k][1] = cmake<M2>(0.0, 0.0);
        }
        if constexpr (std::is_same<C2, bf2>::value) {
            // packed fp32x2 FMAs: u = (re, im) -= h.re (v.re, v.im) and a second
            // pair q += h.im (-v.re, v.im) holding (Im, Re) terms, so neither
            // needs the swapped pair (v.im, v.re): two FMAs per complex product
            float2 q[kPairs][2];
#pragma unroll
            for (int k = 0; k < kPairs; ++k) q[k][0] = q[k][1] = make_float2(0.f, 0.f);
            stream_basis<C2>(stg, cb.C + n0, cb.V + n0, cb.kc, g.nv, j, len, false,
                             [&](int t, int k, int c, M2 vv) {
                const M2 h = hm[t];
                u[k][c] = ffma2(vv, make_float2(-h.x, -h.x), u[k][c]);
                q[k][c] = ffma2(vv, make_float2(-h.y, h.y), q[k][c]);
            });
#pragma unroll
            for (int k = 0; k < kPairs; ++k)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    u[k][c].x += q[k][c].y;
                    u[k][c].y += q[k][c].x;
                }
        } else {
            stream_basis<C2>(stg, cb.C + n0, cb.V + n0, cb.kc, g.nv, j, len, false,
                             [&](int t, int k, int c, M2 vv) {
                const M2 h = hm[t];
                u[k][c].x -= h.x * vv.x - h.y * vv.y;
                u[k][c].y -= h.x * vv.y + h.y * vv.x;
            });
        }
#pragma unroll
        for (int k = 0; k < kPairs; ++k) {
            const int e = pair_node<C2>(k);
            if (e < len) {
                st_pair(w + e, u[k][0], u[k][1]);
                acc += double(cabs2(rounded(w, u[k][0])));
                if (e + 1 < len) acc += double(cabs2(rounded(w, u[k][1])));
            }
        }
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0)
        g.partial[((long long)b * g.nblk + blockIdx.x) * g.ps] = make_double2(acc, 0.0);
    if (!last_block_done(&g.counter[b], ncta)) return;
    orth_finish<C2>(g, b, cb, j, proj, sh, hs, gsS, gcS, ncta);
}

// Bulk-copy form of k_orth: the basis tiles reach shared memory by
// cp.async.bulk (one instruction per chunk tile instead of a 16-byte cp.async
// per thread and unit), issued by one producer thread kOrthStages - 1 tiles
// ahead through a ring of full / empty mbarriers; 256 consumer threads keep
// the node mapping and arithmetic of k_orth. Per chunk the tiles are w (slot
// j+1) then u_0 .. u_j. Every wait is bounded: when one runs out the RHS ends
// with ST_DEVICE_TIMEOUT, the producer waits (bounded) for the copies it has
// in flight, and the CTA leaves.
template <typename S> struct OrthBulk {
    static constexpr int TILE = kChunk * int(sizeof(S));   // bytes per chunk tile
    // stages: a power of two (ring index and phase by mask and shift)
    static constexpr int LOG_STAGES = 2;
    static constexpr int STAGES = 1 << LOG_STAGES;
    static constexpr size_t SMEM = size_t(STAGES) * TILE + 2 * STAGES * sizeof(unsigned long long);
    static constexpr int THREADS = kThreads + 32;           // + the producer warp
};

// values of this thread's pairs from a chunk tile (MASK: nodes >= len read as
// zero; only the last, partial chunk of a vector needs it)
template <typename C2, bool MASK, typename M2>
__device__ __forceinline__ void tile_pairs(const char* tile, int len, M2 (&v)[kPairs][2]) {
    if constexpr (std::is_same<C2, bf2>::value) {
#pragma unroll
        for (int u = 0; u < kPairs / 2; ++u) {
            const int e = 4 * (threadIdx.x + kThreads * u);
            const uint4 raw = reinterpret_cast<const uint4*>(tile)[threadIdx.x + kThreads * u];
            const unsigned w4[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
            for (int c = 0; c < 4; ++c)
                v[2 * u + c / 2][c % 2] = !MASK || e + c < len
                                              ? to_f(*reinterpret_cast<const bf2*>(&w4[c]))
                                              : cmake<M2>(0.0, 0.0);
        }
    } else if constexpr (std::is_same<C2, float2>::value) {
#pragma unroll
        for (int k = 0; k < kPairs; ++k) {
            const int e = pair_node<C2>(k);
            const float4 r = reinterpret_cast<const float4*>(tile)[threadIdx.x + kThreads * k];
            v[k][0] = !MASK || e < len ? make_double2(r.x, r.y) : make_double2(0.0, 0.0);
            v[k][1] = !MASK || e + 1 < len ? make_double2(r.z, r.w) : make_double2(0.0, 0.0);
        }
    } else {
#pragma unroll
        for (int k = 0; k < kPairs; ++k) {
            const int e = pair_node<C2>(k);
            const double2* d = reinterpret_cast<const double2*>(tile) + e;
            v[k][0] = !MASK || e < len ? d[0] : make_double2(0.0, 0.0);
            v[k][1] = !MASK || e + 1 < len ? d[1] : make_double2(0.0, 0.0);
        }
    }
}

template <typename S, bool MS = false>
__global__ void __launch_bounds__(OrthBulk<S>::THREADS) k_orth_bulk(S* V, long long N, GState g,
                                                                   int j, int proj) {
    using C2 = S;
    using P = OrthBulk<S>;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || g.ended[b]) return;
    int nchunk = g.nchunk;
    if constexpr (MS) {
        N = g.slots[b].n;
        nchunk = g.slots[b].nchunk;
    }
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const CycleBasis<C2> cb = cycle_basis(V, g, b);
    if (proj) {
        if (cb.kc == 0) return;
        j = cb.kc - 1;
    } else if (j < cb.kc) {
        return;
    }
    extern __shared__ __align__(128) char ring[];
    unsigned long long* full = reinterpret_cast<unsigned long long*>(ring + size_t(P::STAGES) * P::TILE);
    unsigned long long* empty = full + P::STAGES;
    __shared__ double2 hs[USV_MAX_RESTART + 2];
    __shared__ double2 gsS[USV_MAX_RESTART + 1];
    __shared__ double gcS[USV_MAX_RESTART + 1];
    __shared__ double sh[32];
    __shared__ int failed;
    using M2 = typename MathT<C2>::T2;
    __shared__ M2 hm[USV_MAX_RESTART + 2];
    const int m = g.m;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = threadIdx.x; t <= j; t += blockDim.x) {
        hs[t] = proj ? g.alpha[(long long)b * g.kr + t]
                     : cscale(g.H[((long long)b * m + j) * (m + 1) + t], g.sigma[b * (m + 1) + t]);
        hm[t] = cmake<M2>(hs[t].x, hs[t].y);
    }
    if (threadIdx.x == 0) {
        failed = 0;
        for (int s = 0; s < P::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kThreads / 32);
        }
        mbar_fence_init();
    }
    __syncthreads();  // hs, hm, barriers visible
    const int tpc = j + 2;  // tiles per chunk: w, u_0 .. u_j
    const int nmy = nchunk > int(blockIdx.x) ? int((nchunk - blockIdx.x + ncta - 1) / ncta) : 0;
    double acc = 0.0;
    if (warp == kThreads / 32) {
        // producer: one elected thread issues every tile of this CTA in order
        if (lane == 0) {
            int q = 0;
            bool ok = true;
            for (int i = 0; i < nmy && ok; ++i) {
                const long long n0 = (long long)(blockIdx.x + (long long)i * ncta) * kChunk;
                const int len = int(min((long long)kChunk, N - n0));
                const unsigned bytes = unsigned((size_t(len) * sizeof(C2) + 15) / 16 * 16);
                for (int tt = 0; tt < tpc; ++tt, ++q) {
                    const int s = q & (P::STAGES - 1);
                    if (!mbar_wait(&empty[s], (unsigned(q >> P::LOG_STAGES) & 1u) ^ 1u)) {
                        ok = false;
                        break;
                    }
                    const C2* src = tt == 0 ? cb.V + (long long)(j + 1) * g.nv + n0
                                            : (tt - 1 < cb.kc ? cb.C : cb.V) +
                                                  (long long)(tt - 1) * g.nv + n0;
                    mbar_expect_tx(&full[s], bytes);
                    bulk_g2s(ring + size_t(s) * P::TILE, src, bytes, &full[s]);
                }
            }
            if (!ok) {
                failed = 1;
                g.status[b] = ST_DEVICE_TIMEOUT;
            }
            // copies still in flight (none unless a wait ran out): the last
            // tile issued on each stage must land before the CTA leaves
            for (int r = q > P::STAGES ? q - P::STAGES : 0; r < q; ++r)
                mbar_wait(&full[r & (P::STAGES - 1)], unsigned(r >> P::LOG_STAGES) & 1u);
        }
    } else {
        int q = 0;
        for (int i = 0; i < nmy; ++i) {
            const long long n0 = (long long)(blockIdx.x + (long long)i * ncta) * kChunk;
            const int len = int(min((long long)kChunk, N - n0));
            M2 u[kPairs][2];
            bool ok = true;
            // Tail of a partial last chunk: complex64 / bfloat16 pairs that start
            // before len lie in the copied bytes (rounded up into the zeroed
            // padding), later ones are neither stored nor summed, so only
            // complex128 (a node per 16 bytes) masks the values it reads.
            constexpr bool MASK = std::is_same<C2, double2>::value;
            for (int tt = 0; tt < tpc; ++tt, ++q) {
                const int s = q & (P::STAGES - 1);
                if (!mbar_wait(&full[s], unsigned(q >> P::LOG_STAGES) & 1u)) {
                    ok = false;
                    break;
                }
                if constexpr (std::is_same<C2, bf2>::value) {
                    // packed words straight from the tile; u -= h v as two
                    // fp32x2 FMAs per value: (v.re, v.im) (-h.re, -h.re) and
                    // the swapped pair (v.im, v.re) (h.im, -h.im), both pairs
                    // widened from the word by a shift and a mask
                    uint4 raw[kPairs / 2];
#pragma unroll
                    for (int w4 = 0; w4 < kPairs / 2; ++w4)
                        raw[w4] = reinterpret_cast<const uint4*>(ring + size_t(s) * P::TILE)
                            [threadIdx.x + kThreads * w4];
                    const M2 h = tt > 0 ? hm[tt - 1] : cmake<M2>(0.0, 0.0);
                    const float2 hre = make_float2(-h.x, -h.x), him = make_float2(h.y, -h.y);
#pragma unroll
                    for (int w4 = 0; w4 < kPairs / 2; ++w4) {
                        const unsigned wd[4] = {raw[w4].x, raw[w4].y, raw[w4].z, raw[w4].w};
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const float lo = __uint_as_float(wd[c] << 16);
                            const float hi = __uint_as_float(wd[c] & 0xffff0000u);
                            M2& acc2 = u[2 * w4 + c / 2][c % 2];
                            if (tt == 0) {
                                acc2 = make_float2(lo, hi);
                            } else {
                                acc2 = ffma2(make_float2(lo, hi), hre, acc2);
                                acc2 = ffma2(make_float2(hi, lo), him, acc2);
                            }
                        }
                    }
                } else {
                    M2 v[kPairs][2];
                    tile_pairs<C2, MASK>(ring + size_t(s) * P::TILE, len, v);
                    if (tt == 0) {
#pragma unroll
                        for (int k = 0; k < kPairs; ++k) u[k][0] = v[k][0], u[k][1] = v[k][1];
                    } else {
                        const M2 h = hm[tt - 1];
#pragma unroll
                        for (int k = 0; k < kPairs; ++k)
#pragma unroll
                            for (int c = 0; c < 2; ++c) {
                                u[k][c].x -= h.x * v[k][c].x - h.y * v[k][c].y;
                                u[k][c].y -= h.x * v[k][c].y + h.y * v[k][c].x;
                            }
                    }
                }
                // the stage is released only after its values have been used
                // (their loads have completed), so the producer's next copy
                // into it cannot overtake a read of this warp
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);
            }
            if (!ok) {
                failed = 1;
                g.status[b] = ST_DEVICE_TIMEOUT;
                break;
            }
            C2* w = cb.V + (long long)(j + 1) * g.nv + n0;
#pragma unroll
            for (int k = 0; k < kPairs; ++k) {
                const int e = pair_node<C2>(k);
                if (e < len) {
                    st_pair(w + e, u[k][0], u[k][1]);
                    acc += double(cabs2(rounded(w, u[k][0])));
                    if (e + 1 < len) acc += double(cabs2(rounded(w, u[k][1])));
                }
            }
        }
    }
    acc = block_sum(acc, sh);
    if (failed) return;
    if (threadIdx.x == 0)
        g.partial[((long long)b * g.nblk + blockIdx.x) * g.ps] = make_double2(acc, 0.0);
    if (!last_block_done(&g.counter[b], ncta)) return;
    orth_finish<C2>(g, b, cb, j, proj, sh, hs, gsS, gcS, ncta);
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
    if (g.kr == 0) {
        for (int i = threadIdx.x; i < L; i += blockDim.x)
            g.y[(long long)b * m + i] = cscale(gv[i], g.sigma[b * (m + 1) + i]);
        return;
    }
    // Recycled cycle: y_t (t < kc) multiplies Ut_t = d_t U_t, and the
    // projection x += U alpha of the cycle's first residual is folded in.
    const int* cw = g.ctl + b * kCtl;
    const int kc = cw[CW_KC], pair = cw[CW_PAIR] > 0 ? cw[CW_PAIR] : 0;
    const double* d = g.dU + ((long long)pair * gridDim.x + b) * g.kr;
    for (int i = threadIdx.x; i < L; i += blockDim.x)
        g.y[(long long)b * m + i] =
            i < kc ? cadd(cscale(gv[i], d[i]), g.alpha[(long long)b * g.kr + i])
                   : cscale(gv[i], g.sigma[b * (m + 1) + i]);
    double* hb = g.hb + (long long)b * g.hb_len;
    for (int i = threadIdx.x; i <= m; i += blockDim.x) hb[hb_sigma(m, g.kr) + i] = g.sigma[b * (m + 1) + i];
    for (int i = threadIdx.x; i < g.kr; i += blockDim.x) hb[hb_d(m, g.kr) + i] = i < kc ? d[i] : 0.0;
    if (threadIdx.x == 0) {
        hb[hb_tail(m, g.kr)] = double(L);
        hb[hb_tail(m, g.kr) + 1] = double(kc);
        g.klast[b] = kc;
    }
}

// ------------------------------------------------------------ solution update
template <typename S, bool MS = false>
__global__ void __launch_bounds__(kThreads) k_update(OpView<double> op, const S* V, double2* x,
                                                     long long ld, GState g) {
    using C2 = S;
    using P = Pipe<C2>;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || !g.ended[b]) return;
    int nchunk = g.nchunk;
    if constexpr (MS) {
        op = g.slots[b].op64;
        nchunk = g.slots[b].nchunk;
    }
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    extern __shared__ __align__(16) uint4 stg[];
    __shared__ double2 ys[USV_MAX_RESTART];
    __shared__ float2 yf[USV_MAX_RESTART];
    const int L = g.len[b];
    for (int t = threadIdx.x; t < L; t += kThreads) {
        ys[t] = g.y[(long long)b * g.m + t];
        yf[t] = make_float2(float(ys[t].x), float(ys[t].y));
    }
    const long long N = op.n;
    // solution vectors: U_t (t < kc) of the cycle's pair, then Krylov slots
    const CycleBasis<C2> cb = cycle_basis(const_cast<C2*>(V), g, b);
    __syncthreads();  // ys visible
    for (int ch = blockIdx.x; ch < nchunk; ch += ncta) {
        const long long n0 = (long long)ch * kChunk;
        const int len = int(min((long long)kChunk, N - n0));
        double2 acc[kPairs][2];
#pragma unroll
        for (int k = 0; k < kPairs; ++k) acc[k][0] = acc[k][1] = make_double2(0.0, 0.0);
        if constexpr (std::is_same<C2, bf2>::value) {
            // bfloat16: the correction W y in fp32 (packed fp32x2 FMAs, like
            // k_orth; widening every basis value to FP64 would load the
            // conversion unit), added to the FP64 solution below
            float2 pa[kPairs][2], pb[kPairs][2];
#pragma unroll
            for (int k = 0; k < kPairs; ++k)
                pa[k][0] = pa[k][1] = pb[k][0] = pb[k][1] = make_float2(0.f, 0.f);
            stream_basis<C2>(stg, cb.U + n0, cb.V + n0, cb.kc, g.nv, L - 1, len, false,
                             [&](int t, int k, int c, float2 vv) {
                const float2 y = yf[t];
                pa[k][c] = ffma2(vv, make_float2(y.x, y.x), pa[k][c]);
                pb[k][c] = ffma2(vv, make_float2(y.y, -y.y), pb[k][c]);  // (y.im v.re, -y.im v.im)
            });
#pragma unroll
            for (int k = 0; k < kPairs; ++k)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    acc[k][c] = make_double2(double(pa[k][c].x) + double(pb[k][c].y),
                                             double(pa[k][c].y) + double(pb[k][c].x));
        } else {
            stream_basis<C2>(stg, cb.U + n0, cb.V + n0, cb.kc, g.nv, L - 1, len, false,
                             [&](int t, int k, int c, typename MathT<C2>::T2 vv) {
                acc[k][c] = cadd(acc[k][c], cmul(ys[t], make_double2(vv.x, vv.y)));
            });
        }
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

// ------------------------------------------------------------ recycled space (GCRO-DR)
constexpr int kMaxRecycle = 16;
constexpr int kBdTile = 512;  // nodes of U staged in shared memory per pass

template <typename S> struct Wide { using T = float2; };
template <> struct Wide<double2> { using T = double2; };

// bd[s][i] = <Vhat_s, Ut_i>, s <= m, i < kc: Vhat = [C_0..C_kc-1, sigma_s V_s],
// Ut_i = d_i U_i (the columns of Vhat^H W that are not identity), written to
// the host-read block. Each CTA stages a tile of U in shared memory; warp w
// owns the slots s = w (mod warps) for every tile, so the per-CTA sums are
// accumulated in a fixed order; the last CTA reduces the CTA partials.
template <typename S, int K, bool MS = false>
__global__ void __launch_bounds__(kThreads) k_bdots(S* V, long long N, GState g) {
    using T = typename Wide<S>::T;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || !g.ended[b]) return;
    int nchunk = g.nchunk;
    if constexpr (MS) {
        N = g.slots[b].n;
        nchunk = g.slots[b].nchunk;
    }
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const CycleBasis<S> cb = cycle_basis(V, g, b);
    const int m = g.m;
    if (cb.kc != K) return;  // recycled cycles use all K vectors
    if (!g.ctl[b * kCtl + CW_HARVEST]) return;
    constexpr int kc = K;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* ut = reinterpret_cast<T*>(smem_raw);                                  // [kc][kBdTile]
    double2* tab = reinterpret_cast<double2*>(ut + (size_t)kc * kBdTile);    // [m+1][kc]
    for (int q = threadIdx.x; q < (m + 1) * kc; q += kThreads) tab[q] = make_double2(0.0, 0.0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nw = kThreads / 32;
    for (int ch = blockIdx.x; ch < nchunk; ch += ncta) {
        for (int t0 = 0; t0 < kChunk; t0 += kBdTile) {
            const long long n0 = (long long)ch * kChunk + t0;
            const int len = int(max(0LL, min((long long)kBdTile, N - n0)));
            __syncthreads();
            for (int q = threadIdx.x; q < kc * kBdTile; q += kThreads) {
                const int i = q / kBdTile, e = q % kBdTile;
                ut[q] = e < len ? widen<T>(cb.U[(long long)i * g.nv + n0 + e]) : cmake<T>(0.0, 0.0);
            }
            __syncthreads();
            for (int sl = warp; sl <= m; sl += nw) {
                const S* vs = (sl < kc ? cb.C : cb.V) + (long long)sl * g.nv + n0;
                T acc[K];
#pragma unroll
                for (int i = 0; i < K; ++i) acc[i] = cmake<T>(0.0, 0.0);
#pragma unroll 2
                for (int e = lane; e < len; e += 32) {
                    const T v = widen<T>(vs[e]);
#pragma unroll
                    for (int i = 0; i < K; ++i) {
                        const T u = ut[i * kBdTile + e];
                        acc[i].x += v.x * u.x + v.y * u.y;
                        acc[i].y += v.x * u.y - v.y * u.x;
                    }
                }
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    const double re = warp_sum(double(acc[i].x));
                    const double im = warp_sum(double(acc[i].y));
                    if (lane == 0) tab[sl * kc + i] = cadd(tab[sl * kc + i], make_double2(re, im));
                }
            }
        }
    }
    __syncthreads();
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * g.ps;
    for (int q = threadIdx.x; q < (m + 1) * kc; q += kThreads) part[q] = tab[q];
    if (!last_block_done(&g.counter[b], ncta)) return;
    const double* d = g.dU + ((long long)cb.pair * gridDim.y + b) * g.kr;
    double* out = g.hb + (long long)b * g.hb_len + hb_bd(m);
    for (int q = threadIdx.x; q < (m + 1) * kc; q += kThreads) {
        double re = 0.0, im = 0.0;
        const double2* pq = g.partial + (long long)b * g.nblk * g.ps + q;
        for (int c = 0; c < ncta; ++c) {
            const double2 v = ld_cg(pq + (long long)c * g.ps);
            re += v.x;
            im += v.y;
        }
        const int sl = q / kc, i = q % kc;
        const double sc = (sl < kc ? 1.0 : g.sigma[b * (m + 1) + sl]) * d[i];
        out[2 * (sl + (m + 1) * i)] = re * sc;
        out[2 * (sl + (m + 1) * i) + 1] = im * sc;
    }
    if (threadIdx.x == 0) g.counter[b] = 0;
}

// New recycled pair at the start of a cycle (when CW_COMBINE is set), from the
// data of an earlier cycle: U' = [Ut, V_p] P R^{-1}, C' = [C, V_{p+1}] Q with
// the coefficients (sigma, d folded in) from the host's harmonic Ritz step.
// Inputs: the source pair U_0..U_{kc-1}, C_0..C_{kc-1} and the source Krylov
// slots kc..m; coefficient rows in that order, columns U'_0..U'_{k-1},
// C'_0..C'_{k-1}. Outputs go to a third pair buffer (no aliasing). Also
// d'_i = 1/||U'_i|| for the new pair. One pass over the inputs: every thread
// keeps the 2K outputs of kNpt nodes (coalesced, kThreads apart) in
// registers; the shared coefficient row is read once per kNpt nodes.
template <typename S> constexpr int kCombineNpt = sizeof(S) == 16 ? 1 : 2;
template <typename S, int K, bool MS = false>
__global__ void __launch_bounds__(kThreads) k_combine(S* V, long long N, GState g) {
    using T = typename Wide<S>::T;
    constexpr int NPT = kCombineNpt<S>;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE) return;
    if constexpr (MS) N = g.slots[b].n;
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const int* cw = g.ctl + b * kCtl;
    if (!cw[CW_COMBINE]) return;
    const int m = g.m, skc = cw[CW_SRC_KC];
    const int rows = skc + m + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* cf = reinterpret_cast<T*>(smem_raw);  // [rows][2K]
    __shared__ double sh[32];
    for (int q = threadIdx.x; q < rows * 2 * K; q += kThreads) {
        const double2 c = g.coef[(long long)b * (K + m + 1) * 2 * K + q];
        cf[q] = cmake<T>(c.x, c.y);
    }
    const long long sp = (cw[CW_SRC_PAIR] > 0 ? cw[CW_SRC_PAIR] : 0) * g.pstride + (long long)b * K * g.nv;
    const long long dp = cw[CW_DST] * g.pstride + (long long)b * K * g.nv;
    const S* Uo = static_cast<const S*>(g.Ubuf) + sp;
    const S* Co = static_cast<const S*>(g.Cbuf) + sp;
    S* Un = static_cast<S*>(g.Ubuf) + dp;
    S* Cn = static_cast<S*>(g.Cbuf) + dp;
    const S* Vs = V + cw[CW_SRC_VBUF] * g.vstride + (long long)b * (m + 1) * g.nv;
    __syncthreads();
    double nrm[K];
#pragma unroll
    for (int i = 0; i < K; ++i) nrm[i] = 0.0;
    auto fma_row = [](T (&acc)[NPT][K], const T* crow, const T (&v)[NPT]) {
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const T c = crow[i];
#pragma unroll
            for (int q = 0; q < NPT; ++q) {
                acc[q][i].x += c.x * v[q].x - c.y * v[q].y;
                acc[q][i].y += c.x * v[q].y + c.y * v[q].x;
            }
        }
    };
    const long long step = (long long)ncta * kThreads * NPT;
    for (long long n0 = (long long)blockIdx.x * kThreads * NPT + threadIdx.x; n0 < N; n0 += step) {
        T au[NPT][K], ac[NPT][K];
#pragma unroll
        for (int q = 0; q < NPT; ++q)
#pragma unroll
            for (int i = 0; i < K; ++i) au[q][i] = ac[q][i] = cmake<T>(0.0, 0.0);
        auto load = [&](const S* src, T (&v)[NPT]) {
#pragma unroll
            for (int q = 0; q < NPT; ++q) {
                const long long n = n0 + (long long)q * kThreads;
                v[q] = n < N ? widen<T>(src[n]) : cmake<T>(0.0, 0.0);
            }
        };
        T v[NPT];
        for (int r = 0; r < skc; ++r) {  // U rows feed U' only
            load(Uo + (long long)r * g.nv, v);
            fma_row(au, cf + r * 2 * K, v);
        }
        for (int r = 0; r < skc; ++r) {  // C rows feed C' only
            load(Co + (long long)r * g.nv, v);
            fma_row(ac, cf + (skc + r) * 2 * K + K, v);
        }
        for (int sl = skc; sl <= m; ++sl) {  // Krylov slots feed both (slot m: C' only)
            load(Vs + (long long)sl * g.nv, v);
            const T* crow = cf + (skc + sl) * 2 * K;
            if (sl < m) fma_row(au, crow, v);
            fma_row(ac, crow + K, v);
        }
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            const long long n = n0 + (long long)q * kThreads;
            if (n < N) {
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    const S o = narrow<S>(au[q][i]);
                    Un[(long long)i * g.nv + n] = o;
                    Cn[(long long)i * g.nv + n] = narrow<S>(ac[q][i]);
                    nrm[i] += cabs2(to_d(o));
                }
            }
        }
    }
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * g.ps;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const double t = block_sum(nrm[i], sh);
        if (threadIdx.x == 0) part[i] = make_double2(t, 0.0);
    }
    if (!last_block_done(&g.counter[b], ncta)) return;
    for (int i = threadIdx.x; i < K; i += kThreads) {
        double t = 0.0;
        const double2* pq = g.partial + (long long)b * g.nblk * g.ps + i;
        for (int c = 0; c < ncta; ++c) t += ld_cg(pq + (long long)c * g.ps).x;
        g.dU[((long long)cw[CW_DST] * gridDim.y + b) * K + i] = t > 0.0 ? 1.0 / sqrt(t) : 0.0;
    }
    if (threadIdx.x == 0) g.counter[b] = 0;
}

// The same product for bfloat16 storage on the tensor cores (mma.sync
// m16n8k16, bf16 x bf16 -> fp32): out = In Coef with In = [U_old | C_old |
// Krylov slots] (nodes x rows) and the 2K complex outputs as real columns.
// A row of the product is a node; k runs over (input row, re/im), so a packed
// {re, im} word of an input vector is one k pair of A. Each complex
// coefficient c of output o gives four real columns: {Re, Im} of c v from the
// bfloat16 part hi(c) and from the remainder lo(c) = c - hi(c) (16
// significant bits of c); B fragments are built once per CTA in shared
// memory in fragment order. A warp owns 16-node blocks; lane (g, c) loads the
// words of nodes g and g+8 of input rows 8kb + c and 8kb + c + 4 and keeps
// the accumulators of all K n-tiles (two outputs each).
//   fragments: a = {A[g][2c..], A[g+8][2c..], A[g][2c+8..], A[g+8][2c+8..]},
//   b = {B[2c..][g], B[2c+8..][g]}, d = {D[g][2c], D[g][2c+1], D[g+8][2c], D[g+8][2c+1]}
__device__ __forceinline__ void mma_bf16(float (&d)[4], unsigned a0, unsigned a1, unsigned a2,
                                         unsigned a3, unsigned b0, unsigned b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ unsigned bf_pack(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return unsigned(__bfloat16_as_ushort(lo)) | (unsigned(__bfloat16_as_ushort(hi)) << 16);
}
constexpr int kCombineGroup = 6;  // k-blocks of 8 input rows loaded per batch
static size_t combine_mma_smem(int k, int m) {
    return sizeof(uint2) * size_t((k + m + 1 + 7) / 8) * k * 32;
}
template <int K, bool MS = false>
__global__ void __launch_bounds__(kThreads) k_combine_mma(bf2* V, long long N, GState g) {
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE) return;
    if constexpr (MS) N = g.slots[b].n;
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const int* cw = g.ctl + b * kCtl;
    if (!cw[CW_COMBINE]) return;
    const int m = g.m, skc = cw[CW_SRC_KC];
    const int rows = skc + m + 1, nkb = (rows + 7) / 8;
    extern __shared__ __align__(16) uint2 bfr[];  // [nkb][K][32]
    __shared__ double sh[kThreads / 32][2 * K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g8 = lane >> 2, c4 = lane & 3;
    const double2* coef = g.coef + (long long)b * (K + m + 1) * 2 * K;
    // B fragment word of input row r, real column col (output col/4, part col%4)
    auto bword = [&](int r, int col) -> unsigned {
        if (r >= rows) return 0u;
        const double2 c = coef[(long long)r * 2 * K + col / 4];
        const bool lo = (col & 2) != 0, im = (col & 1) != 0;
        __nv_bfloat16 cr = __double2bfloat16(c.x), ci = __double2bfloat16(c.y);
        if (lo) {
            cr = __double2bfloat16(c.x - double(__bfloat162float(cr)));
            ci = __double2bfloat16(c.y - double(__bfloat162float(ci)));
        }
        // Re(c v) = c.re v.re - c.im v.im ; Im(c v) = c.im v.re + c.re v.im
        return im ? bf_pack(ci, cr) : bf_pack(cr, __hneg(ci));
    };
    for (int q = threadIdx.x; q < nkb * K * 32; q += kThreads) {
        const int ln = q % 32, nt = (q / 32) % K, kb = q / (32 * K);
        const int gg = ln >> 2, cc = ln & 3, col = 8 * nt + gg;
        bfr[q] = make_uint2(bword(8 * kb + cc, col), bword(8 * kb + cc + 4, col));
    }
    const long long sp = (cw[CW_SRC_PAIR] > 0 ? cw[CW_SRC_PAIR] : 0) * g.pstride + (long long)b * K * g.nv;
    const long long dp = cw[CW_DST] * g.pstride + (long long)b * K * g.nv;
    const unsigned* Uo = reinterpret_cast<const unsigned*>(static_cast<const bf2*>(g.Ubuf) + sp);
    const unsigned* Co = reinterpret_cast<const unsigned*>(static_cast<const bf2*>(g.Cbuf) + sp);
    unsigned* Un = reinterpret_cast<unsigned*>(static_cast<bf2*>(g.Ubuf) + dp);
    unsigned* Cn = reinterpret_cast<unsigned*>(static_cast<bf2*>(g.Cbuf) + dp);
    const unsigned* Vs = reinterpret_cast<const unsigned*>(V + cw[CW_SRC_VBUF] * g.vstride +
                                                            (long long)b * (m + 1) * g.nv);
    // input row r (rows past the last read row 0 and are zeroed)
    auto row = [&](int r) {
        r = r < rows ? r : 0;
        return r < skc ? Uo + (long long)r * g.nv
                       : (r < 2 * skc ? Co + (long long)(r - skc) * g.nv : Vs + (long long)(r - skc) * g.nv);
    };
    __syncthreads();
    float nrm[K];
#pragma unroll
    for (int i = 0; i < K; ++i) nrm[i] = 0.f;
    const long long nblk16 = (N + 15) / 16;
    const long long wstride = (long long)ncta * (kThreads / 32);
    for (long long blk = (long long)blockIdx.x * (kThreads / 32) + warp; blk < nblk16; blk += wstride) {
        const long long n0 = blk * 16 + g8, n1 = n0 + 8;
        const long long l0 = n0 < N ? n0 : N - 1, l1 = n1 < N ? n1 : N - 1;
        float acc[K][4];
#pragma unroll
        for (int nt = 0; nt < K; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        // the A words of kCombineGroup k-blocks are loaded before their MMAs
        // (24 loads in flight per lane instead of 4)
        for (int kb0 = 0; kb0 < nkb; kb0 += kCombineGroup) {
            unsigned a[kCombineGroup][4];
#pragma unroll
            for (int u = 0; u < kCombineGroup; ++u) {
                const int ra = 8 * (kb0 + u) + c4, rb = ra + 4;
                const unsigned* pa = row(ra);
                const unsigned* pb = row(rb);
                a[u][0] = __ldg(pa + l0);
                a[u][1] = __ldg(pa + l1);
                a[u][2] = __ldg(pb + l0);
                a[u][3] = __ldg(pb + l1);
                if (ra >= rows) a[u][0] = a[u][1] = 0u;
                if (rb >= rows) a[u][2] = a[u][3] = 0u;
            }
#pragma unroll
            for (int u = 0; u < kCombineGroup; ++u) {
                if (kb0 + u >= nkb) break;
                const uint2* bq = bfr + (size_t)(kb0 + u) * K * 32 + lane;
#pragma unroll
                for (int nt = 0; nt < K; ++nt) {
                    const uint2 bb = bq[nt * 32];
                    mma_bf16(acc[nt], a[u][0], a[u][1], a[u][2], a[u][3], bb.x, bb.y);
                }
            }
        }
        // lanes c and c^1 hold the hi and lo parts of one output: add them;
        // lane (g, 0) then has output 2nt, lane (g, 2) output 2nt+1
#pragma unroll
        for (int nt = 0; nt < K; ++nt) {
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) v[e] = acc[nt][e] + __shfl_xor_sync(0xffffffffu, acc[nt][e], 1);
            if ((c4 & 1) == 0) {
                const int o = 2 * nt + (c4 >> 1);
                const bf2 w0 = __floats2bfloat162_rn(v[0], v[1]);
                const bf2 w1 = __floats2bfloat162_rn(v[2], v[3]);
                unsigned* dst = o < K ? Un + (long long)o * g.nv : Cn + (long long)(o - K) * g.nv;
                if (n0 < N) dst[n0] = *reinterpret_cast<const unsigned*>(&w0);
                if (n1 < N) dst[n1] = *reinterpret_cast<const unsigned*>(&w1);
                if (o < K) {
                    const float2 f0 = to_f(w0), f1 = to_f(w1);
                    float add = 0.f;
                    if (n0 < N) add += f0.x * f0.x + f0.y * f0.y;
                    if (n1 < N) add += f1.x * f1.x + f1.y * f1.y;
                    nrm[nt] += add;
                }
            }
        }
    }
    // ||U'_o||^2: lane (g, c) with c even holds output 2nt + c/2 in nrm[nt]
#pragma unroll
    for (int nt = 0; nt < K; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int o = 2 * nt + h;
            const double t = warp_sum((c4 & 1) == 0 && (c4 >> 1) == h ? double(nrm[nt]) : 0.0);
            if (lane == 0 && o < K) sh[warp][o] = t;
        }
    __syncthreads();
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * g.ps;
    for (int o = threadIdx.x; o < K; o += kThreads) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += sh[w][o];
        part[o] = make_double2(t, 0.0);
    }
    if (!last_block_done(&g.counter[b], ncta)) return;
    for (int i = threadIdx.x; i < K; i += kThreads) {
        double t = 0.0;
        const double2* pq = g.partial + (long long)b * g.nblk * g.ps + i;
        for (int c = 0; c < ncta; ++c) t += ld_cg(pq + (long long)c * g.ps).x;
        g.dU[((long long)cw[CW_DST] * gridDim.y + b) * K + i] = t > 0.0 ? 1.0 / sqrt(t) : 0.0;
    }
    if (threadIdx.x == 0) g.counter[b] = 0;
}

// The new recycled pair on the 5th-generation tensor cores (tcgen05.mma,
// kind::f16, bf16 x bf16 -> fp32 accumulators in tensor memory), for
// bfloat16 storage, K = 4 or 8 and at most kUmmaMaxRows input rows.
// The product is arranged so that the packed {re, im} words of the input
// vectors are an MN-major A operand as they lie in memory: a row of A is a
// (node, part) pair, part = re / im, so 64 nodes give the M = 128 rows of
// one MMA and a 16-byte piece of input vector r (4 nodes) is one row of a
// canonical 8 x 16-byte core matrix (k = input row r). B (K-major, built once
// per CTA) holds four real columns per complex output o: hi(c.re), lo(c.re),
// hi(c.im), lo(c.im) of c = coef[r][o] (bf16 high part + remainder: 16
// significant bits). Row (n, re) of D then holds sum_r v_r.re c_r, row (n, im)
// sum_r v_r.im c_r, and lane pairs of the epilogue form
//   out.re = P_re.re - P_im.im,  out.im = P_re.im + P_im.re.
// Pipeline per CTA (128 threads): input tiles (rows x 64 nodes, 256 B per
// row) reach shared memory by cp.async (16-byte pieces placed straight into
// the core-matrix layout) through a kUmmaStages ring; thread 0 issues the
// nks = ceil(rows / 16) MMAs of a tile into one of two TMEM accumulators and
// commits them to that accumulator's mbarrier; all four warps read the
// previous tile's accumulator (warp w: TMEM lanes 32w..32w+31), combine the
// lane pairs, store U'_o / C'_o and sum ||U'_o||^2 from the stored values.
// Every mbarrier wait is bounded; on a timeout the RHS ends with
// ST_DEVICE_TIMEOUT and the CTA still waits (bounded) for its MMAs and frees
// its tensor memory.
constexpr int kUmmaThreads = 128;
constexpr int kUmmaNodes = 64;      // nodes per tile: M = 128 rows (node, part)
constexpr int kUmmaStages = 4;
constexpr int kUmmaMaxRows = 64;    // input rows: at most 4 k-steps of 16
constexpr size_t kUmmaMinSmem = 56 * 1024;  // <= 4 CTAs per SM: <= 512 TMEM columns
__host__ __device__ constexpr int umma_tmem_cols(int k) { return 16 * k; }  // 2 x 8K, K = 4 or 8
static size_t combine_umma_smem(int k, int m) {
    const int nks = (k + m + 1 + 15) / 16;
    const size_t need = size_t(kUmmaStages) * nks * 4096 + size_t(nks) * 16 * 8 * k * 2;
    return need > kUmmaMinSmem ? need : kUmmaMinSmem;
}
template <int K, bool MS = false>
__global__ void __launch_bounds__(kUmmaThreads) k_combine_umma(bf2* V, long long N, GState g) {
    static_assert(K % 4 == 0 && K <= 8, "N = 8K columns: whole 32-column TMEM loads, <= 64");
    constexpr int NC = 8 * K;  // real columns of B / D
    constexpr int TC = umma_tmem_cols(K);
    constexpr int S = kUmmaStages;
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE) return;
    if constexpr (MS) N = g.slots[b].n;
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const int* cw = g.ctl + b * kCtl;
    if (!cw[CW_COMBINE]) return;
    const int m = g.m, skc = cw[CW_SRC_KC];
    const int rows = skc + m + 1;  // <= kUmmaMaxRows (host)
    const int nks = (rows + 15) / 16, nrg = (rows + 7) / 8;
    const unsigned stage_bytes = unsigned(nks) * 4096u;
    extern __shared__ __align__(128) unsigned char usm[];
    unsigned char* As = usm;                                  // [S][2 nks][16][128 B]
    unsigned char* Bs = usm + size_t(S) * stage_bytes;        // [2 nks][NC / 8][128 B]
    __shared__ __align__(8) unsigned long long mbar[2];
    __shared__ unsigned tmem_s;
    __shared__ double sh[kUmmaThreads / 32][K];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double2* coef = g.coef + (long long)b * (K + m + 1) * 2 * K;
    // A stages zeroed once (rows past `rows` stay zero), B built in its core layout:
    // element (k, n) at ((k / 8) (NC / 8) + n / 8) 128 + (n % 8) 16 + (k % 8) 2
    for (unsigned q = tid; q < unsigned(S) * stage_bytes / 16; q += kUmmaThreads)
        reinterpret_cast<uint4*>(As)[q] = make_uint4(0u, 0u, 0u, 0u);
    for (int q = tid; q < 16 * nks * NC; q += kUmmaThreads) {
        const int r = q / NC, col = q % NC, o = col >> 2, part = col & 3;
        __nv_bfloat16 v = __float2bfloat16(0.f);
        if (r < rows) {
            const double2 c = coef[(long long)r * 2 * K + o];
            const double x = part < 2 ? c.x : c.y;
            const __nv_bfloat16 hi = __double2bfloat16(x);
            v = (part & 1) ? __double2bfloat16(x - double(__bfloat162float(hi))) : hi;
        }
        *reinterpret_cast<__nv_bfloat16*>(Bs + (((r >> 3) * (NC / 8) + (col >> 3)) << 7) +
                                          ((col & 7) << 4) + ((r & 7) << 1)) = v;
    }
    if (warp == 0) tmem_alloc(&tmem_s, TC);
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_fence_init();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_s;

    const long long sp = (cw[CW_SRC_PAIR] > 0 ? cw[CW_SRC_PAIR] : 0) * g.pstride + (long long)b * K * g.nv;
    const long long dp = cw[CW_DST] * g.pstride + (long long)b * K * g.nv;
    const unsigned* Uo = reinterpret_cast<const unsigned*>(static_cast<const bf2*>(g.Ubuf) + sp);
    const unsigned* Co = reinterpret_cast<const unsigned*>(static_cast<const bf2*>(g.Cbuf) + sp);
    unsigned* Un = reinterpret_cast<unsigned*>(static_cast<bf2*>(g.Ubuf) + dp);
    unsigned* Cn = reinterpret_cast<unsigned*>(static_cast<bf2*>(g.Cbuf) + dp);
    const unsigned* Vs = reinterpret_cast<const unsigned*>(V + cw[CW_SRC_VBUF] * g.vstride +
                                                            (long long)b * (m + 1) * g.nv);
    auto row = [&](int r) {
        return r < skc ? Uo + (long long)r * g.nv
                       : (r < 2 * skc ? Co + (long long)(r - skc) * g.nv : Vs + (long long)(r - skc) * g.nv);
    };
    __shared__ const unsigned* rowp[kUmmaMaxRows];
    for (int r = tid; r < rows; r += kUmmaThreads) rowp[r] = row(r);
    __syncthreads();
    const long long ntile = (N + kUmmaNodes - 1) / kUmmaNodes;
    const int my_tiles =
        ntile > blockIdx.x ? int((ntile - 1 - blockIdx.x) / ncta + 1) : 0;
    // tile t of this CTA: nodes [(blockIdx.x + t ncta) 64, +64), inside the
    // zero-padded vectors (their length is a multiple of 64 nodes)
    auto issue = [&](int t) {
        if (t < my_tiles) {
            const long long n0 = ((long long)blockIdx.x + (long long)t * ncta) * kUmmaNodes;
            unsigned char* st = As + size_t(t % S) * stage_bytes;
            for (int c = tid; c < nrg * 128; c += kUmmaThreads) {
                const int r8 = c & 7, q = (c >> 3) & 15, rg = c >> 7, r = rg * 8 + r8;
                if (r < rows) cp_async16(st + ((rg * 16 + q) << 7) + (r8 << 4), rowp[r] + n0 + 4 * q, 16);
            }
        }
        cp_async_commit();
    };
    constexpr unsigned idesc = umma_idesc_bf16(128, NC, true, false);
    const unsigned b_addr = smem_u32(Bs);
    float nrm[K / 2];  // ||U'_o||^2 of this lane's outputs o = 2p + (lane & 1)
#pragma unroll
    for (int i = 0; i < K / 2; ++i) nrm[i] = 0.f;
    bool ok = true;
    int issued = 0;  // MMA groups committed (thread 0)
#pragma unroll 1
    for (int t = 0; t < S - 1; ++t) issue(t);
#pragma unroll 1
    for (int t = 0; t <= my_tiles; ++t) {
        if (t < my_tiles) {
            cp_async_wait<S - 2>();
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                const unsigned a_addr = smem_u32(As + size_t(t % S) * stage_bytes);
                const unsigned d = tmem + unsigned(t & 1) * NC;
                for (int ks = 0; ks < nks; ++ks)
                    umma_bf16(d, umma_desc(a_addr + ks * 4096u, 2048u, 128u),
                              umma_desc(b_addr + ks * 2u * NC * 16u, NC * 16u, 128u), idesc, ks > 0);
                umma_commit(&mbar[t & 1]);
                ++issued;
            }
        }
        if (t >= 1) {
            const int te = t - 1;
            if (ok && !mbar_wait(&mbar[te & 1], unsigned(te >> 1) & 1u)) ok = false;
            ok = __all_sync(0xffffffffu, ok);  // the TMEM loads below are warp-wide
            tc_fence_after();
            if (ok) {
                const long long n0 = ((long long)blockIdx.x + (long long)te * ncta) * kUmmaNodes;
                const long long node = n0 + 16 * warp + (lane >> 1);
                const bool odd = (lane & 1) != 0;
                const unsigned ta = tmem + (unsigned(32 * warp) << 16) + unsigned(te & 1) * NC;
#pragma unroll
                for (int h = 0; h < NC / 32; ++h) {
                    float v[32];
                    tmem_ld32(ta + 32u * h, v);
                    // output pair (oe, oe + 1): the even lane (re row) forms
                    // oe, the odd lane (im row) oe + 1; each sends its partner
                    // the row's products for the partner's output
#pragma unroll
                    for (int jp = 0; jp < 4; ++jp) {
                        const int oe = 8 * h + 2 * jp;
                        const float ae = v[8 * jp] + v[8 * jp + 1], ce = v[8 * jp + 2] + v[8 * jp + 3];
                        const float ao = v[8 * jp + 4] + v[8 * jp + 5], co = v[8 * jp + 6] + v[8 * jp + 7];
                        const float pa = __shfl_xor_sync(0xffffffffu, odd ? ae : ao, 1);
                        const float pc = __shfl_xor_sync(0xffffffffu, odd ? ce : co, 1);
                        const float a = odd ? ao : ae, c = odd ? co : ce;
                        const float re = odd ? pa - c : a - pc;
                        const float im = odd ? pc + a : c + pa;
                        if (node < N) {
                            const bf2 wv = __floats2bfloat162_rn(re, im);
                            unsigned* dst = (oe < K ? Un + (long long)oe * g.nv : Cn + (long long)(oe - K) * g.nv) +
                                            (odd ? g.nv : 0);
                            dst[node] = *reinterpret_cast<const unsigned*>(&wv);
                            if (oe < K) {
                                const float2 f = to_f(wv);
                                nrm[oe >> 1] += f.x * f.x + f.y * f.y;
                            }
                        }
                    }
                }
            }
            tc_fence_before();
        }
        issue(t + S - 1);
    }
    cp_async_wait<0>();
    if (!ok) {
        g.status[b] = ST_DEVICE_TIMEOUT;
        // MMAs still in flight must finish before their tensor memory is freed
        if (tid == 0)
            for (int r = issued > 2 ? issued - 2 : 0; r < issued; ++r)
                mbar_wait(&mbar[r & 1], unsigned(r >> 1) & 1u);
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, TC);
    // ||U'_o||^2 per CTA in a fixed order (lanes, then warps)
#pragma unroll
    for (int o = 0; o < K; ++o) {
        const double t = warp_sum((lane & 1) == (o & 1) ? double(nrm[o >> 1]) : 0.0);
        if (lane == 0) sh[warp][o] = t;
    }
    __syncthreads();
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * g.ps;
    for (int o = tid; o < K; o += kUmmaThreads) {
        double t = 0.0;
        for (int w = 0; w < kUmmaThreads / 32; ++w) t += sh[w][o];
        part[o] = make_double2(t, 0.0);
    }
    if (!last_block_done(&g.counter[b], ncta)) return;
    for (int i = tid; i < K; i += kUmmaThreads) {
        double t = 0.0;
        const double2* pq = g.partial + (long long)b * g.nblk * g.ps + i;
        for (int c = 0; c < ncta; ++c) t += ld_cg(pq + (long long)c * g.ps).x;
        g.dU[((long long)cw[CW_DST] * gridDim.y + b) * K + i] = t > 0.0 ? 1.0 / sqrt(t) : 0.0;
    }
    if (tid == 0) g.counter[b] = 0;
}

// bd = Vhat^H Ut for bfloat16 storage on the tensor cores: D = A B with A
// rows = the slots s <= m of Vhat (16 per row tile), k = (node, re/im), and
// B columns {re, im} -> Re, {im, -re} -> Im of <Vhat_s, U_i> (exact bf16
// words, no split). Lane (g, c) loads the 16-byte unit at node 16j + 4c of
// slots s0 + g and s0 + g + 8 and of U_i, i = 4nt + g/2, and feeds its four
// words to two products. Global warp w owns row tile w % RT and every
// (W / RT)-th 16-node block; fp32 sums are moved to FP64 every 16 blocks and
// the warps of a CTA are added in a fixed order.
static size_t bdots_mma_smem(int k, int m) {
    return sizeof(double2) * (size_t(kThreads / 32) * 16 + size_t(m + 1)) * k;
}
template <int K, bool MS = false>
__global__ void __launch_bounds__(kThreads) k_bdots_mma(bf2* V, long long N, GState g) {
    const int b = blockIdx.y;
    if (g.status[b] != ST_ACTIVE || !g.ended[b]) return;
    if constexpr (MS) N = g.slots[b].n;
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    const CycleBasis<bf2> cb = cycle_basis(V, g, b);
    const int m = g.m;
    if (cb.kc != K) return;  // recycled cycles use all K vectors
    if (!g.ctl[b * kCtl + CW_HARVEST]) return;
    constexpr int NT = (2 * K + 7) / 8;
    const int RT = (m + 16) / 16;  // row tiles of 16 slots covering 0..m
    extern __shared__ __align__(16) double2 wtab[];  // [warps][16][K], then the CTA's [m+1][K]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g8 = lane >> 2, c4 = lane & 3;
    constexpr int nw = kThreads / 32;

    const long long W = (long long)ncta * nw, wg = (long long)blockIdx.x * nw + warp;
    const int rt = int(wg % RT);
    const long long wstride = W / RT;
    const int sa = 16 * rt + g8, sb = sa + 8;
    auto slot_ptr = [&](int sl) {
        sl = sl <= m ? sl : 0;
        return reinterpret_cast<const uint4*>((sl < K ? cb.C : cb.V) + (long long)sl * g.nv);
    };
    const uint4* pa = slot_ptr(sa);
    const uint4* pb = slot_ptr(sb);
    const uint4* pu[NT];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
        const int i = 4 * nt + g8 / 2;
        pu[nt] = reinterpret_cast<const uint4*>(cb.U + (long long)(i < K ? i : 0) * g.nv);
    }
    double2 tot[NT][2];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) tot[nt][0] = tot[nt][1] = make_double2(0.0, 0.0);
    const long long nb16 = (N + 15) / 16, lastu = (N + 3) / 4 - 1;
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    if (wg < wstride * RT) {
        long long blk = wg / RT;
        while (blk < nb16) {
            float d[NT][4];
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.f;
            // two blocks of 16 nodes per batch: their 2 (2 + NT) 16-byte loads
            // are issued before the MMAs of either
            for (int r = 0; r < 16 && blk < nb16; r += 2) {
                uint4 va[2], vb[2], w[2][NT];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const long long bu = blk + u * wstride;
                    const long long uq = 4 * bu + c4;
                    const bool in = bu < nb16 && uq <= lastu;
                    const long long uc = uq < lastu ? uq : lastu;
                    va[u] = __ldg(pa + uc);
                    vb[u] = __ldg(pb + uc);
                    if (!(sa <= m && in)) va[u] = zero;
                    if (!(sb <= m && in)) vb[u] = zero;
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt) {
                        w[u][nt] = __ldg(pu[nt] + uc);
                        if (!(4 * nt + g8 / 2 < K && in)) w[u][nt] = zero;
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; ++u)
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt) {
                        uint4 ww = w[u][nt];
                        if (g8 & 1) {
                            ww.x = (ww.x >> 16) | ((ww.x << 16) ^ 0x80000000u);
                            ww.y = (ww.y >> 16) | ((ww.y << 16) ^ 0x80000000u);
                            ww.z = (ww.z >> 16) | ((ww.z << 16) ^ 0x80000000u);
                            ww.w = (ww.w >> 16) | ((ww.w << 16) ^ 0x80000000u);
                        }
                        mma_bf16(d[nt], va[u].x, vb[u].x, va[u].y, vb[u].y, ww.x, ww.y);
                        mma_bf16(d[nt], va[u].z, vb[u].z, va[u].w, vb[u].w, ww.z, ww.w);
                    }
                blk += 2 * wstride;
            }
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                tot[nt][0] = cadd(tot[nt][0], make_double2(d[nt][0], d[nt][1]));
                tot[nt][1] = cadd(tot[nt][1], make_double2(d[nt][2], d[nt][3]));
            }
        }
    }
    // lane (g, c): <slot sa|sb, U_{4nt+c}> in tot[nt][0|1]
    double2* mine = wtab + (size_t)warp * 16 * K;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
        const int i = 4 * nt + c4;
        if (i < K) {
            mine[g8 * K + i] = tot[nt][0];
            mine[(g8 + 8) * K + i] = tot[nt][1];
        }
    }
    __syncthreads();
    // CTA sums in warp order: slot sl comes from the warps whose row tile is sl/16
    double2* tab = wtab + (size_t)nw * 16 * K;
    for (int q = threadIdx.x; q < (m + 1) * K; q += kThreads) {
        const int sl = q / K, i = q % K;
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < nw; ++w)
            if (int(((long long)blockIdx.x * nw + w) % RT) == sl / 16)
                t = cadd(t, wtab[(size_t)w * 16 * K + (sl % 16) * K + i]);
        tab[q] = t;
    }
    __syncthreads();
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * g.ps;
    for (int q = threadIdx.x; q < (m + 1) * K; q += kThreads) part[q] = tab[q];
    if (!last_block_done(&g.counter[b], ncta)) return;
    const double* dd = g.dU + ((long long)cb.pair * gridDim.y + b) * g.kr;
    double* out = g.hb + (long long)b * g.hb_len + hb_bd(m);
    for (int q = threadIdx.x; q < (m + 1) * K; q += kThreads) {
        double re = 0.0, im = 0.0;
        const double2* pq = g.partial + (long long)b * g.nblk * g.ps + q;
        for (int c = 0; c < ncta; ++c) {
            const double2 v = ld_cg(pq + (long long)c * g.ps);
            re += v.x;
            im += v.y;
        }
        const int sl = q / K, i = q % K;
        const double sc = (sl < K ? 1.0 : g.sigma[b * (m + 1) + sl]) * dd[i];
        out[2 * (sl + (m + 1) * i)] = re * sc;
        out[2 * (sl + (m + 1) * i) + 1] = im * sc;
    }
    if (threadIdx.x == 0) g.counter[b] = 0;
}

// ------------------------------------------------------------ final gates (fp64)
// iterative_solver.py:70-79: ||R(OP x) - Rb|| / ||Rb|| and
// max |OP x - b| / max(|OP||x| + |b|, 1e-30), plus a finiteness check.
template <bool ADJ, bool MS = false>
__global__ void __launch_bounds__(256) k_gates(OpView<double> op, const double2* rhs,
                                               const double2* x, long long ld, GState g) {
    const int b = blockIdx.y;
    if constexpr (MS) op = g.slots[b].op64;
    const int ncta = rhs_ctas<MS>(g, b);
    if (int(blockIdx.x) >= ncta) return;
    __shared__ double sh[32];
    const double2* rb = rhs + b * ld;
    const double2* xb = x + b * ld;
    double s2 = 0.0, b2 = 0.0, bwd = 0.0, bad = 0.0;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < op.n;
         n += (long long)ncta * blockDim.x) {
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
    double2* part = g.partial + ((long long)b * g.nblk + blockIdx.x) * g.ps;
    if (threadIdx.x == 0) {
        part[0] = make_double2(s2, b2);
        part[1] = make_double2(bwd, bad);
    }
    if (!last_block_done(&g.counter[b], ncta)) return;
    double ts = 0, tb = 0, tw = 0, tbad = 0;
    for (int q = threadIdx.x; q < ncta; q += blockDim.x) {
        const double2* pq = g.partial + ((long long)b * g.nblk + q) * g.ps;
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
// A private stream per (host thread, device) for the graph capture, created
// on first use and kept for the life of the thread.
static cudaError_t capture_stream(cudaStream_t* out) {
    constexpr int kMaxDevices = 64;
    static thread_local cudaStream_t streams[kMaxDevices] = {};
    int cur = 0;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    if (cur < 0 || cur >= kMaxDevices) return cudaErrorInvalidDevice;
    if (streams[cur] == nullptr) {
        e = cudaStreamCreateWithFlags(&streams[cur], cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            streams[cur] = nullptr;
            return e;
        }
    }
    *out = streams[cur];
    return cudaSuccess;
}

// Owners of the per-solve graph and timing events: every return path of the
// driver releases them.
struct GraphHold {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~GraphHold() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};
struct EventHold {
    std::vector<cudaEvent_t> v;
    ~EventHold() {
        for (cudaEvent_t e : v)
            if (e) cudaEventDestroy(e);
    }
};


// The recycled-space kernels are instantiated for every k = 1..kMaxRecycle.
// (bfloat16: the new pair on tcgen05 when `umma` and k is 4 or 8, else mma.sync)
template <typename S, int K, bool MS> const void* recycle_kernel_k(bool combine, bool umma) {
    if constexpr (std::is_same<S, bf2>::value) {
        if constexpr (K % 4 == 0 && K <= 8)
            if (combine && umma) return (const void*)k_combine_umma<K, MS>;
        return combine ? (const void*)k_combine_mma<K, MS> : (const void*)k_bdots_mma<K, MS>;
    }
    return combine ? (const void*)k_combine<S, K, MS> : (const void*)k_bdots<S, K, MS>;
}
template <typename S, bool MS> const void* recycle_kernel(int k, bool combine, bool umma = false) {
    switch (k) {
#define USV_K(K) case K: return recycle_kernel_k<S, K, MS>(combine, umma);
        USV_K(1) USV_K(2) USV_K(3) USV_K(4) USV_K(5) USV_K(6) USV_K(7) USV_K(8)
        USV_K(9) USV_K(10) USV_K(11) USV_K(12) USV_K(13) USV_K(14) USV_K(15) USV_K(16)
#undef USV_K
        default: return nullptr;
    }
}

// Coefficients of the next recycled pair from one finished cycle's host-read
// block: the harmonic Ritz update of GCRO-DR (Parks, de Sturler, Mackey,
// Johnson & Maiti, SIAM J. Sci. Comput. 28 (2006), Algorithm 2.1) on
//   G ((L+1) x L): columns t < kc = d_t e_t, columns t >= kc = the raw
//                  Arnoldi columns (K W = Vhat G, W = [Ut, V_kc..V_{L-1}]),
//   Vhat^H W:      columns t < kc = bd[:, t], columns t >= kc = e_t.
// P = the k harmonic Ritz vectors of smallest |theta|, [Q, Rq] = qr(G P),
// U' = W P Rq^{-1}, C' = Vhat Q (so K U' = C', C' orthonormal). Output rows:
// [U_old (kc) | C_old (kc) | Krylov slots kc..m], columns [U' (k) | C' (k)],
// with the storage scales d (U) and sigma (slots) folded in.
static bool recycle_coefficients(int m, int k, const double* hb, std::vector<double2>& coef,
                                 int& src_kc) {
    using dense::cd;
    const int L = int(hb[hb_tail(m, k)]), kc = int(hb[hb_tail(m, k) + 1]);
    src_kc = kc;
    if (L - kc < 1 || L < k || L > m || kc > k) return false;
    const double* graw = hb + hb_graw(m);
    const double* bd = hb + hb_bd(m);
    const double* sigma = hb + hb_sigma(m, k);
    const double* d = hb + hb_d(m, k);
    const int r = L + 1;
    std::vector<cd> G(size_t(r) * L, cd(0.0)), W(size_t(r) * L, cd(0.0));
    for (int t = 0; t < L; ++t) {
        if (t < kc) {
            G[t + size_t(r) * t] = d[t];
            for (int sl = 0; sl < r; ++sl) {
                const double* v = bd + 2 * (sl + (m + 1) * t);
                W[sl + size_t(r) * t] = cd(v[0], v[1]);
            }
        } else {
            for (int sl = 0; sl <= t + 1; ++sl) {
                const double* v = graw + 2 * (t * (m + 1) + sl);
                G[sl + size_t(r) * t] = cd(v[0], v[1]);
            }
            W[t + size_t(r) * t] = 1.0;
        }
    }
    std::vector<cd> P, theta;
    if (!dense::harmonic_ritz(L, k, G, W, P, theta)) return false;
    std::vector<cd> GP(size_t(r) * k, cd(0.0)), Q, Rq;
    for (int c = 0; c < k; ++c)
        for (int t = 0; t < L; ++t) {
            const cd pv = P[t + size_t(L) * c];
            for (int sl = 0; sl < r; ++sl) GP[sl + size_t(r) * c] += G[sl + size_t(r) * t] * pv;
        }
    if (!dense::qr(r, k, GP, Q, Rq)) return false;
    std::vector<cd> Pu(size_t(L) * k);  // P Rq^{-1}
    for (int t = 0; t < L; ++t)
        for (int c = 0; c < k; ++c) {
            cd acc = P[t + size_t(L) * c];
            for (int q = 0; q < c; ++q) acc -= Pu[t + size_t(L) * q] * Rq[q + size_t(k) * c];
            Pu[t + size_t(L) * c] = acc / Rq[c + size_t(k) * c];
        }
    const int rows = kc + m + 1;
    coef.assign(size_t(rows) * 2 * k, make_double2(0.0, 0.0));
    bool finite = true;
    auto put = [&](int row, int col, cd v) {
        finite = finite && std::isfinite(v.real()) && std::isfinite(v.imag());
        coef[size_t(row) * 2 * k + col] = make_double2(v.real(), v.imag());
    };
    for (int c = 0; c < k; ++c) {
        for (int t = 0; t < L; ++t) {
            const cd v = Pu[t + size_t(L) * c];
            if (t < kc) put(t, c, v * d[t]);
            else put(kc + t, c, v * sigma[t]);
        }
        for (int sl = 0; sl < r; ++sl) {
            const cd v = Q[sl + size_t(r) * c];
            put(kc + sl, k + c, sl < kc ? v : v * sigma[sl]);
        }
    }
    return finite;
}

constexpr double kSceneWaves = 4.0;  // multi-scene grids: waves of CTA shares
template <typename R, typename S, bool ADJ, bool MS = false>
static int run_gmres(const usv_scene& s, const void* op_buf, const usv_gmres_params& p,
                     const double2* rhs, double2* x, int B, long long ld, char* ws,
                     const WsLayout& L, GState& g, usv_gmres_stats* stats, cudaStream_t strm,
                     const std::vector<SceneSlot>* slots = nullptr) {
    using C2 = S;  // stored Krylov vector element
    const OpView<double> op64 = make_view<double>(s, op_buf, ADJ);
    const OpView<R> opk = make_view<R>(s, op_buf, ADJ);
    C2* V = reinterpret_cast<C2*>(ws + L.V);
    if constexpr (MS) {
        SceneSlot* dslots = reinterpret_cast<SceneSlot*>(ws + L.slots);
        USV_CUDA_TRY(cudaMemcpyAsync(dslots, slots->data(), sizeof(SceneSlot) * size_t(B),
                                     cudaMemcpyHostToDevice, strm));
        g.slots = dslots;
    }
    const size_t lsq_smem = sizeof(double2) * size_t(g.m) * (g.m + 1);
    const size_t pipe_smem = Pipe<C2>::STAGED ? Pipe<C2>::BYTES : 16;
    const Step step = make_step(kThreads, s.nx, s.ny);
    const Step step_d = make_step(kDotsThreads, s.nx, s.ny);
    USV_CUDA_TRY(cudaFuncSetAttribute(k_orth<S, MS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(pipe_smem)));
    USV_CUDA_TRY(cudaFuncSetAttribute(k_update<S, MS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(pipe_smem)));
    // Grids fill the GPU once (resident CTAs per SM x SMs, shared by the B
    // right-hand sides); every CTA loops over node chunks, so there is no
    // partial last wave and the last CTA reduces one partial per CTA.
    int dev = 0, sms = 0;
    USV_CUDA_TRY(cudaGetDevice(&dev));
    USV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    auto grid_for = [&](const void* fn, int threads, size_t smem, dim3& grid,
                        int fixed_per_sm = 0) -> int {
        int per_sm = fixed_per_sm;
        if (per_sm <= 0)
            USV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
        // one wave of resident CTAs shared by the right-hand sides. For a
        // multi-scene batch the per-RHS shares are proportional to the scene
        // sizes (rhs_ctas) and add up to kSceneWaves waves while every RHS is
        // active: when the small scenes have converged, the large ones still
        // fill the GPU (CTAs of finished right-hand sides return at once)
        long long x = (long long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1) / B;
        if constexpr (MS) {
            double total = 0.0;
            for (const SceneSlot& sl : *slots) total += double(sl.n);
            x = (long long)(kSceneWaves * double((per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1)) *
                            double(g.n) / total);
        }
        if (p.max_ctas > 0 && x > p.max_ctas) x = p.max_ctas;
        x = x < 1 ? 1 : (x > g.nchunk ? g.nchunk : x);
        grid = dim3(unsigned(x), unsigned(B));
        return USV_OK;
    };
    dim3 grid_res, grid_dots, grid_orth, grid_upd, grid_gates;
    if (int e = grid_for((const void*)k_residual<ADJ, C2, MS>, 256, 0, grid_res)) return e;
    // Arnoldi stencil + dots: per-warp dot tasks with direct loads (two
    // bulk-copy layouts measured slower at 128^3, see the dots kernel)
    const void* fn_dots = (const void*)k_dots<R, S, ADJ, kDotsThreads, MS>;
    const int dots_threads = kDotsThreads;
    const size_t dots_smem = 0;
    USV_CUDA_TRY(cudaFuncSetAttribute(fn_dots, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(dots_smem)));
    if (int e = grid_for(fn_dots, dots_threads, dots_smem, grid_dots)) return e;
    // bfloat16 vectors: the Arnoldi stencil from the packed bfloat16 row
    // coefficients (24 B per node; USV_GMRES_DOTS_C64_ROWS: complex64, 48 B)
    const bool rows16 = std::is_same<S, bf2>::value && !(p.kernel_variant & USV_GMRES_DOTS_C64_ROWS);
    auto launch_dots = [&](cudaStream_t st, int j, int proj) -> cudaError_t {
        OpView<R> ov = opk;
        C2* vp = V;
        GState gs = g;
        Step sd = step_d;
        int r16 = rows16;
        void* args[] = {&ov, &vp, &gs, &j, &sd, &proj, &r16};
        return cudaLaunchKernel(fn_dots, grid_dots, dim3(dots_threads), args, dots_smem, st);
    };
    // orthogonalisation kernel: the bulk-copy ring (default for complex64 /
    // bfloat16) or the per-thread pipeline (USV_GMRES_ORTH_CPASYNC; always for
    // complex128, whose unrolled 16-byte loads need no staging)
    const bool orth_cpasync = (p.kernel_variant & USV_GMRES_ORTH_CPASYNC) != 0 ||
                              std::is_same<S, double2>::value;
    const void* fn_orth = orth_cpasync ? (const void*)k_orth<S, MS> : (const void*)k_orth_bulk<S, MS>;
    const int orth_threads = orth_cpasync ? kThreads : OrthBulk<S>::THREADS;
    const size_t orth_smem = orth_cpasync ? pipe_smem : OrthBulk<S>::SMEM;
    USV_CUDA_TRY(cudaFuncSetAttribute(fn_orth, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(orth_smem)));
    if (int e = grid_for(fn_orth, orth_threads, orth_smem, grid_orth)) return e;
    auto launch_orth = [&](cudaStream_t st, int j, int proj) -> cudaError_t {
        C2* vp = V;
        long long nn_ = g.n;
        GState gs = g;
        void* args[] = {&vp, &nn_, &gs, &j, &proj};
        return cudaLaunchKernel(fn_orth, grid_orth, dim3(orth_threads), args, orth_smem, st);
    };
    if (int e = grid_for((const void*)k_update<S, MS>, kThreads, pipe_smem, grid_upd)) return e;
    if (int e = grid_for((const void*)k_gates<ADJ, MS>, 256, 0, grid_gates)) return e;
    if (lsq_smem > 48 * 1024)
        USV_CUDA_TRY(cudaFuncSetAttribute(k_lsq, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(lsq_smem)));
    const int kr = g.kr;
    dim3 grid_bd, grid_comb;
    size_t bd_smem = 0, comb_smem = 0;
    const void* fn_bdots = nullptr;
    const void* fn_comb = nullptr;
    bool comb_umma = false;
    int comb_threads = kThreads;
    if (kr > 0) {
        using T = typename Wide<S>::T;
        bd_smem = std::is_same<S, bf2>::value
                      ? bdots_mma_smem(kr, g.m)
                      : sizeof(T) * size_t(kr) * kBdTile + sizeof(double2) * size_t(g.m + 1) * kr;
        // bfloat16, k = 4 or 8, k + m + 1 <= 64 input rows: the new pair on
        // tcgen05 (USV_GMRES_COMBINE_MMA_SYNC keeps the mma.sync kernel)
        comb_umma = std::is_same<S, bf2>::value && (kr == 4 || kr == 8) &&
                    kr + g.m + 1 <= kUmmaMaxRows &&
                    !(p.kernel_variant & USV_GMRES_COMBINE_MMA_SYNC);
        comb_smem = comb_umma ? combine_umma_smem(kr, g.m)
                    : std::is_same<S, bf2>::value ? combine_mma_smem(kr, g.m)
                                                  : sizeof(T) * size_t(kr + g.m + 1) * 2 * kr;
        comb_threads = comb_umma ? kUmmaThreads : kThreads;
        fn_bdots = recycle_kernel<S, MS>(kr, false);
        fn_comb = recycle_kernel<S, MS>(kr, true, comb_umma);
        if (!fn_bdots || !fn_comb) return USV_ERR_ARG;
        USV_CUDA_TRY(cudaFuncSetAttribute(fn_bdots, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(bd_smem)));
        USV_CUDA_TRY(cudaFuncSetAttribute(fn_comb, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(comb_smem)));
        // the tcgen05 pair kernel holds ~57 KB per CTA: ask for the full
        // shared-memory carveout so that three CTAs share an SM
        if (comb_umma)
            USV_CUDA_TRY(cudaFuncSetAttribute(fn_comb, cudaFuncAttributePreferredSharedMemoryCarveout,
                                              int(cudaSharedmemCarveoutMaxShared)));
        if (int e = grid_for(fn_bdots, kThreads, bd_smem, grid_bd)) return e;
        // tcgen05 pair kernel: as many CTAs per SM as its shared memory allows
        // (the occupancy query answers 1 for it), at most 512 TMEM columns
        int comb_per_sm = 0;
        if (comb_umma) {
            int smem_sm = 0, smem_res = 0;
            cudaFuncAttributes fa{};
            USV_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
            USV_CUDA_TRY(cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, dev));
            USV_CUDA_TRY(cudaFuncGetAttributes(&fa, fn_comb));
            comb_per_sm = int(size_t(smem_sm) / (comb_smem + fa.sharedSizeBytes + size_t(smem_res)));
            const int by_tmem = 512 / umma_tmem_cols(kr);
            comb_per_sm = comb_per_sm < 1 ? 1 : (comb_per_sm > by_tmem ? by_tmem : comb_per_sm);
        }
        if (int e = grid_for(fn_comb, comb_threads, comb_smem, grid_comb, comb_per_sm)) return e;
    }
    // zero the state and the solution
    USV_CUDA_TRY(cudaMemsetAsync(ws + L.state_begin, 0, L.total - L.state_begin, strm));
    if (kr > 0) {
        // Krylov and pair buffers start zero: every load stays finite, padding included
        USV_CUDA_TRY(cudaMemsetAsync(ws + L.V, 0, L.coef - L.V, strm));
    } else if (MS) {
        // scenes smaller than the vector stride: every vector is zero past its
        // scene's last node (the same padding rule as below)
        USV_CUDA_TRY(cudaMemsetAsync(ws + L.V, 0, L.partial - L.V, strm));
    } else if (g.nv > g.n) {
        // paired loads may touch the padding past node n-1 of each basis vector:
        // keep it zero so it contributes nothing to the dots
        USV_CUDA_TRY(cudaMemset2DAsync(V + g.n, g.nv * sizeof(C2), 0, (g.nv - g.n) * sizeof(C2),
                                       size_t(g.m + 1) * B, strm));
    }
    USV_CUDA_TRY(cudaMemset2DAsync(x, ld * sizeof(double2), 0, g.n * sizeof(double2), B, strm));
    if (kr == 0) {
        k_residual<ADJ, C2, MS><<<grid_res, 256, 0, strm>>>(op64, rhs, x, ld, V, g, 1, step);
        USV_CUDA_TRY(cudaGetLastError());
    }
    // Recycling: pinned host blocks for the per-cycle read of the Hessenberg /
    // inner-product data and the upload of the control words and coefficients.
    struct Pinned {
        void* p = nullptr;
        ~Pinned() { if (p) cudaFreeHost(p); }
    } hb_pin, up_pin[2];
    const size_t hb_bytes = sizeof(double) * size_t(B) * (kr > 0 ? g.hb_len : 0);
    const size_t coef_elems = size_t(kr + g.m + 1) * 2 * kr;
    const size_t up_ctl_bytes = sizeof(int) * size_t(B) * kCtl;
    const size_t up_bytes = up_ctl_bytes + sizeof(double2) * coef_elems * B;
    if (kr > 0) {
        USV_CUDA_TRY(cudaMallocHost(&hb_pin.p, hb_bytes));
        for (auto& u : up_pin) USV_CUDA_TRY(cudaMallocHost(&u.p, up_bytes));
    }

    // Event timing: one event before the first kernel of a cycle and one after
    // every kernel; consecutive pairs bracket single launches.
    usv_gmres_profile* prof = p.profile;
    const int kernels_per_cycle = 2 * g.m + 3 + (kr > 0 ? 3 : 0);
    EventHold events;
    std::vector<cudaEvent_t>& ev = events.v;
    std::vector<int> fam;
    if (prof) {
        ev.assign(kernels_per_cycle + 1, nullptr);
        for (auto& e : ev) USV_CUDA_TRY(cudaEventCreate(&e));
    }
    // nodes per right-hand side for the byte counts (multi-scene: the mean)
    double nn = double(g.n);
    if constexpr (MS) {
        nn = 0.0;
        for (const SceneSlot& sl : *slots) nn += double(sl.n);
        nn /= double(B);
    }
    const double vb = double(sizeof(C2));
    std::vector<double> fam_bytes;
    // per measured interval: the Arnoldi step j (-1: none) and whether it
    // only runs in recycled cycles (1) or with a new pair (2), so that the
    // empty launches of a cycle count no bytes
    std::vector<int> fam_step, fam_need;
    std::vector<double> fam_shared;  // bytes read once per launch for all RHS
    auto mark = [&](cudaStream_t st, int idx, bool capturing) {
        if (!prof) return cudaSuccess;
        return capturing ? cudaEventRecordWithFlags(ev[idx], st, cudaEventRecordExternal)
                         : cudaEventRecord(ev[idx], st);
    };
    auto launch_cycle = [&](cudaStream_t st, bool capturing) -> int {
        int k = 0;
        fam.clear();
        fam_bytes.clear();
        fam_step.clear();
        fam_need.clear();
        fam_shared.clear();
        USV_CUDA_TRY(mark(st, k++, capturing));
        if (kr > 0) {
            // new pair (when the host supplied coefficients), FP64 residual into
            // slot kc, projection of it on the recycled C
            {
                C2* vp = V;
                GState gs = g;
                long long nn_ = g.n;
                void* args[] = {&vp, &nn_, &gs};
                USV_CUDA_TRY(cudaLaunchKernel(fn_comb, grid_comb, dim3(comb_threads), args, comb_smem, st));
            }
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(6);
            fam_bytes.push_back(nn * vb * (g.m + 1.0 + 3 * kr));  // read U, C, slots kc..m; write U', C'
            fam_shared.push_back(0.0);
            fam_step.push_back(-1);
            fam_need.push_back(2);
            k_residual<ADJ, C2, MS><<<grid_res, 256, 0, st>>>(op64, rhs, x, ld, V, g, 0, step);
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(4);
            // per RHS: x, b, the stored residual; per launch: node record (R),
            // diagonal and the six FP64 edge coefficients
            fam_bytes.push_back(nn * (2 * sizeof(double2) + vb));
            fam_shared.push_back(nn * (sizeof(double4) + 7 * sizeof(double2)));
            fam_step.push_back(-1);
            fam_need.push_back(0);
            USV_CUDA_TRY(launch_dots(st, 0, 1));
            USV_CUDA_TRY(launch_orth(st, 0, 1));
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(7);
            fam_bytes.push_back(nn * vb * (2.0 * kr + 3));
            fam_shared.push_back(0.0);
            fam_step.push_back(-1);
            fam_need.push_back(1);
        }
        for (int j = 0; j < g.m; ++j) {
            USV_CUDA_TRY(launch_dots(st, j, 0));
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(0);
            // per RHS: read u_0..u_j (u_j also feeds the stencil), write w; per
            // launch: the row coefficients (complex64: 48 B) or node records
            // (complex128: 32 B), the same for every RHS of the batch
            fam_bytes.push_back(nn * vb * (j + 2));
            fam_shared.push_back(nn * (sizeof(R) == 8 ? 32.0 : (rows16 ? 24.0 : 48.0)));
            fam_step.push_back(j);
            fam_need.push_back(0);
            USV_CUDA_TRY(launch_orth(st, j, 0));
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(1);
            fam_bytes.push_back(nn * vb * (j + 3));
            fam_shared.push_back(0.0);
            fam_step.push_back(j);
            fam_need.push_back(0);
        }
        k_lsq<<<B, 128, lsq_smem, st>>>(g);
        USV_CUDA_TRY(mark(st, k++, capturing));
        fam.push_back(2);
        fam_bytes.push_back(0.0);
        fam_shared.push_back(0.0);
        fam_step.push_back(-1);
        fam_need.push_back(0);
        k_update<S, MS><<<grid_upd, kThreads, pipe_smem, st>>>(op64, V, x, ld, g);
        USV_CUDA_TRY(mark(st, k++, capturing));
        fam.push_back(3);
        fam_bytes.push_back(nn * (vb * g.m + 2 * sizeof(double2) + sizeof(double4)));
        fam_shared.push_back(0.0);
        fam_step.push_back(-1);
        fam_need.push_back(0);
        if (kr > 0) {
            // inner products for the harmonic Ritz step, then the host-read block
            {
                C2* vp = V;
                GState gs = g;
                long long nn_ = g.n;
                void* args[] = {&vp, &nn_, &gs};
                USV_CUDA_TRY(cudaLaunchKernel(fn_bdots, grid_bd, dim3(kThreads), args, bd_smem, st));
            }
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(7);
            fam_bytes.push_back(nn * vb * (g.m + 1.0 + kr));
            fam_shared.push_back(0.0);
            fam_step.push_back(-1);
            fam_need.push_back(3);
            USV_CUDA_TRY(cudaMemcpyAsync(hb_pin.p, ws + L.hb, hb_bytes, cudaMemcpyDeviceToHost, st));
        } else {
            k_residual<ADJ, C2, MS><<<grid_res, 256, 0, st>>>(op64, rhs, x, ld, V, g, 0, step);
            USV_CUDA_TRY(mark(st, k++, capturing));
            fam.push_back(4);
            // per RHS: x, b, the stored residual; per launch: node record (R),
            // diagonal and the six FP64 edge coefficients
            fam_bytes.push_back(nn * (2 * sizeof(double2) + vb));
            fam_shared.push_back(nn * (sizeof(double4) + 7 * sizeof(double2)));
            fam_step.push_back(-1);
            fam_need.push_back(0);
        }
        USV_CUDA_TRY(cudaGetLastError());
        return USV_OK;
    };
    // measured cycle's recycled count and new-pair flag (first active RHS)
    int meas_kc = 0, meas_combine = 0, meas_harvest = 0;
    auto accumulate = [&](std::vector<int>& active_counts) -> int {
        if (!prof) return USV_OK;
        for (size_t i = 0; i < fam.size(); ++i) {
            float ms = 0.f;
            USV_CUDA_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            prof->milliseconds[fam[i]] += ms;
            prof->launches[fam[i]] += 1;
            const bool idle = (fam_step[i] >= 0 && fam_step[i] < meas_kc) ||
                              (fam_need[i] == 1 && meas_kc == 0) ||
                              (fam_need[i] == 2 && !meas_combine) ||
                              (fam_need[i] == 3 && (meas_kc == 0 || !meas_harvest));
            if (!idle && active_counts[0] > 0)
                prof->bytes[fam[i]] += fam_bytes[i] * active_counts[0] + fam_shared[i];
        }
        return USV_OK;
    };

    GraphHold cycle_graph;
    cudaGraphExec_t& exec = cycle_graph.exec;
    if (p.use_graph) {
        cudaStream_t cap = nullptr;
        USV_CUDA_TRY(capture_stream(&cap));
        USV_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int st = launch_cycle(cap, true);
        cudaError_t e = cudaStreamEndCapture(cap, &cycle_graph.graph);
        if (st) return st;
        USV_CUDA_TRY(e);
        USV_CUDA_TRY(cudaGraphInstantiate(&exec, cycle_graph.graph, 0));
    }
    std::vector<int> status(B);
    std::vector<int> active(1, 0);
    int rc = USV_OK;
    bool pending = false;
    const int max_cycles = p.maxiter + 2;  // safety bound; the device status ends the loop
    // Recycling bookkeeping per RHS (lagged by one cycle): the pair, recycled
    // count and Krylov buffer of the last two launched cycles, and the
    // coefficients computed from the older one while the newer one runs.
    struct CycleUse { int pair = -1, kc = 0, vbuf = 0; };
    struct Pending { bool ready = false; int src_kc = 0; std::vector<double2> coef; };
    std::vector<CycleUse> last(B), before(B);
    std::vector<Pending> pend(B);
    std::vector<double> hb_cur(kr > 0 ? hb_bytes / sizeof(double) : 0);
    const int every = p.recycle_every > 0 ? p.recycle_every : 1;
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
        if (kr > 0) {
            if (cycle > 0) std::memcpy(hb_cur.data(), hb_pin.p, hb_bytes);
            // control words of this cycle
            int* ctl = static_cast<int*>(up_pin[cycle & 1].p);
            double2* coef = reinterpret_cast<double2*>(static_cast<char*>(up_pin[cycle & 1].p) +
                                                       up_ctl_bytes);
            bool any_combine = false;
            std::vector<CycleUse> now(B);
            for (int b = 0; b < B; ++b) {
                int* cw = ctl + b * kCtl;
                CycleUse u;
                u.vbuf = cycle % kVBufs;
                if (pend[b].ready && before[b].vbuf == u.vbuf) {
                    int dst = 0;
                    while (dst == before[b].pair || dst == last[b].pair) ++dst;
                    cw[CW_KC] = kr;
                    cw[CW_PAIR] = dst;
                    cw[CW_COMBINE] = 1;
                    cw[CW_SRC_PAIR] = before[b].pair;
                    cw[CW_SRC_VBUF] = before[b].vbuf;
                    cw[CW_SRC_KC] = pend[b].src_kc;
                    cw[CW_DST] = dst;
                    std::memcpy(coef + coef_elems * b, pend[b].coef.data(),
                                sizeof(double2) * pend[b].coef.size());
                    u.pair = dst;
                    u.kc = kr;
                    any_combine = true;
                } else {
                    cw[CW_KC] = last[b].kc;
                    cw[CW_PAIR] = last[b].pair > 0 ? last[b].pair : 0;
                    cw[CW_COMBINE] = 0;
                    cw[CW_SRC_PAIR] = cw[CW_SRC_VBUF] = cw[CW_SRC_KC] = cw[CW_DST] = 0;
                    u.pair = last[b].pair;
                    u.kc = last[b].kc;
                }
                cw[CW_VBUF] = u.vbuf;
                cw[CW_HARVEST] = cycle % every == 0;
                pend[b].ready = false;
                now[b] = u;
            }
            e = cudaMemcpyAsync(ws + L.ctl, ctl, up_ctl_bytes, cudaMemcpyHostToDevice, strm);
            if (e == cudaSuccess && any_combine)
                e = cudaMemcpyAsync(ws + L.coef, coef, sizeof(double2) * coef_elems * B,
                                    cudaMemcpyHostToDevice, strm);
            if (e != cudaSuccess) { rc = set_last_cuda_error(e); break; }
            before = last;
            last = now;
            for (int b = 0; b < B; ++b)
                if (status[b] == ST_ACTIVE) {
                    meas_kc = ctl[b * kCtl + CW_KC];
                    meas_combine = ctl[b * kCtl + CW_COMBINE];
                    meas_harvest = ctl[b * kCtl + CW_HARVEST];
                    break;
                }
        }
        if (exec) {
            e = cudaGraphLaunch(exec, strm);
            if (e != cudaSuccess) { rc = set_last_cuda_error(e); break; }
        } else {
            rc = launch_cycle(strm, false);
            if (rc) break;
        }
        pending = true;
        if (kr > 0 && cycle > 0 && (cycle - 1) % every == 0) {
            // harmonic Ritz step on the previous cycle's data while this one runs
            for (int b = 0; b < B; ++b)
                if (status[b] == ST_ACTIVE)
                    pend[b].ready = recycle_coefficients(g.m, kr, hb_cur.data() + size_t(b) * g.hb_len,
                                                         pend[b].coef, pend[b].src_kc) &&
                                    pend[b].src_kc == before[b].kc;
        }
    }
    if (rc) return rc;
    if (prof) USV_CUDA_TRY(cudaEventRecord(ev[0], strm));
    k_gates<ADJ, MS><<<grid_gates, 256, 0, strm>>>(op64, rhs, x, ld, g);
    USV_CUDA_TRY(cudaGetLastError());
    if (prof) {
        USV_CUDA_TRY(cudaEventRecord(ev[1], strm));
        USV_CUDA_TRY(cudaEventSynchronize(ev[1]));
        float ms = 0.f;
        USV_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        prof->milliseconds[5] += ms;
        prof->launches[5] += 1;
        prof->bytes[5] += nn * B * (2 * sizeof(double2) + sizeof(double4) + sizeof(double2));
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
        if (status[b] == ST_DEVICE_TIMEOUT) st.status = USV_ERR_DEVICE_TIMEOUT;
        else if (!finite || status[b] == ST_NONFINITE) st.status = USV_ERR_NONFINITE;
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
    if (p->recycle < 0 || p->recycle_every < 0) return USV_ERR_ARG;
    if (p->max_ctas < 0 || (p->kernel_variant & ~(USV_GMRES_ORTH_CPASYNC | USV_GMRES_COMBINE_MMA_SYNC | USV_GMRES_DOTS_C64_ROWS)))
        return USV_ERR_ARG;
    if (p->recycle > 0 && (p->recycle > kMaxRecycle || p->recycle > *m - 1)) return USV_ERR_ARG;
    *chunk = kChunk;  // node chunk per CTA (block_nodes is reserved)
    if (p->block_nodes != 0 && p->block_nodes != kChunk) return USV_ERR_ARG;
    *nblk = int((*n + *chunk - 1) / *chunk);
    return USV_OK;
}

}  // namespace usv

using namespace usv;

// Device state of one solve inside the caller's workspace.
static GState make_state(char* ws, const WsLayout& L, const usv_gmres_params* params, long long n,
                         int m, int chunk, int nblk, int nrhs) {
    const int kr = params->recycle;
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
    g.ps = partial_slots(m, kr);
    g.kr = kr;
    if (kr > 0) {
        g.hb_len = hb_size(m, kr);
        g.vstride = (long long)nrhs * (m + 1) * g.nv;
        g.pstride = (long long)nrhs * kr * g.nv;
        g.Ubuf = ws + L.U;
        g.Cbuf = ws + L.C;
        g.ctl = reinterpret_cast<int*>(ws + L.ctl);
        g.coef = reinterpret_cast<double2*>(ws + L.coef);
        g.hb = reinterpret_cast<double*>(ws + L.hb);
        g.dU = reinterpret_cast<double*>(ws + L.dU);
        g.alpha = reinterpret_cast<double2*>(ws + L.alpha);
        g.klast = reinterpret_cast<int*>(ws + L.klast);
        g.started = reinterpret_cast<int*>(ws + L.started);
    }
    return g;
}

extern "C" {

int usv_gmres_workspace_bytes(const usv_scene* scene, const usv_gmres_params* params, int nrhs,
                              size_t* bytes) {
    long long n;
    int m, chunk, nblk;
    int st = check_params(scene, params, nrhs, &n, &m, &chunk, &nblk);
    if (st) return st;
    if (!bytes) return USV_ERR_ARG;
    const size_t vb = vector_bytes(params->precision);
    *bytes = ws_layout(n, m, nrhs, nblk, vb, params->history_capacity, params->recycle).total;
    return USV_OK;
}

int usv_harmonic_ritz(int m, int k, const double* G, const double* W, double* P, double* theta) {
    if (m < 1 || k < 1 || k > m || !G || !W || !P || !theta) return USV_ERR_ARG;
    using dense::cd;
    const size_t n = size_t(m + 1) * m;
    std::vector<cd> g(n), w(n), p, th;
    for (size_t i = 0; i < n; ++i) {
        g[i] = cd(G[2 * i], G[2 * i + 1]);
        w[i] = cd(W[2 * i], W[2 * i + 1]);
    }
    if (!dense::harmonic_ritz(m, k, g, w, p, th)) return USV_ERR_NONFINITE;
    for (size_t i = 0; i < size_t(m) * k; ++i) {
        P[2 * i] = p[i].real();
        P[2 * i + 1] = p[i].imag();
    }
    for (int i = 0; i < k; ++i) {
        theta[2 * i] = th[i].real();
        theta[2 * i + 1] = th[i].imag();
    }
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
    const int kr = params->recycle;
    const WsLayout L = ws_layout(n, m, nrhs, nblk, vb, params->history_capacity, kr);
    if (workspace_bytes < L.total) return USV_ERR_WORKSPACE;
    char* ws = static_cast<char*>(workspace);
    GState g = make_state(ws, L, params, n, m, chunk, nblk, nrhs);
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


// Several scenes in one batched solve: right-hand side b belongs to scene
// scene_of_rhs[b] (operator buffer op_bufs[scene]); every launch of a cycle
// covers all right-hand sides of all scenes, each CTA row (blockIdx.y = b)
// reading its scene from the slot table in the workspace. Vectors are laid
// out for the largest scene (ld >= its node count); a right-hand side of a
// smaller scene uses the first n entries of its column.
static int check_scenes(int nscenes, const usv_scene* scenes, const void* const* op_bufs,
                        const int* scene_of_rhs, const usv_gmres_params* params, int nrhs,
                        long long* nmax, int* m, int* chunk, int* nblk) {
    if (nscenes < 1 || !scenes || !scene_of_rhs || !params || nrhs < 1) return USV_ERR_ARG;
    *nmax = 0;
    int mmin = 1 << 30;
    for (int sc = 0; sc < nscenes; ++sc) {
        long long n;
        int mi, ch, nb;
        if (int st = check_params(&scenes[sc], params, nrhs, &n, &mi, &ch, &nb)) return st;
        if (op_bufs && !op_bufs[sc]) return USV_ERR_ARG;
        if (n > *nmax) *nmax = n;
        if (mi < mmin) mmin = mi;
        *chunk = ch;
    }
    for (int b = 0; b < nrhs; ++b)
        if (scene_of_rhs[b] < 0 || scene_of_rhs[b] >= nscenes) return USV_ERR_ARG;
    // one restart length for the batch: every scene must allow the requested m
    if (mmin != (params->restart < *nmax ? params->restart : int(*nmax))) return USV_ERR_ARG;
    *m = mmin;
    *nblk = int((*nmax + *chunk - 1) / *chunk);
    return USV_OK;
}

int usv_gmres_scenes_workspace_bytes(int nscenes, const usv_scene* scenes,
                                     const int* scene_of_rhs, const usv_gmres_params* params,
                                     int nrhs, size_t* bytes) {
    long long n;
    int m, chunk, nblk;
    int st = check_scenes(nscenes, scenes, nullptr, scene_of_rhs, params, nrhs, &n, &m, &chunk, &nblk);
    if (st) return st;
    if (!bytes) return USV_ERR_ARG;
    *bytes = ws_layout(n, m, nrhs, nblk, vector_bytes(params->precision), params->history_capacity,
                       params->recycle).total;
    return USV_OK;
}

int usv_gmres_solve_scenes(int nscenes, const usv_scene* scenes, const void* const* op_bufs,
                           const int* scene_of_rhs, const usv_gmres_params* params,
                           const void* rhs, void* x, int nrhs, int64_t ld, void* workspace,
                           size_t workspace_bytes, usv_gmres_stats* stats, void* stream) {
    long long n;
    int m, chunk, nblk;
    int st = check_scenes(nscenes, scenes, op_bufs, scene_of_rhs, params, nrhs, &n, &m, &chunk,
                          &nblk);
    if (st) return st;
    if (!op_bufs || !rhs || !x || !workspace || !stats || ld < n) return USV_ERR_ARG;
    const size_t vb = vector_bytes(params->precision);
    const WsLayout L = ws_layout(n, m, nrhs, nblk, vb, params->history_capacity, params->recycle);
    if (workspace_bytes < L.total) return USV_ERR_WORKSPACE;
    char* ws = static_cast<char*>(workspace);
    GState g = make_state(ws, L, params, n, m, chunk, nblk, nrhs);
    const bool adj = params->adjoint != 0;
    std::vector<SceneSlot> slots(nrhs);
    for (int b = 0; b < nrhs; ++b) {
        const usv_scene& sc = scenes[scene_of_rhs[b]];
        const void* buf = op_bufs[scene_of_rhs[b]];
        SceneSlot& sl = slots[b];
        sl.op64 = make_view<double>(sc, buf, adj);
        sl.op32 = make_view<float>(sc, buf, adj);
        sl.n = (long long)sc.nx * sc.ny * sc.nz;
        sl.nchunk = int((sl.n + chunk - 1) / chunk);
        sl.step = make_step(kThreads, sc.nx, sc.ny);
        sl.step_d = make_step(kDotsThreads, sc.nx, sc.ny);
    }
    // the zeroing of the solution covers each column's own scene
    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    const double2* b = static_cast<const double2*>(rhs);
    double2* xx = static_cast<double2*>(x);
    // the driver's scene-level set-up (grids, workspace clearing) uses the
    // largest scene; kernels take each right-hand side's own scene
    int big = 0;
    for (int sc = 1; sc < nscenes; ++sc)
        if ((long long)scenes[sc].nx * scenes[sc].ny * scenes[sc].nz >
            (long long)scenes[big].nx * scenes[big].ny * scenes[big].nz)
            big = sc;
#define USV_RUN(R, S, A) run_gmres<R, S, A, true>(scenes[big], op_bufs[big], *params, b, xx, nrhs, ld, ws, L, g, stats, strm, &slots)
    if (params->precision == USV_PREC_FP64)
        return adj ? USV_RUN(double, double2, true) : USV_RUN(double, double2, false);
    if (params->precision == USV_PREC_MIXED_BF16)
        return adj ? USV_RUN(float, bf2, true) : USV_RUN(float, bf2, false);
    return adj ? USV_RUN(float, float2, true) : USV_RUN(float, float2, false);
#undef USV_RUN
}

}  // extern "C"
