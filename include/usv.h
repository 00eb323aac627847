/*
 * usv.h — C ABI of the B200 (sm_100a) gpu_iterative Helmholtz backend.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (USV_OK = 0) and never throws. Device pointers are caller-owned (the
 * Python host allocates them as torch tensors); `stream` is a cudaStream_t
 * passed as void*. All work is stream-ordered; only the GMRES driver and
 * the final gates read results back to the host.
 *
 * Grid nodes use the reference's Fortran order idx = i + nx*(j + ny*k).
 * Complex vectors are interleaved (re, im) pairs: complex128 = double2,
 * complex64 = float2. Multi-RHS blocks are column-major, column b at
 * offset b*ld elements (the reference's (N, nrhs) Fortran arrays).
 *
 * Reference interfaces replaced (paths relative to the reference root):
 *   usv_operator_bytes / usv_operator_build
 *       ConservativeHelmholtz.__init__ + assemble()
 *       (src/algorithm/physics/conservative_helmholtz.py:18-149) and the
 *       row scaling / Jacobi set-up of GpuIterativeSolver.solve
 *       (src/algorithm/solvers/iterative_solver.py:37-56).
 *   usv_operator_apply / usv_operator_apply_kernel
 *       the CSR SpMV `A_gpu @ v` and its variants
 *       (iterative_solver.py:42,71,74-75; helmholtz_solver.py:613-620 for A^H).
 *   usv_gmres_workspace_bytes / usv_gmres_solve
 *       GpuIterativeSolver.solve (iterative_solver.py:30-104) driving
 *       cupyx.scipy.sparse.linalg.gmres, as reached from
 *       HelmholtzDirectSolver._solve_iterative / _solve_gpu_adjoint
 *       (src/algorithm/solvers/helmholtz_solver.py:589-632).
 *   usv_gmres_scenes_workspace_bytes / usv_gmres_solve_scenes
 *       the same solve for the right-hand sides of several scenes at once
 *       (the reference solves scenes one after the other; its column batching
 *       of one scene is phase_response_basis.py:97-115).
 *   usv_materials_blend
 *       WarpAssemblyEngine material stage + blend_obstacle_material
 *       (src/algorithm/physics/warp_utils.py:11-23, 50-77).
 *   usv_source_masses / usv_source_rhs
 *       source_mass_matrix + flux_rhs_columns + assemble_rhs
 *       (src/algorithm/physics/sinc_aperture.py:36-85; warp_utils.py:118-120).
 *   usv_basis_field / usv_basis_adjoint / usv_basis_target_response
 *       PhaseResponseBasis.field / phase_vjp / target_response
 *       (src/algorithm/training/phase_response_basis.py:139-253).
 *   usv_material_vjp
 *       ConservativeHelmholtz.material_vjp (conservative_helmholtz.py:151-175).
 */
#ifndef USV_H
#define USV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define USV_ABI_VERSION 3

/* status codes */
#define USV_OK 0
#define USV_ERR_ARG 1            /* invalid argument / scene (ValueError)        */
#define USV_ERR_CUDA 2           /* CUDA runtime error                           */
#define USV_ERR_WORKSPACE 3      /* workspace too small                          */
#define USV_ERR_NOT_CONVERGED 4  /* GMRES gates failed (RuntimeError)            */
#define USV_ERR_NONFINITE 5      /* non-finite value in the solve                */
#define USV_ERR_SOURCE_PML 6     /* deposited aperture overlaps the PML          */
#define USV_ERR_SOURCE_SOFT 7    /* deposited aperture touches a soft face       */
#define USV_ERR_SOURCE_CLEARANCE 8 /* aperture closer than one cell to a side    */
#define USV_ERR_TOO_LARGE 9      /* size beyond a fixed internal maximum          */
#define USV_ERR_DEVICE_TIMEOUT 10 /* a bounded device-side wait ran out          */

/* face kinds, faces in the reference order -x,+x,-y,+y,-z,+z */
#define USV_FACE_REFLECTING 0
#define USV_FACE_OPEN 1
#define USV_FACE_SOFT 2
#define USV_FACE_IMPEDANCE 3

/* operator variants for usv_operator_apply */
#define USV_APPLY_A 0        /* y = A x                                   (fp64) */
#define USV_APPLY_AH 1       /* y = A^H x                                 (fp64) */
#define USV_APPLY_ABS_A 2    /* y = |A| |x| (backward-error denominator)  (fp64) */
#define USV_APPLY_ABS_AH 3   /* y = |A^H| |x|                             (fp64) */
#define USV_APPLY_K 4        /* y = R A (s x), row-scaled Jacobi operator        */
#define USV_APPLY_KH 5       /* y = R' A^H (s' x), same for the adjoint          */

/* precisions */
#define USV_PREC_FP64 0      /* complex128 vectors, fp64 coefficients            */
#define USV_PREC_MIXED 1     /* complex64 Krylov vectors + FP64 refinement       */
#define USV_PREC_MIXED_BF16 2 /* bfloat16 complex Krylov vectors (4 B), fp32
                                 stencil, FP64 dots/Hessenberg + FP64 refinement
                                 (usv_gmres_* only)                              */

typedef struct usv_scene {
    int32_t nx, ny, nz;
    int32_t face_kind[6];        /* USV_FACE_* per face                          */
    double dx;                   /* node spacing (m)                             */
    double omega;                /* angular frequency (rad/s)                    */
    double impedance_re[6];      /* wall impedance Z (Pa s/m), impedance faces   */
    double impedance_im[6];
    int32_t pml_cells;           /* 0 = no PML                                   */
    int32_t pml_order;
    double pml_strength;
    int32_t pml_faces;           /* bit f set: PML on face f (must be open)      */
    int32_t reserved;
} usv_scene;

/* Per-kernel-family device time of one solve, measured with CUDA events
 * recorded between the launches (also inside the captured cycle graph).
 * Families: 0 Arnoldi stencil+dots, 1 orthogonalisation+norm,
 * 2 least squares, 3 solution update, 4 FP64 residual, 5 final gates,
 * 6 new recycled pair, 7 projection on the recycled space and the inner
 * products of the harmonic Ritz step. `launches` counts measured intervals
 * (a projection interval holds two kernels). */
#define USV_KFAMILIES 8
typedef struct usv_gmres_profile {
    int32_t launches[USV_KFAMILIES];
    double milliseconds[USV_KFAMILIES];
    double bytes[USV_KFAMILIES];   /* algorithmic DRAM bytes, summed over launches */
} usv_gmres_profile;

typedef struct usv_gmres_params {
    int32_t restart;             /* m of GMRES(m)                      (30)      */
    int32_t maxiter;             /* inner-iteration cap               (3000)     */
    double rtol;                 /* scaled relative residual target   (1e-6)     */
    double backward_error_tol;   /* componentwise gate                (1e-4)     */
    int32_t precision;           /* USV_PREC_*                                   */
    int32_t adjoint;             /* 0: solve A x = b, 1: solve A^H x = b         */
    int32_t full_cycles;         /* 1: every cycle runs all m steps (reference)  */
    int32_t use_graph;           /* 1: capture each cycle in a CUDA graph        */
    int32_t block_nodes;         /* nodes per CTA chunk, 0 = default (2048)      */
    int32_t history_capacity;    /* restarts recorded per RHS in `history`       */
    double* history;             /* host, nrhs x capacity: ||r||/||Rb|| at each
                                    restart test after the first (the library's
                                    pr_norm callback values); may be NULL        */
    usv_gmres_profile* profile;  /* host; NULL = no event timing                 */
    int32_t recycle;             /* k > 0: GCRO-DR(m, k), deflated restarting with
                                    k harmonic Ritz vectors carried from cycle to
                                    cycle (k <= min(16, m-1)); 0: plain GMRES(m) */
    int32_t recycle_every;       /* recompute the recycled space after every n-th
                                    cycle (0 or 1: every cycle)                  */
    int32_t max_ctas;            /* cap on the CTAs per right-hand side of the
                                    streaming kernels (each CTA then loops over
                                    more node chunks); 0 = fill the GPU          */
    int32_t kernel_variant;      /* USV_GMRES_* bits; 0 = the measured-fastest
                                    form (bulk-copy orthogonalisation ring)      */
} usv_gmres_params;

/* kernel_variant bits of usv_gmres_params (complex64 / bfloat16 vectors; the
 * complex128 path always uses the per-thread form) */
#define USV_GMRES_ORTH_CPASYNC 1   /* orthogonalisation: per-thread cp.async
                                      pipeline instead of the bulk-copy ring  */
#define USV_GMRES_COMBINE_MMA_SYNC 2  /* bfloat16 GCRO-DR: the new recycled pair
                                      with warp-level mma.sync instead of
                                      tcgen05 (used in any case unless k is
                                      4 or 8 and k + m + 1 <= 64)           */
#define USV_GMRES_DOTS_C64_ROWS 4  /* bfloat16 Arnoldi stencil: complex64 row
                                      coefficients (48 B per node) instead
                                      of packed bfloat16 ones (24 B)       */

typedef struct usv_gmres_stats {
    int32_t status;              /* USV_OK or USV_ERR_*                          */
    int32_t info;                /* the library's info (iters at maxiter)        */
    int32_t iterations;          /* inner iterations                             */
    int32_t cycles;              /* restart cycles                               */
    double scaled_residual;      /* ||R(Ax-b)|| / ||Rb||, fp64                   */
    double backward_error;       /* max |Ax-b| / (|A||x|+|b|), fp64              */
    double initial_residual;     /* ||Rb||                                       */
} usv_gmres_stats;

/* Host-only (no GPU work): the harmonic Ritz step of the recycled cycles.
 * G and W are (m+1) x m complex column-major (interleaved re, im): K W_m =
 * Vhat G and Vhat^H W_m of one cycle. Returns in P (m x k) the k unit
 * solutions z of G^H G z = theta G^H W z with the smallest |theta|, and the
 * theta. USV_ERR_NONFINITE when the eigen-solve fails. */
int usv_harmonic_ritz(int m, int k, const double* G, const double* W, double* P, double* theta);

/* Homogeneous surface solver: for each of `modes` (x, y) modes the backward
 * continued fraction of the z-axis operator (diag[nz], upper[nz-1],
 * lower[nz-1]; upper[j] = Z[j, j+1], lower[j] = Z[j+1, j]) shifted by
 * shift[mode]: history[j][mode] = u[j+1]/u[0], j < nz-1 (complex128 device
 * arrays). Replaces _cuda_z_transfer (homogeneous_surface.py:41-85). */
int usv_z_transfer(const void* shift, const void* diag, const void* upper, const void* lower,
                   void* history, int modes, int nz, void* stream);

/* library identity */
int usv_abi_version(void);
const char* usv_status_string(int status);
int usv_device_info(int* sm_count, int* cc_major, int* cc_minor);

/* ---- operator ---------------------------------------------------------- */
/* Bytes of the device buffer that holds the per-node operator records. */
int usv_operator_bytes(const usv_scene* scene, size_t* bytes);
/* Build coefficients from rho, c (device fp64, N each). */
int usv_operator_build(const usv_scene* scene, const double* rho, const double* c,
                       void* op_buf, size_t op_bytes, void* stream);
/* y[:, b] = OP x[:, b] for b < nrhs; `precision` selects complex128/64 for
 * USV_APPLY_K/KH (the fp64-only variants ignore it). x and y must not
 * overlap (a row reads x at its six neighbours). */
int usv_operator_apply(const usv_scene* scene, const void* op_buf, int variant,
                       int precision, const void* x, void* y, int nrhs, int64_t ld,
                       void* stream);
/* usv_operator_apply with an explicit stencil kernel for USV_APPLY_K / KH in
 * complex64 (USV_PREC_MIXED); other variants and precisions ignore `kernel`.
 * Replaces the same SpMV as usv_operator_apply; the kernel choice is what
 * autotune.StencilTuner measures. */
#define USV_STENCIL_AUTO 0          /* the library's default for the batch     */
#define USV_STENCIL_COEF_ROWS 1     /* precomputed complex64 row coefficients
                                       (48 B per node), one thread per node    */
#define USV_STENCIL_RECORD_TILES 2  /* 16-B node records {rho, R, s}, rows
                                       formed in registers, z-marching tiles;
                                       nrhs <= 4                               */
int usv_operator_apply_kernel(const usv_scene* scene, const void* op_buf, int variant,
                              int precision, int kernel, const void* x, void* y, int nrhs,
                              int64_t ld, void* stream);
/* Copies of the per-node diagonal (complex128), row scale R and Jacobi s
 * (forward, adjoint) for inspection; any pointer may be NULL. */
int usv_operator_export(const usv_scene* scene, const void* op_buf, double* diag,
                        double* row_scale, double* jacobi, double* row_scale_adj,
                        double* jacobi_adj, void* stream);

/* ---- GMRES ------------------------------------------------------------- */
int usv_gmres_workspace_bytes(const usv_scene* scene, const usv_gmres_params* params,
                              int nrhs, size_t* bytes);
/* Solve OP x[:, b] = rhs[:, b] (complex128, device) for b < nrhs. x is
 * overwritten. `stats` is a host array of nrhs entries. Returns USV_OK when
 * the call itself worked; per-RHS outcome is in stats[b].status. */
int usv_gmres_solve(const usv_scene* scene, const void* op_buf,
                    const usv_gmres_params* params, const void* rhs, void* x,
                    int nrhs, int64_t ld, void* workspace, size_t workspace_bytes,
                    usv_gmres_stats* stats, void* stream);

/* Several scenes in one batched solve (the uneven-grid scene batches): the
 * right-hand side b belongs to scene scene_of_rhs[b] < nscenes, whose
 * operator buffer is op_bufs[scene]. Every kernel launch of a restart cycle
 * covers all right-hand sides of all scenes. rhs and x are columns of stride
 * ld >= the largest scene's node count; a right-hand side of a smaller scene
 * uses the first n entries of its column. All scenes share the parameters
 * (restart, recycling, precision, adjoint); the restart length must not be
 * cut by a scene smaller than it. Replaces the per-scene loop over
 * HelmholtzDirectSolver solves (phase_response_basis.py:97-115 batches one
 * scene's columns; scenes were solved one after the other). */
int usv_gmres_scenes_workspace_bytes(int nscenes, const usv_scene* scenes,
                                     const int* scene_of_rhs, const usv_gmres_params* params,
                                     int nrhs, size_t* bytes);
int usv_gmres_solve_scenes(int nscenes, const usv_scene* scenes, const void* const* op_bufs,
                           const int* scene_of_rhs, const usv_gmres_params* params,
                           const void* rhs, void* x, int nrhs, int64_t ld, void* workspace,
                           size_t workspace_bytes, usv_gmres_stats* stats, void* stream);

/* ---- scene set-up ------------------------------------------------------ */
/* rho, c from an SDF: h = sine-smoothed step over +-width, blend 1/rho and
 * 1/(rho c^2) between obstacle and medium. Medium arrays may be NULL (then
 * the scalars rho0, c0 are used). sdf may be NULL with radius>=0: sphere at
 * center (m) in node coordinates (i*dx). */
int usv_materials_blend(const usv_scene* scene, const double* sdf, const double* center,
                        double radius, double width, double rho_obstacle,
                        double c_obstacle, const double* rho_medium,
                        const double* c_medium, double rho0, double c0, double* rho,
                        double* c, void* stream);
/* masses (device fp64, nx*ny x M column-major, followed by ONE spare
 * double used as a check word, so nx*ny*M + 1 doubles) of M apertures with
 * centres given twice, on the host (for the clearance checks) and on the
 * device (M x 3, z must be 0), from a device quadrature of Q points (offsets
 * x, y and weights). Checks clearance, PML and soft-face overlap; `op_buf`
 * must already be built for the same scene. */
int usv_source_masses(const usv_scene* scene, const void* op_buf,
                      const double* centers_host, const double* centers_dev,
                      int m_emitters, double diameter, const double* quad_x,
                      const double* quad_y, const double* quad_w, int q_points,
                      double* masses, void* stream);
/* rhs[:, b] = -2 pi/(rho_ref dx^3) * sum_m masses[:, m] * coeff[b*m_emitters+m]
 * in the z=0 plane, zero elsewhere; coeff is complex128 (device). */
int usv_source_rhs(const usv_scene* scene, const double* masses, int m_emitters,
                   const double* coeff, double rho_ref, void* rhs, int nrhs, int64_t ld,
                   void* stream);

/* ---- phase response basis (G: complex64 columns, N x M, ld = N) -------- */
/* field (complex128, N) = sum_m G[:, m] e^{i phases[m]} */
int usv_basis_field(const void* basis, int64_t n, int m, int basis_precision,
                    const double* phases, void* field, void* stream);
/* response[m] = (G^H g)_m (complex128, may be NULL) and
 * grad[m] = Re(conj(response[m]) i e^{i phases[m]}) (may be NULL);
 * workspace holds per-chunk partial sums. */
int usv_basis_adjoint_workspace_bytes(int64_t n, int m, size_t* bytes);
int usv_basis_adjoint(const void* basis, int64_t n, int m, int basis_precision,
                      const void* cotangent, const double* phases, double* response,
                      double* grad, void* workspace, size_t workspace_bytes,
                      void* stream);
/* usv_basis_adjoint without a workspace, for callers that cannot allocate
 * device memory when they need the gradient (a process whose device memory
 * is owned by its own pool, a real-time loop that must not pay cudaMalloc
 * latency or risk out-of-memory, code running during CUDA graph capture).
 * It has no counterpart in the reference. The partial sums live in a 1 MiB
 * file-scope device array that every GPU loading this library holds until
 * exit; m (emitters) is limited to 4096, larger m returns USV_ERR_TOO_LARGE.
 * The first call on a device looks up the array's address
 * (cudaGetSymbolAddress) and caches it for the life of the process; make
 * that first call before any stream capture, and do not use this entry point
 * on a device after cudaDeviceReset (the cached address is then stale).
 * All calls share the array: calls that overlap on the GPU (other streams or
 * threads) race and must be serialised by the caller. */
int usv_basis_adjoint_noalloc(const void* basis, int64_t n, int m, int basis_precision,
                              const void* cotangent, const double* phases,
                              double* response, double* grad, void* stream);
/* out (device complex128, p x m, row-major) = trilinear interpolation of the
 * basis columns at p points (device fp64, p x 3, metres from node (0,0,0)).
 * Points are expected inside [0, (n-1) dx] per axis (the Python host checks
 * this, as the reference does); a point outside extrapolates linearly from
 * the nearest edge cell and a non-finite point gives NaN, never a load
 * outside the basis. */
int usv_basis_target_response(const void* basis, int64_t nx, int64_t ny, int64_t nz,
                              int m, int basis_precision, const double* points, int p,
                              double dx, void* out, void* stream);

/* ---- focal losses (phase_adjoint_optimizer.py:210-414) ------------------ */
#define USV_LOSS_FOCAL_PRESSURE 0  /* FocalPressureLoss                            */
#define USV_LOSS_FOCAL_CONTRAST 1  /* FocalContrastLoss (soft max over the mask)    */
#define USV_LOSS_CONTRAST_RATIO 2  /* -mean_t |u_t|^2 / mean_mask |u|^2             */
int usv_loss_workspace_bytes(int64_t n, size_t* bytes);
/* value (device, 3 doubles): {loss, mean |u_t|, mean |u_t|^2}; cotangent
 * (device complex128, N, may be NULL) in the dL = Re(g^H du) convention;
 * mask: device bytes (1 = background / shell node) or NULL = every node;
 * targets: device int64 Fortran node indices (repeats accumulate). Replaces
 * FocalPressureLoss / FocalContrastLoss .evaluate_device. */
int usv_loss(int mode, const void* field, int64_t n, const unsigned char* mask,
             const int64_t* targets, int n_targets, double target_weight,
             double background_weight, double temperature, double eps, double* value,
             void* cotangent, void* workspace, size_t workspace_bytes, void* stream);

/* ---- gradients --------------------------------------------------------- */
/* grad_rho, grad_c (device fp64) of dL = -Re(lambda^H dA u). */
int usv_material_vjp(const usv_scene* scene, const void* op_buf, const double* rho,
                     const double* c, const void* field, const void* adjoint,
                     double* grad_rho, double* grad_c, void* stream);
/* grad[m] += Re(conj((B^H lam)_m) * a_m * i e^{i phi_m}) for the z=0 source
 * columns; lam complex128 (device). */
int usv_source_phase_grad(const usv_scene* scene, const double* masses, int m_emitters,
                          const void* lam, const double* phases, const double* amplitudes,
                          double rho_ref, double* grad, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* USV_H */
