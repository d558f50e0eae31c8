/*
 * fvx.h -- C ABI of libfvx.so, the B200 (sm_100a) implementation of
 * finitevolX's explicit-step and elliptic-inversion hot path.
 *
 * finitevolX itself is a Python/JAX library with no C layer: its boundary
 * is the public Python API (finitevolx/__init__.py).  Each entry point below
 * names the reference interface it replaces (file:line inside the
 * finitevolX project).  A foreign-function binding (ctypes here; a jax.ffi
 * custom call where jaxlib's FFI headers exist) calls these directly.
 *
 * Conventions
 *   - Fields are row-major [ny, nx] device arrays with a one-cell ghost
 *     ring (same-index C-grid stagger: U[j,i] at i+1/2, V[j,i] at j+1/2,
 *     X[j,i] at the NE corner).  Masks are uint8 (0/1) device arrays.
 *   - Every pointer is a caller-owned device pointer; hot-path calls
 *     allocate nothing.  ``stream`` is a cudaStream_t (NULL = legacy).
 *   - Return value: 0 on success, otherwise an fvx_status code (1 shape,
 *     2 method, 3 dtype, 4 CUDA error, 5 not converged, 6 bad argument,
 *     7 device-side wait timed out).  No entry point traps on the device.
 *   - _f32 / _f64 suffixes select the arithmetic type.
 *
 * Advection method codes: 0 naive, 1 upwind1, 2 upwind2, 3 upwind3,
 * 4 weno3, 5 weno5, 6 wenoz5, 7 weno7, 8 weno9, 9 minmod, 10 van_leer,
 * 11 superbee, 12 mc, 13 wenoz3 (face fluxes only).
 */
#ifndef FVX_H
#define FVX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- masks ------------------------------------------------------------- */

/* Mask2D.from_mask (mask/cartesian.py:584-739) with pool_bool
 * (mask/utils.py:42-164), dilate_mask (:314-382), count_contiguous
 * (:385-468) and make_sponge (:471-546).  ``irr_flag`` marks the irregular
 * strict-corner boundary cells (compact with fvx_compact_flags); ``sponge``
 * may be NULL. */
int fvx_mask2d_build(const uint8_t* h, int ny, int nx, uint8_t* u, uint8_t* v, uint8_t* xy_corner,
                     uint8_t* xy_corner_strict, uint8_t* y_wall, uint8_t* x_wall, uint8_t* convex,
                     uint8_t* valid, int32_t* classification, uint8_t* irr_flag, int32_t* x_pos,
                     int32_t* x_neg, int32_t* y_pos, int32_t* y_neg, float* sponge, int sponge_width,
                     void* stream);

/* count_contiguous (mask/utils.py:385-468); axis 1 = x, 0 = y. */
int fvx_count_contiguous(const uint8_t* mask, int ny, int nx, int axis, int32_t* pos, int32_t* neg,
                         void* stream);

/* Mask2D.get_adaptive_masks (mask/cartesian.py:495-553): out[k] is the mask
 * of sizes_sorted[k] (device int32 array). */
int fvx_adaptive_masks(const int32_t* pos, const int32_t* neg, int64_t n, const int32_t* sizes_sorted,
                       int nsizes, uint8_t* out, void* stream);

/* Packed (2,4,6) tier codes of Advection2D's pre-built hierarchies
 * (advection/advection.py:310-327): bits 0-1 x tier, bits 2-3 y tier. */
int fvx_tier_codes(const int32_t* x_pos, const int32_t* x_neg, const int32_t* y_pos,
                   const int32_t* y_neg, int64_t n, uint8_t* out, void* stream);

/* np.where row-major compaction used for xy_corner_strict_irrbound_rows/cols
 * (mask/cartesian.py:675-689).  ``work``: 2*ny+1 int32; work[2*ny] = count. */
int fvx_compact_flags(const uint8_t* flags, int ny, int nx, int32_t* work, int32_t* rows, int32_t* cols,
                      void* stream);

/* ---- advection --------------------------------------------------------- */

/* Advection2D.__call__ (advection/advection.py:329-420).  ``tiers`` (packed
 * codes) selects the masked upwind_flux dispatch (advection/flux.py:100-253)
 * and requires ``mask_h``; tiers == NULL with mask_h != NULL is the
 * non-dispatchable masked path (output * mask.h). */
int fvx_advect2d_f32(const float* h, const float* u, const float* v, float* out, int ny, int nx, double dx,
                     double dy, int method, const uint8_t* tiers, const uint8_t* mask_h, void* stream);
int fvx_advect2d_f64(const double* h, const double* u, const double* v, double* out, int ny, int nx,
                     double dx, double dy, int method, const uint8_t* tiers, const uint8_t* mask_h,
                     void* stream);

/* Reconstruction2D.<method>_x / _y (advection/reconstruction.py:582-1306),
 * uv_center_flux (advection/face_flux.py:36-87).  fe or fn may be NULL. */
int fvx_face_flux2d_f32(const float* h, const float* u, const float* v, float* fe, float* fn, int ny, int nx,
                        int method, const uint8_t* tiers, void* stream);
int fvx_face_flux2d_f64(const double* h, const double* u, const double* v, double* fe, double* fn, int ny,
                        int nx, int method, const uint8_t* tiers, void* stream);

/* Flux divergence step of Advection2D.__call__ (advection/advection.py:410-419). */
int fvx_flux_divergence2d_f32(const float* fe, const float* fn, float* out, int ny, int nx, double dx,
                              double dy, const uint8_t* mask_h, void* stream);
int fvx_flux_divergence2d_f64(const double* fe, const double* fn, double* out, int ny, int nx, double dx,
                              double dy, const uint8_t* mask_h, void* stream);

/* upwind_flux tier blend (advection/flux.py:221-253); host arrays of
 * ``ntiers`` device pointers; dim 1 = x faces, 0 = y faces. */
int fvx_upwind_blend_f32(const float* const* fluxes, const uint8_t* const* masks, int ntiers, const float* u,
                         float* out, int ny, int nx, int dim, void* stream);
int fvx_upwind_blend_f64(const double* const* fluxes, const uint8_t* const* masks, int ntiers,
                         const double* u, double* out, int ny, int nx, int dim, void* stream);

/* ---- C-grid operators --------------------------------------------------- */

/* Difference2D (operators/difference.py:165-520) and Interpolation2D
 * (operators/interpolation.py:104-275).  op: 0 diff_x_T_to_U, 1 diff_y_T_to_V,
 * 2 diff_y_U_to_X, 3 diff_x_V_to_X, 4 diff_y_X_to_U, 5 diff_x_X_to_V,
 * 6 diff_x_U_to_T, 7 diff_y_V_to_T, 8 laplacian, 9 divergence(a=u,b=v),
 * 10 curl(a=u,b=v), 11 grad_perp (out=u, out2=v); 16 T_to_U, 17 T_to_V,
 * 18 T_to_X, 19 X_to_U, 20 X_to_V, 21 U_to_T, 22 V_to_T, 23 X_to_T,
 * 24 U_to_X, 25 V_to_X, 26 U_to_V, 27 V_to_U.  mask_out* may be NULL. */
int fvx_cgrid_op2d_f32(int op, const float* a, const float* b, float* out, float* out2, int ny, int nx,
                       double dx, double dy, const uint8_t* mask_out, const uint8_t* mask_out2, void* stream);
int fvx_cgrid_op2d_f64(int op, const double* a, const double* b, double* out, double* out2, int ny, int nx,
                       double dx, double dy, const uint8_t* mask_out, const uint8_t* mask_out2, void* stream);

/* arakawa_jacobian (operators/jacobian.py:22-131); out [batch, ny-2, nx-2]. */
int fvx_arakawa_jacobian_f32(const float* f, const float* g, float* out, int batch, int ny, int nx, double dx,
                             double dy, void* stream);
int fvx_arakawa_jacobian_f64(const double* f, const double* g, double* out, int batch, int ny, int nx,
                             double dx, double dy, void* stream);

/* Diffusion2D.__call__ / .fluxes (diffusion/diffusion.py:120-330); kappa is
 * the scalar unless kappa_field != NULL; any of out/flux_x/flux_y may be NULL. */
int fvx_diffusion2d_f32(const float* h, const float* kappa_field, double kappa, float* out, float* flux_x,
                        float* flux_y, int ny, int nx, double dx, double dy, const uint8_t* mask_u,
                        const uint8_t* mask_v, const uint8_t* mask_h, void* stream);
int fvx_diffusion2d_f64(const double* h, const double* kappa_field, double kappa, double* out, double* flux_x,
                        double* flux_y, int ny, int nx, double dx, double dy, const uint8_t* mask_u,
                        const uint8_t* mask_v, const uint8_t* mask_h, void* stream);

/* BiharmonicDiffusion2D.__call__ (diffusion/diffusion.py:462-574), fused. */
int fvx_biharmonic2d_f32(const float* h, double kappa, float* out, int ny, int nx, double dx, double dy,
                         const uint8_t* mask_h, void* stream);
int fvx_biharmonic2d_f64(const double* h, double kappa, double* out, int ny, int nx, double dx, double dy,
                         const uint8_t* mask_h, void* stream);

/* ---- boundary conditions and time stepping ------------------------------ */

/* enforce_periodic (boundary/boundary.py:52-75), in place, batched. */
int fvx_fill_periodic_f32(float* field, int batch, int ny, int nx, void* stream);
int fvx_fill_periodic_f64(double* field, int batch, int ny, int nx, void* stream);

/* pad_interior(mode="constant") (boundary/boundary.py:17-49), in place. */
int fvx_zero_ring_f32(float* field, int batch, int ny, int nx, void* stream);
int fvx_zero_ring_f64(double* field, int batch, int ny, int nx, void* stream);

/* out = (a*x + b*y) + c*z: stage combinations of euler/heun/rk3_ssp_step
 * (timestepping/explicit_rk.py:22-121); y and z may be NULL. */
int fvx_lincomb_f32(int64_t n, double a, const float* x, double b, const float* y, double c, const float* z,
                    float* out, void* stream);
int fvx_lincomb_f64(int64_t n, double a, const double* x, double b, const double* y, double c,
                    const double* z, double* out, void* stream);


/* ---- Dirichlet Helmholtz by DST-I tensor-core GEMMs --------------------- */

/* Replaces spectraldiffx solve_helmholtz_dst as re-exported by finitevolX
 * (solvers/spectral.py:14-98; called at scripts/qg_1p5_layer.py:444-449):
 * (nabla^2 - lambda) psi = rhs on an interior-only [ny, nx] array, psi = 0
 * outside.  A plan holds the DST-I matrices, eigenvalue grids and
 * workspaces; batch element b uses lambdas[b % n_lambda] (pv_inversion's
 * per-layer lambda, solvers/elliptic.py:517-541).  Creating a plan is the
 * only allocating call. */
typedef struct fvx_dst_plan fvx_dst_plan;
int fvx_dst_plan_create(int ny, int nx, double dx, double dy, int batch_max, const double* lambdas, int n_lambda,
                        int want_fp64, fvx_dst_plan** plan);
int fvx_dst_plan_destroy(fvx_dst_plan* plan);
/* The same plan for the other rectangular spectral solvers that
 * solvers/spectral.py:14-98 re-exports and _spectral_solve (:105-128)
 * dispatches: kind 0 = DST-I (Dirichlet, = fvx_dst_plan_create), 1 =
 * DCT-II (Neumann, solve_helmholtz_dct), 2 = periodic (solve_helmholtz_fft,
 * computed with the real Hartley transform pair, which diagonalises the
 * same periodic 5-point operator).  Input and output are the full [ny, nx]
 * array (no ghost ring); the null mode of a Neumann / periodic Poisson
 * problem is set to zero (the zero-mean solution).  DCT-II and periodic
 * plans take the dense product path; fvx_dst_solve_f64 supports method 0
 * only for them. */
int fvx_spectral_plan_create(int kind, int ny, int nx, double dx, double dy, int batch_max, const double* lambdas,
                             int n_lambda, int want_fp64, fvx_dst_plan** plan);
/* Capacitance-matrix step between the two rectangular solves of a masked
 * solve (the online part of the CapacitanceSolver that
 * solvers/elliptic.py:146-183 builds): out = f, then out[idx[k]] -=
 * sum_l cinv[k][l] u[idx[l]] (FP64 sums), k < nb; f, u, out hold n
 * elements (out may be f); idx are distinct flat indices, cinv is the
 * inverse capacitance matrix (nb x nb, row-major FP64). */
int fvx_capacitance_rhs_f32(const float* f, const float* u, const double* cinv, const long long* idx, int nb,
                            long long n, float* out, void* stream);
int fvx_capacitance_rhs_f64(const double* f, const double* u, const double* cinv, const long long* idx, int nb,
                            long long n, double* out, void* stream);
/* Reads the plan's device error flag (7 if a bounded wait gave up); syncs. */
int fvx_dst_plan_check(fvx_dst_plan* plan, void* stream);
/* Bound on every barrier wait inside the plan's tensor-core products, in SM
 * clock cycles (>= 1000; default 4e9, about 2 s): a wait that runs out ends
 * its CTA without trapping (after the copies and MMAs it issued have
 * landed) and sets the flag fvx_dst_plan_check reports (7) and then clears.
 * No counterpart in finitevolX (its XLA solve has no device waits). */
int fvx_dst_plan_set_wait_limit(fvx_dst_plan* plan, long long cycles);
/* Fault injection for tests only (no counterpart in finitevolX): while on,
 * the single-CTA products' producers issue no loads, so every product's
 * first wait runs out after the wait limit with nothing in flight. */
int fvx_dst_plan_inject_stall(fvx_dst_plan* plan, int on);
/* FP32: 3xBF16 split tcgen05 chain (ny, nx multiples of 8; otherwise the
 * FP64 chain with FP32 output).  Element (b,y,x) at ptr[b*bstride + y*ld + x]. */
int fvx_dst_solve_f32(fvx_dst_plan* plan, const float* rhs, long long rhs_bstride, long long rhs_ld, float* psi,
                      long long psi_bstride, long long psi_ld, int batch, void* stream);
/* FP64: method 0 = FP64 SIMT chain; 1 = split chain + FP64 iterative
 * refinement to normwise backward error <= tol (info: passes, backward
 * error, ||r||/||f||; returns 5 if max_iter passes do not reach tol). */
int fvx_dst_solve_f64(fvx_dst_plan* plan, const double* rhs, long long rhs_bstride, long long rhs_ld, double* psi,
                      long long psi_bstride, long long psi_ld, int batch, int method, double tol, int max_iter,
                      double* info, void* stream);
/* Same chain on an operand already split into the plan workspace (written
 * by fvx_qg_stage_f32's split outputs); fvx_dst_workspace returns it and
 * fvx_dst_operand_layout its layout (0 natural, 1 x de-interleaved: the
 * even/odd products of plans with ny, nx multiples of 256). */
int fvx_dst_solve_presplit_f32(fvx_dst_plan* plan, float* psi, long long psi_bstride, long long psi_ld, int batch,
                               void* stream);
/* FP64-residual iterative refinement of an FP32 Dirichlet result (the
 * accuracy step spectraldiffx's FP64 solve_helmholtz_dst does not need, and
 * this split-precision chain does): ``passes`` times r = rhs - (lap -
 * lambda) psi in FP64 from the FP32 arrays, psi += chain(r).  One pass
 * brings the chain's ~1e-5 relative error down to psi's FP32 rounding.
 * Overwrites the plan's first workspace; no host synchronisation. */
int fvx_dst_refine_f32(fvx_dst_plan* plan, const float* rhs, long long rhs_bstride, long long rhs_ld, float* psi,
                       long long psi_bstride, long long psi_ld, int batch, int passes, void* stream);
int fvx_dst_workspace(fvx_dst_plan* plan, void** w1_hi, void** w1_lo);
/* The FP64 chain's input workspace ([batch_max][ny][nx] doubles, natural
 * layout; plans with an FP64 chain) and the FP64 solve that starts from it
 * (fvx_dst_solve_f64's FP64 chain without its input copy): the FP64 QG
 * stage kernel writes its output's interior there.  Launch plumbing with no
 * counterpart in finitevolX. */
int fvx_dst_workspace_f64(fvx_dst_plan* plan, void** v1);
int fvx_dst_solve_presplit_f64(fvx_dst_plan* plan, double* psi, long long psi_bstride, long long psi_ld, int batch,
                               void* stream);
int fvx_dst_operand_layout(fvx_dst_plan* plan);
/* One product of the chain on the current workspaces (timing only). */
int fvx_dst_gemm_step(fvx_dst_plan* plan, int which, int batch, void* stream);
/* Even/odd product kernel (process-wide, for the autotuner): 0 = one CTA
 * per 128-row tile with 64-element K blocks (3 ring stages, default), 1 =
 * CTA pairs sharing each B block (cta_group::2; row counts that are
 * multiples of 256), 2 = one CTA per tile with 32-element K blocks (6 ring
 * stages); kind < 0 returns the current choice.  No counterpart in
 * finitevolX (launch configuration). */
int fvx_dst_kernel_config(int kind);

/* Allocation-free FP32 DST Helmholtz solve.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc while they run
 * (a framework custom call whose framework owns all device memory, a host
 * that forbids allocation after start-up, a loop that cannot take
 * cudaMalloc's implicit synchronisation).  Same result as
 * fvx_dst_solve_f32, batch 1, one lambda; its scratch is a fixed
 * file-scope device array (about 1.3 MB, held by every GPU that loads the
 * library until exit), so ny and nx must be multiples of 8 and at most 256
 * (otherwise returns 1 and does nothing).  The first call on a device looks
 * up the array's address (make it before any stream capture).  All calls
 * share the array: calls that overlap on the GPU race. */
int fvx_dst_solve_noalloc_f32(const float* rhs, long long rhs_ld, float* psi, long long psi_ld, int ny, int nx,
                              double dx, double dy, double lambda, void* stream);
/* Companion of fvx_dst_solve_noalloc_f32 (no counterpart in the reference):
 * the tensor-core products wait on barriers with a time limit, and a wait
 * that gives up sets an error flag in the scratch array instead of
 * trapping, while the solve itself has already returned 0.  This copies the
 * flag to the host on ``stream``, waits for the stream, and returns 7
 * (timeout: psi is incomplete) if it is set, 0 if not or if no
 * allocation-free solve ran on the current device.  Each solve clears the
 * flag, so check after every solve whose result matters. */
int fvx_dst_noalloc_check(void* stream);

/* ---- fused QG RK stage ---------------------------------------------------- */

/* One Runge-Kutta stage of the QG 1.5-layer PV equation
 * (scripts/qg_1p5_layer.py:454-487 inside rk3_ssp_step,
 * timestepping/explicit_rk.py:74-121): q_out = a*q_start + b*q_stage + c*rhs
 * with rhs = Advection2D(BC(q_stage), u, v) - beta*V_to_T(v) + forcing
 * - drag*laplacian(psi) + viscosity*laplacian(BC(q_stage)), (u, v) the
 * geostrophic velocity of psi_interior (zero outside).  periodic: 1 periodic
 * ghost ring, 0 zero ring.  write_ghost refills q_out's ring.  split_hi/lo
 * (bf16 [ny-2][nx-2], may be NULL) receive q_out's interior for the next DST,
 * in the layout split_layout (fvx_dst_operand_layout of the plan).  FP64
 * stages: split_hi (may be NULL) receives q_out's interior as doubles
 * [ny-2][nx-2] (the FP64 chain's input, fvx_dst_workspace_f64), split_lo
 * must be NULL and split_layout 0.
 * method: 1 upwind1, 3 upwind3, 4 weno3, 5 weno5, 6 wenoz5, 7 weno7,
 * 8 weno9, 9 minmod, 10 van_leer. */
int fvx_qg_stage_f32(const float* q_stage, const float* q_start, const float* psi_interior, const float* forcing,
                     float* q_out, void* split_hi, void* split_lo, int split_layout, int ny, int nx, double dx,
                     double dy,
                     double beta, double drag, double viscosity, double a, double b, double c, int method,
                     int periodic, int write_ghost, void* stream);
int fvx_qg_stage_f64(const double* q_stage, const double* q_start, const double* psi_interior,
                     const double* forcing, double* q_out, void* split_hi, void* split_lo, int split_layout, int ny, int nx,
                     double dx, double dy, double beta, double drag, double viscosity, double a, double b,
                     double c, int method, int periodic, int write_ghost, void* stream);

/* ---- masked multigrid, PCG, vertical modes -------------------------------- */

/* Preconditioner / coarse-solver callback: z = M rho on ``stream``. */
typedef int (*fvx_precond_fn)(void* ctx, const void* rho, void* z, void* stream);

/* build_multigrid_solver (solvers/multigrid.py:905-1062): FP64 host build of
 * the level hierarchy (masks mean>=0.5, face coefficients, inverse
 * diagonals), uploaded in ``dtype`` (0 float32, 1 float64).  coeff may be
 * NULL (c = 1); n_levels 0 = as many as halving allows (>= 8 cells). */
typedef struct fvx_mg fvx_mg;
int fvx_mg_create(const double* mask, const double* coeff, int ny, int nx, double dx, double dy, double lambda,
                  int n_levels, int n_pre, int n_post, int n_coarse, double omega, int dtype, fvx_mg** out);
int fvx_mg_destroy(fvx_mg* g);
int fvx_mg_num_levels(fvx_mg* g);
/* Level metadata and device arrays (mask, cx, cy, inv_diagonal). */
int fvx_mg_level(fvx_mg* g, int level, int* ny, int* nx, double* dx2, void** mask, void** cx, void** cy,
                 void** inv);
/* MultigridSolver.v_cycle (multigrid.py:808-881); u_in NULL = zero guess. */
int fvx_mg_vcycle(fvx_mg* g, const void* u_in, const void* f, void* u_out, void* stream);
/* MultigridSolver._run_vcycles (multigrid.py:885-897). */
int fvx_mg_solve(fvx_mg* g, const void* f, void* u, int n_cycles, void* stream);
/* _apply_operator (multigrid.py:327-405) at a level. */
int fvx_mg_apply(fvx_mg* g, int level, const void* u, void* out, void* stream);
/* masked_laplacian (solvers/iterative.py:144-191). */
int fvx_masked_laplacian_f32(const float* psi, const float* mask, float* out, int ny, int nx, double dx, double dy,
                             double lambda, void* stream);
int fvx_masked_laplacian_f64(const double* psi, const double* mask, double* out, int ny, int nx, double dx,
                             double dy, double lambda, void* stream);

/* Device-resident PCG on the finest MG operator (solve_cg with
 * make_multigrid_preconditioner, iterative.py:48-136 and
 * preconditioners.py:207-244): FP64 iterate and inner products, work vectors
 * in the MG dtype, 2-norm relative residual checked in FP64.  precond 0 none,
 * 1 one V-cycle, 2 the callback (fn, ctx); flexible selects Polak-Ribiere
 * beta.  info = [iterations, relative residual, converged]. */
typedef struct fvx_pcg fvx_pcg;
int fvx_pcg_create(fvx_mg* g, fvx_pcg** out);
int fvx_pcg_destroy(fvx_pcg* P);
int fvx_pcg_bind_vectors(fvx_pcg* P, void* rho, void* z);
int fvx_pcg_solve(fvx_pcg* P, const void* b, double* x, int max_iter, double rtol, int precond, fvx_precond_fn fn,
                  void* ctx, int flexible, int replace_every, int chunk, double* info, void* stream);
/* The same solve in pieces; fvx_pcg_iterate makes no host synchronisation
 * and may be captured in a CUDA graph. */
int fvx_pcg_begin(fvx_pcg* P, const void* b, double* x, double rtol, int precond, fvx_precond_fn fn, void* ctx,
                  double* bb_out, void* stream);
int fvx_pcg_iterate(fvx_pcg* P, const void* b, double* x, int it0, int niter, int precond, fvx_precond_fn fn,
                    void* ctx, int flexible, int replace_every, void* stream);
int fvx_pcg_status(fvx_pcg* P, double* out3, void* stream);
int fvx_pcg_finish(fvx_pcg* P, const void* b, double* x, double bb, double* rel_out, void* stream);
/* FP64-accumulated inner product (one device scalar). */
int fvx_dot_f32(const float* a, const float* b, long long n, double* part, double* out_dev, void* stream);
int fvx_dot_f64(const double* a, const double* b, long long n, double* part, double* out_dev, void* stream);
/* layer_to_mode / mode_to_layer (vertical/vertical_modes.py:204-263). */
int fvx_layer_mix_f32(const double* C, int nl, const float* in, float* out, long long plane, int batch,
                      void* stream);
int fvx_layer_mix_f64(const double* C, int nl, const double* in, double* out, long long plane, int batch,
                      void* stream);

/* ---- learned coarse-grid preconditioner (no counterpart in finitevolX) ---- */

/* Hybrid cycle: the V-cycle's legs on levels 0..lvl-1 (fused kernels,
 * n_pre, n_post <= 16) with the level-lvl correction from ``coarse`` (NULL =
 * zero), scaled by the energy-optimal omega if ``scale``, followed by
 * n_smooth Jacobi sweeps at level lvl. */
int fvx_mg_vcycle_hybrid(fvx_mg* g, const void* f, void* u_out, int lvl, int n_pre, int n_post, int n_smooth,
                         int scale, fvx_precond_fn coarse, void* ctx, void* stream);
/* Downward leg only: f's restricted residual at level lvl into f_lvl. */
int fvx_mg_restrict_residual(fvx_mg* g, const void* f, int lvl, int n_pre, void* f_lvl, void* stream);
/* Batched MG solves at level lvl, one CTA per right-hand side. */
long long fvx_mg_level_work(fvx_mg* g, int lvl);
int fvx_mg_solve_level_batched(fvx_mg* g, int lvl, int batch, const void* f, void* u, int n_cycles, void* work,
                               void* stream);
/* Multigrid (n_cycles cycles) as the level-lvl solver: an fvx_precond_fn
 * with ctx = the fvx_levelsolve (the exact-coarse-solve comparison). */
typedef struct fvx_levelsolve fvx_levelsolve;
int fvx_levelsolve_create(fvx_mg* g, int lvl, int n_cycles, fvx_levelsolve** out);
int fvx_levelsolve_destroy(fvx_levelsolve* s);
int fvx_levelsolve_coarse(void* ctx, const void* f, void* u, void* stream);
/* The hybrid cycle as an fvx_precond_fn (ctx = the fvx_hybrid object). */
typedef struct fvx_hybrid fvx_hybrid;
int fvx_hybrid_create(fvx_mg* g, int lvl, int n_pre, int n_post, int n_smooth, int scale, fvx_precond_fn coarse,
                      void* ctx, fvx_hybrid** out);
int fvx_hybrid_destroy(fvx_hybrid* h);
int fvx_hybrid_precond(void* ctx, const void* rho, void* z, void* stream);

/* 4-level U-Net (16/16/32/32 channels), BF16 weights, FP32 accumulation:
 * create / parameter IO / forward / backward / Adam train step, and the
 * inference callback fvx_unet_coarse (an fvx_precond_fn, ctx = the net).
 * fvx_unet_io which: 0 parameters, 1 gradient, 2 input x, 3 output y, 4 the
 * last coarse solve's scale pair [s, 1/s]. */
typedef struct fvx_unet fvx_unet;
long long fvx_unet_num_params(void);
int fvx_unet_create(int h, int w, int batch_max, fvx_unet** out);
int fvx_unet_destroy(fvx_unet* n);
int fvx_unet_io(fvx_unet* n, int which, long long offset, long long count, const void* src, void* dst,
                void* stream);
int fvx_unet_sync_params(fvx_unet* n, void* stream);
int fvx_unet_forward(fvx_unet* n, int batch, void* stream);
int fvx_unet_backward(fvx_unet* n, int batch, const float* dy, void* stream);
int fvx_unet_train_step(fvx_unet* n, int batch, const float* target, double lr, double beta1, double beta2,
                        double eps, int step, double* loss_out, void* stream);
int fvx_unet_set_level(fvx_unet* n, const float* mask, const float* logc, double sigma, void* stream);
/* fvx_unet_coarse: one launch per layer.  fvx_unet_coarse_fused: the whole
 * solve (RMS, 8 layers, output scaling) as one cooperative launch with grid
 * barriers between the layers; every barrier wait is bounded
 * (fvx_unet_set_wait_limit, SM cycles) and a wait that ran out shows as
 * FVX_ERR_TIMEOUT in fvx_unet_check (which synchronises and resets the
 * barrier state).  fvx_unet_inject_stall: CTA 0 skips the first barrier
 * (the timeout test). */
int fvx_unet_coarse(void* ctx, const void* f, void* u, void* stream);
int fvx_unet_coarse_fused(void* ctx, const void* f, void* u, void* stream);
int fvx_unet_check(fvx_unet* n);
int fvx_unet_set_wait_limit(fvx_unet* n, long long cycles);
int fvx_unet_inject_stall(fvx_unet* n, int stall);
/* Layer-level kernels (conv3x3 with pool/upsample input, backward, MSE, Adam). */
int fvx_nn_conv_fwd(const float* in, int mode, int batch, int cin, const void* w_bf16, const float* bias,
                    const float* skip, float* out, int cout, int h, int w, int relu, void* stream);
int fvx_nn_conv_bwd(const float* in, int mode, int batch, int cin, const void* w_bf16, const float* dy,
                    const float* y, int cout, int h, int w, int relu, float* g, float* dskip, float* dxin,
                    float* dsrc, float* dw, float* db, float* part, void* stream);
int fvx_nn_conv_bwd_blocks(int batch, int h, int w);
int fvx_nn_mse(const float* pred, const float* target, const float* mask, long long plane, int batch, float* dpred,
               double* loss_dev, double mask_sum, void* stream);
int fvx_nn_adam(float* w, void* w_bf16, const float* grad, float* m, float* v, int n, double lr, double beta1,
                double beta2, double eps, int step, void* stream);
int fvx_nn_to_bf16(const float* src, void* dst, int n, void* stream);

/* ---- QG snapshot planes ------------------------------------------------- */
/* record_snapshot of scripts/qg_1p5_layer.py:514-545 on the device: from
 * the full [ny, nx] q, psi (zero ghost ring), u (U points), v (V points) and
 * relative vorticity z (X points), writes out[7][ny-2][nx-2] = q, psi,
 * eta_scale * psi, U_to_T(u), V_to_T(v), speed, X_to_T(z) (interiors). */
int fvx_qg_snapshot_pack_f32(const float* q, const float* psi, const float* u, const float* v, const float* z,
                             int ny, int nx, double eta_scale, float* out, void* stream);
int fvx_qg_snapshot_pack_f64(const double* q, const double* psi, const double* u, const double* v,
                             const double* z, int ny, int nx, double eta_scale, double* out, void* stream);

/* ---- QG fused-stage tile shape (autotuner) -------------------------------- */
/* cfg 0 = 64x16, 1 = 32x16, 2 = 128x8, 3 = 64x32, 4 = 128x16, 5 = 16x16 cells for (method, dtype 0 FP32 / 1
 * FP64); cfg < 0 returns the number of configurations.  No counterpart in
 * finitevolX (launch configuration). */
int fvx_qg_tile_config(int method, int dtype, int cfg);

/* ---- ensemble of multi-layer QG members ------------------------------------ */
/* Members (n[m]^2 interior, nl[m] <= 3 layers; l2m/m2l row-major nl x nl per
 * member, concatenated; lam: per-mode 1/Rd^2) stepped with rk3_ssp_step
 * (timestepping/explicit_rk.py:74-121) of the per-layer 1.5-layer tendency
 * (scripts/qg_1p5_layer.py:454-487) with psi from the vertical modes
 * (vertical_modes.py:193-263, elliptic.py:390-542).  One persistent
 * work-queue launch per RK stage over every tile of every layer. */
typedef struct fvx_ens fvx_ens;
int fvx_ens_create(int n_members, const int* n, const int* nl, const double* l2m, const double* m2l,
                   const double* lam, const double* dx, const double* dy, const double* dt, double beta, int method,
                   fvx_ens** out);
int fvx_ens_destroy(fvx_ens* e);
int fvx_ens_io(fvx_ens* e, int member, int layer, const void* src, void* dst, void* stream);
int fvx_ens_set_blocks_per_sm(fvx_ens* e, int blocks_per_sm);
int fvx_ens_launches_per_step(fvx_ens* e);
/* FP64-residual refinement passes (0-4, default 1) after the batched DST
 * solves of the weakly screened modes (lambda (n dx)^2 < 2000, batched
 * first in each size group): their psi at FP32 rounding instead of the
 * split chain's ~1e-5, which the velocity differences would amplify past
 * the FP32 step bar; no counterpart in finitevolX, whose solve is FP64. */
int fvx_ens_set_refine(fvx_ens* e, int passes);
int fvx_ens_step(fvx_ens* e, int n_steps, void* stream);

/* ---- diagnostics (operators/diagnostics.py) -------------------------------- */
/* op: 0 kinetic_energy(u,v) :35-73, 1 bernoulli_potential(h,u,v; p0 = g)
 * :76-112, 2 shear_strain(u,v; dx,dy) :184-213, 3 tensor_strain :216-245,
 * 4 qg_potential_vorticity(psi, y; f0, beta, dx, dy, y0) :395-452,
 * 5 potential_vorticity(omega, f, h) :150-181, 6 enstrophy :308-329,
 * 7 potential_enstrophy :332-360, 8 strain_magnitude_squared :248-271,
 * 9 okubo_weiss :274-305, 10 available_potential_energy(h, H; g') :363-392. */
int fvx_diag2d_f32(int op, const float* a, const float* b, const float* c, float* out, int ny, int nx, double p0,
                   double p1, double p2, double p3, double p4, void* stream);
int fvx_diag2d_f64(int op, const double* a, const double* b, const double* c, double* out, int ny, int nx,
                   double p0, double p1, double p2, double p3, double p4, void* stream);
/* total_energy / total_enstrophy (:498-555): scale * sum over the interior
 * of (a + b) (b may be NULL) into a device double, deterministic. */
int fvx_interior_sum_f32(const float* a, const float* b, int ny, int nx, double scale, double* part,
                         unsigned* ticket, double* out_dev, void* stream);
int fvx_interior_sum_f64(const double* a, const double* b, int ny, int nx, double scale, double* part,
                         unsigned* ticket, double* out_dev, void* stream);

/* ---- shallow-water operators ----------------------------------------------- */
/* op 0 Coriolis2D (u, v, f) -> (du, dv) (operators/coriolis.py:34-133);
 * 1-3 Vorticity2D.pv_flux_{energy,enstrophy}_conserving / _arakawa_lamb
 * (q, u, v; alpha) -> (qu, qv) (operators/vorticity.py:120-235);
 * 4-6 MomentumAdvection2D energy / enstrophy / al (u, v) -> (du, dv)
 * (diffusion/momentum.py:108-216); 7 Vorticity2D.potential_vorticity
 * (u, v, h, f) -> q (vorticity.py:60-118).  Masks (bool [Ny][Nx]) may be NULL. */
int fvx_sw2d_f32(int op, const float* a, const float* b, const float* c, const float* d, float* out1, float* out2,
                 int ny, int nx, double dx, double dy, double alpha, const uint8_t* mask_h, const uint8_t* mask_u,
                 const uint8_t* mask_v, const uint8_t* mask_xy, void* stream);
int fvx_sw2d_f64(int op, const double* a, const double* b, const double* c, const double* d, double* out1,
                 double* out2, int ny, int nx, double dx, double dy, double alpha, const uint8_t* mask_h,
                 const uint8_t* mask_u, const uint8_t* mask_v, const uint8_t* mask_xy, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FVX_H */
