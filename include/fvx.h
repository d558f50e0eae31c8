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
/* Reads the plan's device error flag (7 if a bounded wait gave up); syncs. */
int fvx_dst_plan_check(fvx_dst_plan* plan, void* stream);
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
 * by fvx_qg_stage_f32's split outputs); fvx_dst_workspace returns it. */
int fvx_dst_solve_presplit_f32(fvx_dst_plan* plan, float* psi, long long psi_bstride, long long psi_ld, int batch,
                               void* stream);
int fvx_dst_workspace(fvx_dst_plan* plan, void** w1_hi, void** w1_lo);
/* One product of the chain on the current workspaces (timing only). */
int fvx_dst_gemm_step(fvx_dst_plan* plan, int which, int batch, void* stream);

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

/* ---- fused QG RK stage ---------------------------------------------------- */

/* One Runge-Kutta stage of the QG 1.5-layer PV equation
 * (scripts/qg_1p5_layer.py:454-487 inside rk3_ssp_step,
 * timestepping/explicit_rk.py:74-121): q_out = a*q_start + b*q_stage + c*rhs
 * with rhs = Advection2D(BC(q_stage), u, v) - beta*V_to_T(v) + forcing
 * - drag*laplacian(psi) + viscosity*laplacian(BC(q_stage)), (u, v) the
 * geostrophic velocity of psi_interior (zero outside).  periodic: 1 periodic
 * ghost ring, 0 zero ring.  write_ghost refills q_out's ring.  split_hi/lo
 * (bf16 [ny-2][nx-2], may be NULL) receive q_out's interior for the next DST.
 * method: 1 upwind1, 3 upwind3, 4 weno3, 5 weno5, 6 wenoz5, 7 weno7,
 * 8 weno9, 9 minmod, 10 van_leer. */
int fvx_qg_stage_f32(const float* q_stage, const float* q_start, const float* psi_interior, const float* forcing,
                     float* q_out, void* split_hi, void* split_lo, int ny, int nx, double dx, double dy,
                     double beta, double drag, double viscosity, double a, double b, double c, int method,
                     int periodic, int write_ghost, void* stream);
int fvx_qg_stage_f64(const double* q_stage, const double* q_start, const double* psi_interior,
                     const double* forcing, double* q_out, void* split_hi, void* split_lo, int ny, int nx,
                     double dx, double dy, double beta, double drag, double viscosity, double a, double b,
                     double c, int method, int periodic, int write_ghost, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FVX_H */
