// Fused QG 1.5-layer RK stage (scripts/qg_1p5_layer.py:115-145, 420-497 with
// timestepping/explicit_rk.py:74-121).  One kernel per Runge-Kutta stage:
//
//   q_b   = BC(q_s)               periodic wrap (boundary.py:52-75) or zero ring
//   X     = interior(T_to_X(psi)) psi from the DST solve, zero ghost ring
//   u, v  = -diff_y_X_to_U(X), diff_x_X_to_V(X)
//   rhs   = Advection2D(q_b, u, v, scheme)              [2:-2, 2:-2]
//         + (-beta * V_to_T(v))                           [1:-1, 1:-1]
//         + forcing - drag * laplacian(psi) + nu * laplacian(q_b)
//   q_out = a * q_n + b * q_s + c * rhs                  (c = stage weight * dt)
//
// q_b is never materialised (ghost values come from wrap-around tile loads),
// face fluxes and velocities stay in shared memory, and the kernel writes
// q_out (interior, plus the ghost ring on the last stage) and optionally the
// bf16 hi/lo split of q_out's interior that the next DST product reads.
#include "qg_stage.cuh"

namespace fvx {
namespace qg {

template <typename T, int S, int TX, int TY>
static int launch_t(const StageArgs& a, cudaStream_t st) {
  size_t sm = smem_bytes<T, S, TX, TY>();
  static fvx_once_per_device attr;
  if (fvx_once_on_device(attr, [sm] { return fvx_set_max_smem(stage_kernel<T, S, TX, TY>, (int)sm); }))
    return FVX_ERR_CUDA;
  const TileSplit ts = tile_split<S, TX, TY>(a.ny, a.nx);
  if (fvx_launch_pdl(stage_kernel<T, S, TX, TY>, dim3(ts.ntx * ts.nty), dim3(THREADS), sm, st, a, ts) !=
      cudaSuccess)
    return FVX_ERR_CUDA;
  return fvx_cuda_status();
}

// Tile configuration per (scheme, dtype), set by the autotuner.
static int g_tile_cfg[32][2] = {};

template <typename T, int S>
static int launch(const StageArgs& a, cudaStream_t st) {
  switch (g_tile_cfg[S][sizeof(T) == 8]) {
    case 1: return launch_t<T, S, kTileTX[1], kTileTY[1]>(a, st);
    case 2: return launch_t<T, S, kTileTX[2], kTileTY[2]>(a, st);
    case 3: return launch_t<T, S, kTileTX[3], kTileTY[3]>(a, st);
    case 4: return launch_t<T, S, kTileTX[4], kTileTY[4]>(a, st);
    case 5: return launch_t<T, S, kTileTX[5], kTileTY[5]>(a, st);
    default: return launch_t<T, S, kTileTX[0], kTileTY[0]>(a, st);
  }
}

template <typename T>
static int dispatch(int method, const StageArgs& a, cudaStream_t st) {
  switch (method) {
    case FVX_UPWIND1: return launch<T, FVX_UPWIND1>(a, st);
    case FVX_UPWIND3: return launch<T, FVX_UPWIND3>(a, st);
    case FVX_WENO3: return launch<T, FVX_WENO3>(a, st);
    case FVX_WENO5: return launch<T, FVX_WENO5>(a, st);
    case FVX_WENOZ5: return launch<T, FVX_WENOZ5>(a, st);
    case FVX_WENO7: return launch<T, FVX_WENO7>(a, st);
    case FVX_WENO9: return launch<T, FVX_WENO9>(a, st);
    case FVX_VAN_LEER: return launch<T, FVX_VAN_LEER>(a, st);
    case FVX_MINMOD: return launch<T, FVX_MINMOD>(a, st);
    default: return FVX_ERR_METHOD;
  }
}

}  // namespace qg
}  // namespace fvx

using namespace fvx;

#define FVX_DEF_QG(SFX, T)                                                                                   \
  extern "C" int fvx_qg_stage_##SFX(const T* q_stage, const T* q_start, const T* psi_interior,             \
                                    const T* forcing, T* q_out, void* split_hi, void* split_lo,              \
                                    int split_layout, int ny, int nx,                                        \
                                    double dx, double dy, double beta, double drag, double viscosity,       \
                                    double a, double b, double c, int method, int periodic, int write_ghost, \
                                    void* stream) {                                                          \
    if (!q_stage || !psi_interior || !q_out) return FVX_ERR_ARG;                                             \
    if (sizeof(T) == 8 ? (split_lo != nullptr || (split_hi && split_layout)) /* FP64: hi = interior copy */  \
                       : ((split_hi == nullptr) != (split_lo == nullptr)))                                      \
      return FVX_ERR_ARG;                                                                                    \
    if (ny < 6 || nx < 6) return FVX_ERR_SHAPE;                                                              \
    qg::StageArgs A;                                                                                         \
    A.qs = q_stage; A.qn = q_start; A.psi = psi_interior; A.forcing = forcing; A.out = q_out;              \
    A.split_hi = (__nv_bfloat16*)split_hi; A.split_lo = (__nv_bfloat16*)split_lo;                          \
    A.split_layout = split_layout;                                                                           \
    A.ny = ny; A.nx = nx; A.a = a; A.b = b; A.c = c; A.dx = dx; A.dy = dy; A.beta = beta;                    \
    A.drag = drag; A.visc = viscosity; A.periodic = periodic; A.write_ghost = write_ghost;                   \
    return qg::dispatch<T>(method, A, fvx_stream(stream));                                                   \
  }

FVX_DEF_QG(f32, float)
FVX_DEF_QG(f64, double)

// Tile shape of the fused stage kernel for one scheme and dtype (0 FP32, 1
// FP64): cfg 0 = 64x16, 1 = 32x16, 2 = 128x8, 3 = 64x32, 4 = 128x16, 5 = 16x16
// cells.  Returns the number of
// configurations when cfg < 0 (and changes nothing).
extern "C" int fvx_qg_tile_config(int method, int dtype, int cfg) {
  if (cfg < 0) return qg::kTileConfigs;
  if (method < 0 || method >= 32 || dtype < 0 || dtype > 1 || cfg >= qg::kTileConfigs) return FVX_ERR_ARG;
  qg::g_tile_cfg[method][dtype] = cfg;
  return FVX_OK;
}
