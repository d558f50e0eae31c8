// Diagnostics on the Arakawa C-grid (finitevolX operators/diagnostics.py):
// pointwise and 5-point quantities in one kernel with an operator code, and
// FP64 domain integrals over the interior with a deterministic reduction
// (per-block partials summed in block order by the last block to finish).
//
// Stencil conventions (operators/stencils.py:84-187) on the interior
// [1:-1, 1:-1], ghost ring written as zero where the reference returns
// interior(...): diff_x_fwd(h) = h[j,i+1] - h[j,i], diff_x_bwd(h) = h[j,i] -
// h[j,i-1], avg_x_bwd(h) = 0.5 (h[j,i] + h[j,i-1]) (y likewise).
#include "fvx_common.cuh"

namespace fvx {
namespace diag {

enum DiagOp {
  KINETIC_ENERGY = 0,       // kinetic_energy(u, v)                 diagnostics.py:35-73
  BERNOULLI = 1,            // bernoulli_potential(h, u, v, g)       :76-112
  SHEAR_STRAIN = 2,         // shear_strain(u, v, dx, dy)            :184-213
  TENSOR_STRAIN = 3,        // tensor_strain(u, v, dx, dy)           :216-245
  QG_PV = 4,                // qg_potential_vorticity(psi, f0, beta, dx, dy, y, y0)  :395-452
  POTENTIAL_VORTICITY = 5,  // potential_vorticity(omega, f, h)      :150-181 (pointwise)
  ENSTROPHY = 6,            // enstrophy(omega)                      :308-329 (pointwise)
  POTENTIAL_ENSTROPHY = 7,  // potential_enstrophy(q, h)             :332-360 (pointwise)
  STRAIN_MAG2 = 8,          // strain_magnitude_squared(sn, ss)      :248-271 (pointwise)
  OKUBO_WEISS = 9,          // okubo_weiss(sn, ss, omega)            :274-305 (pointwise)
  APE = 10,                 // available_potential_energy(h, H, g')  :363-392 (pointwise)
  N_OPS = 11
};

// p[0..3]: op parameters (g; dx, dy; f0, beta, dx, dy, y0; g').
template <typename T>
__global__ void diag_kernel(int op, const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ c,
                            T* __restrict__ out, int ny, int nx, double p0, double p1, double p2, double p3,
                            double p4) {
  const size_t n = (size_t)ny * nx;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(k / nx), i = (int)(k - (size_t)j * nx);
    const bool inter = j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2;
    T r = T(0);
    switch (op) {
      case KINETIC_ENERGY:
      case BERNOULLI: {  // a = u, b = v (KE); a = h, b = u, c = v (Bernoulli)
        const T* u = op == KINETIC_ENERGY ? a : b;
        const T* v = op == KINETIC_ENERGY ? b : c;
        if (inter) {
          const T u2c = u[k] * u[k], u2w = u[k - 1] * u[k - 1];
          const T v2c = v[k] * v[k], v2s = v[k - nx] * v[k - nx];
          const T ke = T(0.5) * (T(0.5) * (u2c + u2w) + T(0.5) * (v2c + v2s));
          r = op == KINETIC_ENERGY ? ke : ke + T(p0) * a[k];
        }
        break;
      }
      case SHEAR_STRAIN:  // a = u, b = v
        if (inter) r = (b[k + 1] - b[k]) / T(p0) + (a[k + nx] - a[k]) / T(p1);
        break;
      case TENSOR_STRAIN:
        if (inter) r = (a[k] - a[k - 1]) / T(p0) - (b[k] - b[k - nx]) / T(p1);
        break;
      case QG_PV: {  // a = psi, b = y; p = f0, beta, dx, dy, y0
        if (inter) {
          const T dx = T(p2), dy = T(p3);
          const T d2x = ((a[k + 1] - a[k]) - (a[k] - a[k - 1])) / (dx * dx);
          const T d2y = ((a[k + nx] - a[k]) - (a[k] - a[k - nx])) / (dy * dy);
          r = (d2x + d2y) / T(p0) + T(p1) * (b[k] - T(p4)) / T(p0);
        }
        break;
      }
      case POTENTIAL_VORTICITY:  // a = omega, b = f, c = h
        r = c[k] == T(0) ? T(NAN) : (a[k] + b[k]) / c[k];
        break;
      case ENSTROPHY:
        r = T(0.5) * (a[k] * a[k]);
        break;
      case POTENTIAL_ENSTROPHY:  // a = q, b = h
        r = T(0.5) * (a[k] * a[k]) * b[k];
        break;
      case STRAIN_MAG2:
        r = a[k] * a[k] + b[k] * b[k];
        break;
      case OKUBO_WEISS:
        r = a[k] * a[k] + b[k] * b[k] - c[k] * c[k];
        break;
      case APE: {
        const T eta = a[k] - b[k];
        r = T(0.5) * T(p0) * (eta * eta);
        break;
      }
    }
    out[k] = r;
  }
}

constexpr int kSumBlocks = 296;

DEV double dblock_sum(double v) {
  __shared__ double sh[32];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
  if (w == 0)
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  return v;
}

// out = scale * sum over the interior of (a + b) (b may be NULL), FP64.
template <typename T>
__global__ void interior_sum_kernel(const T* __restrict__ a, const T* __restrict__ b, int ny, int nx, double scale,
                                    double* part, unsigned* ticket, double* out) {
  const size_t n = (size_t)(ny - 2) * (nx - 2);
  double acc = 0.0;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(k / (nx - 2)) + 1, i = (int)(k % (nx - 2)) + 1;
    const size_t g = (size_t)j * nx + i;
    acc += b ? (double)(a[g] + b[g]) : (double)a[g];
  }
  acc = dblock_sum(acc);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = acc;
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double v = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) v += ((volatile double*)part)[k];
    v = dblock_sum(v);
    if (threadIdx.x == 0) {
      *out = v * scale;
      *ticket = 0u;
    }
  }
}

// The seven interior planes of a QG snapshot (scripts/qg_1p5_layer.py:514-545,
// record_snapshot): q, psi, eta = eta_scale psi, U_to_T(u), V_to_T(v),
// speed = sqrt(u_T^2 + v_T^2), X_to_T(zeta) -- the interpolation formulas of
// operators/interpolation.py (0.5 (c + w), 0.5 (c + s), 0.25 (c + s + w + sw))
// on the full [ny][nx] arrays, written to out[7][ny-2][nx-2] in one pass.
template <typename T>
__global__ void snapshot_pack_kernel(const T* __restrict__ q, const T* __restrict__ psi, const T* __restrict__ u,
                                     const T* __restrict__ v, const T* __restrict__ z, int ny, int nx, T eta_scale,
                                     T* __restrict__ out) {
  const int nyi = ny - 2, nxi = nx - 2;
  const size_t plane = (size_t)nyi * nxi;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < plane; k += (size_t)gridDim.x * blockDim.x) {
    const int jj = (int)(k / nxi), ii = (int)(k - (size_t)jj * nxi);
    const size_t g = (size_t)(jj + 1) * nx + (ii + 1);
    const T uT = T(0.5) * (u[g] + u[g - 1]);
    const T vT = T(0.5) * (v[g] + v[g - nx]);
    out[k] = q[g];
    out[plane + k] = psi[g];
    out[2 * plane + k] = eta_scale * psi[g];
    out[3 * plane + k] = uT;
    out[4 * plane + k] = vT;
    out[5 * plane + k] = sqrt(uT * uT + vT * vT);
    out[6 * plane + k] = T(0.25) * (z[g] + z[g - nx] + z[g - 1] + z[g - nx - 1]);
  }
}

static int grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace diag
}  // namespace fvx

using namespace fvx;
using namespace fvx::diag;

#define FVX_DEF_DIAG(SFX, T)                                                                                     \
  extern "C" int fvx_diag2d_##SFX(int op, const T* a, const T* b, const T* c, T* out, int ny, int nx, double p0, \
                                  double p1, double p2, double p3, double p4, void* stream) {                   \
    if (op < 0 || op >= N_OPS) return FVX_ERR_METHOD;                                                            \
    if (!a || !out) return FVX_ERR_ARG;                                                                          \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                                  \
    const bool need_b = op != ENSTROPHY;                                                                         \
    const bool need_c = op == BERNOULLI || op == POTENTIAL_VORTICITY || op == OKUBO_WEISS;                       \
    if ((need_b && !b) || (need_c && !c)) return FVX_ERR_ARG;                                                    \
    diag_kernel<T><<<grid_for((size_t)ny * nx), 256, 0, fvx_stream(stream)>>>(op, a, b, c, out, ny, nx, p0, p1,  \
                                                                              p2, p3, p4);                       \
    return fvx_cuda_status();                                                                                    \
  }                                                                                                              \
  /* scale * sum_interior(a + b) into out_dev (FP64); part: >= 296 doubles,                                      \
     ticket: one zeroed unsigned (left zeroed). */                                                               \
  extern "C" int fvx_interior_sum_##SFX(const T* a, const T* b, int ny, int nx, double scale, double* part,      \
                                        unsigned* ticket, double* out_dev, void* stream) {                      \
    if (!a || !part || !ticket || !out_dev) return FVX_ERR_ARG;                                                  \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                                  \
    interior_sum_kernel<T><<<kSumBlocks, 256, 0, fvx_stream(stream)>>>(a, b, ny, nx, scale, part, ticket,        \
                                                                       out_dev);                                 \
    return fvx_cuda_status();                                                                                    \
  }

#define FVX_DEF_SNAP(SFX, T)                                                                                  \
  extern "C" int fvx_qg_snapshot_pack_##SFX(const T* q, const T* psi, const T* u, const T* v, const T* z, int ny, \
                                            int nx, double eta_scale, T* out, void* stream) {                   \
    if (!q || !psi || !u || !v || !z || !out) return FVX_ERR_ARG;                                              \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                                \
    snapshot_pack_kernel<T><<<grid_for((size_t)(ny - 2) * (nx - 2)), 256, 0, fvx_stream(stream)>>>(            \
        q, psi, u, v, z, ny, nx, (T)eta_scale, out);                                                           \
    return fvx_cuda_status();                                                                                  \
  }

FVX_DEF_SNAP(f32, float)
FVX_DEF_SNAP(f64, double)

FVX_DEF_DIAG(f32, float)
FVX_DEF_DIAG(f64, double)
