// Capacitance-matrix correction for masked Helmholtz solves on a rectangular
// spectral solver (finitevolX solvers/elliptic.py:146-183, which builds
// spectraldiffx's CapacitanceSolver; algorithm of Buzbee, Golub and Nielson
// as docs/elliptic_solvers.md states it).
//
// With L the rectangular operator, B the N_b inner-boundary points and
// C = (L^-1 E_B)[B, :] (N_b x N_b, built once), the masked solution is
//   u = L^-1 f,  alpha = C^-1 u[B],  psi = u - L^-1 E_B alpha
//                                        = L^-1 (f - E_B alpha),
// which vanishes on B.  This file holds the step between the two
// rectangular solves: rhs2 = f, then rhs2[B] -= C^-1 u[B] (FP64 sums).  The
// second solve replaces the reference's dense N_b x (Ny Nx) Green's-function
// product, so no O(N_b Ny Nx) matrix is stored.
#include "fvx_common.cuh"

namespace fvx {
namespace cap {

template <typename T>
__global__ void copy_kernel(const T* __restrict__ f, T* __restrict__ out, long long n) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = f[k];
}

// One warp per boundary row k: alpha_k = sum_l Cinv[k][l] u[idx[l]], then
// out[idx[k]] -= alpha_k (indices are distinct, so rows never collide).
template <typename T>
__global__ void correct_kernel(const T* __restrict__ u, const double* __restrict__ cinv,
                               const long long* __restrict__ idx, int nb, T* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < nb; k += warps) {
    const double* row = cinv + (long long)k * nb;
    double acc = 0.0;
    for (int l = lane; l < nb; l += 32) acc = fma(row[l], (double)u[idx[l]], acc);
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[idx[k]] = (T)((double)out[idx[k]] - acc);
  }
}

static int grid_for(long long n, int per) {
  long long b = (n + per - 1) / per;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace cap
}  // namespace fvx

using namespace fvx::cap;

#define FVX_DEF_CAP(SFX, T)                                                                                    \
  extern "C" int fvx_capacitance_rhs_##SFX(const T* f, const T* u, const double* cinv, const long long* idx,  \
                                           int nb, long long n, T* out, void* stream) {                       \
    if (!f || !u || !cinv || !idx || !out) return FVX_ERR_ARG;                                                 \
    if (nb < 1 || n < 1) return FVX_ERR_SHAPE;                                                                 \
    cudaStream_t st = fvx_stream(stream);                                                                      \
    if (out != f) copy_kernel<T><<<grid_for(n, 256), 256, 0, st>>>(f, out, n);                                 \
    correct_kernel<T><<<grid_for((long long)nb * 32, 256), 256, 0, st>>>(u, cinv, idx, nb, out);              \
    return fvx_cuda_status();                                                                                  \
  }

FVX_DEF_CAP(f32, float)
FVX_DEF_CAP(f64, double)
