// Stencil operators on the Arakawa C-grid: advection (all finitevolX
// schemes, with mask-aware tier dispatch), face fluxes, C-grid differences
// and interpolations, Arakawa Jacobian, harmonic / biharmonic diffusion and
// the periodic ghost-ring fill.  FP32 and FP64 instantiations of each.
#include "recon.cuh"

namespace fvx {

// ===========================================================================
// Advection: fused face-flux + flux divergence, one smem tile per CTA.
// Restates Advection2D.__call__ (advection/advection.py:329-420):
//   out[2:-2,2:-2] = -((fe[j,i]-fe[j,i-1])/dx + (fn[j,i]-fn[j-1,i])/dy),
//   zero elsewhere, then * mask.h when a mask is given.
// Masked dispatchable methods pick, per face, the reconstruction of the tier
// of the upwind cell (upwind_flux, advection/flux.py:221-253).
// ===========================================================================

constexpr int ATX = 64;   // output tile width (cells)
constexpr int ATY = 16;   // output tile height
constexpr int AH = 5;     // halo covering WENO9 (face i reads i-4 .. i+5)
constexpr int ATHREADS = 256;

// tier byte: bits 0-1 x-tier, bits 2-3 y-tier; 0 none, 1 -> s=2, 2 -> s=4, 3 -> s=6
template <typename T, int S4, int S6>
DEV T tiered_face(const T* p, int st, int i, int N, bool pos, int code) {
  if (code == 0) return T(0);
  if (code == 1) return pos ? p[0] : p[st];  // upwind1
  if (code == 3 && S6 >= 0) return face_value<T, (S6 >= 0 ? S6 : 0)>(p, st, i, N, pos);
  return face_value<T, S4>(p, st, i, N, pos);
}

// One load phase per tile: h (tile + halo), u on the tile's east faces and v
// on its north faces land in one flat shared buffer, four loads in flight
// per thread (eight raise the FP32 kernels' registers from 31 to 59); the
// face fluxes then overwrite u and v in place.
// FP64 WENO7 / WENO9 faces are evaluated through a call: inlined into the
// face loops, the compiler hoists the schemes' ~84 table coefficients out of
// the loop into registers (FP64 WENO7: 134 registers, or spills under a cap
// of three CTAs per SM); behind the call they stay constant-bank operands
// (56-60 registers, no spills).  FP32 inlined needs 39 registers and runs
// faster than through the call.
template <typename T, int S>
struct AdvFaceCall {
  static constexpr bool v = sizeof(T) == 8 && (S == FVX_WENO7 || S == FVX_WENO9);
};
template <typename T, int S>
__noinline__ __device__ T face_value_call(const T* p, int st, int i, int N, bool pos) {
  return face_value<T, S>(p, st, i, N, pos);
}
template <typename T, int S>
DEV T adv_face(const T* p, int st, int i, int N, bool pos) {
  if constexpr (AdvFaceCall<T, S>::v) return face_value_call<T, S>(p, st, i, N, pos);
  else return face_value<T, S>(p, st, i, N, pos);
}
template <typename T, int S, int S4, int S6, bool MASKED>
__global__ void __launch_bounds__(ATHREADS)
advect_tile_kernel(const T* __restrict__ h, const T* __restrict__ u, const T* __restrict__ v,
                   T* __restrict__ out, int ny, int nx, T dx, T dy,
                   const uint8_t* __restrict__ tiers, const uint8_t* __restrict__ mh) {
  constexpr int HW = ATX + 2 * AH, HH = ATY + 2 * AH;
  constexpr int NH = HH * HW, NU = ATY * (ATX + 1), NV = (ATY + 1) * ATX, NTOT = NH + NU + NV;
  constexpr int U = 4;
  __shared__ T tl[NTOT];
  __shared__ uint8_t tx_[ATY][ATX + 2];
  __shared__ uint8_t ty_[ATY + 2][ATX];
  T* hs = tl;             // [HH][HW], origin (y0 - AH, x0 - AH)
  T* fe = tl + NH;        // [ATY][ATX + 1]: u on east faces, then the x flux
  T* fn = tl + NH + NU;   // [ATY + 1][ATX]: v on north faces, then the y flux
  const int x0 = blockIdx.x * ATX, y0 = blockIdx.y * ATY;
  const int tid = threadIdx.x;
  for (int k0 = tid; k0 < NTOT; k0 += U * ATHREADS) {
    T val[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
      int k = k0 + q * ATHREADS;
      T x = T(0);
      if (k < NH) {
        const int ly = k / HW, lx = k - ly * HW;
        const int gy = y0 - AH + ly, gx = x0 - AH + lx;
        if (gy >= 0 && gy < ny && gx >= 0 && gx < nx) x = h[(size_t)gy * nx + gx];
      } else if (k < NH + NU) {
        k -= NH;
        const int ly = k / (ATX + 1), lf = k - ly * (ATX + 1);
        const int gj = y0 + ly, gi = x0 - 1 + lf;
        if (gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2) x = u[(size_t)gj * nx + gi];
      } else if (k < NTOT) {
        k -= NH + NU;
        const int lf = k / ATX, lx = k - lf * ATX;
        const int gj = y0 - 1 + lf, gi = x0 + lx;
        if (gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2) x = v[(size_t)gj * nx + gi];
      }
      val[q] = x;
    }
#pragma unroll
    for (int q = 0; q < U; ++q)
      if (k0 + q * ATHREADS < NTOT) tl[k0 + q * ATHREADS] = val[q];
  }
  if (MASKED) {
    for (int k = tid; k < ATY * (ATX + 2); k += ATHREADS) {
      int ly = k / (ATX + 2), lx = k % (ATX + 2);
      int gy = y0 + ly, gx = x0 - 1 + lx;
      tx_[ly][lx] = (gy < ny && gx >= 0 && gx < nx) ? (tiers[(size_t)gy * nx + gx] & 3) : 0;
    }
    for (int k = tid; k < (ATY + 2) * ATX; k += ATHREADS) {
      int ly = k / ATX, lx = k % ATX;
      int gy = y0 - 1 + ly, gx = x0 + lx;
      ty_[ly][lx] = (gy >= 0 && gy < ny && gx < nx) ? ((tiers[(size_t)gy * nx + gx] >> 2) & 3) : 0;
    }
  }
  __syncthreads();
  // Face fluxes, overwriting u / v in place.  East face (ly, lf) is the
  // face between cells x0-2+lf and x0-1+lf of row y0+ly; north face (lf, lx)
  // the one between rows y0-2+lf and y0-1+lf of column x0+lx.  Each trip of
  // the first loop takes cell (y0+ly, x0+lx)'s east and north faces (two
  // independent reconstructions; ATY x ATX / ATHREADS whole trips), the
  // second the tile's west-most east faces and south-most north faces.
  auto east = [&](int ly, int lf) -> T {
    const int gj = y0 + ly, gi = x0 - 1 + lf;
    if (!(gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2)) return T(0);
    const T uu = fe[ly * (ATX + 1) + lf];
    const bool pos = uu >= T(0);
    const T* p = &hs[(ly + AH) * HW + lf - 1 + AH];
    T hf;
    if (MASKED) hf = tiered_face<T, S4, S6>(p, 1, gi, nx, pos, pos ? tx_[ly][lf] : tx_[ly][lf + 1]);
    else hf = adv_face<T, S>(p, 1, gi, nx, pos);
    return hf * uu;
  };
  auto north = [&](int lf, int lx) -> T {
    const int gj = y0 - 1 + lf, gi = x0 + lx;
    if (!(gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2)) return T(0);
    const T vv = fn[lf * ATX + lx];
    const bool pos = vv >= T(0);
    const T* p = &hs[(lf - 1 + AH) * HW + lx + AH];
    T hf;
    if (MASKED) hf = tiered_face<T, S4, S6>(p, HW, gj, ny, pos, pos ? ty_[lf][lx] : ty_[lf + 1][lx]);
    else hf = adv_face<T, S>(p, HW, gj, ny, pos);
    return hf * vv;
  };
  static_assert((ATY * ATX) % ATHREADS == 0, "whole trips over the tile's cells");
#pragma unroll 1
  for (int k = tid; k < ATY * ATX; k += ATHREADS) {
    const int ly = k / ATX, lx = k - ly * ATX;
    const T a = east(ly, lx + 1), b = north(ly + 1, lx);
    fe[ly * (ATX + 1) + lx + 1] = a;
    fn[(ly + 1) * ATX + lx] = b;
  }
  for (int k = tid; k < ATY + ATX; k += ATHREADS) {
    if (k < ATY) fe[k * (ATX + 1)] = east(k, 0);
    else fn[k - ATY] = north(0, k - ATY);
  }
  __syncthreads();
  for (int k = tid; k < ATY * ATX; k += ATHREADS) {
    int ly = k / ATX, lx = k % ATX;
    int gj = y0 + ly, gi = x0 + lx;
    if (gj >= ny || gi >= nx) continue;
    T r = T(0);
    if (gj >= 2 && gj <= ny - 3 && gi >= 2 && gi <= nx - 3)
      r = -((fe[ly * (ATX + 1) + lx + 1] - fe[ly * (ATX + 1) + lx]) / dx +
            (fn[(ly + 1) * ATX + lx] - fn[ly * ATX + lx]) / dy);
    if (MASKED || mh != nullptr) r = r * T(mh[(size_t)gj * nx + gi]);
    out[(size_t)gj * nx + gi] = r;
  }
}

// ---------------------------------------------------------------------------
// Face fluxes only (uv_center_flux / Reconstruction2D.<m>_x/_y and the
// unfused reference-structured path): one thread per face, global loads.
// ---------------------------------------------------------------------------
template <typename T, int S, int S4, int S6, bool MASKED>
__global__ void face_flux_kernel(const T* __restrict__ h, const T* __restrict__ u,
                                 const T* __restrict__ v, T* __restrict__ fe, T* __restrict__ fn,
                                 int ny, int nx, const uint8_t* __restrict__ tiers) {
  int gi = blockIdx.x * blockDim.x + threadIdx.x;
  int gj = blockIdx.y * blockDim.y + threadIdx.y;
  if (gi >= nx || gj >= ny) return;
  size_t c = (size_t)gj * nx + gi;
  T fx = T(0), fy = T(0);
  if (gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2) {
    T uu = u[c];
    bool pos = uu >= T(0);
    T hf = MASKED ? tiered_face<T, S4, S6>(h + c, 1, gi, nx, pos, tiers[pos ? c : c + 1] & 3)
                  : face_value<T, S>(h + c, 1, gi, nx, pos);
    fx = hf * uu;
    T vv = v[c];
    bool pv = vv >= T(0);
    T hv = MASKED ? tiered_face<T, S4, S6>(h + c, nx, gj, ny, pv, (tiers[pv ? c : c + nx] >> 2) & 3)
                  : face_value<T, S>(h + c, nx, gj, ny, pv);
    fy = hv * vv;
  }
  if (fe) fe[c] = fx;
  if (fn) fn[c] = fy;
}

template <typename T>
__global__ void flux_divergence_kernel(const T* __restrict__ fe, const T* __restrict__ fn,
                                       T* __restrict__ out, int ny, int nx, T dx, T dy,
                                       const uint8_t* __restrict__ mh) {
  int gi = blockIdx.x * blockDim.x + threadIdx.x;
  int gj = blockIdx.y * blockDim.y + threadIdx.y;
  if (gi >= nx || gj >= ny) return;
  size_t c = (size_t)gj * nx + gi;
  T r = T(0);
  if (gj >= 2 && gj <= ny - 3 && gi >= 2 && gi <= nx - 3)
    r = -((fe[c] - fe[c - 1]) / dx + (fn[c] - fn[c - nx]) / dy);
  if (mh) r = r * T(mh[c]);
  out[c] = r;
}

// ===========================================================================
// C-grid differences and interpolations (operators/difference.py:165-520,
// interpolation.py:104-275, stencils.py:84-184, 347-510).  Output written to
// the interior [1:-1,1:-1], ghost ring zero, optional output-stagger mask.
// ===========================================================================
enum CgridOp {
  OP_DX_T2U = 0, OP_DY_T2V, OP_DY_U2X, OP_DX_V2X, OP_DY_X2U, OP_DX_X2V, OP_DX_U2T, OP_DY_V2T,
  OP_LAPLACIAN, OP_DIVERGENCE, OP_CURL, OP_GRAD_PERP,
  OP_T2U = 16, OP_T2V, OP_T2X, OP_X2U, OP_X2V, OP_U2T, OP_V2T, OP_X2T, OP_U2X, OP_V2X, OP_U2V, OP_V2U,
};

template <typename T>
__global__ void cgrid_op_kernel(int op, const T* __restrict__ a, const T* __restrict__ b,
                                T* __restrict__ out, T* __restrict__ out2, int ny, int nx, T dx, T dy,
                                const uint8_t* __restrict__ m1, const uint8_t* __restrict__ m2) {
  int gi = blockIdx.x * blockDim.x + threadIdx.x;
  int gj = blockIdx.y * blockDim.y + threadIdx.y;
  if (gi >= nx || gj >= ny) return;
  size_t c = (size_t)gj * nx + gi;
  bool inner = gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2;
  T r = T(0), r2 = T(0);
  if (inner) {
    const T* A = a + c;
    auto E = [&](const T* p) { return p[1]; };
    auto W = [&](const T* p) { return p[-1]; };
    auto N = [&](const T* p) { return p[nx]; };
    auto Sd = [&](const T* p) { return p[-nx]; };
    switch (op) {
      case OP_DX_T2U: case OP_DX_V2X: r = (E(A) - A[0]) / dx; break;
      case OP_DY_T2V: case OP_DY_U2X: r = (N(A) - A[0]) / dy; break;
      case OP_DY_X2U: case OP_DY_V2T: r = (A[0] - Sd(A)) / dy; break;
      case OP_DX_X2V: case OP_DX_U2T: r = (A[0] - W(A)) / dx; break;
      case OP_LAPLACIAN: {
        T d2x = ((E(A) - A[0]) - (A[0] - W(A))) / (dx * dx);
        T d2y = ((N(A) - A[0]) - (A[0] - Sd(A))) / (dy * dy);
        r = d2x + d2y;
        break;
      }
      case OP_DIVERGENCE: {
        const T* B = b + c;
        r = (A[0] - W(A)) / dx + (B[0] - Sd(B)) / dy;
        break;
      }
      case OP_CURL: {
        const T* B = b + c;  // a = u, b = v
        r = (E(B) - B[0]) / dx - (N(A) - A[0]) / dy;
        break;
      }
      case OP_GRAD_PERP: {
        r = -(A[nx] + A[nx + 1] - A[-nx] - A[-nx + 1]) / (T(4) * dy);
        r2 = (A[1] + A[nx + 1] - A[-1] - A[nx - 1]) / (T(4) * dx);
        break;
      }
      case OP_T2U: case OP_V2X: r = T(0.5) * (A[0] + E(A)); break;
      case OP_T2V: case OP_U2X: r = T(0.5) * (A[0] + N(A)); break;
      case OP_T2X: r = T(0.25) * (A[0] + E(A) + N(A) + A[nx + 1]); break;
      case OP_X2U: case OP_V2T: r = T(0.5) * (A[0] + Sd(A)); break;
      case OP_X2V: case OP_U2T: r = T(0.5) * (A[0] + W(A)); break;
      case OP_X2T: r = T(0.25) * (A[0] + Sd(A) + W(A) + A[-nx - 1]); break;
      case OP_U2V: r = T(0.25) * (A[0] + N(A) + W(A) + A[nx - 1]); break;
      case OP_V2U: r = T(0.25) * (A[0] + Sd(A) + E(A) + A[-nx + 1]); break;
      default: break;
    }
  }
  if (m1) r = r * T(m1[c]);
  out[c] = r;
  if (op == OP_GRAD_PERP) {
    if (m2) r2 = r2 * T(m2[c]);
    out2[c] = r2;
  }
}

// ===========================================================================
// Arakawa Jacobian (operators/jacobian.py:106-131): out [B, Ny-2, Nx-2].
// ===========================================================================
// A thread per output column walking kJacRows rows with a 3 x 3 window of f
// and g in registers (three new values of each per row instead of eight):
// the warp's loads of a row are consecutive columns.  Each output keeps the
// reference's three-form expression and operand order.
constexpr int kJacCols = 128, kJacRows = 16;
template <typename T>
__global__ void __launch_bounds__(kJacCols)
jacobian_kernel(const T* __restrict__ f, const T* __restrict__ g, T* __restrict__ out, int ny, int nx, T scale) {
  const int i = blockIdx.x * kJacCols + threadIdx.x;  // output column 0..nx-3
  const int j0 = blockIdx.y * kJacRows;               // first output row
  const int b = blockIdx.z;
  if (i >= nx - 2 || j0 >= ny - 2) return;
  const int j1 = min(j0 + kJacRows, ny - 2);
  // padded row j0 + r, columns i .. i + 2: window rows a (top), m (middle), c (bottom)
  const T* F = f + (size_t)b * ny * nx + (size_t)j0 * nx + i;
  const T* G = g + (size_t)b * ny * nx + (size_t)j0 * nx + i;
  T fa0 = ldg(F), fa1 = ldg(F + 1), fa2 = ldg(F + 2), ga0 = ldg(G), ga1 = ldg(G + 1), ga2 = ldg(G + 2);
  F += nx;
  G += nx;
  T fm0 = ldg(F), fm1 = ldg(F + 1), fm2 = ldg(F + 2), gm0 = ldg(G), gm1 = ldg(G + 1), gm2 = ldg(G + 2);
  T* o = out + (size_t)b * (ny - 2) * (nx - 2) + (size_t)j0 * (nx - 2) + i;
#pragma unroll 4
  for (int j = j0; j < j1; ++j) {
    F += nx;
    G += nx;
    const T fc0 = ldg(F), fc1 = ldg(F + 1), fc2 = ldg(F + 2), gc0 = ldg(G), gc1 = ldg(G + 1), gc2 = ldg(G + 2);
    // f_(dj, di): dj = -1, 0, 1 -> a, m, c; di = -1, 0, 1 -> 0, 1, 2
    const T Jpp = (fm2 - fm0) * (gc1 - ga1) - (fc1 - fa1) * (gm2 - gm0);
    const T Jpx = fm2 * (gc2 - ga2) - fm0 * (gc0 - ga0) - fc1 * (gc2 - gc0) + fa1 * (ga2 - ga0);
    const T Jxp = gc1 * (fc2 - fc0) - ga1 * (fa2 - fa0) - gm2 * (fc2 - fa2) + gm0 * (fc0 - fa0);
    *o = (Jpp + Jpx + Jxp) * scale;  // scale = 1 / (12 dx dy)
    o += nx - 2;
    fa0 = fm0; fa1 = fm1; fa2 = fm2; ga0 = gm0; ga1 = gm1; ga2 = gm2;
    fm0 = fc0; fm1 = fc1; fm2 = fc2; gm0 = gc0; gm1 = gc1; gm2 = gc2;
  }
}

// ===========================================================================
// Diffusion (diffusion/diffusion.py:120-205).  flux_x lives on faces
// i = 1..Nx-3 (east wall face stays 0), flux_y on j = 1..Ny-3.
// ===========================================================================
template <typename T>
DEV T dflux_x(const T* h, const T* kf, T kap, const uint8_t* mu, int j, int i, int ny, int nx, T dx) {
  if (j < 1 || j > ny - 2 || i < 1 || i > nx - 3) return T(0);
  size_t c = (size_t)j * nx + i;
  T k = kf ? kf[c] : kap;
  T f = k * (h[c + 1] - h[c]) / dx;
  return mu ? f * T(mu[c]) : f;
}
template <typename T>
DEV T dflux_y(const T* h, const T* kf, T kap, const uint8_t* mv, int j, int i, int ny, int nx, T dy) {
  if (j < 1 || j > ny - 3 || i < 1 || i > nx - 2) return T(0);
  size_t c = (size_t)j * nx + i;
  T k = kf ? kf[c] : kap;
  T f = k * (h[c + nx] - h[c]) / dy;
  return mv ? f * T(mv[c]) : f;
}

template <typename T>
__global__ void diffusion_kernel(const T* __restrict__ h, const T* __restrict__ kf, T kap,
                                 T* __restrict__ out, T* __restrict__ fxo, T* __restrict__ fyo,
                                 int ny, int nx, T dx, T dy, const uint8_t* mu, const uint8_t* mv,
                                 const uint8_t* mh) {
  int gi = blockIdx.x * blockDim.x + threadIdx.x;
  int gj = blockIdx.y * blockDim.y + threadIdx.y;
  if (gi >= nx || gj >= ny) return;
  size_t c = (size_t)gj * nx + gi;
  if (fxo) fxo[c] = dflux_x(h, kf, kap, mu, gj, gi, ny, nx, dx);
  if (fyo) fyo[c] = dflux_y(h, kf, kap, mv, gj, gi, ny, nx, dy);
  if (!out) return;
  T r = T(0);
  if (gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2) {
    T du = (dflux_x(h, kf, kap, mu, gj, gi, ny, nx, dx) - dflux_x(h, kf, kap, mu, gj, gi - 1, ny, nx, dx)) / dx;
    T dv = (dflux_y(h, kf, kap, mv, gj, gi, ny, nx, dy) - dflux_y(h, kf, kap, mv, gj - 1, gi, ny, nx, dy)) / dy;
    r = du + dv;
  }
  if (mh) r = r * T(mh[c]);
  out[c] = r;
}

// Biharmonic -kappa * L(L(h)) with L the unmasked flux-form Laplacian
// (BiharmonicDiffusion2D.__call__, diffusion.py:549-574), fused: the
// intermediate L(h) (zero ghost ring) lives in shared memory only.  A 64 x 16
// output tile per 256-thread block (threads as 64 columns x 4 rows, no index
// divisions); the flux quotients are products with 1/dx, 1/dy (within an ulp
// of the quotients).  Tiles whose cells and halo sit at least three cells
// from every edge take a branch-free body (every face flux active).
constexpr int BTX = 64, BTY = 16, BTHREADS = 256;
template <typename T>
__global__ void __launch_bounds__(BTHREADS)
biharmonic_kernel(const T* __restrict__ h, T* __restrict__ out, int ny, int nx, T rdx, T rdy, T kappa,
                  const uint8_t* __restrict__ mh) {
  __shared__ T hs[BTY + 4][BTX + 4];
  __shared__ T l1[BTY + 2][BTX + 2];
  const int x0 = blockIdx.x * BTX, y0 = blockIdx.y * BTY;
  const int tx = threadIdx.x & (BTX - 1), ty = threadIdx.x >> 6;
  const bool inner = x0 >= 3 && x0 + BTX <= nx - 3 && y0 >= 3 && y0 + BTY <= ny - 3;
  {
    // all of this thread's tile loads in flight before any is stored
    constexpr int RY = (BTY + 4 + 3) / 4, RX = (BTX + 4 + BTX - 1) / BTX;
    T v[RY][RX];
#pragma unroll
    for (int a = 0; a < RY; ++a) {
      const int ly = ty + 4 * a, gy = y0 - 2 + ly;
#pragma unroll
      for (int b = 0; b < RX; ++b) {
        const int lx = tx + BTX * b, gx = x0 - 2 + lx;
        const bool use = ly < BTY + 4 && lx < BTX + 4 && (inner || (gy >= 0 && gy < ny && gx >= 0 && gx < nx));
        v[a][b] = use ? h[(size_t)gy * nx + gx] : T(0);
      }
    }
#pragma unroll
    for (int a = 0; a < RY; ++a)
#pragma unroll
      for (int b = 0; b < RX; ++b)
        if (ty + 4 * a < BTY + 4 && tx + BTX * b < BTX + 4) hs[ty + 4 * a][tx + BTX * b] = v[a][b];
  }
  __syncthreads();
  // L(H) at (gy, gx) from the tile (ly, lx): fluxes zero off the interior faces
  auto lap = [&](auto&& H, int gy, int gx, int ly, int lx) -> T {
    if (gy < 1 || gy > ny - 2 || gx < 1 || gx > nx - 2) return T(0);
    const T c = H(ly, lx);
    const T fe = (gx <= nx - 3) ? (T(1) * (H(ly, lx + 1) - c)) * rdx : T(0);
    const T fw = (gx - 1 >= 1) ? (T(1) * (c - H(ly, lx - 1))) * rdx : T(0);
    const T fnn = (gy <= ny - 3) ? (T(1) * (H(ly + 1, lx) - c)) * rdy : T(0);
    const T fs = (gy - 1 >= 1) ? (T(1) * (c - H(ly - 1, lx))) * rdy : T(0);
    return (fe - fw) * rdx + (fnn - fs) * rdy;
  };
  auto lap_in = [&](auto&& H, int ly, int lx) -> T {
    const T c = H(ly, lx);
    const T fe = (H(ly, lx + 1) - c) * rdx, fw = (c - H(ly, lx - 1)) * rdx;
    const T fnn = (H(ly + 1, lx) - c) * rdy, fs = (c - H(ly - 1, lx)) * rdy;
    return (fe - fw) * rdx + (fnn - fs) * rdy;
  };
  auto Hh = [&](int ly, int lx) { return hs[ly][lx]; };
  auto Hl = [&](int ly, int lx) { return l1[ly][lx]; };
  if (inner) {
    for (int ly = ty; ly < BTY + 2; ly += 4)
      for (int lx = tx; lx < BTX + 2; lx += BTX) l1[ly][lx] = lap_in(Hh, ly + 1, lx + 1);
  } else {
    for (int ly = ty; ly < BTY + 2; ly += 4)
      for (int lx = tx; lx < BTX + 2; lx += BTX) l1[ly][lx] = lap(Hh, y0 - 1 + ly, x0 - 1 + lx, ly + 1, lx + 1);
  }
  __syncthreads();
  const int gx = x0 + tx;
  if (gx >= nx) return;
  for (int ly = ty; ly < BTY; ly += 4) {
    const int gy = y0 + ly;
    if (gy >= ny) break;
    T r = -kappa * (inner ? lap_in(Hl, ly + 1, tx + 1) : lap(Hl, gy, gx, ly + 1, tx + 1));
    const size_t c = (size_t)gy * nx + gx;
    if (mh) r = r * T(mh[c]);
    out[c] = r;
  }
}

// ===========================================================================
// Periodic ghost fill (boundary/boundary.py:52-75; S, N, W, E order so the
// corners end up as the doubly-wrapped interior values).
// ===========================================================================
template <typename T>
__global__ void fill_periodic_kernel(T* __restrict__ f, int ny, int nx) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int nring = 2 * nx + 2 * (ny - 2);
  if (k >= nring) return;
  T* F = f + (size_t)blockIdx.y * ny * nx;
  int j, i;
  if (k < nx) { j = 0; i = k; }
  else if (k < 2 * nx) { j = ny - 1; i = k - nx; }
  else if (k < 2 * nx + ny - 2) { j = k - 2 * nx + 1; i = 0; }
  else { j = k - 2 * nx - (ny - 2) + 1; i = nx - 1; }
  int sj = j == 0 ? ny - 2 : (j == ny - 1 ? 1 : j);
  int si = i == 0 ? nx - 2 : (i == nx - 1 ? 1 : i);
  F[(size_t)j * nx + i] = F[(size_t)sj * nx + si];
}

template <typename T>
__global__ void zero_ring_kernel(T* __restrict__ f, int ny, int nx) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int nring = 2 * nx + 2 * (ny - 2);
  if (k >= nring) return;
  T* F = f + (size_t)blockIdx.y * ny * nx;
  int j, i;
  if (k < nx) { j = 0; i = k; }
  else if (k < 2 * nx) { j = ny - 1; i = k - nx; }
  else if (k < 2 * nx + ny - 2) { j = k - 2 * nx + 1; i = 0; }
  else { j = k - 2 * nx - (ny - 2) + 1; i = nx - 1; }
  F[(size_t)j * nx + i] = T(0);
}

// ===========================================================================
// out = a*x + b*y + c*z (z optional), evaluated as ((a*x + b*y) + c*z) in T:
// the Shu-Osher combinations of rk3_ssp_step / heun_step / euler_step
// (timestepping/explicit_rk.py:22-121).
// ===========================================================================
template <typename T>
__global__ void lincomb_kernel(size_t n, T a, const T* __restrict__ x, T b, const T* __restrict__ y, T c,
                               const T* __restrict__ z, T* __restrict__ out) {
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; k < n; k += stride) {
    T r = a * x[k];
    if (y) r = r + b * y[k];
    if (z) r = r + c * z[k];
    out[k] = r;
  }
}

// upwind_flux blend (advection/flux.py:221-253): per interior face, the flux
// of the tier whose mask is set at the upwind cell; ghost ring zero.
constexpr int kMaxTiers = 8;
template <typename T>
struct BlendArgs {
  const T* flux[kMaxTiers];
  const uint8_t* mask[kMaxTiers];
  int n;
};
template <typename T>
__global__ void upwind_blend_kernel(BlendArgs<T> A, const T* __restrict__ u, T* __restrict__ out, int ny,
                                    int nx, int dim) {
  int gi = blockIdx.x * blockDim.x + threadIdx.x;
  int gj = blockIdx.y * blockDim.y + threadIdx.y;
  if (gi >= nx || gj >= ny) return;
  size_t c = (size_t)gj * nx + gi;
  T r = T(0);
  if (gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2) {
    size_t up = u[c] >= T(0) ? c : (dim == 1 ? c + 1 : c + nx);
    for (int s = 0; s < A.n; ++s)
      if (A.mask[s][up]) r = r + A.flux[s][c];
  }
  out[c] = r;
}

// ===========================================================================
// Host dispatch
// ===========================================================================
template <typename T, int S>
static void launch_advect_unmasked(const T* h, const T* u, const T* v, T* out, int ny, int nx, T dx, T dy,
                                   const uint8_t* mh, cudaStream_t st) {
  dim3 g((nx + ATX - 1) / ATX, (ny + ATY - 1) / ATY);
  advect_tile_kernel<T, S, 0, -1, false><<<g, ATHREADS, 0, st>>>(h, u, v, out, ny, nx, dx, dy, nullptr, mh);
}
template <typename T, int S4, int S6>
static void launch_advect_masked(const T* h, const T* u, const T* v, T* out, int ny, int nx, T dx, T dy,
                                 const uint8_t* tiers, const uint8_t* mh, cudaStream_t st) {
  dim3 g((nx + ATX - 1) / ATX, (ny + ATY - 1) / ATY);
  advect_tile_kernel<T, 0, S4, S6, true><<<g, ATHREADS, 0, st>>>(h, u, v, out, ny, nx, dx, dy, tiers, mh);
}

// Minimum line length each scheme's boundary ladder is defined for.
static int min_len(int m) {
  switch (m) {
    case FVX_WENO9: return 8;   // shortest line the reference's ladder concatenation accepts
    case FVX_WENO7: return 6;
    case FVX_WENO5: case FVX_WENOZ5: return 4;
    default: return 3;
  }
}

template <typename T>
static int advect2d(const T* h, const T* u, const T* v, T* out, int ny, int nx, double dx, double dy,
                    int method, const uint8_t* tiers, const uint8_t* mh, cudaStream_t st) {
  if (!h || !u || !v || !out) return FVX_ERR_ARG;
  if (method < 0 || method >= FVX_WENOZ3) return FVX_ERR_METHOD;
  if (ny < min_len(method) || nx < min_len(method)) return FVX_ERR_SHAPE;
  T tdx = T(dx), tdy = T(dy);
  if (tiers) {
    if (!mh) return FVX_ERR_ARG;
    switch (method) {
      case FVX_WENO5: launch_advect_masked<T, FVX_WENO3, FVX_WENO5>(h, u, v, out, ny, nx, tdx, tdy, tiers, mh, st); break;
      case FVX_WENOZ5: launch_advect_masked<T, FVX_WENOZ3, FVX_WENOZ5>(h, u, v, out, ny, nx, tdx, tdy, tiers, mh, st); break;
      case FVX_WENO3: launch_advect_masked<T, FVX_WENO3, -1>(h, u, v, out, ny, nx, tdx, tdy, tiers, mh, st); break;
      case FVX_MINMOD: launch_advect_masked<T, FVX_MINMOD, -1>(h, u, v, out, ny, nx, tdx, tdy, tiers, mh, st); break;
      case FVX_VAN_LEER: launch_advect_masked<T, FVX_VAN_LEER, -1>(h, u, v, out, ny, nx, tdx, tdy, tiers, mh, st); break;
      case FVX_SUPERBEE: launch_advect_masked<T, FVX_SUPERBEE, -1>(h, u, v, out, ny, nx, tdx, tdy, tiers, mh, st); break;
      case FVX_MC: launch_advect_masked<T, FVX_MC, -1>(h, u, v, out, ny, nx, tdx, tdy, tiers, mh, st); break;
      default: return FVX_ERR_METHOD;
    }
    return fvx_cuda_status();
  }
  switch (method) {
#define FVX_CASE(M) case M: launch_advect_unmasked<T, M>(h, u, v, out, ny, nx, tdx, tdy, mh, st); break;
    FVX_CASE(FVX_NAIVE) FVX_CASE(FVX_UPWIND1) FVX_CASE(FVX_UPWIND2) FVX_CASE(FVX_UPWIND3)
    FVX_CASE(FVX_WENO3) FVX_CASE(FVX_WENO5) FVX_CASE(FVX_WENOZ5) FVX_CASE(FVX_WENO7)
    FVX_CASE(FVX_WENO9) FVX_CASE(FVX_MINMOD) FVX_CASE(FVX_VAN_LEER) FVX_CASE(FVX_SUPERBEE)
    FVX_CASE(FVX_MC)
#undef FVX_CASE
    default: return FVX_ERR_METHOD;
  }
  return fvx_cuda_status();
}

template <typename T, int S, int S4, int S6, bool MK>
static void launch_ff(const T* h, const T* u, const T* v, T* fe, T* fn, int ny, int nx, const uint8_t* tiers,
                      cudaStream_t st) {
  dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);
  face_flux_kernel<T, S, S4, S6, MK><<<g, b, 0, st>>>(h, u, v, fe, fn, ny, nx, tiers);
}

template <typename T>
static int face_flux2d(const T* h, const T* u, const T* v, T* fe, T* fn, int ny, int nx, int method,
                       const uint8_t* tiers, cudaStream_t st) {
  if (!h || !u || !v) return FVX_ERR_ARG;
  if (method < 0 || method >= FVX_NUM_SCHEMES) return FVX_ERR_METHOD;
  if (ny < min_len(method) || nx < min_len(method)) return FVX_ERR_SHAPE;
  if (tiers) {
    switch (method) {
      case FVX_WENO5: launch_ff<T, 0, FVX_WENO3, FVX_WENO5, true>(h, u, v, fe, fn, ny, nx, tiers, st); break;
      case FVX_WENOZ5: launch_ff<T, 0, FVX_WENOZ3, FVX_WENOZ5, true>(h, u, v, fe, fn, ny, nx, tiers, st); break;
      case FVX_WENO3: launch_ff<T, 0, FVX_WENO3, -1, true>(h, u, v, fe, fn, ny, nx, tiers, st); break;
      case FVX_MINMOD: launch_ff<T, 0, FVX_MINMOD, -1, true>(h, u, v, fe, fn, ny, nx, tiers, st); break;
      case FVX_VAN_LEER: launch_ff<T, 0, FVX_VAN_LEER, -1, true>(h, u, v, fe, fn, ny, nx, tiers, st); break;
      case FVX_SUPERBEE: launch_ff<T, 0, FVX_SUPERBEE, -1, true>(h, u, v, fe, fn, ny, nx, tiers, st); break;
      case FVX_MC: launch_ff<T, 0, FVX_MC, -1, true>(h, u, v, fe, fn, ny, nx, tiers, st); break;
      default: return FVX_ERR_METHOD;
    }
    return fvx_cuda_status();
  }
  switch (method) {
#define FVX_CASE(M) case M: launch_ff<T, M, 0, -1, false>(h, u, v, fe, fn, ny, nx, nullptr, st); break;
    FVX_CASE(FVX_NAIVE) FVX_CASE(FVX_UPWIND1) FVX_CASE(FVX_UPWIND2) FVX_CASE(FVX_UPWIND3)
    FVX_CASE(FVX_WENO3) FVX_CASE(FVX_WENO5) FVX_CASE(FVX_WENOZ5) FVX_CASE(FVX_WENO7)
    FVX_CASE(FVX_WENO9) FVX_CASE(FVX_MINMOD) FVX_CASE(FVX_VAN_LEER) FVX_CASE(FVX_SUPERBEE)
    FVX_CASE(FVX_MC) FVX_CASE(FVX_WENOZ3)
#undef FVX_CASE
    default: return FVX_ERR_METHOD;
  }
  return fvx_cuda_status();
}

}  // namespace fvx

using namespace fvx;

// ===========================================================================
// C ABI
// ===========================================================================
#define FVX_DTYPES(X) X(f32, float) X(f64, double)

#define FVX_DEF_ADVECT(SFX, T)                                                                       \
  extern "C" int fvx_advect2d_##SFX(const T* h, const T* u, const T* v, T* out, int ny, int nx,      \
                                    double dx, double dy, int method, const uint8_t* tiers,          \
                                    const uint8_t* mask_h, void* stream) {                           \
    return advect2d<T>(h, u, v, out, ny, nx, dx, dy, method, tiers, mask_h, fvx_stream(stream));      \
  }                                                                                                  \
  extern "C" int fvx_face_flux2d_##SFX(const T* h, const T* u, const T* v, T* fe, T* fn, int ny,     \
                                       int nx, int method, const uint8_t* tiers, void* stream) {     \
    return face_flux2d<T>(h, u, v, fe, fn, ny, nx, method, tiers, fvx_stream(stream));               \
  }                                                                                                  \
  extern "C" int fvx_flux_divergence2d_##SFX(const T* fe, const T* fn, T* out, int ny, int nx,      \
                                             double dx, double dy, const uint8_t* mask_h,            \
                                             void* stream) {                                         \
    if (!fe || !fn || !out) return FVX_ERR_ARG;                                                      \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                      \
    dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);                                                   \
    flux_divergence_kernel<T><<<g, b, 0, fvx_stream(stream)>>>(fe, fn, out, ny, nx, T(dx), T(dy),    \
                                                                 mask_h);                            \
    return fvx_cuda_status();                                                                        \
  }                                                                                                  \
  extern "C" int fvx_cgrid_op2d_##SFX(int op, const T* a, const T* b, T* out, T* out2, int ny,       \
                                      int nx, double dx, double dy, const uint8_t* mask_out,         \
                                      const uint8_t* mask_out2, void* stream) {                      \
    if (!a || !out) return FVX_ERR_ARG;                                                              \
    if ((op == OP_DIVERGENCE || op == OP_CURL) && !b) return FVX_ERR_ARG;                            \
    if (op == OP_GRAD_PERP && !out2) return FVX_ERR_ARG;                                             \
    if (!((op >= 0 && op <= OP_GRAD_PERP) || (op >= OP_T2U && op <= OP_V2U))) return FVX_ERR_METHOD;  \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                      \
    dim3 bl(32, 8), g((nx + 31) / 32, (ny + 7) / 8);                                                  \
    cgrid_op_kernel<T><<<g, bl, 0, fvx_stream(stream)>>>(op, a, b, out, out2, ny, nx, T(dx), T(dy),  \
                                                           mask_out, mask_out2);                     \
    return fvx_cuda_status();                                                                        \
  }                                                                                                  \
  extern "C" int fvx_arakawa_jacobian_##SFX(const T* f, const T* g, T* out, int batch, int ny,       \
                                            int nx, double dx, double dy, void* stream) {            \
    if (!f || !g || !out) return FVX_ERR_ARG;                                                        \
    if (ny < 3 || nx < 3 || batch < 1 || batch > 65535) return FVX_ERR_SHAPE;                        \
    dim3 gr((nx - 2 + kJacCols - 1) / kJacCols, (ny - 2 + kJacRows - 1) / kJacRows, batch);              \
    jacobian_kernel<T><<<gr, kJacCols, 0, fvx_stream(stream)>>>(f, g, out, ny, nx, T(1.0 / (12.0 * dx * dy))); \
    return fvx_cuda_status();                                                                        \
  }                                                                                                  \
  extern "C" int fvx_diffusion2d_##SFX(const T* h, const T* kappa_field, double kappa, T* out,       \
                                       T* flux_x, T* flux_y, int ny, int nx, double dx, double dy,   \
                                       const uint8_t* mask_u, const uint8_t* mask_v,                 \
                                       const uint8_t* mask_h, void* stream) {                        \
    if (!h || (!out && !flux_x && !flux_y)) return FVX_ERR_ARG;                                      \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                      \
    dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);                                                   \
    diffusion_kernel<T><<<g, b, 0, fvx_stream(stream)>>>(h, kappa_field, T(kappa), out, flux_x,     \
                                                           flux_y, ny, nx, T(dx), T(dy), mask_u,     \
                                                           mask_v, mask_h);                          \
    return fvx_cuda_status();                                                                        \
  }                                                                                                  \
  extern "C" int fvx_biharmonic2d_##SFX(const T* h, double kappa, T* out, int ny, int nx, double dx, \
                                        double dy, const uint8_t* mask_h, void* stream) {            \
    if (!h || !out) return FVX_ERR_ARG;                                                              \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                      \
    dim3 g((nx + BTX - 1) / BTX, (ny + BTY - 1) / BTY);                                               \
    biharmonic_kernel<T><<<g, BTHREADS, 0, fvx_stream(stream)>>>(h, out, ny, nx, T(1.0 / dx),         \
                                                                   T(1.0 / dy), T(kappa), mask_h);   \
    return fvx_cuda_status();                                                                        \
  }                                                                                                  \
  extern "C" int fvx_fill_periodic_##SFX(T* field, int batch, int ny, int nx, void* stream) {        \
    if (!field) return FVX_ERR_ARG;                                                                  \
    if (ny < 3 || nx < 3 || batch < 1 || batch > 65535) return FVX_ERR_SHAPE;                        \
    int n = 2 * nx + 2 * (ny - 2);                                                                   \
    fill_periodic_kernel<T><<<dim3((n + 255) / 256, batch), 256, 0, fvx_stream(stream)>>>(field, ny, \
                                                                                          nx);       \
    return fvx_cuda_status();                                                                        \
  }                                                                                                  \
  extern "C" int fvx_zero_ring_##SFX(T* field, int batch, int ny, int nx, void* stream) {            \
    if (!field) return FVX_ERR_ARG;                                                                  \
    if (ny < 3 || nx < 3 || batch < 1 || batch > 65535) return FVX_ERR_SHAPE;                        \
    int n = 2 * nx + 2 * (ny - 2);                                                                   \
    zero_ring_kernel<T><<<dim3((n + 255) / 256, batch), 256, 0, fvx_stream(stream)>>>(field, ny, nx); \
    return fvx_cuda_status();                                                                        \
  }

FVX_DTYPES(FVX_DEF_ADVECT)

#define FVX_DEF_MISC(SFX, T)                                                                          \
  extern "C" int fvx_lincomb_##SFX(int64_t n, double a, const T* x, double b, const T* y, double c,   \
                                   const T* z, T* out, void* stream) {                                \
    if (!x || !out || n < 0) return FVX_ERR_ARG;                                                      \
    if (n == 0) return FVX_OK;                                                                        \
    int blocks = (int)((n + 255) / 256);                                                              \
    if (blocks > 148 * 16) blocks = 148 * 16;                                                         \
    lincomb_kernel<T><<<blocks, 256, 0, fvx_stream(stream)>>>((size_t)n, T(a), x, T(b), y, T(c), z,  \
                                                              out);                                   \
    return fvx_cuda_status();                                                                         \
  }                                                                                                   \
  extern "C" int fvx_upwind_blend_##SFX(const T* const* fluxes, const uint8_t* const* masks,          \
                                        int ntiers, const T* u, T* out, int ny, int nx, int dim,     \
                                        void* stream) {                                               \
    if (!fluxes || !masks || !u || !out) return FVX_ERR_ARG;                                          \
    if (ntiers < 1 || ntiers > kMaxTiers) return FVX_ERR_SHAPE;                                       \
    if (dim != 0 && dim != 1) return FVX_ERR_ARG;                                                     \
    BlendArgs<T> A;                                                                                   \
    A.n = ntiers;                                                                                     \
    for (int s = 0; s < ntiers; ++s) { A.flux[s] = fluxes[s]; A.mask[s] = masks[s]; }                  \
    dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);                                                    \
    upwind_blend_kernel<T><<<g, b, 0, fvx_stream(stream)>>>(A, u, out, ny, nx, dim);                  \
    return fvx_cuda_status();                                                                         \
  }

FVX_DTYPES(FVX_DEF_MISC)
