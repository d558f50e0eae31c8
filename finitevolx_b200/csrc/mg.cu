// Geometric multigrid for the masked, variable-coefficient Helmholtz
// operator and the preconditioned CG built on it.
//
// Restates finitevolX solvers/multigrid.py: _apply_operator (:327-405),
// _weighted_jacobi (:408-461), _restrict (:464-507), _prolongate (:510-598),
// MultigridSolver.v_cycle (:808-881) and build_multigrid_solver
// (:905-1062, level hierarchy built on the host in FP64 like the
// reference's offline NumPy setup), plus masked_laplacian
// (solvers/iterative.py:144-191) and a PCG whose stopping test follows
// solve_cg (iterative.py:48-136).
//
// Device layout per level: mask, cx, cy, inv_diag, u, f, tmp (T = float or
// double, row-major [ny, nx]).  Levels at or below kCoarseCells cells run
// inside one CTA (one launch for the whole coarse part of the V-cycle);
// finer levels use one launch per leg (all of its sweeps and the transfer).
#include "fvx_common.cuh"

#include <cmath>
#include <vector>

namespace fvx {
namespace mg {

constexpr int kCoarseCells = 32 * 32;
constexpr int kCoarseThreads = 1024;

template <typename T>
struct Lev {
  int ny, nx;
  T rdx2, rdy2;    // 1/dx^2, 1/dy^2 at this level
  T dx2, dy2;      // dx^2, dy^2 (FP64 divides like the reference)
  T lam;
  T *mask, *cx, *cy, *inv, *u, *f, *tmp;
};

DEV double block_sum(double v) {
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

// Grid-stride walk over the cells of an ny x nx array: f(c, j, i) for
// c = global thread index, + stride, ... with the row j and column i
// advanced by additions (one division per thread, at the start), so the
// loop body carries no 64-bit division.
template <typename F>
DEV void grid_cells(int ny, int nx, F&& f) {
  const size_t n = (size_t)ny * nx, stride = (size_t)gridDim.x * blockDim.x;
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  int j = (int)(c / (size_t)nx), i = (int)(c - (size_t)j * nx);
  const int dj = (int)(stride / (size_t)nx), di = (int)(stride - (size_t)dj * nx);
  for (; c < n; c += stride) {
    f(c, j, i);
    i += di;
    j += dj;
    if (i >= nx) {
      i -= nx;
      ++j;
    }
  }
}

// True in the one block that finishes last (an atomic ticket taken after a
// fence); that block then sums the partials in block order.
DEV bool pcg_last_block(unsigned* ticket) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  return last;
}

template <typename T> DEV T divd(T a, T d2, T rd2) {
  if constexpr (sizeof(T) == 8) return a / d2;
  else return a * rd2;
}

// (A u)[j,i] of _apply_operator: u masked first, zero-padded neighbours,
// conservative 5-point stencil, output masked.
template <typename T>
DEV T apply_at(const Lev<T>& L, const T* u, int j, int i) {
  const int nx = L.nx, ny = L.ny;
  const size_t c = (size_t)j * nx + i;
  const T m = L.mask[c];
  const T um = u[c] * m;
  const T ue = i + 1 < nx ? u[c + 1] * L.mask[c + 1] : T(0);
  const T uw = i > 0 ? u[c - 1] * L.mask[c - 1] : T(0);
  const T un = j + 1 < ny ? u[c + nx] * L.mask[c + nx] : T(0);
  const T us = j > 0 ? u[c - nx] * L.mask[c - nx] : T(0);
  const T cxw = i > 0 ? L.cx[c - 1] : T(0);
  const T cys = j > 0 ? L.cy[c - nx] : T(0);
  const T lap = divd(L.cx[c] * (ue - um) - cxw * (um - uw), L.dx2, L.rdx2) +
                divd(L.cy[c] * (un - um) - cys * (um - us), L.dy2, L.rdy2);
  return (lap - L.lam * um) * m;
}

template <typename T>
DEV void jacobi_at(const Lev<T>& L, const T* u, const T* f, T* out, T omega, int j, int i, size_t c) {
  const T r = f[c] - apply_at(L, u, j, i);
  out[c] = (u[c] + omega * L.inv[c] * r) * L.mask[c];
}

// coarse cell (J, I): r = (f - A u) * m on the 4 fine cells, mask-weighted mean
template <typename T>
DEV void restrict_at(const Lev<T>& F, const T* u, const T* f, const Lev<T>& C, T* fc, int J, int I, size_t cc) {
  T s[4], m[4];
  const int dj[4] = {0, 1, 0, 1}, di[4] = {0, 0, 1, 1};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int j = 2 * J + dj[k], i = 2 * I + di[k];
    const size_t c = (size_t)j * F.nx + i;
    const T mf = F.mask[c];
    const T r = (f[c] - apply_at(F, u, j, i)) * mf;
    s[k] = r * mf;
    m[k] = mf;
  }
  const T sum4 = ((s[0] + s[1]) + s[2]) + s[3];
  const T cnt = ((m[0] + m[1]) + m[2]) + m[3];
  fc[cc] = (sum4 / (cnt > T(1) ? cnt : T(1))) * C.mask[cc];
}

// fine cell: u = (u + P e_c) * m_f, P the mask-normalised 9/3/3/1 bilinear form
template <typename T>
DEV void prolong_at(const Lev<T>& F, T* u, const Lev<T>& C, const T* ec, int j, int i, size_t c) {
  const int J = j >> 1, I = i >> 1, dj = j & 1, di = i & 1;
  const int sj = 2 * dj - 1, si = 2 * di - 1;
  auto V = [&](int jj, int ii) -> T {
    if (jj < 0 || jj >= C.ny || ii < 0 || ii >= C.nx) return T(0);
    const size_t k = (size_t)jj * C.nx + ii;
    return ec[k] * C.mask[k];
  };
  auto M = [&](int jj, int ii) -> T {
    if (jj < 0 || jj >= C.ny || ii < 0 || ii >= C.nx) return T(0);
    return C.mask[(size_t)jj * C.nx + ii];
  };
  const T ws = ((T(9) * V(J, I) + T(3) * V(J, I + si)) + T(3) * V(J + sj, I)) + T(1) * V(J + sj, I + si);
  const T ds = ((T(9) * M(J, I) + T(3) * M(J, I + si)) + T(3) * M(J + sj, I)) + T(1) * M(J + sj, I + si);
  const T e = (ws / (ds > T(1) ? ds : T(1))) * F.mask[c];
  u[c] = (u[c] + e) * F.mask[c];
}

template <typename T>
__global__ void jacobi_kernel(Lev<T> L, const T* u, const T* f, T* out, T omega) {
  const size_t n = (size_t)L.ny * L.nx;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(c / L.nx), i = (int)(c - (size_t)j * L.nx);
    jacobi_at(L, u, f, out, omega, j, i, c);
  }
}
template <typename T>
__global__ void restrict_kernel(Lev<T> F, const T* u, const T* f, Lev<T> C, T* fc) {
  const size_t n = (size_t)C.ny * C.nx;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int J = (int)(c / C.nx), I = (int)(c - (size_t)J * C.nx);
    restrict_at(F, u, f, C, fc, J, I, c);
  }
}
template <typename T>
__global__ void prolong_kernel(Lev<T> F, T* u, Lev<T> C, const T* ec) {
  const size_t n = (size_t)F.ny * F.nx;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(c / F.nx), i = (int)(c - (size_t)j * F.nx);
    prolong_at(F, u, C, ec, j, i, c);
  }
}
template <typename T>
__global__ void apply_kernel(Lev<T> L, const T* u, T* out) {
  const size_t n = (size_t)L.ny * L.nx;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(c / L.nx), i = (int)(c - (size_t)j * L.nx);
    out[c] = apply_at(L, u, j, i);
  }
}
template <typename T>
__global__ void fill_kernel(T* p, size_t n, T v) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) p[c] = v;
}
template <typename T>
__global__ void copy_kernel(T* dst, const T* src, size_t n) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    dst[c] = src[c];
}

constexpr int kMaxLevels = 16;
template <typename T>
struct LevArray {
  Lev<T> L[kMaxLevels];
};

// fnc(j, i, c) on this thread's cells c = tid, tid + kCoarseThreads, ... of
// an ny x nx level (row j, column i), the indices advanced without divisions.
template <typename F>
DEV void coarse_cells(int ny, int nx, F&& fnc) {
  const int cells = ny * nx;
  const int dq = kCoarseThreads / nx, dr = kCoarseThreads - dq * nx;
  int j = (int)threadIdx.x / nx, i = (int)threadIdx.x - j * nx;
  for (int c = threadIdx.x; c < cells; c += kCoarseThreads) {
    fnc(j, i, (size_t)c);
    i += dr;
    j += dq;
    if (i >= nx) { i -= nx; ++j; }
  }
}

// The coarsest-grid solve -- n Jacobi sweeps from u = 0 -- of a level of at
// most kWarpSolveCells cells on shared-memory copies of the level's arrays
// (sh: 7 * kWarpSolveCells values): one cell per thread of the first
// ceil(cells / 32) warps, which alone meet at a named barrier between sweeps.
// jacobi_at's arithmetic on the same values as the block-wide form over
// global memory.  f_src: the right-hand side (of type F, widened as it is
// copied); the solution goes to u_dst (of type U, rounded if narrower).
// Called by the whole CTA; returns with it synchronised.
constexpr int kWarpSolveCells = 256;
template <typename T, typename F, typename U>
DEV void coarsest_warp_solve(const Lev<T>& L, const F* f_src, U* u_dst, int n, T omega, T* sh) {
  const int cells = L.ny * L.nx;
  Lev<T> S = L;
  S.mask = sh;
  S.cx = sh + kWarpSolveCells;
  S.cy = sh + 2 * kWarpSolveCells;
  S.inv = sh + 3 * kWarpSolveCells;
  S.f = sh + 4 * kWarpSolveCells;
  S.u = sh + 5 * kWarpSolveCells;
  S.tmp = sh + 6 * kWarpSolveCells;
  for (int c = threadIdx.x; c < cells; c += blockDim.x) {
    S.mask[c] = L.mask[c];
    S.cx[c] = L.cx[c];
    S.cy[c] = L.cy[c];
    S.inv[c] = L.inv[c];
    S.f[c] = (T)f_src[c];
    S.u[c] = T(0);
  }
  __syncthreads();
  const int nthr = (cells + 31) & ~31;
  const int c = threadIdx.x;
  if (c < nthr) {
    const int j = c / L.nx, i = c - j * L.nx;
    T* a = S.u;
    T* b = S.tmp;
    for (int s = 0; s < n; ++s) {
      if (c < cells) jacobi_at(S, a, S.f, b, omega, j, i, (size_t)c);
      asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory");
      T* t = a;
      a = b;
      b = t;
    }
    if (c < cells) u_dst[c] = (U)a[c];
  }
  __syncthreads();
}

// Whole coarse part of a V-cycle in one CTA: levels lc .. nl-1, entered with
// f[lc] set and u[lc] = 0 (the recursion's zero initial guess).  S is the
// level table in shared memory; each level's entry is copied to registers
// before its loops (its fields are read at every cell).
// D (may be null): the coarsest level in FP64; its n_coarse sweeps -- the
// coarsest-grid solve -- then run in FP64 on the widened right-hand side and
// the result is rounded back into S[nl-1].u.
// wsh (may be null): shared memory for coarsest_warp_solve (7 *
// kWarpSolveCells values of the coarsest solve's type), used when the
// coarsest level fits it.
template <typename T>
DEV void coarse_cycle(const Lev<T>* S, int lc, int nl, int n_pre, int n_post, int n_coarse, T omega,
                      const Lev<double>* D = nullptr, void* wsh = nullptr) {
  const int tid = threadIdx.x;
  auto sweeps = [&](const Lev<T> L, int n) {
    const size_t cells = (size_t)L.ny * L.nx;
    T* a = L.u;
    T* b = L.tmp;
    for (int s = 0; s < n; ++s) {
      coarse_cells(L.ny, L.nx, [&](int j, int i, size_t c) { jacobi_at(L, a, L.f, b, omega, j, i, c); });
      __syncthreads();
      T* t = a; a = b; b = t;
    }
    if (a != L.u) {
      for (size_t c = tid; c < cells; c += kCoarseThreads) L.u[c] = a[c];
      __syncthreads();
    }
  };
  for (int l = lc; l < nl; ++l) {
    const Lev<T> L = S[l];
    const size_t cells = (size_t)L.ny * L.nx;
    for (size_t c = tid; c < cells; c += kCoarseThreads) L.u[c] = T(0);
    __syncthreads();
    if (l == nl - 1) {
      const bool warp = wsh && cells <= (size_t)kWarpSolveCells;
      if (D && warp) {
        coarsest_warp_solve<double, T, T>(*D, L.f, L.u, n_coarse, (double)omega, (double*)wsh);
      } else if (!D && warp) {
        coarsest_warp_solve<T, T, T>(L, L.f, L.u, n_coarse, omega, (T*)wsh);
      } else if (D) {
        const Lev<double> E = *D;
        for (size_t c = tid; c < cells; c += kCoarseThreads) { E.f[c] = (double)L.f[c]; E.u[c] = 0.0; }
        __syncthreads();
        double* a = E.u;
        double* b = E.tmp;
        for (int s = 0; s < n_coarse; ++s) {
          coarse_cells(E.ny, E.nx, [&](int j, int i, size_t c) { jacobi_at(E, a, E.f, b, (double)omega, j, i, c); });
          __syncthreads();
          double* t = a; a = b; b = t;
        }
        for (size_t c = tid; c < cells; c += kCoarseThreads) L.u[c] = (T)a[c];
        __syncthreads();
      } else {
        sweeps(L, n_coarse);
      }
      break;
    }
    sweeps(L, n_pre);
    const Lev<T> C = S[l + 1];
    const size_t cc = (size_t)C.ny * C.nx;
    coarse_cells(C.ny, C.nx, [&](int J, int I, size_t c) { restrict_at(L, L.u, L.f, C, C.f, J, I, c); });
    __syncthreads();
  }
  for (int l = nl - 2; l >= lc; --l) {
    const Lev<T> L = S[l];
    const Lev<T> C = S[l + 1];
    const size_t cells = (size_t)L.ny * L.nx;
    coarse_cells(L.ny, L.nx, [&](int j, int i, size_t c) { prolong_at(L, L.u, C, C.u, j, i, c); });
    __syncthreads();
    sweeps(L, n_post);
  }
}

template <typename T>
__global__ void __launch_bounds__(kCoarseThreads)
coarse_vcycle_kernel(LevArray<T> A, int lc, int nl, int n_pre, int n_post, int n_coarse, T omega) {
  __shared__ Lev<T> S[kMaxLevels];
  __shared__ T wsh[7 * kWarpSolveCells];
  if (threadIdx.x < nl) S[threadIdx.x] = A.L[threadIdx.x];
  __syncthreads();
  coarse_cycle(S, lc, nl, n_pre, n_post, n_coarse, omega, (const Lev<double>*)nullptr, (void*)wsh);
}

// An FP32 plan's single-CTA coarse cycle with the coarsest-grid solve (the
// n_coarse Jacobi sweeps on the coarsest level) in FP64, on the FP64 copy of
// that level (operators from the same FP64 host hierarchy).
__global__ void __launch_bounds__(kCoarseThreads)
coarse_vcycle_f64_kernel(LevArray<float> A, Lev<double> D, int lc, int nl, int n_pre, int n_post, int n_coarse,
                         float omega) {
  __shared__ Lev<float> S[kMaxLevels];
  __shared__ Lev<double> E;
  __shared__ double wsh[7 * kWarpSolveCells];
  if (threadIdx.x < nl) S[threadIdx.x] = A.L[threadIdx.x];
  if (threadIdx.x == 0) E = D;
  __syncthreads();
  coarse_cycle(S, lc, nl, n_pre, n_post, n_coarse, omega, &E, (void*)wsh);
}

// Many independent solves of A_lc u = f at level lc, one CTA per right-hand
// side: u = sum of n_cycles V-cycle corrections, u += V(f - A u).  Each
// block's level arrays u, f, tmp come from its own slice of ``work``
// (3 * sum of the cells of levels lc .. nl-1 per block).
template <typename T>
__global__ void __launch_bounds__(kCoarseThreads)
coarse_solve_batched_kernel(LevArray<T> A, int lc, int nl, int n_pre, int n_post, int n_coarse, T omega,
                            const T* __restrict__ f, T* __restrict__ u, T* work, size_t work_per_block,
                            int n_cycles) {
  __shared__ Lev<T> S[kMaxLevels];
  __shared__ T wsh[7 * kWarpSolveCells];
  if (threadIdx.x == 0) {
    T* w = work + (size_t)blockIdx.x * work_per_block;
    for (int l = lc; l < nl; ++l) {
      S[l] = A.L[l];
      const size_t c = (size_t)S[l].ny * S[l].nx;
      S[l].u = w;
      S[l].f = w + c;
      S[l].tmp = w + 2 * c;
      w += 3 * c;
    }
  }
  __syncthreads();
  const Lev<T>& L = S[lc];
  const size_t cells = (size_t)L.ny * L.nx;
  const T* fb = f + (size_t)blockIdx.x * cells;
  T* ub = u + (size_t)blockIdx.x * cells;
  for (size_t c = threadIdx.x; c < cells; c += kCoarseThreads) ub[c] = T(0);
  __syncthreads();
  for (int k = 0; k < n_cycles; ++k) {
    coarse_cells(L.ny, L.nx, [&](int j, int i, size_t c) { L.f[c] = (fb[c] - apply_at(L, ub, j, i)) * L.mask[c]; });
    __syncthreads();
    coarse_cycle(S, lc, nl, n_pre, n_post, n_coarse, omega, (const Lev<double>*)nullptr, (void*)wsh);
    for (size_t c = threadIdx.x; c < cells; c += kCoarseThreads) ub[c] += L.u[c];
    __syncthreads();
  }
}

// Energy-optimal scaling of a coarse correction d = C.u:
// omega = (d . f) / (d . A d) minimises |e* - omega d| in the energy norm of
// -A (A negative definite), so the scaled correction never increases the
// level-lvl error; omega = 0 when d . A d = 0.
template <typename T>
__global__ void __launch_bounds__(256)
k_coarse_omega(Lev<T> C, double* part, unsigned* ticket, double* omega) {
  const size_t n = (size_t)C.ny * C.nx;
  double df = 0.0, dad = 0.0;
  (void)n;
  grid_cells(C.ny, C.nx, [&](size_t c, int j, int i) {
    const double d = (double)C.u[c];
    df += d * (double)C.f[c];
    dad += d * (double)apply_at(C, C.u, j, i);
  });
  df = block_sum(df);
  dad = block_sum(dad);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = df; part[2 * blockIdx.x + 1] = dad; }
  if (pcg_last_block(ticket)) {
    __threadfence();
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
      a += ((volatile double*)part)[2 * k];
      b += ((volatile double*)part)[2 * k + 1];
    }
    a = block_sum(a);
    b = block_sum(b);
    if (threadIdx.x == 0) {
      *omega = b != 0.0 ? a / b : 0.0;
      *ticket = 0u;
    }
  }
}

template <typename T>
__global__ void k_scale(T* u, size_t n, const double* omega) {
  const T w = (T)*omega;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    u[c] *= w;
}

constexpr int kOmegaBlocks = 64;

// ---------------------------------------------------------------------------
// Fused V-cycle legs for the host-driven (fine) levels, one launch per leg:
//   down: u = k Jacobi sweeps from u_init (NULL = 0) on f, then the
//         restricted residual R (f - A u) into the next level's f;
//   up:   u = u_pre + P e_coarse, then k Jacobi sweeps, into ``out``.
// A CTA covers its output tile plus a halo of H = k (+1 for the residual):
// an RW x RH region.  Thread tid owns column c = tid % RW of the region and
// rows r0 .. r0 + LR - 1 of it (r0 = (tid / RW) LR): those cells' u, f,
// omega * inv_diag, cx, cy and mask stay in its registers for the whole leg;
// shared memory holds u (two buffers, for the neighbours' reads) and cx
// (for the west face).  Every sweep updates the whole region but its outer
// ring: a cell d cells from the region's edge is exact after d sweeps, so
// after k sweeps the tile and a ring of H - k around it hold the global
// Jacobi iterate, as in the shrinking-region form.  The arithmetic of every
// cell is jacobi_at / restrict_at / prolong_at's, in the same order.
// ---------------------------------------------------------------------------
constexpr int kLegMaxSweeps = 16;
constexpr int kLegFewTiles = 148;  // legs with fewer tiles use more threads per CTA

template <typename T> struct LegTile;
template <> struct LegTile<float> { static constexpr int TX = 64, TY = 32; };
template <> struct LegTile<double> { static constexpr int TX = 32, TY = 16; };

// One weighted-Jacobi update of a cell from its own and its neighbours'
// values: jacobi_at's arithmetic with the multiplications by the 0/1 mask
// dropped (u is masked -- zero on dry cells -- and winv = omega * inv_diag
// is zero there).  On a wet cell those multiply by 1 (exact); on a dry cell
// the result is u + 0 * r = 0, as the masked form gives (up to the sign of
// zero), so the values are the same.
template <typename T>
DEV T jac_v(T um, T ue, T uw, T un, T us, T cx, T cxw, T cy, T cys, T f, T winv, T dx2, T rdx2, T dy2, T rdy2,
            T lam) {
  const T lap = divd(cx * (ue - um) - cxw * (um - uw), dx2, rdx2) + divd(cy * (un - um) - cys * (um - us), dy2, rdy2);
  const T r = f - (lap - lam * um);
  return um + winv * r;
}

// Region geometry of a leg with halo H on a TX x TY tile.
struct LegShape {
  int RW, RH, RN, LR;  // LR: rows per thread
};
template <typename T>
__host__ __device__ inline LegShape leg_shape(int H, int nt) {
  LegShape g;
  g.RW = LegTile<T>::TX + 2 * H;
  g.RH = LegTile<T>::TY + 2 * H;
  g.RN = g.RW * g.RH;
  const int nseg = nt / g.RW;
  g.LR = nseg > 0 ? (g.RH + nseg - 1) / nseg : 1 << 20;
  return g;
}

// Coarse window of an up leg (prolongation sources of the region).
struct CoarseWin {
  int CX0, CY0, CW, CH;
};
__host__ __device__ inline CoarseWin coarse_win(int x0, int y0, int RW, int RH) {
  CoarseWin w;
  w.CX0 = (x0 >> 1) - 1;
  w.CY0 = (y0 >> 1) - 1;
  w.CW = ((x0 + RW - 1) >> 1) + 1 - w.CX0 + 1;
  w.CH = ((y0 + RH - 1) >> 1) + 1 - w.CY0 + 1;
  return w;
}

// Shared memory of a leg with k sweeps (both kinds): cx and two u buffers
// over the halo-(k + 1) region, and the up leg's coarse window (twice).
template <typename T>
static size_t leg_smem(int k) {
  const LegShape g = leg_shape<T>(k + 1, 1);
  const size_t CN = (size_t)((g.RW + 1) / 2 + 3) * ((g.RH + 1) / 2 + 3);
  return (3 * (size_t)g.RN + 2 * CN) * sizeof(T);
}

// Per-thread cell state of a leg: R register slots for the thread's rows.
template <typename T, int R>
struct LegCells {
  T u[R], f[R], w[R], cx[R], cy[R];
  unsigned wet = 0;   // bit i: row slot i is a wet cell
  T cy_south = T(0);  // cy of the row below the thread's first row
};

// The level's constants of the thread's cells (zero outside the level):
// mask bits, cx, cy, omega * inv_diag; cx also into the shared tile.
template <typename T, int R>
DEV void leg_load_constants(const Lev<T>& L, LegCells<T, R>& s, T* scx, int x0, int y0, int RW, int RH, int c,
                            int r0, int LR, bool act, T omega) {
  const int gx = x0 + c;
  const bool colg = act && gx >= 0 && gx < L.nx;
  T mv[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = r0 + i, gy = y0 + r;
    const bool in = colg && i < LR && r < RH && gy >= 0 && gy < L.ny;
    const size_t g = in ? (size_t)gy * L.nx + gx : 0;
    mv[i] = in ? L.mask[g] : T(0);
    s.cx[i] = in ? L.cx[g] : T(0);
    s.cy[i] = in ? L.cy[g] : T(0);
    s.w[i] = in ? L.inv[g] : T(0);
  }
  {
    const int gy = y0 + r0 - 1;
    const bool in = colg && r0 >= 1 && gy >= 0 && gy < L.ny;
    s.cy_south = in ? L.cy[(size_t)gy * L.nx + gx] : T(0);
  }
  s.wet = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    s.w[i] = omega * s.w[i];
    if (mv[i] != T(0)) s.wet |= 1u << i;
    if (act && i < LR && r0 + i < RH) scx[(r0 + i) * RW + c] = s.cx[i];
  }
}

// k Jacobi sweeps of the region held in (registers, A); returns the buffer
// holding the final u (the registers hold the thread's own final values).
template <typename T, int R>
DEV T* leg_sweeps(const Lev<T>& L, LegCells<T, R>& s, T* A, T* B, const T* scx, int k, int RW, int RH, int c,
                  int r0, int LR, bool act) {
  const bool colin = act && c >= 1 && c <= RW - 2;
  for (int sw = 0; sw < k; ++sw) {
    T us = (colin && r0 >= 1) ? A[(r0 - 1) * RW + c] : T(0);  // old u of the row below
    T cys = s.cy_south;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = r0 + i;
      if (act && i < LR && r < RH) {
        const T um = s.u[i];
        T nv = um;
        if (colin && r >= 1 && r <= RH - 2) {
          const int q = r * RW + c;
          const T un = (i + 1 < R && i + 1 < LR) ? s.u[i + 1 < R ? i + 1 : i] : A[q + RW];
          nv = jac_v(um, A[q + 1], A[q - 1], un, us, s.cx[i], scx[q - 1], s.cy[i], cys, s.f[i], s.w[i], L.dx2,
                     L.rdx2, L.dy2, L.rdy2, L.lam);
        }
        us = um;
        cys = s.cy[i];
        s.u[i] = nv;
        B[r * RW + c] = nv;
      }
    }
    __syncthreads();
    T* t = A;
    A = B;
    B = t;
  }
  return A;
}

// The legs' thread configurations: NT threads with R register rows each; the
// host takes the first that covers the region (LR <= R).  The legs are
// programmatic dependents: what the kernel before them wrote (f, u_init,
// u_pre, ec, ec_scale) is read only after grid_dep_wait, through L2
// (ld.global.cg), from pointers not marked __restrict__ -- a restrict-const
// load may be served by the read-only path or moved above the wait.
template <typename T, int NT, int R>
__global__ void __launch_bounds__(NT)
down_leg_kernel(Lev<T> L, const T* f, const T* u_init, int k, T omega, Lev<T> C) {
  constexpr int TX = LegTile<T>::TX, TY = LegTile<T>::TY;
  const int H = k + 1;
  const LegShape g = leg_shape<T>(H, NT);
  const int RW = g.RW, RH = g.RH, LR = g.LR;
  extern __shared__ __align__(16) unsigned char leg_raw[];
  T* scx = (T*)leg_raw;
  T* A = scx + g.RN;
  T* B = A + g.RN;
  const int x0 = blockIdx.x * TX - H, y0 = blockIdx.y * TY - H;
  const int seg = threadIdx.x / RW, c = threadIdx.x - seg * RW, r0 = seg * LR;
  const bool act = r0 < RH;
  LegCells<T, R> s;
  // the level's constants, then (after the previous kernel, which wrote f
  // and u_init) f and u_init
  leg_load_constants<T, R>(L, s, scx, x0, y0, RW, RH, c, r0, LR, act, omega);
  grid_dep_wait();
  {
    const int gx = x0 + c;
    const bool colg = act && gx >= 0 && gx < L.nx;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = r0 + i, gy = y0 + r;
      const bool in = colg && i < LR && r < RH && gy >= 0 && gy < L.ny;
      const size_t gg = in ? (size_t)gy * L.nx + gx : 0;
      s.f[i] = in ? __ldcg(f + gg) : T(0);
      s.u[i] = (in && u_init) ? __ldcg(u_init + gg) : T(0);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if (u_init) s.u[i] *= ((s.wet >> i) & 1u) ? T(1) : T(0);  // the sweeps take u masked
      if (act && i < LR && r0 + i < RH) A[(r0 + i) * RW + c] = s.u[i];
    }
  }
  __syncthreads();
  grid_dep_launch();  // the next kernel may start loading its constants
  A = leg_sweeps<T, R>(L, s, A, B, scx, k, RW, RH, c, r0, LR, act);
  B = A == scx + g.RN ? A + g.RN : scx + g.RN;
  // the tile's u, and its residual * mask (u is masked, so the neighbours'
  // masks multiply by 1 or meet a zero: restrict_at's values)
  T rm[R];
  {
    const bool colt = act && c >= H && c < H + TX;
    const int gx = x0 + c;
    T us = (colt && r0 >= 1) ? A[(r0 - 1) * RW + c] : T(0);
    T cys = s.cy_south;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = r0 + i;
      rm[i] = T(0);
      if (act && i < LR && r < RH) {
        const T um = s.u[i];
        if (colt && r >= H && r < H + TY) {
          const int gy = y0 + r;
          if (gy < L.ny && gx < L.nx) L.u[(size_t)gy * L.nx + gx] = um;
          const int q = r * RW + c;
          const T un = (i + 1 < R && i + 1 < LR) ? s.u[i + 1 < R ? i + 1 : i] : A[q + RW];
          const T ue = A[q + 1], uw = A[q - 1];
          const T mc = ((s.wet >> i) & 1u) ? T(1) : T(0);
          const T lap = divd(s.cx[i] * (ue - um) - scx[q - 1] * (um - uw), L.dx2, L.rdx2) +
                        divd(s.cy[i] * (un - um) - cys * (um - us), L.dy2, L.rdy2);
          rm[i] = ((s.f[i] - (lap - L.lam * um) * mc) * mc) * mc;
        }
        us = um;
        cys = s.cy[i];
      }
    }
  }
  __syncthreads();  // every read of A is done: A <- r * m, B <- m on the tile
  {
    const bool colt = act && c >= H && c < H + TX;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = r0 + i;
      if (colt && i < LR && r >= H && r < H + TY) {
        A[r * RW + c] = rm[i];
        B[r * RW + c] = ((s.wet >> i) & 1u) ? T(1) : T(0);
      }
    }
  }
  __syncthreads();
  constexpr int CX = TX / 2, CY = TY / 2;
  for (int q = threadIdx.x; q < CX * CY; q += NT) {
    const int Jl = q / CX, Il = q % CX;
    const int J = blockIdx.y * CY + Jl, I = blockIdx.x * CX + Il;
    if (J >= C.ny || I >= C.nx) continue;
    T sv[4], mv[4];
    const int dj[4] = {0, 1, 0, 1}, di[4] = {0, 0, 1, 1};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int kk = (H + 2 * Jl + dj[t]) * RW + (H + 2 * Il + di[t]);
      sv[t] = A[kk];
      mv[t] = B[kk];
    }
    const T sum4 = ((sv[0] + sv[1]) + sv[2]) + sv[3];
    const T cnt = ((mv[0] + mv[1]) + mv[2]) + mv[3];
    const size_t cc = (size_t)J * C.nx + I;
    C.f[cc] = (sum4 / (cnt > T(1) ? cnt : T(1))) * C.mask[cc];
  }
}

// out (tile) <- k sweeps from u_pre + P ec.  Halo k.
// ec_scale (may be null): the coarse correction is read as ec * (T)*ec_scale
// (the hybrid cycle's energy-optimal scaling, applied as the window loads).
template <typename T, int NT, int R>
__global__ void __launch_bounds__(NT)
up_leg_kernel(Lev<T> L, const T* f, const T* u_pre, Lev<T> C, const T* ec, int k, T omega, T* __restrict__ out,
              const double* ec_scale) {
  constexpr int TX = LegTile<T>::TX, TY = LegTile<T>::TY;
  const int H = k;
  const LegShape g = leg_shape<T>(H, NT);
  const int RW = g.RW, RH = g.RH, LR = g.LR;
  // the buffer layout of leg_smem(k) (sized for halo k + 1)
  const int RNmax = leg_shape<T>(k + 1, 1).RN;
  extern __shared__ __align__(16) unsigned char leg_raw[];
  T* scx = (T*)leg_raw;
  T* A = scx + RNmax;
  T* B = A + RNmax;
  T* sv = B + RNmax;  // coarse e * mask
  const int x0 = blockIdx.x * TX - H, y0 = blockIdx.y * TY - H;
  const CoarseWin cw = coarse_win(x0, y0, RW, RH);
  T* scm = sv + cw.CW * cw.CH;  // coarse mask
  const int seg = threadIdx.x / RW, c = threadIdx.x - seg * RW, r0 = seg * LR;
  const bool act = r0 < RH;
  LegCells<T, R> s;
  // constants first; the coarse correction ec, f and u_pre come from the
  // kernels before this one
  leg_load_constants<T, R>(L, s, scx, x0, y0, RW, RH, c, r0, LR, act, omega);
  grid_dep_wait();
  const T ew = ec_scale ? (T)__ldcg(ec_scale) : T(1);
  for (int q = threadIdx.x; q < cw.CW * cw.CH; q += NT) {
    const int J = cw.CY0 + q / cw.CW, I = cw.CX0 + q % cw.CW;
    const bool in = J >= 0 && J < C.ny && I >= 0 && I < C.nx;
    const size_t cc = in ? (size_t)J * C.nx + I : 0;
    const T cm = in ? C.mask[cc] : T(0);
    sv[q] = in ? (__ldcg(ec + cc) * ew) * cm : T(0);
    scm[q] = cm;
  }
  T up[R];
  const int gx = x0 + c;
  const bool colg = act && gx >= 0 && gx < L.nx;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = r0 + i, gy = y0 + r;
    const bool in = colg && i < LR && r < RH && gy >= 0 && gy < L.ny;
    const size_t gg = in ? (size_t)gy * L.nx + gx : 0;
    s.f[i] = in ? __ldcg(f + gg) : T(0);
    up[i] = in ? __ldcg(u_pre + gg) : T(0);
  }
  __syncthreads();
  grid_dep_launch();
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = r0 + i, gy = y0 + r;
    if (!(act && i < LR && r < RH)) continue;
    const bool in = colg && gy >= 0 && gy < L.ny;
    const T mf = ((s.wet >> i) & 1u) ? T(1) : T(0);
    T u = T(0);
    if (in) {
      const int J = gy >> 1, I = gx >> 1, sj = 2 * (gy & 1) - 1, si = 2 * (gx & 1) - 1;
      auto V = [&](int jj, int ii) -> T { return sv[(jj - cw.CY0) * cw.CW + (ii - cw.CX0)]; };
      auto M = [&](int jj, int ii) -> T { return scm[(jj - cw.CY0) * cw.CW + (ii - cw.CX0)]; };
      const T ws = ((T(9) * V(J, I) + T(3) * V(J, I + si)) + T(3) * V(J + sj, I)) + T(1) * V(J + sj, I + si);
      const T ds = ((T(9) * M(J, I) + T(3) * M(J, I + si)) + T(3) * M(J + sj, I)) + T(1) * M(J + sj, I + si);
      const T e = (ws / (ds > T(1) ? ds : T(1))) * mf;
      u = (up[i] + e) * mf;
    }
    s.u[i] = u;
    A[r * RW + c] = u;
  }
  __syncthreads();
  A = leg_sweeps<T, R>(L, s, A, B, scx, k, RW, RH, c, r0, LR, act);
  const bool colt = act && c >= H && c < H + TX && gx < L.nx;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = r0 + i, gy = y0 + r;
    if (colt && i < LR && r >= H && r < H + TY && gy < L.ny) out[(size_t)gy * L.nx + gx] = s.u[i];
  }
}

// masked_laplacian (iterative.py:144-191): periodic roll, (lap - lam psi_m) * m
template <typename T>
__global__ void masked_laplacian_kernel(const T* psi, const T* m, T* out, int ny, int nx, T dx, T dy, T lam) {
  const size_t n = (size_t)ny * nx;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(c / nx), i = (int)(c - (size_t)j * nx);
    const int ie = i + 1 == nx ? 0 : i + 1, iw = i == 0 ? nx - 1 : i - 1;
    const int jn = j + 1 == ny ? 0 : j + 1, js = j == 0 ? ny - 1 : j - 1;
    auto P = [&](int jj, int ii) { size_t k = (size_t)jj * nx + ii; return psi[k] * m[k]; };
    const T pm = P(j, i);
    const T lap = ((P(j, iw) + P(j, ie)) - T(2) * pm) / (dx * dx) + ((P(js, i) + P(jn, i)) - T(2) * pm) / (dy * dy);
    out[c] = (lap - lam * pm) * m[c];
  }
}

static int grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace mg
}  // namespace fvx

using namespace fvx;
using namespace fvx::mg;

struct fvx_mg {
  int nl = 0, lc = 0, n_pre = 6, n_post = 6, n_coarse = 50, dtype = 0;
  double* omega_scratch = nullptr;  // [2 * kOmegaBlocks partials, omega], ticket after it
  double omega = 0.95, lam = 0.0;
  std::vector<void*> allocs;
  LevArray<float> A32;
  LevArray<double> A64;  // FP64 plans: every level; FP32 plans: the coarsest level only
  Lev<double> L0d;  // finest operator in FP64 (residual checks of FP32 solves)
};

template <typename T>
static LevArray<T>& levs(fvx_mg* g);
template <>
LevArray<float>& levs<float>(fvx_mg* g) { return g->A32; }
template <>
LevArray<double>& levs<double>(fvx_mg* g) { return g->A64; }

static void mg_free(fvx_mg* g) {
  for (void* p : g->allocs) cudaFree(p);
  g->allocs.clear();
}

// Host FP64 hierarchy (build_multigrid_solver, multigrid.py:905-1062).
struct HostLevel {
  int ny, nx;
  double dx, dy;
  std::vector<double> mask, coeff, cx, cy, inv;
};

static void host_level_ops(HostLevel& L, double lam) {
  const int ny = L.ny, nx = L.nx;
  const size_t n = (size_t)ny * nx;
  L.cx.assign(n, 0.0);
  L.cy.assign(n, 0.0);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t c = (size_t)j * nx + i;
      if (i + 1 < nx) L.cx[c] = (0.5 * (L.coeff[c] + L.coeff[c + 1])) * (L.mask[c] * L.mask[c + 1]);
      if (j + 1 < ny) L.cy[c] = (0.5 * (L.coeff[c] + L.coeff[c + nx])) * (L.mask[c] * L.mask[c + nx]);
    }
  L.inv.assign(n, 0.0);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t c = (size_t)j * nx + i;
      const double cxw = i > 0 ? L.cx[c - 1] : 0.0, cys = j > 0 ? L.cy[c - nx] : 0.0;
      double d = -(L.cx[c] + cxw) / (L.dx * L.dx) - (L.cy[c] + cys) / (L.dy * L.dy) - lam;
      d *= L.mask[c];
      L.inv[c] = (std::fabs(d) > 1e-30 ? 1.0 / d : 0.0) * L.mask[c];
    }
}

template <typename T>
static int upload_levels(fvx_mg* g, std::vector<HostLevel>& H, int first = 0) {
  LevArray<T>& A = levs<T>(g);
  for (int l = first; l < g->nl; ++l) {
    HostLevel& h = H[l];
    Lev<T>& L = A.L[l];
    L.ny = h.ny; L.nx = h.nx;
    L.dx2 = (T)(h.dx * h.dx); L.dy2 = (T)(h.dy * h.dy);
    L.rdx2 = (T)(1.0 / (h.dx * h.dx)); L.rdy2 = (T)(1.0 / (h.dy * h.dy));
    L.lam = (T)g->lam;
    const size_t n = (size_t)h.ny * h.nx;
    T** bufs[7] = {&L.mask, &L.cx, &L.cy, &L.inv, &L.u, &L.f, &L.tmp};
    for (T** b : bufs) {
      if (cudaMalloc((void**)b, n * sizeof(T)) != cudaSuccess) return FVX_ERR_CUDA;
      g->allocs.push_back(*b);
      cudaMemset(*b, 0, n * sizeof(T));
    }
    std::vector<T> tmp(n);
    const std::vector<double>* src[4] = {&h.mask, &h.cx, &h.cy, &h.inv};
    T* dst[4] = {L.mask, L.cx, L.cy, L.inv};
    for (int k = 0; k < 4; ++k) {
      for (size_t c = 0; c < n; ++c) tmp[c] = (T)(*src[k])[c];
      if (cudaMemcpy(dst[k], tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return FVX_ERR_CUDA;
    }
  }
  return FVX_OK;
}

// mask: [ny, nx] float64 0/1 (host); coeff: [ny, nx] float64 or NULL.
extern "C" int fvx_mg_create(const double* mask, const double* coeff, int ny, int nx, double dx, double dy,
                             double lambda, int n_levels, int n_pre, int n_post, int n_coarse, double omega, int dtype,
                             fvx_mg** out) {
  if (!mask || !out) return FVX_ERR_ARG;
  *out = nullptr;
  if (ny < 1 || nx < 1 || n_pre < 0 || n_post < 0 || n_coarse < 0) return FVX_ERR_SHAPE;
  if (n_pre > kLegMaxSweeps || n_post > kLegMaxSweeps) return FVX_ERR_ARG;  // fused legs: <= 16 sweeps
  if (dtype != 0 && dtype != 1) return FVX_ERR_DTYPE;
  if (n_levels <= 0) {  // _compute_n_levels (multigrid.py:50-76)
    int a = ny, b = nx;
    n_levels = 1;
    while (a % 2 == 0 && b % 2 == 0 && a / 2 >= 8 && b / 2 >= 8) { a /= 2; b /= 2; ++n_levels; }
  }
  if (n_levels > kMaxLevels) return FVX_ERR_SHAPE;
  const int fac = 1 << (n_levels - 1);
  if (ny % fac || nx % fac) return FVX_ERR_SHAPE;
  std::vector<HostLevel> H(n_levels);
  H[0].ny = ny; H[0].nx = nx; H[0].dx = dx; H[0].dy = dy;
  const size_t n0 = (size_t)ny * nx;
  H[0].mask.assign(mask, mask + n0);
  H[0].coeff.resize(n0);
  for (size_t c = 0; c < n0; ++c) H[0].coeff[c] = (coeff ? coeff[c] : 1.0) * H[0].mask[c];
  for (int l = 0; l < n_levels; ++l) {
    host_level_ops(H[l], lambda);
    if (l + 1 < n_levels) {
      HostLevel& F = H[l];
      HostLevel& C = H[l + 1];
      C.ny = F.ny / 2; C.nx = F.nx / 2; C.dx = F.dx * 2.0; C.dy = F.dy * 2.0;
      const size_t nc = (size_t)C.ny * C.nx;
      C.mask.resize(nc);
      C.coeff.resize(nc);
      for (int J = 0; J < C.ny; ++J)
        for (int I = 0; I < C.nx; ++I) {
          const size_t a = (size_t)(2 * J) * F.nx + 2 * I, b = a + F.nx, c = a + 1, d = b + 1;
          const double avg = (((F.mask[a] + F.mask[b]) + F.mask[c]) + F.mask[d]) / 4.0;  // _restrict_mask
          const double mc = avg >= 0.5 ? 1.0 : 0.0;
          C.mask[(size_t)J * C.nx + I] = mc;
          const double s4 = ((F.coeff[a] * F.mask[a] + F.coeff[b] * F.mask[b]) + F.coeff[c] * F.mask[c]) +
                            F.coeff[d] * F.mask[d];
          const double cnt = ((F.mask[a] + F.mask[b]) + F.mask[c]) + F.mask[d];
          C.coeff[(size_t)J * C.nx + I] = (s4 / (cnt > 1.0 ? cnt : 1.0)) * mc;  // _restrict_coeff
        }
    }
  }
  fvx_mg* g = new fvx_mg();
  g->nl = n_levels; g->n_pre = n_pre; g->n_post = n_post; g->n_coarse = n_coarse;
  g->omega = omega; g->lam = lambda; g->dtype = dtype;
  g->lc = n_levels - 1;
  while (g->lc > 0 && (size_t)H[g->lc - 1].ny * H[g->lc - 1].nx <= (size_t)kCoarseCells) --g->lc;
  int rc = dtype == 0 ? upload_levels<float>(g, H) : upload_levels<double>(g, H);
  // FP32 plans keep an FP64 copy of the coarsest level: the coarsest-grid
  // solve of every V-cycle runs in FP64
  if (!rc && dtype == 0) rc = upload_levels<double>(g, H, n_levels - 1);
  if (!rc) {
    Lev<double>& D = g->L0d;
    D.ny = ny; D.nx = nx; D.dx2 = dx * dx; D.dy2 = dy * dy; D.rdx2 = 1.0 / (dx * dx); D.rdy2 = 1.0 / (dy * dy);
    D.lam = lambda; D.inv = D.u = D.f = D.tmp = nullptr;
    double** bufs[3] = {&D.mask, &D.cx, &D.cy};
    const std::vector<double>* src[3] = {&H[0].mask, &H[0].cx, &H[0].cy};
    for (int k = 0; k < 3 && !rc; ++k) {
      if (cudaMalloc((void**)bufs[k], n0 * sizeof(double)) != cudaSuccess) { rc = FVX_ERR_CUDA; break; }
      g->allocs.push_back(*bufs[k]);
      if (cudaMemcpy(*bufs[k], src[k]->data(), n0 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = FVX_ERR_CUDA;
    }
  }
  if (!rc) {
    // partial sums, omega and ticket of the hybrid cycle's energy-scaled
    // coarse correction, allocated here so that no solve-time call allocates
    const size_t bytes = (2 * kOmegaBlocks + 2) * sizeof(double);
    if (cudaMalloc((void**)&g->omega_scratch, bytes) != cudaSuccess) {
      g->omega_scratch = nullptr;
      rc = FVX_ERR_CUDA;
    } else {
      g->allocs.push_back(g->omega_scratch);
      if (cudaMemset(g->omega_scratch, 0, bytes) != cudaSuccess) rc = FVX_ERR_CUDA;
    }
  }
  if (rc) { mg_free(g); delete g; return rc; }
  if (cudaDeviceSynchronize() != cudaSuccess) { mg_free(g); delete g; return FVX_ERR_CUDA; }
  *out = g;
  return FVX_OK;
}

extern "C" int fvx_mg_destroy(fvx_mg* g) {
  if (!g) return FVX_ERR_ARG;
  cudaDeviceSynchronize();
  mg_free(g);
  delete g;
  return fvx_cuda_status();
}

// Level metadata and device arrays (mask, cx, cy, inv_diag) for inspection.
extern "C" int fvx_mg_level(fvx_mg* g, int level, int* ny, int* nx, double* dx2, void** mask, void** cx, void** cy,
                            void** inv) {
  if (!g || level < 0 || level >= g->nl) return FVX_ERR_ARG;
  if (g->dtype == 0) {
    Lev<float>& L = g->A32.L[level];
    *ny = L.ny; *nx = L.nx; *dx2 = L.dx2; *mask = L.mask; *cx = L.cx; *cy = L.cy; *inv = L.inv;
  } else {
    Lev<double>& L = g->A64.L[level];
    *ny = L.ny; *nx = L.nx; *dx2 = L.dx2; *mask = L.mask; *cx = L.cx; *cy = L.cy; *inv = L.inv;
  }
  return FVX_OK;
}

extern "C" int fvx_mg_num_levels(fvx_mg* g) { return g ? g->nl : -1; }

// The legs' thread configurations: 0 = (512 threads, 4 register rows),
// 1 = (512, 8), 2 = (1024, 4), 3 = (1024, 8); the first in the type's order
// whose rows cover the region is used.  FP32 prefers 1024 x 4 (63 registers:
// one CTA of 32 warps per SM); FP64 prefers 512 x 4 (1024 x 4 would spill),
// except on levels with fewer tiles than SMs, where more threads per tile
// shorten each CTA's sweeps.
constexpr int kLegNT[4] = {512, 512, 1024, 1024}, kLegR[4] = {4, 8, 4, 8};
template <typename T>
static int leg_config(int H, bool few) {
  static constexpr int order32[4] = {2, 3, 1, 0}, order64[4] = {0, 1, 2, 3}, order_few[4] = {2, 3, 0, 1};
  const int* order = few ? order_few : (sizeof(T) == 4 ? order32 : order64);
  for (int j = 0; j < 4; ++j) {
    const int i = order[j];
    if (leg_shape<T>(H, kLegNT[i]).LR <= kLegR[i]) return i;
  }
  return -1;
}

template <typename T>
static int leg_attr() {
  static fvx_once_per_device attr;
  return fvx_once_on_device(attr, [] {
    const int bytes = (int)leg_smem<T>(kLegMaxSweeps);
    return fvx_set_max_smem(down_leg_kernel<T, 512, 4>, bytes) && fvx_set_max_smem(down_leg_kernel<T, 512, 8>, bytes) &&
           fvx_set_max_smem(down_leg_kernel<T, 1024, 4>, bytes) &&
           fvx_set_max_smem(down_leg_kernel<T, 1024, 8>, bytes) && fvx_set_max_smem(up_leg_kernel<T, 512, 4>, bytes) &&
           fvx_set_max_smem(up_leg_kernel<T, 512, 8>, bytes) && fvx_set_max_smem(up_leg_kernel<T, 1024, 4>, bytes) &&
           fvx_set_max_smem(up_leg_kernel<T, 1024, 8>, bytes);
  });
}

// The single-CTA coarse V-cycle from level l (FP32 plans: in FP64).
template <typename T>
static int coarse_vcycle(fvx_mg* g, int l, cudaStream_t st) {
  if constexpr (sizeof(T) == 4)
    coarse_vcycle_f64_kernel<<<1, kCoarseThreads, 0, st>>>(g->A32, g->A64.L[g->nl - 1], l, g->nl, g->n_pre,
                                                           g->n_post, g->n_coarse, (float)g->omega);
  else
    coarse_vcycle_kernel<T><<<1, kCoarseThreads, 0, st>>>(levs<T>(g), l, g->nl, g->n_pre, g->n_post, g->n_coarse,
                                                          (T)g->omega);
  return fvx_cuda_status();
}

// Downward leg at host-driven level l: L.u <- k sweeps on f from u_init
// (NULL = 0), level l+1's f <- the restricted residual.
template <typename T>
static int leg_down(fvx_mg* g, int l, const T* f, const T* u_init, int k, cudaStream_t st) {
  if (k > kLegMaxSweeps) return FVX_ERR_ARG;
  int rc = leg_attr<T>();
  if (rc) return rc;
  LevArray<T>& A = levs<T>(g);
  Lev<T>& L = A.L[l];
  constexpr int TX = LegTile<T>::TX, TY = LegTile<T>::TY;
  dim3 gr((L.nx + TX - 1) / TX, (L.ny + TY - 1) / TY);
  // programmatic launch: the constants load while the kernel before
  // finishes (the kernel waits before reading f and u_init)
  const int cfg = leg_config<T>(k + 1, (size_t)gr.x * gr.y < (size_t)kLegFewTiles);
  const size_t sm = leg_smem<T>(k);
  const Lev<T>& C = A.L[l + 1];
  const T om = (T)g->omega;
  cudaError_t e = cudaErrorInvalidValue;
  switch (cfg) {
    case 0: e = fvx_launch_pdl(down_leg_kernel<T, 512, 4>, gr, dim3(512), sm, st, L, f, u_init, k, om, C); break;
    case 1: e = fvx_launch_pdl(down_leg_kernel<T, 512, 8>, gr, dim3(512), sm, st, L, f, u_init, k, om, C); break;
    case 2: e = fvx_launch_pdl(down_leg_kernel<T, 1024, 4>, gr, dim3(1024), sm, st, L, f, u_init, k, om, C); break;
    case 3: e = fvx_launch_pdl(down_leg_kernel<T, 1024, 8>, gr, dim3(1024), sm, st, L, f, u_init, k, om, C); break;
    default: return FVX_ERR_ARG;
  }
  if (e != cudaSuccess) return FVX_ERR_CUDA;
  return fvx_cuda_status();
}

// Upward leg at host-driven level l: out <- k sweeps on f from L.u + P ec.
template <typename T>
static int leg_up(fvx_mg* g, int l, const T* f, const T* ec, int k, T* out, cudaStream_t st,
                  const double* ec_scale = nullptr) {
  if (k > kLegMaxSweeps) return FVX_ERR_ARG;
  int rc = leg_attr<T>();
  if (rc) return rc;
  LevArray<T>& A = levs<T>(g);
  Lev<T>& L = A.L[l];
  constexpr int TX = LegTile<T>::TX, TY = LegTile<T>::TY;
  dim3 gr((L.nx + TX - 1) / TX, (L.ny + TY - 1) / TY);
  const int cfg = leg_config<T>(k + 1, (size_t)gr.x * gr.y < (size_t)kLegFewTiles);
  const size_t sm = leg_smem<T>(k);
  const Lev<T>& C = A.L[l + 1];
  const T om = (T)g->omega;
  const T* up = L.u;
  cudaError_t e = cudaErrorInvalidValue;
  switch (cfg) {
    case 0: e = fvx_launch_pdl(up_leg_kernel<T, 512, 4>, gr, dim3(512), sm, st, L, f, up, C, ec, k, om, out, ec_scale); break;
    case 1: e = fvx_launch_pdl(up_leg_kernel<T, 512, 8>, gr, dim3(512), sm, st, L, f, up, C, ec, k, om, out, ec_scale); break;
    case 2: e = fvx_launch_pdl(up_leg_kernel<T, 1024, 4>, gr, dim3(1024), sm, st, L, f, up, C, ec, k, om, out, ec_scale); break;
    case 3: e = fvx_launch_pdl(up_leg_kernel<T, 1024, 8>, gr, dim3(1024), sm, st, L, f, up, C, ec, k, om, out, ec_scale); break;
    default: return FVX_ERR_ARG;
  }
  if (e != cudaSuccess) return FVX_ERR_CUDA;
  return fvx_cuda_status();
}

// V-cycle below the finest level of a host-driven cycle: entered with
// L[l].f set, zero initial guess; returns where level l's result lives
// (L[l].u for the single-CTA coarse levels, L[l].tmp for host-driven ones).
template <typename T>
static int vcycle_levels(fvx_mg* g, int l, T** result, cudaStream_t st) {
  LevArray<T>& A = levs<T>(g);
  const T om = (T)g->omega;
  if (l >= g->lc) {
    *result = A.L[l].u;
    return coarse_vcycle<T>(g, l, st);
  }
  Lev<T>& L = A.L[l];
  int rc = leg_down<T>(g, l, L.f, nullptr, g->n_pre, st);
  if (rc) return rc;
  T* ec = nullptr;
  if ((rc = vcycle_levels<T>(g, l + 1, &ec, st))) return rc;
  if ((rc = leg_up<T>(g, l, L.f, ec, g->n_post, L.tmp, st))) return rc;
  *result = L.tmp;
  return FVX_OK;
}

// One V-cycle at level 0: u_out = V(u_in, f) (u_in NULL = zero initial
// guess).  u_in and u_out may alias.  Arrays are [ny, nx] of the plan dtype.
template <typename T>
static int vcycle0(fvx_mg* g, const T* u_in, const T* f, T* u_out, cudaStream_t st) {
  LevArray<T>& A = levs<T>(g);
  Lev<T>& L = A.L[0];
  const size_t n = (size_t)L.ny * L.nx;
  const int gr = grid_for(n);
  const T om = (T)g->omega;
  if (g->nl == 1) {
    if (u_in) copy_kernel<T><<<gr, 256, 0, st>>>(L.u, u_in, n);
    else fill_kernel<T><<<gr, 256, 0, st>>>(L.u, n, T(0));
    copy_kernel<T><<<gr, 256, 0, st>>>(L.f, f, n);
    T* a = L.u; T* b = L.tmp;
    for (int s = 0; s < g->n_coarse; ++s) { jacobi_kernel<T><<<gr, 256, 0, st>>>(L, a, L.f, b, om); T* t = a; a = b; b = t; }
    copy_kernel<T><<<gr, 256, 0, st>>>(u_out, a, n);
    return fvx_cuda_status();
  }
  if (g->lc == 0 && !u_in) {  // whole cycle fits the single-CTA kernel
    copy_kernel<T><<<gr, 256, 0, st>>>(L.f, f, n);
    int rc = coarse_vcycle<T>(g, 0, st);
    if (rc) return rc;
    copy_kernel<T><<<gr, 256, 0, st>>>(u_out, L.u, n);
    return fvx_cuda_status();
  }
  int rc = leg_down<T>(g, 0, f, u_in, g->n_pre, st);
  if (rc) return rc;
  T* ec = nullptr;
  if ((rc = vcycle_levels<T>(g, 1, &ec, st))) return rc;
  return leg_up<T>(g, 0, f, ec, g->n_post, u_out, st);
}

extern "C" int fvx_mg_vcycle(fvx_mg* g, const void* u_in, const void* f, void* u_out, void* stream) {
  if (!g || !f || !u_out) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  return g->dtype == 0 ? vcycle0<float>(g, (const float*)u_in, (const float*)f, (float*)u_out, st)
                       : vcycle0<double>(g, (const double*)u_in, (const double*)f, (double*)u_out, st);
}

// ---------------------------------------------------------------------------
// Hybrid cycle for a learned coarse solver: the V-cycle's legs on levels
// 0 .. lvl-1 (n_pre / n_post weighted-Jacobi sweeps from a zero guess, the
// reference's restriction and prolongation) with the level-lvl correction
// supplied by ``coarse(ctx, f_lvl, u_lvl, stream)``, which reads the
// restricted residual f_lvl and writes u_lvl (both [ny_lvl, nx_lvl], plan
// dtype).  With ``coarse`` NULL the correction is zero.
template <typename T>
static int hybrid_down(fvx_mg* g, const T* f, int lvl, int n_pre, cudaStream_t st) {
  LevArray<T>& A = levs<T>(g);
  for (int l = 0; l < lvl; ++l) {
    int rc = leg_down<T>(g, l, l == 0 ? f : A.L[l].f, nullptr, n_pre, st);
    if (rc) return rc;
  }
  return FVX_OK;
}

// ec_scale (may be null): scale of the level-lvl correction, applied by the
// first upward leg as it reads it.
template <typename T>
static int hybrid_up(fvx_mg* g, const T* f, T* u_out, int lvl, int n_post, cudaStream_t st,
                     const double* ec_scale = nullptr) {
  LevArray<T>& A = levs<T>(g);
  for (int l = lvl - 1; l >= 0; --l) {
    const T* ec = l + 1 == lvl ? A.L[lvl].u : A.L[l + 1].tmp;
    int rc = leg_up<T>(g, l, l == 0 ? f : A.L[l].f, ec, n_post, l == 0 ? u_out : A.L[l].tmp, st,
                       l + 1 == lvl ? ec_scale : nullptr);
    if (rc) return rc;
  }
  return FVX_OK;
}

// n_smooth: weighted-Jacobi sweeps on A_lvl e = f_lvl after the coarse
// correction (they damp the high-frequency error a learned solver leaves).
// scale: the coarse correction is first scaled by the energy-optimal omega.
template <typename T>
static int hybrid_cycle(fvx_mg* g, const T* f, T* u_out, int lvl, int n_pre, int n_post, int n_smooth, int scale,
                        fvx_precond_fn coarse, void* ctx, cudaStream_t st) {
  if (n_pre > kLegMaxSweeps || n_post > kLegMaxSweeps || n_smooth < 0) return FVX_ERR_ARG;
  int rc = hybrid_down<T>(g, f, lvl, n_pre, st);
  if (rc) return rc;
  Lev<T>& C = levs<T>(g).L[lvl];
  const size_t nc = (size_t)C.ny * C.nx;
  const double* omega_in_leg = nullptr;
  if (coarse) {
    if ((rc = coarse(ctx, C.f, C.u, st))) return rc;
    if (scale) {
      double* part = g->omega_scratch;
      double* om = part + 2 * kOmegaBlocks;
      unsigned* ticket = (unsigned*)(om + 1);
      k_coarse_omega<T><<<kOmegaBlocks, 256, 0, st>>>(C, part, ticket, om);
      // without smoothing sweeps at level lvl the first upward leg applies
      // omega as it reads the correction; the sweeps need it applied first
      if (n_smooth > 0) k_scale<T><<<grid_for(nc), 256, 0, st>>>(C.u, nc, om);
      else omega_in_leg = om;
    }
  } else {
    fill_kernel<T><<<grid_for(nc), 256, 0, st>>>(C.u, nc, T(0));
  }
  if (n_smooth > 0) {
    T* a = C.u;
    T* b = C.tmp;
    for (int k = 0; k < n_smooth; ++k) {
      jacobi_kernel<T><<<grid_for(nc), 256, 0, st>>>(C, a, C.f, b, (T)g->omega);
      T* t = a; a = b; b = t;
    }
    if (a != C.u) copy_kernel<T><<<grid_for(nc), 256, 0, st>>>(C.u, a, nc);
  }
  return hybrid_up<T>(g, f, u_out, lvl, n_post, st, omega_in_leg);
}

extern "C" int fvx_mg_vcycle_hybrid(fvx_mg* g, const void* f, void* u_out, int lvl, int n_pre, int n_post,
                                    int n_smooth, int scale, fvx_precond_fn coarse, void* ctx, void* stream) {
  if (!g || !f || !u_out || n_pre < 0 || n_post < 0) return FVX_ERR_ARG;
  if (lvl < 1 || lvl >= g->nl) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  return g->dtype == 0 ? hybrid_cycle<float>(g, (const float*)f, (float*)u_out, lvl, n_pre, n_post, n_smooth, scale,
                                             coarse, ctx, st)
                       : hybrid_cycle<double>(g, (const double*)f, (double*)u_out, lvl, n_pre, n_post, n_smooth,
                                              scale, coarse, ctx, st);
}

// The hybrid cycle packaged as a preconditioner callback (ctx = the
// fvx_hybrid object) for fvx_pcg_solve / fvx_pcg_iterate with precond 2.
struct fvx_hybrid {
  fvx_mg* g;
  int lvl, n_pre, n_post, n_smooth, scale;
  fvx_precond_fn coarse;
  void* ctx;
};

extern "C" int fvx_hybrid_create(fvx_mg* g, int lvl, int n_pre, int n_post, int n_smooth, int scale,
                                 fvx_precond_fn coarse, void* ctx, fvx_hybrid** out) {
  if (!g || !out || n_pre < 0 || n_post < 0 || n_smooth < 0) return FVX_ERR_ARG;
  if (n_pre > kLegMaxSweeps || n_post > kLegMaxSweeps) return FVX_ERR_ARG;
  if (lvl < 1 || lvl >= g->nl) return FVX_ERR_SHAPE;
  *out = new fvx_hybrid{g, lvl, n_pre, n_post, n_smooth, scale, coarse, ctx};
  return FVX_OK;
}

extern "C" int fvx_hybrid_destroy(fvx_hybrid* h) {
  delete h;
  return FVX_OK;
}

extern "C" int fvx_hybrid_precond(void* ctx, const void* rho, void* z, void* stream) {
  fvx_hybrid* h = (fvx_hybrid*)ctx;
  if (!h) return FVX_ERR_ARG;
  return fvx_mg_vcycle_hybrid(h->g, rho, z, h->lvl, h->n_pre, h->n_post, h->n_smooth, h->scale, h->coarse, h->ctx,
                              stream);
}


// Multigrid as the level-lvl solver of the hybrid cycle (n_cycles cycles
// from zero, one CTA): the exact-coarse-solve limit a learned coarse solver
// is measured against.  An fvx_precond_fn with ctx = the fvx_levelsolve.
struct fvx_levelsolve {
  fvx_mg* g;
  int lvl, n_cycles;
  void* work;
};

extern "C" int fvx_mg_solve_level_batched(fvx_mg* g, int lvl, int batch, const void* f, void* u, int n_cycles,
                                          void* work, void* stream);
extern "C" long long fvx_mg_level_work(fvx_mg* g, int lvl);

extern "C" int fvx_levelsolve_create(fvx_mg* g, int lvl, int n_cycles, fvx_levelsolve** out) {
  if (!g || !out || n_cycles < 1) return FVX_ERR_ARG;
  if (lvl < 0 || lvl >= g->nl) return FVX_ERR_SHAPE;
  void* w = nullptr;
  const size_t bytes = (size_t)fvx_mg_level_work(g, lvl) * (g->dtype == 0 ? 4 : 8);
  if (cudaMalloc(&w, bytes) != cudaSuccess) return FVX_ERR_CUDA;
  *out = new fvx_levelsolve{g, lvl, n_cycles, w};
  return FVX_OK;
}

extern "C" int fvx_levelsolve_destroy(fvx_levelsolve* s) {
  if (!s) return FVX_OK;
  cudaDeviceSynchronize();
  cudaFree(s->work);
  delete s;
  return fvx_cuda_status();
}

extern "C" int fvx_levelsolve_coarse(void* ctx, const void* f, void* u, void* stream) {
  fvx_levelsolve* s = (fvx_levelsolve*)ctx;
  if (!s) return FVX_ERR_ARG;
  return fvx_mg_solve_level_batched(s->g, s->lvl, 1, f, u, s->n_cycles, s->work, stream);
}

// The downward leg only: the level-lvl restricted residual of f, copied to
// f_lvl ([ny_lvl, nx_lvl]); used to generate training inputs.
extern "C" int fvx_mg_restrict_residual(fvx_mg* g, const void* f, int lvl, int n_pre, void* f_lvl, void* stream) {
  if (!g || !f || !f_lvl || n_pre < 0) return FVX_ERR_ARG;
  if (lvl < 1 || lvl >= g->nl) return FVX_ERR_SHAPE;
  cudaStream_t st = fvx_stream(stream);
  if (g->dtype == 0) {
    int rc = hybrid_down<float>(g, (const float*)f, lvl, n_pre, st);
    Lev<float>& C = g->A32.L[lvl];
    const size_t n = (size_t)C.ny * C.nx;
    copy_kernel<float><<<grid_for(n), 256, 0, st>>>((float*)f_lvl, C.f, n);
    return rc ? rc : fvx_cuda_status();
  }
  int rc = hybrid_down<double>(g, (const double*)f, lvl, n_pre, st);
  Lev<double>& C = g->A64.L[lvl];
  const size_t n = (size_t)C.ny * C.nx;
  copy_kernel<double><<<grid_for(n), 256, 0, st>>>((double*)f_lvl, C.f, n);
  return rc ? rc : fvx_cuda_status();
}

// Scratch elements per right-hand side for fvx_mg_solve_level_batched.
extern "C" long long fvx_mg_level_work(fvx_mg* g, int lvl) {
  if (!g || lvl < 0 || lvl >= g->nl) return -1;
  long long w = 0;
  for (int l = lvl; l < g->nl; ++l)
    w += g->dtype == 0 ? 3LL * g->A32.L[l].ny * g->A32.L[l].nx : 3LL * g->A64.L[l].ny * g->A64.L[l].nx;
  return w;
}

// ``batch`` independent solves A_lvl u_b = f_b at level lvl (MG cycles run
// by one CTA each); f, u: [batch, ny_lvl, nx_lvl]; work: batch *
// fvx_mg_level_work(g, lvl) elements of the plan dtype.
extern "C" int fvx_mg_solve_level_batched(fvx_mg* g, int lvl, int batch, const void* f, void* u, int n_cycles,
                                          void* work, void* stream) {
  if (!g || !f || !u || !work || batch < 0 || n_cycles < 1) return FVX_ERR_ARG;
  if (lvl < 0 || lvl >= g->nl) return FVX_ERR_SHAPE;
  if (batch == 0) return FVX_OK;
  cudaStream_t st = fvx_stream(stream);
  const size_t wpb = (size_t)fvx_mg_level_work(g, lvl);
  if (g->dtype == 0)
    coarse_solve_batched_kernel<float><<<batch, kCoarseThreads, 0, st>>>(
        g->A32, lvl, g->nl, g->n_pre, g->n_post, g->n_coarse, (float)g->omega, (const float*)f, (float*)u,
        (float*)work, wpb, n_cycles);
  else
    coarse_solve_batched_kernel<double><<<batch, kCoarseThreads, 0, st>>>(
        g->A64, lvl, g->nl, g->n_pre, g->n_post, g->n_coarse, g->omega, (const double*)f, (double*)u,
        (double*)work, wpb, n_cycles);
  return fvx_cuda_status();
}

// MultigridSolver._run_vcycles (multigrid.py:885-897): n_cycles V-cycles from 0.
extern "C" int fvx_mg_solve(fvx_mg* g, const void* f, void* u, int n_cycles, void* stream) {
  if (!g || !f || !u || n_cycles < 0) return FVX_ERR_ARG;
  int rc = FVX_OK;
  for (int k = 0; k < n_cycles && rc == FVX_OK; ++k) rc = fvx_mg_vcycle(g, k == 0 ? nullptr : u, f, u, stream);
  if (n_cycles == 0) {
    const size_t n = g->dtype == 0 ? (size_t)g->A32.L[0].ny * g->A32.L[0].nx : (size_t)g->A64.L[0].ny * g->A64.L[0].nx;
    rc = cudaMemsetAsync(u, 0, n * (g->dtype == 0 ? 4 : 8), fvx_stream(stream)) == cudaSuccess ? FVX_OK : FVX_ERR_CUDA;
  }
  return rc;
}

// _apply_operator at a level: out = A u.
extern "C" int fvx_mg_apply(fvx_mg* g, int level, const void* u, void* out, void* stream) {
  if (!g || !u || !out || level < 0 || level >= g->nl) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  if (g->dtype == 0) {
    Lev<float>& L = g->A32.L[level];
    apply_kernel<float><<<grid_for((size_t)L.ny * L.nx), 256, 0, st>>>(L, (const float*)u, (float*)out);
  } else {
    Lev<double>& L = g->A64.L[level];
    apply_kernel<double><<<grid_for((size_t)L.ny * L.nx), 256, 0, st>>>(L, (const double*)u, (double*)out);
  }
  return fvx_cuda_status();
}

#define FVX_DEF_MLAP(SFX, T)                                                                                   \
  extern "C" int fvx_masked_laplacian_##SFX(const T* psi, const T* mask, T* out, int ny, int nx, double dx,   \
                                            double dy, double lambda, void* stream) {                         \
    if (!psi || !mask || !out) return FVX_ERR_ARG;                                                             \
    if (ny < 1 || nx < 1) return FVX_ERR_SHAPE;                                                                \
    masked_laplacian_kernel<T><<<grid_for((size_t)ny * nx), 256, 0, fvx_stream(stream)>>>(psi, mask, out, ny,  \
                                                                                          nx, T(dx), T(dy),     \
                                                                                          T(lambda));           \
    return fvx_cuda_status();                                                                                  \
  }
FVX_DEF_MLAP(f32, float)
FVX_DEF_MLAP(f64, double)

// ===========================================================================
// Preconditioned CG on the finest operator A (negative definite, like
// solve_cg's operators, iterative.py:97-127): CG with A and a negative-
// definite preconditioner M is the SPD recurrence on (-A, -M) written with
// the natural residual rho = b - A x.  x is FP64; rho, z, p, A p are T;
// every inner product accumulates in FP64 (warp shuffles, then one block
// per reduction in a fixed order, so results are deterministic); every
// ``replace_every`` iterations rho is recomputed from x in FP64.  All
// scalars stay on the device and every kernel returns at once when the
// convergence flag is set, so the host only reads the flag every ``chunk``
// iterations.
// ===========================================================================
namespace fvx {
namespace mg {

enum Slot { S_GAMMA = 0, S_PAP, S_ALPHA, S_BETA, S_RR, S_BB, S_CONV, S_ITER, S_TOL2, S_FLEX_A, S_NSLOTS = 16 };
constexpr int kRedBlocks = 296;  // 2 per SM


template <typename T>
__global__ void k_apply_dot(Lev<T> L, const T* p, T* Ap, double* part, const double* s) {
  if (s[S_CONV] != 0.0) return;
  const size_t n = (size_t)L.ny * L.nx;
  double acc = 0.0;
  (void)n;
  grid_cells(L.ny, L.nx, [&](size_t c, int j, int i) {
    const T a = apply_at(L, p, j, i);
    Ap[c] = a;
    acc += (double)p[c] * (double)a;
  });
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

template <typename T>
__global__ void k_update(double* x, const T* p, const T* Ap, T* rho, T* rho_prev, double* part, const double* s,
                         size_t N) {
  if (s[S_CONV] != 0.0) return;
  const double a = s[S_ALPHA];
  double acc = 0.0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (size_t)gridDim.x * blockDim.x) {
    x[c] += a * (double)p[c];
    if (rho_prev) rho_prev[c] = rho[c];
    const T r = rho[c] - (T)a * Ap[c];
    rho[c] = r;
    acc += (double)r * (double)r;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// rho = b - A x in FP64 (x FP64, b of type T), rho stored as T; part = |rho|^2
template <typename T>
__global__ void k_residual64(Lev<double> D, const double* x, const T* b, T* rho, double* part, const double* s,
                             int force) {
  if (!force && s[S_CONV] != 0.0) return;
  const size_t n = (size_t)D.ny * D.nx;
  double acc = 0.0;
  (void)n;
  grid_cells(D.ny, D.nx, [&](size_t c, int j, int i) {
    const double r = (double)b[c] - apply_at(D, x, j, i);
    if (rho) rho[c] = (T)r;
    acc += r * r;
  });
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

template <typename T>
__global__ void k_dot(const T* a, const T* b, const T* c2, double* part, double* part2, const double* s, size_t n) {
  if (s[S_CONV] != 0.0) return;
  double acc = 0.0, acc2 = 0.0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    acc += (double)a[c] * (double)b[c];
    if (c2) acc2 += (double)a[c] * (double)c2[c];
  }
  acc = block_sum(acc);
  if (c2) acc2 = block_sum(acc2);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = acc;
    if (c2) part2[blockIdx.x] = acc2;
  }
}

template <typename T>
__global__ void k_pupdate(T* p, const T* z, const double* s, size_t n) {
  if (s[S_CONV] != 0.0) return;
  const T b = (T)s[S_BETA];
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    p[c] = z[c] + b * p[c];
}

template <typename T>
__global__ void k_copy_if(T* dst, const T* src, size_t n, const double* s) {
  if (s[S_CONV] != 0.0) return;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    dst[c] = src[c];
}

enum RedMode { R_STORE = 0, R_ALPHA, R_BETA, R_RR, R_BETA_FLEX };

// One block: fixed-order sum of the partials, then the scalar update.
__global__ void k_reduce(const double* part, const double* part2, int np, double* s, int slot, int mode, int force) {
  if (!force && s[S_CONV] != 0.0) return;
  double v = 0.0, v2 = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) {
    v += part[k];
    if (part2) v2 += part2[k];
  }
  v = block_sum(v);
  if (part2) v2 = block_sum(v2);
  if (threadIdx.x != 0) return;
  switch (mode) {
    case R_STORE: s[slot] = v; break;
    case R_ALPHA: s[S_PAP] = v; s[S_ALPHA] = s[S_GAMMA] / v; break;
    case R_BETA: s[S_BETA] = v / s[S_GAMMA]; s[S_GAMMA] = v; break;
    case R_BETA_FLEX: s[S_BETA] = (v - v2) / s[S_GAMMA]; s[S_GAMMA] = v; break;  // Polak-Ribiere
    case R_RR:
      s[S_RR] = v;
      s[S_ITER] += 1.0;
      if (v <= s[S_TOL2]) s[S_CONV] = 1.0;
      break;
  }
}

template <typename T>
__global__ void k_zero_x(double* x, size_t n) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) x[c] = 0.0;
}

// ---- fused iteration kernels (one pass each over the level-0 arrays) ------
constexpr int kPcgBlocks = 148 * 4;

// A u at (j, i) with u given as a function of the flat index (apply_at's
// arithmetic, in its order).
template <typename T, typename U>
DEV T apply_fn(const Lev<T>& L, int j, int i, U u) {
  const int nx = L.nx, ny = L.ny;
  const size_t c = (size_t)j * nx + i;
  const T m = L.mask[c];
  const T um = u(c) * m;
  const T ue = i + 1 < nx ? u(c + 1) * L.mask[c + 1] : T(0);
  const T uw = i > 0 ? u(c - 1) * L.mask[c - 1] : T(0);
  const T un = j + 1 < ny ? u(c + nx) * L.mask[c + nx] : T(0);
  const T us = j > 0 ? u(c - nx) * L.mask[c - nx] : T(0);
  const T cxw = i > 0 ? L.cx[c - 1] : T(0);
  const T cys = j > 0 ? L.cy[c - nx] : T(0);
  const T lap = divd(L.cx[c] * (ue - um) - cxw * (um - uw), L.dx2, L.rdx2) +
                divd(L.cy[c] * (un - um) - cys * (um - us), L.dy2, L.rdy2);
  return (lap - L.lam * um) * m;
}


DEV double pcg_sum_parts(const double* part, int np) {
  __threadfence();
  double v = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) v += ((volatile const double*)part)[k];
  return block_sum(v);
}

// p_new = z + beta p_old (recomputed at the neighbours), Ap = A p_new,
// partial p.Ap; the last block sets alpha = gamma / p.Ap.  p ping-pongs
// between p0 and p1 by the iteration count.
template <typename T>
__global__ void __launch_bounds__(256)
k_dir_apply(Lev<T> L, const T* __restrict__ z, T* p0, T* p1, T* __restrict__ Ap, double* part, double* s,
            unsigned* ticket) {
  if (s[S_CONV] != 0.0) return;
  const int it = (int)s[S_ITER];
  const T* po = (it & 1) ? p1 : p0;
  T* pn = (it & 1) ? p0 : p1;
  const T beta = (T)s[S_BETA];
  const size_t n = (size_t)L.ny * L.nx;
  double acc = 0.0;
  auto P = [&](size_t k) -> T { return z[k] + beta * po[k]; };
  (void)n;
  grid_cells(L.ny, L.nx, [&](size_t c, int j, int i) {
    const T pc = P(c);
    const T a = apply_fn(L, j, i, P);
    pn[c] = pc;
    Ap[c] = a;
    acc += (double)pc * (double)a;
  });
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
  if (pcg_last_block(ticket)) {
    const double v = pcg_sum_parts(part, gridDim.x);
    if (threadIdx.x == 0) {
      s[S_PAP] = v;
      s[S_ALPHA] = s[S_GAMMA] / v;
      *ticket = 0u;
    }
  }
}

// x_new = x + alpha p (FP64, ping-pong x0/x1), then rho: every
// ``replace_every``-th iteration the true residual b - A x_new in FP64
// (x_new recomputed at the neighbours, A the FP64 operator), otherwise the
// recursion rho - alpha Ap; partial |rho|^2.  The last block counts the
// iteration and sets the convergence flag.
template <typename T>
__global__ void __launch_bounds__(256)
k_step(Lev<double> D, const T* p0, const T* p1, const T* __restrict__ Ap, double* x0, double* x1,
       const T* __restrict__ b, T* rho, T* rho_prev, int replace_every, double* part, double* s, unsigned* ticket) {
  if (s[S_CONV] != 0.0) return;
  const int it = (int)s[S_ITER];
  const T* pn = (it & 1) ? p0 : p1;
  const double* xo = (it & 1) ? x1 : x0;
  double* xn = (it & 1) ? x0 : x1;
  const double a = s[S_ALPHA];
  const bool true_res = replace_every > 0 && (it + 1) % replace_every == 0;
  const size_t n = (size_t)D.ny * D.nx;
  double acc = 0.0;
  auto X = [&](size_t k) -> double { return xo[k] + a * (double)pn[k]; };
  (void)n;
  grid_cells(D.ny, D.nx, [&](size_t c, int j, int i) {
    const double xc = X(c);
    xn[c] = xc;
    const T ro = rho[c];
    if (rho_prev) rho_prev[c] = ro;
    if (true_res) {
      const double r = (double)b[c] - apply_fn(D, j, i, X);
      rho[c] = (T)r;
      acc += r * r;
    } else {
      const T r = ro - (T)a * Ap[c];
      rho[c] = r;
      acc += (double)r * (double)r;
    }
  });
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
  if (pcg_last_block(ticket)) {
    const double v = pcg_sum_parts(part, gridDim.x);
    if (threadIdx.x == 0) {
      s[S_RR] = v;
      s[S_ITER] += 1.0;
      if (v <= s[S_TOL2]) s[S_CONV] = 1.0;
      *ticket = 0u;
    }
  }
}

// gamma_new = z.rho; flexible: beta = (z.rho - z.rho_prev) / gamma
// (Polak-Ribiere), else gamma_new / gamma.
template <typename T>
__global__ void __launch_bounds__(256)
k_dot_beta(const T* __restrict__ z, const T* __restrict__ rho, const T* __restrict__ rho_prev, size_t n,
           double* part, double* part2, double* s, unsigned* ticket) {
  if (s[S_CONV] != 0.0) return;
  double acc = 0.0, acc2 = 0.0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const double zc = (double)z[c];
    acc += zc * (double)rho[c];
    if (rho_prev) acc2 += zc * (double)rho_prev[c];
  }
  acc = block_sum(acc);
  if (rho_prev) acc2 = block_sum(acc2);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = acc;
    if (rho_prev) part2[blockIdx.x] = acc2;
  }
  if (pcg_last_block(ticket)) {
    const double v = pcg_sum_parts(part, gridDim.x);
    const double v2 = rho_prev ? pcg_sum_parts(part2, gridDim.x) : 0.0;
    if (threadIdx.x == 0) {
      s[S_BETA] = (v - v2) / s[S_GAMMA];
      s[S_GAMMA] = v;
      *ticket = 0u;
    }
  }
}

}  // namespace mg
}  // namespace fvx

struct fvx_pcg {
  fvx_mg* mg = nullptr;
  int dtype = 0;
  size_t n = 0;
  void *rho = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *rho_prev = nullptr, *p1 = nullptr;
  double* x1 = nullptr;                       // second FP64 iterate buffer (ping-pong with the caller's x)
  void *own_rho = nullptr, *own_z = nullptr;  // allocations replaced by bound caller buffers
  double *part = nullptr, *part2 = nullptr, *s = nullptr;
  unsigned* ticket = nullptr;
};

extern "C" int fvx_pcg_create(fvx_mg* g, fvx_pcg** out) {
  if (!g || !out) return FVX_ERR_ARG;
  fvx_pcg* P = new fvx_pcg();
  P->mg = g;
  P->dtype = g->dtype;
  P->n = g->dtype == 0 ? (size_t)g->A32.L[0].ny * g->A32.L[0].nx : (size_t)g->A64.L[0].ny * g->A64.L[0].nx;
  const size_t es = g->dtype == 0 ? 4 : 8;
  bool ok = true;
  void** vecs[6] = {&P->rho, &P->z, &P->p, &P->Ap, &P->rho_prev, &P->p1};
  for (void** v : vecs)
    if (ok && cudaMalloc(v, P->n * es) != cudaSuccess) ok = false;
  const size_t np = kPcgBlocks > kRedBlocks ? kPcgBlocks : kRedBlocks;
  if (ok && cudaMalloc((void**)&P->x1, P->n * sizeof(double)) != cudaSuccess) ok = false;
  if (ok && cudaMalloc((void**)&P->part, np * sizeof(double)) != cudaSuccess) ok = false;
  if (ok && cudaMalloc((void**)&P->part2, np * sizeof(double)) != cudaSuccess) ok = false;
  if (ok && cudaMalloc((void**)&P->s, (S_NSLOTS + 2) * sizeof(double)) != cudaSuccess) ok = false;
  if (ok && cudaMalloc((void**)&P->ticket, 4 * sizeof(unsigned)) != cudaSuccess) ok = false;
  if (ok && cudaMemset(P->ticket, 0, 4 * sizeof(unsigned)) != cudaSuccess) ok = false;
  if (!ok) {
    void* ps[] = {P->rho, P->z, P->p, P->Ap, P->rho_prev, P->p1, P->x1, P->part, P->part2, P->s, P->ticket};
    for (void* q : ps) if (q) cudaFree(q);
    delete P;
    return FVX_ERR_CUDA;
  }
  *out = P;
  return FVX_OK;
}

extern "C" int fvx_pcg_destroy(fvx_pcg* P) {
  if (!P) return FVX_ERR_ARG;
  cudaDeviceSynchronize();
  if (P->own_rho) { P->rho = P->own_rho; P->z = P->own_z; }
  void* ps[] = {P->rho, P->z, P->p, P->Ap, P->rho_prev, P->p1, P->x1, P->part, P->part2, P->s, P->ticket};
  for (void* q : ps) if (q) cudaFree(q);
  delete P;
  return fvx_cuda_status();
}

// The PCG in four entry points so a host can capture fvx_pcg_iterate (and
// the preconditioner launches it makes) in a CUDA graph and replay it:
// begin (rho = b, z = M rho, p = z, gamma), iterate (n iterations, no host
// synchronisation; kernels return at once after convergence), status (reads
// the flag, synchronises), finish (FP64 true residual).
struct PcgCall {
  int precond;
  fvx_precond_fn fn;
  void* ctx;
  int flexible;
  int replace_every;
};

template <typename T>
static int pcg_apply_M(fvx_pcg* P, const PcgCall& c, cudaStream_t st) {
  if (c.precond == 1) return fvx_mg_vcycle(P->mg, nullptr, P->rho, P->z, st);
  if (c.precond == 2) return c.fn(c.ctx, P->rho, P->z, st);
  k_copy_if<T><<<kRedBlocks, 256, 0, st>>>((T*)P->z, (const T*)P->rho, P->n, P->s);
  return fvx_cuda_status();
}

template <typename T>
static int pcg_begin_t(fvx_pcg* P, const T* b, double* x, double rtol, const PcgCall& c, double* bb_out,
                       cudaStream_t st) {
  fvx_mg* g = P->mg;
  const size_t n = P->n;
  double* s = P->s;
  const int G = kRedBlocks;
  double init[S_NSLOTS] = {0};
  cudaMemcpyAsync(s, init, sizeof(init), cudaMemcpyHostToDevice, st);
  k_zero_x<T><<<G, 256, 0, st>>>(x, n);
  k_residual64<T><<<G, 256, 0, st>>>(g->L0d, x, b, (T*)P->rho, P->part, s, 1);
  k_reduce<<<1, 256, 0, st>>>(P->part, nullptr, G, s, S_BB, R_STORE, 1);
  double bb = 0;
  cudaMemcpyAsync(&bb, s + S_BB, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return FVX_ERR_CUDA;
  *bb_out = bb;
  const double tol2 = rtol * rtol * bb;
  double conv = bb == 0.0 ? 1.0 : 0.0;
  cudaMemcpyAsync(s + S_TOL2, &tol2, sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s + S_CONV, &conv, sizeof(double), cudaMemcpyHostToDevice, st);
  if (bb == 0.0) return FVX_OK;
  int rc = pcg_apply_M<T>(P, c, st);
  if (rc) return rc;
  // p_old = 0 and beta = 0 (S_BETA starts at 0): the first iteration takes p = z
  cudaMemsetAsync(P->p, 0, n * sizeof(T), st);
  k_dot<T><<<G, 256, 0, st>>>((const T*)P->rho, (const T*)P->z, nullptr, P->part, nullptr, s, n);
  k_reduce<<<1, 256, 0, st>>>(P->part, nullptr, G, s, S_GAMMA, R_STORE, 0);
  return fvx_cuda_status();
}

// ``niter`` iterations; the iteration count, the iterate/direction
// ping-pong and the residual-replacement schedule all follow the device's
// own counter, so the launches are the same for every call (CUDA graphs).
// Per iteration: k_dir_apply, k_step, the preconditioner, k_dot_beta.
template <typename T>
static int pcg_iterate_t(fvx_pcg* P, const T* b, double* x, int niter, const PcgCall& c, cudaStream_t st) {
  fvx_mg* g = P->mg;
  Lev<T>& L = levs<T>(g).L[0];
  T *rho = (T*)P->rho, *z = (T*)P->z, *p0 = (T*)P->p, *p1 = (T*)P->p1, *Ap = (T*)P->Ap;
  T* rp = c.flexible ? (T*)P->rho_prev : nullptr;
  double* s = P->s;
  const int G = kPcgBlocks;
  for (int k = 0; k < niter; ++k) {
    k_dir_apply<T><<<G, 256, 0, st>>>(L, z, p0, p1, Ap, P->part, s, P->ticket);
    k_step<T><<<G, 256, 0, st>>>(g->L0d, p0, p1, Ap, x, P->x1, b, rho, rp, c.replace_every, P->part, s,
                                 P->ticket + 1);
    int rc = pcg_apply_M<T>(P, c, st);
    if (rc) return rc;
    k_dot_beta<T><<<G, 256, 0, st>>>(z, rho, rp, P->n, P->part, P->part2, s, P->ticket + 2);
  }
  return fvx_cuda_status();
}

// Final iterate into x (odd iteration counts leave it in the second
// buffer) and its FP64 true relative residual.
template <typename T>
static int pcg_finish_t(fvx_pcg* P, const T* b, double* x, double bb, double* rel_out, cudaStream_t st) {
  double iters = 0;
  cudaMemcpyAsync(&iters, P->s + S_ITER, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return FVX_ERR_CUDA;
  if (((long long)iters) & 1)
    cudaMemcpyAsync(x, P->x1, P->n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  const int G = kRedBlocks;
  k_residual64<T><<<G, 256, 0, st>>>(P->mg->L0d, x, b, (T*)nullptr, P->part, P->s, 1);
  k_reduce<<<1, 256, 0, st>>>(P->part, nullptr, G, P->s, S_RR, R_STORE, 1);
  double rr = 0;
  cudaMemcpyAsync(&rr, P->s + S_RR, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return FVX_ERR_CUDA;
  // bb = 0: the zero solution is exact; a NaN (or negative) bb or rr is not
  // a converged solve: the relative residual stays NaN
  *rel_out = bb == 0.0 ? 0.0 : sqrt(rr / bb);
  return FVX_OK;
}

extern "C" int fvx_pcg_begin(fvx_pcg* P, const void* b, double* x, double rtol, int precond, fvx_precond_fn fn,
                             void* ctx, double* bb_out, void* stream) {
  if (!P || !b || !x || !bb_out || (precond == 2 && !fn)) return FVX_ERR_ARG;
  PcgCall c{precond, fn, ctx, 0, 0};
  cudaStream_t st = fvx_stream(stream);
  return P->dtype == 0 ? pcg_begin_t<float>(P, (const float*)b, x, rtol, c, bb_out, st)
                       : pcg_begin_t<double>(P, (const double*)b, x, rtol, c, bb_out, st);
}

extern "C" int fvx_pcg_iterate(fvx_pcg* P, const void* b, double* x, int it0, int niter, int precond,
                               fvx_precond_fn fn, void* ctx, int flexible, int replace_every, void* stream) {
  if (!P || !b || !x || niter < 0 || (precond == 2 && !fn)) return FVX_ERR_ARG;
  PcgCall c{precond, fn, ctx, flexible, replace_every};
  cudaStream_t st = fvx_stream(stream);
  (void)it0;  // the schedule follows the device iteration counter
  return P->dtype == 0 ? pcg_iterate_t<float>(P, (const float*)b, x, niter, c, st)
                       : pcg_iterate_t<double>(P, (const double*)b, x, niter, c, st);
}

// Reads [converged flag, iterations, last |rho|^2]; synchronises the stream.
extern "C" int fvx_pcg_status(fvx_pcg* P, double* out3, void* stream) {
  if (!P || !out3) return FVX_ERR_ARG;
  double hs[S_NSLOTS];
  cudaStream_t st = fvx_stream(stream);
  if (cudaMemcpyAsync(hs, P->s, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return FVX_ERR_CUDA;
  out3[0] = hs[S_CONV];
  out3[1] = hs[S_ITER];
  out3[2] = hs[S_RR];
  return FVX_OK;
}

extern "C" int fvx_pcg_finish(fvx_pcg* P, const void* b, double* x, double bb, double* rel_out, void* stream) {
  if (!P || !b || !x || !rel_out) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  return P->dtype == 0 ? pcg_finish_t<float>(P, (const float*)b, x, bb, rel_out, st)
                       : pcg_finish_t<double>(P, (const double*)b, x, bb, rel_out, st);
}

// Iterations to run before the next read of the convergence flag: the
// number the last chunk's residual reduction predicts to reach tol2 (so
// few iterations run after convergence), between 1 and chunk_max.
static int pcg_next_chunk(double rr_prev, double rr, int done, double tol2, int chunk_max) {
  if (!(rr > 0.0) || !(rr_prev > 0.0) || rr >= rr_prev || done < 1) return chunk_max;
  const double per_it = log(rr / rr_prev) / done;  // < 0
  const double need = log(tol2 / rr) / per_it;
  int m = need <= 1.0 ? 1 : (int)ceil(need);
  return m < 1 ? 1 : (m > chunk_max ? chunk_max : m);
}

template <typename T>
static int pcg_run(fvx_pcg* P, const T* b, double* x, int max_iter, double rtol, int precond, fvx_precond_fn fn,
                   void* ctx, int flexible, int replace_every, int chunk, double* info, cudaStream_t st) {
  PcgCall c{precond, fn, ctx, flexible, replace_every};
  double bb = 0;
  int rc = pcg_begin_t<T>(P, b, x, rtol, c, &bb, st);
  if (rc) return rc;
  if (bb == 0.0) {
    if (info) { info[0] = 0; info[1] = 0; info[2] = 1; }
    return FVX_OK;
  }
  int it = 0;
  double hs[3] = {0, 0, 0};
  double rr_prev = bb;
  int m = chunk < 2 ? chunk : 2;
  while (it < max_iter && hs[0] == 0.0) {
    if (m > max_iter - it) m = max_iter - it;
    if ((rc = pcg_iterate_t<T>(P, b, x, m, c, st))) return rc;
    it += m;
    if ((rc = fvx_pcg_status(P, hs, st))) return rc;
    m = pcg_next_chunk(rr_prev, hs[2], m, rtol * rtol * bb, chunk);
    rr_prev = hs[2];
  }
  double rel = 0;
  if ((rc = pcg_finish_t<T>(P, b, x, bb, &rel, st))) return rc;
  if (info) { info[0] = hs[1]; info[1] = rel; info[2] = rel <= rtol ? 1.0 : 0.0; }
  return rel <= rtol ? FVX_OK : FVX_ERR_NOT_CONVERGED;
}

// Whole solve: begin, chunks of ``chunk`` iterations between reads of the
// device convergence flag, FP64 true residual at the end.
extern "C" int fvx_pcg_solve(fvx_pcg* P, const void* b, double* x, int max_iter, double rtol, int precond,
                             fvx_precond_fn fn, void* ctx, int flexible, int replace_every, int chunk, double* info,
                             void* stream) {
  if (!P || !b || !x || max_iter < 0 || chunk < 1 || (precond == 2 && !fn)) return FVX_ERR_ARG;
  cudaStream_t st = fvx_stream(stream);
  return P->dtype == 0 ? pcg_run<float>(P, (const float*)b, x, max_iter, rtol, precond, fn, ctx, flexible,
                                        replace_every, chunk, info, st)
                       : pcg_run<double>(P, (const double*)b, x, max_iter, rtol, precond, fn, ctx, flexible,
                                         replace_every, chunk, info, st);
}

// Use caller-owned device buffers (plan dtype, [ny, nx]) as the residual rho
// and preconditioned residual z, so a preconditioner callback can read rho
// and write z through the caller's own handles.
extern "C" int fvx_pcg_bind_vectors(fvx_pcg* P, void* rho, void* z) {
  if (!P || !rho || !z) return FVX_ERR_ARG;
  if (!P->own_rho) { P->own_rho = P->rho; P->own_z = P->z; }
  P->rho = rho;
  P->z = z;
  return FVX_OK;
}

// ---- small linear-algebra helpers ----------------------------------------
namespace fvx {
namespace mg {
template <typename T>
__global__ void k_dot_plain(const T* a, const T* b, size_t n, double* part) {
  double acc = 0.0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    acc += (double)a[c] * (double)b[c];
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}
__global__ void k_sum_parts(const double* part, int np, double* out) {
  double v = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) v += part[k];
  v = block_sum(v);
  if (threadIdx.x == 0) *out = v;
}
// out[b, k, c] = sum_l C[k][l] in[b, l, c]  (layer_to_mode / mode_to_layer,
// vertical/vertical_modes.py:193-263), C given by value.
constexpr int kMaxLayers = 8;
struct Mix { double c[kMaxLayers * kMaxLayers]; };
template <typename T>
__global__ void k_layer_mix(Mix M, const T* in, T* out, int nl, size_t plane, int batch) {
  const size_t n = plane * (size_t)batch;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const size_t b = t / plane, c = t - b * plane;
    const T* src = in + b * nl * plane + c;
    T v[kMaxLayers];
    for (int l = 0; l < nl; ++l) v[l] = src[l * plane];
    T* dst = out + b * nl * plane + c;
    for (int k = 0; k < nl; ++k) {
      T acc = T(0);
      for (int l = 0; l < nl; ++l) acc = acc + (T)M.c[k * nl + l] * v[l];
      dst[k * plane] = acc;
    }
  }
}
}  // namespace mg
}  // namespace fvx

// sum a*b in FP64 into *out_dev (device double); ``part`` holds 296 doubles.
#define FVX_DEF_LA(SFX, T)                                                                                      \
  extern "C" int fvx_dot_##SFX(const T* a, const T* b, int64_t n, double* part, double* out_dev, void* stream) { \
    if (!a || !b || !part || !out_dev || n < 0) return FVX_ERR_ARG;                                             \
    cudaStream_t st = fvx_stream(stream);                                                                       \
    fvx::mg::k_dot_plain<T><<<fvx::mg::kRedBlocks, 256, 0, st>>>(a, b, (size_t)n, part);                        \
    fvx::mg::k_sum_parts<<<1, 256, 0, st>>>(part, fvx::mg::kRedBlocks, out_dev);                                \
    return fvx_cuda_status();                                                                                   \
  }                                                                                                             \
  extern "C" int fvx_layer_mix_##SFX(const double* C, int nl, const T* in, T* out, int64_t plane, int batch,    \
                                     void* stream) {                                                            \
    if (!C || !in || !out || in == out) return FVX_ERR_ARG;                                                     \
    if (nl < 1 || nl > fvx::mg::kMaxLayers || plane < 1 || batch < 1) return FVX_ERR_SHAPE;                     \
    fvx::mg::Mix M;                                                                                             \
    for (int k = 0; k < nl * nl; ++k) M.c[k] = C[k];                                                            \
    fvx::mg::k_layer_mix<T><<<fvx::mg::grid_for((size_t)plane * batch), 256, 0, fvx_stream(stream)>>>(          \
        M, in, out, nl, (size_t)plane, batch);                                                                  \
    return fvx_cuda_status();                                                                                   \
  }
FVX_DEF_LA(f32, float)
FVX_DEF_LA(f64, double)
