// Fused QG RK stage: the per-tile body shared by the single-field kernel
// (qg.cu) and the ensemble's persistent work-queue kernel (ensemble.cu).
#pragma once
#include "recon.cuh"

#include <cuda_bf16.h>

#include <type_traits>

namespace fvx {
namespace qg {

constexpr int THREADS = 256;
// Tile shapes the autotuner chooses from (fvx_qg_tile_config): TX x TY cells.
// (16 x 16: small FP64 grids, where 32 x 16 tiles leave SMs idle.)
constexpr int kTileTX[6] = {64, 32, 128, 64, 128, 16};
constexpr int kTileTY[6] = {16, 16, 8, 32, 16, 16};
constexpr int kTileConfigs = 6;

// a / d: exact division in FP64; multiplication by the rounded reciprocal in
// FP32 (<= 1 ulp from the quotient).
template <typename T> DEV T divr(T a, T d, T rd) {
  if constexpr (sizeof(T) == 8) return a / d;
  else return a * rd;
}

struct StageArgs {
  const void* qs;      // stage state [Ny][Nx]
  const void* qn;      // step-start state (null on stage 1)
  const void* psi;     // interior-only [Ny-2][Nx-2]
  const void* forcing; // [Ny][Nx] or null
  void* out;           // [Ny][Nx]
  __nv_bfloat16* split_hi;  // [Ny-2][Nx-2] or null (FP64 stages: a double [Ny-2][Nx-2] interior copy)
  __nv_bfloat16* split_lo;  // (FP64 stages: null)
  int split_layout;         // 1: x de-interleaved (the even/odd DST operand layout)
  int ny, nx;
  double a, b, c;      // out = a*qn + b*qs + c*rhs
  double dx, dy, beta, drag, visc;
  int periodic;        // 1: periodic ghost ring, 0: zero (wall) ghost ring
  int write_ghost;
};

// Face value on a line segment far from both ends: a WENO scheme at its full
// reach (what face_value's boundary ladder picks when d >= reach), other
// schemes through face_value itself.
template <typename T, int S>
DEV T face_value_full(const T* p, int st, int i, int N, bool pos) {
  if constexpr (SchemeInfo<S>::is_weno) {
    constexpr bool Z = SchemeInfo<S>::zfam;
    constexpr int R = SchemeInfo<S>::reach;
    const T* b = pos ? p : p + st;
    const int s = pos ? st : -st;
    auto e = [&](int k) -> T { return b[k * s]; };
    if constexpr (R >= 4) {
      T v[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) v[k] = e(k - 4);
      return weno_generic<T, 5>(v);
    } else if constexpr (R == 3) {
      T v[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) v[k] = e(k - 3);
      return weno_generic<T, 4>(v);
    } else if constexpr (R == 2) {
      return weno5<T, Z>(e(-2), e(-1), e(0), e(1), e(2));
    } else {
      return Z ? wenoz3(e(-1), e(0), e(1)) : weno3(e(-1), e(0), e(1));
    }
  } else {
    return face_value<T, S>(p, st, i, N, pos);
  }
}

// WENO7 / WENO9 faces through calls: inlined into the stage's face loops,
// the compiler hoists the schemes' table coefficients out of the loops into
// registers (FP32 WENO9: 195 registers per thread); behind a call they stay
// constant-bank operands.
template <int S>
struct StageFaceCall {
  static constexpr bool v = S == FVX_WENO7 || S == FVX_WENO9;
};
template <typename T, int S>
__noinline__ __device__ T stage_face_full_call(const T* p, int st, int i, int N, bool pos) {
  return face_value_full<T, S>(p, st, i, N, pos);
}
template <typename T, int S>
__noinline__ __device__ T stage_face_ladder_call(const T* p, int st, int i, int N, bool pos) {
  return face_value<T, S>(p, st, i, N, pos);
}
template <typename T, int S>
DEV T stage_face_full(const T* p, int st, int i, int N, bool pos) {
  if constexpr (StageFaceCall<S>::v) return stage_face_full_call<T, S>(p, st, i, N, pos);
  else return face_value_full<T, S>(p, st, i, N, pos);
}
template <typename T, int S>
DEV T stage_face(const T* p, int st, int i, int N, bool pos) {
  if constexpr (StageFaceCall<S>::v) return stage_face_ladder_call<T, S>(p, st, i, N, pos);
  else return face_value<T, S>(p, st, i, N, pos);
}

// ---- asynchronous global -> shared copies (cp.async, no register staging) --
// Interior tiles' loads are plain copies: issue them all, then wait once, so
// the tile load costs one memory latency instead of one per loop iteration.
// (The q rows' pitch, Nx elements, is not 16-byte aligned in general, which
// rules out TMA tiles here.)
template <typename T>
DEV void cp_async_elem(T* dst, const T* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
DEV void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
DEV void cp_async_8(void* dst, const void* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

// ---- tile geometry ----------------------------------------------------------
// The q tile covers rows y0-H .. y0+TY+H-1 and columns x0-H .. x0+TX+H-1;
// element (ly, lx) sits at [ly * QW + SH + lx].  The SH leading elements
// make each stored row start at column x0-H-SH, an even column (x0 is even),
// so that FP32 rows can be copied in 8-byte pieces; the pitch QW is even and,
// for FP32, 2 mod 4 (a row per lane then spreads over the banks).
template <typename T, int S, int TX, int TY>
struct Geom {
  static constexpr int H = SchemeInfo<S>::halo_hi > 3 ? SchemeInfo<S>::halo_hi : 3;
  static constexpr int QWD = TX + 2 * H;  // q columns the body reads
  static constexpr int SH = sizeof(T) == 4 ? (H & 1) : 0;
  static constexpr int QWL = sizeof(T) == 4 ? ((QWD + SH + 1) & ~1) : QWD;  // columns per 8-byte row copy
  static constexpr int QW = sizeof(T) == 4 ? (QWL % 4 == 0 ? QWL + 2 : QWL) : QWD;
  static constexpr int QH = TY + 2 * H;
  static constexpr int NQ = QH * QW;
  static constexpr int NP = (TY + 2) * (TX + 2);  // psi, origin (y0-1, x0-1)
  static constexpr int NWORK = (TY + 1) * (TX + 1) + TY * (TX + 1) + 2 * (TY + 1) * TX;  // X, fe, fn, v
};

// ---- packed FP32 pairs (Blackwell f32x2 arithmetic) -----------------------
// Two independent values per instruction; each lane is an IEEE round-to-
// nearest FP32 operation, the same as its scalar form.
DEV unsigned long long f2pack(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
DEV float2 f2unpack(unsigned long long r) {
  float2 d;
  asm("mov.b64 {%0,%1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(r));
  return d;
}
DEV float2 f2fma(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2pack(a)), "l"(f2pack(b)), "l"(f2pack(c)));
  return f2unpack(d);
}
DEV float2 f2add(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2pack(a)), "l"(f2pack(b)));
  return f2unpack(d);
}
DEV float2 f2mul(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2pack(a)), "l"(f2pack(b)));
  return f2unpack(d);
}
DEV float2 f2s(float c) { return make_float2(c, c); }

// WENO5 / WENO-Z5 (weno5<float, Z> in recon.cuh, the same formulas) on two
// stencils at once.  WENO5 normalises with one reciprocal per lane (the
// common-denominator weights of weno5_core), WENO-Z5 with four; stencils
// whose WENO5 products overflow go through the scalar four-division form.
__noinline__ DEV float2 weno5_js_x2_fallback(float2 qi1, float2 qi2, float2 qi3, float2 b1, float2 b2, float2 b3) {
  const float e = 1e-8f;
  float r[2];
  for (int l = 0; l < 2; ++l) {
    const float w1 = fdiv(0.1f, sq((l ? b1.y : b1.x) + e)), w2 = fdiv(0.6f, sq((l ? b2.y : b2.x) + e)),
                w3 = fdiv(0.3f, sq((l ? b3.y : b3.x) + e));
    r[l] = fdiv(w1 * (l ? qi1.y : qi1.x) + w2 * (l ? qi2.y : qi2.x) + w3 * (l ? qi3.y : qi3.x), w1 + w2 + w3);
  }
  return make_float2(r[0], r[1]);
}
DEV float2 f2rcp(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
template <bool Z>
DEV float2 weno5_x2(float2 qmm, float2 qm, float2 q0, float2 qp, float2 qpp) {
  const float2 qi1 = f2fma(f2s(11.f / 6.f), q0, f2fma(f2s(-7.f / 6.f), qm, f2mul(f2s(1.f / 3.f), qmm)));
  const float2 qi2 = f2fma(f2s(1.f / 3.f), qp, f2fma(f2s(5.f / 6.f), q0, f2mul(f2s(-1.f / 6.f), qm)));
  const float2 qi3 = f2fma(f2s(-1.f / 6.f), qpp, f2fma(f2s(5.f / 6.f), qp, f2mul(f2s(1.f / 3.f), q0)));
  const float2 k1 = f2s(13.f / 12.f), k2 = f2s(0.25f);
  const float2 a1 = f2add(f2fma(f2s(-2.f), qm, qmm), q0);
  const float2 c1 = f2fma(f2s(3.f), q0, f2fma(f2s(-4.f), qm, qmm));
  const float2 b1 = f2fma(k2, f2mul(c1, c1), f2mul(k1, f2mul(a1, a1)));
  const float2 a2 = f2add(f2fma(f2s(-2.f), q0, qm), qp);
  const float2 c2 = f2add(qm, f2mul(f2s(-1.f), qp));
  const float2 b2 = f2fma(k2, f2mul(c2, c2), f2mul(k1, f2mul(a2, a2)));
  const float2 a3 = f2add(f2fma(f2s(-2.f), qp, q0), qpp);
  const float2 c3 = f2add(f2fma(f2s(-4.f), qp, f2mul(f2s(3.f), q0)), qpp);
  const float2 b3 = f2fma(k2, f2mul(c3, c3), f2mul(k1, f2mul(a3, a3)));
  if (Z) {
    const float2 eps = f2s(1e-16f);
    const float2 tau = make_float2(fabsf(b1.x - b3.x), fabsf(b1.y - b3.y));
    const float2 r1 = f2mul(tau, f2rcp(f2add(b1, eps)));
    const float2 r2 = f2mul(tau, f2rcp(f2add(b2, eps)));
    const float2 r3 = f2mul(tau, f2rcp(f2add(b3, eps)));
    const float2 w1 = f2mul(f2s(0.1f), f2add(f2s(1.f), r1));
    const float2 w2 = f2mul(f2s(0.6f), f2add(f2s(1.f), r2));
    const float2 w3 = f2mul(f2s(0.3f), f2add(f2s(1.f), r3));
    const float2 num = f2fma(w3, qi3, f2fma(w2, qi2, f2mul(w1, qi1)));
    return f2mul(num, f2rcp(f2add(f2add(w1, w2), w3)));
  } else {
    const float2 eps = f2s(1e-8f);
    const float2 d1 = f2add(b1, eps), d2 = f2add(b2, eps), d3 = f2add(b3, eps);
    const float2 s1 = f2mul(d1, d1), s2 = f2mul(d2, d2), s3 = f2mul(d3, d3);
    const float2 W1 = f2mul(f2s(0.1f), f2mul(s2, s3)), W2 = f2mul(f2s(0.6f), f2mul(s1, s3));
    const float2 W3 = f2mul(f2s(0.3f), f2mul(s1, s2));
    const float2 num = f2fma(W3, qi3, f2fma(W2, qi2, f2mul(W1, qi1)));
    const float2 den = f2add(f2add(W1, W2), W3);
    const float2 r = f2mul(num, f2rcp(den));
    if (den.x < 3e38f && den.y < 3e38f && fabsf(r.x) < 3.4e38f && fabsf(r.y) < 3.4e38f) return r;
    return weno5_js_x2_fallback(qi1, qi2, qi3, b1, b2, b3);
  }
}

// IN: the tile and its halo lie inside the interior and every face is at
// least the scheme's reach from both ends (the kernel decides per block):
// no bounds tests, wrap-around loads, ghost writes or boundary ladder.
template <typename T, int S, bool IN, int TX, int TY>
DEV void stage_body(const StageArgs& A, uint8_t* sm, const int x0, const int y0) {
  using G = Geom<T, S, TX, TY>;
  constexpr int H = G::H, QW = G::QW, QWD = G::QWD, QH = G::QH;
  T* base = (T*)sm;
  T* qt = base + G::SH;                    // q (ly, lx) at qt[ly * QW + lx]
  T* pt = base + G::NQ;                    // psi [TY+2][TX+2], origin (y0-1, x0-1)
  T* xt = pt + G::NP;                      // X [TY+1][TX+1], origin (y0-1, x0-1)
  T* fe = xt + (TY + 1) * (TX + 1);        // [TY][TX+1]
  T* fn = fe + TY * (TX + 1);              // [TY+1][TX]
  T* vs = fn + (TY + 1) * TX;              // v on north faces [TY+1][TX], origin (y0-1, x0)
  const int ny = A.ny, nx = A.nx;
  const int tid = threadIdx.x;
  const T* qs = (const T*)A.qs;
  const T* psi = (const T*)A.psi;
  const int nxi = nx - 2;
  // ---- loads: q with BC applied on the fly, psi with zero outside --------
  if constexpr (IN) {
    {
      const bool v8 = sizeof(T) == 8 || (((uintptr_t)qs | (uintptr_t)psi) & 7) == 0 && (nx & 1) == 0;
      if (v8) {
        // 8-byte pieces; each thread keeps one column of pieces and walks
        // the rows with pointer increments
        constexpr int E = 8 / (int)sizeof(T);
        constexpr int CQ = G::QWL / E, RQ = THREADS / CQ;
        constexpr int CP = (TX + 2) / E, RP = THREADS / CP;
        static_assert(RQ >= 1 && RP >= 1, "tile rows wider than the block");
        int r = tid / CQ;
        if (r < RQ) {
          const int c = tid - r * CQ;
          const T* src = qs + (size_t)(y0 - H + r) * nx + (x0 - H - G::SH + c * E);
          T* dst = base + r * QW + c * E;
          for (; r < QH; r += RQ, src += (size_t)RQ * nx, dst += RQ * QW) cp_async_8(dst, src);
        }
        r = tid / CP;
        if (r < RP) {
          const int c = tid - r * CP;
          const T* src = psi + (size_t)(y0 - 2 + r) * nxi + (x0 - 2 + c * E);
          T* dst = pt + r * (TX + 2) + c * E;
          for (; r < TY + 2; r += RP, src += (size_t)RP * nxi, dst += RP * (TX + 2)) cp_async_8(dst, src);
        }
      } else {
        for (int k = tid; k < QH * QWD; k += THREADS) {
          const int ly = k / QWD, lx = k - ly * QWD;
          cp_async_elem(qt + ly * QW + lx, qs + (size_t)(y0 - H + ly) * nx + (x0 - H + lx));
        }
        for (int k = tid; k < (TY + 2) * (TX + 2); k += THREADS) {
          const int ly = k / (TX + 2), lx = k - ly * (TX + 2);
          cp_async_elem(pt + k, psi + (size_t)(y0 - 2 + ly) * nxi + (x0 - 2 + lx));
        }
      }
      cp_async_wait_all();
    }
  } else {
  // general tiles: wrap-around / zero-ring sources resolved per element, the
  // copies themselves asynchronous (one wait for the whole tile)
  for (int k = tid; k < QH * QWD; k += THREADS) {
    int ly = k / QWD, lx = k - ly * QWD;
    int gy = y0 - H + ly, gx = x0 - H + lx;
    const T* src = nullptr;
    if (gy >= 0 && gy < ny && gx >= 0 && gx < nx) {
      bool gh = gy == 0 || gy == ny - 1 || gx == 0 || gx == nx - 1;
      if (!gh) src = qs + (size_t)gy * nx + gx;
      else if (A.periodic) {
        int sy = gy == 0 ? ny - 2 : (gy == ny - 1 ? 1 : gy);
        int sx = gx == 0 ? nx - 2 : (gx == nx - 1 ? 1 : gx);
        src = qs + (size_t)sy * nx + sx;
      }
    }
    if (src) cp_async_elem(qt + ly * QW + lx, src);
    else qt[ly * QW + lx] = T(0);
  }
  for (int k = tid; k < (TY + 2) * (TX + 2); k += THREADS) {
    int ly = k / (TX + 2), lx = k - ly * (TX + 2);
    int gy = y0 - 1 + ly, gx = x0 - 1 + lx;
    if (gy >= 1 && gy <= ny - 2 && gx >= 1 && gx <= nx - 2) cp_async_elem(pt + k, psi + (size_t)(gy - 1) * nxi + (gx - 1));
    else pt[k] = T(0);
  }
  cp_async_wait_all();
  }
  __syncthreads();
  constexpr int SEG = TX * TY / THREADS;
  constexpr bool WIN = IN && sizeof(T) == 4 && (S == FVX_WENO5 || S == FVX_WENOZ5) && SEG >= 2 && SEG % 2 == 0 &&
                       SEG * THREADS == TX * TY && TX % SEG == 0 && TY % SEG == 0;
  // ---- X = interior(T_to_X(psi)) on rows y0-1.., cols x0-1.. -------------
  // (not built by the WIN body, which takes u and v from psi directly)
  if constexpr (WIN) {
  } else if constexpr (IN && THREADS % TX == 0 && THREADS / TX <= TY + 1) {
    // a column of X per thread group, walking down the rows (two new psi
    // loads per row); the last column by the first TY + 1 threads
    constexpr int RG = THREADS / TX, RPG = (TY + 1 + RG - 1) / RG;
    const int lx = tid % TX, g = tid / TX;
    const int r0 = g * RPG, r1 = r0 + RPG < TY + 1 ? r0 + RPG : TY + 1;
    const T* p = pt + r0 * (TX + 2) + lx;
    T a0 = p[0] + p[1];
    for (int ly = r0; ly < r1; ++ly) {
      p += TX + 2;
      const T a1 = p[0] + p[1];
      xt[ly * (TX + 1) + lx] = T(0.25) * (a0 + a1);
      a0 = a1;
    }
    if (tid < TY + 1) {
      const T* q = pt + tid * (TX + 2) + TX;
      xt[tid * (TX + 1) + TX] = T(0.25) * (q[0] + q[1] + q[TX + 2] + q[TX + 3]);
    }
  } else
  for (int k = tid; k < (TY + 1) * (TX + 1); k += THREADS) {
    int ly = k / (TX + 1), lx = k - ly * (TX + 1);
    int gy = y0 - 1 + ly, gx = x0 - 1 + lx;
    T val = T(0);
    if (IN || (gy >= 1 && gy <= ny - 2 && gx >= 1 && gx <= nx - 2)) {
      const T* p = pt + ly * (TX + 2) + lx;  // psi at (gy, gx)
      val = T(0.25) * (p[0] + p[1] + p[TX + 2] + p[TX + 3]);
    }
    xt[k] = val;
  }
  if constexpr (!WIN) __syncthreads();
  const T dx = T(A.dx), dy = T(A.dy);
  const T rdx = T(1.0 / A.dx), rdy = T(1.0 / A.dy);
  // u at U-point (j, i) = -(X[j,i] - X[j-1,i]) / dy on [1, N-2]^2
  auto uvel = [&](int gy, int gx) -> T {
    if (!IN && (gy < 1 || gy > ny - 2 || gx < 1 || gx > nx - 2)) return T(0);
    const T* p = xt + (gy - (y0 - 1)) * (TX + 1) + (gx - (x0 - 1));
    return -divr(p[0] - p[-(TX + 1)], dy, rdy);
  };
  auto vvel = [&](int gy, int gx) -> T {
    if (!IN && (gy < 1 || gy > ny - 2 || gx < 1 || gx > nx - 2)) return T(0);
    const T* p = xt + (gy - (y0 - 1)) * (TX + 1) + (gx - (x0 - 1));
    return divr(p[0] - p[-1], dx, rdx);
  };
  // ---- face fluxes --------------------------------------------------------
  // FP32 WENO5 / WENO-Z5 interior tiles (WIN): each thread reconstructs a
  // run of SEG east faces along a row and a run of SEG north faces along a
  // column from a register window of SEG + 5 cells (one shared-memory load
  // per face instead of six), the upwind stencil picked from the window and
  // two neighbouring faces evaluated as one packed f32x2 pair.  Velocities
  // come straight from psi: u = -(X[j] - X[j-1]) / dy with
  // X = T_to_X(psi) is -(psi[j+1][i] + psi[j+1][i+1] - psi[j-1][i] -
  // psi[j-1][i+1]) / (4 dy) (the psi[j] terms cancel), v likewise, summed as
  // sliding differences along the walk, so no X array is built.
  if constexpr (WIN) {
    const float cu = -0.25f * (float)rdy, cv = 0.25f * (float)rdx;
    const float* ps = (const float*)pt;  // psi (gy, gx) at ps[(gy - y0 + 1) * (TX + 2) + gx - x0 + 1]
    constexpr bool Z = SchemeInfo<S>::zfam;
    const float* q32 = (const float*)qt;
    {  // east faces of cells x0 + xs .. x0 + xs + SEG - 1 on row ly
      const int ly = tid % TY, xs = (tid / TY) * SEG;
      const float* p = q32 + (ly + H) * QW + (xs + H);  // q at (y0 + ly, x0 + xs)
      float w[SEG + 5];
#pragma unroll
      for (int k = 0; k < SEG + 5; ++k) w[k] = p[k - 2];
      // d[m] = psi(j+1, i) - psi(j-1, i) at i = x0 + xs + m, j = y0 + ly
      float d[SEG + 1];
      const float* pn = ps + (ly + 2) * (TX + 2) + (xs + 1);
      const float* pm = ps + ly * (TX + 2) + (xs + 1);
#pragma unroll
      for (int m = 0; m <= SEG; ++m) d[m] = pn[m] - pm[m];
#pragma unroll
      for (int f = 0; f < SEG; f += 2) {  // faces f and f + 1 as one packed pair
        const float u0 = cu * (d[f] + d[f + 1]), u1 = cu * (d[f + 1] + d[f + 2]);
        const bool p0 = u0 >= 0.f, p1 = u1 >= 0.f;
        float2 e[5];
#pragma unroll
        for (int j = 0; j < 5; ++j)
          e[j] = make_float2(p0 ? w[f + j] : w[f + 5 - j], p1 ? w[f + 1 + j] : w[f + 6 - j]);
        const float2 r = weno5_x2<Z>(e[0], e[1], e[2], e[3], e[4]);
        fe[ly * (TX + 1) + xs + f + 1] = (T)(r.x * u0);
        fe[ly * (TX + 1) + xs + f + 2] = (T)(r.y * u1);
      }
    }
    {  // north faces of cells y0 + ys .. y0 + ys + SEG - 1 in column lx
      const int lx = tid % TX, ys = (tid / TX) * SEG;
      const float* p = q32 + (ys + H) * QW + (lx + H);  // q at (y0 + ys, x0 + lx)
      float w[SEG + 5];
#pragma unroll
      for (int k = 0; k < SEG + 5; ++k) w[k] = p[(k - 2) * QW];
      // e[m] = psi(j, i+1) - psi(j, i-1) at j = y0 + ys + m, i = x0 + lx
      float e2[SEG + 1];
      const float* pc = ps + (ys + 1) * (TX + 2) + lx;
#pragma unroll
      for (int m = 0; m <= SEG; ++m) e2[m] = pc[m * (TX + 2) + 2] - pc[m * (TX + 2)];
#pragma unroll
      for (int f = 0; f < SEG; f += 2) {
        const float v0 = cv * (e2[f] + e2[f + 1]), v1 = cv * (e2[f + 1] + e2[f + 2]);
        const bool p0 = v0 >= 0.f, p1 = v1 >= 0.f;
        float2 e[5];
#pragma unroll
        for (int j = 0; j < 5; ++j)
          e[j] = make_float2(p0 ? w[f + j] : w[f + 5 - j], p1 ? w[f + 1 + j] : w[f + 6 - j]);
        const float2 r = weno5_x2<Z>(e[0], e[1], e[2], e[3], e[4]);
        fn[(ys + f + 1) * TX + lx] = (T)(r.x * v0);
        fn[(ys + f + 2) * TX + lx] = (T)(r.y * v1);
        vs[(ys + f + 1) * TX + lx] = (T)v0;
        vs[(ys + f + 2) * TX + lx] = (T)v1;
      }
    }
    // the tile's west-most east faces and south-most north faces
    for (int k = tid; k < TY + TX; k += THREADS) {
      if (k < TY) {
        const int ly = k, gi = x0 - 1;
        const float* a = ps + ly * (TX + 2);  // psi rows j-1 and j+1 at columns x0-1, x0
        const T uu = (T)(cu * ((a[2 * (TX + 2)] - a[0]) + (a[2 * (TX + 2) + 1] - a[1])));
        fe[ly * (TX + 1)] = stage_face_full<T, S>(qt + (ly + H) * QW + (H - 1), 1, gi, nx, uu >= T(0)) * uu;
      } else {
        const int lx = k - TY, gj = y0 - 1;
        const float* a = ps + lx;  // psi rows y0-1, y0 at columns i-1, i+1
        const T vv = (T)(cv * ((a[2] - a[0]) + (a[(TX + 2) + 2] - a[TX + 2])));
        fn[lx] = stage_face_full<T, S>(qt + (H - 1) * QW + (lx + H), QW, gj, ny, vv >= T(0)) * vv;
        vs[lx] = vv;
      }
    }
  } else {
  for (int k = tid; k < TY * (TX + 1); k += THREADS) {
    int ly = k / (TX + 1), lf = k - ly * (TX + 1);
    int gj = y0 + ly, gi = x0 - 1 + lf;
    T f = T(0);
    if (IN) {
      T uu = uvel(gj, gi);
      f = stage_face_full<T, S>(qt + (ly + H) * QW + (lf - 1 + H), 1, gi, nx, uu >= T(0)) * uu;
    } else if (gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2) {
      T uu = uvel(gj, gi);
      f = stage_face<T, S>(qt + (ly + H) * QW + (lf - 1 + H), 1, gi, nx, uu >= T(0)) * uu;
    }
    fe[k] = f;
  }
  for (int k = tid; k < (TY + 1) * TX; k += THREADS) {
    int lf = k / TX, lx = k - lf * TX;
    int gj = y0 - 1 + lf, gi = x0 + lx;
    T f = T(0);
    T vv = vvel(gj, gi);
    if (IN)
      f = stage_face_full<T, S>(qt + (lf - 1 + H) * QW + (lx + H), QW, gj, ny, vv >= T(0)) * vv;
    else if (gj >= 1 && gj <= ny - 2 && gi >= 1 && gi <= nx - 2)
      f = stage_face<T, S>(qt + (lf - 1 + H) * QW + (lx + H), QW, gj, ny, vv >= T(0)) * vv;
    fn[k] = f;
    vs[k] = vv;
  }
  }
  __syncthreads();
  // ---- tendency, RK combination, stores ------------------------------------
  const T* qn = (const T*)A.qn;
  const T* F = (const T*)A.forcing;
  T* out = (T*)A.out;
  const T beta = T(A.beta), drag = T(A.drag), visc = T(A.visc);
  const T ca = T(A.a), cb = T(A.b), cc = T(A.c);
  constexpr int SEGT = TX * TY / THREADS;
  if constexpr (IN && SEGT >= 1 && SEGT * THREADS == TX * TY && TY % SEGT == 0) {
    if (!F && A.drag == 0.0 && A.visc == 0.0) {
      // interior tile without forcing, drag or viscosity: a run of SEGT
      // cells down one column per thread (coalesced rows across a warp),
      // each north face / v reused as the next cell's south one
      const int lx = tid % TX, ly0 = (tid / TX) * SEGT;
      const int gi = x0 + lx;
      size_t g = (size_t)(y0 + ly0) * nx + gi;
      const T* fep = fe + ly0 * (TX + 1) + lx;
      const T* fnp = fn + ly0 * TX + lx;
      const T* vsp = vs + ly0 * TX + lx;
      const T* qp = qt + (ly0 + H) * QW + (lx + H);
      const int xi = gi - 1;
      const int scol = A.split_layout ? ((xi & 1) ? (nxi >> 1) + (xi >> 1) : (xi >> 1)) : xi;
      size_t sidx = (size_t)(y0 + ly0 - 1) * nxi + scol;
      // one loop per (q_n present, split wanted) pair: no per-cell branches
      auto run = [&](auto has_qn, auto do_split) {
        T fs = fnp[0], vsv = vsp[0];
        const T* qnp = decltype(has_qn)::value ? qn + g : nullptr;
        T* op = out + g;
        __nv_bfloat16* hp = decltype(do_split)::value ? A.split_hi + sidx : nullptr;
        double* dp = (sizeof(T) == 8 && decltype(do_split)::value) ? (double*)(void*)A.split_hi + sidx : nullptr;
        __nv_bfloat16* lp = decltype(do_split)::value ? A.split_lo + sidx : nullptr;
#pragma unroll
        for (int f = 0; f < SEGT; ++f) {
          const T fnn = fnp[(f + 1) * TX], vn = vsp[(f + 1) * TX];
          T rhs = -(divr(fep[f * (TX + 1) + 1] - fep[f * (TX + 1)], dx, rdx) + divr(fnn - fs, dy, rdy));
          rhs = rhs + (-beta * (T(0.5) * (vn + vsv)));
          T r = cb * qp[f * QW];
          if constexpr (decltype(has_qn)::value) r = ca * qnp[(size_t)f * nx] + r;
          r = r + cc * rhs;
          op[(size_t)f * nx] = r;
          if constexpr (decltype(do_split)::value) {
            if constexpr (sizeof(T) == 8) {
              dp[(size_t)f * nxi] = r;  // FP64: the interior itself (the FP64 chain's input)
            } else {
              const float fv = (float)r;
              const __nv_bfloat16 h = __float2bfloat16_rn(fv);
              hp[(size_t)f * nxi] = h;
              lp[(size_t)f * nxi] = __float2bfloat16_rn(fv - __bfloat162float(h));
            }
          }
          fs = fnn;
          vsv = vn;
        }
      };
      using yes = std::true_type;
      using no = std::false_type;
      if (qn) {
        if (A.split_hi) run(yes{}, yes{});
        else run(yes{}, no{});
      } else {
        if (A.split_hi) run(no{}, yes{});
        else run(no{}, no{});
      }
      return;
    }
  }
  for (int k = tid; k < TY * TX; k += THREADS) {
    int ly = k / TX, lx = k - ly * TX;
    int gj = y0 + ly, gi = x0 + lx;
    if (!IN && (gj < 1 || gj > ny - 2 || gi < 1 || gi > nx - 2)) continue;  // ghost ring written below
    T rhs = T(0);
    if (IN || (gj >= 2 && gj <= ny - 3 && gi >= 2 && gi <= nx - 3))
      rhs = -(divr(fe[ly * (TX + 1) + lx + 1] - fe[ly * (TX + 1) + lx], dx, rdx) +
              divr(fn[(ly + 1) * TX + lx] - fn[ly * TX + lx], dy, rdy));
    T vc = T(0.5) * (vs[(ly + 1) * TX + lx] + vs[ly * TX + lx]);
    rhs = rhs + (-beta * vc);
    size_t g = (size_t)gj * nx + gi;
    if (F) rhs = rhs + F[g];
    if (A.drag != 0.0) {
      const T* p = pt + (ly + 1) * (TX + 2) + (lx + 1);
      T d2x = divr((p[1] - p[0]) - (p[0] - p[-1]), dx * dx, rdx * rdx);
      T d2y = divr((p[TX + 2] - p[0]) - (p[0] - p[-(TX + 2)]), dy * dy, rdy * rdy);
      rhs = rhs - drag * (d2x + d2y);
    }
    if (A.visc != 0.0) {
      const T* q = qt + (ly + H) * QW + (lx + H);
      T d2x = divr((q[1] - q[0]) - (q[0] - q[-1]), dx * dx, rdx * rdx);
      T d2y = divr((q[QW] - q[0]) - (q[0] - q[-QW]), dy * dy, rdy * rdy);
      rhs = rhs + visc * (d2x + d2y);
    }
    T qsv = qt[(ly + H) * QW + (lx + H)];
    T r = cb * qsv;
    if (qn) r = ca * qn[g] + r;
    r = r + cc * rhs;
    out[g] = r;
    if (A.split_hi) {
      const int xi = gi - 1;
      size_t s = (size_t)(gj - 1) * nxi + (A.split_layout ? ((xi & 1) ? (nxi >> 1) + (xi >> 1) : (xi >> 1)) : xi);
      if constexpr (sizeof(T) == 8) {
        ((double*)(void*)A.split_hi)[s] = r;  // FP64: the interior itself
      } else {
        float fv = (float)r;
        __nv_bfloat16 h = __float2bfloat16_rn(fv);
        A.split_hi[s] = h;
        A.split_lo[s] = __float2bfloat16_rn(fv - __bfloat162float(h));
      }
    }
    if (!IN && A.write_ghost && A.periodic) {
      // copies of this interior cell into the ghost ring (S, N, W, E fill)
      int ys[2] = {gj, gj == ny - 2 ? 0 : (gj == 1 ? ny - 1 : -1)};
      int xs[2] = {gi, gi == nx - 2 ? 0 : (gi == 1 ? nx - 1 : -1)};
      for (int a2 = 0; a2 < 2; ++a2)
        for (int b2 = 0; b2 < 2; ++b2) {
          if ((a2 == 0 && b2 == 0) || ys[a2] < 0 || xs[b2] < 0) continue;
          out[(size_t)ys[a2] * nx + xs[b2]] = r;
        }
    }
  }
  if (!IN && A.write_ghost && !A.periodic) {
    for (int k = tid; k < TY * TX; k += THREADS) {
      int ly = k / TX, lx = k - ly * TX;
      int gj = y0 + ly, gi = x0 + lx;
      if (gj < ny && gi < nx && (gj == 0 || gj == ny - 1 || gi == 0 || gi == nx - 1))
        out[(size_t)gj * nx + gi] = T(0);
    }
  }
}

// Tile (x0, y0) of one field: the interior body when the tile, its halo and
// every face's reach lie inside the interior, the general body otherwise.
template <typename T, int S, int TX, int TY>
DEV void stage_tile(const StageArgs& A, uint8_t* sm, int x0, int y0) {
  constexpr int H = SchemeInfo<S>::halo_hi > 3 ? SchemeInfo<S>::halo_hi : 3;
  constexpr int R = SchemeInfo<S>::reach;
  const bool in = x0 - H >= 1 && x0 + TX + H - 1 <= A.nx - 2 && y0 - H >= 1 && y0 + TY + H - 1 <= A.ny - 2 &&
                  x0 - 1 >= R && x0 + TX <= A.nx - 1 - R && y0 - 1 >= R && y0 + TY <= A.ny - 1 - R;
  if (in) stage_body<T, S, true, TX, TY>(A, sm, x0, y0);
  else stage_body<T, S, false, TX, TY>(A, sm, x0, y0);
}

// Interior tile rectangle [txa, txb] x [tya, tyb] (empty when txa > txb or
// tya > tyb): the tiles stage_tile runs with the interior body.  The same
// bounds as stage_tile's test, solved for the tile index.
struct TileSplit {
  int ntx, nty, txa, txb, tya, tyb;
};

template <int S, int TX, int TY>
static TileSplit tile_split(int ny, int nx) {
  constexpr int H = SchemeInfo<S>::halo_hi > 3 ? SchemeInfo<S>::halo_hi : 3;
  constexpr int R = SchemeInfo<S>::reach;
  TileSplit t;
  t.ntx = (nx + TX - 1) / TX;
  t.nty = (ny + TY - 1) / TY;
  auto in_x = [&](int x0) {
    return x0 - H >= 1 && x0 + TX + H - 1 <= nx - 2 && x0 - 1 >= R && x0 + TX <= nx - 1 - R;
  };
  auto in_y = [&](int y0) {
    return y0 - H >= 1 && y0 + TY + H - 1 <= ny - 2 && y0 - 1 >= R && y0 + TY <= ny - 1 - R;
  };
  t.txa = 0; while (t.txa < t.ntx && !in_x(t.txa * TX)) ++t.txa;
  t.txb = t.txa; while (t.txb + 1 < t.ntx && in_x((t.txb + 1) * TX)) ++t.txb;
  t.tya = 0; while (t.tya < t.nty && !in_y(t.tya * TY)) ++t.tya;
  t.tyb = t.tya; while (t.tyb + 1 < t.nty && in_y((t.tyb + 1) * TY)) ++t.tyb;
  if (t.txa >= t.ntx || t.tya >= t.nty) { t.txa = 1; t.txb = 0; t.tya = 1; t.tyb = 0; }  // no interior tile
  return t;
}

// Block b -> tile: the boundary tiles (the slow, general body) get the
// lowest block indices so that they start first instead of forming the
// launch's tail, then the interior rectangle row by row.
DEV void tile_of_block(const TileSplit& t, int b, int& tx, int& ty) {
  const int wi = t.txb - t.txa + 1, hi = t.tyb - t.tya + 1;
  const int ni = (wi > 0 && hi > 0) ? wi * hi : 0;
  const int nb = t.ntx * t.nty - ni;
  if (b >= nb) {
    const int k = b - nb;
    ty = t.tya + k / wi;
    tx = t.txa + k % wi;
    return;
  }
  // rows below the rectangle, rows beside it (the columns outside), rows above
  const int full_lo = ni ? t.tya * t.ntx : nb;
  if (b < full_lo) { ty = b / t.ntx; tx = b % t.ntx; return; }
  const int side = t.ntx - wi;
  const int mid = hi * side;
  if (b < full_lo + mid) {
    const int k = b - full_lo;
    ty = t.tya + k / side;
    const int c = k % side;
    tx = c < t.txa ? c : c + wi;
    return;
  }
  const int k = b - full_lo - mid;
  ty = t.tyb + 1 + k / t.ntx;
  tx = k % t.ntx;
}

template <typename T, int S, int TX, int TY>
__global__ void __launch_bounds__(THREADS)
stage_kernel(StageArgs A, TileSplit ts) {
  extern __shared__ __align__(16) uint8_t sm[];
  // launched programmatically: psi comes from the kernel before this one
  grid_dep_wait();
  grid_dep_launch();
  int tx, ty;
  tile_of_block(ts, blockIdx.x, tx, ty);
  stage_tile<T, S, TX, TY>(A, sm, tx * TX, ty * TY);
}

template <typename T, int S, int TX, int TY>
static size_t smem_bytes() {
  using G = Geom<T, S, TX, TY>;
  return (size_t)(G::NQ + G::NP + G::NWORK) * sizeof(T);
}

}  // namespace qg
}  // namespace fvx
