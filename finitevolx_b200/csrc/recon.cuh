// Face-value reconstructions for flux-form advection on the C-grid.
//
// Point formulas restate finitevolX advection/weno.py (WENO3/5 JS and Z,
// WENO7/9 via the generic Jiang-Shu form) and advection/limiters.py, with
// the same operation order so the FP64 build tracks the reference to
// rounding.  The boundary fallback ladders of advection/reconstruction.py
// (WENO5 :834-864, WENO7/9 :74-236, upwind2/3 and TVD east-boundary
// fallbacks) all reduce to one rule, used by face_value() below:
//
//   c = upwind cell of face i (i for u >= 0, i+1 for u < 0), N = line length,
//   d = min(c, N-1-c) cells available on the short side of c,
//   reach = min(scheme reach, d): 0 -> first-order upwind h[c],
//   1 -> WENO3, 2 -> WENO5, 3 -> WENO7, 4 -> WENO9 (same bias and family).
#pragma once
#include "fvx_common.cuh"
#include "weno_tables.cuh"

namespace fvx {

template <typename T> DEV T sq(T x) { return x * x; }
// FP32 reciprocal by the hardware approximation (rcp.approx.ftz.f32, at
// most 1 ulp): +inf for 0, 0 for |b| > 2^126 (the result would be
// subnormal and is flushed).
DEV float rcp_approx(float b) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
  return r;
}
// Division in the reconstruction formulas: exact IEEE division in FP64 (the
// correctness path tracks the reference's operation order), a times the
// approximate reciprocal of b in FP32 (<= 2 ulp; its 2^126 < |b| < 2^128
// corner maps to the weights an FP32 reference overflows on anyway).
template <typename T> DEV T fdiv(T a, T b) {
  if constexpr (sizeof(T) == 8) return a / b;
  else return a * rcp_approx(b);
}
template <typename T> DEV T tabs(T x) { return x < T(0) ? -x : x; }
template <typename T> DEV T tmax(T a, T b) { return a > b ? a : b; }
template <typename T> DEV T tmin(T a, T b) { return a < b ? a : b; }

// ---- WENO3 (advection/weno.py:297-347) ------------------------------------
// The right-biased forms (:413-459, :462-522, :597-665) are these functions on
// the mirrored stencil; face_value() below feeds them that way.
template <typename T> DEV T weno3(T qm, T q0, T qp) {
  const T eps = T(1e-8);
  T qi1 = T(-0.5) * qm + T(1.5) * q0;
  T qi2 = T(0.5) * (q0 + qp);
  T w1 = fdiv(T(1.0 / 3.0), sq(sq(q0 - qm) + eps));
  T w2 = fdiv(T(2.0 / 3.0), sq(sq(qp - q0) + eps));
  return fdiv(w1 * qi1 + w2 * qi2, w1 + w2);
}
template <typename T> DEV T wenoz3(T qm, T q0, T qp) {
  const T eps = T(1e-14);
  T qi1 = T(-0.5) * qm + T(1.5) * q0;
  T qi2 = T(0.5) * (q0 + qp);
  T b1 = sq(q0 - qm), b2 = sq(qp - q0);
  T tau = tabs(b2 - b1);
  T w1 = T(1.0 / 3.0) * (T(1) + fdiv(tau, b1 + eps));
  T w2 = T(2.0 / 3.0) * (T(1) + fdiv(tau, b2 + eps));
  return fdiv(w1 * qi1 + w2 * qi2, w1 + w2);
}
// ---- WENO5 (advection/weno.py:350-410, :462-522) -------------------------
template <typename T, bool Z>
DEV T weno5_core(T qi1, T qi2, T qi3, T b1, T b2, T b3) {
  if (Z) {
    const T eps = T(1e-16);
    T tau5 = tabs(b1 - b3);
    T w1 = T(0.1) * (T(1) + fdiv(tau5, b1 + eps));
    T w2 = T(0.6) * (T(1) + fdiv(tau5, b2 + eps));
    T w3 = T(0.3) * (T(1) + fdiv(tau5, b3 + eps));
    return fdiv(w1 * qi1 + w2 * qi2 + w3 * qi3, w1 + w2 + w3);
  } else {
    const T eps = T(1e-8);
    if constexpr (sizeof(T) == 4) {
      // FP32: the weights d_k / s_k (s_k = (b_k + eps)^2) times s1 s2 s3,
      // d_k prod_{j != k} s_j, give the same normalised combination with one
      // reciprocal instead of four.  s_k >= 1e-16, so no product underflows;
      // the few stencils whose products overflow (|q| jumps above ~1e4) take
      // the four-division form.
      const float s1 = sq(b1 + eps), s2 = sq(b2 + eps), s3 = sq(b3 + eps);
      const float W1 = 0.1f * (s2 * s3), W2 = 0.6f * (s1 * s3), W3 = 0.3f * (s1 * s2);
      const float den = W1 + W2 + W3;
      const float r = (W1 * qi1 + W2 * qi2 + W3 * qi3) * rcp_approx(den);
      if (den < 3e38f && fabsf(r) < 3.4e38f) return r;
    }
    T w1 = fdiv(T(0.1), sq(b1 + eps));
    T w2 = fdiv(T(0.6), sq(b2 + eps));
    T w3 = fdiv(T(0.3), sq(b3 + eps));
    return fdiv(w1 * qi1 + w2 * qi2 + w3 * qi3, w1 + w2 + w3);
  }
}
template <typename T, bool Z> DEV T weno5(T qmm, T qm, T q0, T qp, T qpp) {
  const T k1 = T(13.0 / 12.0), k2 = T(0.25);
  T qi1 = T(1.0 / 3.0) * qmm - T(7.0 / 6.0) * qm + T(11.0 / 6.0) * q0;
  T qi2 = T(-1.0 / 6.0) * qm + T(5.0 / 6.0) * q0 + T(1.0 / 3.0) * qp;
  T qi3 = T(1.0 / 3.0) * q0 + T(5.0 / 6.0) * qp - T(1.0 / 6.0) * qpp;
  T b1 = k1 * sq(qmm - T(2) * qm + q0) + k2 * sq(qmm - T(4) * qm + T(3) * q0);
  T b2 = k1 * sq(qm - T(2) * q0 + qp) + k2 * sq(qm - qp);
  T b3 = k1 * sq(q0 - T(2) * qp + qpp) + k2 * sq(T(3) * q0 - T(4) * qp + qpp);
  return weno5_core<T, Z>(qi1, qi2, qi3, b1, b2, b3);
}
// ---- WENO7 / WENO9, generic Jiang-Shu form (advection/weno.py:268-294) ---
template <typename T> DEV T tab_c(int R, int k, int j) {
  if constexpr (sizeof(T) == 8) return R == 4 ? kW7_C[k][j] : kW9_C[k][j];
  else return R == 4 ? kW7_Cf[k][j] : kW9_Cf[k][j];
}
template <typename T> DEV T tab_w(int R, int k) {
  if constexpr (sizeof(T) == 8) return R == 4 ? kW7_W[k] : kW9_W[k];
  else return R == 4 ? kW7_Wf[k] : kW9_Wf[k];
}
template <typename T> DEV T tab_b(int R, int k, int i, int j) {
  if constexpr (sizeof(T) == 8) return R == 4 ? kW7_B[k][i][j] : kW9_B[k][i][j];
  else return R == 4 ? kW7_Bf[k][i][j] : kW9_Bf[k][i][j];
}

// v[0..2R-2]: the 2R-1 cells of the big stencil ordered in the upwind
// direction (the mirrored, negative-flow tables of the reference are the
// left-biased tables on the reversed stencil).
//
// FP32: the quadratic forms have O(10^3) alternating coefficients, so on raw
// values they lose ~4 digits to cancellation against the local mean.  The
// FP32 build evaluates them (and the candidates) on values shifted by the
// stencil centre s: exact algebra, because every form annihilates constants
// (B 1 = 0) and every candidate's weights sum to one, so
// cand(v) = s + cand(v - s) and beta(v) = beta(v - s).  FP64 keeps the
// reference's raw-value evaluation order.
template <typename T, int R>
DEV T weno_generic(const T* vin) {
  const T eps = T(1e-8);
  constexpr bool SHIFT = sizeof(T) == 4;
  const T s = SHIFT ? vin[R - 1] : T(0);
  T v[2 * R - 1];
#pragma unroll
  for (int k = 0; k < 2 * R - 1; ++k) v[k] = SHIFT ? vin[k] - s : vin[k];
  T num = T(0), den = T(0);
#pragma unroll
  for (int k = 0; k < R; ++k) {
    T cand = T(0);
#pragma unroll
    for (int j = 0; j < R; ++j) cand = cand + tab_c<T>(R, k, j) * v[k + j];
    T beta = T(0);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      T row = T(0);
#pragma unroll
      for (int j = 0; j < R; ++j) row = row + tab_b<T>(R, k, i, j) * v[k + j];
      beta = beta + v[k + i] * row;
    }
    T a = fdiv(tab_w<T>(R, k), sq(beta + eps));
    den = den + a;
    num = num + a * cand;
  }
  return SHIFT ? s + fdiv(num, den) : num / den;
}

// ---- limiters (advection/limiters.py:34-123) -----------------------------
template <typename T, int S> DEV T limiter(T r) {
  if (S == FVX_MINMOD) return tmax(T(0), tmin(T(1), r));
  if (S == FVX_VAN_LEER) { T ra = tabs(r); return (r + ra) / (T(1) + ra); }
  if (S == FVX_SUPERBEE) return tmax(T(0), tmax(tmin(T(2) * r, T(1)), tmin(r, T(2))));
  return tmax(T(0), tmin(tmin((T(1) + r) / T(2), T(2) * r), T(2)));  // MC
}

template <int S> struct SchemeInfo {
  static constexpr bool is_weno = (S == FVX_WENO3 || S == FVX_WENOZ3 || S == FVX_WENO5 ||
                                   S == FVX_WENOZ5 || S == FVX_WENO7 || S == FVX_WENO9);
  static constexpr int reach = (S == FVX_WENO3 || S == FVX_WENOZ3) ? 1
                               : (S == FVX_WENO5 || S == FVX_WENOZ5) ? 2
                               : (S == FVX_WENO7) ? 3 : (S == FVX_WENO9) ? 4 : 1;
  static constexpr bool zfam = (S == FVX_WENOZ3 || S == FVX_WENOZ5);
  static constexpr bool tvd = (S == FVX_MINMOD || S == FVX_VAN_LEER || S == FVX_SUPERBEE || S == FVX_MC);
  // cells read on each side of the face's left cell i: [i - lo, i + hi]
  static constexpr int halo_lo = is_weno ? reach + 1 : 1;
  static constexpr int halo_hi = is_weno ? reach + 1 : 2;
};

// Face value at face i (between cells i and i+1) of a line of N cells.
// ``p`` points at cell i; neighbours are p[k*st].  pos: u >= 0.
// Valid for 1 <= i <= N-2 (the faces the reference reconstructs).
template <typename T, int S>
DEV T face_value(const T* p, int st, int i, int N, bool pos) {
  auto at = [&](int k) -> T { return p[k * st]; };
  if (S == FVX_NAIVE) return T(0.5) * (at(0) + at(1));
  if (S == FVX_UPWIND1) return pos ? at(0) : at(1);
  if (S == FVX_UPWIND2) {
    if (pos) return T(1.5) * at(0) - T(0.5) * at(-1);
    return (i <= N - 3) ? T(1.5) * at(1) - T(0.5) * at(2) : at(1);
  }
  if (S == FVX_UPWIND3) {
    if (pos) return T(-1.0 / 6.0) * at(-1) + T(5.0 / 6.0) * at(0) + T(1.0 / 3.0) * at(1);
    return (i <= N - 3) ? T(1.0 / 3.0) * at(0) + T(5.0 / 6.0) * at(1) - T(1.0 / 6.0) * at(2) : at(1);
  }
  if constexpr (SchemeInfo<S>::tvd) {
    if (pos) {
      T dfwd = at(1) - at(0);
      T dbwd = at(0) - at(-1);
      T r = dbwd / (dfwd + T(1e-8));
      return at(0) + T(0.5) * limiter<T, S>(r) * dfwd;
    }
    if (i > N - 3) return at(1);
    T dn = at(0) - at(1);
    T dn2 = at(1) - at(2);
    T r = dn2 / (dn + T(1e-8));
    return at(1) + T(0.5) * limiter<T, S>(r) * dn;
  }
  if constexpr (SchemeInfo<S>::is_weno) {
    // Upwind-oriented stencil: e(k) is the cell k steps downstream of the
    // upwind cell c (pos: h[i+k], neg: h[i+1-k]).  Every right-biased formula
    // of the reference is the left-biased one on the mirrored stencil (same
    // candidates, same smoothness squares, same weights), so both flow
    // directions run one code path and warps do not diverge on the sign.
    constexpr bool Z = SchemeInfo<S>::zfam;
    const int c = pos ? i : i + 1;
    const int d = min(c, N - 1 - c);
    const int r = min(SchemeInfo<S>::reach, d);
    const T* b = pos ? p : p + st;
    const int s = pos ? st : -st;
    auto e = [&](int k) -> T { return b[k * s]; };
    if (r >= 4) {
      T v[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) v[k] = e(k - 4);
      return weno_generic<T, 5>(v);
    }
    if (r == 3) {
      T v[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) v[k] = e(k - 3);
      return weno_generic<T, 4>(v);
    }
    if (r == 2) return weno5<T, Z>(e(-2), e(-1), e(0), e(1), e(2));
    if (r == 1) return Z ? wenoz3(e(-1), e(0), e(1)) : weno3(e(-1), e(0), e(1));
    return e(0);
  }
  return T(0);
}

}  // namespace fvx
