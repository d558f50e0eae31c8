// Shallow-water operators on the Arakawa C-grid, each one fused kernel:
// Coriolis2D (operators/coriolis.py:34-133), Vorticity2D's potential
// vorticity and PV fluxes (operators/vorticity.py:60-235) and
// MomentumAdvection2D (diffusion/momentum.py:35-216).
//
// The reference composes Interpolation2D / Difference2D calls, each writing
// a full staggered array with a zero ghost ring and (under a mask) the
// output stagger's mask applied.  Here every output cell recomputes the
// intermediates it needs at its neighbours with the same arithmetic, ring
// and mask rules (T -> mask.h, U -> mask.u, V -> mask.v, X ->
// mask.xy_corner_strict), so no intermediate array is written.
#include "fvx_common.cuh"

namespace fvx {
namespace sw {

enum SwOp {
  CORIOLIS = 0,        // (u, v, f) -> (du, dv)
  PV_FLUX_ENERGY = 1,  // (q, u, v) -> (qu, qv)
  PV_FLUX_ENSTROPHY = 2,
  PV_FLUX_AL = 3,      // alpha blend
  MOM_ENERGY = 4,      // (u, v) -> (du, dv)
  MOM_ENSTROPHY = 5,
  MOM_AL = 6,
  POT_VORTICITY = 7,   // (u, v, h, f) -> q
  N_OPS = 8
};

template <typename T>
struct Fields {
  const T *a, *b, *c, *d;
  int ny, nx;
  T dx, dy, alpha, beta;  // beta = 1 - alpha, rounded once from the double
  const uint8_t *mh, *mu, *mv, *mxy;
  int pass_down;  // 1: intermediates carry their stagger's mask (Vorticity2D, MomentumAdvection2D)

  DEV bool in(int j, int i) const { return j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2; }
  DEV T m(const uint8_t* k, int j, int i) const { return (k && pass_down) ? T(k[(size_t)j * nx + i]) : T(1); }
  DEV T at(const T* p, int j, int i) const { return p[(size_t)j * nx + i]; }

  // Interpolation2D / Difference2D primitives at (j, i), ring zero, masked
  DEV T T2U(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j, i + 1)) * m(mu, j, i) : T(0); }
  DEV T T2V(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j + 1, i)) * m(mv, j, i) : T(0); }
  DEV T T2X(const T* p, int j, int i) const {
    return in(j, i) ? T(0.25) * (at(p, j, i) + at(p, j, i + 1) + at(p, j + 1, i) + at(p, j + 1, i + 1)) * m(mxy, j, i)
                    : T(0);
  }
  DEV T X2U(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j - 1, i)) * m(mu, j, i) : T(0); }
  DEV T X2V(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j, i - 1)) * m(mv, j, i) : T(0); }
  DEV T U2X(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j + 1, i)) * m(mxy, j, i) : T(0); }
  DEV T V2X(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j, i + 1)) * m(mxy, j, i) : T(0); }
  DEV T U2T(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j, i - 1)) * m(mh, j, i) : T(0); }
  DEV T V2T(const T* p, int j, int i) const { return in(j, i) ? T(0.5) * (at(p, j, i) + at(p, j - 1, i)) * m(mh, j, i) : T(0); }
  DEV T V2U(const T* p, int j, int i) const {
    return in(j, i) ? T(0.25) * (at(p, j, i) + at(p, j - 1, i) + at(p, j, i + 1) + at(p, j - 1, i + 1)) * m(mu, j, i)
                    : T(0);
  }
  DEV T U2V(const T* p, int j, int i) const {
    return in(j, i) ? T(0.25) * (at(p, j, i) + at(p, j + 1, i) + at(p, j, i - 1) + at(p, j + 1, i - 1)) * m(mv, j, i)
                    : T(0);
  }
  // curl (difference.py:47-59) of (u, v) at X-points
  DEV T curl(const T* u, const T* v, int j, int i) const {
    return in(j, i) ? ((at(v, j, i + 1) - at(v, j, i)) / dx - (at(u, j + 1, i) - at(u, j, i)) / dy) * m(mxy, j, i)
                    : T(0);
  }
  // kinetic energy K at T-points (momentum.py:108-122), ring zero, no mask
  DEV T kin(const T* u, const T* v, int j, int i) const {
    if (!in(j, i)) return T(0);
    const T ut = U2T(u, j, i), vt = V2T(v, j, i);
    return T(0.5) * (ut * ut + vt * vt);
  }
};

template <typename T>
__global__ void sw_kernel(int op, Fields<T> F, T* __restrict__ o1, T* __restrict__ o2) {
  const int ny = F.ny, nx = F.nx;
  const size_t n = (size_t)ny * nx;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(k / nx), i = (int)(k - (size_t)j * nx);
    const bool in = F.in(j, i);
    T r1 = T(0), r2 = T(0);
    switch (op) {
      case CORIOLIS: {  // a = u, b = v, c = f; unmasked interpolation, final mask
        if (in) {
          r1 = F.T2U(F.c, j, i) * F.V2U(F.b, j, i);
          r2 = -F.T2V(F.c, j, i) * F.U2V(F.a, j, i);
        }
        if (F.mu) r1 = r1 * T(F.mu[k]);
        if (F.mv) r2 = r2 * T(F.mv[k]);
        break;
      }
      case PV_FLUX_ENERGY:
      case PV_FLUX_ENSTROPHY:
      case PV_FLUX_AL: {  // a = q, b = u, c = v
        const T* q = F.a;
        T e1 = T(0), e2 = T(0), s1 = T(0), s2 = T(0);
        if (op != PV_FLUX_ENSTROPHY && in) {  // vorticity.py:120-152
          e1 = F.X2U(q, j, i) * F.at(F.b, j, i);
          e2 = F.X2V(q, j, i) * F.at(F.c, j, i);
        }
        if (op != PV_FLUX_ENERGY) {  // vorticity.py:154-188: X_to_U(q * U_to_X(u))
          auto qu = [&](int jj, int ii) { return F.in(jj, ii) ? F.at(q, jj, ii) * F.U2X(F.b, jj, ii) : T(0); };
          auto qv = [&](int jj, int ii) { return F.in(jj, ii) ? F.at(q, jj, ii) * F.V2X(F.c, jj, ii) : T(0); };
          if (in) {
            s1 = T(0.5) * (qu(j, i) + qu(j - 1, i)) * F.m(F.mu, j, i);
            s2 = T(0.5) * (qv(j, i) + qv(j, i - 1)) * F.m(F.mv, j, i);
          }
        }
        if (op == PV_FLUX_ENERGY) { r1 = e1; r2 = e2; }
        else if (op == PV_FLUX_ENSTROPHY) { r1 = s1; r2 = s2; }
        else {  // vorticity.py:190-235
          r1 = F.alpha * e1 + F.beta * s1;
          r2 = F.alpha * e2 + F.beta * s2;
        }
        break;
      }
      case MOM_ENERGY:
      case MOM_ENSTROPHY:
      case MOM_AL: {  // a = u, b = v; momentum.py:124-216
        const T *u = F.a, *v = F.b;
        if (j >= 2 && j <= ny - 3 && i >= 2 && i <= nx - 3) {
          T e1 = T(0), e2 = T(0), s1 = T(0), s2 = T(0);
          auto z = [&](int jj, int ii) { return F.curl(u, v, jj, ii); };
          if (op != MOM_ENSTROPHY) {  // E-scheme
            const T zu = F.in(j, i) ? T(0.5) * (z(j, i) + z(j - 1, i)) * F.m(F.mu, j, i) : T(0);
            const T zv = F.in(j, i) ? T(0.5) * (z(j, i) + z(j, i - 1)) * F.m(F.mv, j, i) : T(0);
            e1 = zu * F.V2U(v, j, i);
            e2 = zv * F.U2V(u, j, i);
          }
          if (op != MOM_ENERGY) {  // Z-scheme
            auto zvq = [&](int jj, int ii) { return F.in(jj, ii) ? z(jj, ii) * F.V2X(v, jj, ii) : T(0); };
            auto zuq = [&](int jj, int ii) { return F.in(jj, ii) ? z(jj, ii) * F.U2X(u, jj, ii) : T(0); };
            s1 = T(0.5) * (zvq(j, i) + zvq(j - 1, i)) * F.m(F.mu, j, i);
            s2 = T(0.5) * (zuq(j, i) + zuq(j, i - 1)) * F.m(F.mv, j, i);
          }
          T zvu, zuv;
          if (op == MOM_ENERGY) { zvu = e1; zuv = e2; }
          else if (op == MOM_ENSTROPHY) { zvu = s1; zuv = s2; }
          else { zvu = F.alpha * e1 + F.beta * s1; zuv = F.alpha * e2 + F.beta * s2; }
          const T dkdx = (F.kin(u, v, j, i + 1) - F.kin(u, v, j, i)) / F.dx * F.m(F.mu, j, i);
          const T dkdy = (F.kin(u, v, j + 1, i) - F.kin(u, v, j, i)) / F.dy * F.m(F.mv, j, i);
          r1 = zvu - dkdx;
          r2 = -zuv - dkdy;
        }
        if (F.mu) r1 = r1 * T(F.mu[k]);
        if (F.mv) r2 = r2 * T(F.mv[k]);
        break;
      }
      case POT_VORTICITY: {  // a = u, b = v, c = h, d = f; vorticity.py:60-118
        if (in) {
          const T num = F.curl(F.a, F.b, j, i) + F.T2X(F.d, j, i);
          const T den = F.T2X(F.c, j, i);
          r1 = den == T(0) ? T(NAN) : num / den;
        }
        if (F.mxy && F.pass_down && !F.mxy[k]) r1 = T(0);
        break;
      }
    }
    o1[k] = r1;
    if (o2) o2[k] = r2;
  }
}

static int grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace sw
}  // namespace fvx

using namespace fvx;
using namespace fvx::sw;

// op as SwOp; a..d inputs (see SwOp); masks may be NULL (unmasked);
// out2 unused (NULL) for POT_VORTICITY.  Coriolis applies mask_u / mask_v
// to its outputs only; the others pass the masks down to every
// intermediate like the reference's masked Difference2D / Interpolation2D.
#define FVX_DEF_SW(SFX, T)                                                                                        \
  extern "C" int fvx_sw2d_##SFX(int op, const T* a, const T* b, const T* c, const T* d, T* out1, T* out2, int ny, \
                                int nx, double dx, double dy, double alpha, const uint8_t* mask_h,               \
                                const uint8_t* mask_u, const uint8_t* mask_v, const uint8_t* mask_xy,            \
                                void* stream) {                                                                   \
    if (op < 0 || op >= N_OPS) return FVX_ERR_METHOD;                                                             \
    if (!a || !b || !out1 || (op != POT_VORTICITY && !out2)) return FVX_ERR_ARG;                                  \
    if ((op <= PV_FLUX_AL || op == POT_VORTICITY) && !c) return FVX_ERR_ARG;                                      \
    if (op == POT_VORTICITY && !d) return FVX_ERR_ARG;                                                            \
    if (ny < 3 || nx < 3) return FVX_ERR_SHAPE;                                                                   \
    Fields<T> F{a, b, c, d, ny, nx, T(dx), T(dy), T(alpha), T(1.0 - alpha), mask_h, mask_u, mask_v, mask_xy,     \
                op == CORIOLIS ? 0 : 1};                                                                          \
    sw_kernel<T><<<grid_for((size_t)ny * nx), 256, 0, fvx_stream(stream)>>>(op, F, out1, out2);                   \
    return fvx_cuda_status();                                                                                     \
  }

FVX_DEF_SW(f32, float)
FVX_DEF_SW(f64, double)
