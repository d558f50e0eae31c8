"""FP64 NumPy restatement of finitevolX's hot path -- TEST INFRASTRUCTURE ONLY.

This module is the oracle for the parity tests of ``finitevolx_b200``.  It is
never imported by the product library; only ``tests/``, ``__graft_entry__``'s
``smoke()`` and ``bench.py``'s CPU-baseline legs use it.

Every function cites the reference file:line (paths inside the finitevolX
project) whose arithmetic it restates.  Array conventions follow the
reference: total shape ``[Ny, Nx]`` with a one-cell ghost ring; same-index
stagger (U[j,i] at i+1/2, V[j,i] at j+1/2, X[j,i] at the NE corner).

Pinning (which results are checked against the reference's own data):
  * masks, Advection2D upwind1/weno5, Difference2D, Interpolation2D,
    Diffusion2D, BiharmonicDiffusion2D: the reference's FP64 golden ``.npz``
    fixtures (tests/fixtures/golden) at rtol 1e-12 / atol 1e-14;
  * WENO point reconstructions, limiters, Jacobian, RK steppers, masks:
    known-answer tests restated from the reference's test suite;
  * solve_helmholtz_dst: third-party (spectraldiffx v0.0.10, commit
    eac31a578ae31da61fa855cccc594459722e1517); pinned by the exact discrete
    identity (5-point Dirichlet operator minus lambda applied to the
    solution reproduces the right-hand side), not by a golden vector;
  * CG: third-party (lineax 0.1.0); iterate-level parity unpinned, pinned by
    the outcome tests (converged flag, residual bound);
  * solve_helmholtz_dct / solve_helmholtz_fft / capacitance_solve:
    third-party (spectraldiffx v0.0.10, as above); pinned by the discrete
    identities (the Neumann / periodic 5-point operator minus lambda applied
    to the solution reproduces the right-hand side, less its mean when
    lambda = 0) and by the reference's own capacitance tests (the solution
    vanishes on the inner-boundary points; no boundary point is an error).
"""

from __future__ import annotations

import math

import numpy as np

# ---------------------------------------------------------------------------
# Grid  (grid/cartesian.py:83-108)
# ---------------------------------------------------------------------------


def grid_from_interior(nx_interior, ny_interior, Lx, Ly):
    """CartesianGrid2D.from_interior (grid/cartesian.py:83-108)."""
    return dict(Nx=nx_interior + 2, Ny=ny_interior + 2, Lx=Lx, Ly=Ly,
                dx=Lx / nx_interior, dy=Ly / ny_interior)


# ---------------------------------------------------------------------------
# Mask primitives  (mask/utils.py)
# ---------------------------------------------------------------------------


def pool_bool(arr, kernel, threshold, direction="leading"):
    """Windowed mean of a 0/1 mask vs a threshold (mask/utils.py:42-164)."""
    arr_f = np.asarray(arr).astype(float)
    if direction == "leading":
        pads = tuple((k - 1, 0) for k in kernel)
    else:
        pads = tuple((0, k - 1) for k in kernel)
    padded = np.pad(arr_f, pads)
    total = np.zeros_like(arr_f)
    import itertools
    for offs in itertools.product(*(range(k) for k in kernel)):
        sl = tuple(slice(o, o + s) for o, s in zip(offs, arr_f.shape))
        total += padded[sl]
    return total / float(np.prod(kernel)) > threshold


def dilate_mask(mask):
    """Cross-shaped binary dilation, zero border (mask/utils.py:314-382)."""
    m = np.asarray(mask, dtype=bool)
    out = m.copy()
    for ax in range(m.ndim):
        lo = [slice(None)] * m.ndim
        hi = [slice(None)] * m.ndim
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        out[tuple(lo)] |= m[tuple(hi)]
        out[tuple(hi)] |= m[tuple(lo)]
    return out


def count_contiguous(arr, axis, forward):
    """Run length of wet cells from each cell (mask/utils.py:385-468)."""
    a = np.moveaxis(np.asarray(arr, dtype=np.int32), axis, 0)
    n = a.shape[0]
    c = np.zeros_like(a)
    if forward:
        c[-1] = a[-1]
        for i in range(n - 2, -1, -1):
            c[i] = a[i] * (1 + c[i + 1])
    else:
        c[0] = a[0]
        for i in range(1, n):
            c[i] = a[i] * (1 + c[i - 1])
    return np.moveaxis(c, 0, axis)


def make_sponge(shape, width):
    """Linear float32 sponge ramp (mask/utils.py:471-546)."""
    if width is None or width <= 0:
        return np.ones(shape, dtype=np.float32)
    w = float(width)
    out = np.ones(shape, dtype=np.float32)
    for ax, n in enumerate(shape):
        idx = np.arange(n, dtype=np.float32)
        ramp = np.clip(np.minimum(idx, (n - 1) - idx) / w, 0.0, 1.0)
        bshape = [1] * len(shape)
        bshape[ax] = n
        out = out * ramp.reshape(bshape)
    return out


def mask2d_from_mask(mask_hgrid, sponge_width=None):
    """Mask2D.from_mask (mask/cartesian.py:584-739); returns a dict."""
    h = np.asarray(mask_hgrid, dtype=bool)
    Ny, Nx = h.shape
    hf = h.astype(np.float32)
    u = pool_bool(hf, (1, 2), 3.0 / 4.0, "trailing")
    v = pool_bool(hf, (2, 1), 3.0 / 4.0, "trailing")
    xy = pool_bool(hf, (2, 2), 1.0 / 8.0, "trailing")
    xys = pool_bool(hf, (2, 2), 7.0 / 8.0, "trailing")
    u_north = np.pad(u[1:, :], ((0, 1), (0, 0)))
    v_east = np.pad(v[:, 1:], ((0, 0), (0, 1)))
    y_wall = xy & (~u | ~u_north)
    x_wall = xy & (~v | ~v_east)
    convex = y_wall & x_wall
    valid = xy & u & u_north & v & v_east
    if Ny >= 3 and Nx >= 3:
        psif = xys.astype(np.float32)
        pool3 = np.zeros((Ny - 2, Nx - 2), dtype=np.float32)
        for di in range(3):
            for dj in range(3):
                pool3 += psif[di:Ny - 2 + di, dj:Nx - 2 + dj]
        pool3 /= 9.0
        irr = (~xys[1:-1, 1:-1]) & (pool3 > 1.0 / 18.0)
        rows, cols = np.where(irr)
        rows = (rows + 1).astype(np.int32)
        cols = (cols + 1).astype(np.int32)
    else:
        rows = np.empty(0, np.int32)
        cols = np.empty(0, np.int32)
    land = ~h
    d1 = dilate_mask(land)
    coast = h & d1
    d2 = dilate_mask(d1)
    near = h & d2 & ~coast
    ocean = h & ~d2
    cls = np.zeros((Ny, Nx), np.int32)
    cls[coast] = 1
    cls[near] = 2
    cls[ocean] = 3
    if sponge_width is None or sponge_width == 0:
        sponge = np.ones((Ny, Nx), np.float32)
    else:
        if sponge_width < 0:
            raise ValueError(f"sponge_width must be non-negative; got {sponge_width!r}")
        sponge = make_sponge((Ny, Nx), sponge_width)
    return dict(
        h=h, u=u, v=v, xy_corner=xy, xy_corner_strict=xys,
        not_h=~h, not_u=~u, not_v=~v, not_xy_corner=~xy, not_xy_corner_strict=~xys,
        xy_corner_y_wall=y_wall, xy_corner_x_wall=x_wall,
        xy_corner_convex=convex, xy_corner_valid=valid,
        xy_corner_strict_irrbound_rows=rows, xy_corner_strict_irrbound_cols=cols,
        classification=cls,
        x_pos=count_contiguous(h, 1, True), x_neg=count_contiguous(h, 1, False),
        y_pos=count_contiguous(h, 0, True), y_neg=count_contiguous(h, 0, False),
        sponge=sponge,
    )


def adaptive_masks(cnt_pos, cnt_neg, sizes):
    """Mask2D.get_adaptive_masks tier split (mask/cartesian.py:495-553)."""
    max_s = np.zeros(cnt_pos.shape, np.int32)
    for s in sorted(sizes):
        hw = s // 2
        can = (cnt_pos >= hw) & (cnt_neg >= hw)
        max_s = np.where(can, s, max_s)
    return {s: (max_s == s) for s in sizes}


def narrow_mask_hierarchy(hier, sizes):
    """OR-fold tiers >= the largest target (advection/flux.py:41-97)."""
    ss = sorted(sizes)
    out = {s: hier[s] for s in ss[:-1]}
    fold = None
    for s, m in hier.items():
        if s >= ss[-1]:
            fold = m if fold is None else (fold | m)
    out[ss[-1]] = fold
    return out


# ---------------------------------------------------------------------------
# WENO point reconstructions  (advection/weno.py)
# ---------------------------------------------------------------------------


def weno3(qm, q0, qp):
    """weno_3pts (advection/weno.py:297-320)."""
    eps = 1e-8
    qi1 = -1.0 / 2.0 * qm + 3.0 / 2.0 * q0
    qi2 = 1.0 / 2.0 * (q0 + qp)
    b1 = (q0 - qm) ** 2
    b2 = (qp - q0) ** 2
    w1 = (1.0 / 3.0) / (b1 + eps) ** 2
    w2 = (2.0 / 3.0) / (b2 + eps) ** 2
    return (w1 * qi1 + w2 * qi2) / (w1 + w2)


def wenoz3(qm, q0, qp):
    """weno_3pts_improved (advection/weno.py:323-347)."""
    eps = 1e-14
    qi1 = -1.0 / 2.0 * qm + 3.0 / 2.0 * q0
    qi2 = 1.0 / 2.0 * (q0 + qp)
    b1 = (q0 - qm) ** 2
    b2 = (qp - q0) ** 2
    tau = np.abs(b2 - b1)
    w1 = (1.0 / 3.0) * (1.0 + tau / (b1 + eps))
    w2 = (2.0 / 3.0) * (1.0 + tau / (b2 + eps))
    return (w1 * qi1 + w2 * qi2) / (w1 + w2)


def weno3_right(q0, qp, qpp):
    """weno_3pts_right (advection/weno.py:413-435)."""
    eps = 1e-8
    qi1 = 0.5 * (q0 + qp)
    qi2 = 1.5 * qp - 0.5 * qpp
    b1 = (qp - q0) ** 2
    b2 = (qpp - qp) ** 2
    w1 = (2.0 / 3.0) / (b1 + eps) ** 2
    w2 = (1.0 / 3.0) / (b2 + eps) ** 2
    return (w1 * qi1 + w2 * qi2) / (w1 + w2)


def wenoz3_right(q0, qp, qpp):
    """weno_3pts_improved_right (advection/weno.py:438-459)."""
    eps = 1e-14
    qi1 = 0.5 * (q0 + qp)
    qi2 = 1.5 * qp - 0.5 * qpp
    b1 = (qp - q0) ** 2
    b2 = (qpp - qp) ** 2
    tau = np.abs(b2 - b1)
    w1 = (2.0 / 3.0) * (1.0 + tau / (b1 + eps))
    w2 = (1.0 / 3.0) * (1.0 + tau / (b2 + eps))
    return (w1 * qi1 + w2 * qi2) / (w1 + w2)


def weno5(qmm, qm, q0, qp, qpp):
    """weno_5pts (advection/weno.py:350-376)."""
    eps = 1e-8
    qi1 = 1.0 / 3.0 * qmm - 7.0 / 6.0 * qm + 11.0 / 6.0 * q0
    qi2 = -1.0 / 6.0 * qm + 5.0 / 6.0 * q0 + 1.0 / 3.0 * qp
    qi3 = 1.0 / 3.0 * q0 + 5.0 / 6.0 * qp - 1.0 / 6.0 * qpp
    k1, k2 = 13.0 / 12.0, 0.25
    b1 = k1 * (qmm - 2 * qm + q0) ** 2 + k2 * (qmm - 4 * qm + 3 * q0) ** 2
    b2 = k1 * (qm - 2 * q0 + qp) ** 2 + k2 * (qm - qp) ** 2
    b3 = k1 * (q0 - 2 * qp + qpp) ** 2 + k2 * (3 * q0 - 4 * qp + qpp) ** 2
    w1 = 0.1 / (b1 + eps) ** 2
    w2 = 0.6 / (b2 + eps) ** 2
    w3 = 0.3 / (b3 + eps) ** 2
    return (w1 * qi1 + w2 * qi2 + w3 * qi3) / (w1 + w2 + w3)


def wenoz5(qmm, qm, q0, qp, qpp):
    """weno_5pts_improved (advection/weno.py:379-410)."""
    eps = 1e-16
    qi1 = 1.0 / 3.0 * qmm - 7.0 / 6.0 * qm + 11.0 / 6.0 * q0
    qi2 = -1.0 / 6.0 * qm + 5.0 / 6.0 * q0 + 1.0 / 3.0 * qp
    qi3 = 1.0 / 3.0 * q0 + 5.0 / 6.0 * qp - 1.0 / 6.0 * qpp
    k1, k2 = 13.0 / 12.0, 0.25
    b1 = k1 * (qmm - 2 * qm + q0) ** 2 + k2 * (qmm - 4 * qm + 3 * q0) ** 2
    b2 = k1 * (qm - 2 * q0 + qp) ** 2 + k2 * (qm - qp) ** 2
    b3 = k1 * (q0 - 2 * qp + qpp) ** 2 + k2 * (3 * q0 - 4 * qp + qpp) ** 2
    tau5 = np.abs(b1 - b3)
    w1 = 0.1 * (1 + tau5 / (b1 + eps))
    w2 = 0.6 * (1 + tau5 / (b2 + eps))
    w3 = 0.3 * (1 + tau5 / (b3 + eps))
    return (w1 * qi1 + w2 * qi2 + w3 * qi3) / (w1 + w2 + w3)


def weno5_right(qm, q0, qp, qpp, qppp):
    """weno_5pts_right (advection/weno.py:462-491)."""
    eps = 1e-8
    qi1 = 1.0 / 3.0 * qppp - 7.0 / 6.0 * qpp + 11.0 / 6.0 * qp
    qi2 = -1.0 / 6.0 * qpp + 5.0 / 6.0 * qp + 1.0 / 3.0 * q0
    qi3 = 1.0 / 3.0 * qp + 5.0 / 6.0 * q0 - 1.0 / 6.0 * qm
    k1, k2 = 13.0 / 12.0, 0.25
    b1 = k1 * (qp - 2 * qpp + qppp) ** 2 + k2 * (3 * qp - 4 * qpp + qppp) ** 2
    b2 = k1 * (q0 - 2 * qp + qpp) ** 2 + k2 * (q0 - qpp) ** 2
    b3 = k1 * (qm - 2 * q0 + qp) ** 2 + k2 * (qm - 4 * q0 + 3 * qp) ** 2
    w1 = 0.1 / (b1 + eps) ** 2
    w2 = 0.6 / (b2 + eps) ** 2
    w3 = 0.3 / (b3 + eps) ** 2
    return (w1 * qi1 + w2 * qi2 + w3 * qi3) / (w1 + w2 + w3)


def wenoz5_right(qm, q0, qp, qpp, qppp):
    """weno_5pts_improved_right (advection/weno.py:494-522)."""
    eps = 1e-16
    qi1 = 1.0 / 3.0 * qppp - 7.0 / 6.0 * qpp + 11.0 / 6.0 * qp
    qi2 = -1.0 / 6.0 * qpp + 5.0 / 6.0 * qp + 1.0 / 3.0 * q0
    qi3 = 1.0 / 3.0 * qp + 5.0 / 6.0 * q0 - 1.0 / 6.0 * qm
    k1, k2 = 13.0 / 12.0, 0.25
    b1 = k1 * (qp - 2 * qpp + qppp) ** 2 + k2 * (3 * qp - 4 * qpp + qppp) ** 2
    b2 = k1 * (q0 - 2 * qp + qpp) ** 2 + k2 * (q0 - qpp) ** 2
    b3 = k1 * (qm - 2 * q0 + qp) ** 2 + k2 * (qm - 4 * q0 + 3 * qp) ** 2
    tau5 = np.abs(b1 - b3)
    w1 = 0.1 * (1 + tau5 / (b1 + eps))
    w2 = 0.6 * (1 + tau5 / (b2 + eps))
    w3 = 0.3 * (1 + tau5 / (b3 + eps))
    return (w1 * qi1 + w2 * qi2 + w3 * qi3) / (w1 + w2 + w3)


# WENO7 / WENO9 tables: finite-volume Jiang-Shu coefficients, optimal weights
# and smoothness quadratic forms (advection/weno.py:7-253, mirrored :525-535).
# These are published constants of the scheme; they are generated here from
# their definition (Lagrange cell-average reconstruction and the Jiang-Shu
# integral of squared derivatives) rather than typed in, and a unit test
# checks the generated tables against the reference's values.


def _fv_inverse(r, k):
    """Exact map from the r cell averages of candidate k to polynomial coeffs.

    Candidate k (k = 0..r-1) covers cells at offsets -(r-1-k) .. k relative
    to the target cell, which spans [-1/2, 1/2] (unit spacing).  Returns
    Ainv (Fractions) with p(x) = sum_a c_a x^a, c = Ainv @ averages.
    """
    from fractions import Fraction
    shift = r - 1 - k
    offs = [j - shift for j in range(r)]
    A = []
    for o in offs:
        hi, lo = Fraction(2 * o + 1, 2), Fraction(2 * o - 1, 2)
        A.append([(hi ** (a + 1) - lo ** (a + 1)) / (a + 1) for a in range(r)])
    n = r
    M = [A[i][:] + [Fraction(int(i == j)) for j in range(n)] for i in range(n)]
    for c in range(n):
        p = next(i for i in range(c, n) if M[i][c] != 0)
        M[c], M[p] = M[p], M[c]
        pv = M[c][c]
        M[c] = [x / pv for x in M[c]]
        for i in range(n):
            if i != c and M[i][c] != 0:
                f = M[i][c]
                M[i] = [x - f * y for x, y in zip(M[i], M[c])]
    return [row[n:] for row in M]


def _fv_face_coeffs_exact(r, k):
    """Weights of candidate k's reconstruction at the face x = +1/2."""
    from fractions import Fraction
    Ainv = _fv_inverse(r, k)
    return [sum(Ainv[a][j] * Fraction(1, 2) ** a for a in range(r)) for j in range(r)]


def _fv_candidate_coeffs(r):
    """r-point candidate reconstructions at x_{i+1/2} (Shu 1998, sec. 2.2)."""
    return tuple(tuple(float(c) for c in _fv_face_coeffs_exact(r, k)) for k in range(r))


def _fv_linear_weights(r):
    """Optimal linear weights of the (2r-1)-point scheme (exact, Fractions)."""
    big = _fv_face_coeffs_exact(2 * r - 1, r - 1)
    small = [_fv_face_coeffs_exact(r, k) for k in range(r)]
    d = []
    for p in range(r):
        acc = sum(d[k] * small[k][p - k] for k in range(p))
        d.append((big[p] - acc) / small[p][0])
    return tuple(float(x) for x in d)


def _fv_beta_matrix(r, k):
    """Jiang-Shu smoothness quadratic form of candidate k (r cells).

    beta = sum_{l=1}^{r-1} int_{-1/2}^{1/2} (d^l p / dx^l)^2 dx (unit
    spacing), p the candidate's polynomial; returned as the symmetric matrix
    B with beta = v^T B v.
    """
    from fractions import Fraction
    Ainv = _fv_inverse(r, k)
    n = r
    B = [[Fraction(0)] * n for _ in range(n)]
    for l in range(1, r):
        for a in range(l, r):
            fa = Fraction(math.factorial(a), math.factorial(a - l))
            for b in range(l, r):
                fb = Fraction(math.factorial(b), math.factorial(b - l))
                e = (a - l) + (b - l)
                integ = (Fraction(1, 2) ** (e + 1) - Fraction(-1, 2) ** (e + 1)) / (e + 1)
                w = fa * fb * integ
                for i in range(n):
                    for j in range(n):
                        B[i][j] += w * Ainv[a][i] * Ainv[b][j]
    return np.array([[float(x) for x in row] for row in B])


WENO7_COEFFS = _fv_candidate_coeffs(4)
WENO7_WEIGHTS = _fv_linear_weights(4)
WENO7_BETA = tuple(_fv_beta_matrix(4, k) for k in range(4))
WENO9_COEFFS = _fv_candidate_coeffs(5)
WENO9_WEIGHTS = _fv_linear_weights(5)
WENO9_BETA = tuple(_fv_beta_matrix(5, k) for k in range(5))
WENO7_COEFFS_R = tuple(tuple(reversed(c)) for c in reversed(WENO7_COEFFS))
WENO7_WEIGHTS_R = tuple(reversed(WENO7_WEIGHTS))
WENO7_BETA_R = tuple(m[::-1, ::-1] for m in reversed(WENO7_BETA))
WENO9_COEFFS_R = tuple(tuple(reversed(c)) for c in reversed(WENO9_COEFFS))
WENO9_WEIGHTS_R = tuple(reversed(WENO9_WEIGHTS))
WENO9_BETA_R = tuple(m[::-1, ::-1] for m in reversed(WENO9_BETA))


def _weno_generic(stencils, coeffs, betas, weights, eps=1e-8):
    """_weno_reconstruct (advection/weno.py:268-294)."""
    cands = []
    for cs, st in zip(coeffs, stencils):
        acc = 0
        for c, v in zip(cs, st):
            acc = acc + c * v
        cands.append(acc)
    bs = []
    for B, st in zip(betas, stencils):
        vals = np.stack([np.asarray(s, dtype=float) for s in st], 0)
        bs.append(np.einsum("i...,ij,j...->...", vals, B, vals))
    alphas = [w / (b + eps) ** 2 for w, b in zip(weights, bs)]
    asum = 0
    for a in alphas:
        asum = asum + a
    num = 0
    for a, c in zip(alphas, cands):
        num = num + a * c
    return num / asum


def weno7(qmmm, qmm, qm, q0, qp, qpp, qppp):
    """weno_7pts (advection/weno.py:538-563)."""
    st = ((qmmm, qmm, qm, q0), (qmm, qm, q0, qp), (qm, q0, qp, qpp), (q0, qp, qpp, qppp))
    return _weno_generic(st, WENO7_COEFFS, WENO7_BETA, WENO7_WEIGHTS)


def weno7_right(qmm, qm, q0, qp, qpp, qppp, qpppp):
    """weno_7pts_right (advection/weno.py:597-628)."""
    st = ((qmm, qm, q0, qp), (qm, q0, qp, qpp), (q0, qp, qpp, qppp), (qp, qpp, qppp, qpppp))
    return _weno_generic(st, WENO7_COEFFS_R, WENO7_BETA_R, WENO7_WEIGHTS_R)


def weno9(a, b, c, d, e, f, g, h, i):
    """weno_9pts (advection/weno.py:566-594)."""
    st = ((a, b, c, d, e), (b, c, d, e, f), (c, d, e, f, g), (d, e, f, g, h), (e, f, g, h, i))
    return _weno_generic(st, WENO9_COEFFS, WENO9_BETA, WENO9_WEIGHTS)


def weno9_right(a, b, c, d, e, f, g, h, i):
    """weno_9pts_right (advection/weno.py:631-665)."""
    st = ((a, b, c, d, e), (b, c, d, e, f), (c, d, e, f, g), (d, e, f, g, h), (e, f, g, h, i))
    return _weno_generic(st, WENO9_COEFFS_R, WENO9_BETA_R, WENO9_WEIGHTS_R)


# ---------------------------------------------------------------------------
# Limiters  (advection/limiters.py:34-123)
# ---------------------------------------------------------------------------


def minmod(r):
    return np.maximum(0.0, np.minimum(1.0, r))


def van_leer(r):
    ra = np.abs(r)
    return (r + ra) / (1.0 + ra)


def superbee(r):
    return np.maximum(0.0, np.maximum(np.minimum(2.0 * r, 1.0), np.minimum(r, 2.0)))


def mc(r):
    return np.maximum(0.0, np.minimum(np.minimum((1.0 + r) / 2.0, 2.0 * r), 2.0))


LIMITERS = {"minmod": minmod, "van_leer": van_leer, "superbee": superbee, "mc": mc}
TVD_EPS = 1e-8  # advection/reconstruction.py:43

# ---------------------------------------------------------------------------
# Face reconstructions along the last axis (advection/reconstruction.py)
#
# ``_face_values(h, scheme)`` takes rows ``h`` of length N (the full padded
# line) and returns (h_pos, h_neg), each of length N-2: the face values at
# faces i = 1..N-2 (face i sits between cells i and i+1) for positive and
# negative flow, including the reference's boundary fallback ladders.
# ---------------------------------------------------------------------------


def _face_values(h, scheme):
    N = h.shape[-1]
    H = lambda a, b=None: h[..., a:b]  # noqa: E731
    if scheme == "naive":
        v = 0.5 * (H(1, -1) + H(2))
        return v, v
    if scheme == "upwind1":
        return H(1, -1), H(2)
    if scheme == "upwind2":  # reconstruction.py:632-656
        pos = 1.5 * H(1, -1) - 0.5 * H(0, -2)
        neg = np.concatenate([1.5 * H(2, -1) - 0.5 * H(3), H(N - 1)], -1)
        return pos, neg
    if scheme == "upwind3":  # reconstruction.py:684-715
        pos = -1.0 / 6.0 * H(0, -2) + 5.0 / 6.0 * H(1, -1) + 1.0 / 3.0 * H(2)
        neg = np.concatenate(
            [1.0 / 3.0 * H(1, -2) + 5.0 / 6.0 * H(2, -1) - 1.0 / 6.0 * H(3), H(N - 1)], -1)
        return pos, neg
    if scheme in ("weno3", "wenoz3"):  # reconstruction.py:749-832
        f, fr = (weno3, weno3_right) if scheme == "weno3" else (wenoz3, wenoz3_right)
        pos = f(H(0, -2), H(1, -1), H(2))
        neg = np.concatenate([fr(H(1, -2), H(2, -1), H(3)), H(N - 1)], -1)
        return pos, neg
    if scheme in ("weno5", "wenoz5"):  # reconstruction.py:834-864, 896-926
        f5, f5r, f3, f3r = ((weno5, weno5_right, weno3, weno3_right) if scheme == "weno5"
                            else (wenoz5, wenoz5_right, wenoz3, wenoz3_right))
        p5 = f5(H(0, -4), H(1, -3), H(2, -2), H(3, -1), H(4))
        p3f = f3(H(0, 1), H(1, 2), H(2, 3))
        p3l = f3(H(N - 3, N - 2), H(N - 2, N - 1), H(N - 1))
        pos = np.concatenate([p3f, p5, p3l], -1)
        n5 = f5r(H(0, -4), H(1, -3), H(2, -2), H(3, -1), H(4))
        n3 = f3r(H(N - 3, N - 2), H(N - 2, N - 1), H(N - 1))
        neg = np.concatenate([n5, n3, H(N - 1)], -1)
        return pos, neg
    if scheme == "weno7":  # reconstruction.py:74-118
        pos = np.concatenate([
            weno3(H(0, 1), H(1, 2), H(2, 3)),
            weno5(H(0, 1), H(1, 2), H(2, 3), H(3, 4), H(4, 5)),
            weno7(H(0, -6), H(1, -5), H(2, -4), H(3, -3), H(4, -2), H(5, -1), H(6)),
            weno5(H(N - 5, N - 4), H(N - 4, N - 3), H(N - 3, N - 2), H(N - 2, N - 1), H(N - 1)),
            weno3(H(N - 3, N - 2), H(N - 2, N - 1), H(N - 1)),
        ], -1)
        neg = np.concatenate([
            weno5_right(H(0, 1), H(1, 2), H(2, 3), H(3, 4), H(4, 5)),
            weno7_right(H(0, -6), H(1, -5), H(2, -4), H(3, -3), H(4, -2), H(5, -1), H(6)),
            weno5_right(H(N - 5, N - 4), H(N - 4, N - 3), H(N - 3, N - 2), H(N - 2, N - 1), H(N - 1)),
            weno3_right(H(N - 3, N - 2), H(N - 2, N - 1), H(N - 1)),
            H(N - 1),
        ], -1)
        return pos, neg
    if scheme == "weno9":  # reconstruction.py:121-236
        def sl(k):
            return [H(j, j + 1) for j in range(k)]
        def tl(k):
            return [H(N - k + j, N - k + j + 1) for j in range(k)]
        mid = [H(j, (j - 8) if j < 8 else None) for j in range(9)]
        pos = np.concatenate([
            weno3(*sl(3)), weno5(*sl(5)), weno7(*sl(7)), weno9(*mid),
            weno7(*tl(7)), weno5(*tl(5)), weno3(*tl(3)),
        ], -1)
        neg = np.concatenate([
            weno5_right(*sl(5)), weno7_right(*sl(7)), weno9_right(*mid),
            weno7_right(*tl(7)), weno5_right(*tl(5)), weno3_right(*tl(3)), H(N - 1),
        ], -1)
        return pos, neg
    if scheme in LIMITERS:  # tvd_x, reconstruction.py:1003-1040
        phi = LIMITERS[scheme]
        dfwd = H(2) - H(1, -1)
        dbwd = H(1, -1) - H(0, -2)
        r = dbwd / (dfwd + TVD_EPS)
        pos = H(1, -1) + 0.5 * phi(r) * dfwd
        dn = H(1, -2) - H(2, -1)
        dn2 = H(2, -1) - H(3)
        rn = dn2 / (dn + TVD_EPS)
        neg = np.concatenate([H(2, -1) + 0.5 * phi(rn) * dn, H(N - 1)], -1)
        return pos, neg
    raise ValueError(f"Unknown method: {scheme!r}")


ADVECTION_METHODS = ("naive", "upwind1", "upwind2", "upwind3", "weno3", "weno5",
                     "wenoz5", "weno7", "weno9", "minmod", "van_leer", "superbee", "mc")
MASK_DISPATCHABLE = ("weno3", "weno5", "wenoz5", "minmod", "van_leer", "superbee", "mc")


def _interior(values, like, ghost=1):
    """operators/_ghost.py:9-28."""
    out = np.zeros(like.shape, dtype=np.result_type(like, values))
    sl = tuple(slice(ghost, -ghost) for _ in range(like.ndim))
    out[sl] = values
    return out


def face_flux_x(h, u, scheme):
    """Reconstruction2D.<scheme>_x (advection/reconstruction.py:582-1040).

    East-face flux fe[j, i] (face i+1/2), zero ghost ring.
    """
    pos, neg = _face_values(h[1:-1, :], scheme)
    uu = u[1:-1, 1:-1]
    return _interior(np.where(uu >= 0.0, pos, neg) * uu, h)


def face_flux_y(h, v, scheme):
    """Reconstruction2D.<scheme>_y (mirror of the x form along axis 0)."""
    return face_flux_x(h.T, v.T, scheme).T


_RECON_TIERS = {  # advection/advection.py:91-136
    "weno5": {2: "upwind1", 4: "weno3", 6: "weno5"},
    "wenoz5": {2: "upwind1", 4: "wenoz3", 6: "wenoz5"},
    "weno3": {2: "upwind1", 4: "weno3"},
}


def tiers_for_method(method):
    if method in _RECON_TIERS:
        return _RECON_TIERS[method]
    if method in LIMITERS:
        return {2: "upwind1", 4: method}
    raise ValueError(f"Method {method!r} does not support mask-based stencil dispatch")


def upwind_flux_x(h, u, tier_masks, rec):
    """upwind_flux with dim=1 (advection/flux.py:100-253).

    ``tier_masks``: {size: bool mask}, ``rec``: {size: scheme name}.
    """
    pos = u[1:-1, 1:-1] >= 0.0
    acc = np.zeros_like(h[1:-1, 1:-1])
    for s in sorted(rec):
        f = face_flux_x(h, u, rec[s])
        m = tier_masks[s]
        fm = np.where(pos, m[1:-1, 1:-1], m[1:-1, 2:])
        acc = acc + np.where(fm, f[1:-1, 1:-1], 0.0)
    out = np.zeros_like(h)
    out[1:-1, 1:-1] = acc
    return out


def advection2d(h, u, v, dx, dy, method="upwind1", mask=None):
    """Advection2D.__call__ (advection/advection.py:329-420).

    ``mask``: dict from :func:`mask2d_from_mask` or None.
    """
    if mask is not None and method in MASK_DISPATCHABLE:
        rec = tiers_for_method(method)
        sizes = tuple(sorted(rec))
        hx = adaptive_masks(mask["x_pos"], mask["x_neg"], (2, 4, 6))
        hy = adaptive_masks(mask["y_pos"], mask["y_neg"], (2, 4, 6))
        mx = narrow_mask_hierarchy(hx, sizes)
        my = narrow_mask_hierarchy(hy, sizes)
        fe = upwind_flux_x(h, u, mx, rec)
        fn = upwind_flux_x(h.T, v.T, {s: m.T for s, m in my.items()}, rec).T
    else:
        if method not in ADVECTION_METHODS:
            raise ValueError(f"Unknown method: {method!r}")
        fe = face_flux_x(h, u, method)
        fn = face_flux_y(h, v, method)
    out = _interior(
        -((fe[2:-2, 2:-2] - fe[2:-2, 1:-3]) / dx + (fn[2:-2, 2:-2] - fn[1:-3, 2:-2]) / dy),
        h, ghost=2)
    if mask is not None:
        out = out * mask["h"]
    return out


# ---------------------------------------------------------------------------
# Difference / interpolation  (operators/stencils.py, difference.py,
# interpolation.py)
# ---------------------------------------------------------------------------


def _fwd_x(h):
    return h[1:-1, 2:] - h[1:-1, 1:-1]


def _fwd_y(h):
    return h[2:, 1:-1] - h[1:-1, 1:-1]


def _bwd_x(h):
    return h[1:-1, 1:-1] - h[1:-1, :-2]


def _bwd_y(h):
    return h[1:-1, 1:-1] - h[:-2, 1:-1]


def _mask_out(out, m):
    return out if m is None else out * m


def diff2d(name, a, dx, dy, mask=None, b=None):
    """Difference2D (operators/difference.py:165-520).  Returns array(s)."""
    M = (lambda k: None) if mask is None else (lambda k: mask[k])  # noqa: E731
    if name == "diff_x_T_to_U":
        return _mask_out(_interior(_fwd_x(a) / dx, a), M("u"))
    if name == "diff_y_T_to_V":
        return _mask_out(_interior(_fwd_y(a) / dy, a), M("v"))
    if name == "diff_y_U_to_X":
        return _mask_out(_interior(_fwd_y(a) / dy, a), M("xy_corner_strict"))
    if name == "diff_x_V_to_X":
        return _mask_out(_interior(_fwd_x(a) / dx, a), M("xy_corner_strict"))
    if name == "diff_y_X_to_U":
        return _mask_out(_interior(_bwd_y(a) / dy, a), M("u"))
    if name == "diff_x_X_to_V":
        return _mask_out(_interior(_bwd_x(a) / dx, a), M("v"))
    if name == "diff_x_U_to_T":
        return _mask_out(_interior(_bwd_x(a) / dx, a), M("h"))
    if name == "diff_y_V_to_T":
        return _mask_out(_interior(_bwd_y(a) / dy, a), M("h"))
    if name == "laplacian":
        d2x = (_fwd_x(a) - _bwd_x(a)) / dx ** 2
        d2y = (_fwd_y(a) - _bwd_y(a)) / dy ** 2
        return _mask_out(_interior(d2x + d2y, a), M("h"))
    if name == "divergence":
        like = np.zeros(a.shape, dtype=np.result_type(a, b))
        return _mask_out(_interior(_bwd_x(a) / dx + _bwd_y(b) / dy, like), M("h"))
    if name == "curl":
        return _mask_out(_interior(_fwd_x(b) / dx - _fwd_y(a) / dy, a), M("xy_corner_strict"))
    if name == "grad_perp":
        psi = a
        u = _interior(-(psi[2:, 1:-1] + psi[2:, 2:] - psi[:-2, 1:-1] - psi[:-2, 2:]) / (4.0 * dy), psi)
        v = _interior((psi[1:-1, 2:] + psi[2:, 2:] - psi[1:-1, :-2] - psi[2:, :-2]) / (4.0 * dx), psi)
        return _mask_out(u, M("u")), _mask_out(v, M("v"))
    raise ValueError(name)


def interp2d(name, a, mask=None):
    """Interpolation2D (operators/interpolation.py:104-275)."""
    M = (lambda k: None) if mask is None else (lambda k: mask[k])  # noqa: E731
    c, e, w, n, s = a[1:-1, 1:-1], a[1:-1, 2:], a[1:-1, :-2], a[2:, 1:-1], a[:-2, 1:-1]
    table = {
        "T_to_U": (0.5 * (c + e), "u"),
        "T_to_V": (0.5 * (c + n), "v"),
        "T_to_X": (0.25 * (c + e + n + a[2:, 2:]), "xy_corner_strict"),
        "X_to_U": (0.5 * (c + s), "u"),
        "X_to_V": (0.5 * (c + w), "v"),
        "U_to_T": (0.5 * (c + w), "h"),
        "V_to_T": (0.5 * (c + s), "h"),
        "X_to_T": (0.25 * (c + s + w + a[:-2, :-2]), "h"),
        "U_to_X": (0.5 * (c + n), "xy_corner_strict"),
        "V_to_X": (0.5 * (c + e), "xy_corner_strict"),
        "U_to_V": (0.25 * (c + n + w + a[2:, :-2]), "v"),
        "V_to_U": (0.25 * (c + s + e + a[:-2, 2:]), "u"),
    }
    vals, mk = table[name]
    return _mask_out(_interior(vals, a), M(mk))


def arakawa_jacobian(f, g, dx, dy):
    """Arakawa (1966) J(f, g) (operators/jacobian.py:106-131)."""
    Jpp = (f[..., 1:-1, 2:] - f[..., 1:-1, :-2]) * (g[..., 2:, 1:-1] - g[..., :-2, 1:-1]) - (
        f[..., 2:, 1:-1] - f[..., :-2, 1:-1]) * (g[..., 1:-1, 2:] - g[..., 1:-1, :-2])
    Jpx = (f[..., 1:-1, 2:] * (g[..., 2:, 2:] - g[..., :-2, 2:])
           - f[..., 1:-1, :-2] * (g[..., 2:, :-2] - g[..., :-2, :-2])
           - f[..., 2:, 1:-1] * (g[..., 2:, 2:] - g[..., 2:, :-2])
           + f[..., :-2, 1:-1] * (g[..., :-2, 2:] - g[..., :-2, :-2]))
    Jxp = (g[..., 2:, 1:-1] * (f[..., 2:, 2:] - f[..., 2:, :-2])
           - g[..., :-2, 1:-1] * (f[..., :-2, 2:] - f[..., :-2, :-2])
           - g[..., 1:-1, 2:] * (f[..., 2:, 2:] - f[..., :-2, 2:])
           + g[..., 1:-1, :-2] * (f[..., 2:, :-2] - f[..., :-2, :-2]))
    return (Jpp + Jpx + Jxp) / (12.0 * dx * dy)


# ---------------------------------------------------------------------------
# Diffusion  (diffusion/diffusion.py:120-176, 462-574)
# ---------------------------------------------------------------------------


def diffusion_fluxes(h, kappa, dx, dy, mu=None, mv=None):
    """_diffusion_2d_fluxes_impl (diffusion/diffusion.py:179-205)."""
    k = np.asarray(kappa, dtype=float)
    if k.ndim >= 2:
        kx, ky = k[1:-1, 1:-2], k[1:-2, 1:-1]
    else:
        kx = ky = k
    fx = np.zeros_like(h)
    fx[1:-1, 1:-2] = kx * (h[1:-1, 2:-1] - h[1:-1, 1:-2]) / dx
    if mu is not None:
        fx = fx * mu
    fy = np.zeros_like(h)
    fy[1:-2, 1:-1] = ky * (h[2:-1, 1:-1] - h[1:-2, 1:-1]) / dy
    if mv is not None:
        fy = fy * mv
    return fx, fy


def diffusion2d(h, kappa, dx, dy, mask=None):
    """Diffusion2D.__call__ / _diffusion_2d_impl (diffusion/diffusion.py:120-176)."""
    mu = None if mask is None else mask["u"]
    mv = None if mask is None else mask["v"]
    fx, fy = diffusion_fluxes(h, kappa, dx, dy, mu, mv)
    du = (fx[1:-1, 1:-1] - fx[1:-1, :-2]) / dx
    dv = (fy[1:-1, 1:-1] - fy[:-2, 1:-1]) / dy
    out = _interior(du + dv, h)
    if mask is not None:
        out = out * mask["h"]
    return out


def biharmonic2d(h, kappa, dx, dy, mask=None):
    """BiharmonicDiffusion2D.__call__ (diffusion/diffusion.py:549-574)."""
    lap1 = diffusion2d(h, 1.0, dx, dy)
    lap2 = diffusion2d(lap1, 1.0, dx, dy)
    out = -kappa * lap2
    if mask is not None:
        out = out * mask["h"]
    return out


# ---------------------------------------------------------------------------
# Boundary conditions  (boundary/boundary.py:17-75, bc_set.py:35-66,
# bc_1d.py:125-142)
# ---------------------------------------------------------------------------


def enforce_periodic(f):
    out = np.array(f, copy=True)
    out[0, :] = out[-2, :]
    out[-1, :] = out[1, :]
    out[:, 0] = out[:, -2]
    out[:, -1] = out[:, 1]
    return out


def pad_interior_constant(f):
    out = np.zeros_like(f)
    out[1:-1, 1:-1] = f[1:-1, 1:-1]
    return out


# ---------------------------------------------------------------------------
# Time stepping  (timestepping/explicit_rk.py:43-121)
# ---------------------------------------------------------------------------


def euler_step(y, f, dt):
    return y + dt * f(y)


def heun_step(y, f, dt):
    k1 = f(y)
    k2 = f(y + dt * k1)
    return y + 0.5 * dt * (k1 + k2)


def rk3_ssp_step(y, f, dt):
    k1 = f(y)
    y1 = y + dt * k1
    k2 = f(y1)
    y2 = 0.75 * y + 0.25 * y1 + 0.25 * dt * k2
    k3 = f(y2)
    return (1.0 / 3.0) * y + (2.0 / 3.0) * y2 + (2.0 / 3.0) * dt * k3


# ---------------------------------------------------------------------------
# Spectral Dirichlet Helmholtz (spectraldiffx v0.0.10 solve_helmholtz_dst,
# re-exported at solvers/spectral.py:14-98; math docs/elliptic_solvers.md:55-76)
# ---------------------------------------------------------------------------


def dst1_eigenvalues(n, d):
    k = np.arange(n)
    return -4.0 / d ** 2 * np.sin(np.pi * (k + 1) / (2 * (n + 1))) ** 2


def solve_helmholtz_dst(rhs, dx, dy, lambda_=0.0):
    """(nabla^2 - lambda) psi = rhs, psi = 0 outside, via DST-I."""
    from scipy.fft import dstn, idstn
    rhs = np.asarray(rhs, dtype=float)
    ny, nx = rhs.shape[-2:]
    fh = dstn(rhs, type=1, axes=(-2, -1))
    lam = np.asarray(lambda_, dtype=float)
    den = dst1_eigenvalues(ny, dy)[:, None] + dst1_eigenvalues(nx, dx)[None, :]
    den = den - (lam[..., None, None] if lam.ndim else lam)
    return idstn(fh / den, type=1, axes=(-2, -1))


def dirichlet_helmholtz_apply(psi, dx, dy, lambda_=0.0):
    """5-point (nabla^2 - lambda) on an interior-only array, zero outside."""
    p = np.pad(psi, ((0, 0),) * (psi.ndim - 2) + ((1, 1), (1, 1)))
    c = p[..., 1:-1, 1:-1]
    lap = (p[..., 1:-1, 2:] - 2 * c + p[..., 1:-1, :-2]) / dx ** 2 + (
        p[..., 2:, 1:-1] - 2 * c + p[..., :-2, 1:-1]) / dy ** 2
    lam = np.asarray(lambda_, dtype=float)
    return lap - (lam[..., None, None] if lam.ndim else lam) * c


def dct2_eigenvalues(n, d):
    """-4/d^2 sin^2(pi k / (2n)): the Neumann (cell-centred) 3-point second
    difference's eigenvalues (docs/elliptic_solvers.md eigenvalue table)."""
    k = np.arange(n)
    return -4.0 / d ** 2 * np.sin(np.pi * k / (2 * n)) ** 2


def fft_eigenvalues(n, d):
    """-4/d^2 sin^2(pi k / n): the periodic 3-point second difference."""
    k = np.arange(n)
    return -4.0 / d ** 2 * np.sin(np.pi * k / n) ** 2


def _spectral_den(ny, nx, dx, dy, lambda_, ey, ex):
    den = ey(ny, dy)[:, None] + ex(nx, dx)[None, :]
    lam = np.asarray(lambda_, dtype=float)
    return den - (lam[..., None, None] if lam.ndim else lam)


def _safe_div(a, den):
    # the null mode (den == 0: Neumann / periodic Poisson) -> 0, the zero-mean gauge
    return np.where(den == 0.0, 0.0, a / np.where(den == 0.0, 1.0, den))


def solve_helmholtz_dct(rhs, dx, dy, lambda_=0.0):
    """(nabla^2 - lambda) psi = rhs with homogeneous Neumann walls by DCT-II
    (spectraldiffx solve_helmholtz_dct, re-exported at solvers/spectral.py:14-98;
    published algorithm: forward DCT-II, divide by the eigenvalue grid,
    inverse; null mode set to zero)."""
    from scipy.fft import dctn, idctn
    rhs = np.asarray(rhs, dtype=float)
    ny, nx = rhs.shape[-2:]
    den = _spectral_den(ny, nx, dx, dy, lambda_, dct2_eigenvalues, dct2_eigenvalues)
    return idctn(_safe_div(dctn(rhs, type=2, axes=(-2, -1)), den), type=2, axes=(-2, -1))


def solve_helmholtz_fft(rhs, dx, dy, lambda_=0.0):
    """(nabla^2 - lambda) psi = rhs, doubly periodic, by FFT (spectraldiffx
    solve_helmholtz_fft; null mode set to zero)."""
    rhs = np.asarray(rhs, dtype=float)
    ny, nx = rhs.shape[-2:]
    den = _spectral_den(ny, nx, dx, dy, lambda_, fft_eigenvalues, fft_eigenvalues)
    return np.real(np.fft.ifft2(_safe_div(np.fft.fft2(rhs, axes=(-2, -1)), den), axes=(-2, -1)))


def neumann_helmholtz_apply(psi, dx, dy, lambda_=0.0):
    """5-point (nabla^2 - lambda) with mirror ghosts (zero normal gradient)."""
    p = np.pad(psi, ((0, 0),) * (psi.ndim - 2) + ((1, 1), (1, 1)), mode="edge")
    c = p[..., 1:-1, 1:-1]
    lap = (p[..., 1:-1, 2:] - 2 * c + p[..., 1:-1, :-2]) / dx ** 2 + (
        p[..., 2:, 1:-1] - 2 * c + p[..., :-2, 1:-1]) / dy ** 2
    return lap - float(lambda_) * c


def periodic_helmholtz_apply(psi, dx, dy, lambda_=0.0):
    """5-point (nabla^2 - lambda) with periodic wrap."""
    lap = (np.roll(psi, -1, -1) - 2 * psi + np.roll(psi, 1, -1)) / dx ** 2 + (
        np.roll(psi, -1, -2) - 2 * psi + np.roll(psi, 1, -2)) / dy ** 2
    return lap - float(lambda_) * psi


def spectral_solve(rhs, dx, dy, lambda_, bc):
    """_spectral_solve (solvers/spectral.py:105-128)."""
    f = {"fft": solve_helmholtz_fft, "dst": solve_helmholtz_dst, "dct": solve_helmholtz_dct}.get(bc)
    if f is None:
        raise ValueError(f"base_bc must be 'fft', 'dst', or 'dct'; got {bc!r}")
    return f(rhs, dx, dy, lambda_)


def inner_boundary_indices(mask):
    """Interior (True) cells 4-connected to an exterior (False) cell; cells
    beyond the array edge count as interior (the reference test helper's
    binary_dilation of ~mask with the cross structure, tests/test_elliptic.py:492-503)."""
    m = np.asarray(mask, dtype=bool)
    land = ~m
    d = land.copy()
    d[1:, :] |= land[:-1, :]
    d[:-1, :] |= land[1:, :]
    d[:, 1:] |= land[:, :-1]
    d[:, :-1] |= land[:, 1:]
    return np.where(m & d)


def capacitance_solve(rhs, mask, dx, dy, lambda_=0.0, base_bc="fft"):
    """Capacitance-matrix masked solve (elliptic.py:146-183 builds it;
    Buzbee-Golub-Nielson as docs/elliptic_solvers.md states): Green's
    functions g_l = L^-1 e_{b_l} of the rectangular solver, C = G[B, :],
    alpha = C^-1 u[B] with u = L^-1 rhs, psi = u - G alpha (zero on B)."""
    jb, ib = inner_boundary_indices(mask)
    nb = len(jb)
    if nb == 0:
        raise ValueError("No inner-boundary points found in mask")
    ny, nx = np.asarray(mask).shape
    E = np.zeros((nb, ny, nx))
    E[np.arange(nb), jb, ib] = 1.0
    G = spectral_solve(E, dx, dy, lambda_, base_bc)
    C = G[:, jb, ib].T                       # C[k, l] = g_l(b_k)
    u = spectral_solve(np.asarray(rhs, float), dx, dy, lambda_, base_bc)
    alpha = np.linalg.solve(C, u[jb, ib])
    return u - np.tensordot(alpha, G, axes=(0, 0))


def dst1_matrix(n):
    """S[j, k] = sin(pi (j+1)(k+1) / (n+1)); dst type 1 = 2 S."""
    j = np.arange(n)
    return np.sin(np.pi * np.outer(j + 1, j + 1) / (n + 1))


# ---------------------------------------------------------------------------
# Masked operators and CG (solvers/iterative.py)
# ---------------------------------------------------------------------------


def masked_laplacian(psi, mask, dx, dy, lambda_=0.0):
    """masked_laplacian (solvers/iterative.py:144-191), periodic roll."""
    pm = psi * mask
    lap = (np.roll(pm, 1, 1) + np.roll(pm, -1, 1) - 2.0 * pm) / dx ** 2 + (
        np.roll(pm, 1, 0) + np.roll(pm, -1, 0) - 2.0 * pm) / dy ** 2
    return (lap - lambda_ * pm) * mask


def pcg(matvec, rhs, x0=None, precond=None, rtol=1e-6, atol=1e-6, max_steps=500,
        stabilise_every=10):
    """Preconditioned CG for a negative-definite operator.

    Restates the iteration that solve_cg delegates to lineax.CG
    (solvers/iterative.py:105-136): the system is negated to (-A) x = -b with
    preconditioner -M; stop when max|r| < atol + rtol * max|b|; the residual
    is recomputed from scratch every ``stabilise_every`` steps.  Iterate-level
    parity with lineax is unpinned.
    """
    b = -np.asarray(rhs, float)
    A = lambda x: -matvec(x)  # noqa: E731
    P = (lambda r: r) if precond is None else (lambda r: -precond(r))  # noqa: E731
    x = np.zeros_like(b) if x0 is None else np.array(x0, float)
    r = b - A(x)
    z = P(r)
    p = z.copy()
    gamma = float(np.vdot(r, z))
    tol = atol + rtol * np.max(np.abs(b))
    k = 0
    conv = np.max(np.abs(r)) < tol
    while not conv and k < max_steps and gamma > 0:
        Ap = A(p)
        alpha = gamma / float(np.vdot(p, Ap))
        x = x + alpha * p
        k += 1
        if k % stabilise_every == 0:
            r = b - A(x)
        else:
            r = r - alpha * Ap
        z = P(r)
        g_new = float(np.vdot(r, z))
        p = z + (g_new / gamma) * p
        gamma = g_new
        conv = np.max(np.abs(r)) < tol
    res = np.linalg.norm(matvec(x) - rhs)
    return x, dict(iterations=k, residual_norm=res, converged=bool(conv))


# ---------------------------------------------------------------------------
# Geometric multigrid  (solvers/multigrid.py)
# ---------------------------------------------------------------------------


def mg_compute_n_levels(ny, nx, min_coarse=8):
    """multigrid.py:50-76."""
    n = 1
    while ny % 2 == 0 and nx % 2 == 0 and ny // 2 >= min_coarse and nx // 2 >= min_coarse:
        ny //= 2
        nx //= 2
        n += 1
    return n


def mg_restrict_mask(m, thr=0.5):
    """multigrid.py:79-104."""
    avg = (m[::2, ::2] + m[1::2, ::2] + m[::2, 1::2] + m[1::2, 1::2]) / 4.0
    return (avg >= thr).astype(np.float64)


def mg_face_coeffs(coeff, mask):
    """_compute_face_masks + _interpolate_coeff_to_faces (multigrid.py:107-179)."""
    mcx = np.zeros_like(mask)
    mcx[:, :-1] = mask[:, :-1] * mask[:, 1:]
    mcy = np.zeros_like(mask)
    mcy[:-1, :] = mask[:-1, :] * mask[1:, :]
    cx = np.zeros_like(coeff)
    cx[:, :-1] = 0.5 * (coeff[:, :-1] + coeff[:, 1:])
    cx *= mcx
    cy = np.zeros_like(coeff)
    cy[:-1, :] = 0.5 * (coeff[:-1, :] + coeff[1:, :])
    cy *= mcy
    return cx, cy


def mg_restrict_coeff(c, mf, mc_):
    """multigrid.py:182-218."""
    cm = c * mf
    s4 = cm[::2, ::2] + cm[1::2, ::2] + cm[::2, 1::2] + cm[1::2, 1::2]
    cnt = mf[::2, ::2] + mf[1::2, ::2] + mf[::2, 1::2] + mf[1::2, 1::2]
    return (s4 / np.maximum(cnt, 1.0)) * mc_


def mg_inv_diagonal(cx, cy, mask, dx, dy, lam):
    """multigrid.py:221-266."""
    cxw = np.zeros_like(cx)
    cxw[:, 1:] = cx[:, :-1]
    cys = np.zeros_like(cy)
    cys[1:, :] = cy[:-1, :]
    d = -(cx + cxw) / dx ** 2 - (cy + cys) / dy ** 2 - lam
    d *= mask
    safe = np.where(np.abs(d) > 1e-30, d, 1.0)
    inv = np.where(np.abs(d) > 1e-30, 1.0 / safe, 0.0)
    return inv * mask


def mg_build(mask, dx, dy, lambda_=0.0, coeff=None, n_levels=None, n_pre=6, n_post=6,
             n_coarse=50, omega=0.95, n_cycles=5):
    """build_multigrid_solver (multigrid.py:905-1062)."""
    m = np.asarray(mask, dtype=np.float64)
    ny, nx = m.shape
    if n_levels is None:
        n_levels = mg_compute_n_levels(ny, nx)
    fac = 2 ** (n_levels - 1)
    if ny % fac or nx % fac:
        raise ValueError(
            f"Grid shape ({ny}, {nx}) is not divisible by 2^(n_levels-1) = {fac}.  "
            "Choose a different n_levels or pad the grid.")
    c = np.ones_like(m) if coeff is None else np.asarray(coeff, np.float64)
    c = c * m
    levels = []
    cm, cc, cdx, cdy = m, c, float(dx), float(dy)
    for lev in range(n_levels):
        cx, cy = mg_face_coeffs(cc, cm)
        inv = mg_inv_diagonal(cx, cy, cm, cdx, cdy, lambda_)
        levels.append(dict(mask=cm, cx=cx, cy=cy, dx=cdx, dy=cdy, lam=float(lambda_), inv=inv))
        if lev < n_levels - 1:
            nm = mg_restrict_mask(cm)
            cc = mg_restrict_coeff(cc, cm, nm)
            cm = nm
            cdx *= 2.0
            cdy *= 2.0
    return dict(levels=levels, n_levels=n_levels, n_pre=n_pre, n_post=n_post,
                n_coarse=n_coarse, omega=omega, n_cycles=n_cycles)


def mg_apply(u, L):
    """_apply_operator (multigrid.py:327-405)."""
    um = u * L["mask"]
    cx, cy = L["cx"], L["cy"]
    e = np.zeros_like(um); e[:, :-1] = um[:, 1:]
    w = np.zeros_like(um); w[:, 1:] = um[:, :-1]
    n = np.zeros_like(um); n[:-1, :] = um[1:, :]
    s = np.zeros_like(um); s[1:, :] = um[:-1, :]
    cxw = np.zeros_like(cx); cxw[:, 1:] = cx[:, :-1]
    cys = np.zeros_like(cy); cys[1:, :] = cy[:-1, :]
    lap = (cx * (e - um) - cxw * (um - w)) / L["dx"] ** 2 + (cy * (n - um) - cys * (um - s)) / L["dy"] ** 2
    return (lap - L["lam"] * um) * L["mask"]


def mg_jacobi(u, f, L, omega, n):
    """_weighted_jacobi (multigrid.py:408-461)."""
    for _ in range(n):
        r = f - mg_apply(u, L)
        u = (u + omega * L["inv"] * r) * L["mask"]
    return u


def mg_restrict(v, mf, mc_):
    """_restrict (multigrid.py:464-507)."""
    vm = v * mf
    s4 = vm[::2, ::2] + vm[1::2, ::2] + vm[::2, 1::2] + vm[1::2, 1::2]
    cnt = mf[::2, ::2] + mf[1::2, ::2] + mf[::2, 1::2] + mf[1::2, 1::2]
    return (s4 / np.maximum(cnt, 1.0)) * mc_


def mg_prolong(vc, mc_, mf):
    """_prolongate (multigrid.py:510-598)."""
    nyc, nxc = vc.shape
    vm = vc * mc_
    vp = np.pad(vm, 1)
    mp = np.pad(mc_, 1)
    out = np.zeros((2 * nyc, 2 * nxc))
    for dj in (0, 1):
        for di in (0, 1):
            sj, si = 2 * dj - 1, 2 * di - 1
            vsi = vp[1:-1, 1 + si:nxc + 1 + si]
            msi = mp[1:-1, 1 + si:nxc + 1 + si]
            vsj = vp[1 + sj:nyc + 1 + sj, 1:-1]
            msj = mp[1 + sj:nyc + 1 + sj, 1:-1]
            vd = vp[1 + sj:nyc + 1 + sj, 1 + si:nxc + 1 + si]
            md = mp[1 + sj:nyc + 1 + sj, 1 + si:nxc + 1 + si]
            ws = 9 * vp[1:-1, 1:-1] + 3 * vsi + 3 * vsj + 1 * vd
            ds = 9 * mp[1:-1, 1:-1] + 3 * msi + 3 * msj + 1 * md
            out[dj::2, di::2] = ws / np.maximum(ds, 1.0)
    return out * mf


def mg_vcycle(mg, u, f, lev=0):
    """MultigridSolver.v_cycle (multigrid.py:808-881)."""
    L = mg["levels"][lev]
    if lev == mg["n_levels"] - 1:
        return mg_jacobi(u, f, L, mg["omega"], mg["n_coarse"])
    u = mg_jacobi(u, f, L, mg["omega"], mg["n_pre"])
    r = (f - mg_apply(u, L)) * L["mask"]
    C = mg["levels"][lev + 1]
    rc = mg_restrict(r, L["mask"], C["mask"])
    ec = mg_vcycle(mg, np.zeros_like(rc), rc, lev + 1)
    u = (u + mg_prolong(ec, C["mask"], L["mask"])) * L["mask"]
    return mg_jacobi(u, f, L, mg["omega"], mg["n_post"])


def mg_solve(mg, f):
    """MultigridSolver._run_vcycles (multigrid.py:885-897)."""
    u = np.zeros_like(f)
    for _ in range(mg["n_cycles"]):
        u = mg_vcycle(mg, u, f)
    return u


def mg_restrict_residual(mg, f, lvl, n_pre):
    """Downward leg of the learned preconditioner's hybrid cycle (no reference
    counterpart; built from mg_vcycle's pieces): per level, n_pre sweeps from
    zero, then restrict the residual.  Returns (per-level u, f) and f_lvl."""
    us, fs = [], [f]
    for lev in range(lvl):
        L = mg["levels"][lev]
        u = mg_jacobi(np.zeros_like(fs[-1]), fs[-1], L, mg["omega"], n_pre)
        r = (fs[-1] - mg_apply(u, L)) * L["mask"]
        C = mg["levels"][lev + 1]
        us.append(u)
        fs.append(mg_restrict(r, L["mask"], C["mask"]))
    return us, fs


def mg_hybrid(mg, f, lvl, n_pre, n_post, coarse=None):
    """Hybrid cycle: mg_vcycle's legs on levels 0..lvl-1 with the level-lvl
    correction e = coarse(f_lvl) (zero when coarse is None)."""
    us, fs = mg_restrict_residual(mg, f, lvl, n_pre)
    e = np.zeros_like(fs[lvl]) if coarse is None else coarse(fs[lvl])
    for lev in range(lvl - 1, -1, -1):
        L = mg["levels"][lev]
        C = mg["levels"][lev + 1]
        u = (us[lev] + mg_prolong(e, C["mask"], L["mask"])) * L["mask"]
        e = mg_jacobi(u, fs[lev], L, mg["omega"], n_post)
    return e


def mg_level_solve(mg, lvl, f, n_cycles):
    """u += V_lvl(f - A_lvl u) from u = 0, n_cycles times (the training targets)."""
    L = mg["levels"][lvl]
    u = np.zeros_like(f)
    for _ in range(n_cycles):
        r = (f - mg_apply(u, L)) * L["mask"]
        u = u + mg_vcycle(mg, np.zeros_like(r), r, lvl)
    return u


# ---------------------------------------------------------------------------
# Vertical modes  (vertical/vertical_modes.py:50-263)
# ---------------------------------------------------------------------------


def build_coupling_matrix(H, gp):
    H = np.asarray(H, float)
    g = np.asarray(gp, float)
    nl = H.shape[0]
    A = np.zeros((nl, nl))
    if nl == 1:
        A[0, 0] = 1.0 / (H[0] * g[0])
    else:
        A[0, 0] = 1.0 / (H[0] * g[0]) + 1.0 / (H[0] * g[1])
        A[0, 1] = -1.0 / (H[0] * g[1])
        for i in range(1, nl - 1):
            A[i, i - 1] = -1.0 / (H[i] * g[i])
            A[i, i] = (1.0 / H[i]) * (1.0 / g[i + 1] + 1.0 / g[i])
            A[i, i + 1] = -1.0 / (H[i] * g[i + 1])
        A[-1, -1] = 1.0 / (H[nl - 1] * g[nl - 1])
        A[-1, -2] = -1.0 / (H[nl - 1] * g[nl - 1])
    return A


def decompose_vertical_modes(A, f0):
    """decompose_vertical_modes (vertical_modes.py:124-190); jnp.linalg.eigh
    symmetrises its input by default, so the restatement uses (A + A^T)/2."""
    lam, R = np.linalg.eigh(0.5 * (A + A.T))
    pos = lam > 0
    safe = np.where(pos, lam, 1.0)
    rr = np.where(pos, 1.0 / (abs(f0) * np.sqrt(safe)), np.inf)
    return rr, R.T, R


# ---------------------------------------------------------------------------
# QG 1.5-layer tendency and step (scripts/qg_1p5_layer.py:115-145, 420-497)
# ---------------------------------------------------------------------------


def qg_velocity(psi, dx, dy):
    """geostrophic_velocity_from_streamfunction (qg_1p5_layer.py:115-145)."""
    px = interp2d("T_to_X", psi)
    return -diff2d("diff_y_X_to_U", px, dx, dy), diff2d("diff_x_X_to_V", px, dx, dy)


def qg_snapshot(q, dx, dy, lam, eta_scale):
    """record_snapshot (qg_1p5_layer.py:514-545) on a full [Ny, Nx] state:
    psi by the DST with a zero ghost ring, geostrophic u, v, relative
    vorticity (Vorticity2D.relative_vorticity, the curl at X points), then the
    seven interior planes q, psi, eta, U_to_T(u), V_to_T(v), speed,
    X_to_T(zeta) and 0.5 mean(q^2)."""
    psi = np.zeros_like(q)
    psi[1:-1, 1:-1] = solve_helmholtz_dst(q[1:-1, 1:-1], dx, dy, lam)
    u, v = qg_velocity(psi, dx, dy)
    zeta = diff2d("curl", u, dx, dy, None, v)
    uc, vc, zc = interp2d("U_to_T", u), interp2d("V_to_T", v), interp2d("X_to_T", zeta)
    i = (slice(1, -1), slice(1, -1))
    planes = np.stack([q[i], psi[i], eta_scale * psi[i], uc[i], vc[i], np.sqrt(uc[i] ** 2 + vc[i] ** 2), zc[i]])
    return planes, float(0.5 * np.mean(q[i] ** 2))


def qg_tendency(q, dx, dy, beta, lam, method="weno5", bc="periodic", forcing=None,
                drag=0.0, viscosity=0.0):
    """PV tendency (qg_1p5_layer.py:454-487), psi by DST with zero ghosts."""
    qb = enforce_periodic(q) if bc == "periodic" else pad_interior_constant(q)
    psi = np.zeros_like(qb)
    psi[1:-1, 1:-1] = solve_helmholtz_dst(qb[1:-1, 1:-1], dx, dy, lam)
    return qg_tendency_psi(qb, psi, dx, dy, beta, method, forcing, drag, viscosity)


def qg_tendency_psi(qb, psi, dx, dy, beta, method="weno5", forcing=None, drag=0.0, viscosity=0.0):
    """The same tendency for a given (BC-filled) q and streamfunction psi."""
    u, v = qg_velocity(psi, dx, dy)
    rhs = advection2d(qb, u, v, dx, dy, method)
    vc = interp2d("V_to_T", v)
    rhs[1:-1, 1:-1] += -beta * vc[1:-1, 1:-1]
    if forcing is not None:
        rhs = rhs + forcing
    if drag:
        rhs = rhs - drag * diff2d("laplacian", psi, dx, dy)
    if viscosity:
        rhs = rhs + viscosity * diff2d("laplacian", qb, dx, dy)
    return rhs


def mlqg_tendency(q, l2m, m2l, lams, dx, dy, beta, method="weno5"):
    """Multi-layer QG tendency, q [nl, Ny, Nx]: modes (layer_to_mode,
    vertical_modes.py:193-227), one DST Helmholtz per mode (pv_inversion,
    elliptic.py:390-542), back to layers (mode_to_layer, :230-263), then each
    layer's 1.5-layer tendency with its own psi (periodic q)."""
    nl = q.shape[0]
    qb = np.stack([enforce_periodic(q[k]) for k in range(nl)])
    qm = np.einsum("kl,lyx->kyx", l2m, qb[:, 1:-1, 1:-1])
    psim = np.stack([solve_helmholtz_dst(qm[k], dx, dy, lams[k]) for k in range(nl)])
    psil = np.einsum("kl,lyx->kyx", m2l, psim)
    out = np.zeros_like(qb)
    for k in range(nl):
        psi = np.zeros_like(qb[k])
        psi[1:-1, 1:-1] = psil[k]
        out[k] = qg_tendency_psi(qb[k], psi, dx, dy, beta, method)
    return out


def mlqg_step(q, l2m, m2l, lams, dx, dy, beta, dt, method="weno5"):
    """One rk3_ssp_step of the multi-layer tendency, ghost rings refilled."""
    f = lambda y: mlqg_tendency(y, l2m, m2l, lams, dx, dy, beta, method)  # noqa: E731
    out = rk3_ssp_step(q, f, dt)
    return np.stack([enforce_periodic(out[k]) for k in range(q.shape[0])])


def qg_step(q, dx, dy, beta, lam, dt, method="weno5", bc="periodic", **kw):
    """One rk3_ssp_step of the QG tendency followed by the BC refill."""
    f = lambda y: qg_tendency(y, dx, dy, beta, lam, method, bc, **kw)  # noqa: E731
    out = rk3_ssp_step(q, f, dt)
    return enforce_periodic(out) if bc == "periodic" else pad_interior_constant(out)


# ---------------------------------------------------------------------------
# Seeded synthetic inputs (the configurations' value distributions)
# ---------------------------------------------------------------------------


def kminus3_field(ny, nx, seed, std=1.0, slope=-3.0):
    """Seeded Gaussian random field with an isotropic k^slope power spectrum."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = np.inf
    amp = k ** (slope / 2.0)
    f = np.fft.irfft2(np.fft.rfft2(w) * amp, s=(ny, nx))
    f -= f.mean()
    return f * (std / f.std())


def fourier_streamfunction(ny, nx, dx, dy, seed, n_modes=8, umax=1.0):
    """Sum of seeded Fourier modes (wavenumbers 1..8), scaled to max|u|=umax."""
    rng = np.random.default_rng(seed)
    y = np.arange(ny)[:, None] / ny
    x = np.arange(nx)[None, :] / nx
    psi = np.zeros((ny, nx))
    for _ in range(n_modes):
        kx, ky = rng.integers(1, 9, size=2)
        a, ph = rng.standard_normal(), rng.uniform(0, 2 * np.pi)
        psi += a * np.sin(2 * np.pi * (kx * x + ky * y) + ph)
    full = np.zeros((ny + 2, nx + 2))
    full[1:-1, 1:-1] = psi
    full = enforce_periodic(full)
    u, v = diff2d("grad_perp", full, dx, dy)
    s = max(np.abs(u).max(), np.abs(v).max())
    return full * (umax / s)


# ---------------------------------------------------------------------------
# Diagnostics (operators/diagnostics.py)
# ---------------------------------------------------------------------------


def _ring0(x):
    out = np.zeros_like(x)
    out[1:-1, 1:-1] = x[1:-1, 1:-1]
    return out


def kinetic_energy(u, v):
    """diagnostics.py:35-73: 0.5 (avg_x_bwd(u^2) + avg_y_bwd(v^2)), zero ring."""
    u2, v2 = u ** 2, v ** 2
    ke = np.zeros_like(u)
    ke[1:-1, 1:-1] = 0.5 * (0.5 * (u2[1:-1, 1:-1] + u2[1:-1, :-2]) + 0.5 * (v2[1:-1, 1:-1] + v2[:-2, 1:-1]))
    return ke


def bernoulli_potential(h, u, v, gravity=9.81):
    """diagnostics.py:76-112."""
    return _ring0(kinetic_energy(u, v) + gravity * h)


def shear_strain(u, v, dx, dy):
    """diagnostics.py:184-213: diff_x_fwd(v)/dx + diff_y_fwd(u)/dy."""
    out = np.zeros_like(u)
    out[1:-1, 1:-1] = (v[1:-1, 2:] - v[1:-1, 1:-1]) / dx + (u[2:, 1:-1] - u[1:-1, 1:-1]) / dy
    return out


def tensor_strain(u, v, dx, dy):
    """diagnostics.py:216-245: diff_x_bwd(u)/dx - diff_y_bwd(v)/dy."""
    out = np.zeros_like(u)
    out[1:-1, 1:-1] = (u[1:-1, 1:-1] - u[1:-1, :-2]) / dx - (v[1:-1, 1:-1] - v[:-2, 1:-1]) / dy
    return out


def qg_potential_vorticity(psi, f0, beta, dx, dy, y, y0):
    """diagnostics.py:395-452."""
    d2x = ((psi[1:-1, 2:] - psi[1:-1, 1:-1]) - (psi[1:-1, 1:-1] - psi[1:-1, :-2])) / dx ** 2
    d2y = ((psi[2:, 1:-1] - psi[1:-1, 1:-1]) - (psi[1:-1, 1:-1] - psi[:-2, 1:-1])) / dy ** 2
    out = np.zeros_like(psi)
    out[1:-1, 1:-1] = (d2x + d2y) / f0 + beta * (y[1:-1, 1:-1] - y0) / f0
    return out


def potential_vorticity(omega, f, h):
    """diagnostics.py:150-181."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(h == 0, np.nan, (omega + f) / h)


def enstrophy(omega):
    return 0.5 * omega ** 2


def potential_enstrophy(q, h):
    return 0.5 * q ** 2 * h


def strain_magnitude_squared(sn, ss):
    return sn ** 2 + ss ** 2


def okubo_weiss(sn, ss, omega):
    return sn ** 2 + ss ** 2 - omega ** 2


def available_potential_energy(h, H, g_prime):
    return 0.5 * g_prime * (h - H) ** 2


def total_energy(ke, ape, dx, dy):
    """diagnostics.py:498-524."""
    return np.sum(ke[1:-1, 1:-1] + ape[1:-1, 1:-1]) * dx * dy


def total_enstrophy(ens, dx, dy):
    """diagnostics.py:527-555."""
    return np.sum(ens[1:-1, 1:-1]) * dx * dy


# ---------------------------------------------------------------------------
# Shallow-water operators: Coriolis2D (operators/coriolis.py:34-133),
# Vorticity2D (operators/vorticity.py:60-235), MomentumAdvection2D
# (diffusion/momentum.py:35-216) -- composed from interp2d / diff2d exactly as
# the reference composes Interpolation2D / Difference2D.
# ---------------------------------------------------------------------------


def coriolis2d(u, v, f, mask=None):
    """coriolis.py:86-133 (unmasked interpolation, masked outputs)."""
    f_on_u, f_on_v = interp2d("T_to_U", f), interp2d("T_to_V", f)
    v_on_u, u_on_v = interp2d("V_to_U", v), interp2d("U_to_V", u)
    du = _interior(f_on_u[1:-1, 1:-1] * v_on_u[1:-1, 1:-1], u)
    dv = _interior(-f_on_v[1:-1, 1:-1] * u_on_v[1:-1, 1:-1], v)
    if mask is not None:
        du, dv = du * mask["u"], dv * mask["v"]
    return du, dv


def potential_vorticity_x(u, v, h, f, dx, dy, mask=None):
    """Vorticity2D.potential_vorticity (vorticity.py:60-118)."""
    zeta = diff2d("curl", u, dx, dy, mask, v)
    f_on_q, h_on_q = interp2d("T_to_X", f, mask), interp2d("T_to_X", h, mask)
    num = zeta[1:-1, 1:-1] + f_on_q[1:-1, 1:-1]
    den = h_on_q[1:-1, 1:-1]
    with np.errstate(divide="ignore", invalid="ignore"):
        pv = np.where(den == 0, np.nan, num / den)
    out = _interior(pv, h)
    if mask is not None:
        out = np.where(mask["xy_corner_strict"] != 0, out, 0.0)
    return out


def pv_flux(q, u, v, scheme, alpha=1.0 / 3.0, mask=None):
    """Vorticity2D.pv_flux_{energy,enstrophy}_conserving / _arakawa_lamb
    (vorticity.py:120-235)."""
    def energy():
        q_on_u, q_on_v = interp2d("X_to_U", q, mask), interp2d("X_to_V", q, mask)
        return (_interior(q_on_u[1:-1, 1:-1] * u[1:-1, 1:-1], u),
                _interior(q_on_v[1:-1, 1:-1] * v[1:-1, 1:-1], v))

    def enstrophy():
        u_on_q, v_on_q = interp2d("U_to_X", u, mask), interp2d("V_to_X", v, mask)
        qu_at_q = _interior(q[1:-1, 1:-1] * u_on_q[1:-1, 1:-1], q)
        qv_at_q = _interior(q[1:-1, 1:-1] * v_on_q[1:-1, 1:-1], q)
        return interp2d("X_to_U", qu_at_q, mask), interp2d("X_to_V", qv_at_q, mask)

    if scheme == "energy":
        return energy()
    if scheme == "enstrophy":
        return enstrophy()
    (ue, ve), (us, vs) = energy(), enstrophy()
    return alpha * ue + (1.0 - alpha) * us, alpha * ve + (1.0 - alpha) * vs


def momentum_advection(u, v, dx, dy, scheme="energy", mask=None):
    """MomentumAdvection2D.__call__ (momentum.py:108-216)."""
    zeta = diff2d("curl", u, dx, dy, mask, v)
    u_on_T, v_on_T = interp2d("U_to_T", u, mask), interp2d("V_to_T", v, mask)
    K = _interior(0.5 * (u_on_T[1:-1, 1:-1] ** 2 + v_on_T[1:-1, 1:-1] ** 2), u)
    dK_dx, dK_dy = diff2d("diff_x_T_to_U", K, dx, dy, mask), diff2d("diff_y_T_to_V", K, dx, dy, mask)

    def e_scheme():
        zeta_on_u, zeta_on_v = interp2d("X_to_U", zeta, mask), interp2d("X_to_V", zeta, mask)
        v_on_u, u_on_v = interp2d("V_to_U", v, mask), interp2d("U_to_V", u, mask)
        return (_interior(zeta_on_u[1:-1, 1:-1] * v_on_u[1:-1, 1:-1], u),
                _interior(zeta_on_v[1:-1, 1:-1] * u_on_v[1:-1, 1:-1], v))

    def z_scheme():
        v_on_q, u_on_q = interp2d("V_to_X", v, mask), interp2d("U_to_X", u, mask)
        zv_at_q = _interior(zeta[1:-1, 1:-1] * v_on_q[1:-1, 1:-1], u)
        zu_at_q = _interior(zeta[1:-1, 1:-1] * u_on_q[1:-1, 1:-1], v)
        return interp2d("X_to_U", zv_at_q, mask), interp2d("X_to_V", zu_at_q, mask)

    if scheme == "energy":
        zv_u, zu_v = e_scheme()
    elif scheme == "enstrophy":
        zv_u, zu_v = z_scheme()
    elif scheme == "al":
        a = 1.0 / 3.0
        (e1, e2), (s1, s2) = e_scheme(), z_scheme()
        zv_u = _interior(a * e1[1:-1, 1:-1] + (1.0 - a) * s1[1:-1, 1:-1], u)
        zu_v = _interior(a * e2[1:-1, 1:-1] + (1.0 - a) * s2[1:-1, 1:-1], v)
    else:
        raise ValueError(f"Unknown scheme: {scheme!r}.  Choose 'energy', 'enstrophy', or 'al'.")
    du = _interior(zv_u[2:-2, 2:-2] - dK_dx[2:-2, 2:-2], u, ghost=2)
    dv = _interior(-zu_v[2:-2, 2:-2] - dK_dy[2:-2, 2:-2], v, ghost=2)
    if mask is not None:
        du, dv = du * mask["u"], dv * mask["v"]
    return du, dv
