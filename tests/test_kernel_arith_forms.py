"""CPU checks of arithmetic reformulations the CUDA kernels rely on (NumPy
emulation of the kernels' FP32 formulas and index walks; the GPU parity
tests check the kernels themselves against the oracle).

* FP32 WENO5 (Jiang-Shu) weights normalised with one reciprocal: the
  weights d_k / s_k times s_1 s_2 s_3 give the same reconstruction as the
  four-division form (csrc/recon.cuh weno5_core, csrc/qg_stage.cuh
  weno5_x2), and stencils whose products overflow are the ones the kernels
  send to the four-division fallback.
* Division-free (row, column) walks of the multigrid kernels (csrc/mg.cu
  coarse_cells, grid_cells): the same cells as c -> (c / w, c % w).
* The multigrid legs' thread layout (csrc/mg.cu leg_shape, leg_config):
  every cell of a leg's region is owned by exactly one thread, within that
  thread's register rows, for every sweep count a leg accepts.
"""

import numpy as np
import pytest

F = np.float32


def _smoothness(qmm, qm, q0, qp, qpp):
    k1, k2 = F(13.0 / 12.0), F(0.25)
    b1 = k1 * (qmm - F(2) * qm + q0) ** 2 + k2 * (qmm - F(4) * qm + F(3) * q0) ** 2
    b2 = k1 * (qm - F(2) * q0 + qp) ** 2 + k2 * (qm - qp) ** 2
    b3 = k1 * (q0 - F(2) * qp + qpp) ** 2 + k2 * (F(3) * q0 - F(4) * qp + qpp) ** 2
    qi1 = F(1.0 / 3.0) * qmm - F(7.0 / 6.0) * qm + F(11.0 / 6.0) * q0
    qi2 = F(-1.0 / 6.0) * qm + F(5.0 / 6.0) * q0 + F(1.0 / 3.0) * qp
    qi3 = F(1.0 / 3.0) * q0 + F(5.0 / 6.0) * qp - F(1.0 / 6.0) * qpp
    return (b1, b2, b3), (qi1, qi2, qi3)


def weno5_four_divisions(b, qi):
    eps = F(1e-8)
    w = [F(d) / (bk + eps) ** 2 for d, bk in zip((0.1, 0.6, 0.3), b)]
    return (w[0] * qi[0] + w[1] * qi[1] + w[2] * qi[2]) / (w[0] + w[1] + w[2])


def weno5_one_reciprocal(b, qi):
    """The kernels' form; returns (value, takes_fallback)."""
    eps = F(1e-8)
    s1, s2, s3 = ((bk + eps) ** 2 for bk in b)
    with np.errstate(over="ignore", invalid="ignore"):
        W1, W2, W3 = F(0.1) * (s2 * s3), F(0.6) * (s1 * s3), F(0.3) * (s1 * s2)
        den = W1 + W2 + W3
        r = (W1 * qi[0] + W2 * qi[1] + W3 * qi[2]) * (F(1) / den)
        ok = (den < F(3e38)) & (np.abs(r) < F(3.4e38))
    return r, ~ok


@pytest.mark.parametrize("scale", [1e-5, 1.0, 1e3])
def test_weno5_one_reciprocal_matches_four_divisions(scale):
    rng = np.random.default_rng(7)
    q = (rng.standard_normal((5, 200000)) * scale).astype(F)
    b, qi = _smoothness(*q)
    ref = weno5_four_divisions(b, qi)
    got, fb = weno5_one_reciprocal(b, qi)
    assert not fb.any()
    # the reconstruction is a convex combination of qi: bound the difference
    # by a few FP32 ulps of the largest candidate
    mag = np.maximum.reduce([np.abs(x) for x in qi]) + np.float32(1e-30)
    assert np.max(np.abs(got - ref) / mag) < 8 * np.finfo(F).eps


def test_weno5_overflowing_products_take_the_fallback():
    # jumps of 1e5 make s ~ 1e20 and the products overflow: the kernels'
    # test routes exactly these stencils to the four-division form, which
    # stays finite
    q = np.array([[0.0], [0.0], [1e5], [0.0], [0.0]], dtype=F)
    b, qi = _smoothness(*q)
    _, fb = weno5_one_reciprocal(b, qi)
    assert fb.all()
    assert np.isfinite(weno5_four_divisions(b, qi)).all()


def _walk(n_cells, w, nthreads, tid):
    """(j, i) sequence of csrc/mg.cu's division-free walk for one thread."""
    dq, dr = nthreads // w, nthreads % w
    j, i = tid // w, tid % w
    out = []
    for _ in range(tid, n_cells, nthreads):
        out.append((j, i))
        i += dr
        j += dq
        if i >= w:
            i -= w
            j += 1
    return out


@pytest.mark.parametrize("h,w,nthreads", [(32, 32, 1024), (16, 16, 1024), (8, 8, 1024), (46, 78, 256),
                                          (44, 76, 1024), (3, 2000, 256), (5, 1, 1024), (30, 37, 256)])
def test_division_free_walk_visits_the_same_cells(h, w, nthreads):
    n = h * w
    for tid in range(nthreads):
        ref = [divmod(c, w) for c in range(tid, n, nthreads)]
        assert _walk(n, w, nthreads, tid) == ref


def test_mask_free_jacobi_equals_masked_form():
    # the multigrid legs' sweeps drop the multiplications by the 0/1 mask:
    # u is kept masked, inv_diag (mask-multiplied by construction) carries
    # omega; on wet cells the dropped factors are 1, on dry cells both forms
    # give zero -- the same values as jacobi_at (multigrid.py:408-461)
    import oracle.fvx_oracle as O
    rng = np.random.default_rng(3)
    n = 40
    mask = (rng.random((n, n)) > 0.3).astype(np.float64)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 0.0
    coeff = np.exp(0.5 * rng.standard_normal((n, n)))
    L = O.mg_build(mask, 0.1, 0.1, lambda_=2.0, coeff=coeff, n_levels=1)["levels"][0]
    u = rng.standard_normal((n, n)) * mask
    f = rng.standard_normal((n, n))
    omega = 0.95
    ref = O.mg_jacobi(u, f, L, omega, 1)
    pad = lambda a: np.pad(a, 1)  # noqa: E731
    up, cxp, cyp = pad(u), pad(L["cx"]), pad(L["cy"])
    c = (slice(1, -1), slice(1, -1))
    um, ue, uw = up[c], up[1:-1, 2:], up[1:-1, :-2]
    un, us = up[2:, 1:-1], up[:-2, 1:-1]
    lap = (cxp[c] * (ue - um) - cxp[1:-1, :-2] * (um - uw)) / 0.1 ** 2 + \
          (cyp[c] * (un - um) - cyp[:-2, 1:-1] * (um - us)) / 0.1 ** 2
    r = f - (lap - 2.0 * um)
    got = um + (omega * L["inv"]) * r
    np.testing.assert_array_equal(got, ref)


def _leg_shape(tx, ty, halo, nt):
    rw, rh = tx + 2 * halo, ty + 2 * halo
    nseg = nt // rw
    return rw, rh, (-(-rh // nseg) if nseg > 0 else 1 << 20)


@pytest.mark.parametrize("tile", [(64, 32), (32, 16)])
def test_leg_threads_own_every_region_cell_once(tile):
    nt_r = [(512, 4), (512, 8), (1024, 4), (1024, 8)]  # leg_config's candidates
    for k in range(0, 17):  # sweeps per leg (kLegMaxSweeps = 16)
        for halo in (k + 1, k):  # down leg, up leg
            for order in ((2, 3, 1, 0), (0, 1, 2, 3)):
                cfg = next(i for i in order if _leg_shape(*tile, k + 1, nt_r[i][0])[2] <= nt_r[i][1])
                nt, rows = nt_r[cfg]
                rw, rh, lr = _leg_shape(*tile, halo, nt)
                assert lr <= rows
                owned = np.zeros((rh, rw), np.int64)
                for tid in range(nt):
                    seg, c = divmod(tid, rw)
                    r0 = seg * lr
                    if r0 >= rh:
                        continue
                    for i in range(rows):
                        r = r0 + i
                        if i < lr and r < rh:
                            owned[r, c] += 1
                assert (owned == 1).all(), (tile, k, halo, cfg)
