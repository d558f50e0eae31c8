"""Mask2D / StencilCapability2D built on the device.

Mirrors finitevolX mask/cartesian.py:345-739 and mask/base.py:60-105.  All
construction runs in libfvx.so (``fvx_mask2d_build``, ``fvx_compact_flags``,
``fvx_adaptive_masks``); stored arrays are CUDA tensors (bool / int32 /
float32), bit-exact with the reference's NumPy construction.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import I, I64, P, check, fn, stream_ptr


@dataclass
class StencilCapability2D:
    """Directional contiguous-wet-cell counts (mask/base.py:60-105)."""

    x_pos: torch.Tensor
    x_neg: torch.Tensor
    y_pos: torch.Tensor
    y_neg: torch.Tensor

    @classmethod
    def from_mask(cls, h) -> "StencilCapability2D":
        m = L.as_mask(h)
        ny, nx = m.shape
        out = [torch.empty((ny, nx), dtype=torch.int32, device=m.device) for _ in range(4)]
        check(fn("fvx_count_contiguous")(P(m), I(ny), I(nx), I(1), P(out[0]), P(out[1]), stream_ptr()),
              "count_contiguous")
        check(fn("fvx_count_contiguous")(P(m), I(ny), I(nx), I(0), P(out[2]), P(out[3]), stream_ptr()),
              "count_contiguous")
        return cls(*out)


def count_contiguous(arr, axis: int, forward: bool) -> torch.Tensor:
    """mask/utils.py:385-468 for 2-D masks (int32, on the device)."""
    m = L.as_mask(arr)
    if m.ndim != 2:
        raise ValueError("count_contiguous: 2-D masks only")
    if axis not in (0, 1, -1, -2):
        raise ValueError(f"axis {axis} out of range for a 2-D mask")
    axis = axis % 2
    ny, nx = m.shape
    pos = torch.empty((ny, nx), dtype=torch.int32, device=m.device)
    neg = torch.empty_like(pos)
    check(fn("fvx_count_contiguous")(P(m), I(ny), I(nx), I(axis), P(pos), P(neg), stream_ptr()),
          "count_contiguous")
    return pos if forward else neg


def make_sponge(shape, width) -> torch.Tensor:
    """mask/utils.py:471-546 for 2-D shapes (float32 on the device)."""
    ny, nx = shape
    h = torch.ones((ny, nx), dtype=torch.bool, device=L.require_cuda())
    return Mask2D.from_mask(h, sponge_width=width).sponge


class Mask2D:
    """Arakawa C-grid mask for a 2-D Cartesian domain (mask/cartesian.py:345-739)."""

    def __init__(self, **fields):
        for k, v in fields.items():
            setattr(self, k, v)

    # -- construction -------------------------------------------------------
    @classmethod
    def from_mask(cls, mask_hgrid, sponge_width: int | None = None, k_bottom=None) -> "Mask2D":
        h = L.as_mask(mask_hgrid)
        if h.ndim != 2:
            raise ValueError("Mask2D.from_mask expects a 2-D mask")
        if sponge_width is not None and sponge_width < 0:
            raise ValueError(f"sponge_width must be non-negative; got {sponge_width!r}")
        ny, nx = h.shape
        dev = h.device
        b = lambda: torch.empty((ny, nx), dtype=torch.bool, device=dev)  # noqa: E731
        i32 = lambda: torch.empty((ny, nx), dtype=torch.int32, device=dev)  # noqa: E731
        u, v, xy, xys, yw, xw, cv, va, irr = (b() for _ in range(9))
        cls_ = i32()
        xp, xn, yp, yn = (i32() for _ in range(4))
        sponge = torch.empty((ny, nx), dtype=torch.float32, device=dev)
        sw = 0 if sponge_width is None else int(sponge_width)
        check(fn("fvx_mask2d_build")(P(h), I(ny), I(nx), P(u), P(v), P(xy), P(xys), P(yw), P(xw), P(cv),
                                     P(va), P(cls_), P(irr), P(xp), P(xn), P(yp), P(yn), P(sponge), I(sw),
                                     stream_ptr()), "Mask2D.from_mask")
        rows, cols = _compact(irr)
        return cls(h=h, u=u, v=v, xy_corner=xy, xy_corner_strict=xys,
                   xy_corner_y_wall=yw, xy_corner_x_wall=xw, xy_corner_convex=cv, xy_corner_valid=va,
                   xy_corner_strict_irrbound_rows=rows, xy_corner_strict_irrbound_cols=cols,
                   classification=cls_, stencil_capability=StencilCapability2D(xp, xn, yp, yn),
                   sponge=sponge, k_bottom=None if k_bottom is None else L.as_field(k_bottom),
                   _tiers=None)

    @classmethod
    def from_dimensions(cls, ny: int, nx: int, sponge_width: int | None = None) -> "Mask2D":
        return cls.from_mask(torch.ones((ny, nx), dtype=torch.bool, device=L.require_cuda()),
                             sponge_width=sponge_width)

    @classmethod
    def from_center(cls, field, sponge_width: int | None = None, k_bottom=None) -> "Mask2D":
        """NaN marks dry cells (mask/cartesian.py:741-770)."""
        if isinstance(field, torch.Tensor):
            h = torch.isfinite(field.to(L.require_cuda()))
        else:
            h = np.isfinite(np.asarray(field))
        return cls.from_mask(h, sponge_width=sponge_width, k_bottom=k_bottom)

    # -- inverted masks and classification accessors -----------------------
    @property
    def not_h(self):
        return ~self.h

    @property
    def not_u(self):
        return ~self.u

    @property
    def not_v(self):
        return ~self.v

    @property
    def not_xy_corner(self):
        return ~self.xy_corner

    @property
    def not_xy_corner_strict(self):
        return ~self.xy_corner_strict

    @property
    def ind_land(self):
        return self.classification == 0

    @property
    def ind_coast(self):
        return self.classification == 1

    @property
    def ind_near_coast(self):
        return self.classification == 2

    @property
    def ind_ocean(self):
        return self.classification == 3

    @property
    def shape(self):
        return tuple(self.h.shape)

    # -- adaptive stencil masks --------------------------------------------
    def _stencil_capability_for(self, source: str) -> StencilCapability2D:
        grid_map = {"h": self.h, "u": self.u, "v": self.v, "xy_corner": self.xy_corner,
                    "xy_corner_strict": self.xy_corner_strict}
        if source not in grid_map:
            raise ValueError(f"source must be one of {list(grid_map)!r}, got {source!r}")
        if source == "h":
            return self.stencil_capability
        return StencilCapability2D.from_mask(grid_map[source])

    def get_adaptive_masks(self, direction: str = "x", source: str = "h",
                           stencil_sizes=(2, 4, 6, 8, 10)) -> dict:
        """Mutually exclusive tier masks (mask/cartesian.py:495-553)."""
        sc = self._stencil_capability_for(source)
        if direction == "x":
            pos, neg = sc.x_pos, sc.x_neg
        elif direction == "y":
            pos, neg = sc.y_pos, sc.y_neg
        else:
            raise ValueError(f"direction must be 'x' or 'y', got {direction!r}")
        sizes = sorted(int(s) for s in stencil_sizes)
        n = pos.numel()
        dev_sizes = torch.tensor(sizes, dtype=torch.int32, device=pos.device)
        out = torch.empty((len(sizes),) + tuple(pos.shape), dtype=torch.bool, device=pos.device)
        check(fn("fvx_adaptive_masks")(P(pos), P(neg), I64(n), P(dev_sizes), I(len(sizes)), P(out),
                                       stream_ptr()), "get_adaptive_masks")
        by_size = {s: out[k] for k, s in enumerate(sizes)}
        return {int(s): by_size[int(s)] for s in stencil_sizes}

    def tier_codes(self) -> torch.Tensor:
        """Packed (2, 4, 6) tier codes used by the masked advection kernels."""
        if self._tiers is None:
            sc = self.stencil_capability
            t = torch.empty(self.h.shape, dtype=torch.uint8, device=self.h.device)
            check(fn("fvx_tier_codes")(P(sc.x_pos), P(sc.x_neg), P(sc.y_pos), P(sc.y_neg),
                                       I64(t.numel()), P(t), stream_ptr()), "tier_codes")
            self._tiers = t
        return self._tiers


def _compact(flags: torch.Tensor):
    ny, nx = flags.shape
    work = torch.empty(2 * ny + 1, dtype=torch.int32, device=flags.device)
    rows = torch.empty(ny * nx, dtype=torch.int32, device=flags.device)
    cols = torch.empty(ny * nx, dtype=torch.int32, device=flags.device)
    check(fn("fvx_compact_flags")(P(flags), I(ny), I(nx), P(work), P(rows), P(cols), stream_ptr()),
          "compact_flags")
    total = int(work[2 * ny].item())
    return rows[:total].clone(), cols[:total].clone()


def narrow_mask_hierarchy(hierarchy: dict, target_sizes) -> dict:
    """advection/flux.py:41-97 (OR-fold tiers >= the largest target)."""
    sizes = sorted(target_sizes)
    if not sizes:
        raise ValueError("target_sizes must not be empty")
    out = {}
    for s in sizes[:-1]:
        if s not in hierarchy:
            raise ValueError(f"hierarchy is missing stencil size {s}; available: {sorted(hierarchy.keys())}")
        out[s] = hierarchy[s]
    fold = None
    for s, m in hierarchy.items():
        if s >= sizes[-1]:
            fold = m if fold is None else (fold | m)
    if fold is None:
        raise ValueError(f"hierarchy has no tier >= biggest target size {sizes[-1]}; "
                         f"available: {sorted(hierarchy.keys())}")
    out[sizes[-1]] = fold
    return out
