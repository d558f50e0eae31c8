"""Arakawa C-grid metadata (finitevolX grid/base.py:61-96, grid/cartesian.py:56-108)."""

from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class ArakawaCGrid2D:
    """Total shape [Ny, Nx] including a one-cell ghost ring on every side.

    Same-index stagger: T[j,i] cell centre, U[j,i] east face (i+1/2),
    V[j,i] north face (j+1/2), X[j,i] north-east corner.
    """

    Nx: int
    Ny: int
    Lx: float
    Ly: float
    dx: float
    dy: float

    @classmethod
    def from_interior(cls, nx_interior: int, ny_interior: int, Lx: float, Ly: float):
        """grid/cartesian.py:83-108: Nx = nx+2, dx = Lx / nx."""
        return cls(Nx=nx_interior + 2, Ny=ny_interior + 2, Lx=Lx, Ly=Ly,
                   dx=Lx / nx_interior, dy=Ly / ny_interior)

    @property
    def shape(self):
        return (self.Ny, self.Nx)


CartesianGrid2D = ArakawaCGrid2D
