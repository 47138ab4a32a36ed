"""Index space of a GETM domain as laid out in memory (cppdefs.h:146-159).

A 3D field covers ``(imin-2:imax+2, jmin-2:jmax+2, 0:kmax)`` with i fastest: as a C-contiguous
array its shape is ``(kmax+1, nj, ni)`` (identical bytes to the Fortran column-major array);
a 2D field is ``(nj, ni)``. Indices below are the reference's (Fortran) indices.
"""
from __future__ import annotations

import ctypes as C

HALO = 2


class GetmDomain(C.Structure):
    """Mirror of ``getm_domain`` in include/getm_b200.h."""

    _fields_ = [
        ("imin", C.c_int32), ("imax", C.c_int32), ("jmin", C.c_int32), ("jmax", C.c_int32), ("kmax", C.c_int32),
        ("sj", C.c_int64), ("sk", C.c_int64),
        ("dx", C.c_double), ("dy", C.c_double), ("ard1", C.c_double),
    ]


class Grid:
    """Cartesian GETM grid: nx x ny interior columns, kmax layers, halo 2 (domain.F90)."""

    def __init__(self, nx: int, ny: int, kmax: int, dx: float, dy: float, imin: int = 1, jmin: int = 1):
        if nx < 1 or ny < 1 or kmax < 0:
            raise ValueError("bad grid size")
        self.nx, self.ny, self.kmax = int(nx), int(ny), int(kmax)
        self.imin, self.jmin = int(imin), int(jmin)
        self.imax, self.jmax = self.imin + self.nx - 1, self.jmin + self.ny - 1
        self.ni, self.nj, self.nk = self.nx + 2 * HALO, self.ny + 2 * HALO, self.kmax + 1
        self.dx, self.dy = float(dx), float(dy)
        self.ard1 = 1.0 / (self.dx * self.dy)  # domain.F90:596

    # array index of reference index i / j
    def ii(self, i: int) -> int:
        return i - (self.imin - HALO)

    def jj(self, j: int) -> int:
        return j - (self.jmin - HALO)

    def shape3(self):
        return (self.nk, self.nj, self.ni)

    def shape2(self):
        return (self.nj, self.ni)

    def interior(self):
        """Slices of the interior imin..imax, jmin..jmax in array indices (j, i)."""
        return (slice(HALO, HALO + self.ny), slice(HALO, HALO + self.nx))

    def cells(self) -> int:
        return self.nx * self.ny * self.kmax

    def domain(self) -> GetmDomain:
        return GetmDomain(self.imin, self.imax, self.jmin, self.jmax, self.kmax, self.ni, self.ni * self.nj,
                          self.dx, self.dy, self.ard1)

    def __repr__(self):
        return f"Grid({self.nx}x{self.ny}x{self.kmax}, dx={self.dx}, dy={self.dy})"
