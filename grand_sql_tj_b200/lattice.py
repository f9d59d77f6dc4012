"""Lattice and coupling tables of the square t-J cylinder (host-side set-up).

These are the module globals that the hot path reads (neib, neiba, inb1,
nleg11, nposi, nposi_dm, nposi_lat, jt, jz, jd, jn, esite).  The Fortran
caller owns them; this module rebuilds them for the standalone driver, the
tests and the benchmark, following

  * main.f90:40-47            couplings (jz, jd = -sqrt(3) jz, jt, jn = -jz/4, esite)
  * dmrg_sub.f90:1-29         dmrg_setup0 (inb1, nleg11 from the full lattice)
  * dmrg_sub.f90:31-143,271-279  dmrg_setup for the square lattice

Only the square lattice (square = 1, nly = 1, nc = 1) is built; the
triangle and honeycomb branches of dmrg_setup are not on the hot path.
"""
from __future__ import annotations

import math

import numpy as np

from .structs import Lattice

NEIBT = 12
NEIBT1 = 8


class Geometry:
    """Nx x Ny cylinder (periodic in y when Ny > 2, open in x), sites numbered
    column by column: site = y + (x-1)*Ny (Get_Lattice, dmrg_sub.f90:350-365)."""

    def __init__(self, nx: int, ny: int, t: float = 1.0, J: float = 1.0 / 3.0, t2: float = 0.0,
                 esite: float = 0.0, up_bias: int = 1, open_x: int = 1):
        self.nx, self.ny, self.nleg = nx, ny, ny
        self.num_site = nx * ny
        self.open = open_x
        self.up_bias = up_bias
        ns1 = self.num_site + 1
        # couplings (main.f90:36-47) in units where hopping carries the SU(2) sqrt(2)
        self.jz = np.zeros((NEIBT, ns1))
        self.jd = np.zeros((NEIBT, ns1))
        self.jt = np.zeros((NEIBT, ns1))
        self.jn = np.zeros(NEIBT)
        r = t2 / t if t != 0 else 0.0
        self.jz[0:4, 1:] = J
        self.jz[4:8, 1:] = J * r * r
        self.jd[:, 1:] = self.jz[:, 1:] * (-math.sqrt(3.0))
        self.jt[0:4, 1:] = -math.sqrt(2.0) * t
        self.jt[4:8, 1:] = -math.sqrt(2.0) * t2
        self.jn[:] = -self.jz[:, 1] / 4.0
        self.esite = np.full(ns1, float(esite))
        # full-lattice tables, then dmrg_setup0 (main.f90:50-52)
        self.setup(self.num_site // 2 - 1, self.num_site // 2 - 1)
        self._setup0()

    # dmrg_setup0 (dmrg_sub.f90:1-29)
    def _setup0(self):
        ns1 = self.num_site + 1
        self.inb1 = np.zeros((ns1, ns1), dtype=np.int32)
        self.nleg11 = np.zeros(self.num_site, dtype=np.int32)
        for ns in range(1, self.num_site - 1):
            k0 = 0
            for i1 in range(1, ns + 1):
                self.inb1[i1, ns] = 10000
                k00 = int(np.sum(self.neib[i1, 1:] >= ns))
                if k00 != 0:
                    k0 += 1
                    self.inb1[i1, ns] = k0
            self.nleg11[ns - 1] = k0

    # dmrg_setup (dmrg_sub.f90:31-143, 271-279), square lattice
    def setup(self, ns: int, ns21: int):
        nleg, ns1 = self.nleg, self.num_site + 1
        nn = ns + ns21 + 2
        nxc = (nn - 1) // nleg + 1
        self.ns, self.ns21 = ns, ns21
        nposi = np.zeros(ns1 + 2, dtype=np.int32)
        nposi_lat = np.zeros(ns1 + 2, dtype=np.int32)
        nposi_dm = np.zeros(ns1 + 2, dtype=np.int32)
        neib = np.zeros((ns1 + 2 * nleg + 2, NEIBT + 1), dtype=np.int32)   # neib(i, k), 1-based k
        neiba = np.zeros((ns1 + 2 * nleg + 2, ns1 + 2 * nleg + 2), dtype=np.int32)
        totsite = nleg * nxc
        for i in range(1, ns + 2):
            nposi[i] = 1
            nposi_lat[i] = i
            nposi_dm[i] = i
        nposi[ns + 1] = 2
        for i in range(1, ns21 + 2):
            nposi[ns + 1 + i] = 3
            nposi_dm[totsite + 1 - i] = i + (ns + 1)
            nposi_lat[i + ns + 1] = totsite + 1 - i
        nposi[ns + 1 + ns21 + 1] = 4

        def link(a, b, ka, kb):
            neib[a, ka] = b
            neib[b, kb] = a
            neiba[a, b] = ka
            neiba[b, a] = kb

        for ix in range(1, nxc + 1):
            for iy in range(1, nleg + 1):
                ii = iy + (ix - 1) * nleg
                jy = ii - iy + (iy % nleg) + 1
                if iy != nleg or nleg != 2:
                    link(ii, jy, 1, 2)
                jx = ii + nleg
                if jx > nleg * nxc:
                    jx = jx - nleg * nxc if (self.open == 0 and nxc >= 3) else 0
                if jx != 0:
                    link(ii, jx, 3, 4)
                    jy = jx - 1
                    if iy == 1:
                        jy += nleg
                    if jy != 0:
                        link(ii, jy, 5, 6)
                    jy = jx + 1
                    if iy == nleg:
                        jy -= nleg
                    if jy != 0:
                        link(ii, jy, 7, 8)
        for i in range(1, self.num_site + 1):
            for j in range(NEIBT1 + 1, NEIBT + 1):
                if abs(self.jz[j - 1, 1]) + abs(self.jd[j - 1, 1]) + abs(self.jt[j - 1, 1]) + abs(self.jn[j - 1]) == 0.0:
                    b = neib[i, j]
                    neiba[i, b] = 0
                    neiba[b, i] = 0
                    neib[i, j] = 0
        self.neib = neib[:ns1, :]
        self.neiba = neiba[:ns1, :ns1]
        self.nposi = nposi[:ns1]
        self.nposi_dm = nposi_dm[:ns1]
        self.nposi_lat = nposi_lat[:ns1]

    def lattice(self, sys_len: int, env_len: int) -> Lattice:
        """Tables for the superblock [sys_len + 1 + 1 + env_len]."""
        self.setup(sys_len, env_len)
        return Lattice(self.num_site, NEIBT, self.up_bias,
                       np.asfortranarray(self.neib[:, 1:]), self.neiba, self.inb1, self.nleg11,
                       self.nposi, self.nposi_dm, self.nposi_lat, self.jt, self.jz, self.jd,
                       self.jn, self.esite)
