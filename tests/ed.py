"""Exact diagonalisation of the t-J model on small clusters (test helper, CPU).

An independent check of the Hamiltonian that the DMRG path builds: the full
Fock space of the t-J model (each site empty, up or down; no double
occupancy) in the sector of fixed electron number N and S_z = 0, with

  H = sum_<ij> [ -t_ij sum_s (c+_is c_js + h.c.) + J_ij (S_i.S_j - n_i n_j / 4) ]
      + sum_i esite_i n_i

-- the model the reference states in code/tjsq/common.f90:1-4 -- on the
bonds and couplings of the same neighbour tables the DMRG uses
(grand_sql_tj_b200.lattice.Geometry: t_ij = -jt_ij / sqrt(2), J_ij = jz_ij).
The SU(2) DMRG targets total spin S = tot_num_down / 2, so the lowest
eigenvalue among the states with S(S+1) = that value is returned.

This module shares no code with the oracle or the product: states are bit
masks, fermion signs come from the Jordan-Wigner order (site, spin), and the
matrix is diagonalised with scipy's sparse Lanczos.
"""
from __future__ import annotations

import itertools
import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla


def bonds_of(geo):
    """(i, j, t_ij, J_ij) for every bond of the full lattice, 0-based sites."""
    geo.setup(geo.num_site // 2 - 1, geo.num_site // 2 - 1)
    out = []
    n = geo.num_site
    for i in range(1, n + 1):
        for k in (1, 3, 5, 7, 9, 11):        # forward directions; k + 1 is the reverse
            j = int(geo.neib[i, k])
            if j == 0:
                continue
            t = -float(geo.jt[k - 1, i]) / math.sqrt(2.0)
            J = float(geo.jz[k - 1, i])
            if t != 0.0 or J != 0.0:
                out.append((i - 1, j - 1, t, J))
    return out


def _states(n, n_elec, n_up=None):
    ups, dns = [], []
    nu = n_elec // 2 if n_up is None else n_up
    for occ in itertools.combinations(range(n), n_elec):
        for upset in itertools.combinations(occ, nu):
            u = 0
            for s in upset:
                u |= 1 << s
            o = 0
            for s in occ:
                o |= 1 << s
            ups.append(u)
            dns.append(o & ~u)
    return np.array(ups, dtype=np.int64), np.array(dns, dtype=np.int64)


def _popcount(x):
    x = x.copy()
    c = np.zeros_like(x)
    while np.any(x):
        c += x & 1
        x >>= 1
    return c


class TJCluster:
    def __init__(self, n_site, bonds, esite, n_elec, n_up=None):
        assert n_up is not None or n_elec % 2 == 0
        self.n, self.bonds, self.N = n_site, bonds, n_elec
        self.up, self.dn = _states(n_site, n_elec, n_up)
        self.key = (self.up << n_site) | self.dn
        order = np.argsort(self.key)
        self.up, self.dn, self.key = self.up[order], self.dn[order], self.key[order]
        self.dim = len(self.key)
        self.esite = np.asarray(esite, dtype=float)

    def _index(self, up, dn):
        k = (up << self.n) | dn
        idx = np.searchsorted(self.key, k)
        assert np.all(self.key[idx] == k)
        return idx

    def _between(self, i, j):
        lo, hi = min(i, j), max(i, j)
        m = 0
        for s in range(lo + 1, hi):
            m |= 1 << s
        return m

    def hamiltonian(self):
        rows, cols, vals = [], [], []
        up, dn = self.up, self.dn
        occ = up | dn
        idx = np.arange(self.dim)
        diag = np.zeros(self.dim)
        for s in range(self.n):
            diag += self.esite[s] * ((occ >> s) & 1)
        for (i, j, t, J) in self.bonds:
            bi, bj = 1 << i, 1 << j
            between = self._between(i, j)
            nb = _popcount(occ & between)
            sign = np.where(nb % 2 == 0, 1.0, -1.0)
            if t != 0.0:
                for (a, b) in ((i, j), (j, i)):      # c+_a c_b, both spins
                    ba, bb = 1 << a, 1 << b
                    for spin in (0, 1):
                        src = up if spin == 0 else dn
                        ok = ((src & bb) != 0) & ((occ & ba) == 0)
                        if not np.any(ok):
                            continue
                        nu, nd = up[ok].copy(), dn[ok].copy()
                        if spin == 0:
                            nu = nu ^ bb ^ ba
                        else:
                            nd = nd ^ bb ^ ba
                        rows.append(self._index(nu, nd))
                        cols.append(idx[ok])
                        vals.append(-t * sign[ok])
            if J != 0.0:
                both = ((occ & bi) != 0) & ((occ & bj) != 0)
                anti = both & (((up & bi) != 0) != ((up & bj) != 0))
                diag[anti] += J * (-0.5)                 # Sz Sz - n n / 4 = -1/2 for antiparallel
                # (S+_i S-_j + S-_i S+_j) / 2 flips an antiparallel pair
                nu, nd = up[anti] ^ bi ^ bj, dn[anti] ^ bi ^ bj
                rows.append(self._index(nu, nd))
                cols.append(idx[anti])
                vals.append(np.full(int(anti.sum()), 0.5 * J))
        rows.append(idx)
        cols.append(idx)
        vals.append(diag)
        r, c, v = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
        return sp.csr_matrix((v, (r, c)), shape=(self.dim, self.dim))

    def spin_squared(self):
        """S_tot^2 = sum_i 3/4 n_i + 2 sum_{i<j} S_i.S_j."""
        up, dn = self.up, self.dn
        occ = up | dn
        idx = np.arange(self.dim)
        diag = 0.75 * _popcount(occ).astype(float)
        rows, cols, vals = [], [], []
        for i in range(self.n):
            for j in range(i + 1, self.n):
                bi, bj = 1 << i, 1 << j
                both = ((occ & bi) != 0) & ((occ & bj) != 0)
                par = both & (((up & bi) != 0) == ((up & bj) != 0))
                anti = both & ~par
                diag[par] += 2 * 0.25
                diag[anti] += 2 * -0.25
                nu, nd = up[anti] ^ bi ^ bj, dn[anti] ^ bi ^ bj
                rows.append(self._index(nu, nd))
                cols.append(idx[anti])
                vals.append(np.full(int(anti.sum()), 1.0))
        rows.append(idx)
        cols.append(idx)
        vals.append(diag)
        r, c, v = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
        return sp.csr_matrix((v, (r, c)), shape=(self.dim, self.dim))


def ground_energy(geo, n_elec, two_s=0, k=8):
    """Lowest energy with total spin two_s / 2 in the N = n_elec, S_z = 0 sector,
    and the state's <S_i . S_j> matrix."""
    cl = TJCluster(geo.num_site, bonds_of(geo), geo.esite[1:geo.num_site + 1], n_elec)
    H = cl.hamiltonian()
    S2 = cl.spin_squared()
    target = 0.25 * two_s * (two_s + 2)
    if cl.dim <= 400:
        w, v = np.linalg.eigh(H.toarray())
    else:
        w, v = sla.eigsh(H, k=min(k, cl.dim - 2), which="SA", tol=1e-13)
        o = np.argsort(w)
        w, v = w[o], v[:, o]
    for a in range(len(w)):
        s2 = float(v[:, a] @ (S2 @ v[:, a]))
        if abs(s2 - target) < 1e-6:
            return float(w[a]), v[:, a], cl
    raise RuntimeError("no state with the target spin among the lowest %d" % len(w))


def spin_correlation(cl, psi, i, j):
    """<psi| S_i . S_j |psi> (0-based sites i != j)."""
    up, dn = cl.up, cl.dn
    occ = up | dn
    bi, bj = 1 << i, 1 << j
    both = ((occ & bi) != 0) & ((occ & bj) != 0)
    par = both & (((up & bi) != 0) == ((up & bj) != 0))
    anti = both & ~par
    v = 0.25 * float(np.sum(psi[par] ** 2)) - 0.25 * float(np.sum(psi[anti] ** 2))
    src = np.nonzero(anti)[0]
    dst = cl._index(up[anti] ^ bi ^ bj, dn[anti] ^ bi ^ bj)
    v += 0.5 * float(np.sum(psi[dst] * psi[src]))
    return v


def grand_canonical_ground_energy(geo):
    """min over even N of the S = 0 ground energy (the shipped up_bias = 0 mode)."""
    best = None
    for n in range(0, geo.num_site + 1, 2):
        if n == 0:
            e = 0.0
        else:
            e, _, _ = ground_energy(geo, n)
        best = e if best is None else min(best, e)
    return best


def density_correlation(cl, psi, i, j):
    """<psi| n_i n_j |psi> (0-based sites i != j)."""
    occ = cl.up | cl.dn
    both = ((occ >> i) & 1) & ((occ >> j) & 1)
    return float(np.sum(psi[both == 1] ** 2))


def annihilate(cl, vec, site, spin, target):
    """c_(site, spin) |vec> as a vector of the cluster `target` (one electron
    less).  Fermion order: modes by site, up (spin 0) before down (spin 1) on a
    site -- the order whose string the hopping of TJCluster.hamiltonian counts
    (electrons on the sites between the two ends)."""
    src = cl.up if spin == 0 else cl.dn
    b = 1 << site
    ok = (src & b) != 0
    up, dn = cl.up[ok], cl.dn[ok]
    below = b - 1
    # occupied modes before (site, spin): every electron on a lower site, and
    # the up electron of this site when a down electron is removed
    nbefore = _popcount(up & below) + _popcount(dn & below) + (spin == 1) * ((up & b) != 0)
    if spin == 0:
        up = up ^ b
    else:
        dn = dn ^ b
    out = np.zeros(target.dim)
    out[target._index(up, dn)] = vec[ok] * np.where(nbefore % 2 == 0, 1.0, -1.0)
    return out


_SECTORS = {}


def _sector(n, n_elec, n_up):
    """The basis of n sites with n_elec electrons, n_up of them up (memoised)."""
    key = (n, n_elec, n_up)
    if key not in _SECTORS:
        _SECTORS[key] = TJCluster(n, [], np.zeros(n), n_elec, n_up)
    return _SECTORS[key]


def singlet_pair_correlation(cl, psi, a, b, c, d):
    """<psi| D+_(a,b) D_(c,d) |psi> with D_(i,j) = (c_(j,dn) c_(i,up) - c_(j,up) c_(i,dn)) / sqrt(2),
    the annihilator of the singlet pair (c+_(i,up) c+_(j,dn) - c+_(i,dn) c+_(j,up)) / sqrt(2)."""
    n, N = cl.n, cl.N
    nu = N // 2
    m_up = _sector(n, N - 1, nu - 1)    # after removing an up electron
    m_dn = _sector(n, N - 1, nu)        # after removing a down electron
    two = _sector(n, N - 2, nu - 1)

    def pair(i, j):
        x = annihilate(m_up, annihilate(cl, psi, i, 0, m_up), j, 1, two)
        y = annihilate(m_dn, annihilate(cl, psi, i, 1, m_dn), j, 0, two)
        return (x - y) / np.sqrt(2.0)

    return float(pair(a, b) @ pair(c, d))


def hopping_correlation(cl, psi, i, j):
    """<psi| sum_s c+_(i,s) c_(j,s) |psi>, i != j."""
    total = 0.0
    for spin in (0, 1):
        nu = cl.N // 2
        m = _sector(cl.n, cl.N - 1, nu - 1 if spin == 0 else nu)
        total += float(annihilate(cl, psi, i, spin, m) @ annihilate(cl, psi, j, spin, m))
    return total
