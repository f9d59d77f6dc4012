"""Truncation (den_mat.f90) and correlator contractions (measure.f90) on the
B200 against the oracle.

Truncation: identical kept count, truncation error and entropies to 1e-10
against LAPACK dsyev in the oracle (the device eigenvalues come from
Householder tridiagonalisation and Sturm multisection), kept eigenvectors
orthonormal to 1e-12 and spanning the same space: projector difference
<= max(1e-8, 1e-15 / gap), gap = the sector's distance between its smallest
kept and largest dropped eigenvalue (a subspace is determined by FP64 data
only to about eps ||rho|| / gap, for any backward-stable solver;
eigenvector signs and degenerate bases are free).  Correlators: relative
1e-12.
"""
import numpy as np
import pytest

from grand_sql_tj_b200 import synth
from grand_sql_tj_b200.structs import block_transfer_trans
from tests.test_cor_cpu import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(product_lib):
    from grand_sql_tj_b200.lib import Context
    c = Context(0)
    yield c
    c.close()


def _sector_gaps(psi, side, blk):
    """Per kept sector: gap between its smallest kept and largest dropped eigenvalue of rho."""
    rho = {}
    for k, sec in enumerate(psi.sectors):
        o = int(psi.offsets[k])
        m = psi.data[o:o + sec.sys_dim * sec.env_dim].reshape(sec.env_dim, sec.sys_dim).T
        key = (sec.sys_num_up, sec.sys_num_down) if side == 0 else (sec.env_num_up, sec.env_num_down)
        r = m @ m.T if side == 0 else m.T @ m
        rho[key] = rho.get(key, 0) + r
    gaps = {}
    for s in blk.subs:
        key = (s.num_up, s.num_down)
        w = np.sort(np.linalg.eigvalsh(rho[key]))[::-1]
        n = s.mat.shape[1]
        gaps[key] = w[n - 1] - w[n] if n < len(w) else np.inf
    return gaps


def _projectors(blk):
    out = {}
    for s in blk.subs:
        q = s.mat
        out[(s.num_up, s.num_down)] = q @ q.T
    return out


@pytest.mark.parametrize("wl,side,kmin,kmax", [("small", 0, 6, 12), ("small", 1, 4, 8),
                                               ("small_gc", 0, 10, 20), ("cyl4", 0, 20, 40),
                                               ("cyl4", 1, 8, 64), ("ladder16_m256", 0, 96, 128)])
def test_truncation(ctx, oracle_lib, wl, side, kmin, kmax):
    from oracle import oracle
    sb = synth.workload(wl, seed=5)
    _, _, psi = oracle.lanczos(sb, 1e-8)          # a ground-state-like wavefunction
    r0, t0, _ = oracle.truncation(psi, side, kmin, kmax, 1e-12)
    r1, t1 = ctx.truncation(psi, side, kmin, kmax, 1e-12)
    assert r1.num_state == r0.num_state
    assert abs(r1.trunc_err - r0.trunc_err) <= 1e-10
    for k in ("entropy1", "entropy2", "entropys"):
        assert abs(getattr(r1, k) - getattr(r0, k)) <= 1e-10, k
    for sb1 in t1.subs:
        q = sb1.mat
        assert np.max(np.abs(q.T @ q - np.eye(q.shape[1]))) <= 1e-12
    p0, p1 = _projectors(t0), _projectors(t1)
    assert p0.keys() == p1.keys()
    gaps = _sector_gaps(psi, side, t0)
    for k in p0:
        tol = max(1e-8, 1e-15 / max(gaps[k], 1e-300))
        assert np.max(np.abs(p0[k] - p1[k])) <= tol, (k, gaps[k])
    # the two-call protocol returns the same result when called again
    r2, t2 = ctx.truncation(psi, side, kmin, kmax, 1e-12)
    assert r2.num_state == r1.num_state and all(np.array_equal(a.mat, b.mat) for a, b in zip(t1.subs, t2.subs))


@pytest.mark.parametrize("wl,kmin,kmax", [("cyl4x24_m2000", 3000, 6000), ("cyl6x24_m6000", 2000, 3000)])
def test_truncation_cluster_sizes(ctx, oracle_lib, wl, kmin, kmax):
    """Sectors of 320 states and more go to the cluster paths: the reduction
    by 16 CTAs (from step 0 in shared memory at 359-481 states; moving into
    shared memory part-way at 900-1524 states) and the cluster
    orthonormalisation of kept blocks with k^2 d >= 3e7 (full sectors of
    359-481 states; up to 605 of 1524).  The synthetic wavefunctions of the
    two headline superblocks, against dsyev in the oracle, with the bounds of
    test_truncation."""
    from oracle import oracle
    psi = synth.workload(wl).wave
    r0, t0, _ = oracle.truncation(psi, 0, kmin, kmax, 1e-12)
    r1, t1 = ctx.truncation(psi, 0, kmin, kmax, 1e-12)
    assert max(s.mat.shape[0] for s in t1.subs) >= 359
    assert r1.num_state == r0.num_state
    assert abs(r1.trunc_err - r0.trunc_err) <= 1e-10
    for k in ("entropy1", "entropy2", "entropys"):
        assert abs(getattr(r1, k) - getattr(r0, k)) <= 1e-10, k
    for sb1 in t1.subs:
        q = sb1.mat
        assert np.max(np.abs(q.T @ q - np.eye(q.shape[1]))) <= 1e-12
    p0, p1 = _projectors(t0), _projectors(t1)
    assert p0.keys() == p1.keys()
    gaps = _sector_gaps(psi, 0, t0)
    for k in p0:
        tol = max(1e-8, 1e-15 / max(gaps[k], 1e-300))
        assert np.max(np.abs(p0[k] - p1[k])) <= tol, (k, gaps[k])


def test_truncation_rank_deficient(ctx, oracle_lib):
    """Density matrices with large null spaces -- the truncations of an
    untruncated 2x6 ladder run, system block much longer than the
    environment -- with every state kept: the columns are orthonormal, each
    spans an invariant subspace of its rho (residual <= 1e-13 ||rho||), and
    the spectrum summaries equal the oracle's (DSYEV)."""
    from grand_sql_tj_b200.lattice import Geometry
    from grand_sql_tj_b200.sweep import Dmrg, DmrgParams
    from oracle.oracle import OracleBackend

    class Rec:
        def __init__(self):
            self.o, self.waves = OracleBackend(), []

        def __getattr__(self, k):
            return getattr(self.o, k)

        def truncation(self, wave, side, kmin, kmax, err):
            self.waves.append((wave.copy(), side))
            return self.o.truncation(wave, side, kmin, kmax, err)

    geo = Geometry(6, 2, t=1.0, J=1.0 / 3.0, esite=-0.1, up_bias=1)
    be = Rec()
    d = Dmrg(geo, be, DmrgParams(n_elec=10, kept_min=10 ** 5, kept_max=10 ** 6, lanzero=1e-12, lanzero_warm=1e-12,
                                 seed=3))
    d.warm_up()
    d.left_to_right(5, 10, restart=False)
    from oracle import oracle
    checked = 0
    for w, side in be.waves[-3:]:
        r0, _, _ = oracle.truncation(w, side, 10 ** 5, 10 ** 6, 1e-18)
        r1, t1 = ctx.truncation(w, side, 10 ** 5, 10 ** 6, 1e-18)
        assert r1.num_state == r0.num_state
        for k in ("trunc_err", "entropy1", "entropy2", "entropys"):
            assert abs(getattr(r1, k) - getattr(r0, k)) <= 1e-10, k
        nrm2 = float(w.data[:w.dim] @ w.data[:w.dim])
        for sub in t1.subs:
            q = sub.mat
            assert np.max(np.abs(q.T @ q - np.eye(q.shape[1]))) <= 1e-12
            assert side == 0
            i = next(i for i, sc in enumerate(w.sectors) if (sc.sys_num_up, sc.sys_num_down) == (sub.num_up, sub.num_down))
            x = w.sector(i)
            rho = (x @ x.T) / nrm2
            lam = np.einsum("ij,ij->j", q, rho @ q)
            res = np.max(np.abs(rho @ q - q * lam))
            assert res <= 1e-13 * max(np.max(np.abs(rho)), 1e-300), (sub.num_up, sub.num_down, res)
            checked += q.shape[1]
    assert checked > 500


@pytest.mark.parametrize("wl", ["small", "small_gc", "cyl4"])
def test_correlators(ctx, oracle_lib, wl):
    from oracle import oracle
    sb = synth.workload(wl, seed=8)
    site = lambda k: oracle.site_operator(k, sb.lat.up_bias)
    for name, a, b, flag in cases(sb, site):
        ref = oracle.correlator(name, a, b, sb.sys_bs, sb.env_bs, sb.wave, flag)
        got = ctx.correlator(name, a, b, sb.sys_bs, sb.env_bs, sb.wave, flag)
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (name, flag, got, ref)
