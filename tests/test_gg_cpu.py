"""The synthetic grouped block-GEMM batch (grand_sql_tj_b200/gg.py): seeded,
inside its stated ranges, every operand window inside the pool, and the
numpy reference consistent with a direct evaluation of one term."""
import numpy as np

from grand_sql_tj_b200 import gg


def test_batch_is_seeded_and_in_range():
    a = gg.make_batch(n_cells=40, seed=5, pool_len=1 << 20)
    b = gg.make_batch(n_cells=40, seed=5, pool_len=1 << 20)
    assert np.array_equal(a.pool, b.pool)
    assert [(c.M, c.N, c.t_begin, c.t_end) for c in a.cells] == [(c.M, c.N, c.t_begin, c.t_end) for c in b.cells]
    for c in a.cells:
        assert 8 <= c.M <= 1024 and 8 <= c.N <= 1024 and 4 <= c.t_end - c.t_begin <= 16
        for t in range(c.t_begin, c.t_end):
            x = a.terms[t]
            assert 8 <= x.K <= 1024 and -1.0 <= x.coef <= 1.0
            lrows, lcols = (x.K, c.M) if x.l_trans else (c.M, x.K)
            rrows, rcols = (c.N, x.K) if x.r_trans else (x.K, c.N)
            assert x.l_ld == lrows and x.r_ld == rrows
            assert x.l_off + lrows * lcols <= a.pool.size and x.r_off + rrows * rcols <= a.pool.size
    assert a.out_len == sum(c.M * c.N for c in a.cells)
    assert abs(a.flops - sum(2.0 * c.M * c.N * a.terms[t].K for c in a.cells
                             for t in range(c.t_begin, c.t_end))) < 1.0


def test_reference_of_one_term():
    b = gg.make_batch(n_cells=3, dmax=64, seed=9, pool_len=1 << 16)
    c = b.cells[0]
    ref = gg.reference(b, [0])[0]
    y = np.zeros((c.M, c.N))
    for t in range(c.t_begin, c.t_end):
        x = b.terms[t]
        for i in range(c.M):
            for j in range(c.N):
                s = 0.0
                for k in range(x.K):
                    lv = b.pool[x.l_off + i * x.l_ld + k] if x.l_trans else b.pool[x.l_off + k * x.l_ld + i]
                    rv = b.pool[x.r_off + k * x.r_ld + j] if x.r_trans else b.pool[x.r_off + j * x.r_ld + k]
                    s += lv * rv
                y[i, j] += x.coef * s
    assert np.max(np.abs(ref - y)) <= 1e-12 * max(1.0, np.max(np.abs(y)))
