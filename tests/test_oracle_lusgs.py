"""CPU checks of the oracle's coloured LU-SGS (bcsr_parallel_lusgs,
sparse_bcsr_linear_module.F90:1438-1502): with one colour it is the block-Jacobi
bcsr_diag bit for bit, and with a proper colouring it is the exact inverse of
(I + L)(D + U) for the colour-ordered splitting (the forward sweep of the reference
subtracts the lower-colour blocks without a diagonal solve; the backward sweep ends
with the diagonal block's LU solve)."""
import numpy as np


def _dense(A):
    bs = A.blc_size
    M = np.zeros((A.m * bs, A.m * bs))
    for i in range(A.m):
        for j in range(A.row[i] - 1, A.row[i + 1] - 1):
            c = A.col[j] - 1
            M[bs * i:bs * i + bs, bs * c:bs * c + bs] = A.v[j].T
    return M


def test_lusgs_one_colour_is_block_jacobi(oracle_lib):
    from oracle.oracle import OracleBcsr
    from subfv_b200.bcsr import grid_matrix
    A = grid_matrix(4, 3, 3, bs=5, stencil=7, seed=21)
    o = OracleBcsr(A)
    b = np.random.default_rng(1).normal(size=o.n)
    np.testing.assert_array_equal(o.parallel_lusgs(b, 1, np.ones(A.m, np.int32)), o.diag(b))


def test_lusgs_inverts_the_colour_splitting(oracle_lib):
    from oracle.oracle import OracleBcsr
    from subfv_b200.bcsr import grid_matrix, greedy_colors
    A = grid_matrix(4, 4, 2, bs=3, stencil=7, seed=22)
    ncs, color = greedy_colors(A)
    o = OracleBcsr(A)
    M = _dense(A)
    bs = A.blc_size
    cb = np.repeat(color, bs)
    lower = M * (cb[:, None] > cb[None, :])  # row colour above the column's: the forward sweep's blocks
    upper = M * (cb[:, None] < cb[None, :])
    D = M * (cb[:, None] == cb[None, :]) * np.kron(np.eye(A.m), np.ones((bs, bs)))
    P = (np.eye(M.shape[0]) + lower) @ (D + upper)
    b = np.random.default_rng(2).normal(size=o.n)
    x = o.parallel_lusgs(b, ncs, color)
    np.testing.assert_allclose(P @ x, b, rtol=1e-10, atol=1e-10 * np.abs(b).max())


def test_oracle_pcgm_solves_spd(oracle_lib):
    """The oracle's bcsr_pcgm restatement reaches the exact solution of an SPD system."""
    import sys
    sys.path.insert(0, __file__.rsplit("/", 1)[0])
    from test_bcsr_gpu import _spd
    from oracle.oracle import OracleBcsr
    A = _spd(4, 3, 3, 3, 11)
    o = OracleBcsr(A)
    b = np.random.default_rng(3).normal(size=o.n)
    x, it, st, res = o.pcgm(b, 1e-11 * np.linalg.norm(b))
    assert st == 0 and 0 < it < o.n
    np.testing.assert_allclose(_dense(A) @ x, b, rtol=0, atol=1e-9 * np.abs(b).max())
