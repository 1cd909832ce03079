"""BCSR SpMV, block-Jacobi and restarted GMRES on the GPU against the oracle restatement
of src/linear_algebra/sparse_bcsr_linear_module.F90.

SpMV and the block-Jacobi application are bit-identical (same per-block order, no FMA).
GMRES sums its dot products and norms by a fixed tree instead of left to right, so its
iterates agree to round-off: the solution within 1e-9 relative of the oracle's, the
first Hessenberg within 1e-10, the same restart count and convergence flag."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    "b5_27pt": dict(nx=6, ny=5, nz=4, bs=5, stencil=27, seed=1),
    "b5_7pt_periodic": dict(nx=5, ny=4, nz=3, bs=5, stencil=7, seed=2, periodic=True),
    "b4_27pt": dict(nx=4, ny=4, nz=3, bs=4, stencil=27, seed=3),
    "b3_7pt": dict(nx=6, ny=3, nz=2, bs=3, stencil=7, seed=4),
    "b1_7pt": dict(nx=9, ny=7, nz=3, bs=1, stencil=7, seed=5),
}


def _mat(name):
    from subfv_b200.bcsr import grid_matrix
    c = dict(CASES[name])
    return grid_matrix(c.pop("nx"), c.pop("ny"), c.pop("nz"), **c)


def _dense(A):
    bs = A.blc_size
    M = np.zeros((A.m * bs, A.m * bs))
    for i in range(A.m):
        for j in range(A.row[i] - 1, A.row[i + 1] - 1):
            c = A.col[j] - 1
            M[bs * i:bs * i + bs, bs * c:bs * c + bs] = A.v[j].T
    return M


@pytest.mark.parametrize("case", list(CASES))
def test_matmul_and_diag_bit_exact(native, oracle_lib, cuda_ok, case):
    from oracle.oracle import OracleBcsr
    from subfv_b200.bcsr import DeviceBcsr
    A = _mat(case)
    d, o = DeviceBcsr(A), OracleBcsr(A)
    x = np.random.default_rng(7).normal(size=d.n)
    np.testing.assert_array_equal(d.matmul(x), o.matmul(x))
    np.testing.assert_allclose(d.matmul(x), _dense(A) @ x, rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(d.diag(x), o.diag(x))


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("precond", [True, False])
def test_gmres_matches_oracle(native, oracle_lib, cuda_ok, case, precond):
    from oracle.oracle import OracleBcsr
    from subfv_b200.bcsr import DeviceBcsr
    A = _mat(case)
    d, o = DeviceBcsr(A), OracleBcsr(A)
    b = np.random.default_rng(8).normal(size=d.n)
    tol = 1e-8 * np.linalg.norm(b)
    m = 30 if d.n > 40 else 8
    x, conv, it, rho, H = d.gmres(b, tol, m, precond=precond, want_h=True)
    xo, convo, ito, rhoo, Ho = o.gmres(b, tol, m, precond=precond)
    assert conv == convo and it == ito
    assert np.abs(x - xo).max() <= 1e-9 * np.abs(xo).max()
    # upper Hessenberg part only (entries below the subdiagonal are never defined;
    # H(m+1, m) is stored column-major: H[j, i] = H(i+1, j+1)), and only the columns
    # built before the Krylov space reaches round-off: these matrices converge within a
    # few columns, after which the Arnoldi vectors are rounding noise of either order.
    i, j = np.meshgrid(np.arange(m + 1), np.arange(m), indexing="xy")
    hess = (i <= j + 1) & (j < min(m, 6))
    np.testing.assert_allclose(H[hess], Ho[hess], rtol=1e-9, atol=1e-9 * np.abs(Ho).max())
    if conv:
        assert np.linalg.norm(b - _dense(A) @ x) < 1.5 * tol


def test_gmres_not_converged_is_reported(native, cuda_ok):
    """A matrix block-Jacobi cannot fix within 40 restarts of GMRES(2): conv = .false."""
    from subfv_b200.bcsr import DeviceBcsr, grid_matrix
    A = grid_matrix(6, 6, 4, bs=5, stencil=27, seed=9, diag_shift=0.05)
    d = DeviceBcsr(A)
    b = np.random.default_rng(10).normal(size=d.n)
    x, conv, it, rho = d.gmres(b, 1e-14 * np.linalg.norm(b), 2, precond=True)
    assert not conv and it == 40


def test_iterative_refinement_fp32_matrix(native, cuda_ok):
    from subfv_b200.bcsr import DeviceBcsr, grid_matrix
    A = grid_matrix(8, 8, 6, bs=5, stencil=27, seed=11)
    d = DeviceBcsr(A)
    b = np.random.default_rng(12).normal(size=d.n)
    x, conv, outer, rho = d.gmres_refine(b, rel_tol=1e-8, m=30)
    assert conv and outer >= 1
    assert np.linalg.norm(b - _dense(A) @ x) < 1e-8 * np.linalg.norm(b)
    x64, conv64, _, _ = d.gmres(b, 1e-8 * np.linalg.norm(b), 30)
    assert np.abs(x - x64).max() <= 1e-6 * np.abs(x64).max()


@pytest.mark.parametrize("case", list(CASES))
def test_parallel_lusgs_bit_exact(native, oracle_lib, cuda_ok, case):
    """bcsr_parallel_lusgs (:1438-1502) with a greedy colouring: bit-identical."""
    from oracle.oracle import OracleBcsr
    from subfv_b200.bcsr import DeviceBcsr, greedy_colors
    A = _mat(case)
    ncs, color = greedy_colors(A)
    d, o = DeviceBcsr(A), OracleBcsr(A)
    d.set_colors(ncs, color)
    b = np.random.default_rng(9).normal(size=d.n)
    np.testing.assert_array_equal(d.parallel_lusgs(b), o.parallel_lusgs(b, ncs, color))


@pytest.mark.parametrize("case", list(CASES))
def test_gmres_parallel_lusgs_matches_oracle(native, oracle_lib, cuda_ok, case):
    """bcsr_gmres_parallel_lusgs (:885-993): same restarts and convergence flag, solution
    within 1e-9 of the oracle's (dot products by a fixed tree), true residual below tol."""
    from oracle.oracle import OracleBcsr
    from subfv_b200.bcsr import DeviceBcsr, greedy_colors
    A = _mat(case)
    ncs, color = greedy_colors(A)
    d, o = DeviceBcsr(A), OracleBcsr(A)
    d.set_colors(ncs, color)
    b = np.random.default_rng(10).normal(size=d.n)
    tol = 1e-8 * np.linalg.norm(b)
    m = 30 if d.n > 40 else 8
    x, conv, it, rho = d.gmres_lusgs(b, tol, m)
    xo, convo, ito, rhoo = o.gmres_lusgs(b, tol, m, ncs, color)
    assert conv == convo and it == ito
    assert np.abs(x - xo).max() <= 1e-9 * np.abs(xo).max()
    if conv:
        assert np.linalg.norm(b - _dense(A) @ x) < 1.5 * tol


def _spd(nx, ny, nz, bs, seed):
    """A block-symmetric, block-diagonally dominant (SPD) matrix on the 7-point pattern."""
    from subfv_b200.bcsr import BcsrMatrix, grid_matrix
    A = grid_matrix(nx, ny, nz, bs=bs, stencil=7, seed=seed)
    rng = np.random.default_rng(seed + 100)
    row, col = A.row - 1, A.col - 1
    v = np.zeros_like(A.v)
    pos = {}
    for i in range(A.m):
        for j in range(row[i], row[i + 1]):
            pos[(i, col[j])] = j
    for (i, c), j in pos.items():
        if c > i:
            B = rng.uniform(-0.2, 0.2, (bs, bs))
            v[j] = B  # v[j, c, r]: the Fortran block is v[j].T
            v[pos[(c, i)]] = B.T
    for i in range(A.m):
        S = rng.uniform(-0.3, 0.3, (bs, bs))
        v[pos[(i, i)]] = S @ S.T + (2.0 * bs) * np.eye(bs)
    return BcsrMatrix(A.m, bs, A.row, A.col, v)


@pytest.mark.parametrize("bs", [3, 5])
def test_pcgm_matches_oracle(native, oracle_lib, cuda_ok, bs):
    """bcsr_pcgm (:1110-1169) on an SPD matrix from a nonzero initial guess: the same
    iteration count as the oracle, the solution within 1e-9 of it, residual below tol."""
    from oracle.oracle import OracleBcsr
    from subfv_b200.bcsr import DeviceBcsr
    A = _spd(5, 4, 3, bs, 31)
    d, o = DeviceBcsr(A), OracleBcsr(A)
    rng = np.random.default_rng(32)
    b, x0 = rng.normal(size=d.n), rng.normal(size=d.n)
    tol = 1e-9 * np.linalg.norm(b)
    x, it, st, res = d.pcgm(b, tol, x0)
    xo, ito, sto, reso = o.pcgm(b, tol, x0)
    assert st == sto == 0 and it == ito
    assert np.abs(x - xo).max() <= 1e-9 * np.abs(xo).max()
    assert np.linalg.norm(b - _dense(A) @ x) <= 1.01 * tol


def test_zero_right_hand_side_is_solved_by_zero(native, cuda_ok):
    """b = 0: every Krylov entry returns x = 0, converged, without an Arnoldi cycle, also
    at tol = 0 (a relative tolerance on b = 0), where the reference's recurrences would
    divide the zero residual by its zero norm; PCG from x0 = 0 likewise."""
    from subfv_b200.bcsr import DeviceBcsr, greedy_colors, grid_matrix
    A = grid_matrix(4, 4, 3, bs=5, stencil=27, seed=13)
    d = DeviceBcsr(A)
    d.set_colors(*greedy_colors(A))
    b = np.zeros(d.n)
    for tol in (0.0, 1e-10):
        for pc in (True, False):
            x, conv, it, rho = d.gmres(b, tol, 30, precond=pc)
            assert conv and it == 0 and rho == 0.0 and not x.any(), (tol, pc)
        x, conv, it, rho = d.gmres_lusgs(b, tol)
        assert conv and it == 0 and not x.any()
    x, conv, outer, rho = d.gmres_refine(b, rel_tol=1e-8)
    assert conv and not x.any() and np.isfinite(rho)
    S = DeviceBcsr(_spd(3, 3, 2, 5, 41))
    for tol in (0.0, 1e-10):
        x, it, st, res = S.pcgm(np.zeros(S.n), tol)
        assert st == 0 and it == 0 and res == 0.0 and not x.any()
