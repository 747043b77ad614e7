"""Batched per-l implicit solves on the device (LU_Decompose_full / LU_Solve_full,
Linear_Solve.F90:1028-1036, 1088-1110) through the C ABI (ra_lu_*).

The batched-solve workload: for l = 0..1023 the linked W-P-T operator
(3 N_r x 3 N_r; the reference couples T into W for the Boussinesq set) and
the Z operator (N_r x N_r) of the Crank-Nicolson step at Ekman 1e-4,
dt 1e-5, N_r in {128, 256}, with 8 complex (16 real) Gaussian right-hand
sides per l, solved as one launch by FP64 block substitution and by FP32
substitution with FP64-residual iterative refinement.

Parity criterion.  The W-P-T operators have condition numbers of 1e8 - 1e10,
so two correct LU solves of a random right-hand side may differ by up to
cond x 2^-53 in the solution; what a correct solve guarantees is a backward
error at the rounding level.  Each column is checked with LAPACK's own test
ratio (xGET02: ||b - A x||_1 / (||A||_1 ||x||_1 eps) < 30), and the
difference to SciPy's LU solve is bounded by cond_1(A) x 2^-53 x 64 on a
sample of l (and is printed)."""
import numpy as np
import pytest
import scipy.linalg as sla

import rayleigh_b200 as rb

pytestmark = pytest.mark.gpu
EPS = 2.0 ** -53


def _get02(M_cm, x, b):
    """LAPACK xGET02 ratio per column: ||b - A x||_1 / (||A||_1 ||x||_1 eps), batched over l;
    M_cm[l][j][i] = A_l[i][j] (column-major storage), x and b as [l][column][i]."""
    r = b - np.matmul(x, M_cm)
    an = np.abs(M_cm).sum(axis=2).max(axis=1)        # ||A||_1 per l (largest column sum)
    return np.abs(r).sum(axis=2) / (an[:, None] * np.abs(x).sum(axis=2) * EPS)


def _systems(nr, lmax=1023):
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    cfg = rb.Config(n_r=nr, l_max=lmax, dt=1e-5, ekman=1e-4, rayleigh=1e5)
    wpt = rb.build_matrices(cfg, 0, 0, lmax + 1)       # [l][col][row]
    z = rb.build_matrices(cfg, 1, 1, lmax)            # l = 1 .. l_max (Z is not solved at l = 0)
    return wpt, z


@pytest.mark.parametrize("nr", [128, 256])
def test_batched_solves_workload(nr):
    rng = np.random.Generator(np.random.PCG64(0x5241594C))
    wpt_cm, z_cm = _systems(nr)
    report = {}
    for name, mats_cm in (("W-P-T", wpt_cm), ("Z", z_cm)):
        count, n, _ = mats_cm.shape
        b = rng.standard_normal((count, 16, n))
        with rb.BatchedLU(n, count) as lu:
            t_fact = lu.factor(mats_cm)
            x64, _, t64 = lu.solve(b, rb.SOLVE_FP64)
            xir, its, tir = lu.solve(b, rb.SOLVE_REFINE)
        for form, x in (("fp64", x64), ("refine", xir)):
            ratio = _get02(mats_cm, x, b)
            assert ratio.max() < 30.0, (name, form, float(ratio.max()))
        # difference to SciPy's LU on a sample of l, bounded by the conditioning
        worst = 0.0
        for l in sorted({0, 1, 2, 3, 10, 100, count // 2, count - 1}):
            A = mats_cm[l].T
            ref = sla.lu_solve(sla.lu_factor(A), b[l].T).T
            cond = np.linalg.cond(A, 1)
            for x in (x64, xir):
                d = np.abs(x[l] - ref).max() / np.abs(ref).max()
                worst = max(worst, d)
                assert d <= max(64 * cond * EPS, 1e-13), (name, l, d, cond)
        assert its.max() < 30, its.max()          # converged before the iteration cap
        report[name] = dict(factor_ms=round(t_fact, 2), fp64_solve_ms=round(t64, 3), refine_ms=round(tir, 3),
                            refine_iters=np.bincount(its.ravel()).tolist(), max_diff_to_scipy=f"{worst:.1e}")
    print(f"N_r={nr}", report)


def test_singular_matrix_reported():
    """A zero row in one per-l matrix: RA_ERR_SINGULAR names that matrix; the
    others were not harmed (a refactor after fixing it succeeds)."""
    wpt_cm, _ = _systems(24, lmax=15)
    bad = wpt_cm.copy()
    bad[5][:, 30] = 0.0           # row 30 of A_5 (column-major storage: [col][row])
    count, n, _ = bad.shape
    with rb.BatchedLU(n, count) as lu:
        with pytest.raises(rb.RayleighError) as ei:
            lu.factor(bad)
        assert ei.value.code == rb.RA_ERR_SINGULAR and "matrix 5" in str(ei.value)
        lu.factor(wpt_cm)
        b = np.ones((count, 2, n))
        x, _, _ = lu.solve(b)
        assert np.all(np.isfinite(x))


def test_nonfinite_matrix_refused():
    wpt_cm, _ = _systems(24, lmax=7)
    bad = wpt_cm.copy()
    bad[3][7, 7] = np.nan
    count, n, _ = bad.shape
    with rb.BatchedLU(n, count) as lu:
        with pytest.raises(rb.RayleighError) as ei:
            lu.factor(bad)
        assert ei.value.code == rb.RA_ERR_NONFINITE
