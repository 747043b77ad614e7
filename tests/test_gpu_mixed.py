"""Split-precision (int8 digit) tensor-core products against exact products.

Each operand element is cut into six 7-bit digits after a power-of-two scaling
of its row (A) or column (B); the 21 leading digit products are exact in int32.
The error of entry (i, j) is therefore bounded by a small multiple of
2^-40 K max_k|a_ik| max_k|b_kj|, which the tests check entry by entry."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx():
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    return rb.Rayleigh(rb.Config(n_r=16, l_max=15, n_theta=24))


@pytest.fixture(scope="module")
def ctx():
    return _ctx()


def _check(ctx, a, b):
    c = ctx.mixed_gemm(a, b)
    exact = (a.astype(np.longdouble) @ b.astype(np.longdouble)).astype(np.float64)
    k = a.shape[1]
    bound = 2.0**-36 * k * np.abs(a).max(axis=1)[:, None] * np.abs(b).max(axis=0)[None, :]
    err = np.abs(c - exact)
    assert np.all(err <= bound + 1e-300), (err / np.maximum(bound, 1e-300)).max()
    scale = np.abs(exact).max()
    if scale == 0.0 or not np.isfinite(scale):
        return 0.0
    return float(np.linalg.norm((c - exact) / scale) / np.linalg.norm(exact / scale))


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 64, 32), (130, 65, 33), (257, 200, 384), (77, 513, 100)])
def test_random_shapes(ctx, m, n, k):
    rng = np.random.Generator(np.random.PCG64(m * 1000003 + n * 1009 + k))
    a = rng.standard_normal((m, k))
    b = rng.standard_normal((k, n))
    rel = _check(ctx, a, b)
    assert rel < 1e-10, rel


def test_wide_dynamic_range(ctx):
    # rows and columns spanning 2^-300 .. 2^300, zero rows and columns, and
    # entries of mixed sign inside a row: the per-row scaling keeps each exact
    rng = np.random.Generator(np.random.PCG64(5))
    m, n, k = 150, 90, 70
    a = rng.standard_normal((m, k)) * np.ldexp(1.0, rng.integers(-300, 300, m))[:, None]
    b = rng.standard_normal((k, n)) * np.ldexp(1.0, rng.integers(-300, 300, n))[None, :]
    a[3] = 0.0
    b[:, 7] = 0.0
    c = ctx.mixed_gemm(a, b)
    assert np.all(c[3] == 0.0) and np.all(c[:, 7] == 0.0)
    _check(ctx, a, b)


def test_two_calls_agree(ctx):
    rng = np.random.Generator(np.random.PCG64(9))
    a = rng.standard_normal((200, 96))
    b = rng.standard_normal((96, 130))
    assert np.array_equal(ctx.mixed_gemm(a, b), ctx.mixed_gemm(a, b))


def test_legendre_table_product(ctx):
    # the products the mixed Legendre transforms make: a P_l^m table (K = number
    # of l of one parity) times spectral coefficients
    import oracle as O
    lmax, nth = 127, 192
    h = O.Horizontal(lmax, nth)
    rng = np.random.Generator(np.random.PCG64(3))
    for m in (0, 1, 40, 127):
        p = np.asarray(h.p_even[m], dtype=np.float64)        # [nl][nth/2]
        s = rng.standard_normal((p.shape[0], 96))
        rel = _check(ctx, np.ascontiguousarray(p.T), s)
        assert rel < 1e-10, (m, rel)
