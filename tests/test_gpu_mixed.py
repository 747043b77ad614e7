"""Split-precision (int8 digit) tensor-core products against exact products.

Each operand element is rounded to a 39-bit integer after a power-of-two
scaling of its row (A) or column (B) and cut into five balanced base-256 digits;
the 15 leading digit products are exact in int32.  The error of entry (i, j) is
therefore bounded by 2^-33 K max_k|a_ik| max_k|b_kj|, which the tests check entry
by entry (measured errors are far below it)."""
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
    # per term: digit truncation <= 2^-37 and dropped digit products <= 2^-34 of max|a_i.| max|b_.j|
    bound = 2.0**-33 * k * np.abs(a).max(axis=1)[:, None] * np.abs(b).max(axis=0)[None, :]
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


# ---------------------------------------------------------------------------
# The mixed-precision step (RA_PREC_MIXED) against the oracle and the FP64 step
# ---------------------------------------------------------------------------
MIXED_TOL = 1e-9


def _fields(wpt, z, nr):
    return {"W": wpt[:, :, :nr], "P": wpt[:, :, nr:2 * nr], "T": wpt[:, :, 2 * nr:], "Z": z}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _run(cfg, precision, wpt, z, steps):
    import rayleigh_b200 as rb
    g = rb.Rayleigh(rb.Config(**dict(cfg, precision=precision, use_graph=True)))
    g.put_state(wpt, z, None, iteration=1)
    g.step(steps)
    w, zz, _ = g.get_state()
    g.close()
    return w, zz


@pytest.mark.parametrize("cfg,steps", [
    (dict(n_r=24, l_max=15, dt=2e-4), 20),
    (dict(n_r=48, l_max=63, dt=1e-4), 10),
])
def test_mixed_step_vs_oracle(cfg, steps):
    import oracle as O
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    oc = O.Config(**{k: v for k, v in cfg.items() if k in O.Config.__dataclass_fields__})
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=min(20, oc.l_max))
    o.init_state(wpt, z)
    for _ in range(steps):
        o.step()
    w, zz = _run(cfg, rb.PREC_MIXED, wpt, z, steps)
    ref = _fields(o.rhs_wpt, o.rhs_z, oc.n_r)
    errs = {k: _rel(v, ref[k]) for k, v in _fields(w, zz, oc.n_r).items()}
    print(cfg, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < MIXED_TOL, errs


def test_mixed_step_vs_fp64_large():
    # l_max = 255: the GPU FP64 form against the GPU mixed form, 5 steps
    import oracle as O
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    cfg = dict(n_r=64, l_max=255, dt=1e-5, ekman=1e-4, rayleigh=1e7)
    oc = O.Config(**{k: v for k, v in cfg.items() if k in O.Config.__dataclass_fields__})
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=20)
    w64, z64 = _run(cfg, rb.PREC_FP64, wpt, z, 5)
    wmx, zmx = _run(cfg, rb.PREC_MIXED, wpt, z, 5)
    ref = _fields(w64, z64, oc.n_r)
    errs = {k: _rel(v, ref[k]) for k, v in _fields(wmx, zmx, oc.n_r).items()}
    print(cfg, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < MIXED_TOL, errs


@pytest.mark.parametrize("lmax", [255, 511])
def test_mixed_stages_per_lmax(lmax):
    """The split-precision form stage by stage against the FP64 oracle at
    l_max = 255 and 511 (N_r = 8), errors printed per l_max: the inverse and
    forward Legendre transforms (split products), the physical-space stage they
    feed and the implicit solve (split product).  The solution after the step
    is held to 1e-9 (relative L2 per field); each intermediate buffer to 1e-7
    of its own norm: the nonlinear terms are products of the velocity fields,
    which are small beside T, so their relative error is larger than that of
    the transformed buffer they come from."""
    from test_gpu_parity import _stage_compare
    errs = _stage_compare(dict(n_r=8, l_max=lmax, dt=1e-6, rayleigh=1e5, ekman=1e-3, precision=1), steps_before=1)
    print(f"l_max {lmax}:", {k: f"{v:.2e}" for k, v in errs.items()})
    state = {k: v for k, v in errs.items() if k.startswith("sol_")}
    assert max(state.values()) <= MIXED_TOL, errs
    bad = {k: v for k, v in errs.items() if v > 1e-7}
    assert not bad, errs
