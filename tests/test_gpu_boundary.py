"""The drop-in boundary entry points for a Fortran driver that owns its own
matrices, boundary values and rank-distributed state (through the C ABI):
ra_load_matrices + ra_factor (Load_Linear_Coefficients / LU_Decompose_Matrices,
Sphere_Linear_Terms.F90:196-1100, Linear_Solve.F90:459-539), ra_set_bc_mask
(bc_values, BoundaryConditions.F90:364-531, Apply_Boundary_Mask
Linear_Solve.F90:401-418), ra_put/get_state_modes (a rank's (l, m) list,
Load_Balance.F90:311-470), and the error codes RA_ERR_SINGULAR and
RA_ERR_NONFINITE raised by faults injected on the host."""
import numpy as np
import pytest

import oracle as O
import rayleigh_b200 as rb
from layouts import rel_err

pytestmark = pytest.mark.gpu
CFG = dict(n_r=24, l_max=15, dt=2e-4, rayleigh=1e5, ekman=1e-3)


def _ctx(cfg, **kw):
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    return rb.Rayleigh(rb.Config(**dict(cfg, **kw)))


def _start(cfg, amp=1e-2):
    oc = O.Config(**cfg)
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=amp, lmax_pert=10)
    o.init_state(wpt, z)
    return oc, o, wpt, z


def _errs(g, o, nr):
    wg, zg, _ = g.get_state()
    return {"W": rel_err(wg[:, :, :nr], o.rhs_wpt[:, :, :nr]), "P": rel_err(wg[:, :, nr:2 * nr], o.rhs_wpt[:, :, nr:2 * nr]),
            "T": rel_err(wg[:, :, 2 * nr:], o.rhs_wpt[:, :, 2 * nr:]), "Z": rel_err(zg, o.rhs_z)}


@pytest.mark.parametrize("precision", [0, 1])
def test_loaded_own_matrices_match_built_in(precision):
    """The library's own matrices and coefficients loaded back through the C ABI
    reproduce the built-in run bit for bit."""
    oc, o, wpt, z = _start(CFG)
    a = _ctx(CFG, precision=precision)
    b = _ctx(CFG, precision=precision)
    L = oc.l_max + 1
    rc = rb.Config(**CFG)
    lw, cw = rb.build_matrices(rc, 0, 0, L, coefs=True)
    lz, cz = rb.build_matrices(rc, 1, 0, L, coefs=True)
    b.load_matrices(0, lw, cw)
    b.load_matrices(1, lz, cz)
    b.factor(CFG["dt"])
    for g in (a, b):
        g.put_state(wpt, z, None, iteration=1)
        g.step(6)
    sa, sb = a.get_state(), b.get_state()
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)


def test_loaded_oracle_matrices_step_with_the_oracle():
    """The oracle's own per-l matrices (the driver's, here) drive the device solve:
    10 steps agree with the oracle at 1e-12 per field."""
    oc, o, wpt, z = _start(CFG)
    g = _ctx(CFG)
    L, nr = oc.l_max + 1, oc.n_r
    lw = np.stack([m.T for m in o.mat_wpt])                              # column-major per l
    lz = np.stack([np.zeros((nr, nr))] + [m.T for m in o.mat_z[1:]])
    g.load_matrices(0, lw)
    g.load_matrices(1, lz)
    g.factor(CFG["dt"])
    g.put_state(wpt, z, None, iteration=1)
    for _ in range(10):
        o.step()
    g.step(10)
    errs = _errs(g, o, nr)
    assert max(errs.values()) < 1e-12, errs


def test_singular_loaded_matrix():
    oc, o, wpt, z = _start(CFG)
    g = _ctx(CFG)
    L = oc.l_max + 1
    rc = rb.Config(**CFG)
    lw = rb.build_matrices(rc, 0, 0, L)
    lz = rb.build_matrices(rc, 1, 0, L)
    lw[3][:, 40] = 0.0                # zero row 40 of A_3 (column-major: [col][row])
    g.load_matrices(0, lw)
    g.load_matrices(1, lz)
    with pytest.raises(rb.RayleighError) as ei:
        g.factor(CFG["dt"])
    assert ei.value.code == rb.RA_ERR_SINGULAR
    assert "W-P-T" in str(ei.value) and "l = 3" in str(ei.value)


def test_nonfinite_state_refused():
    oc, o, wpt, z = _start(CFG)
    g = _ctx(CFG)
    bad = wpt.copy()
    bad[7, 1, 5] = np.nan
    with pytest.raises(rb.RayleighError) as ei:
        g.put_state(bad, z, None, iteration=1)
    assert ei.value.code == rb.RA_ERR_NONFINITE
    with pytest.raises(rb.RayleighError) as ei:
        g.step(1)                     # no state was accepted
    assert ei.value.code == rb.RA_ERR_STATE
    ab = np.zeros((4, len(o.ls), 2, oc.n_r))
    ab[2, 3, 0, 4] = np.inf
    with pytest.raises(rb.RayleighError) as ei:
        g.put_state(wpt, z, ab, iteration=2)
    assert ei.value.code == rb.RA_ERR_NONFINITE
    g.put_state(wpt, z, None, iteration=1)   # a finite state is accepted again
    g.step(2)


def test_nonfinite_reached_in_step():
    """A coefficient near the overflow threshold (finite, so the load accepts it)
    drives the state to Inf/NaN within a few steps; the step reports
    RA_ERR_NONFINITE from the device flag instead of returning garbage."""
    oc, o, wpt, z = _start(CFG)
    g = _ctx(CFG, use_graph=True)
    L = oc.l_max + 1
    rc = rb.Config(**CFG)
    lw, cw = rb.build_matrices(rc, 0, 0, L, coefs=True)
    cw[:, 10, :] = 1e308             # slot (T, T, 0) of every l
    g.load_matrices(0, lw, cw)
    g.load_matrices(1, rb.build_matrices(rc, 1, 0, L))
    g.factor(CFG["dt"])
    g.put_state(wpt, z, None, iteration=1)
    code = None
    for _ in range(8):
        try:
            g.step(1)
        except rb.RayleighError as e:
            code = e.code
            break
    assert code == rb.RA_ERR_NONFINITE


def test_boundary_values_mask():
    """bc_values with non-zero entries beyond l = 0 (a fixed-T perturbation at the
    top for (l, m) = (2, 1), (3, 0), a dT pattern at the bottom) against the
    oracle's Apply_Boundary_Mask with the same values; NULL restores the default."""
    oc, o, wpt, z = _start(CFG)
    g = _ctx(CFG)
    nlm = len(o.ls)
    bv = np.zeros((4, nlm, 2, 2))
    s4 = np.sqrt(4 * np.pi)
    bv[2, 0, 0, 0] = oc.t_top * s4
    bv[2, 0, 0, 1] = oc.t_bottom * s4
    lm = lambda l, m: l * (l + 1) // 2 + m
    bv[2, lm(2, 1), 0, 0] = 0.3
    bv[2, lm(2, 1), 1, 0] = -0.1
    bv[2, lm(3, 0), 0, 0] = 0.05
    bv[2, lm(5, 4), 1, 1] = 0.02
    o.bc_values = bv
    g.set_bc_mask(bv)
    g.put_state(wpt, z, None, iteration=1)
    for _ in range(5):
        o.step()
    g.step(5)
    errs = _errs(g, o, oc.n_r)
    assert max(errs.values()) < 1e-12, errs
    # back to the built-in values: the same as a context that never had a mask
    h = _ctx(CFG)
    g.set_bc_mask(None)
    for c in (g, h):
        c.put_state(wpt, z, None, iteration=1)
        c.step(3)
    for x, y in zip(g.get_state(), h.get_state()):
        assert np.array_equal(x, y)


def _rank_modes(lmax, nranks):
    """The reference's layout of modes over ranks: m values dealt high-low
    (Load_Balance.F90), each rank's (l, m) pairs ordered l slowest, m fastest."""
    ms = list(range(lmax + 1))
    owner = {}
    for i, m in enumerate(ms):
        k = i % (2 * nranks)
        owner[m] = k if k < nranks else 2 * nranks - 1 - k
    out = []
    for r in range(nranks):
        mine = sorted(m for m in ms if owner[m] == r)
        pairs = [(l, m) for l in range(lmax + 1) for m in mine if m <= l]
        out.append((np.array([p[0] for p in pairs]), np.array([p[1] for p in pairs])))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_rank_local_state_exchange(precision):
    """The state put as four ranks' slices and read back the same way equals the
    whole-state path bit for bit, after steps."""
    oc, o, wpt, z = _start(CFG)
    nr = oc.n_r
    rng = np.random.Generator(np.random.PCG64(3))
    ab = rng.standard_normal((4, len(o.ls), 2, nr)) * 1e-3
    full = _ctx(CFG, precision=precision)
    part = _ctx(CFG, precision=precision)
    full.put_state(wpt, z, ab, iteration=2)
    lm = lambda l, m: l * (l + 1) // 2 + m
    ranks = _rank_modes(oc.l_max, 4)
    for ls, ms in reversed(ranks):
        idx = np.array([lm(l, m) for l, m in zip(ls, ms)])
        part.put_state_modes(ls, ms, wpt[idx], z[idx], ab[:, idx], iteration=2)
    for g in (full, part):
        g.step(4)
    fw, fz, fab = full.get_state()
    for ls, ms in ranks:
        idx = np.array([lm(l, m) for l, m in zip(ls, ms)])
        w, zz, a = part.get_state_modes(ls, ms)
        assert np.array_equal(w, fw[idx]) and np.array_equal(zz, fz[idx]) and np.array_equal(a, fab[:, idx])
    with pytest.raises(rb.RayleighError):
        part.put_state_modes([2, 2], [1, 1], wpt[:2], z[:2])          # a repeated mode
    with pytest.raises(rb.RayleighError):
        part.put_state_modes([3], [4], wpt[:1], z[:1])                # m > l
