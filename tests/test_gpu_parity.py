"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64 form: every stage and the state after N steps agree with the oracle to a
relative L2 error (per field) of 1e-12 or better."""
import numpy as np
import pytest

import oracle as O
from layouts import p2_eo_to_full, p2_fold, p2_to_dev, rel_err, row_index, s2_to_rows

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _ctx(cfg):
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    return rb.Rayleigh(rb.Config(**cfg))


def _ocfg(cfg):
    keys = {k: v for k, v in cfg.items() if k in O.Config.__dataclass_fields__}
    return O.Config(**keys)


@pytest.mark.parametrize("lmax,nth", [(15, 24), (63, 96), (255, 384)])
def test_plm_tables(lmax, nth):
    cfg = dict(n_r=16, l_max=lmax, n_theta=nth)
    g = _ctx(cfg)
    h = O.Horizontal(lmax, nth)
    L = lmax + 1
    P = g.debug_buffer("ptab").reshape(-1, nth // 2)
    iP = g.debug_buffer("iptab").reshape(-1, nth // 2)
    worst = 0.0
    for m in range(L):
        for par, (ref, iref) in enumerate(((h.p_even[m], h.ip_even[m]), (h.p_odd[m], h.ip_odd[m]))):
            nl = ref.shape[0]
            if nl == 0:
                continue
            rows = [row_index(m, m + par + 2 * j, L) for j in range(nl)]
            scale = max(np.abs(ref).max(), 1e-300)
            worst = max(worst, np.abs(P[rows] - ref).max() / scale)
            iscale = max(np.abs(iref).max(), 1e-300)
            worst = max(worst, np.abs(iP[rows] - iref.T).max() / iscale)
    # FP64 recurrence with a carried exponent vs the REAL*16 (longdouble) one:
    # error grows ~ l eps relative to the largest entry of each m table
    assert worst < 5e-12, worst


@pytest.mark.parametrize("lmax,nth,nf,nr", [(15, 24, 3, 5), (63, 96, 2, 7)])
def test_legendre_transforms(lmax, nth, nf, nr):
    g = _ctx(dict(n_r=16, l_max=lmax, n_theta=nth))
    h = O.Horizontal(lmax, nth)
    rng = np.random.Generator(np.random.PCG64(11))
    s2 = [rng.standard_normal((nf, 2, nr, lmax - m + 1)) for m in range(lmax + 1)]
    ref = h.s2p(s2)
    got = g.legendre_s2p(s2)
    assert rel_err(np.stack(got), np.stack(ref)) < 1e-14
    p2 = [rng.standard_normal((nf, 2, nr, nth)) for m in range(lmax + 1)]
    ref = h.p2s(p2)
    got = g.legendre_p2s(p2)
    assert rel_err(np.concatenate([a.ravel() for a in got]), np.concatenate([a.ravel() for a in ref])) < 1e-14


@pytest.mark.parametrize("lmax", [15, 63, 511])
def test_fft(lmax):
    g = _ctx(dict(n_r=16, l_max=lmax))
    nphi = g.n_phi
    rng = np.random.Generator(np.random.PCG64(5))
    x = rng.standard_normal((7, nphi + 2))
    x[:, nphi:] = 0
    np.testing.assert_allclose(g.fft_r2c(x), O.fft_r2c(x, nphi), rtol=0, atol=1e-12 * np.abs(O.fft_r2c(x, nphi)).max())
    X = O.fft_r2c(x, nphi)
    ref = O.fft_c2r(X, nphi)
    got = g.fft_c2r(X)
    assert rel_err(got[:, :nphi], ref[:, :nphi]) < 1e-14


def test_chebyshev_operators():
    g = _ctx(dict(n_r=48, l_max=15))
    cfg = _ocfg(dict(n_r=48, l_max=15))
    o = O.Oracle(cfg)
    np.testing.assert_allclose(g.radius(), o.radius, rtol=1e-15)
    rng = np.random.Generator(np.random.PCG64(9))
    f = rng.standard_normal((10, 48))
    assert rel_err(g.cheby_to_spectral(f), o.cg.to_spectral(f)) < 1e-13
    assert rel_err(g.cheby_from_spectral(f), o.cg.from_spectral(f)) < 1e-13
    for order in (1, 2, 3):
        assert rel_err(g.cheby_deriv(f, order), o.cg.deriv(f, order)) < 1e-13


SMALL = dict(n_r=24, l_max=15, dt=2e-4, rayleigh=1e5, ekman=1e-3)


def _stage_compare(cfg, steps_before=0, amp=1e-2, choices=None):
    """Run one step stage by stage on both sides; return {stage: rel err}."""
    oc = _ocfg(cfg)
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=amp, lmax_pert=min(10, oc.l_max))
    o.init_state(wpt, z)
    g = _ctx(dict(cfg, use_graph=False))
    for knob, v in (choices or {}).items():
        g.set_choice(knob, v)
    g.put_state(wpt, z, None, iteration=1)
    for _ in range(steps_before):
        o.step()
        g.step(1)
    wg, zg, abg = g.get_state()
    errs = {"state_in_wpt": rel_err(wg, o.rhs_wpt), "state_in_z": rel_err(zg, o.rhs_z)}
    # ---- oracle stages with intermediates ----
    L, nr, nth = oc.l_max + 1, oc.n_r, oc.n_theta
    cg = o.cg
    c = cg.dealias(o.get_all_rhs())
    W, P, T, Z = c
    grids = cg.from_spectral(cg.dealias(np.stack([W, cg.deriv(W, 1), cg.deriv(W, 2), cg.deriv(W, 3), P, cg.deriv(P, 1),
                                                  T, cg.deriv(T, 1), cg.deriv(T, 2), Z, cg.deriv(Z, 1), cg.deriv(Z, 2)])))
    g8 = o.post_solve()
    rhs_w, rhs_z = o.rhs_wpt.copy(), o.rhs_z.copy()
    s2a = o.transpose_1a2a(g8)
    s2a12 = o.rlm_spacea(s2a)
    p2a = o.h.s2p(s2a12)
    p3b = o.physical_space(o.transpose_2a3a(p2a))
    cfl_ref = o.last_cfl
    p2b = o.transpose_3b2b(p3b)
    s2b = o.h.p2s(p2b)
    ab = o.transpose_2b1b(o.rlm_spaceb(s2b))
    o.advance_time(ab)
    # ---- device stages ----
    g.post_solve()
    errs["grid"] = rel_err(g.debug_buffer("grid").reshape(grids.shape), grids)
    errs["rhs_wpt"] = rel_err(g.debug_buffer("rhs_wpt"), rhs_w.ravel())
    errs["rhs_z"] = rel_err(g.debug_buffer("rhs_z"), rhs_z.ravel())
    errs["s2a"] = rel_err(g.debug_buffer("s2a"), s2_to_rows(s2a, [0, 2, 3, 4, 5, 6, 7]).ravel())
    g.rlm_spacea()
    # device field order DVRDT, DVTDR, VR, VT, VP, DVRDR, DVPDR, OMR, DTDR, DTDT, T as oracle indexes
    a_fields = [6, 10, 0, 8, 9, 4, 11, 3, 5, 7, 2]
    errs["s2a11"] = rel_err(g.debug_buffer("s2a11"), s2_to_rows(s2a12, a_fields, r_major=True).ravel())
    errs["p2a"] = rel_err(p2_eo_to_full(g.debug_buffer("p2a"), L, nth, len(a_fields), nr),
                          p2_to_dev(p2a, a_fields))
    cfl = g.physical_space()
    errs["cfl"] = abs(cfl - cfl_ref) / max(cfl_ref, 1e-300)
    errs["p2b"] = rel_err(g.debug_buffer("p2b"), p2_fold(p2_to_dev(p2b, [0, 1, 2, 3])).ravel())
    g.rlm_spaceb()
    errs["s2b"] = rel_err(g.debug_buffer("s2b"), s2_to_rows(s2b, [0, 1, 2, 3], r_major=True).ravel())
    errs["ab"] = rel_err(g.debug_buffer("ab"), ab.ravel())
    g.advance_time()
    wg, zg, _ = g.get_state()
    errs["sol_wpt"] = rel_err(wg, o.rhs_wpt)
    errs["sol_z"] = rel_err(zg, o.rhs_z)
    return errs


def test_step_stages_first_step():
    errs = _stage_compare(SMALL)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


def test_step_stages_ab2_step():
    errs = _stage_compare(SMALL, steps_before=2)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


@pytest.mark.parametrize("physics", [0, 1, 2])
def test_step_stages_768_point_phi_transform(physics):
    """l_max = 511, n_theta = 768 (the l_max = 511 grid's angular size, few
    radii): the largest phi transform, through each physical-space kernel
    (0, 2: the three-pass 16 x 16 x 3 FFT at two or one CTA per SM; 1: the
    four-pass one, where each thread owns two points of a row)."""
    errs = _stage_compare(dict(n_r=8, l_max=511, dt=1e-6, rayleigh=1e5, ekman=1e-3), steps_before=1,
                          choices={"physics": physics})
    print(physics, {k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


def test_step_stages_1536_point_phi_transform():
    """l_max = 1023, n_theta = 1536, n_phi = 3072 (the transform sweep's largest
    size, few radii): the physical-space kernel with 512 threads per row."""
    errs = _stage_compare(dict(n_r=8, l_max=1023, dt=1e-6, rayleigh=1e5, ekman=1e-3), steps_before=1)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


@pytest.mark.parametrize("physics", [0, 1])
def test_step_stages_384_point_phi_transform(physics):
    """l_max = 255, n_theta = 384: the three-pass kernel's 16 x 8 x 3 plan."""
    errs = _stage_compare(dict(n_r=8, l_max=255, dt=1e-6, rayleigh=1e5, ekman=1e-3), steps_before=1,
                          choices={"physics": physics})
    print(physics, {k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


def test_autotune_choices():
    """The set-up autotuner picks a candidate of each knob; every candidate of
    the solve's column block gives the same state to rounding."""
    cfg = dict(n_r=96, l_max=63, dt=1e-5, ekman=1e-4, rayleigh=1e6)
    oc = _ocfg(cfg)
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=10)
    g = _ctx(dict(cfg, autotune=True))
    res = g.autotune(2)
    assert res["physics"][0] in (0, 1, 2) and res["solve_nc"][0] in (16, 32), res
    states = []
    for nc in (16, 32):
        g.set_choice("solve_nc", nc)
        g.put_state(wpt, z, None, iteration=1)
        g.step(4)
        states.append(g.get_state())
    for a, b in zip(states[0], states[1]):
        assert rel_err(a, b) < 1e-14
    with pytest.raises(Exception):
        g.set_choice("physics", 7)


def _fields(wpt, z, nr):
    return {"W": wpt[:, :, :nr], "P": wpt[:, :, nr:2 * nr], "T": wpt[:, :, 2 * nr:], "Z": z}


@pytest.mark.parametrize("cfg,steps", [
    (dict(n_r=24, l_max=15, dt=2e-4), 20),
    (dict(n_r=48, l_max=63, dt=1e-4), 100),         # the FP64 timestep-loop case: l_max = 63, N_r = 48, 100 steps
    (dict(n_r=32, l_max=31, dt=1e-4, no_slip_top=False, no_slip_bottom=False, fix_tvar_bottom=False,
          dtdr_bottom=-1.0, rotation=False), 10),
])
def test_multi_step_parity(cfg, steps):
    oc = _ocfg(cfg)
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=min(20, oc.l_max))
    o.init_state(wpt, z)
    g = _ctx(dict(cfg, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    for _ in range(steps):
        o.step()
    g.step(steps)
    wg, zg, _ = g.get_state()
    nr = oc.n_r
    errs = {k: rel_err(v, _fields(o.rhs_wpt, o.rhs_z, nr)[k]) for k, v in _fields(wg, zg, nr).items()}
    print(cfg, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < TOL, errs


@pytest.mark.parametrize("precision,tol", [(0, TOL), (1, 1e-9)])
def test_headline_radial_size(precision, tol):
    """N_r = 192 with the dynamo case's Ekman number and time step (Ek = 1e-5,
    dt = 1e-6) on a small angular grid (l_max = 15): the per-l W-P-T operators
    have condition numbers up to ~1e11 here, so this pins the device LU solve
    (and, in the mixed form, the split products of the explicit inverses)
    against the oracle's LAPACK solve over 10 steps."""
    cfg = dict(n_r=192, l_max=15, dt=1e-6, ekman=1e-5, rayleigh=5e6)
    oc = _ocfg(cfg)
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=10)
    o.init_state(wpt, z)
    g = _ctx(dict(cfg, precision=precision, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    for _ in range(10):
        o.step()
    g.step(10)
    wg, zg, _ = g.get_state()
    nr = oc.n_r
    errs = {k: rel_err(v, _fields(o.rhs_wpt, o.rhs_z, nr)[k]) for k, v in _fields(wg, zg, nr).items()}
    print(precision, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < tol, errs


@pytest.mark.parametrize("precision,tol", [(0, TOL), (1, 1e-9)])
def test_timestep_change(precision, tol):
    """Reset_Linear_Equations on a dt change (Sphere_Linear_Terms.F90:67-76):
    the implicit matrices are rebuilt and factored again (and their inverses' digits
    split again in the mixed form), the AB2 factors of the first step after
    the change use the unequal steps, and the replayed step graph is captured
    again; the state then follows the oracle as before."""
    cfg = dict(n_r=24, l_max=15, dt=2e-4, rayleigh=1e5, ekman=1e-3)
    oc = _ocfg(cfg)
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=1e-2, lmax_pert=10)
    o.init_state(wpt, z)
    g = _ctx(dict(cfg, precision=precision, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    for _ in range(4):
        o.step()
    g.step(4)
    o.set_dt(1.3e-4)
    g.set_dt(1.3e-4)
    for _ in range(4):
        o.step()
    g.step(4)
    wg, zg, _ = g.get_state()
    nr = oc.n_r
    errs = {k: rel_err(v, _fields(o.rhs_wpt, o.rhs_z, nr)[k]) for k, v in _fields(wg, zg, nr).items()}
    print(precision, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < tol, errs
