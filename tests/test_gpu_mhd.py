"""The dynamo (magnetic) equation set on the device against the oracle.

Magnetism adds the poloidal and toroidal potentials C and A of B: their
Chebyshev synthesis and Post_Solve terms, B and curl B in rlm_spacea
(Compute_BandCurlB, Sphere_Hybrid_Space.F90:357-435), the Lorentz force and
the EMF in physical space (Sphere_Physical_Space.F90:512-581), Adjust_Emf in
rlm_spaceb (:557-602), Finalize_EMF's radial derivative and the C and A solves
with insulating boundaries (Sphere_Spectral_Space.F90:436-488,
Sphere_Linear_Terms.F90:473-499, 1041-1077).  FP64 form: every stage and the
state after N steps to 1e-12 relative L2 per field; mixed form: 1e-9."""
import numpy as np
import pytest

import oracle as O
from layouts import p2_eo_to_full, p2_fold, p2_to_dev, rel_err, s2_to_rows

pytestmark = pytest.mark.gpu
TOL = 1e-12
MHD = dict(n_r=24, l_max=15, dt=2e-4, rayleigh=1e5, ekman=1e-3, magnetism=True, magnetic_prandtl=5.0)


def _ctx(cfg):
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    return rb.Rayleigh(rb.Config(**cfg))


def _ocfg(cfg):
    return O.Config(**{k: v for k, v in cfg.items() if k in O.Config.__dataclass_fields__})


def _seed(oc, amp_u=1e-2, amp_b=1e-1):
    wpt, z = O.seeded_state(oc, amp=amp_u, lmax_pert=min(10, oc.l_max))
    c, a = O.seeded_magnetic_state(oc, amp=amp_b, lmax_pert=min(10, oc.l_max))
    return wpt, z, c, a


def _state_errs(o, g):
    nr = o.cfg.n_r
    wg, zg, _ = g.get_state()
    cg, ag, _ = g.get_magnetic_state()
    return {"W": rel_err(wg[:, :, :nr], o.rhs_wpt[:, :, :nr]), "P": rel_err(wg[:, :, nr:2 * nr], o.rhs_wpt[:, :, nr:2 * nr]),
            "T": rel_err(wg[:, :, 2 * nr:], o.rhs_wpt[:, :, 2 * nr:]), "Z": rel_err(zg, o.rhs_z),
            "C": rel_err(cg, o.rhs_c), "A": rel_err(ag, o.rhs_a)}


def _stage_compare(cfg, steps_before=0):
    oc = _ocfg(cfg)
    o = O.Oracle(oc)
    wpt, z, c, a = _seed(oc)
    o.init_state(wpt, z, c_coeffs=c, a_coeffs=a)
    g = _ctx(dict(cfg, use_graph=False))
    g.put_state(wpt, z, None, iteration=1)
    g.put_magnetic_state(c, a)
    for _ in range(steps_before):
        o.step()
        g.step(1)
    errs = {"state_in_" + k: v for k, v in _state_errs(o, g).items()}
    L, nr, nth = oc.l_max + 1, oc.n_r, oc.n_theta
    cg = o.cg
    cc = cg.dealias(o.get_all_rhs())
    W, P, T, Z, C, A = cc
    d = cg.deriv
    grids = cg.from_spectral(cg.dealias(np.stack([W, d(W, 1), d(W, 2), d(W, 3), P, d(P, 1), T, d(T, 1), d(T, 2), Z,
                                                  d(Z, 1), d(Z, 2), C, d(C, 1), d(C, 2), A, d(A, 1), d(A, 2)])))
    g13 = o.post_solve()
    rhs_c, rhs_a = o.rhs_c.copy(), o.rhs_a.copy()
    s2a = o.transpose_1a2a(g13)
    s2a18 = o.rlm_spacea(s2a)
    p2a = o.h.s2p(s2a18)
    p3b = o.physical_space(o.transpose_2a3a(p2a))
    cfl_ref = o.last_cfl
    p2b = o.transpose_3b2b(p3b)
    s2b = o.h.p2s(p2b)
    o.advance_time(o.transpose_2b1b(o.rlm_spaceb(s2b)))
    g.post_solve()
    errs["grid"] = rel_err(g.debug_buffer("grid").reshape(grids.shape), grids)
    errs["rhs_c"] = rel_err(g.debug_buffer("rhs_c"), rhs_c.ravel())
    errs["rhs_a"] = rel_err(g.debug_buffer("rhs_a"), rhs_a.ravel())
    errs["s2am"] = rel_err(g.debug_buffer("s2am"), s2_to_rows(s2a, [8, 9, 10, 11, 12]).ravel())
    g.rlm_spacea()
    a_fields = [6, 10, 0, 8, 9, 4, 11, 3, 5, 7, 2, 12, 13, 14, 15, 16, 17]
    dev = g.debug_buffer("s2a11").reshape(-1, nr, 17, 2)
    ref = s2_to_rows(s2a18, a_fields, r_major=True)
    errs["s2a_hydro"] = rel_err(dev[:, :, :11], ref[:, :, :11])
    for i, name in enumerate(("br", "curlbr", "curlbt", "curlbp", "bt", "bp")):
        errs["s2a_" + name] = rel_err(dev[:, :, 11 + i], ref[:, :, 11 + i])
    errs["p2a"] = rel_err(p2_eo_to_full(g.debug_buffer("p2a"), L, nth, 17, nr), p2_to_dev(p2a, a_fields))
    cfl = g.physical_space()
    errs["cfl"] = abs(cfl - cfl_ref) / max(cfl_ref, 1e-300)
    devb = g.debug_buffer("p2b").reshape(L, 2, nth // 2, nr, 7, 2)
    refb = p2_fold(p2_to_dev(p2b, list(range(7))))
    for i, name in enumerate(("W", "P", "T", "Z", "emft", "emfr", "emfp")):
        errs["p2b_" + name] = rel_err(devb[..., i, :], refb[..., i, :])
    g.rlm_spaceb()
    errs["s2b"] = rel_err(g.debug_buffer("s2b"), s2_to_rows(s2b, list(range(7)), r_major=True).ravel())
    abd = g.debug_buffer("ab").reshape(6, -1)
    for i, name in enumerate(("W", "P", "T", "Z", "C", "A")):
        errs["ab_" + name] = rel_err(abd[i], o.ab[i].ravel())
    g.advance_time()
    errs.update({"sol_" + k: v for k, v in _state_errs(o, g).items()})
    return errs


def test_mhd_stages_first_step():
    errs = _stage_compare(MHD)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


def test_mhd_stages_ab2_step():
    errs = _stage_compare(MHD, steps_before=2)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


@pytest.mark.parametrize("cfg,steps,precision,tol", [
    (MHD, 20, 0, TOL),
    (dict(MHD, n_r=48, l_max=63, dt=1e-4, magnetic_prandtl=1.0), 20, 0, TOL),   # the l_max = 63, N_r = 48 grid
    (dict(MHD, rotation=False, no_slip_top=False, no_slip_bottom=False), 10, 0, TOL),
    (MHD, 20, 1, 1e-9),
    (dict(MHD, n_r=48, l_max=63, dt=1e-4, magnetic_prandtl=1.0), 20, 1, 1e-9),
])
def test_mhd_multi_step_parity(cfg, steps, precision, tol):
    oc = _ocfg(cfg)
    o = O.Oracle(oc)
    wpt, z, c, a = _seed(oc)
    o.init_state(wpt, z, c_coeffs=c, a_coeffs=a)
    g = _ctx(dict(cfg, precision=precision, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    g.put_magnetic_state(c, a)
    for _ in range(steps):
        o.step()
    cfl = g.step(steps)
    errs = _state_errs(o, g)
    print(cfg, precision, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < tol, errs
    assert abs(cfl - o.last_cfl) <= 1e-9 * o.last_cfl


def test_mhd_headline_radial_size():
    """N_r = 192 with the dynamo case's Ekman number and time step on a small angular grid:
    the C and A operators' potential-field rows at the radial size of the headline case."""
    cfg = dict(n_r=192, l_max=15, dt=1e-6, ekman=1e-5, rayleigh=5e6, magnetism=True, magnetic_prandtl=1.0)
    oc = _ocfg(cfg)
    o = O.Oracle(oc)
    wpt, z, c, a = _seed(oc, amp_u=1e-3, amp_b=1e-3)
    o.init_state(wpt, z, c_coeffs=c, a_coeffs=a)
    g = _ctx(dict(cfg, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    g.put_magnetic_state(c, a)
    for _ in range(5):
        o.step()
    g.step(5)
    errs = _state_errs(o, g)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < TOL, errs


def test_mhd_restart_and_dt_change():
    """A checkpoint through get/put (hydrodynamic and magnetic parts) continues bit for bit;
    a dt change rebuilds and refactors the C and A systems with the others."""
    oc = _ocfg(MHD)
    wpt, z, c, a = _seed(oc)
    g = _ctx(dict(MHD, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    g.put_magnetic_state(c, a)
    g.step(3)
    w3, z3, ab3 = g.get_state()
    c3, a3, abm3 = g.get_magnetic_state()
    g.step(3)
    ref = g.get_state(), g.get_magnetic_state()
    h = _ctx(dict(MHD, use_graph=True))
    h.put_state(w3, z3, ab3, iteration=4)
    h.put_magnetic_state(c3, a3, abm3)
    h.step(3)
    got = h.get_state(), h.get_magnetic_state()
    for x, y in zip(ref, got):
        for u, v in zip(x, y):
            assert np.array_equal(u, v)
    o = O.Oracle(oc)
    o.init_state(wpt, z, c_coeffs=c, a_coeffs=a)
    g2 = _ctx(dict(MHD, use_graph=True))
    g2.put_state(wpt, z, None, iteration=1)
    g2.put_magnetic_state(c, a)
    for _ in range(3):
        o.step()
    g2.step(3)
    o.set_dt(1.3e-4)
    g2.set_dt(1.3e-4)
    for _ in range(3):
        o.step()
    g2.step(3)
    errs = _state_errs(o, g2)
    assert max(errs.values()) < TOL, errs


def test_mhd_loaded_matrices():
    """The driver's own C and A matrices through ra_load_matrices (systems 2 and 3) and
    ra_factor step like the library's own assembly."""
    import rayleigh_b200 as rb
    oc = _ocfg(MHD)
    wpt, z, c, a = _seed(oc)
    rc = rb.Config(**MHD)
    L = oc.l_max + 1
    g = _ctx(dict(MHD, use_graph=False))
    for sys in range(4):
        lhs, cf = rb.build_matrices(rc, sys, 0, L, coefs=True)
        g.load_matrices(sys, lhs, cf)
    g.factor(MHD["dt"])
    ref = _ctx(dict(MHD, use_graph=False))
    for ctx in (g, ref):
        ctx.put_state(wpt, z, None, iteration=1)
        ctx.put_magnetic_state(c, a)
        ctx.step(4)
    for x, y in zip(g.get_magnetic_state(), ref.get_magnetic_state()):
        assert rel_err(x, y) < 1e-14
