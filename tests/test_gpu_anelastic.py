"""The anelastic equation sets on the device against the oracle.

reference_type 3 (Polytropic_ReferenceND, PDE_Coefficients.F90:437-537) and 2
(Polytropic_Reference, :925-1051): the density-weighted velocity of rlm_spacea
(over_rhor, over_rhorsq, drho_term, Sphere_Hybrid_Space.F90:44-62, 240-350), the
density factors of the momentum terms, the viscous and ohmic heating
(Sphere_Physical_Space.F90:337-466) and the variable-coefficient implicit terms
(Compute_Diffusion_Coefs, PDE_Coefficients.F90:2032-2098, in Load_Linear_Coefficients,
Sphere_Linear_Terms.F90:196-537).  FP64 form: every stage and the state after N steps
to 1e-12 relative L2 per field; mixed form: 1e-9.  The anelastic MHD workload
(N_r = 128, l_max = 255, 200 graph-captured steps) reports the mixed form's error
against the FP64 form and is checked against the oracle over its first step."""
import dataclasses
import time

import numpy as np
import pytest

import oracle as O
import test_gpu_mhd as M
import test_gpu_parity as H
from layouts import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12
# the anelastic MHD workload's physics on a small grid
ANEL = dict(n_r=24, l_max=15, dt=1e-4, reference_type=3, poly_n=2.0, poly_nrho=5.0, modified_rayleigh=0.5,
            ekman=1e-3, prandtl=1.0, magnetic_prandtl=2.0, no_slip_top=False, no_slip_bottom=False)
ANEL_MHD = dict(ANEL, magnetism=True)
# the dimensional polytrope of the Jones et al. benchmarks (Benchmarking.F90:202-300), cgs
J2011 = dict(n_r=24, l_max=15, dt=30.0, reference_type=2, shell_depth=4.55e9, aspect_ratio=0.35, poly_n=2.0,
             poly_nrho=5.0, poly_mass=1.9e30, poly_rho_i=1.1, pressure_specific_heat=1.0509e8,
             angular_velocity=1.76e-4, nu_top=3.64364e12, kappa_top=3.64364e12, no_slip_top=False,
             no_slip_bottom=False, t_bottom=851225.7)


@pytest.mark.parametrize("steps_before", [0, 2])
def test_anelastic_mhd_stages(steps_before):
    errs = M._stage_compare(ANEL_MHD, steps_before=steps_before)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


@pytest.mark.parametrize("cfg", [ANEL, dict(ANEL, nu_type=2, nu_power=-0.5, kappa_type=2, kappa_power=-0.5)])
def test_anelastic_hydro_stages(cfg):
    """After two steps (the seeded state has no velocity yet), so that the viscous heating
    and the density-weighted advection are exercised stage by stage."""
    errs = H._stage_compare(cfg, steps_before=2)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


@pytest.mark.parametrize("cfg,steps,precision,tol", [
    (ANEL_MHD, 20, 0, TOL),
    (ANEL_MHD, 20, 1, 1e-9),
    (dict(ANEL_MHD, n_r=48, l_max=63, eta_type=2, eta_power=-0.5, no_slip_bottom=True), 20, 0, TOL),
    (dict(ANEL_MHD, n_r=48, l_max=63, eta_type=2, eta_power=-0.5, no_slip_bottom=True), 20, 1, 1e-9),
    (dict(ANEL, viscous_heating=False), 20, 0, TOL),
])
def test_anelastic_mhd_multi_step_parity(cfg, steps, precision, tol):
    oc = M._ocfg(cfg)
    o = O.Oracle(oc)
    mag = bool(cfg.get("magnetism"))
    wpt, z, c, a = M._seed(oc, amp_u=1e-3, amp_b=1e-2)
    o.init_state(wpt, z, c_coeffs=c if mag else None, a_coeffs=a if mag else None)
    g = M._ctx(dict(cfg, precision=precision, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    if mag:
        g.put_magnetic_state(c, a)
    for _ in range(steps):
        o.step()
    cfl = g.step(steps)
    if mag:
        errs = M._state_errs(o, g)
    else:
        wg, zg, _ = g.get_state()
        nr = oc.n_r
        errs = {k: rel_err(v, H._fields(o.rhs_wpt, o.rhs_z, nr)[k]) for k, v in H._fields(wg, zg, nr).items()}
    print(cfg, precision, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < tol, errs
    assert abs(cfl - o.last_cfl) <= max(1e-9, 10 * tol) * o.last_cfl


@pytest.mark.parametrize("precision,tol", [(0, 1e-11), (1, 1e-9)])
def test_dimensional_polytrope_parity(precision, tol):
    """The cgs polytrope (reference_type 2) of the Jones et al. hydrodynamic benchmark:
    10 steps of 30 s against the oracle.  Its W-P-T matrices are ill conditioned (the
    smallest LU pivot, after row and column equilibration, is ~1e-2 n 2^-53), so two
    backward-stable LU solves (the device's and LAPACK's) agree to ~2e-12 in P after 10
    steps; the mixed form solves these systems by the FP64 block substitution (an
    explicit inverse of them loses all digits) and keeps its split products for the
    Legendre transforms."""
    oc = M._ocfg(J2011)
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=1e3, lmax_pert=10)
    o.init_state(wpt, z)
    g = M._ctx(dict(J2011, precision=precision, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    for _ in range(10):
        o.step()
    g.step(10)
    wg, zg, _ = g.get_state()
    nr = oc.n_r
    errs = {k: rel_err(v, H._fields(o.rhs_wpt, o.rhs_z, nr)[k]) for k, v in H._fields(wg, zg, nr).items()}
    print(precision, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < tol, errs


def test_anelastic_mhd_workload():
    """The anelastic MHD step at its own size: the nondimensional polytrope with 5 density
    scale heights, n = 2, radius ratio 0.35, N_r = 128, l_max = 255 (N_theta = 384,
    N_phi = 768); fields W, Z, P, S, C, A; seeded entropy and magnetic perturbations of
    amplitude 1e-4 with (l+1)^-2 decay; 200 graph-captured steps in each form.  The FP64
    form matches the oracle over the first step to 1e-12.  The mixed form's difference
    from the FP64 form grows by ~5e-12 per step, as it does on the Boussinesq dynamo
    (6e-10 after 100 steps at l_max = 511): measured 1.0e-9 after 200 steps, bounded here
    at 2e-9."""
    import rayleigh_b200 as rb
    oc = O.anelastic_mhd_config()
    names = {f.name for f in dataclasses.fields(rb.Config)}
    cfg = {k: v for k, v in dataclasses.asdict(oc).items() if k in names}
    wpt, z = O.seeded_state(oc, amp=1e-4, lmax_pert=20)
    c, a = O.seeded_magnetic_state(oc, amp=1e-4, lmax_pert=20)
    # the first step against the oracle, FP64
    o = O.Oracle(oc)
    o.init_state(wpt, z, c_coeffs=c, a_coeffs=a)
    o.step()
    g = M._ctx(dict(cfg, precision=rb.PREC_FP64, use_graph=True))
    g.put_state(wpt, z, None, iteration=1)
    g.put_magnetic_state(c, a)
    g.step(1)
    errs = M._state_errs(o, g)
    print("first step vs oracle", {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < TOL, errs
    del g
    states, rates = {}, {}
    for prec in (rb.PREC_FP64, rb.PREC_MIXED):
        g = M._ctx(dict(cfg, precision=prec, use_graph=True))
        g.put_state(wpt, z, None, iteration=1)
        g.put_magnetic_state(c, a)
        g.step(2)
        g.get_state()   # synchronises
        t0 = time.perf_counter()
        g.step(198)
        w, zz, _ = g.get_state()
        rates[prec] = 198 / (time.perf_counter() - t0)
        cc, aa, _ = g.get_magnetic_state()
        states[prec] = {"W": w[:, :, :oc.n_r], "P": w[:, :, oc.n_r:2 * oc.n_r], "S": w[:, :, 2 * oc.n_r:], "Z": zz,
                        "C": cc, "A": aa}
        del g
    errs = {k: rel_err(states[rb.PREC_MIXED][k], states[rb.PREC_FP64][k]) for k in states[rb.PREC_FP64]}
    print(f"anelastic MHD l_max 255 N_r 128: FP64 {rates[rb.PREC_FP64]:.1f} steps/s, mixed "
          f"{rates[rb.PREC_MIXED]:.1f} steps/s (host-timed, with a state copy); mixed vs FP64 after 200 steps",
          {k: f"{v:.2e}" for k, v in errs.items()})
    assert all(np.isfinite(v) for v in errs.values())
    assert max(errs.values()) < 2e-9, errs


def test_driver_reference_state():
    """ra_set_reference with the polytrope's profiles (density, dlnrho, the heating
    coefficients, Coriolis and Lorentz coefficients) on a context created with the
    Boussinesq reference, with the polytrope's matrices loaded through ra_load_matrices and
    ra_factor, steps as the context that restates the polytrope itself: the route by which
    reference states the library does not restate (custom files, reference_type 4 and 5)
    reach the device.  A dt change then needs the driver's matrices (RA_ERR_STATE)."""
    import rayleigh_b200 as rb
    oc = M._ocfg(ANEL_MHD)
    o = O.Oracle(oc)
    wpt, z, c, a = M._seed(oc, amp_u=1e-3, amp_b=1e-2)
    ref = M._ctx(dict(ANEL_MHD, use_graph=True))
    g = M._ctx(dict(ANEL_MHD, reference_type=1, use_graph=True))
    rc = rb.Config(**ANEL_MHD)
    L = oc.l_max + 1
    for sys in range(4):
        lhs, cf = rb.build_matrices(rc, sys, 0, L, coefs=True)
        g.load_matrices(sys, lhs, cf)
    g.factor(ANEL_MHD["dt"])
    g.set_reference(o.density, o.dlnrho, o.viscous_heating_coeff, o.ohmic_heating_coeff, o.coriolis, o.lorentz)
    for ctx in (g, ref):
        ctx.put_state(wpt, z, None, iteration=1)
        ctx.put_magnetic_state(c, a)
        ctx.step(5)
    for x, y in zip(g.get_state()[:2] + g.get_magnetic_state()[:2], ref.get_state()[:2] + ref.get_magnetic_state()[:2]):
        assert rel_err(x, y) < 1e-13
    with pytest.raises(rb.RayleighError) as ei:
        g.set_dt(2e-4)
    assert ei.value.code == rb.RA_ERR_STATE
    with pytest.raises(rb.RayleighError) as ei:
        g.set_reference(-o.density, o.dlnrho)
    assert ei.value.code == rb.RA_ERR_ARG
