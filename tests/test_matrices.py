"""The library's own assembly of the per-l implicit matrices (ra_build_matrices,
host only, no GPU) against the oracle's restatement of Load_Linear_Coefficients +
Set_Boundary_Conditions (Sphere_Linear_Terms.F90:196-1100, Linear_Solve.F90:494-539),
and the Post_Solve coefficients of the same terms."""
import numpy as np
import pytest

import oracle as O


ANEL = dict(n_r=32, l_max=7, dt=1e-4, reference_type=3, poly_n=2.0, poly_nrho=5.0, modified_rayleigh=0.5,
            ekman=1e-3, no_slip_top=False, no_slip_bottom=False)


def _slots():
    # (eq, var, dorder) of the 16 coefficient slots, in the order the C ABI documents
    W, P, T, Z = O.WVAR, O.PVAR, O.TVAR, O.ZVAR
    WE, PE, TE, ZE = O.WEQ, O.PEQ, O.TEQ, O.ZEQ
    return [(WE, W, 0), (WE, W, 1), (WE, W, 2), (WE, P, 1), (WE, T, 0), (PE, W, 0), (PE, W, 1), (PE, W, 2),
            (PE, W, 3), (PE, P, 0), (TE, T, 0), (TE, T, 1), (TE, T, 2), (ZE, Z, 0), (ZE, Z, 1), (ZE, Z, 2)]


@pytest.mark.parametrize("cfg", [
    dict(n_r=24, l_max=7, dt=2e-4, ekman=1e-3, rayleigh=1e5),
    dict(n_r=32, l_max=7, dt=1e-4, no_slip_top=False, no_slip_bottom=False, fix_tvar_bottom=False, dtdr_bottom=-1.0,
         rotation=False),
    dict(n_r=128, l_max=7, dt=1e-5, ekman=1e-4, rayleigh=1e5),   # the batched-solve workload's radial size
    # anelastic: the nondimensional polytrope (5 scale heights, n = 2), constant and
    # density-dependent diffusivities, and the dimensional (cgs) polytrope of the Jones et al.
    # hydrodynamic benchmark (Benchmarking.F90:202-247)
    ANEL,
    dict(ANEL, nu_type=2, nu_power=-0.5, kappa_type=2, kappa_power=-0.5, no_slip_bottom=True),
    dict(n_r=32, l_max=7, dt=30.0, reference_type=2, shell_depth=4.55e9, aspect_ratio=0.35, poly_n=2.0,
         poly_nrho=5.0, poly_mass=1.9e30, poly_rho_i=1.1, pressure_specific_heat=1.0509e8,
         angular_velocity=1.76e-4, nu_top=3.64364e12, kappa_top=3.64364e12, no_slip_top=False,
         no_slip_bottom=False, t_bottom=851225.7),
    # the finite-difference radial mode (uniform grid, 5-point stencils): no-slip and stress-free
    dict(n_r=48, l_max=7, dt=1e-4, chebyshev=False),
    dict(n_r=32, l_max=7, dt=1e-4, chebyshev=False, no_slip_top=False, no_slip_bottom=False,
         fix_tvar_bottom=False, dtdr_bottom=-1.0),
])
def test_build_matrices_match_oracle(cfg):
    import rayleigh_b200 as rb
    oc = O.Config(**cfg)
    o = O.Oracle(oc)
    L = oc.l_max + 1
    rc = rb.Config(**cfg)
    wpt, cw = rb.build_matrices(rc, 0, 0, L, coefs=True)
    z = rb.build_matrices(rc, 1, 1, L - 1)
    for l in range(L):
        ref = o.mat_wpt[l]
        got = wpt[l].T                          # column-major per l
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-13 * scale, l
        if l > 0:
            assert np.abs(z[l - 1].T - o.mat_z[l]).max() <= 1e-13 * np.abs(o.mat_z[l]).max(), l
        for s, key in enumerate(_slots()):
            ref_c = o.coefs[l].get(key)
            if ref_c is None:
                assert not np.any(cw[l, s]), (l, key)
            else:
                np.testing.assert_allclose(cw[l, s], ref_c, rtol=1e-13, atol=1e-15 * np.abs(ref_c).max())


def test_build_matrices_argument_errors():
    import rayleigh_b200 as rb
    rc = rb.Config(n_r=24, l_max=7)
    with pytest.raises(rb.RayleighError):
        rb.build_matrices(rc, 0, 5, 4)       # l beyond l_max
    with pytest.raises(rb.RayleighError):
        rb.build_matrices(rb.Config(n_r=7, l_max=7), 0, 0, 1)


@pytest.mark.parametrize("n_r,anelastic,chebyshev", [(24, False, True), (128, False, True), (32, True, True),
                                                     (32, False, False)])
def test_build_magnetic_matrices_match_oracle(n_r, anelastic, chebyshev):
    """The C (poloidal) and A (toroidal) systems of the dynamo equation set with the
    insulating (potential-field) boundary rows (Sphere_Linear_Terms.F90:473-499, 1041-1077)
    and their Post_Solve coefficients; on the polytrope with a density-dependent eta the
    A equation carries A_Diffusion_Coefs_1 = eta dln(eta)/dr."""
    import rayleigh_b200 as rb
    cfg = dict(n_r=n_r, l_max=7, dt=2e-4, ekman=1e-3, rayleigh=1e5, magnetism=True, magnetic_prandtl=5.0)
    if anelastic:
        cfg.update(ANEL, n_r=n_r, magnetism=True, magnetic_prandtl=2.0, eta_type=2, eta_power=-0.5)
    cfg["chebyshev"] = chebyshev
    o = O.Oracle(O.Config(**cfg))
    L = 8
    rc = rb.Config(**cfg)
    cm, cc = rb.build_matrices(rc, 2, 1, L - 1, coefs=True)
    am, ac = rb.build_matrices(rc, 3, 1, L - 1, coefs=True)
    C, A = O.CVAR, O.AVAR
    for l in range(1, L):
        for got, ref in ((cm[l - 1].T, o.mat_c[l]), (am[l - 1].T, o.mat_a[l])):
            assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), l
        for s, d in enumerate((0, 2)):
            ref_c = o.coefs[l][(O.CEQ, C, d)]
            np.testing.assert_allclose(cc[l - 1, s], ref_c, rtol=1e-13, atol=1e-15 * np.abs(ref_c).max())
        for s, d in enumerate((0, 1, 2)):
            ref_c = o.coefs[l][(O.AEQ, A, d)]
            np.testing.assert_allclose(ac[l - 1, s], ref_c, rtol=1e-13, atol=1e-15 * np.abs(ref_c).max())
    with pytest.raises(rb.RayleighError):   # no magnetic systems without magnetism
        rb.build_matrices(rb.Config(n_r=24, l_max=7), 2, 1, 2)
