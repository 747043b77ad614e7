"""CPU tests of the oracle (the parity checker) against the reference's own
NumPy port (committed golden fixtures) and the known answers of
src/Test_Suite/Test_SHT.F90."""
import math
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "sht_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("lmax,nth", [(15, 24), (41, 64), (63, 96)])
def test_plm_tables_match_reference_port(gold, lmax, nth):
    # with the port's Newton tolerance the restatement reproduces it to rounding
    h = O.Horizontal(lmax, nth, eps="3e-15")
    tag = f"l{lmax}"
    assert np.array_equal(h.xq.astype(np.float64), gold[tag + "_x"])
    assert np.array_equal(h.wq.astype(np.float64), gold[tag + "_w"])
    for m in gold[tag + "_ms"]:
        for name, mine in (("p_lm_even", h.p_even), ("p_lm_odd", h.p_odd),
                           ("ip_lm_even", h.ip_even), ("ip_lm_odd", h.ip_odd)):
            k = f"{tag}_{name}_{m}"
            if k in gold:
                ref = gold[k]
                assert np.abs(mine[m] - ref).max() <= 1e-14 * np.abs(ref).max()
    # with the Fortran tolerance (3e-14) the weights differ by O(eps): tables agree to 1e-12
    h2 = O.Horizontal(lmax, nth)
    for m in gold[tag + "_ms"]:
        k = f"{tag}_ip_lm_even_{m}"
        ref = gold[k]
        assert np.abs(h2.ip_even[m] - ref).max() <= 1e-12 * np.abs(ref).max()


def _spec_to_s2(spec, lmax):
    nk = spec.shape[2]
    out = []
    for m in range(lmax + 1):
        a = np.zeros((nk, 2, 1, lmax - m + 1))
        a[:, 0, 0, :] = spec[m:, m, :].real.T
        a[:, 1, 0, :] = spec[m:, m, :].imag.T
        out.append(a)
    return out


@pytest.mark.parametrize("lmax,nth", [(15, 24), (41, 64), (63, 96)])
def test_legendre_transforms_match_reference_port(gold, lmax, nth):
    h = O.Horizontal(lmax, nth, eps="3e-15")
    tag = f"l{lmax}"
    spec = gold[tag + "_spec_in"]
    p2 = h.s2p(_spec_to_s2(spec, lmax))
    mine = np.stack([p2[m][:, 0, 0, :].T + 1j * p2[m][:, 1, 0, :].T for m in range(lmax + 1)], axis=1)
    ref = gold[tag + "_hyb_out"]
    assert np.abs(mine - ref).max() <= 1e-14 * np.abs(ref).max()
    hin = gold[tag + "_hyb_in"]
    nk = hin.shape[2]
    p2in = []
    for m in range(lmax + 1):
        a = np.zeros((nk, 2, 1, nth))
        a[:, 0, 0, :] = hin[:, m, :].real.T
        a[:, 1, 0, :] = hin[:, m, :].imag.T
        p2in.append(a)
    s2 = h.p2s(p2in)
    ref = gold[tag + "_spec_out"]
    mine = np.zeros_like(ref)
    for m in range(lmax + 1):
        mine[m:, m, :] = (s2[m][:, 0, 0, :] + 1j * s2[m][:, 1, 0, :]).T
    assert np.abs(mine - ref).max() <= 1e-14 * np.abs(ref).max()


def test_single_mode_known_answer():
    """Test_SHT.F90:47-200: Y_2^1 with (2f+1) r and -(3f^2+2) r^2 amplitudes."""
    lmax, nth = 41, 64
    h = O.Horizontal(lmax, nth)
    nf, nr = 3, 4
    radius = np.linspace(0.5, 1.5, nr)
    s2 = [np.zeros((nf, 2, nr, lmax - m + 1)) for m in range(lmax + 1)]
    for f in range(1, nf + 1):
        s2[1][f - 1, 0, :, 1] = (2 * f + 1) * radius * 2.0          # norm = 1/to_phys_norm (m=1)
        s2[1][f - 1, 1, :, 1] = -(3 * f * f + 2) * radius ** 2 * 2.0
    p2 = h.s2p(s2)
    true = math.sqrt(5.0 / (4.0 * math.pi * 6.0)) * (-3.0 * h.costheta * h.sintheta)
    for f in range(1, nf + 1):
        np.testing.assert_allclose(p2[1][f - 1, 0], np.outer((2 * f + 1) * radius, true), rtol=0, atol=1e-12 * 40)
        np.testing.assert_allclose(p2[1][f - 1, 1], np.outer(-(3 * f * f + 2) * radius ** 2, true), rtol=0,
                                   atol=1e-12 * 40)
    back = h.p2s(p2)
    # undo the FFT normalisations folded into the tables (Test_SHT.F90:67-73)
    for m in range(lmax + 1):
        back[m] = back[m] * (nth if m else 2 * nth) * (0.5 if m else 1.0) ** -1 / (nth if m else 2 * nth)
    for f in range(1, nf + 1):
        got = back[1][f - 1, 0, :, 1] / (1.0 / nth)
        np.testing.assert_allclose(got, (2 * f + 1) * radius * 2.0, rtol=1e-10)


def test_white_noise_round_trip():
    """Test_SHT.F90:328-447: every mode, s -> p -> s reproduces the input (l < l_max)."""
    lmax, nth = 31, 48
    h = O.Horizontal(lmax, nth)
    rng = np.random.Generator(np.random.PCG64(7))
    s2 = [rng.standard_normal((2, 2, 3, lmax - m + 1)) for m in range(lmax + 1)]
    back = h.p2s(h.s2p(s2))
    for m in range(lmax + 1):
        norm = (1.0 * (1.0 / (2 * nth))) if m == 0 else (0.5 * (1.0 / nth))
        np.testing.assert_allclose(back[m] / norm, s2[m], rtol=1e-10, atol=1e-10)


def test_fft_conventions():
    n = 24
    rng = np.random.Generator(np.random.PCG64(3))
    y = np.zeros((5, n + 2))
    y[:, :n] = rng.standard_normal((5, n))
    X = O.fft_r2c(y, n)
    direct = np.array([[np.sum(y[i, :n] * np.exp(-2j * np.pi * k * np.arange(n) / n)) for k in range(n // 2 + 1)]
                       for i in range(5)])
    np.testing.assert_allclose(X[:, 0::2], direct.real, atol=1e-12)
    np.testing.assert_allclose(X[:, 1::2], direct.imag, atol=1e-12)
    back = O.fft_c2r(X, n)
    np.testing.assert_allclose(back[:, :n], n * y[:, :n], atol=1e-11)


def test_chebyshev_round_trip_and_derivative():
    cg = O.Chebyshev(32, 0.5, 1.5)
    r = cg.radius
    f = r ** 3 - 2 * r
    c = cg.to_spectral(f[None])[0]
    np.testing.assert_allclose(cg.from_spectral(c[None])[0], f, atol=1e-13)
    d1 = cg.from_spectral(cg.deriv(c[None], 1))[0]
    np.testing.assert_allclose(d1, 3 * r ** 2 - 2, atol=1e-11)
    d2 = cg.from_spectral(cg.deriv(c[None], 2))[0]
    np.testing.assert_allclose(d2, 6 * r, atol=1e-9)
    # the derivative matrices reproduce the recursion
    np.testing.assert_allclose(cg.dcheby[1] @ c, d1, atol=1e-11)


def test_conduction_state_is_steady():
    cfg = O.Config(n_r=40, l_max=7, dt=1e-3)   # 1/r is resolved below the dealiasing cut
    o = O.Oracle(cfg)
    wpt, z = O.seeded_state(cfg, amp=0.0)
    o.init_state(wpt, z)
    t0 = o.rhs_wpt[:, :, 2 * cfg.n_r:].copy()
    for _ in range(3):
        o.step()
    assert np.abs(o.rhs_wpt[:, :, 2 * cfg.n_r:] - t0).max() < 1e-12
    assert np.abs(o.rhs_wpt[:, :, :cfg.n_r]).max() == 0.0
    assert np.abs(o.rhs_z).max() == 0.0


def test_perturbation_evolves_and_stays_finite():
    cfg = O.Config(n_r=16, l_max=15, dt=1e-4)
    o = O.Oracle(cfg)
    wpt, z = O.seeded_state(cfg, amp=1e-2, lmax_pert=8)
    o.init_state(wpt, z)
    for _ in range(4):
        cfl = o.step()
    assert np.isfinite(o.rhs_wpt).all() and np.isfinite(o.rhs_z).all()
    assert np.abs(o.rhs_wpt[:, :, :cfg.n_r]).max() > 0.0      # buoyancy drives W
    assert cfl > 0.0


@pytest.mark.parametrize("golden", ["c2001_case0.json", "c2001_case0_fd_uniform.json"])
def test_c2001_case0_matches_the_reference_regression_report(golden):
    """The reference's own regression runs of its accuracy benchmark
    (tests/c2001_case0: Christensen et al. 2001 case 0 from Benchmark_Init_Hydro,
    N_r = 48, N_theta = 64, 400 steps of dt = 1e-4, alpha = 0.50001; and
    tests/c2001_case0_FD_uniform, the same run in the finite-difference radial mode on
    its uniform grid): mean and standard deviation of the volume-averaged kinetic
    energy at iterations 100, 200, 300, 400, and of the point observations T and
    v_phi where v_r = 0 at mid-depth on the equator, as each run's
    Benchmark_Reports/00000400 prints them (6 decimals).  This pins the oracle's whole
    time step, not only its transforms, in both radial discretisations."""
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", golden)))
    cfg = O.c2001_case0_config(gold["n_r"], gold["n_theta"], chebyshev=gold.get("chebyshev", True))
    o = O.Oracle(cfg)
    wpt, z = o.benchmark_init_hydro()
    o.init_state(wpt, z)
    samples = {"Kinetic Energy": [], "Vphi": [], "Temperature": []}
    for it in range(1, gold["max_iterations"] + 1):
        o.step()
        if it % gold["integration_interval"] == 0:
            samples["Kinetic Energy"].append(o.benchmark_kinetic_energy())
            vphi, temp = o.benchmark_point_observations()
            samples["Vphi"].append(vphi)
            samples["Temperature"].append(temp)
    for name, vals in samples.items():
        vals = np.array(vals)
        ref = gold["observables"][name]
        assert len(vals) == gold["samples"]
        assert abs(vals.mean() - ref["measured"]) < 5e-6, (name, vals.mean(), ref)
        assert abs(vals.std() - ref["sdev"]) < 5e-6, (name, vals.std(), ref)


def _spectral_d(o, f, d):
    c = o.cg.to_spectral(f[None, None, :])
    return o.cg.from_spectral(o.cg.deriv(c, d))[0, 0]


def test_nondimensional_polytrope_known_answers():
    """Polytropic_ReferenceND (PDE_Coefficients.F90:437-537): T = rho = 1 at the outer
    radius, rho(r_i) / rho(r_o) = exp(N_rho), the adiabatic gradient dT/dr = -D g with
    D = beta (exp(N_rho / n) - 1), and dln(rho)/dr, d2ln(rho)/dr2 the derivatives of ln rho."""
    o = O.Oracle(O.anelastic_mhd_config(n_r=64, l_max=7))
    cfg = o.cfg
    assert abs(o.temperature[0] - 1.0) < 1e-14 and abs(o.density[0] - 1.0) < 1e-14
    assert abs(o.density[-1] / o.density[0] - math.exp(cfg.poly_nrho)) < 1e-12 * math.exp(cfg.poly_nrho)
    diss = cfg.aspect_ratio * (math.exp(cfg.poly_nrho / cfg.poly_n) - 1.0)
    g = o.rmax ** 2 / o.radius ** 2
    np.testing.assert_allclose(_spectral_d(o, o.temperature, 1), -diss * g, rtol=1e-9)
    lr = np.log(o.density)
    np.testing.assert_allclose(_spectral_d(o, lr, 1), o.dlnrho, rtol=1e-9)
    np.testing.assert_allclose(_spectral_d(o, lr, 2), o.d2lnrho, rtol=1e-7)
    # Boussinesq limits of the anelastic coefficients vanish; here they do not
    assert np.abs(o.w_diff0).max() > 0 and np.abs(o.s_diff1).max() > 0


def test_dimensional_polytrope_is_hydrostatic():
    """Polytropic_Reference (PDE_Coefficients.F90:925-1051) on the Jones et al. benchmark's
    values: rho(r_i) = poly_rho_i, rho(r_i) / rho(r_o) = exp(N_rho), and the ideal-gas
    pressure P = c_P rho T / (n + 1) is in hydrostatic balance, dP/dr = -rho G M / r^2."""
    cfg = O.Config(n_r=64, l_max=7, reference_type=2, shell_depth=4.55e9, aspect_ratio=0.35, poly_n=2.0,
                   poly_nrho=5.0, poly_mass=1.9e30, poly_rho_i=1.1, pressure_specific_heat=1.0509e8,
                   angular_velocity=1.76e-4, nu_top=3.64364e12, kappa_top=3.64364e12, dt=30.0)
    o = O.Oracle(cfg)
    assert abs(o.density[-1] - 1.1) < 1e-13
    assert abs(o.density[-1] / o.density[0] - math.exp(5.0)) < 1e-11 * math.exp(5.0)
    P = cfg.pressure_specific_heat * o.density * o.temperature / (cfg.poly_n + 1.0)
    g = 6.67e-8 * cfg.poly_mass / o.radius ** 2
    np.testing.assert_allclose(_spectral_d(o, P, 1), -o.density * g, rtol=1e-8)
    np.testing.assert_allclose(_spectral_d(o, np.log(o.density), 1), o.dlnrho, rtol=1e-9)
    np.testing.assert_allclose(_spectral_d(o, np.log(o.temperature), 1), o.dlnT, rtol=1e-9)
    np.testing.assert_allclose(_spectral_d(o, np.log(o.density), 2), o.d2lnrho, rtol=1e-7)


def _t_nonlinear(o, wpt, z, c=None, a=None):
    """T's nonlinear term of one physical-space stage from a state (spectral, per m)."""
    o.init_state(wpt, z, c_coeffs=c, a_coeffs=a)
    s2a = o.transpose_1a2a(o.post_solve())
    p3b = o.physical_space(o.transpose_2a3a(o.h.s2p(o.rlm_spacea(s2a))))
    return p3b[O.TVAR]


def test_anelastic_viscous_heating_of_rotations():
    """Compute_Viscous_Heating (Sphere_Physical_Space.F90:337-443) on the polytrope: a
    solid-body rotation about the polar axis (Z_10 proportional to rho r^2, so that
    v_phi = Omega r sin(theta)) has no strain and heats nothing, while a differential
    rotation (Z_10 proportional to rho r^3) heats; T has no angular structure and
    v_r = 0, so advection adds nothing to T's term."""
    oc = O.anelastic_mhd_config(n_r=64, l_max=15, magnetism=False)
    o = O.Oracle(oc)
    assert o.viscous_heating_coeff is not None and np.all(o.viscous_heating_coeff > 0)
    wpt, _ = O.seeded_state(oc, amp=0.0)
    r = o.radius
    out = []
    for p in (2, 3):
        z = np.zeros((o.n_lm, 2, oc.n_r))
        z[1, 0] = o.cg.to_spectral((1e-3 * o.density * r ** p)[None, None, :])[0, 0]   # lm(1, 0) = 1
        out.append(np.abs(_t_nonlinear(o, wpt, z)).max())
    assert out[1] > 0 and out[0] < 1e-9 * out[1], out


def test_anelastic_heating_coefficients():
    """Both heating terms are on for the polytropes (Controls.F90:64-65) with positive
    coefficients, and off for the Boussinesq reference (Constant_Reference)."""
    o = O.Oracle(O.anelastic_mhd_config(n_r=24, l_max=15))
    assert np.all(o.viscous_heating_coeff > 0) and np.all(o.ohmic_heating_coeff > 0)
    b = O.Oracle(O.Config(n_r=24, l_max=15, magnetism=True))
    assert b.viscous_heating_coeff is None and b.ohmic_heating_coeff is None
