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


def test_c2001_case0_matches_the_reference_regression_report():
    """The reference's own regression run of its accuracy benchmark
    (tests/c2001_case0: Christensen et al. 2001 case 0 from Benchmark_Init_Hydro,
    N_r = 48, N_theta = 64, 400 steps of dt = 1e-4, alpha = 0.50001): mean and
    standard deviation of the volume-averaged kinetic energy at iterations 100,
    200, 300, 400, and of the point observations T and v_phi where v_r = 0 at
    mid-depth on the equator, as its Benchmark_Reports/00000400 prints them (6
    decimals).  This pins the oracle's whole time step, not only its transforms."""
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "c2001_case0.json")))
    cfg = O.c2001_case0_config(gold["n_r"], gold["n_theta"])
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
