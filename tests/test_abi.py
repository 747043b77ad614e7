"""The C-ABI library loads and exports every symbol that include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?(?:int|long|void|char)\s*\**\s*(ra_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("ra_create", "ra_step", "ra_post_solve", "ra_rlm_a", "ra_physical", "ra_rlm_b", "ra_advance",
                 "ra_legendre_s2p", "ra_legendre_p2s", "ra_fft_c2r", "ra_fft_r2c", "ra_set_dt"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from rayleigh_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_default_config_and_argument_errors_without_gpu():
    import rayleigh_b200 as rb
    lib = rb.load_library()
    cfg = rb._Config()
    assert lib.ra_default_config(ctypes.byref(cfg)) == 0
    assert cfg.n_r == 48 and cfg.l_max == 63 and abs(cfg.alpha_implicit - 0.5) < 1e-15
    assert lib.ra_default_config(None) == rb.RA_ERR_ARG
    # a context-less call reports a state error instead of touching the device
    assert lib.ra_step(None, 1, None) == rb.RA_ERR_STATE
    # an invalid configuration is rejected before any CUDA call
    bad = rb.Config(n_r=7).to_c()
    h = ctypes.c_void_p()
    assert lib.ra_create(ctypes.byref(h), ctypes.byref(bad)) == rb.RA_ERR_ARG
    buf = ctypes.create_string_buffer(256)
    lib.ra_last_error(h, buf, 256)
    assert b"n_r" in buf.value
    lib.ra_destroy(h)


def test_config_layout_and_defaults_agree():
    """The Python dataclass, its ctypes mirror and ra_default_config describe the same
    struct: every field of the C defaults equals the dataclass default."""
    import dataclasses
    import rayleigh_b200 as rb
    lib = rb.load_library()
    c = rb._Config()
    assert lib.ra_default_config(ctypes.byref(c)) == 0
    names = [f[0] for f in rb._Config._fields_]
    assert names == [f.name for f in dataclasses.fields(rb.Config)]
    py = rb.Config().to_c()
    for n in names:
        assert getattr(c, n) == getattr(py, n), n


def test_contextless_calls_of_the_newer_entry_points():
    """ra_set_reference, ra_transform_dev and ra_step_adaptive without a context report a state
    error before touching a device."""
    import rayleigh_b200 as rb
    lib = rb.load_library()
    assert lib.ra_set_reference(None, None, None, None, None, 0.0, 0.0) == rb.RA_ERR_STATE
    assert lib.ra_transform_dev(None, 0, 0, None, None, None, 1, None) == rb.RA_ERR_STATE
    ctl = rb.DtControls().to_c()
    assert lib.ra_step_adaptive(None, 1, ctypes.byref(ctl), None, None) == rb.RA_ERR_STATE


def test_reference_state_arguments_are_checked():
    import rayleigh_b200 as rb
    lib = rb.load_library()
    for kw, word in ((dict(reference_type=4), b"reference_type"), (dict(reference_type=3), b"poly"),
                     (dict(reference_type=3, poly_n=2.0, poly_nrho=5.0), b"modified_rayleigh"),
                     (dict(reference_type=2, poly_n=2.0, poly_nrho=5.0), b"poly_mass"),
                     (dict(nu_type=3), b"transport")):
        cfg = rb.Config(**kw).to_c()
        h = ctypes.c_void_p()
        assert lib.ra_create(ctypes.byref(h), ctypes.byref(cfg)) == rb.RA_ERR_ARG, kw
        buf = ctypes.create_string_buffer(256)
        lib.ra_last_error(h, buf, 256)
        assert word in buf.value, (kw, buf.value)
        lib.ra_destroy(h)


def test_diagnostic_quantity_codes_are_the_references():
    """RA_Q_* in the header, the Python names and the reference's output codes
    (velocity_field_codes.F: voffset = 0; vorticity_field_codes.F: vort_off = 300;
    thermal_field_codes.F: pt_off = 500; magnetic_field_codes.F: boffset = teoffset + 100 = 800;
    current_density_codes.F: joffset = boffset + 200)
    agree; context-less diagnostic calls report a state error."""
    import rayleigh_b200 as rb
    src = open(os.path.join(ROOT, "include", "rayleigh_b200.h")).read()
    header = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(r"#define RA_Q_(\w+)\s+(\d+)", src)}
    assert header == rb.Rayleigh.QUANTITIES
    reference = {"v_r": 1, "v_theta": 2, "v_phi": 3, "dv_r_dr": 10, "dv_theta_dr": 11, "dv_phi_dr": 12,
                 "dv_r_dt": 19, "dv_r_dp": 28, "dv_theta_dp": 29, "dv_phi_dp": 30, "vort_r": 300 + 1,
                 "entropy": 500 + 1, "entropy_dr": 500 + 7, "entropy_dtheta": 500 + 13, "entropy_dphi": 500 + 19,
                 "pressure": 500 + 2, "pressure_dr": 500 + 8, "pressure_dphi": 500 + 20,
                 "b_r": 800 + 1, "b_theta": 800 + 2, "b_phi": 800 + 3,
                 "j_r": 800 + 200 + 1, "j_theta": 800 + 200 + 4, "j_phi": 800 + 200 + 7,
                 "vp_r": 4, "vp_theta": 5, "vp_phi": 6, "vm_r": 7, "vm_theta": 8, "vm_phi": 9,
                 "dvp_r_dr": 13, "dvp_theta_dr": 14, "dvp_phi_dr": 15, "dvm_r_dr": 16, "dvm_theta_dr": 17,
                 "dvm_phi_dr": 18, "dvp_r_dt": 22, "dvm_r_dt": 25, "dv_theta_dt": 20, "dv_phi_dt": 21,
                 "dvp_theta_dt": 23, "dvp_phi_dt": 24, "dvm_theta_dt": 26, "dvm_phi_dt": 27, "dvp_r_dp": 31, "dvp_theta_dp": 32,
                 "dvp_phi_dp": 33, "dvm_r_dp": 34, "dvm_theta_dp": 35, "dvm_phi_dp": 36,
                 "vortp_r": 300 + 4, "vortm_r": 300 + 7, "vort_theta": 300 + 2, "vort_phi": 300 + 3,
                 "vortp_theta": 300 + 5, "vortp_phi": 300 + 6, "vortm_theta": 300 + 8, "vortm_phi": 300 + 9,
                 "entropy_p": 500 + 3, "pressure_p": 500 + 4, "entropy_m": 500 + 5, "pressure_m": 500 + 6,
                 "entropy_p_dr": 500 + 9, "pressure_p_dr": 500 + 10, "entropy_m_dr": 500 + 11,
                 "pressure_m_dr": 500 + 12, "entropy_p_dtheta": 500 + 15, "entropy_m_dtheta": 500 + 17,
                 "entropy_p_dphi": 500 + 21, "pressure_p_dphi": 500 + 22, "entropy_m_dphi": 500 + 23,
                 "pressure_m_dphi": 500 + 24,
                 "bp_r": 800 + 4, "bp_theta": 800 + 5, "bp_phi": 800 + 6, "bm_r": 800 + 7, "bm_theta": 800 + 8,
                 "bm_phi": 800 + 9, "jp_r": 1000 + 2, "jm_r": 1000 + 3, "jp_theta": 1000 + 5, "jm_theta": 1000 + 6,
                 "jp_phi": 1000 + 8, "jm_phi": 1000 + 9, "db_r_dp": 800 + 28, "db_theta_dp": 800 + 29,
                 "db_phi_dp": 800 + 30, "dbp_r_dp": 800 + 31, "dbp_theta_dp": 800 + 32, "dbp_phi_dp": 800 + 33,
                 "dbm_r_dp": 800 + 34, "dbm_theta_dp": 800 + 35, "dbm_phi_dp": 800 + 36}
    # kinetic_energy_codes.F: keoffset = vort_off + 100; magnetic_energy_codes.F: meoffset = joffset + 100
    reference.update({"kinetic_energy": 400 + 1, "radial_ke": 400 + 2, "theta_ke": 400 + 3,
                      "phi_ke": 400 + 4, "mkinetic_energy": 400 + 5, "radial_mke": 400 + 6,
                      "theta_mke": 400 + 7, "phi_mke": 400 + 8, "pkinetic_energy": 400 + 9,
                      "radial_pke": 400 + 10, "theta_pke": 400 + 11, "phi_pke": 400 + 12, "vsq": 400 + 13,
                      "radial_vsq": 400 + 14, "theta_vsq": 400 + 15, "phi_vsq": 400 + 16, "mvsq": 400 + 17,
                      "radial_mvsq": 400 + 18, "theta_mvsq": 400 + 19, "phi_mvsq": 400 + 20,
                      "pvsq": 400 + 21, "radial_pvsq": 400 + 22, "theta_pvsq": 400 + 23,
                      "phi_pvsq": 400 + 24})
    reference.update({"j_sq": 1000 + 10, "jp_sq": 1000 + 11, "jm_sq": 1000 + 12, "j_r_sq": 1000 + 14,
                      "jp_r_sq": 1000 + 15, "jm_r_sq": 1000 + 16, "j_theta_sq": 1000 + 17,
                      "jp_theta_sq": 1000 + 18, "jm_theta_sq": 1000 + 19, "j_phi_sq": 1000 + 20,
                      "jp_phi_sq": 1000 + 21, "jm_phi_sq": 1000 + 22})
    reference.update({"magnetic_energy": 1100 + 1, "radial_me": 1100 + 2, "theta_me": 1100 + 3,
                      "phi_me": 1100 + 4, "mmagnetic_energy": 1100 + 5, "radial_mme": 1100 + 6,
                      "theta_mme": 1100 + 7, "phi_mme": 1100 + 8, "pmagnetic_energy": 1100 + 9,
                      "radial_pme": 1100 + 10, "theta_pme": 1100 + 11, "phi_pme": 1100 + 12})
    # mass_flux_codes.F: rhovoffset = voffset + 200
    reference.update({"rhov_r": 200 + 1, "rhov_theta": 200 + 2, "rhov_phi": 200 + 3, "rhovp_r": 200 + 4,
                      "rhovp_theta": 200 + 5, "rhovp_phi": 200 + 6, "rhovm_r": 200 + 7, "rhovm_theta": 200 + 8,
                      "rhovm_phi": 200 + 9})
    # thermal_energy_codes.F: teoffset = pt_off + 200
    reference.update({"thermal_energy_full": 700 + 1, "thermal_energy_p": 700 + 2, "thermal_energy_m": 700 + 3,
                      "thermal_energy_sq": 700 + 7, "thermal_energyp_sq": 700 + 8, "thermal_energym_sq": 700 + 9})
    # vorticity_field_codes.F: enstrophy = vort_off + 10 ... kin_helicity_pm = vort_off + 43
    reference.update({"enstrophy": 300 + 10, "enstrophy_pm": 300 + 11, "enstrophy_mm": 300 + 12,
                      "enstrophy_pp": 300 + 13, "vort_r_sq": 300 + 14, "vort_theta_sq": 300 + 15,
                      "vort_phi_sq": 300 + 16, "vortp_r_sq": 300 + 17, "vortp_theta_sq": 300 + 18,
                      "vortp_phi_sq": 300 + 19, "vortm_r_sq": 300 + 20, "vortm_theta_sq": 300 + 21,
                      "vortm_phi_sq": 300 + 22, "kin_helicity_r": 300 + 24, "kin_helicity_theta": 300 + 25,
                      "kin_helicity_phi": 300 + 26, "kin_helicity_pp_r": 300 + 27,
                      "kin_helicity_pp_theta": 300 + 28, "kin_helicity_pp_phi": 300 + 29,
                      "kin_helicity_mm_r": 300 + 30, "kin_helicity_mm_theta": 300 + 31,
                      "kin_helicity_mm_phi": 300 + 32, "kin_helicity_mp_r": 300 + 33,
                      "kin_helicity_mp_theta": 300 + 34, "kin_helicity_mp_phi": 300 + 35,
                      "kin_helicity_pm_r": 300 + 36, "kin_helicity_pm_theta": 300 + 37,
                      "kin_helicity_pm_phi": 300 + 38, "kin_helicity": 300 + 39,
                      "kin_helicity_pp": 300 + 40, "kin_helicity_mm": 300 + 41,
                      "kin_helicity_mp": 300 + 42, "kin_helicity_pm": 300 + 43, "jpm_sq": 1000 + 13})
    assert header == reference
    lib = rb.load_library()
    ke = ctypes.c_double()
    assert lib.ra_kinetic_energy(None, ctypes.byref(ke)) == rb.RA_ERR_STATE
    q = (ctypes.c_int * 1)(1)
    assert lib.ra_shell_slices(None, q, 1, q, 1, None) == rb.RA_ERR_STATE
    assert lib.ra_shell_averages(None, q, 1, None) == rb.RA_ERR_STATE
    assert lib.ra_azimuthal_averages(None, q, 1, None) == rb.RA_ERR_STATE
    assert lib.ra_shell_spectra(None, q, 1, q, 1, None) == rb.RA_ERR_STATE
    assert lib.ra_equatorial_slices(None, q, 1, None) == rb.RA_ERR_STATE
    assert lib.ra_meridional_slices(None, q, 1, q, 1, None) == rb.RA_ERR_STATE
    assert lib.ra_global_averages(None, q, 1, None) == rb.RA_ERR_STATE
    assert lib.ra_point_probes(None, q, 1, q, 1, q, 1, q, 1, None) == rb.RA_ERR_STATE


def test_cfl_time_step_control_without_gpu():
    """ra_next_dt restates Adjust_TimeStep (Sphere_Hybrid_Space.F90:604-649): grow to
    cflmax * t_cross (capped by max_time_step) when dt < cflmin * t_cross, shrink to
    cflmax * t_cross, by at least min_dt_change, when dt > cflmax * t_cross, else keep dt."""
    import rayleigh_b200 as rb
    ctl = rb.DtControls(max_time_step=1e-4)
    t = 1e-3                                   # crossing time: cfl cargo = 1 / t^2
    cfl = 1.0 / t ** 2
    assert rb.next_dt(ctl, 1e-5, cfl) == 1e-4                  # grows, capped by max_time_step
    assert rb.next_dt(rb.DtControls(), 1e-5, cfl) == 0.6 * t   # grows to cflmax * t
    assert rb.next_dt(rb.DtControls(), 0.5 * t, cfl) == 0.5 * t   # inside [cflmin, cflmax]: kept
    assert rb.next_dt(rb.DtControls(), 0.62 * t, cfl) == 0.62 * t * 0.9   # small decrease bumped to 10 %
    assert abs(rb.next_dt(rb.DtControls(), 2.0 * t, cfl) - 0.6 * t) < 1e-18
    assert rb.next_dt(ctl, 5e-5, 0.0) == 5e-5                   # no cargo: kept
    with pytest.raises(rb.RayleighError):
        rb.next_dt(rb.DtControls(min_time_step=1e-3), 2.0 * t, cfl)
