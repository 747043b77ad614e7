"""rayleigh_b200 -- B200 (sm_100a) implementation of Rayleigh's per-timestep
spectral-transform + implicit-solve path, behind the C ABI declared in
``include/rayleigh_b200.h``.

This module is the Python mirror of the host side: it loads the in-tree
``librayleigh_b200.so`` through ctypes and exposes the stage calls that the
reference's main loop makes (``Post_Solve``, ``rlm_spacea``,
``physical_space``, ``rlm_spaceb``, ``AdvanceTime``; Sphere_Driver.F90:305-328)
and the math-layer operators (Legendre transforms, phi FFTs, Chebyshev
transforms).  There is no CPU fallback: if the shared library or a CUDA device
is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, fields

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librayleigh_b200.so")

RA_OK = 0
RA_ERR_ARG = -1
RA_ERR_CUDA = -2
RA_ERR_SINGULAR = -3
RA_ERR_NOMEM = -4
RA_ERR_STATE = -5
RA_ERR_NONFINITE = -6
PREC_FP64 = 0
PREC_MIXED = 1


class RayleighError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rayleigh_b200 error {code}: {msg}")
        self.code = code


class _Config(ctypes.Structure):
    _fields_ = [
        ("n_r", ctypes.c_int), ("l_max", ctypes.c_int), ("n_theta", ctypes.c_int),
        ("aspect_ratio", ctypes.c_double), ("shell_depth", ctypes.c_double),
        ("rayleigh", ctypes.c_double), ("ekman", ctypes.c_double), ("prandtl", ctypes.c_double),
        ("magnetic_prandtl", ctypes.c_double), ("gravity_power", ctypes.c_double),
        ("rotation", ctypes.c_int), ("magnetism", ctypes.c_int),
        ("no_slip_top", ctypes.c_int), ("no_slip_bottom", ctypes.c_int),
        ("fix_tvar_top", ctypes.c_int), ("fix_tvar_bottom", ctypes.c_int),
        ("t_top", ctypes.c_double), ("t_bottom", ctypes.c_double),
        ("dtdr_top", ctypes.c_double), ("dtdr_bottom", ctypes.c_double),
        ("dt", ctypes.c_double), ("alpha_implicit", ctypes.c_double),
        ("precision", ctypes.c_int), ("use_graph", ctypes.c_int), ("device", ctypes.c_int),
        ("autotune", ctypes.c_int),
        ("reference_type", ctypes.c_int),
        ("poly_n", ctypes.c_double), ("poly_nrho", ctypes.c_double), ("poly_mass", ctypes.c_double),
        ("poly_rho_i", ctypes.c_double), ("pressure_specific_heat", ctypes.c_double),
        ("angular_velocity", ctypes.c_double), ("modified_rayleigh", ctypes.c_double),
        ("nu_type", ctypes.c_int), ("kappa_type", ctypes.c_int), ("eta_type", ctypes.c_int),
        ("nu_power", ctypes.c_double), ("kappa_power", ctypes.c_double), ("eta_power", ctypes.c_double),
        ("nu_top", ctypes.c_double), ("kappa_top", ctypes.c_double), ("eta_top", ctypes.c_double),
        ("viscous_heating", ctypes.c_int), ("ohmic_heating", ctypes.c_int),
        ("chebyshev", ctypes.c_int),
    ]


class _DtControls(ctypes.Structure):
    _fields_ = [("cflmin", ctypes.c_double), ("cflmax", ctypes.c_double), ("max_time_step", ctypes.c_double),
                ("min_time_step", ctypes.c_double), ("min_dt_change", ctypes.c_double)]


@dataclass
class DtControls:
    """Temporal_Controls of the CFL time-step control (Controls.F90:113-115, ClockInfo.F90:27)."""

    cflmin: float = 0.4
    cflmax: float = 0.6
    max_time_step: float = 1.0
    min_time_step: float = 1.0e-13
    min_dt_change: float = 0.1

    def to_c(self):
        c = _DtControls()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c


def next_dt(ctl: DtControls, dt, cfl):
    """Adjust_TimeStep (Sphere_Hybrid_Space.F90:604-649) on the host: the next dt after a step of
    size dt whose CFL cargo is cfl."""
    lib = load_library()
    c = ctl.to_c()
    out = ctypes.c_double()
    rc = lib.ra_next_dt(ctypes.byref(c), float(dt), float(cfl), ctypes.byref(out))
    if rc != RA_OK:
        raise RayleighError(rc, f"time step {out.value} below min_time_step")
    return out.value


@dataclass
class Config:
    """Namelist values the path reads (defaults follow the reference's Controls/PDE_Coefficients)."""

    n_r: int = 48
    l_max: int = 63
    n_theta: int = 0
    aspect_ratio: float = 0.35
    shell_depth: float = 1.0
    rayleigh: float = 1.0e5
    ekman: float = 1.0e-3
    prandtl: float = 1.0
    magnetic_prandtl: float = 1.0
    gravity_power: float = 1.0
    rotation: bool = True
    magnetism: bool = False
    no_slip_top: bool = True
    no_slip_bottom: bool = True
    fix_tvar_top: bool = True
    fix_tvar_bottom: bool = True
    t_top: float = 0.0
    t_bottom: float = 1.0
    dtdr_top: float = 0.0
    dtdr_bottom: float = 0.0
    dt: float = 1.0e-4
    alpha_implicit: float = 0.5
    precision: int = PREC_FP64
    use_graph: bool = True
    device: int = 0
    autotune: bool = False
    # reference state: 1 Boussinesq, 2 dimensional polytrope, 3 nondimensional polytrope
    reference_type: int = 1
    poly_n: float = 0.0
    poly_nrho: float = 0.0
    poly_mass: float = 0.0
    poly_rho_i: float = 0.0
    pressure_specific_heat: float = 1.0
    angular_velocity: float = -1.0
    modified_rayleigh: float = -1.0
    nu_type: int = 1
    kappa_type: int = 1
    eta_type: int = 1
    nu_power: float = 0.0
    kappa_power: float = 0.0
    eta_power: float = 0.0
    nu_top: float = -1.0
    kappa_top: float = -1.0
    eta_top: float = -1.0
    viscous_heating: bool = True
    ohmic_heating: bool = True
    chebyshev: bool = True           # False: the finite-difference radial mode

    def to_c(self):
        c = _Config()
        for f in fields(self):
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        return c


_lib = None
_DP = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p


def load_library(path: str | None = None):
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RayleighError(RA_ERR_STATE, f"{p} is missing; build it with `python -m rayleigh_b200.build`")
    lib = ctypes.CDLL(p)
    sig = {
        "ra_default_config": ([ctypes.POINTER(_Config)], ctypes.c_int),
        "ra_create": ([ctypes.POINTER(_VP), ctypes.POINTER(_Config)], ctypes.c_int),
        "ra_destroy": ([_VP], ctypes.c_int),
        "ra_last_error": ([_VP, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
        "ra_sizes": ([_VP, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int),
                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "ra_set_dt": ([_VP, ctypes.c_double], ctypes.c_int),
        "ra_put_state": ([_VP, _VP, _VP, _VP, ctypes.c_int], ctypes.c_int),
        "ra_get_state": ([_VP, _VP, _VP, _VP], ctypes.c_int),
        "ra_step": ([_VP, ctypes.c_int, _DP], ctypes.c_int),
        "ra_post_solve": ([_VP], ctypes.c_int),
        "ra_rlm_a": ([_VP], ctypes.c_int),
        "ra_physical": ([_VP, _DP], ctypes.c_int),
        "ra_rlm_b": ([_VP], ctypes.c_int),
        "ra_advance": ([_VP], ctypes.c_int),
        "ra_kinetic_energy": ([_VP, _DP], ctypes.c_int),
        "ra_magnetic_energy": ([_VP, _DP], ctypes.c_int),
        "ra_default_dt_controls": ([ctypes.POINTER(_DtControls)], ctypes.c_int),
        "ra_next_dt": ([ctypes.POINTER(_DtControls), ctypes.c_double, ctypes.c_double, _DP], ctypes.c_int),
        "ra_step_adaptive": ([_VP, ctypes.c_int, ctypes.POINTER(_DtControls), _DP, ctypes.POINTER(ctypes.c_int)],
                             ctypes.c_int),
        "ra_shell_slices": ([_VP, _VP, ctypes.c_int, _VP, ctypes.c_int, _VP], ctypes.c_int),
        "ra_shell_averages": ([_VP, _VP, ctypes.c_int, _VP], ctypes.c_int),
        "ra_azimuthal_averages": ([_VP, _VP, ctypes.c_int, _VP], ctypes.c_int),
        "ra_shell_spectra": ([_VP, _VP, ctypes.c_int, _VP, ctypes.c_int, _VP], ctypes.c_int),
        "ra_equatorial_slices": ([_VP, _VP, ctypes.c_int, _VP], ctypes.c_int),
        "ra_meridional_slices": ([_VP, _VP, ctypes.c_int, _VP, ctypes.c_int, _VP], ctypes.c_int),
        "ra_global_averages": ([_VP, _VP, ctypes.c_int, _VP], ctypes.c_int),
        "ra_point_probes": ([_VP, _VP, ctypes.c_int, _VP, ctypes.c_int, _VP, ctypes.c_int, _VP, ctypes.c_int, _VP],
                            ctypes.c_int),
        "ra_sync": ([_VP], ctypes.c_int),
        "ra_legendre_s2p": ([_VP, _VP, _VP, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "ra_legendre_p2s": ([_VP, _VP, _VP, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "ra_fft_c2r": ([_VP, _VP, ctypes.c_long], ctypes.c_int),
        "ra_fft_r2c": ([_VP, _VP, ctypes.c_long], ctypes.c_int),
        "ra_cheby_to_spectral": ([_VP, _VP, _VP, ctypes.c_long], ctypes.c_int),
        "ra_cheby_from_spectral": ([_VP, _VP, _VP, ctypes.c_long], ctypes.c_int),
        "ra_cheby_deriv": ([_VP, _VP, _VP, ctypes.c_int, ctypes.c_long], ctypes.c_int),
        "ra_radius": ([_VP, _VP], ctypes.c_int),
        "ra_costheta": ([_VP, _VP], ctypes.c_int),
        "ra_launch_count": ([_VP], ctypes.c_long),
        "ra_time_steps": ([_VP, ctypes.c_int, _DP, _DP, ctypes.c_int], ctypes.c_int),
        "ra_step_timed": ([_VP, ctypes.c_int, _DP], ctypes.c_int),
        "ra_get_choice": ([_VP, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "ra_set_choice": ([_VP, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
        "ra_autotune": ([_VP, ctypes.c_int, _DP], ctypes.c_int),
        "ra_kernels_per_step": ([], ctypes.c_int),
        "ra_kernel_name": ([ctypes.c_int], ctypes.c_char_p),
        "ra_mixed_gemm": ([_VP, _VP, _VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "ra_mixed_gemm_noalloc": ([_VP, _VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_char_p,
                                   ctypes.c_int], ctypes.c_int),
        "ra_debug_buffer": ([_VP, ctypes.c_int, _VP, ctypes.c_long, ctypes.POINTER(ctypes.c_long)], ctypes.c_int),
        "ra_write_checkpoint": ([_VP, ctypes.c_char_p, ctypes.c_double], ctypes.c_int),
        "ra_read_checkpoint": ([_VP, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), _DP], ctypes.c_int),
        "ra_checkpoint_write_field": ([ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _VP], ctypes.c_int),
        "ra_checkpoint_read_field": ([ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _VP], ctypes.c_int),
        "ra_put_magnetic_state": ([_VP, _VP, _VP, _VP], ctypes.c_int),
        "ra_get_magnetic_state": ([_VP, _VP, _VP, _VP], ctypes.c_int),
        "ra_put_state_modes": ([_VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP, ctypes.c_int], ctypes.c_int),
        "ra_get_state_modes": ([_VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP], ctypes.c_int),
        "ra_build_matrices": ([ctypes.POINTER(_Config), ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, _VP],
                              ctypes.c_int),
        "ra_load_matrices": ([_VP, ctypes.c_int, _VP, _VP], ctypes.c_int),
        "ra_factor": ([_VP, ctypes.c_double], ctypes.c_int),
        "ra_set_bc_mask": ([_VP, _VP], ctypes.c_int),
        "ra_set_reference": ([_VP, _VP, _VP, _VP, _VP, ctypes.c_double, ctypes.c_double], ctypes.c_int),
        "ra_transform_dev": ([_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, ctypes.c_int, _DP], ctypes.c_int),
        "ra_lu_create": ([ctypes.POINTER(_VP), ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "ra_lu_destroy": ([_VP], ctypes.c_int),
        "ra_lu_last_error": ([_VP, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
        "ra_lu_factor": ([_VP, _VP, _DP], ctypes.c_int),
        "ra_lu_solve": ([_VP, _VP, _VP, ctypes.c_int, ctypes.c_int, _VP, _DP], ctypes.c_int),
        "ra_lu_tiles": ([_VP, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(_VP) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Rayleigh:
    """One simulation context on one GPU (mirrors the reference's module state)."""

    def __init__(self, cfg: Config):
        self.lib = load_library()
        self.cfg = cfg
        self._c = cfg.to_c()
        h = _VP()
        rc = self.lib.ra_create(ctypes.byref(h), ctypes.byref(self._c))
        self.h = h
        if rc != RA_OK:
            msg = self._err()
            self.lib.ra_destroy(h)
            self.h = None
            raise RayleighError(rc, msg)
        n_lm = ctypes.c_long()
        nr, nth, nphi = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.ra_sizes(h, ctypes.byref(n_lm), ctypes.byref(nr), ctypes.byref(nth), ctypes.byref(nphi)))
        self.n_lm, self.n_r, self.n_theta, self.n_phi = n_lm.value, nr.value, nth.value, nphi.value
        self.l_max = cfg.l_max

    def _err(self):
        buf = ctypes.create_string_buffer(1024)
        if self.h:
            self.lib.ra_last_error(self.h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc):
        if rc != RA_OK:
            raise RayleighError(rc, self._err())

    def close(self):
        if self.h:
            self.lib.ra_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state (equation-set RHS layout: wpt[lm][ri][3 nr], z[lm][ri][nr], ab[4][lm][ri][nr]) ----
    def put_state(self, wpt, z, ab=None, iteration=1):
        self._wpt = _f64(wpt)
        self._z = _f64(z)
        self._ab = None if ab is None else _f64(ab)
        if self._wpt.size != self.n_lm * 2 * 3 * self.n_r or self._z.size != self.n_lm * 2 * self.n_r:
            raise ValueError("state arrays have the wrong size")
        self._check(self.lib.ra_put_state(self.h, _ptr(self._wpt), _ptr(self._z), _ptr(self._ab), int(iteration)))

    def get_state(self):
        wpt = np.empty((self.n_lm, 2, 3 * self.n_r))
        z = np.empty((self.n_lm, 2, self.n_r))
        ab = np.empty((4, self.n_lm, 2, self.n_r))
        self._check(self.lib.ra_get_state(self.h, _ptr(wpt), _ptr(z), _ptr(ab)))
        return wpt, z, ab

    # ---- magnetic state (magnetism = True): c[lm][ri][nr], a[lm][ri][nr], ab[2][lm][ri][nr] (C, A) ----
    def put_magnetic_state(self, c, a, ab=None):
        self._mc = _f64(c)
        self._ma = _f64(a)
        self._mab = None if ab is None else _f64(ab)
        if self._mc.size != self.n_lm * 2 * self.n_r or self._ma.size != self.n_lm * 2 * self.n_r:
            raise ValueError("magnetic state arrays have the wrong size")
        self._check(self.lib.ra_put_magnetic_state(self.h, _ptr(self._mc), _ptr(self._ma), _ptr(self._mab)))

    def get_magnetic_state(self):
        c = np.empty((self.n_lm, 2, self.n_r))
        a = np.empty((self.n_lm, 2, self.n_r))
        ab = np.empty((2, self.n_lm, 2, self.n_r))
        self._check(self.lib.ra_get_magnetic_state(self.h, _ptr(c), _ptr(a), _ptr(ab)))
        return c, a, ab

    # ---- checkpoint files in the reference's format ----
    def write_checkpoint(self, directory, elapsed_time=0.0):
        self._check(self.lib.ra_write_checkpoint(self.h, os.fsencode(directory), float(elapsed_time)))

    def read_checkpoint(self, directory):
        """Returns (iteration of the checkpoint, its elapsed time); the context continues from the next."""
        it = ctypes.c_int()
        t = ctypes.c_double()
        self._check(self.lib.ra_read_checkpoint(self.h, os.fsencode(directory), ctypes.byref(it), ctypes.byref(t)))
        return it.value, t.value

    # ---- one rank's slice of the modes (the reference's per-rank equation-set layout) ----
    def put_state_modes(self, l_of, m_of, wpt, z, ab=None, iteration=1):
        """Put the modes (l_of[i], m_of[i]): wpt[mode][ri][3 nr], z[mode][ri][nr], ab[4][mode][ri][nr]."""
        lo = np.ascontiguousarray(l_of, dtype=np.int32)
        mo = np.ascontiguousarray(m_of, dtype=np.int32)
        w, zz = _f64(wpt), _f64(z)
        a = None if ab is None else _f64(ab)
        self._check(self.lib.ra_put_state_modes(self.h, len(lo), lo.ctypes.data, mo.ctypes.data, _ptr(w), _ptr(zz),
                                                _ptr(a), int(iteration)))

    def get_state_modes(self, l_of, m_of):
        lo = np.ascontiguousarray(l_of, dtype=np.int32)
        mo = np.ascontiguousarray(m_of, dtype=np.int32)
        k = len(lo)
        w = np.empty((k, 2, 3 * self.n_r))
        z = np.empty((k, 2, self.n_r))
        ab = np.empty((4, k, 2, self.n_r))
        self._check(self.lib.ra_get_state_modes(self.h, k, lo.ctypes.data, mo.ctypes.data, _ptr(w), _ptr(z), _ptr(ab)))
        return w, z, ab

    # ---- the driver's own implicit system ----
    def load_matrices(self, sys, lhs=None, coefs=None):
        """lhs[l][col][row] (each matrix column-major, as the reference stores it), coefs[l][slot][r]."""
        self._lhs_keep = None if lhs is None else _f64(lhs)
        self._coef_keep = None if coefs is None else _f64(coefs)
        self._check(self.lib.ra_load_matrices(self.h, int(sys), _ptr(self._lhs_keep), _ptr(self._coef_keep)))

    def factor(self, dt):
        self._check(self.lib.ra_factor(self.h, float(dt)))

    def set_bc_mask(self, bc_values):
        """bc_values[eq W/P/T/Z][lm][re/im][top/bottom] (Fortran bc_values(2, 2, n_lm, 4)), or None."""
        self._bcv = None if bc_values is None else _f64(bc_values)
        self._check(self.lib.ra_set_bc_mask(self.h, _ptr(self._bcv)))

    def transform_dev(self, direction, precision, d_spec, d_grid, d_work, nfr):
        """ra_transform_dev on device buffers given by address (e.g. torch tensors' data_ptr());
        returns the stage times [Legendre product, relayout, FFT] in ms."""
        ms = (ctypes.c_double * 3)()
        self._check(self.lib.ra_transform_dev(self.h, int(direction), int(precision), ctypes.c_void_p(d_spec),
                                              ctypes.c_void_p(d_grid), ctypes.c_void_p(d_work), int(nfr),
                                              ctypes.cast(ms, _DP)))
        return list(ms)

    def set_reference(self, density, dlnrho, viscous_heating_coeff=None, ohmic_heating_coeff=None,
                      coriolis_coeff=0.0, lorentz_coeff=0.0):
        """The driver's reference state for the explicit terms (ra_set_reference): per-radius
        density, dlnrho and heating coefficients (None: off), the Coriolis and Lorentz coefficients."""
        arrs = [None if a is None else _f64(a) for a in (density, dlnrho, viscous_heating_coeff,
                                                          ohmic_heating_coeff)]
        self._refs = arrs
        self._check(self.lib.ra_set_reference(self.h, *[_ptr(a) for a in arrs], float(coriolis_coeff),
                                               float(lorentz_coeff)))

    def step(self, nsteps=1):
        cfl = ctypes.c_double()
        self._check(self.lib.ra_step(self.h, int(nsteps), ctypes.byref(cfl)))
        return cfl.value

    KNOBS = ("physics", "solve_nc")

    def get_choice(self, knob):
        v = ctypes.c_int()
        self._check(self.lib.ra_get_choice(self.h, knob.encode(), ctypes.byref(v)))
        return v.value

    def set_choice(self, knob, value):
        self._check(self.lib.ra_set_choice(self.h, knob.encode(), int(value)))

    def autotune(self, nreps=3):
        """Times every candidate of each knob on this context and keeps the fastest;
        returns {knob: (choice, ms)}."""
        ms = (ctypes.c_double * len(self.KNOBS))()
        self._check(self.lib.ra_autotune(self.h, int(nreps), ms))
        return {k: (self.get_choice(k), ms[i]) for i, k in enumerate(self.KNOBS)}

    def step_timed(self, nsteps):
        """nsteps steps as ra_step runs them (graph replays), device-timed with CUDA events
        on the context's stream: total milliseconds."""
        ms = ctypes.c_double()
        self._check(self.lib.ra_step_timed(self.h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def time_steps(self, nsteps):
        """Device-timed steps (CUDA events on the context's stream): (total_ms, {kernel: ms})."""
        nk = self.lib.ra_kernels_per_step()
        total = ctypes.c_double()
        per = (ctypes.c_double * nk)()
        self._check(self.lib.ra_time_steps(self.h, int(nsteps), ctypes.byref(total), per, nk))
        names = [self.lib.ra_kernel_name(i).decode() for i in range(nk)]
        return total.value, dict(zip(names, list(per)))

    def set_dt(self, dt):
        self._check(self.lib.ra_set_dt(self.h, float(dt)))

    def sync(self):
        self._check(self.lib.ra_sync(self.h))

    def launch_count(self):
        return self.lib.ra_launch_count(self.h)

    # the five stage calls
    def post_solve(self):
        self._check(self.lib.ra_post_solve(self.h))

    def rlm_spacea(self):
        self._check(self.lib.ra_rlm_a(self.h))

    def physical_space(self):
        cfl = ctypes.c_double()
        self._check(self.lib.ra_physical(self.h, ctypes.byref(cfl)))
        return cfl.value

    def rlm_spaceb(self):
        self._check(self.lib.ra_rlm_b(self.h))

    def advance_time(self):
        self._check(self.lib.ra_advance(self.h))

    def kinetic_energy(self):
        """Benchmark_Checkup's volume-averaged kinetic energy of the current state
        (Benchmarking.F90:645-656, 733-736), reduced on the device."""
        ke = ctypes.c_double()
        self._check(self.lib.ra_kinetic_energy(self.h, ctypes.byref(ke)))
        return ke.value

    # the reference's output codes of the quantities ra_shell_slices provides
    def magnetic_energy(self):
        """The benchmark report's magnetic energy of the current state (magnetism only):
        the volume average of |B|^2 over 2 Ek Pm (Benchmarking.F90:689-696, 846)."""
        me = ctypes.c_double()
        self._check(self.lib.ra_magnetic_energy(self.h, ctypes.byref(me)))
        return me.value

    def step_adaptive(self, nsteps, ctl: DtControls):
        """nsteps steps with the CFL time-step control; returns (dt of the next step, dt changes)."""
        c = ctl.to_c()
        dt = ctypes.c_double()
        nch = ctypes.c_int()
        self._check(self.lib.ra_step_adaptive(self.h, int(nsteps), ctypes.byref(c), ctypes.byref(dt),
                                              ctypes.byref(nch)))
        return dt.value, nch.value

    QUANTITIES = {"v_r": 1, "v_theta": 2, "v_phi": 3, "dv_r_dr": 10, "dv_theta_dr": 11, "dv_phi_dr": 12,
                  "dv_r_dt": 19, "dv_r_dp": 28, "dv_theta_dp": 29, "dv_phi_dp": 30, "vort_r": 301,
                  "entropy": 501, "entropy_dr": 507, "entropy_dtheta": 513, "entropy_dphi": 519,
                  "pressure": 502, "pressure_dr": 508, "pressure_dphi": 520, "b_r": 801, "b_theta": 802,
                  "b_phi": 803, "j_r": 1001, "j_theta": 1004, "j_phi": 1007,
                  # fluctuating (m > 0) and azimuthal-mean (m = 0) parts, the reference's codes
                  "vp_r": 4, "vp_theta": 5, "vp_phi": 6, "vm_r": 7, "vm_theta": 8, "vm_phi": 9,
                  "dvp_r_dr": 13, "dvp_theta_dr": 14, "dvp_phi_dr": 15, "dvm_r_dr": 16, "dvm_theta_dr": 17,
                  "dvm_phi_dr": 18, "dvp_r_dt": 22, "dvm_r_dt": 25, "dv_theta_dt": 20, "dv_phi_dt": 21,
                  "dvp_theta_dt": 23, "dvp_phi_dt": 24, "dvm_theta_dt": 26, "dvm_phi_dt": 27, "dvp_r_dp": 31, "dvp_theta_dp": 32,
                  "dvp_phi_dp": 33, "dvm_r_dp": 34, "dvm_theta_dp": 35, "dvm_phi_dp": 36, "vortp_r": 304,
                  "vortm_r": 307, "vort_theta": 302, "vort_phi": 303, "vortp_theta": 305, "vortp_phi": 306,
                  "vortm_theta": 308, "vortm_phi": 309, "entropy_p": 503, "pressure_p": 504,
                  "entropy_m": 505, "pressure_m": 506, "entropy_p_dr": 509, "pressure_p_dr": 510,
                  "entropy_m_dr": 511, "pressure_m_dr": 512, "entropy_p_dtheta": 515,
                  "entropy_m_dtheta": 517, "entropy_p_dphi": 521, "pressure_p_dphi": 522,
                  "entropy_m_dphi": 523, "pressure_m_dphi": 524, "bp_r": 804, "bp_theta": 805, "bp_phi": 806,
                  "bm_r": 807, "bm_theta": 808, "bm_phi": 809, "jp_r": 1002, "jm_r": 1003, "jp_theta": 1005,
                  "jm_theta": 1006, "jp_phi": 1008, "jm_phi": 1009, "db_r_dp": 828, "db_theta_dp": 829,
                  "db_phi_dp": 830, "dbp_r_dp": 831, "dbp_theta_dp": 832, "dbp_phi_dp": 833, "dbm_r_dp": 834,
                  "dbm_theta_dp": 835, "dbm_phi_dp": 836,
                  "rhov_r": 201, "rhov_theta": 202, "rhov_phi": 203, "rhovp_r": 204, "rhovp_theta": 205,
                  "rhovp_phi": 206, "rhovm_r": 207, "rhovm_theta": 208, "rhovm_phi": 209,
                  "thermal_energy_full": 701, "thermal_energy_p": 702, "thermal_energy_m": 703,
                  "thermal_energy_sq": 707, "thermal_energyp_sq": 708, "thermal_energym_sq": 709,
                  # products: enstrophy, squared vorticity, kinetic helicity, mean J . J'
                  "enstrophy": 310, "enstrophy_pm": 311, "enstrophy_mm": 312, "enstrophy_pp": 313,
                  "vort_r_sq": 314, "vort_theta_sq": 315, "vort_phi_sq": 316, "vortp_r_sq": 317,
                  "vortp_theta_sq": 318, "vortp_phi_sq": 319, "vortm_r_sq": 320, "vortm_theta_sq": 321,
                  "vortm_phi_sq": 322, "kin_helicity_r": 324, "kin_helicity_theta": 325,
                  "kin_helicity_phi": 326, "kin_helicity_pp_r": 327, "kin_helicity_pp_theta": 328,
                  "kin_helicity_pp_phi": 329, "kin_helicity_mm_r": 330, "kin_helicity_mm_theta": 331,
                  "kin_helicity_mm_phi": 332, "kin_helicity_mp_r": 333, "kin_helicity_mp_theta": 334,
                  "kin_helicity_mp_phi": 335, "kin_helicity_pm_r": 336, "kin_helicity_pm_theta": 337,
                  "kin_helicity_pm_phi": 338, "kin_helicity": 339, "kin_helicity_pp": 340,
                  "kin_helicity_mm": 341, "kin_helicity_mp": 342, "kin_helicity_pm": 343, "jpm_sq": 1013,
                  # sums of squares: kinetic energy densities, v^2, J.J, magnetic energy densities
                  "kinetic_energy": 401, "radial_ke": 402, "theta_ke": 403, "phi_ke": 404,
                  "mkinetic_energy": 405, "radial_mke": 406, "theta_mke": 407, "phi_mke": 408,
                  "pkinetic_energy": 409, "radial_pke": 410, "theta_pke": 411, "phi_pke": 412, "vsq": 413,
                  "radial_vsq": 414, "theta_vsq": 415, "phi_vsq": 416, "mvsq": 417, "radial_mvsq": 418,
                  "theta_mvsq": 419, "phi_mvsq": 420, "pvsq": 421, "radial_pvsq": 422, "theta_pvsq": 423,
                  "phi_pvsq": 424, "j_sq": 1010, "jp_sq": 1011, "jm_sq": 1012, "j_r_sq": 1014,
                  "jp_r_sq": 1015, "jm_r_sq": 1016, "j_theta_sq": 1017, "jp_theta_sq": 1018,
                  "jm_theta_sq": 1019, "j_phi_sq": 1020, "jp_phi_sq": 1021, "jm_phi_sq": 1022,
                  "magnetic_energy": 1101, "radial_me": 1102, "theta_me": 1103, "phi_me": 1104,
                  "mmagnetic_energy": 1105, "radial_mme": 1106, "theta_mme": 1107, "phi_mme": 1108,
                  "pmagnetic_energy": 1109, "radial_pme": 1110, "theta_pme": 1111, "phi_pme": 1112}

    def shell_slices(self, quantities, levels):
        """Shell slices of the current state: array [quantity][level][theta][phi] of the
        quantities (output codes or names of QUANTITIES) at the radial grid indices."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        lv = np.ascontiguousarray(levels, dtype=np.int32)
        out = np.empty((len(q), len(lv), self.n_theta, self.n_phi))
        self._check(self.lib.ra_shell_slices(self.h, q.ctypes.data, len(q), lv.ctypes.data, len(lv),
                                             out.ctypes.data))
        return out

    def shell_averages(self, quantities):
        """Shell averages of the current state: array [quantity][moment][r], moment 0 the
        mean over the sphere, 1-3 the averages of (q - mean)^2, ^3, ^4."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        out = np.empty((len(q), 4, self.n_r))
        self._check(self.lib.ra_shell_averages(self.h, q.ctypes.data, len(q), out.ctypes.data))
        return out

    def azimuthal_averages(self, quantities):
        """Azimuthal (phi) averages of the current state: array [quantity][theta][r]."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        out = np.empty((len(q), self.n_theta, self.n_r))
        self._check(self.lib.ra_azimuthal_averages(self.h, q.ctypes.data, len(q), out.ctypes.data))
        return out

    def shell_spectra(self, quantities, levels):
        """Shell spectra of the current state: array [quantity][level][re/im][m][l]
        (l, m = 0 .. l_max; zero for l < m)."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        lv = np.ascontiguousarray(levels, dtype=np.int32)
        L = self.l_max + 1
        out = np.empty((len(q), len(lv), 2, L, L))
        self._check(self.lib.ra_shell_spectra(self.h, q.ctypes.data, len(q), lv.ctypes.data, len(lv),
                                              out.ctypes.data))
        return out

    def equatorial_slices(self, quantities):
        """Equatorial slices of the current state: array [quantity][r][phi], the mean of
        the two theta rows nearest the equator."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        out = np.empty((len(q), self.n_r, self.n_phi))
        self._check(self.lib.ra_equatorial_slices(self.h, q.ctypes.data, len(q), out.ctypes.data))
        return out

    def meridional_slices(self, quantities, phi_indices):
        """Meridional slices of the current state: array [quantity][phi index][theta][r]."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        ph = np.ascontiguousarray(phi_indices, dtype=np.int32)
        out = np.empty((len(q), len(ph), self.n_theta, self.n_r))
        self._check(self.lib.ra_meridional_slices(self.h, q.ctypes.data, len(q), ph.ctypes.data, len(ph),
                                                  out.ctypes.data))
        return out

    def global_averages(self, quantities):
        """Volume averages of the current state: array [quantity]."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        out = np.empty(len(q))
        self._check(self.lib.ra_global_averages(self.h, q.ctypes.data, len(q), out.ctypes.data))
        return out

    def point_probes(self, quantities, r_idx, theta_idx, phi_idx):
        """Point probes of the current state: array [quantity][r][theta][phi] at the
        tensor product of the grid indices."""
        q = np.ascontiguousarray([self.QUANTITIES.get(x, x) for x in quantities], dtype=np.int32)
        ri, ti, pi = (np.ascontiguousarray(a, dtype=np.int32) for a in (r_idx, theta_idx, phi_idx))
        out = np.empty((len(q), len(ri), len(ti), len(pi)))
        self._check(self.lib.ra_point_probes(self.h, q.ctypes.data, len(q), ri.ctypes.data, len(ri), ti.ctypes.data,
                                             len(ti), pi.ctypes.data, len(pi), out.ctypes.data))
        return out

    BUFFERS = {"grid": 0, "s2a": 1, "s2a11": 2, "p2a": 3, "p2b": 4, "s2b": 5, "ab": 6,
               "rhs_wpt": 7, "rhs_z": 8, "ptab": 9, "iptab": 10, "s2am": 11, "rhs_c": 12, "rhs_a": 13}

    def debug_buffer(self, name):
        """Copy of an internal device buffer (diagnostics for the stage-by-stage parity tests)."""
        which = self.BUFFERS[name]
        n = ctypes.c_long()
        self._check(self.lib.ra_debug_buffer(self.h, which, None, 0, ctypes.byref(n)))
        out = np.empty(n.value)
        self._check(self.lib.ra_debug_buffer(self.h, which, _ptr(out), n.value, ctypes.byref(n)))
        return out

    # ---- grids ----
    def radius(self):
        r = np.empty(self.n_r)
        self._check(self.lib.ra_radius(self.h, _ptr(r)))
        return r

    def costheta(self):
        c = np.empty(self.n_theta)
        self._check(self.lib.ra_costheta(self.h, _ptr(c)))
        return c

    # ---- math-layer operators on reference layouts ----
    def legendre_s2p(self, s2):
        """StP: s2 = list over m of arrays (nf, 2, nr, l_max-m+1) -> list over m of (nf, 2, nr, n_theta)."""
        nf, _, nr, _ = s2[0].shape
        flat = _f64(np.concatenate([np.ascontiguousarray(a).ravel() for a in s2]))
        out = np.empty(((self.l_max + 1), nf, 2, nr, self.n_theta))
        self._check(self.lib.ra_legendre_s2p(self.h, _ptr(flat), _ptr(out), nf, nr))
        return [out[m] for m in range(self.l_max + 1)]

    def legendre_p2s(self, p2):
        nf, _, nr, _ = p2[0].shape
        flat = _f64(np.stack(p2))
        out = np.empty(sum(nf * 2 * nr * (self.l_max + 1 - m) for m in range(self.l_max + 1)))
        self._check(self.lib.ra_legendre_p2s(self.h, _ptr(flat), _ptr(out), nf, nr))
        res, off = [], 0
        for m in range(self.l_max + 1):
            n = nf * 2 * nr * (self.l_max + 1 - m)
            res.append(out[off:off + n].reshape(nf, 2, nr, self.l_max + 1 - m))
            off += n
        return res

    def fft_c2r(self, x):
        x = _f64(x).copy()
        self._check(self.lib.ra_fft_c2r(self.h, _ptr(x), x.size // (self.n_phi + 2)))
        return x

    def fft_r2c(self, x):
        x = _f64(x).copy()
        self._check(self.lib.ra_fft_r2c(self.h, _ptr(x), x.size // (self.n_phi + 2)))
        return x

    def mixed_gemm(self, a, b):
        """Split-precision tensor-core product a @ b (FP64 in and out)."""
        a = _f64(a)
        b = _f64(b)
        m, k = a.shape
        k2, n = b.shape
        if k != k2:
            raise ValueError("inner dimensions differ")
        out = np.empty((m, n))
        self._check(self.lib.ra_mixed_gemm(self.h, _ptr(a), _ptr(b), _ptr(out), m, n, k))
        return out

    def cheby_to_spectral(self, f):
        f = _f64(f)
        out = np.empty_like(f)
        self._check(self.lib.ra_cheby_to_spectral(self.h, _ptr(f), _ptr(out), f.size // self.n_r))
        return out

    def cheby_from_spectral(self, c):
        c = _f64(c)
        out = np.empty_like(c)
        self._check(self.lib.ra_cheby_from_spectral(self.h, _ptr(c), _ptr(out), c.size // self.n_r))
        return out

    def cheby_deriv(self, c, order):
        c = _f64(c)
        out = np.empty_like(c)
        self._check(self.lib.ra_cheby_deriv(self.h, _ptr(c), _ptr(out), int(order), c.size // self.n_r))
        return out


def build_matrices(cfg: Config, sys, l0, nl, coefs=False):
    """The library's own assembly of the per-l implicit matrices (host only): lhs[l][col][row]
    (column-major per l) of system sys (0 = W-P-T, 1 = Z, 2 = C, 3 = A with magnetism) for
    l = l0 .. l0+nl-1, and with coefs=True also coefs[l][slot][r] (16 slots for systems 0
    and 1, 2 for C, 3 for A)."""
    lib = load_library()
    c = cfg.to_c()
    n = cfg.n_r * (1 if sys else 3)
    lhs = np.empty((nl, n, n))
    cf = np.empty((nl, {0: 16, 1: 16, 2: 2, 3: 3}[int(sys)], cfg.n_r)) if coefs else None
    rc = lib.ra_build_matrices(ctypes.byref(c), int(sys), int(l0), int(nl), _ptr(lhs), _ptr(cf))
    if rc != RA_OK:
        raise RayleighError(rc, "ra_build_matrices refused the configuration or range")
    return (lhs, cf) if coefs else lhs


def checkpoint_write_field(path, field, n_r, l_max):
    """One checkpoint field file from a state-layout array [lm][re/im][r] (host only)."""
    f = _f64(field)
    if f.size != n_r * (l_max + 1) * (l_max + 2):
        raise ValueError("field has the wrong size")
    rc = load_library().ra_checkpoint_write_field(os.fsencode(path), int(n_r), int(l_max), _ptr(f))
    if rc != RA_OK:
        raise RayleighError(rc, f"cannot write {path}")


def checkpoint_read_field(path, n_r, l_max):
    """A checkpoint field file as a state-layout array [lm][re/im][r] (host only)."""
    n_lm = (l_max + 1) * (l_max + 2) // 2
    out = np.empty((n_lm, 2, n_r))
    rc = load_library().ra_checkpoint_read_field(os.fsencode(path), int(n_r), int(l_max), _ptr(out))
    if rc != RA_OK:
        raise RayleighError(rc, f"cannot read {path} (missing, or not a field of this grid)")
    return out


SOLVE_FP64 = 0
SOLVE_REFINE = 1


class BatchedLU:
    """Batched per-l LU factorisation and solves on one device (LU_Decompose_full /
    LU_Solve_full, Linear_Solve.F90:1028-1036, 1088-1110), independent of a context."""

    def __init__(self, n, count, device=0):
        self.lib = load_library()
        h = _VP()
        rc = self.lib.ra_lu_create(ctypes.byref(h), int(n), int(count), int(device))
        self.h = h
        self.n, self.count = n, count
        if rc != RA_OK:
            msg = self._err()
            self.lib.ra_lu_destroy(h)
            self.h = None
            raise RayleighError(rc, msg)

    def _err(self):
        buf = ctypes.create_string_buffer(1024)
        if self.h:
            self.lib.ra_lu_last_error(self.h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc):
        if rc != RA_OK:
            raise RayleighError(rc, self._err())

    def factor(self, mats_colmajor):
        """mats[l][col][row] (column-major per matrix); returns the device time in ms."""
        a = _f64(mats_colmajor)
        if a.size != self.count * self.n * self.n:
            raise ValueError("matrices have the wrong size")
        ms = ctypes.c_double()
        self._check(self.lib.ra_lu_factor(self.h, _ptr(a), ctypes.byref(ms)))
        return ms.value

    def solve(self, b, mode=SOLVE_FP64):
        """b[l][col][row]; returns (x, iterations[l][column tile], device ms)."""
        b = _f64(b)
        ncols = b.size // (self.count * self.n)
        x = np.empty_like(b)
        nt = self.lib.ra_lu_tiles(self.h, ncols, int(mode))
        if nt < 0:
            self._check(nt)
        it = np.empty(nt, dtype=np.int32)
        ms = ctypes.c_double()
        self._check(self.lib.ra_lu_solve(self.h, _ptr(b), _ptr(x), ncols, int(mode), it.ctypes.data, ctypes.byref(ms)))
        return x, it.reshape(self.count, -1), ms.value

    def close(self):
        if self.h:
            self.lib.ra_lu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


__all__ = ["Config", "Rayleigh", "RayleighError", "load_library", "LIB_PATH", "PREC_FP64", "PREC_MIXED",
           "BatchedLU", "build_matrices", "SOLVE_FP64", "SOLVE_REFINE"]
