"""The finite-difference radial mode (chebyshev = .false.) on the device against the oracle.

The state holds grid values on the uniform grid; to_spectral, from_spectral and dealiasing
are the identity, and every radial derivative is a banded matrix (the 5-point stencils of
Generate_Coefs, Finite_Difference.F90:525-689, one-sided at the ends).  Post_Solve_FD
(Sphere_Spectral_Space.F90:37-176) hands rlm_spacea D_1 D_1 W in place of D_2 W (the
deriv_cluge), while Add_Derivative builds the explicit terms from D_2 W; Finalize_EMF's
radial derivative is D_1.  FP64 form: every stage and the state after N steps to 1e-12
relative L2 per field; mixed form: 1e-9 (it keeps its split products for the Legendre
transforms and solves by the FP64 block substitution: applied by split products, the
explicit grid-space inverse of the W-P-T system left W 8.7e-9 from the oracle after 20
steps; through the LU factors 1.1e-10).  Checkpoints of a finite-difference context carry
grid_type 1 and are refused by a Chebyshev context."""
import numpy as np
import pytest

import oracle as O
import test_gpu_mhd as M
import test_gpu_parity as H
from layouts import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12
FD = dict(n_r=24, l_max=15, dt=2e-4, chebyshev=False)
FD_MHD = dict(M.MHD, chebyshev=False)
FD_ANEL = dict(n_r=24, l_max=15, dt=1e-4, reference_type=3, poly_n=2.0, poly_nrho=3.0, modified_rayleigh=0.5,
               ekman=1e-3, prandtl=1.0, magnetic_prandtl=2.0, no_slip_top=False, no_slip_bottom=False,
               magnetism=True, chebyshev=False)


@pytest.mark.parametrize("steps_before", [0, 2])
def test_fd_hydro_stages(steps_before):
    errs = H._stage_compare(FD, steps_before=steps_before)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


@pytest.mark.parametrize("cfg", [FD_MHD, FD_ANEL])
def test_fd_mhd_stages(cfg):
    errs = M._stage_compare(cfg, steps_before=2)
    print({k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if v > TOL}
    assert not bad, errs


@pytest.mark.parametrize("cfg,steps,precision,tol", [
    (FD, 20, 0, TOL),
    (FD, 20, 1, 1e-9),
    (dict(FD, n_r=48, l_max=63, dt=1e-4, no_slip_top=False, no_slip_bottom=False), 20, 0, TOL),
    (FD_MHD, 20, 0, TOL),
    (FD_MHD, 20, 1, 1e-9),
    (FD_ANEL, 10, 0, TOL),
])
def test_fd_multi_step_parity(cfg, steps, precision, tol):
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


def test_fd_checkpoint_grid_type(tmp_path):
    import rayleigh_b200 as rb
    oc = M._ocfg(FD)
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=10)
    run = M._ctx(FD)
    run.put_state(wpt, z, None, iteration=1)
    run.step(3)
    ck = str(tmp_path / "00000003")
    run.write_checkpoint(ck, elapsed_time=6e-4)
    run.step(4)
    ref = run.get_state()
    fresh = M._ctx(FD)
    assert fresh.read_checkpoint(ck) == (3, 6e-4)
    fresh.step(4)
    for u, v in zip(ref, fresh.get_state()):
        assert np.array_equal(u, v)
    cheb = M._ctx(dict(FD, chebyshev=True))
    with pytest.raises(rb.RayleighError):
        cheb.read_checkpoint(ck)
    with pytest.raises(rb.RayleighError) as ei:
        run.cheby_deriv(np.zeros((4, FD["n_r"])), 1)
    assert ei.value.code == rb.RA_ERR_STATE


def test_fd_step_rate():
    """The finite-difference step against the Chebyshev step on one grid (Boussinesq
    hydrodynamic, N_r = 128, l_max = 255, N_theta = 384), FP64 and mixed: steps/s over 50
    graph-replayed steps, host-timed between two state copies; prints the four rates
    (measured: Chebyshev 81.1 / 97.5, finite differences 79.7 / 81.7 steps/s FP64 / mixed; the
    finite-difference mixed form solves by the FP64 substitution)."""
    import time
    cfg = dict(n_r=128, l_max=255, dt=1e-6, rayleigh=1e5, ekman=1e-3, use_graph=True)
    oc = M._ocfg(cfg)
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=20)
    rates = {}
    for chebyshev in (True, False):
        for precision in (0, 1):
            g = M._ctx(dict(cfg, chebyshev=chebyshev, precision=precision))
            g.put_state(wpt, z, None, iteration=1)
            g.step(2)
            g.get_state()
            t0 = time.perf_counter()
            g.step(50)
            w, _, _ = g.get_state()
            rates[("chebyshev" if chebyshev else "fd", "fp64" if precision == 0 else "mixed")] = \
                50 / (time.perf_counter() - t0)
            assert np.isfinite(w).all()
            g.close()
    print({f"{a} {b}": f"{v:.1f} steps/s" for (a, b), v in rates.items()})
    assert min(rates.values()) > 0
