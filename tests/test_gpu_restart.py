"""Restart from a checkpoint taken through the C ABI.

Rayleigh restarts from checkpoint files holding the solution and the
Adams-Bashforth history (Checkpointing.F90:143-801); here the checkpoint is
what ra_get_state returns (solution, AB2 history), restored with ra_put_state
into a fresh context at the next iteration number.  The continued run must
reproduce the uninterrupted one bit for bit, in both precision forms: every
kernel of the step is deterministic (no atomics other than the CFL maximum)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _ctx(cfg):
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    return rb.Rayleigh(rb.Config(**cfg))


@pytest.mark.parametrize("precision", [0, 1])
def test_restart_reproduces_the_uninterrupted_run(precision):
    cfg = dict(n_r=24, l_max=31, dt=2e-4, rayleigh=1e5, ekman=1e-3, precision=precision)
    oc = O.Config(**{k: v for k, v in cfg.items() if k in O.Config.__dataclass_fields__})
    wpt, z = O.seeded_state(oc, amp=1e-2, lmax_pert=10)
    first, second = 6, 5

    run = _ctx(cfg)
    run.put_state(wpt, z, None, iteration=1)
    run.step(first)
    ck_wpt, ck_z, ck_ab = run.get_state()          # the checkpoint
    run.step(second)
    ref_wpt, ref_z, ref_ab = run.get_state()

    restarted = _ctx(cfg)
    restarted.put_state(ck_wpt, ck_z, ck_ab, iteration=first + 1)
    restarted.step(second)
    got_wpt, got_z, got_ab = restarted.get_state()

    assert np.array_equal(got_wpt, ref_wpt)
    assert np.array_equal(got_z, ref_z)
    assert np.array_equal(got_ab, ref_ab)
    # and the run did move: the checkpoint is not the final state
    assert not np.array_equal(ck_wpt, ref_wpt)


@pytest.mark.parametrize("mag,precision", [(False, 0), (True, 0), (True, 1)])
def test_checkpoint_files_restart(tmp_path, mag, precision):
    """Write_Checkpoint / Read_Checkpoint through files in the reference's format
    (ra_write_checkpoint, ra_read_checkpoint): the run continued from the files, in a
    fresh context whose dt differs (the checkpoint's next dt is restored with its
    matrices), reproduces the uninterrupted run bit for bit; a checkpoint of another
    grid is refused."""
    import rayleigh_b200 as rb
    cfg = dict(n_r=24, l_max=31, dt=2e-4, rayleigh=1e5, ekman=1e-3, precision=precision, magnetism=mag,
               magnetic_prandtl=5.0)
    oc = O.Config(**{k: v for k, v in cfg.items() if k in O.Config.__dataclass_fields__})
    wpt, z = O.seeded_state(oc, amp=1e-2, lmax_pert=10)
    run = _ctx(cfg)
    run.put_state(wpt, z, None, iteration=1)
    if mag:
        c, a = O.seeded_magnetic_state(oc, amp=1e-1, lmax_pert=10)
        run.put_magnetic_state(c, a)
    run.step(4)
    run.set_dt(1.5e-4)                     # the checkpoint carries dt 2e-4 (last) and 1.5e-4 (next)
    ck = str(tmp_path / "00000004")
    run.write_checkpoint(ck, elapsed_time=8e-4)
    run.step(5)
    ref = [run.get_state()] + ([run.get_magnetic_state()] if mag else [])

    fresh = _ctx(dict(cfg, dt=3e-4))
    it, t = fresh.read_checkpoint(ck)
    assert it == 4 and t == 8e-4
    fresh.step(5)
    got = [fresh.get_state()] + ([fresh.get_magnetic_state()] if mag else [])
    for x, y in zip(ref, got):
        for u, v in zip(x, y):
            assert np.array_equal(u, v)
    other = _ctx(dict(cfg, n_r=32))
    with pytest.raises(rb.RayleighError):
        other.read_checkpoint(ck)
