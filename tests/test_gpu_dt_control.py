"""ra_step_adaptive's CFL time-step control (Adjust_TimeStep, Sphere_Hybrid_Space.F90:604-649)
on the device against the same control on the host.

ra_step_adaptive runs the steady steps as one graph launch whose conditional WHILE node
replays the step and a one-thread Adjust_TimeStep kernel until dt must change (or the count
is reached); the host then rebuilds and factors the matrices (Reset_Linear_Equations) and the
first step of the new dt runs with its unequal AB2 factors.  The reference decides after every
step on the host; here that decision is restated as: step(1), ra_next_dt on the returned CFL
cargo, ra_set_dt on a change.  Both give the same states bit for bit and the same dt history."""
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
def test_device_dt_control_matches_host_control(precision):
    import rayleigh_b200 as rb
    cfg = dict(n_r=24, l_max=15, dt=1e-4, rayleigh=1e5, ekman=1e-3, precision=precision, use_graph=True)
    oc = O.Config(**{k: v for k, v in cfg.items() if k in O.Config.__dataclass_fields__})
    wpt, z = O.seeded_state(oc, amp=3e-1, lmax_pert=10)
    ctl = rb.DtControls(cflmin=0.4, cflmax=0.6, max_time_step=2e-3)
    a = _ctx(cfg)
    b = _ctx(cfg)
    for g in (a, b):
        g.put_state(wpt, z, None, iteration=1)
    changes_a, dts_a = 0, []
    for _ in range(6):   # several calls: the loop graph is re-entered with new counts
        dt, n = a.step_adaptive(50, ctl)
        changes_a += n
        dts_a.append(dt)
    dt, changes_b, dts_b = cfg["dt"], 0, []
    for k in range(300):
        cfl = b.step(1)
        nd = rb.next_dt(ctl, dt, cfl)
        if nd != dt:
            b.set_dt(nd)
            dt = nd
            changes_b += 1
        if (k + 1) % 50 == 0:
            dts_b.append(dt)
    print("dt after each 50 steps", dts_a, "changes", changes_a)
    assert changes_a == changes_b and changes_a >= 3
    assert dts_a == dts_b
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
