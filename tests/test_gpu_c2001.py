"""The reference's regression run of its accuracy benchmark, on the GPU.

tests/c2001_case0 of the reference (Christensen et al. 2001 case 0 from
Benchmark_Init_Hydro, N_r = 48, N_theta = 64, 400 steps of dt = 1e-4) reports
the mean and standard deviation of the volume-averaged kinetic energy and of
the point observations T and v_phi at iterations 100, 200, 300 and 400.  The
CUDA path runs those steps through the C ABI; at each sample iteration k its
state after k - 1 steps goes through one oracle step, whose physical-space
stage forms the fields Benchmark_Checkup reads.  The sample itself comes from
the device: the kinetic energy is its own reduction (ra_kinetic_energy), and
the point observations are the oracle's restatement of Point_Observations run
on v_r, v_phi and T shell slices formed on the device (ra_shell_slices), as the
host side of the benchmark would; both are checked against the oracle's step
on the way.  Both precision forms must reproduce the reference's report to its
6 printed decimals, for the Chebyshev run and for tests/c2001_case0_FD_uniform, the same
run in the finite-difference radial mode (uniform grid, chebyshev = .false.)."""
import dataclasses
import json
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("report", ["c2001_case0.json", "c2001_case0_fd_uniform.json"])
@pytest.mark.parametrize("precision", [0, 1])
def test_c2001_case0_reproduces_the_reference_report(precision, report):
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", report)))
    ocfg = O.c2001_case0_config(gold["n_r"], gold["n_theta"], chebyshev=gold.get("chebyshev", True))
    o = O.Oracle(ocfg)
    wpt, z = o.benchmark_init_hydro()
    names = {f.name for f in dataclasses.fields(rb.Config)}
    cfg = {k: v for k, v in dataclasses.asdict(ocfg).items() if k in names}
    ke = []
    with rb.Rayleigh(rb.Config(**cfg, precision=precision, use_graph=True)) as g:
        g.put_state(wpt, z, None, iteration=1)
        done = 0
        levels = list(range(gold["n_r"]))
        every = gold["integration_interval"]
        for k in range(every, gold["max_iterations"] + 1, every):
            g.step(k - 1 - done)
            done = k - 1
            ke_dev = g.kinetic_energy()                # reduced on the device
            sl = g.shell_slices(["v_r", "v_phi", "entropy"], levels)   # formed on the device
            vphi, temp = o.benchmark_point_observations(fields=tuple(a.transpose(1, 0, 2) for a in sl))
            sw, sz, sab = g.get_state()
            o.init_state(sw, sz, sab)
            o.step()                                   # its physical-space stage sees iteration k's velocity
            ke_o = o.benchmark_kinetic_energy()
            vphi_o, temp_o = o.benchmark_point_observations()
            tol = 1e-12 if precision == 0 else 1e-9
            assert abs(ke_dev - ke_o) <= tol * ke_o, (k, ke_dev, ke_o)
            # the linear interpolation at the v_r zero crossings divides by the jump of v_r
            ptol = 1e-11 if precision == 0 else 1e-8
            assert abs(vphi - vphi_o) <= ptol * abs(vphi_o), (k, vphi, vphi_o)
            assert abs(temp - temp_o) <= ptol * abs(temp_o), (k, temp, temp_o)
            ke.append((ke_dev, vphi, temp))
    ke = np.array(ke)
    print(precision, ke)
    assert len(ke) == gold["samples"]
    for col, name in enumerate(("Kinetic Energy", "Vphi", "Temperature")):
        ref = gold["observables"][name]
        assert abs(ke[:, col].mean() - ref["measured"]) < 5e-6, (name, ke[:, col].mean(), ref)
        assert abs(ke[:, col].std() - ref["sdev"]) < 5e-6, (name, ke[:, col].std(), ref)
