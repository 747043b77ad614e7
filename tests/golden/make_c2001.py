"""Extract the reference's own regression result for its accuracy benchmark.

The reference ships a short run of the Christensen et al. (2001) hydrodynamic
case 0 as a regression test: ``tests/c2001_case0/main_input`` (N_r = 48,
N_theta = 64, benchmark_mode = 1, 400 iterations at dt = 1e-4) and the report
its run wrote, ``tests/c2001_case0/Benchmark_Reports/00000400``: mean and
standard deviation over the samples at iterations 100, 200, 300 and 400 of the
volume-averaged kinetic energy and the point observables.

Run from the repository root in a container that has the reference tree:

    python tests/golden/make_c2001.py /path/to/reference

The reference also ships the same run in its finite-difference radial mode,
``tests/c2001_case0_FD_uniform`` (chebyshev = .false., uniform grid); its report goes
to ``tests/golden/c2001_case0_fd_uniform.json``.

The outputs are committed; nothing at test time reads the reference tree.
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python %s /path/to/reference" % os.path.relpath(__file__))
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))


def extract(case, out_name):
    CASE = os.path.join(REF, "tests", case)
    inp = open(os.path.join(CASE, "main_input")).read()
    rep = open(os.path.join(CASE, "Benchmark_Reports", "00000400")).read()

    def nml(name):
        m = re.search(r"^\s*%s\s*=\s*([-+0-9.dDeE]+)" % name, inp, re.M)
        return float(m.group(1).replace("d", "e").replace("D", "e"))

    def iline(label):
        return int(re.search(label + r"\s*:\s*(\d+)", rep).group(1))

    obs = {}
    for name in ("Kinetic Energy", "Temperature", "Vphi", "Drift Frequency"):
        m = re.search(re.escape(name) + r"\s*:\s*([-0-9.]+)\s+([-0-9.]+)\s+([-0-9.]+)\s+([-0-9.]+)", rep)
        obs[name] = {"measured": float(m.group(1)), "suggested": float(m.group(2)), "sdev": float(m.group(4))}
    out = {
        "source": "tests/%s/main_input and tests/%s/Benchmark_Reports/00000400 of the reference" % (case, case),
        "chebyshev": not re.search(r"chebyshev\s*=\s*\.false\.", inp, re.I),
        "n_r": int(nml("n_r")),
        "n_theta": int(nml("n_theta")),
        "max_time_step": nml("max_time_step"),
        "max_iterations": int(nml("max_iterations")),
        "integration_interval": int(nml("benchmark_integration_interval")),
        "first_sample_iteration": iline("Beginning Iteration"),
        "last_sample_iteration": iline("Ending Iteration"),
        "samples": iline("Number of Samples"),
        "observables": obs,
    }
    with open(os.path.join(HERE, out_name), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


def main():
    extract("c2001_case0", "c2001_case0.json")
    extract("c2001_case0_FD_uniform", "c2001_case0_fd_uniform.json")


if __name__ == "__main__":
    main()
