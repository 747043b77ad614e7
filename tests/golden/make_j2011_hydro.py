"""Extract the reference's known answer for its anelastic hydrodynamic benchmark.

Jones et al. (2011), the anelastic hydrodynamic case, is set up by the reference's
``input_examples/j2011_steady_hydro_minimal`` (N_r = 128, N_theta = 192,
benchmark_mode = 3, 200000 iterations) and the benchmark_mode = 3 blocks of
``src/Physics/Benchmarking.F90``: the first imposes the physics (the cgs polytrope,
stress-free, fixed-entropy boundaries, dt <= 30 s, the CFL limits), the second names
the reported observables and quotes their suggested values (the published solution),
the integration interval (every 100 iterations) and the report interval (the last
10000 iterations).

Run from the repository root in a container that has the reference tree:

    python tests/golden/make_j2011_hydro.py /path/to/reference

The output ``tests/golden/j2011_hydro.json`` is committed; nothing at test time
reads the reference tree.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _num(v):
    return float(v.replace("d", "e").replace("D", "e"))


def main(ref):
    inp = open(os.path.join(ref, "input_examples", "j2011_steady_hydro_minimal")).read()
    src = open(os.path.join(ref, "src", "Physics", "Benchmarking.F90")).read()

    def nml(name):
        m = re.search(r"^\s*%s\s*=\s*([-+0-9.dDeE]+)" % name, inp, re.M | re.I)
        return _num(m.group(1))

    blocks = []
    for m in re.finditer(r"If \(benchmark_mode \.eq\. 3\) Then", src):
        nxt = re.compile(r"If \(benchmark_mode \.eq\. \d\) Then").search(src, m.end())
        blocks.append(src[m.start():nxt.start() if nxt else len(src)])
    setup = next(b for b in blocks if "max_time_step" in b)
    report = next(b for b in blocks if "suggested_vals(1)" in b)

    def val(block, name):
        return _num(re.search(r"^\s*%s\s*=\s*([-+0-9.dDeE]+)" % name, block, re.M | re.I).group(1))

    names = {int(i): n.strip(" :") for i, n in re.findall(r"report_names\((\d)\) = '([^']*)'", report)}
    sugg = {int(i): _num(v) for i, v in re.findall(r"suggested_vals\((\d)\) = ([-0-9.dDeE]+)", report)}
    out = {
        "source": "input_examples/j2011_steady_hydro_minimal and the benchmark_mode = 3 blocks of "
                  "src/Physics/Benchmarking.F90 of the reference",
        "n_r": int(nml("n_r")),
        "n_theta": int(nml("n_theta")),
        "max_iterations": int(nml("max_iterations")),
        "max_time_step": val(setup, "max_time_step"),
        "cflmin": val(setup, "cflmin"),
        "cflmax": val(setup, "cflmax"),
        "alpha_implicit": val(setup, "alpha_implicit"),
        "t_bottom": val(setup, "T_Bottom"),
        "rmin": val(setup, "rmin"),
        "rmax": val(setup, "rmax"),
        "poly_n": val(setup, "poly_n"),
        "poly_nrho": val(setup, "poly_Nrho"),
        "poly_mass": val(setup, "poly_mass"),
        "poly_rho_i": val(setup, "poly_rho_i"),
        "pressure_specific_heat": val(setup, "pressure_specific_heat"),
        "angular_velocity": val(setup, "angular_velocity"),
        "nu_top": val(setup, "nu_top"),
        "kappa_top": val(setup, "kappa_top"),
        "integration_interval": int(re.search(r"integration_interval = (\d+)", report).group(1)),
        "report_interval": int(re.search(r"report_interval = (\d+)", report).group(1)),
        "msymm": int(re.search(r"msymm = (\d+)", report).group(1)),
        "suggested": {names[i]: sugg[i] for i in sorted(sugg)},
    }
    with open(os.path.join(HERE, "j2011_hydro.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_j2011_hydro.py /path/to/reference")
    main(sys.argv[1])
