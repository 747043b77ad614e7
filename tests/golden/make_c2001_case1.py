"""Extract the reference's known answer for its MHD accuracy benchmark.

Christensen et al. (2001) dynamo case 1 is set up by the reference's
``input_examples/c2001_case1_input`` (N_r = 64, N_theta = 96, benchmark_mode = 2,
150000 iterations, CFL-limited dt <= 1e-4) and ``src/Physics/Benchmarking.F90``,
whose benchmark_mode = 2 block names the reported observables and quotes their
suggested values (the published benchmark solution), the integration interval
(every 100 iterations) and the report interval (the last 10000 iterations).

Run from the repository root in a container that has the reference tree:

    python tests/golden/make_c2001_case1.py /path/to/reference

The output ``tests/golden/c2001_case1.json`` is committed; nothing at test
time reads the reference tree.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    inp = open(os.path.join(ref, "input_examples", "c2001_case1_input")).read()
    src = open(os.path.join(ref, "src", "Physics", "Benchmarking.F90")).read()

    def nml(name):
        m = re.search(r"^\s*%s\s*=\s*([-+0-9.dDeE]+)" % name, inp, re.M | re.I)
        return float(m.group(1).replace("d", "e").replace("D", "e"))

    # the benchmark_mode = 2 block of Benchmarking.F90's report set-up
    blocks = [m.start() for m in re.finditer(r"If \(benchmark_mode \.eq\. 2\) Then", src)]
    block = None
    for b in blocks:
        e = src.index("Endif", b)
        if "suggested_vals(1)" in src[b:e]:
            block = src[b:e]
    names = {int(i): n.strip(" :") for i, n in re.findall(r"report_names\((\d)\) = '([^']*)'", block)}
    sugg = {int(i): float(v.replace("d", "e")) for i, v in re.findall(r"suggested_vals\((\d)\) = ([-0-9.dD]+)", block)}
    interval = int(re.search(r"integration_interval = (\d+)", block).group(1))
    report = int(re.search(r"report_interval = (\d+)", block).group(1))
    out = {
        "source": "input_examples/c2001_case1_input and the benchmark_mode = 2 block of "
                  "src/Physics/Benchmarking.F90 of the reference",
        "n_r": int(nml("n_r")),
        "n_theta": int(nml("n_theta")),
        "max_time_step": nml("max_time_step"),
        "max_iterations": int(nml("max_iterations")),
        "cflmin": nml("cflmin"),
        "cflmax": nml("cflmax"),
        "integration_interval": interval,
        "report_interval": report,
        "suggested": {names[i]: sugg[i] for i in sorted(sugg)},
    }
    with open(os.path.join(HERE, "c2001_case1.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_c2001_case1.py /path/to/reference")
    main(sys.argv[1])
