"""Benchmark: Rayleigh timesteps/s at l_max = 511, N_r = 192 on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]
                    [--impl ours|reference] [--lmax 511] [--nr 192] [--err-steps 100]
                    [--equation-set dynamo|hydro|anelastic]

One JSON line on rank 0.  The workload is the large Boussinesq dynamo (the
magnetic equation set: W, P, T, Z and the potentials C, A of B; Ek = 1e-5,
Pr = Pm = 1) with seeded T and B perturbations.  A step is one pass of the hot
path (Post_Solve, rlm_spacea, physical_space, rlm_spaceb, AdvanceTime) over the
whole state; the state (~50 GB of buffers) stays resident in HBM and is far
larger than L2.
By default both forms run from the same seeded state: the line reports the
mixed-precision step, with the FP64 step and the per-field relative error of
the mixed state against the FP64 state after --err-steps steps beside it (the
FP64 form is reported instead if that error exceeds 1e-9).
``--impl reference`` times the reference algorithm on the host cores: the
NumPy restatement under ``oracle/`` (the Fortran reference cannot be built in
this image) on a sample of each stage; the line gives the timed seconds, the
factor that scales each stage's sample to the whole stage, and the full-step
estimate they make, plus whole steps measured at the l_max = 63, N_r = 48 size.
With N > 1 (torchrun) every rank runs an independent simulation, as the
reference's multi-run mode does (-nruns); the value sums the ranks' steps.
``--equation-set anelastic`` runs the anelastic MHD workload instead (the
nondimensional polytrope with 5 density scale heights and index 2, radius ratio
0.35, l_max = 255, N_r = 128, W, Z, P, S, C, A with viscous and ohmic heating,
seeded perturbations of amplitude 1e-4, mixed vs FP64 after 200 steps).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "steps/s at lmax=511,N_r=192: mixed-prec vs FP64 GPU at rel err≤1e-9; % roofline"
SEED = 0x5241594C


def headline_config(lmax, nr, precision, mag=True):
    """The large Boussinesq dynamo: rotating convection with the magnetic equation set
    (C, A potentials; insulating boundaries), radius ratio 0.35, Ek = 1e-5, Pr = Pm = 1,
    on an l_max x N_r grid (default l_max = 511, N_r = 192).  mag=False gives the same
    case without the magnetic field (the hydrodynamic equation set)."""
    return dict(n_r=nr, l_max=lmax, aspect_ratio=0.35, shell_depth=1.0, rayleigh=2.0e8, ekman=1.0e-5,
                prandtl=1.0, magnetic_prandtl=1.0, gravity_power=1.0, rotation=True, magnetism=mag,
                no_slip_top=True, no_slip_bottom=True, fix_tvar_top=True, fix_tvar_bottom=True, t_top=0.0,
                t_bottom=1.0, dt=1.0e-6, precision=precision)


def anelastic_config(lmax, nr, precision):
    """The anelastic MHD workload: the nondimensional polytrope (reference_type 3) with 5
    density scale heights and polytropic index 2 in a shell of radius ratio 0.35; the
    magnetic equation set with insulating boundaries; stress-free, fixed-entropy boundaries;
    viscous and ohmic heating on; Ek = 1e-3, Pr = 1, Pm = 2, Ra* = 0.5, dt = 1e-4."""
    return dict(n_r=nr, l_max=lmax, aspect_ratio=0.35, shell_depth=1.0, reference_type=3, poly_n=2.0,
                poly_nrho=5.0, modified_rayleigh=0.5, ekman=1.0e-3, prandtl=1.0, magnetic_prandtl=2.0,
                rotation=True, magnetism=True, no_slip_top=False, no_slip_bottom=False, fix_tvar_top=True,
                fix_tvar_bottom=True, t_top=0.0, t_bottom=1.0, dt=1.0e-4, precision=precision)


def workload_config(equation_set, lmax, nr, precision):
    if equation_set == "anelastic":
        return anelastic_config(lmax, nr, precision)
    return headline_config(lmax, nr, precision, equation_set == "dynamo")


SET_LABEL = {"dynamo": "dynamo (W, P, T, Z, C, A; insulating boundaries)",
             "hydro": "hydrodynamic (W, P, T, Z)",
             "anelastic": "anelastic dynamo (polytrope, 5 density scale heights; W, P, S, Z, C, A; "
                          "viscous and ohmic heating)"}


def workload_name(lmax, nr, mag, equation_set=None):
    if equation_set == "anelastic":
        return f"anelastic_dynamo_polytrope_nrho5_lmax{lmax}_nr{nr}"
    return f"boussinesq_{'dynamo' if mag else 'rotating_convection'}_lmax{lmax}_nr{nr}"


def initial_magnetic_state(ctx, lmax, nr, rng, amp=1e-3):
    """Seeded B: poloidal and toroidal potentials C, A on l in [1, 20], amplitude amp (l+1)^-2,
    as Chebyshev coefficients on the first 16 modes (m = 0 imaginary parts zero)."""
    n_lm = (lmax + 1) * (lmax + 2) // 2
    out = []
    ncoef = min(16, nr // 2)
    for _ in range(2):
        a = np.zeros((n_lm, 2, nr))
        for l in range(1, min(20, lmax) + 1):
            s = l * (l + 1) // 2
            block = rng.standard_normal((l + 1, 2, ncoef)) * amp * (l + 1.0) ** -2 / (1.0 + np.arange(ncoef)) ** 2
            block[0, 1] = 0.0
            a[s:s + l + 1, :, :ncoef] = block
        out.append(a)
    return out


def initial_state(ctx, lmax, nr, rng, amp=1e-3):
    """Conductive T plus a seeded perturbation on l in [1, 20] with (l+1)^-2 decay (coefficient space)."""
    n_lm = (lmax + 1) * (lmax + 2) // 2
    wpt = np.zeros((n_lm, 2, 3 * nr))
    z = np.zeros((n_lm, 2, nr))
    r = ctx.radius()
    r_out, r_in = r[0], r[-1]
    tcond = r_out * r_in / (r_in - r_out) * (1.0 / r_out - 1.0 / r) * math.sqrt(4 * math.pi)
    wpt[0, 0, 2 * nr:] = ctx.cheby_to_spectral(tcond[None])[0]
    ncoef = min(16, nr // 2)
    for l in range(1, min(20, lmax) + 1):
        s = l * (l + 1) // 2
        a = amp * (l + 1.0) ** -2
        block = rng.standard_normal((l + 1, 2, ncoef)) * a / (1.0 + np.arange(ncoef)) ** 2
        block[0, 1] = 0.0
        wpt[s:s + l + 1, :, 2 * nr:2 * nr + ncoef] = block
    return wpt, z


# ---------------------------------------------------------------------------
# algorithmic work per kernel (one launch = one step), FP64
# ---------------------------------------------------------------------------
def kernel_work(lmax, nr, nth, mag=True):
    """Algorithmic work of each stage per step: FLOPs (2 M N K per product) for the products,
    bytes (one read of the inputs, one write of the outputs) for the rest.  The magnetic set
    adds 6 fields to the inverse transform and the physical-space input (17 + 3 d/dphi),
    3 to the forward transform (7), 6 grids to the synthesis (18) and 2 per-l N_r x N_r solves."""
    L = lmax + 1
    n_lm = L * (L + 1) // 2
    nth2 = nth // 2
    kc = (2 * nr) // 3
    cols = 2 * n_lm
    nfa, nfb, ng = (17, 7, 18) if mag else (11, 4, 12)
    w = {}
    w["lt_inverse"] = ("tensor", 2.0 * nth2 * (nfa * nr * 2) * n_lm)
    w["lt_forward"] = ("tensor", 2.0 * nth2 * (nfb * nr * 2) * n_lm)
    w["cheb_synthesis"] = ("tensor", ng * 2.0 * (nr // 2) * kc * cols)
    w["solve"] = ("tensor", 2.0 * (9 + 1 + (2 if mag else 0)) * nr * nr * cols)
    plane = n_lm * 2 * nr * 8.0
    # post_assemble: grids + AB in, RHS + s2a out; magnetism: 6 grids + 2 AB in, 2 RHS + 5 s2am out
    w["post_assemble"] = ("hbm", ((12 + 4 + 4 + 7) + (15 if mag else 0)) * plane)
    # rlm_a: s2a in, s2a11 out; magnetism: s2am (5) in, 6 fields out
    w["rlm_a"] = ("hbm", ((7 + 11) + (11 if mag else 0)) * plane)
    # rlm_b: s2b in, ab out, rhs read and written; magnetism: 3 EMF fields in, C and A
    # histories, X written and read, the C and A right-hand sides read and written
    w["rlm_b"] = ("hbm", ((4 + 4 + 8) + (13 if mag else 0)) * plane)
    w["physics"] = ("hbm", L * nth * (nfa + nfb) * nr * 2 * 8.0)
    return w


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_peak_tflops(torch):
    """cuBLAS DGEMM 8192^3 on this GPU (best of 5): the FP64 tensor-pipe denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU leg: the oracle, sampled per stage (every number below is timed here)
# ---------------------------------------------------------------------------
class CpuSample:
    """One sampled step of the oracle at the benchmark size: every stage runs on a
    strided subset of its independent units (l for Post_Solve and the solve, m for
    the Legendre and rlm stages, a few theta rows for physical space).  The timed
    seconds of each stage and the factor that scales it to the whole stage are
    reported separately; the full-step estimate is their dot product."""

    def __init__(self, lmax, nr, stride=32, ntheta_rows=4, mag=True, equation_set=None):
        import oracle as O
        self.O = O
        self.mag = mag
        self.cores = os.cpu_count()
        O.set_fft_workers(self.cores)
        cfgd = workload_config(equation_set, lmax, nr, 0) if equation_set else headline_config(lmax, nr, 0, mag)
        cfg = O.Config(**{k: v for k, v in cfgd.items() if k in O.Config.__dataclass_fields__})
        t0 = time.perf_counter()
        self.o = O.Oracle(cfg)
        self.init_s = time.perf_counter() - t0
        self.cfg = cfg
        L = lmax + 1
        self.L = L
        n_lm = L * (L + 1) // 2
        self.ms = list(range(0, L, stride))
        self.ls = list(range(stride // 2, L, stride))
        f_m = sum(L - m for m in self.ms) / n_lm
        f_l = sum(l + 1 for l in self.ls) / n_lm
        self.thetas = np.linspace(0, cfg.n_theta - 1, ntheta_rows).astype(int)
        f_t = ntheta_rows / cfg.n_theta
        self.scale = {"post_solve": 1 / f_l, "rlm_a": 1 / f_m, "lt_inverse": 1 / f_m, "physics": 1 / f_t,
                      "lt_forward": 1 / f_m, "rlm_b": 1 / f_m, "solve": 1 / f_l}
        rng = np.random.Generator(np.random.PCG64(SEED))
        o = self.o
        self.s2a = {m: rng.standard_normal((o.NF1A, 2, nr, L - m)) for m in self.ms}
        self.s2a12 = {m: rng.standard_normal((o.NF2A, 2, nr, L - m)) for m in self.ms}
        self.p2b = {m: rng.standard_normal((o.NFB, 2, nr, cfg.n_theta)) for m in self.ms}
        self.s2b = {m: rng.standard_normal((o.NFB, 2, nr, L - m)) for m in self.ms}
        self.p3a = rng.standard_normal((o.NF2A, ntheta_rows, nr, cfg.n_phi + 2))
        lm_idx = np.concatenate([np.arange(l * (l + 1) // 2, l * (l + 1) // 2 + l + 1) for l in self.ls])
        self.lm_idx = lm_idx
        nv = 6 if mag else 4
        self.c = rng.standard_normal((nv, len(lm_idx), 2, nr))
        self.ab = rng.standard_normal((nv, len(lm_idx), 2, nr))
        self.rhs = {l: rng.standard_normal((3 * nr, 2 * (l + 1))) for l in self.ls}
        self.rhsz = {l: rng.standard_normal((nr, 2 * (l + 1))) for l in self.ls}
        self.sample = (f"per step: Post_Solve on l = {self.ls[0]}::{stride} ({f_l:.3f} of the (l,m) columns), "
                       f"rlm_spacea/StP/PtS/rlm_spaceb on m = 0::{stride} ({f_m:.3f} of the (l,m) rows), "
                       f"physical_space on {ntheta_rows} of {cfg.n_theta} theta rows, Implicit_Solve on l = "
                       f"{self.ls[0]}::{stride}; NumPy/BLAS and the phi FFTs on {self.cores} threads")

    def step_seconds(self):
        """Timed seconds of each stage's sample (nothing scaled)."""
        import scipy.linalg as sla
        o, cg = self.o, self.o.cg
        t = {}
        # Post_Solve: radial derivatives, From_Spectral, Add_Derivative on the sampled columns
        t0 = time.perf_counter()
        c = cg.dealias(self.c)
        W, P, T, Z = c[:4]
        ct = [cg.deriv(W, 3), cg.deriv(P, 1), cg.deriv(T, 2), cg.deriv(Z, 2)]
        gl = [W, P, T, Z, cg.deriv(W, 1), cg.deriv(T, 1), cg.deriv(Z, 1), cg.deriv(W, 2)]
        if self.mag:
            C, A = c[4], c[5]
            ct.append(cg.deriv(A, 2))
            gl += [C, A, cg.deriv(C, 1), cg.deriv(A, 1), cg.deriv(C, 2)]
        ctemp = cg.from_spectral(cg.dealias(np.stack(ct)))
        g = cg.from_spectral(cg.dealias(np.stack(gl)))
        p1b = self.ab * 0.5
        src = {(0, 0): g[0], (0, 1): g[4], (0, 2): g[7], (0, 3): ctemp[0], (1, 0): g[1], (1, 1): ctemp[1],
               (2, 0): g[2], (2, 1): g[5], (2, 2): ctemp[2], (3, 0): g[3], (3, 1): g[6], (3, 2): ctemp[3]}
        if self.mag:
            src.update({(4, 0): g[8], (4, 2): g[12], (5, 0): g[9], (5, 1): g[11], (5, 2): ctemp[4]})
        off = 0
        for l in self.ls:
            sl = slice(off, off + l + 1)
            for (eq, var, d), cf in o.coefs[l].items():
                if (var, d) in src:
                    p1b[eq, sl] += src[(var, d)][sl] * cf
            off += l + 1
        t["post_solve"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        o.rlm_spacea(self.s2a, ms=self.ms)
        t["rlm_a"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        o.h.s2p(self.s2a12, ms=self.ms)
        t["lt_inverse"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        o.physical_space(self.p3a, thetas=self.thetas, diagnostics=False)
        t["physics"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        o.h.p2s(self.p2b, ms=self.ms)
        t["lt_forward"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        o.rlm_spaceb(self.s2b, ms=self.ms)
        t["rlm_b"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        if self.mag:   # Finalize_EMF's radial derivative on the sampled columns (AdvanceTime)
            cg.from_spectral(cg.dealias(cg.deriv(cg.to_spectral(self.c[5]), 1)))
        for l in self.ls:
            sla.lu_solve(o.lu_wpt[l], self.rhs[l], check_finite=False)
            if l > 0:
                sla.lu_solve(o.lu_z[l], self.rhsz[l], check_finite=False)
                if self.mag:
                    sla.lu_solve(o.lu_c[l], self.rhsz[l], check_finite=False)
                    sla.lu_solve(o.lu_a[l], self.rhsz[l], check_finite=False)
        t["solve"] = time.perf_counter() - t0
        return t

    def full_step_estimate(self, timed):
        return sum(timed[k] * self.scale[k] for k in timed)

    def report(self, timed_steps):
        """cpu_baseline fields from a list of per-stage timings (one dict per sampled step)."""
        mean = {k: float(np.mean([t[k] for t in timed_steps])) for k in timed_steps[0]}
        full = self.full_step_estimate(mean)
        return {"value": 1.0 / full, "unit": "steps/s", "cores": self.cores, "kind": "port", "sample": self.sample,
                "timed_seconds_per_sampled_step": round(sum(mean.values()), 4),
                "timed_seconds_per_stage": {k: round(v, 4) for k, v in mean.items()},
                "scale_to_full_stage": {k: round(v, 3) for k, v in self.scale.items()},
                "full_step_seconds_estimate": round(full, 3),
                "value_how": "1 / sum over stages of (timed sample seconds x scale to the full stage)"}


C1_CFG = dict(n_r=48, l_max=63, dt=1.0e-4, rayleigh=1.0e5, ekman=1.0e-3)   # the FP64 timestep-loop case


def cpu_c1_steps_per_s(nsteps=3):
    """Whole oracle steps (nothing sampled) at the l_max = 63, N_r = 48 timestep-loop size."""
    import oracle as O
    O.set_fft_workers(os.cpu_count())
    oc = O.Config(**C1_CFG)
    o = O.Oracle(oc)
    wpt, z = O.seeded_state(oc, amp=1e-3, lmax_pert=20)
    o.init_state(wpt, z)
    o.step()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        o.step()
    return nsteps / (time.perf_counter() - t0)


def run_reference(args, rank):
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    mag = args.equation_set in ("dynamo", "anelastic")
    cs = CpuSample(args.lmax, args.nr, mag=mag, equation_set=args.equation_set)
    for _ in range(args.warmup):
        cs.step_seconds()
    timed = [cs.step_seconds() for _ in range(args.steps)]
    cpu = cs.report(timed)
    cpu["c1_full_steps_per_s"] = round(cpu_c1_steps_per_s(), 4)
    value = cpu["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        # the time actually spent per timed (sampled) step; value is the full-step estimate
        "ms_per_step": cpu["timed_seconds_per_sampled_step"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": workload_name(args.lmax, args.nr, mag, args.equation_set), "l_max": args.lmax,
                   "n_r": args.nr, "n_theta": cs.cfg.n_theta, "n_phi": cs.cfg.n_phi,
                   "equation_set": SET_LABEL[args.equation_set],
                   "l2": "working set larger than L2"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def max_over_ranks(value, world, dist, torch, device):
    """The largest value over all ranks (a device-timed duration: the job's time is its slowest rank's)."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def ensemble_rate(steps_per_rank, max_ms, world):
    """Whole-job steps/s of `world` independent replicas that each ran `steps_per_rank` steps."""
    return world * steps_per_rank / (max_ms * 1e-3)


def run_precision(args, prec_name, rank, world, torch, dist, fp64_peak, peaks, peak_kind):
    """Times one precision form on this rank; returns (line fields or None off rank 0, state at step err_steps)."""
    import ctypes
    import rayleigh_b200 as rb
    local = int(os.environ.get("LOCAL_RANK", "0"))
    prec = rb.PREC_MIXED if prec_name == "mixed" else rb.PREC_FP64
    mag = args.equation_set in ("dynamo", "anelastic")
    cfgd = workload_config(args.equation_set, args.lmax, args.nr, prec)
    ctx = rb.Rayleigh(rb.Config(**cfgd, use_graph=True, device=local))
    rng = np.random.Generator(np.random.PCG64(SEED + rank))
    amp = 1e-4 if args.equation_set == "anelastic" else 1e-3
    wpt, z = initial_state(ctx, args.lmax, args.nr, rng, amp)
    ctx.put_state(wpt, z, None, iteration=1)
    if mag:
        cpol, ator = initial_magnetic_state(ctx, args.lmax, args.nr, rng, amp)
        ctx.put_magnetic_state(cpol, ator)
    # warm-up (includes the Euler first step and the capture of the step graph)
    ctx.step(max(3, args.warmup))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms = ctx.step_timed(args.steps)          # graph replays, CUDA events on the context stream
    launches = ctx.launch_count()
    torch.cuda.synchronize()
    max_ms = max_over_ranks(total_ms, world, dist, torch, "cuda")
    if world > 1:
        dist.barrier()
    value = ensemble_rate(args.steps, max_ms, world)
    # per-kernel times (eager launches, an event around each kernel) for the breakdown and roofline
    nk_steps = min(args.steps, 5)
    k_total, per_kernel = ctx.time_steps(nk_steps)
    # continue (untimed) to err_steps for the mixed-vs-FP64 comparison
    done = max(3, args.warmup) + args.steps + nk_steps
    if args.err_steps > done:
        ctx.step(args.err_steps - done)
    state = (ctx.get_state()[:2] + (ctx.get_magnetic_state()[:2] if mag else ())) if rank == 0 else None

    # end to end through the C ABI with host buffers: H2D of the full state, one
    # step, D2H of the new state and its CFL cargo, every step
    n_lm = ctx.n_lm
    nr = args.nr
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    h_wpt, h_z, h_ab = pin(n_lm * 2 * 3 * nr), pin(n_lm * 2 * nr), pin(4 * n_lm * 2 * nr)
    o_wpt, o_z, o_ab = pin(n_lm * 2 * 3 * nr), pin(n_lm * 2 * nr), pin(4 * n_lm * 2 * nr)
    w0, z0, ab0 = ctx.get_state()
    h_wpt[:] = w0.ravel()
    h_z[:] = z0.ravel()
    h_ab[:] = ab0.ravel()
    if mag:   # the magnetic part: C, A and their AB terms, both ways
        hm = [pin(n_lm * 2 * nr), pin(n_lm * 2 * nr), pin(2 * n_lm * 2 * nr)]
        om = [pin(n_lm * 2 * nr), pin(n_lm * 2 * nr), pin(2 * n_lm * 2 * nr)]
        for dst, src in zip(hm, ctx.get_magnetic_state()):
            dst[:] = src.ravel()
    lib = ctx.lib
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    e2e_steps = max(1, min(args.steps, 5))
    cfl = ctypes.c_double()
    it = 1000
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx._check(lib.ra_put_state(ctx.h, P(h_wpt), P(h_z), P(h_ab), it))
        if mag:
            ctx._check(lib.ra_put_magnetic_state(ctx.h, P(hm[0]), P(hm[1]), P(hm[2])))
        ctx._check(lib.ra_step(ctx.h, 1, ctypes.byref(cfl)))
        ctx._check(lib.ra_get_state(ctx.h, P(o_wpt), P(o_z), P(o_ab)))
        if mag:
            ctx._check(lib.ra_get_magnetic_state(ctx.h, P(om[0]), P(om[1]), P(om[2])))
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    h2d = (h_wpt.nbytes + h_z.nbytes + h_ab.nbytes) + (sum(a.nbytes for a in hm) if mag else 0)
    d2h = (o_wpt.nbytes + o_z.nbytes + o_ab.nbytes + 8) + (sum(a.nbytes for a in om) if mag else 0)
    e2e_value = world / max_over_ranks(e2e_s, world, dist, torch, "cuda")
    n_theta, n_phi = ctx.n_theta, ctx.n_phi
    ctx.close()
    del h_wpt, h_z, h_ab, o_wpt, o_z, o_ab
    if mag:
        del hm, om
    if rank != 0:
        return None, None
    # roofline of the dominant kernel
    work = kernel_work(args.lmax, args.nr, n_theta, mag)
    dom = max(per_kernel, key=lambda k: per_kernel[k])
    bound, amount = work[dom]
    avg_s = per_kernel[dom] / nk_steps * 1e-3
    traffic = None
    binding = None
    tpath = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            traffic = tj.get(f"{dom}_{args.equation_set}_{prec_name}_lmax{args.lmax}_nr{args.nr}")
            binding = tj.get(f"{dom}_binding_unit")   # the unit ncu shows saturated, when it is not HBM
        except Exception:
            traffic = None
    if bound == "tensor":
        achieved = amount / avg_s / 1e12
        peak, unit = fp64_peak, "TFLOP/s"
        peak_note = "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe)"
    else:
        achieved = amount / avg_s / 1e9
        peak, unit = peaks["hbm_gbs"], "GB/s"
        peak_note = f"{peak_kind} HBM copy bandwidth (MEASURED_PEAKS.json)"
    kernels = {}
    for k, ms in per_kernel.items():
        b, amt = work[k]
        sec = ms / nk_steps * 1e-3
        rate = amt / sec / (1e12 if b == "tensor" else 1e9)
        kernels[k] = {"ms_per_step": round(ms / nk_steps, 4), "share": round(ms / k_total, 4),
                      ("tflops" if b == "tensor" else "gbs"): round(rate, 2)}
        # fraction of the measured peak: HBM copy for byte-bound kernels; for the FP64
        # form's products, the cuBLAS DGEMM rate (FP64 tensor pipe) of this run
        if b != "tensor":
            kernels[k]["frac_of_hbm"] = round(rate / peaks["hbm_gbs"], 3)
        elif prec_name == "fp64" and fp64_peak:
            kernels[k]["frac_of_dgemm"] = round(rate / fp64_peak, 3)
    fields = {
        "value": value, "ms_per_step": max_ms / args.steps, "precision": prec_name,
        "timing": f"value: {args.steps} steps replayed from the captured step graph, CUDA events on the context "
                  f"stream; kernels: {nk_steps} eager steps with an event around each kernel",
        "config": {"workload": workload_name(args.lmax, args.nr, mag, args.equation_set), "l_max": args.lmax,
                   "n_r": args.nr, "n_theta": n_theta, "n_phi": n_phi, "ekman": cfgd["ekman"],
                   "rayleigh": cfgd.get("rayleigh", cfgd.get("modified_rayleigh")), "prandtl": cfgd["prandtl"],
                   "magnetic_prandtl": cfgd["magnetic_prandtl"] if mag else None, "dt": cfgd["dt"],
                   "l2": "working set (GBs of state and buffers) larger than the 126 MB L2; no flush needed",
                   "equation_set": SET_LABEL[args.equation_set],
                   "parallelism": "replicas (multi-run ensemble)" if world > 1 else "single GPU"},
        "roofline": {"kernel": dom, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                     "frac": achieved / peak if peak else None, "traffic": traffic,
                     "traffic_unit": "GB per launch (ncu dram bytes read + written)" if traffic is not None else None,
                     "algorithmic": amount / (1e12 if bound == "tensor" else 1e9),
                     "algorithmic_unit": "TFLOP per launch" if bound == "tensor" else "GB per launch",
                     "peak_source": peak_note, "binding_unit": binding},
        "kernels": kernels,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "how": "ra_put_state (pinned host) + ra_step(1) + ra_get_state (pinned host) per step"},
    }
    return fields, state


def _field_errors(mixed_state, fp64_state, nr):
    wm, zm = mixed_state[:2]
    wf, zf = fp64_state[:2]
    pairs = [("W", wm[:, :, :nr], wf[:, :, :nr]), ("P", wm[:, :, nr:2 * nr], wf[:, :, nr:2 * nr]),
             ("T", wm[:, :, 2 * nr:], wf[:, :, 2 * nr:]), ("Z", zm, zf)]
    if len(mixed_state) == 4:
        pairs += [("C", mixed_state[2], fp64_state[2]), ("A", mixed_state[3], fp64_state[3])]
    out = {}
    for name, a, b in pairs:
        den = float(np.linalg.norm(b))
        out[name] = float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a))
    return out


def run_ours(args, rank, world, torch, dist):
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    peaks, peak_kind = measured_peaks()
    fp64_peak = fp64_peak_tflops(torch) if rank == 0 else None
    forms = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    res = {}
    for f in forms:
        res[f] = run_precision(args, f, rank, world, torch, dist, fp64_peak, peaks, peak_kind)
    if rank != 0:
        return
    head_form = "mixed" if "mixed" in res else "fp64"
    head, _ = res[head_form]
    line = {"metric": METRIC, "value": head["value"], "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "precision": head_form,
            "data": "synthetic (seeded)", "fp64_dgemm_tflops": fp64_peak}
    for k in ("config", "roofline", "kernels", "gpu_launches", "clocks", "e2e", "timing"):
        line[k] = head[k]
    if len(res) == 2:
        f64, _ = res["fp64"]
        errs = _field_errors(res["mixed"][1], res["fp64"][1], args.nr)
        worst = max(errs.values())
        line["fp64"] = {k: f64[k] for k in ("value", "ms_per_step", "roofline", "kernels", "gpu_launches",
                                            "clocks", "e2e")}
        line["mixed_vs_fp64"] = {"speedup": head["value"] / f64["value"],
                                 "rel_err_per_field": errs, "max_rel_err": worst, "tolerance": 1e-9,
                                 "within_tolerance": worst <= 1e-9, "steps_compared": args.err_steps,
                                 "how": "relative L2 norm per field of the state after the same steps from the "
                                        "same seeded initial state"}
        if worst > 1e-9:
            # the mixed number does not meet the accuracy bound: report the FP64 form as the headline
            line["value"] = f64["value"]
            line["ms_per_step"] = f64["ms_per_step"]
            line["precision"] = "fp64"
            for k in ("roofline", "kernels", "gpu_launches", "clocks", "e2e"):
                line[k] = f64[k]
    if args.c1:
        line["c1_measured"] = c1_comparison(args, torch)
    if not args.no_cpu:
        cs = CpuSample(args.lmax, args.nr, mag=args.equation_set in ("dynamo", "anelastic"),
                       equation_set=args.equation_set)
        cs.step_seconds()
        line["cpu_baseline"] = cs.report([cs.step_seconds()])
    print(json.dumps(line), flush=True)


def c1_comparison(args, torch):
    """Whole steps, nothing sampled, at the l_max = 63, N_r = 48 timestep-loop size: the GPU
    (FP64 form, graph replays) against the oracle on the host cores."""
    import rayleigh_b200 as rb
    ctx = rb.Rayleigh(rb.Config(**C1_CFG, use_graph=True, precision=rb.PREC_FP64,
                                device=int(os.environ.get("LOCAL_RANK", "0"))))
    rng = np.random.Generator(np.random.PCG64(SEED))
    wpt, z = initial_state(ctx, C1_CFG["l_max"], C1_CFG["n_r"], rng)
    ctx.put_state(wpt, z, None, iteration=1)
    ctx.step(5)
    n = 200
    gpu = n / (ctx.step_timed(n) * 1e-3)
    ctx.close()
    cpu = cpu_c1_steps_per_s()
    return {"config": "l_max=63, N_r=48, hydrodynamic Boussinesq (the FP64 timestep-loop case)",
            "gpu_fp64_steps_per_s": gpu, "cpu_oracle_steps_per_s": cpu, "cpu_cores": os.cpu_count(),
            "ratio": gpu / cpu, "how": f"{n} GPU steps (graph replays, CUDA events) vs 3 whole oracle steps"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: time the FP64 and the mixed form, report the mixed one with its error vs FP64")
    ap.add_argument("--err-steps", type=int, default=None,
                    help="steps after which the mixed and FP64 states are compared (100; 200 anelastic)")
    ap.add_argument("--lmax", type=int, default=None, help="511 (255 anelastic)")
    ap.add_argument("--nr", type=int, default=None, help="192 (128 anelastic)")
    ap.add_argument("--equation-set", default="dynamo", choices=["dynamo", "hydro", "anelastic"],
                    help="dynamo: the magnetic equation set (the large Boussinesq dynamo); hydro: without B; "
                         "anelastic: the anelastic MHD workload (polytrope, l_max 255, N_r 128)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-c1", dest="c1", action="store_false",
                    help="skip the whole-step GPU/CPU comparison at the l_max = 63, N_r = 48 size")
    args = ap.parse_args()
    anel = args.equation_set == "anelastic"
    if args.lmax is None:
        args.lmax = 255 if anel else 511
    if args.nr is None:
        args.nr = 128 if anel else 192
    if args.err_steps is None:
        args.err_steps = 200 if anel else 100
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(args, rank, world, torch, dist)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
