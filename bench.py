#!/usr/bin/env python
"""DOF-updates/s of the fused DGSEM tendency + LSRK(5,4) path on B200.

Workload (default): 3-D compressible Euler, periodic 32^3 brick of hex elements on
[0,10]^3, N = 7 (512 nodes/element, 16.8 M nodes, 83.9 M DOF), Kennedy-Gruber
flux-differencing volume term, Rusanov surface flux, isentropic vortex (strength 5,
background Mach 0.5, z-invariant), LSRK(5,4) at CFL 0.4, FP64.  One bench step is one
LSRK(5,4) time step (5 fused stage kernels).  The 1.3 GB state is larger than L2
(126 MB), so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Serving workload (--workload serve_poisson_mix_fp32bulk): a seeded stream of --requests
independent solves arriving as a Poisson process at --rate per second (dim 2 or 3,
advection or Euler, N in {3, 5, 7}, 8-64 (2-D) or 4-32 (3-D) elements per side,
50-500 LSRK(5,4) steps, FP32 bulk) is replayed against the serving loop; the line
reports p50/p99 latency and solves/s beside the DOF-update rate.

Multi-GPU (torchrun): the workload's elements are partitioned over the ranks, which
exchange face traces before every stage (strong scaling; `--replicas` runs one
independent replica per rank instead); time is the max over ranks.

The default line also carries the FP32-bulk form of the same workload timed in the same
process (`fp32_bulk`), its accuracy against the FP64 form and the exact solution after
`--accuracy-steps` steps, and a short serving stream (`serving`).
"""

import argparse
import ctypes
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: dim, N, elements per side, domain side, law, volume flux, precision, warp
    "euler3d_kg_n7_32_fp64": dict(dim=3, N=7, K=32, L=10.0, law="euler", vflux="kg", precision="fp64", warp=False),
    "euler3d_kg_n7_32_fp32bulk": dict(dim=3, N=7, K=32, L=10.0, law="euler", vflux="kg", precision="fp32_bulk",
                                      warp=False),
    "euler3d_kg_n7_32_fp32bulk_warped": dict(dim=3, N=7, K=32, L=10.0, law="euler", vflux="kg",
                                             precision="fp32_bulk", warp=True),
    "euler3d_kg_n7_32_fp64_warped": dict(dim=3, N=7, K=32, L=10.0, law="euler", vflux="kg", precision="fp64",
                                         warp=True),
    "adv2d_weak_n4_16_fp64": dict(dim=2, N=4, K=16, L=1.0, law="advection", vflux="weak", precision="fp64",
                                  warp=False),
    # one field, velocity (1, 0.5, 0.25), sine + Gaussian: the pipelined advection kernel
    "adv3d_weak_n7_32_fp64": dict(dim=3, N=7, K=32, L=1.0, law="advection", vflux="weak", precision="fp64",
                                  warp=False),
    "adv3d_weak_n7_32_fp32bulk": dict(dim=3, N=7, K=32, L=1.0, law="advection", vflux="weak",
                                      precision="fp32_bulk", warp=False),
    # adapted: 4^3 trees on the periodic unit cube, refined twice within radius 0.25 of the
    # centre (2:1 balanced, hanging faces coupled by mortars), N = 5, density pulse
    "euler3d_kg_n5_adapted_fp32bulk": dict(dim=3, N=5, K=4, L=1.0, law="euler", vflux="kg", precision="fp32_bulk",
                                           warp=False, adapted=True),
}
ADV_VELOCITY = (1.0, 0.5, 0.25)  # advection workloads (the first dim components)
SERVE_WORKLOAD = "serve_poisson_mix_fp32bulk"
DEFAULT = "euler3d_kg_n7_32_fp64"
METRIC = "DOF-updates/s per RHS"
UNIT = "DOF-updates/s"


def load_product():
    if "raven_b200" in sys.modules:
        return sys.modules["raven_b200"]
    pkg = os.path.join(ROOT, "raven.jl_b200")
    spec = importlib.util.spec_from_file_location("raven_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["raven_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def config_json(name, w, grid=None):
    if grid is not None and w.get("adapted"):
        return {
            "workload": name,
            "equation": "euler",
            "dim": w["dim"],
            "polynomial_order": w["N"],
            "elements": grid.E,
            "nodes": grid.E * grid.np,
            "trees": w["K"] ** w["dim"],
            "refinement": "two rounds within radius 0.25 of the centre of the periodic unit cube, 2:1 face balance",
            "mortars": int(grid.mortars.shape[1]),
            "volume_form": "flux_differencing_kennedy_gruber",
            "surface_flux": "rusanov",
            "precision": w["precision"],
            "geometry": "adapted brick (hanging faces coupled by mortars)",
            "time_stepper": "LSRK54",
            "initial_data": "density pulse 1 + 0.2 exp(-|x - c|^2 / 0.01) at rest, pressure 1",
            "l2_flush": "none: the state (6.4 MB) is L2-resident",
            "parallelism": "replicas",
        }
    return {
        "workload": name,
        "equation": "euler" if w["law"] == "euler" else "advection",
        "dim": w["dim"],
        "polynomial_order": w["N"],
        "elements": w["K"] ** w["dim"],
        "nodes": w["K"] ** w["dim"] * (w["N"] + 1) ** w["dim"],
        "volume_form": "flux_differencing_kennedy_gruber" if w["vflux"] == "kg" else "weak",
        "surface_flux": "rusanov",
        "precision": w["precision"],
        "geometry": "warped" if w["warp"] else "brick",
        "time_stepper": "LSRK54",
        "initial_data": "isentropic_vortex" if w["law"] == "euler" else "sine_plus_gaussian",
        "l2_flush": "not needed: state larger than L2" if w["K"] >= 32 else "state is L2-resident",
        "parallelism": "replicas",
    }


def sine_warp(L, dim):
    import numpy as np

    def warp(*x):
        s = 1.0
        for d in range(dim):
            s = s * np.sin(np.pi * (x[d] / L))
        return [x[d] + (0.1 * L) * s for d in range(dim)]

    return warp


def setup(rb, w, device):
    grid, law, form, q0, dt = problem(rb, w)
    dg = rb.DGSEM(law=law, grid=grid, volume_form=form, surface_numericalflux=rb.RusanovFlux(),
                  precision=w["precision"], device=device)
    return grid, law, dg, q0, dt


def problem(rb, w):
    """The workload's grid, law, volume form, initial state and time step."""
    from raven_b200 import initial_conditions as ic

    dim, N, K, L = w["dim"], w["N"], w["K"], w["L"]
    cell = rb.LobattoCell(*([N + 1] * dim))
    coords = tuple(rb.jl_range(0.0, L, K + 1) for _ in range(dim))
    cg = rb.brick(coords, (True,) * dim)
    gm = rb.GridManager(cell, cg)
    if w.get("adapted"):
        from raven_b200.forest import sphere_refinement_flags

        centre = (L / 2,) * dim
        for _ in range(2):
            rb.adapt(gm, sphere_refinement_flags(gm.forest, coords, centre, L / 4))
    grid = rb.generate(sine_warp(L, dim), gm) if w["warp"] else rb.generate(gm)
    if w.get("adapted"):
        # density pulse rho = 1 + 0.2 exp(-|x - c|^2 / 0.01) at rest, uniform pressure 1
        law = rb.EulerLaw(dim)
        q0 = ic.density_pulse(grid, law, center=(L / 2,) * dim, amplitude=0.2, width2=0.01)
        form = rb.FluxDifferencingForm(rb.KennedyGruberFlux())
        dt = 0.4 * grid.min_node_distance() / ic.max_wavespeed(grid, law, q0)
    elif w["law"] == "euler":
        law = rb.EulerLaw(dim)
        u0 = 0.5 * math.sqrt(law.gamma)
        q0 = ic.isentropic_vortex(grid, law, beta=5.0, u0=u0, center=(L / 2, L / 2))
        form = rb.FluxDifferencingForm(rb.KennedyGruberFlux())
        # CFL on Raven's min_node_distance (grids.jl:122-145); the Δx/N form is unstable
        # for N = 7 in 3-D at CFL 0.4 (the oracle blows up after 22 steps as well)
        dt = 0.4 * grid.min_node_distance() / ic.max_wavespeed(grid, law, q0)
    else:
        law = rb.AdvectionLaw(dim, ADV_VELOCITY[:dim])
        q0 = ic.sine_plus_gaussian(grid, law, sigma=0.05)
        form = rb.WeakForm()
        dt = 0.5 * grid.min_node_distance() / math.hypot(*law.u)
    return grid, law, form, q0, dt


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_figure(name, key):
    """A figure of the stage kernel from the committed ncu summary of this workload
    (`dram_bytes_per_launch`, `fp64_flops_per_node`), if any."""
    path = os.path.join(ROOT, "profiles", f"stage_kernel_{name}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def profiled_traffic(name):
    """dram bytes per launch of the stage kernel from the committed ncu summary, if any."""
    return profiled_figure(name, "dram_bytes_per_launch")


FP64_NOMINAL_TFLOPS = 37.0  # B200 datasheet FP64, used only if the measurement fails


def measured_fp64_tflops(rb):
    """FP64 fma throughput of this GPU (rb200_probe_fp64_rate: 8 CTAs per SM x 256
    threads x 8 independent fma chains, CUDA events, best of 3), or None."""
    out = ctypes.c_double(0.0)
    st = rb._lib.lib().rb200_probe_fp64_rate(1 << 16, ctypes.byref(out), None)
    return out.value if st == 0 and out.value > 0 else None


def stage_bytes_per_launch(w, nodes, ns):
    """Algorithmic HBM bytes of one stage launch, averaged over the 5 stages of a step:
    q read + q write (FP64) + dq write every stage + dq read in stages 2-5 (stage 1 has
    rka = 0), plus the per-node metrics of a curved grid (wJ*dRdX rows + MJI, and n,
    wsJ on 0.75 face slots per node at N = 7)."""
    dqb = 4 if w["precision"] == "fp32_bulk" else 8
    per_step = nodes * ns * (5 * 16 + 5 * dqb + 4 * dqb)
    if w["warp"]:
        dim, nq = w["dim"], w["N"] + 1
        per_node_geo = (dim * dim + 1) * 8 + (2 * dim * nq ** (dim - 1)) * (dim + 1) * 8 / nq**dim
        per_step += 5 * nodes * per_node_geo
    return per_step / 5.0


def timed_launches(dg, steps):
    """Kernels of ours launched by one lsrk54_steps call of `steps` steps: one for the
    cluster step kernel, else the stage (and mortar) kernels of each step."""
    return 1 if getattr(dg, "cluster_ctas", 0) > 0 else int(dg.info[6]) * steps


def kernel_name(w, dg):
    """The stage kernel the handle launches for this workload."""
    if w.get("serve"):
        return "batched_stage_kernel (all running solves of a class per launch)"
    if getattr(dg, "cluster_ctas", 0) > 0:
        return (f"cluster_adv_steps_kernel (one thread-block cluster of {dg.cluster_ctas} CTAs runs every stage "
                "of the timed steps in one launch)")
    if dg.pipelined_ctas > 0:
        if dg.geometry == "curved":
            if w["precision"] == "fp64":
                return "pipelined_curved64_kernel (3-D Nq=8 curved, FP64, fused volume + surface + LSRK stage)"
            return "pipelined_curved_kernel (3-D Nq=8 curved, FP32 bulk, fused volume + surface + LSRK stage)"
        extra = " with mortar fluxes" if w.get("adapted") else ""
        if w.get("law") == "advection":
            return f"pipelined_adv_kernel (3-D Nq={w['N'] + 1} brick{extra}, weak-form advection, fused stage)"
        return f"pipelined_stage_kernel (3-D Nq={w['N'] + 1} brick{extra}, fused volume + surface + LSRK stage)"
    return "stage_kernel (fused volume + surface + LSRK stage)"


def rel_max_norm(rb, dg, a, b):
    """max |a| / max |b| through the library's max-norm (weightednorm(dg, q, Inf))."""
    return rb.weightednorm(dg, a, math.inf) / rb.weightednorm(dg, b, math.inf)


def fp64_comparison(rb, w, grid, law, dg, q0, dt, steps, device, exact=None):
    """The FP32-bulk run against an FP64 run on the same grid from the same state, every
    100 steps (untimed): relative L2 (MJ-weighted) and max-norm differences.  With
    `exact(t)` (the exact state at time t) both runs' errors against it at the end."""
    form = rb.FluxDifferencingForm(rb.KennedyGruberFlux() if w["vflux"] == "kg" else rb.EntropyConservativeFlux())
    dg64 = rb.DGSEM(law=law, grid=grid, volume_form=form, surface_numericalflux=rb.RusanovFlux(), precision="fp64",
                    device=device)
    q32, q64 = rb.GridArray.from_numpy(q0), rb.GridArray.from_numpy(q0)
    dq32, dq64 = q32.similar(), q64.similar()
    rows, done = [], 0
    while done < steps:
        n = min(100, steps - done)
        dg.lsrk54_steps(q32, dq32, done * dt, dt, n)
        dg64.lsrk54_steps(q64, dq64, done * dt, dt, n)
        done += n
        diff = q64.copy()
        diff.data.sub_(q32.data)
        rows.append({"step": done, "l2_diff_relative": rb.weightednorm(dg64, diff) / rb.weightednorm(dg64, q64),
                     "max_diff_relative": rel_max_norm(rb, dg64, diff, q64)})
        del diff
    I0 = rb.integrals(dg64, rb.GridArray.from_numpy(q0))
    I32, I64 = rb.integrals(dg64, q32), rb.integrals(dg64, q64)
    out = {"every_100_steps": rows,
           "conservation_drift_fp32bulk": [abs(a - b) / max(abs(b), abs(I0[0])) for a, b in zip(I32, I0)],
           "conservation_drift_fp64": [abs(a - b) / max(abs(b), abs(I0[0])) for a, b in zip(I64, I0)]}
    if exact is not None:
        qe = rb.GridArray.from_numpy(exact(done * dt))
        errs = {}
        for name, q in (("fp32bulk", q32), ("fp64", q64)):
            d = qe.copy()
            d.data.sub_(q.data)
            errs[name] = (rb.weightednorm(dg64, d), rel_max_norm(rb, dg64, d, qe))
            del d
        out.update({"steps": done,
                    "l2_error_vs_exact_fp32bulk": errs["fp32bulk"][0], "l2_error_vs_exact_fp64": errs["fp64"][0],
                    "l2_error_ratio_fp32bulk_over_fp64": errs["fp32bulk"][0] / errs["fp64"][0],
                    "max_error_vs_exact_relative_fp32bulk": errs["fp32bulk"][1],
                    "max_error_vs_exact_relative_fp64": errs["fp64"][1]})
        del qe
    del q32, q64, dq32, dq64, dg64
    return out


def timed_steps(dg, q, dq, t0, dt, steps, stream, barrier, dist):
    """Device time (ms) of `steps` LSRK(5,4) steps on `stream`, CUDA events bracketed by a
    barrier and a synchronize on both sides, max over ranks."""
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    dg.lsrk54_steps(q, dq, t0, dt, steps)
    e1.record(stream)
    e1.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def fp32_bulk_leg(rb, w, grid, law, q0, dt, args, ms64, local, stream, barrier, dist, world):
    """The FP32-bulk form of the same workload in the same process: the same grid,
    initial state, steps and timing as the FP64 line, then (untimed) its accuracy
    against the FP64 form and the exact solution after `--accuracy-steps` steps."""
    from raven_b200 import initial_conditions as ic

    w32 = dict(w, precision="fp32_bulk")
    dg32 = rb.DGSEM(law=law, grid=grid, volume_form=rb.FluxDifferencingForm(rb.KennedyGruberFlux()),
                    surface_numericalflux=rb.RusanovFlux(), precision="fp32_bulk", device=local)
    q = rb.GridArray.from_numpy(q0)
    dq = q.similar()
    dg32.lsrk54_steps(q, dq, 0.0, dt, args.warmup)
    ms = timed_steps(dg32, q, dq, args.warmup * dt, dt, args.steps, stream, barrier, dist)
    del q, dq
    nodes, ns = grid.np * grid.E, law.ns
    peak, peak_kind = measured_peaks()
    bytes_launch = stage_bytes_per_launch(w32, nodes, ns)
    achieved = bytes_launch / (ms / 1e3 / (5 * args.steps)) / 1e9
    out = {
        "workload": args.workload.replace("fp64", "fp32bulk"),
        "precision": "fp32_bulk: FP32 volume/surface arithmetic, FP64 geometry, state and reductions, FP32 register",
        "ms_per_step": ms / args.steps,
        "value": world * nodes * ns * 5 * args.steps / (ms / 1e3),
        "unit": UNIT,
        "speedup_vs_fp64": ms64 / ms,
        "gpu_launches": 5 * args.steps,
        "kernel": kernel_name(w32, dg32),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": bytes_launch,
                     "traffic": profiled_traffic(args.workload.replace("fp64", "fp32bulk"))},
    }
    if args.accuracy_steps > 0:
        u0 = 0.5 * math.sqrt(law.gamma)
        exact = lambda t: ic.isentropic_vortex(grid, law, beta=5.0, u0=u0, center=(w["L"] / 2, w["L"] / 2), t=t)
        out["accuracy"] = fp64_comparison(rb, w32, grid, law, dg32, q0, dt, args.accuracy_steps, local, exact=exact)
    del dg32
    return out


# The other configurations, timed in the default run after its own legs so that one record
# holds them all: (label, workload, steps; None = the run's --steps).
OTHER_CONFIGS = [
    ("config 1: 2-D advection 16^2, N=4, 100 steps", "adv2d_weak_n4_16_fp64", 100),
    ("config 3: warped 32^3 Euler KG, FP32 bulk", "euler3d_kg_n7_32_fp32bulk_warped", None),
    ("config 3's FP64 comparison run: the same warped grid in FP64", "euler3d_kg_n7_32_fp64_warped", None),
    ("config 5: adapted 3-D Euler KG, N=5, FP32 bulk", "euler3d_kg_n5_adapted_fp32bulk", 100),
]


def other_configs_leg(rb, args, local, stream, barrier, dist, world):
    """Each of OTHER_CONFIGS timed like the main line (warm-up, CUDA events over the
    steps), with its roofline where its state is larger than L2."""
    out = []
    problems = {}
    for label, name, steps in OTHER_CONFIGS:
        w = dict(WORKLOADS[name])
        key = (w["dim"], w["N"], w["K"], w["law"], w["warp"], bool(w.get("adapted")))
        if key not in problems:
            problems = {key: problem(rb, w)}  # keep one grid alive at a time
        grid, law, form, q0, dt = problems[key]
        dg = rb.DGSEM(law=law, grid=grid, volume_form=form, surface_numericalflux=rb.RusanovFlux(),
                      precision=w["precision"], device=local)
        n = steps or args.steps
        q = rb.GridArray.from_numpy(q0)
        dq = q.similar()
        dg.lsrk54_steps(q, dq, 0.0, dt, args.warmup)
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.2)
        ms = timed_steps(dg, q, dq, args.warmup * dt, dt, n, stream, barrier, dist)
        sampler.stop()
        nodes, ns = grid.np * grid.E, law.ns
        launches = timed_launches(dg, n)
        rec = {
            "label": label,
            "config": config_json(name, w, grid),
            "steps": n,
            "warmup": args.warmup,
            "ms_per_step": ms / n,
            "value": world * nodes * ns * 5 * n / (ms / 1e3),
            "unit": UNIT,
            "gpu_launches": launches,
            "kernel": kernel_name(w, dg),
            "clocks": sampler.summary(),
        }
        if w["K"] >= 32:
            peak, peak_kind = measured_peaks()
            bytes_launch = stage_bytes_per_launch(w, nodes, ns)
            achieved = bytes_launch / (ms / 1e3 / (5 * n)) / 1e9
            rec["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": achieved / peak, "peak_source": peak_kind,
                               "algorithmic_bytes_per_launch": bytes_launch, "traffic": profiled_traffic(name)}
        else:
            rec["roofline"] = None
            rec["note"] = "state is L2-resident (a few MB): no HBM roofline"
        out.append(rec)
        del q, dq, dg
    return out


def adapted_oracle(w):
    """The adapted workload's grid and initial state for the oracle: the forest and its
    arrays are generated on the host (setup, untimed), the oracle couples the hanging
    faces with its own mortar restatement."""
    import numpy as np

    import oracle as O

    rb = load_product()
    from raven_b200 import initial_conditions as ic
    from raven_b200.forest import sphere_refinement_flags

    dim, N, K, L = w["dim"], w["N"], w["K"], w["L"]
    coords = tuple(rb.jl_range(0.0, L, K + 1) for _ in range(dim))
    gm = rb.GridManager(rb.LobattoCell(*([N + 1] * dim)), rb.brick(coords, (True,) * dim))
    for _ in range(2):
        rb.adapt(gm, sphere_refinement_flags(gm.forest, coords, (L / 2,) * dim, L / 4))
    grid = rb.generate(gm)
    og = O.Grid.from_arrays(dim, N + 1, grid.points, grid.volume_metrics, grid.surface_metrics, grid.vmapM,
                            grid.vmapP, grid.boundarycodes, grid.mortars, grid.tohalves)
    law = O.Law(O.LAW_EULER, dim, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_KG)
    q = ic.density_pulse(grid, rb.EulerLaw(dim), center=(L / 2,) * dim, amplitude=0.2, width2=0.01)
    return og, law, np.asfortranarray(q), f"the adapted grid itself ({grid.E} elements, {grid.mortars.shape[1]} mortars)"


def oracle_workload(w):
    """The workload's own grid, law and initial state on the oracle (C++ FP64
    restatement of Raven's CPU path): the same elements, order and data the GPU steps."""
    import oracle as O

    O.build()
    dim, N, K, L = w["dim"], w["N"], w["K"], w["L"]
    if w.get("adapted"):
        return adapted_oracle(w)
    warp = O.WARP_SINE if w["warp"] else O.WARP_NONE
    og = O.Grid(dim, N + 1, [K] * dim, [0.0] * dim, [L] * dim, [True] * dim, warp, 0.1)
    where = f"the workload's own {K}^{dim}-element periodic {'warped ' if w['warp'] else ''}brick"
    if w["law"] == "euler":
        law = O.Law(O.LAW_EULER, dim, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_KG)
        q = og.initial_condition(law, 4, [5.0, 0.5 * math.sqrt(1.4), L / 2, L / 2])
    else:
        law = O.Law(O.LAW_ADVECTION, dim, adv=list(ADV_VELOCITY[:dim]))
        q = og.initial_condition(law, 3, [0.05, 0.5, 0.5, 0.5])
    return og, law, q, where


def time_oracle_steps(og, law, q, warmup, steps, budget_s):
    """Untimed warm-up steps, then up to `steps` timed LSRK(5,4) steps of the oracle on
    its grid, stopping early once `budget_s` seconds of timed work have been spent (at
    least one step).  Returns (timed steps, seconds)."""
    dq = og.state(law)
    dt = 1e-4
    for i in range(warmup):
        og.lsrk54_step(law, q, dq, i * dt, dt)
    n, t0 = 0, time.perf_counter()
    while n < steps:
        og.lsrk54_step(law, q, dq, (warmup + n) * dt, dt)
        n += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    return n, time.perf_counter() - t0


def cpu_sample(w, max_seconds=20.0):
    """The oracle (C++ FP64 restatement) on the host cores: LSRK(5,4) steps on the
    workload's own grid and initial state (one untimed warm-up step, then timed steps
    until ~max_seconds have passed)."""
    import oracle as O

    og, law, q, where = oracle_workload(w)
    steps, el = time_oracle_steps(og, law, q, 1, 1000, max_seconds)
    nodes = og.np * og.E
    return {
        "value": nodes * law.ns * 5 * steps / el,
        "unit": UNIT,
        "cores": O.num_threads(),
        "kind": "port",
        "sample": f"{steps} LSRK(5,4) steps (after 1 untimed) of the same scheme (dim {w['dim']}, N {w['N']}, "
                  f"{w['vflux']}) on {where} ({og.E} elements), FP64, OpenMP over elements, {el:.1f} s",
    }


# timed seconds the reference arm spends at most (its warm-up is one step)
REFERENCE_BUDGET_S = 150.0


def run_reference(args, w):
    """Reference arm: Raven's CPU path restated (the oracle port; Raven is a Julia package
    and no Julia exists on these machines) on the workload's own grid and initial state,
    all host threads.  Timed LSRK(5,4) steps stop early once REFERENCE_BUDGET_S seconds
    have been spent; `timed_steps` says how many ran."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle as O

    og, law, q, where = oracle_workload(w)
    n, el = time_oracle_steps(og, law, q, min(args.warmup, 1), args.steps, REFERENCE_BUDGET_S)
    nodes = og.np * og.E
    value = nodes * law.ns * 5 * n / el
    cfg = config_json(args.workload, w)
    cfg["elements"], cfg["nodes"] = og.E, nodes
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "timed_steps": n,
        "warmup": args.warmup,
        "ms_per_step": el / n * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": O.num_threads(),
            "kind": "port",
            "sample": f"{n} of {args.steps} LSRK(5,4) steps (after {min(args.warmup, 1)} untimed; the timed steps "
                      f"stop after {REFERENCE_BUDGET_S:.0f} s) of the same scheme on {where} ({og.E} elements, "
                      f"N {w['N']}), FP64 C++ restatement of Raven's CPU path, OpenMP over elements",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def serve_bytes_per_dof(precision):
    """Algorithmic HBM bytes per DOF update (per RHS) of the batched stage kernel,
    averaged over the 5 stages: q read + write (16 B), dq write (every stage) and dq
    read (stages 2-5); the per-element geometry is negligible (32 B per element)."""
    dqb = 4 if precision == "fp32_bulk" else 8
    return 16 + dqb + 4 * dqb / 5


def serve_cpu_sample(arrivals, max_seconds=20.0):
    """The oracle on the host cores over a bounded sample of the stream: the solves of
    the stream in order, each run for at most 5 steps, until ~max_seconds have passed."""
    import numpy as np

    import oracle as O

    done_dof, t0, solves = 0, time.perf_counter(), 0
    for a in arrivals:
        s = a.spec
        og = O.Grid(s.dim, s.nq, list(s.K), list(s.lo), list(s.hi), [1] * s.dim)
        if s.law == 1:
            law = O.Law(O.LAW_EULER, s.dim, form=O.FORM_FLUXDIFF, volume_flux=O.FLUX_KG)
            q = og.initial_condition(law, 4, [s.init_params[0], s.init_params[1], 5.0, 5.0])
        else:
            law = O.Law(O.LAW_ADVECTION, s.dim, adv=list(s.advection_velocity[: s.dim]))
            q = og.initial_condition(law, 3, list(s.init_params[:4]))
        dq = og.state(law)
        n = min(5, s.nsteps)
        for i in range(n):
            og.lsrk54_step(law, q, dq, i * s.dt, s.dt)
        done_dof += og.np * og.E * law.ns * 5 * n
        solves += 1
        if time.perf_counter() - t0 >= max_seconds:
            break
    el = time.perf_counter() - t0
    return {
        "value": done_dof / el,
        "unit": UNIT,
        "cores": O.num_threads(),
        "kind": "port",
        "sample": f"the first {solves} solves of the same seeded stream, 5 LSRK(5,4) steps each, FP64 C++ "
                  f"restatement of Raven's CPU path, OpenMP over elements, {el:.1f} s including grid set-up",
    }


def serving_warm_specs(rb, S):
    """One short solve per class of the stream: creates the class, captures its graphs
    and lets the autotuner pick its tile."""
    warm = []
    for dim in (2, 3):
        for nq in (4, 6, 8):
            for law in (0, 1):
                f = S.vortex_spec if law == 1 else S.wave_spec
                warm.append(f(dim, nq, (4,) * dim if dim == 3 else (8, 8), 10,
                              precision=rb._lib.PRECISION_FP32_BULK))
    return warm


def serving_leg(rb, local, requests, rates, seed):
    """A short seeded stream of the serving workload (config 4's generator) replayed at
    each arrival rate in `rates` against one warm server: p50/p99 latency (submit to
    final state on the host), solves/s and DOF updates/s per rate."""
    import numpy as np

    from raven_b200 import serving as S

    srv = S.Server(arena_bytes=48 << 30, device=local)
    try:
        for t in [srv.submit(sp, keep_result=False) for sp in serving_warm_specs(rb, S)]:
            srv.wait(t)
        out = []
        for rate in rates:
            arrivals = S.poisson_mix(seed, requests, rate=rate)
            t0 = time.perf_counter()
            res = S.run_load(srv, arrivals, keep_results=True)
            wall = time.perf_counter() - t0
            lat = res["latencies"]
            dof = float(sum(a.spec.dof_updates() for a in arrivals))
            out.append({
                "arrival_rate_per_s": rate,
                "requests": requests,
                "seed": seed,
                "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3),
                "max_ms": float(lat.max() * 1e3),
                "solves_per_s": requests / wall,
                "dof_updates_per_s": dof / wall,
                "offered_dof_updates_per_s": dof / max(arrivals[-1].t, 1e-9),
                "seconds": wall,
            })
        return out
    finally:
        srv.close()


def run_serving(args):
    """The serving loop under the seeded Poisson stream (one server per GPU; replicas)."""
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        return run_serving_reference(args)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    rb = load_product()
    from raven_b200 import serving as S

    arrivals = S.poisson_mix(args.seed, args.requests, rate=args.rate)
    srv = S.Server(arena_bytes=48 << 30, device=local)
    warm = serving_warm_specs(rb, S)
    for _ in range(max(1, args.warmup)):
        for t in [srv.submit(sp, keep_result=False) for sp in warm]:
            srv.wait(t)
    srv.close()
    # the timed stream on a fresh server whose classes are warm in the process (module
    # loading, kernel attributes); class graphs are captured again at first use
    srv = S.Server(arena_bytes=48 << 30, device=local)
    for t in [srv.submit(sp, keep_result=False) for sp in warm]:
        srv.wait(t)
    base = srv.stats()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    sampler.start()
    time.sleep(0.3)
    t0 = time.perf_counter()
    res = S.run_load(srv, arrivals, keep_results=True)
    wall = time.perf_counter() - t0
    sampler.stop()
    st = srv.stats()
    tiles = srv.class_tiles()
    class_stats = srv.class_stats()
    srv.close()
    lat = res["latencies"]
    dof = float(sum(a.spec.dof_updates() for a in arrivals))
    first_t = arrivals[0].t
    # busy time of the stream: first arrival to last completion (the server's clock)
    busy = wall
    if dist is not None:
        t = torch.tensor([busy], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        busy = float(t.item())
    value = world * dof / busy
    ticks = st["ticks"] - base["ticks"]
    peak, peak_kind = measured_peaks()
    bpd = serve_bytes_per_dof("fp32_bulk")
    achieved = dof * bpd / busy / 1e9
    h2d = sum(a.spec.num_elements * (32 + 8 * a.spec.dim + 16 * a.spec.dim) for a in arrivals)
    d2h = sum(a.spec.np * a.spec.ns * a.spec.num_elements * 8 for a in arrivals)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = serve_cpu_sample(arrivals)
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.requests,
            "warmup": args.warmup,
            "ms_per_step": busy / args.requests * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64",
            "data": "synthetic",
            "config": {
                "workload": SERVE_WORKLOAD,
                "requests": args.requests,
                "arrival_rate_per_s": args.rate,
                "seed": args.seed,
                "dims": [2, 3],
                "equations": ["advection (weak form)", "euler (kennedy-gruber flux differencing)"],
                "polynomial_orders": [3, 5, 7],
                "elements_per_side": {"2d": [8, 64], "3d": [4, 32], "distribution": "log-uniform"},
                "lsrk_steps": [50, 500],
                "precision": "fp32_bulk",
                "initial_data": "sine_plus_gaussian (advection), isentropic vortex strength 3 (euler)",
                "step_meaning": "one request of the stream; value = DOF updates of all requests / busy time",
                "l2_flush": "not needed: the running solves' state (GBs) is larger than L2",
                "parallelism": "replicas",
            },
            "serving": {
                "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3),
                "max_ms": float(lat.max() * 1e3),
                "solves_per_s": world * args.requests / busy,
                "busy_seconds": busy,
                "stream_seconds": arrivals[-1].t - first_t,
                "total_dof_updates": dof,
                "arena_peak_bytes": st["arena_peak"],
                "class_tiles": [list(t) for t in tiles],
                # per class: device time of its ticks (classes overlap) and DOF updates/s there
                "classes": [dict(r, dof_per_s=r["dof_updates"] / (r["device_ms"] / 1e3) if r["device_ms"] else None)
                            for r in class_stats],
            },
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": None,
                "peak_source": peak_kind,
                "kernel": "batched_stage_kernel (all running solves of a class per launch)",
                "algorithmic_bytes_per_dof_update": bpd,
            },
            "cpu_baseline": cpu,
            "e2e": {
                "value": value,
                "unit": UNIT,
                "h2d_bytes_per_step": h2d / args.requests,
                "d2h_bytes_per_step": d2h / args.requests,
                "note": "the value is already end to end: host requests in, final states copied to host",
            },
            "gpu_launches": int(6 * ticks + args.requests),
            "clocks": sampler.summary(),
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_serving_reference(args):
    """Reference arm of the serving workload: the oracle port runs the stream's solves
    one after another on the host cores (the reference has no serving loop), each
    truncated to its first 5 steps; value = DOF updates per second."""
    import oracle as O

    O.build()
    rb = load_product()
    from raven_b200 import serving as S

    arrivals = S.poisson_mix(args.seed, args.requests, rate=args.rate)
    cpu = serve_cpu_sample(arrivals, max_seconds=60.0)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": cpu["value"],
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.requests,
        "warmup": args.warmup,
        "ms_per_step": None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": SERVE_WORKLOAD, "requests": args.requests, "arrival_rate_per_s": args.rate,
                   "seed": args.seed},
        "cpu_baseline": cpu,
        "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_sharded(args, w):
    """The workload's grid partitioned over the ranks (raven_b200.distributed): each rank
    steps its own elements stage by stage and exchanges face traces with its neighbour
    ranks over NCCL before every stage.  value = global DOF updates / max-over-ranks time
    (strong scaling: the grid is fixed as the ranks grow)."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist

    if w.get("adapted"):
        raise SystemExit("--sharded: the adapted workload has mortars, which the partitioned path does not take")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1 and "MASTER_PORT" not in os.environ:
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    try:
        rb = load_product()
        from raven_b200 import distributed as D

        grid, law, form, q0, dt = problem(rb, w)
        ddg = D.DistributedDGSEM(law=law, grid=grid, volume_form=form, surface_numericalflux=rb.RusanovFlux(),
                                 precision=w["precision"], device=local)
        q = ddg.state(q0)
        dq = q.similar()
        stream = torch.cuda.current_stream()

        def barrier():
            torch.cuda.synchronize()
            dist.barrier()
            torch.cuda.synchronize()

        ddg.lsrk54_steps(q, dq, 0.0, dt, args.warmup)
        barrier()
        sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
        sampler.start()
        time.sleep(0.3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(stream)
        ddg.lsrk54_steps(q, dq, args.warmup * dt, dt, args.steps)
        e1.record(stream)
        e1.synchronize()
        barrier()
        sampler.stop()
        t = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        nodes, ns = grid.np * grid.E, law.ns
        value = nodes * ns * 5 * args.steps / (ms / 1e3)
        norm = ddg.weightednorm(q)
        pat = ddg.pattern
        exch = torch.tensor([len(pat.recvindices) * 8.0, ddg.local.num_ghosts, ddg.local.num_local],
                            device="cuda", dtype=torch.float64)
        dist.all_reduce(exch)
        if rank == 0:
            packs = 2 if len(pat.recvindices) or len(pat.sendindices) else 0
            line = {
                "metric": METRIC,
                "value": value,
                "unit": UNIT,
                "n_gpus": world,
                "steps": args.steps,
                "warmup": args.warmup,
                "ms_per_step": ms / args.steps,
                "higher_is_better": True,
                "scaling": "strong",
                "vs_baseline": None,
                "dtype": "f32+f64" if w["precision"] == "fp32_bulk" else "f64",
                "data": "synthetic",
                "config": dict(config_json(args.workload, w, grid),
                               parallelism=f"element partition over {world} ranks, face traces exchanged "
                                           "over NCCL before every stage"),
                "exchange": {"bytes_received_per_stage_all_ranks": exch[0].item(),
                             "ghost_elements_all_ranks": int(exch[1].item()), "elements": grid.E},
                "weightednorm": norm,
                # rank 0's launches: 5 stage kernels a step, plus a pack and an unpack
                # kernel a stage when the rank has neighbour ranks
                "gpu_launches": 5 * args.steps * (1 + packs),
                "clocks": sampler.summary(),
            }
            print(json.dumps(line), flush=True)
    finally:
        dist.destroy_process_group()
    return 0


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS) + [SERVE_WORKLOAD])
    p.add_argument("--requests", type=int, default=200, help="serving workload: solves in the timed stream")
    p.add_argument("--rate", type=float, default=200.0, help="serving workload: arrivals per second")
    p.add_argument("--seed", type=int, default=0, help="serving workload: stream seed")
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--elements-per-side", type=int, default=None,
                   help="override the workload's elements per side (smaller cases for profiling)")
    p.add_argument("--sharded", action="store_true",
                   help="partition the workload's elements over the ranks (face-trace exchange between "
                        "stages, strong scaling); the default when more than one rank runs")
    p.add_argument("--replicas", action="store_true",
                   help="with more than one rank: one independent replica of the workload per rank instead "
                        "of the element partition")
    p.add_argument("--accuracy-steps", type=int, default=1000,
                   help="steps of the untimed FP32-bulk vs FP64 accuracy comparison (0: skip)")
    p.add_argument("--no-fp32-leg", action="store_true", help="skip the FP32-bulk sub-measurement")
    p.add_argument("--serving-requests", type=int, default=40,
                   help="requests of the short serving stream of the default line (0: skip)")
    p.add_argument("--no-other-configs", action="store_true",
                   help="skip timing the other configurations (1, 3, 5) in the default run")
    args = p.parse_args(argv)
    if args.workload == SERVE_WORKLOAD:
        return run_serving(args)
    w = dict(WORKLOADS[args.workload])
    if args.elements_per_side:
        w["K"] = int(args.elements_per_side)
    if args.impl == "reference":
        return run_reference(args, w)
    multi = int(os.environ.get("WORLD_SIZE", "1")) > 1 or args.gpus > 1
    if args.sharded or (multi and not args.replicas and not w.get("adapted")):
        return run_sharded(args, w)

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    rb = load_product()
    grid, law, dg, q0, dt = setup(rb, w, local)
    nodes, ns = grid.np * grid.E, law.ns
    q = rb.GridArray.from_numpy(q0)
    dq = q.similar()
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    dg.lsrk54_steps(q, dq, 0.0, dt, args.warmup)
    barrier()
    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    sampler.start()
    time.sleep(0.3)
    ms = timed_steps(dg, q, dq, args.warmup * dt, dt, args.steps, stream, barrier, dist)
    sampler.stop()
    value = world * nodes * ns * 5 * args.steps / (ms / 1e3)
    launches = timed_launches(dg, args.steps)

    # the FP32-bulk form of the same workload, timed the same way in the same process
    fp32_leg = None
    if (w["law"] == "euler" and w["precision"] == "fp64" and not w["warp"] and not w.get("adapted")
            and not args.no_fp32_leg):
        sampler32 = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
        sampler32.start()
        time.sleep(0.3)
        fp32_leg = fp32_bulk_leg(rb, w, grid, law, q0, dt, args, ms, local, stream, barrier, dist, world)
        sampler32.stop()
        fp32_leg["clocks"] = sampler32.summary()

    # accuracy of the run: L2 distance to the exactly advected vortex, and conservation
    l2_err = None
    fp64_cmp = None
    accuracy = None
    if w.get("adapted"):
        # the FP32-bulk state against an FP64 run of the same steps (the FP64 path is
        # parity-tested against the oracle), and the drift of the conserved integrals
        dg64 = rb.DGSEM(law=law, grid=grid, volume_form=rb.FluxDifferencingForm(rb.KennedyGruberFlux()),
                        surface_numericalflux=rb.RusanovFlux(), precision="fp64", device=local)
        q64 = rb.GridArray.from_numpy(q0)
        dq64 = q64.similar()
        dg64.lsrk54_steps(q64, dq64, 0.0, dt, args.warmup + args.steps)
        I0 = rb.integrals(dg64, rb.GridArray.from_numpy(q0))
        I32, I64 = rb.integrals(dg, q), rb.integrals(dg64, q64)
        diff = q64.copy()
        diff.data.sub_(q.data)
        fp64_cmp = {
            "l2_diff_vs_fp64_relative": rb.weightednorm(dg64, diff) / rb.weightednorm(dg64, q64),
            "max_diff_vs_fp64_relative": rel_max_norm(rb, dg64, diff, q64),
            # |integral(t) - integral(0)| over max(|integral(0)|, mass): the momenta start at 0
            "conservation_drift_fp32bulk": [abs(a - b) / max(abs(b), abs(I0[0])) for a, b in zip(I32, I0)],
            "conservation_drift_fp64": [abs(a - b) / max(abs(b), abs(I0[0])) for a, b in zip(I64, I0)],
            "elements": grid.E,
            "mortars": int(grid.mortars.shape[1]),
            "levels": [int(c) for c in np.bincount([L_[1] for L_ in grid.forest.leaves])],
        }
        del diff, q64, dq64, dg64
    elif w["law"] == "euler":
        from raven_b200 import initial_conditions as ic

        if w["precision"] == "fp32_bulk":
            fp64_cmp = fp64_comparison(rb, w, grid, law, dg, q0, dt, args.steps, local)

        T = (args.warmup + args.steps) * dt
        qe = rb.GridArray.from_numpy(ic.isentropic_vortex(grid, law, beta=5.0, u0=0.5 * math.sqrt(law.gamma),
                                                          center=(w["L"] / 2, w["L"] / 2), t=T))
        qmax = rb.weightednorm(dg, qe, math.inf)
        qe.data.sub_(q.data)
        l2_err = rb.weightednorm(dg, qe)
        I0, I1 = rb.integrals(dg, rb.GridArray.from_numpy(q0)), rb.integrals(dg, q)
        accuracy = {
            "l2_error_vs_exact": l2_err,
            "max_error_vs_exact_relative": rb.weightednorm(dg, qe, math.inf) / qmax,
            # |integral(t) - integral(0)| over max(|integral(0)|, mass): the vortex's z momentum is 0
            "conservation_drift": [abs(a - b) / max(abs(b), abs(I0[0])) for a, b in zip(I1, I0)],
            "steps": args.warmup + args.steps,
        }
        del qe

    # end to end through the C ABI with host buffers: every step copies the state in from
    # pinned host memory, runs one LSRK(5,4) step and copies the state back
    e2e = None
    if args.e2e_steps > 0:
        qh_t = torch.empty((grid.E, ns, grid.np), dtype=torch.float64, pin_memory=True)
        qh = qh_t.numpy().transpose(2, 1, 0)
        qh[...] = q0
        dg.lsrk54_steps_host(qh, 0.0, dt, 1)  # warm-up
        barrier()
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            dg.lsrk54_steps_host(qh, i * dt, dt, 1)
        e2e_s = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {
            "value": world * nodes * ns * 5 * args.e2e_steps / e2e_s,
            "unit": UNIT,
            "h2d_bytes_per_step": nodes * ns * 8,
            "d2h_bytes_per_step": nodes * ns * 8,
            "ms_per_step": e2e_s / args.e2e_steps * 1e3,
            "note": "rb200_lsrk54_step_host, one synchronous call per step: the whole state is copied in "
                    "from pinned host memory and back every step, so PCIe copies dominate",
        }
        # the same entry point used as solve! is: one call for all the steps, the state copied
        # in once and back once (informational; the per-step form above is the e2e figure)
        qh[...] = q0
        barrier()
        t0 = time.perf_counter()
        dg.lsrk54_steps_host(qh, 0.0, dt, args.steps)
        solve_s = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([solve_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            solve_s = float(t.item())
        e2e["one_call_solve"] = {
            "value": world * nodes * ns * 5 * args.steps / solve_s,
            "unit": UNIT,
            "steps": args.steps,
            "h2d_bytes_per_call": nodes * ns * 8,
            "d2h_bytes_per_call": nodes * ns * 8,
            "ms_per_call": solve_s * 1e3,
            "note": "rb200_lsrk54_step_host(q, nsteps = steps): one synchronous call, the state copied in "
                    "and back once, as a solve! over host arrays would use it",
        }

    peak, peak_kind = measured_peaks()
    bytes_launch = stage_bytes_per_launch(w, nodes, ns)
    achieved = bytes_launch / (ms / 1e3 / (5 * args.steps)) / 1e9  # per stage-kernel launch
    traffic = profiled_traffic(args.workload)
    roofline = {
        "bound": "hbm",
        "achieved": achieved,
        "peak": peak,
        "unit": "GB/s",
        "frac": achieved / peak,
        "traffic": traffic,
        "peak_source": peak_kind,
        "kernel": kernel_name(w, dg),
        "algorithmic_bytes_per_launch": bytes_launch,
    }
    fp64_pipe = None
    flops_node = profiled_figure(args.workload, "fp64_flops_per_node")
    if flops_node and w["precision"] == "fp64":
        # the second roofline of the FP64 path: FP64 flops the kernel executes (ncu counters
        # of the committed summary, DFMA = 2) per launch over the launch time
        tf = flops_node * nodes / (ms / 1e3 / (5 * args.steps)) / 1e12
        peak64 = measured_fp64_tflops(rb)
        src = "measured (rb200_probe_fp64_rate, after the timed region)"
        if peak64 is None:
            peak64, src = FP64_NOMINAL_TFLOPS, "nominal (datasheet)"
        fp64_pipe = {"achieved": tf, "peak": peak64, "unit": "TFLOP/s", "frac": tf / peak64,
                     "peak_source": src, "flops_per_node_stage": flops_node}
    # a short serving stream (config 4's generator) on the same GPU, after the timed work
    serving = None
    if args.serving_requests > 0 and args.workload == DEFAULT and w["K"] == WORKLOADS[DEFAULT]["K"]:
        del q, dq
        serving = {"note": "config 4's seeded stream (FP32 bulk), shortened; latency = submit to final "
                           "state on the host; at 200/s the stream offers more work than the GPU drains, "
                           "so latency there includes queueing; the lower rate is below the drain rate",
                   "streams": serving_leg(rb, local, args.serving_requests, (200.0, 10.0), args.seed)}

    others = None
    if (world == 1 and not args.no_other_configs and args.workload == DEFAULT
            and w["K"] == WORKLOADS[DEFAULT]["K"]):
        if serving is None:
            del q, dq
        del dg
        others = other_configs_leg(rb, args, local, stream, barrier, dist, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(w)
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64" if w["precision"] == "fp32_bulk" else "f64",
            "data": "synthetic",
            "config": config_json(args.workload, w, grid),
            "roofline": roofline,
            "fp64_roofline": fp64_pipe,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": sampler.summary(),
            "l2_error_vs_exact": l2_err,
            "accuracy": accuracy,
            "vs_fp64": fp64_cmp,
            "fp32_bulk": fp32_leg,
            "serving": serving,
            "other_configs": others,
            "dt": dt,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
