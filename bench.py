#!/usr/bin/env python3
"""Benchmark of the spectral-element hot path: SSP-Knoth Rosenbrock-W steps/s.

Workload (default): the FP64 drop-in configuration - cubed sphere nPanel 30
(5,400 elements), OrdPoly 4, nz 45 levels stretched quadratically to 30 km,
2 passive tracers, dt 120 s, dry baroclinic wave + seeded theta noise;
synthetic initial state, no I/O.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

One step = one full Rosenbrock-W step (3 stages of tendency + DSS + column
Schur solve) of the whole grid.  With N > 1 (torchrun, one process per GPU)
every rank advances its own ensemble member (seed + rank): the work per GPU is
fixed ("weak"), no collective on the data path; timing is the max over ranks.

Rank 0 prints one JSON line.  ``value`` is device-resident throughput
(inputs in HBM); ``e2e`` drives the same C ABI call with a pinned host state,
so every step includes the state's host->device and device->host copies.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cgdycore.jl_b200"))

METRIC = "Rosenbrock-W steps/s @nPanel30 p4 nz45: FP64 vs mixed FP32; adjoint/fwd time"
UNIT = "steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="dropin")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision sub-measurement")
    ap.add_argument("--mixed-days", type=float, default=1.0, help="simulated days of the mixed accuracy run")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint sub-measurement")
    ap.add_argument("--no-mixed-cfg3", action="store_true",
                    help="skip the mixed form at its own configuration (nPanel 60, nz 64, 1 simulated day)")
    ap.add_argument("--cfg3-days", type=float, default=1.0, help="simulated days of the nPanel-60 accuracy run")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble sub-measurement")
    ap.add_argument("--ensemble-steps", type=int, default=10, help="timed ensemble steps per precision")
    ap.add_argument("--adjoint-steps", "--adjoint-window", dest="adjoint_steps", type=int, default=120,
                    help="steps of the adjoint sensitivity study (120 x 120 s = 4 h)")
    ap.add_argument("--adjoint-fd", action="store_true",
                    help="add central-difference checks of the sensitivity gradient (about a minute)")
    ap.add_argument("--no-output", action="store_true", help="skip the output-interpolation sub-measurement")
    ap.add_argument("--parallel", default="member", choices=["member", "shard"],
                    help="N > 1: one ensemble member per GPU (weak scaling) or one grid decomposed over the "
                         "GPUs with halo exchanges of the DSS (strong scaling)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class Ranks:
    """Rank plumbing: one process per GPU, no collective on the data path.
    A barrier brackets the timed region and the reported time is the max over
    ranks.  `device` is the CUDA device for NCCL, None for a CPU (gloo) group."""

    def __init__(self, rank, world, device=None):
        self.rank, self.world, self.device = rank, world, device

    def barrier(self):
        import torch
        if self.world > 1:
            torch.distributed.barrier()
        if self.device is not None:
            torch.cuda.synchronize()

    def max(self, x):
        import torch
        if self.world > 1:
            t = torch.tensor([float(x)], dtype=torch.float64,
                             device=self.device if self.device is not None else "cpu")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            return float(t.item())
        return float(x)


def member_config(cfg, rank):
    """Ensemble member of a rank: the configuration with its theta-noise seed
    offset by the rank."""
    import dataclasses
    return dataclasses.replace(cfg, seed_theta=cfg.seed_theta + rank)


def aggregate(world, steps, t):
    """Whole-job steps/s: every rank advanced its own member `steps` times
    within the max-over-ranks time t."""
    return world * steps / t


def workload_config(cfg, precision):
    return {"workload": f"{cfg.name}: cubed sphere nPanel {cfg.nPanel} ({6 * cfg.nPanel ** 2} elements), "
                        f"OrdPoly {cfg.OrdPoly}, nz {cfg.nz} {cfg.stretch}, NumTr {cfg.NumTr}, "
                        f"dt {cfg.dt:g} s, SSP-Knoth Rosenbrock-W, {precision.upper()}",
            "dt_note": "dt 300 s (and 150 s) is unstable for this W-method, whose horizontal acoustics "
                       "are explicit, on this grid (NaN by step 5 at 300 s, by step 40 at 150 s); "
                       "120 s is stable for 600+ steps; work per step does not depend on dt",
            "nPanel": cfg.nPanel, "OrdPoly": cfg.OrdPoly, "nz": cfg.nz, "NumTr": cfg.NumTr, "dt": cfg.dt,
            "parallelism": "ensemble member per GPU",
            "l2": "inputs larger than L2 (state 218 MB + element metric 826 MB per member)"}


def unique_dof(cfg):
    numg = 6 * cfg.nPanel ** 2 * cfg.OrdPoly ** 2 + 2
    return numg * cfg.nz * (5 + cfg.NumTr)


# ---------------------------------------------------------------------------
def oracle_steps_per_s(cfg, nsteps, warmup, threads):
    """The CPU restatement of the reference path (oracle/) on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from cgd_b200 import physics as Ph
    oracle.build()
    n = oracle.set_threads(threads)
    z = cfg.levels()
    o = oracle.Oracle(cfg.nPanel, cfg.OrdPoly, cfg.nz, cfg.NumTr, z, H=cfg.H,
                      nu=Ph.hyperdiffusion(cfg.nPanel, cfg.OrdPoly), Up=cfg.Up)
    U = o.init_state(Ph.tracer_centres(cfg.NumTr, cfg.seed_tracer) if cfg.NumTr else None)
    Ph.theta_noise(U, cfg.theta_noise, cfg.seed_theta)
    if warmup:
        U = o.ros_step(U, cfg.dt, warmup)
    t0 = time.perf_counter()
    U = o.ros_step(U, cfg.dt, nsteps)
    t = time.perf_counter() - t0
    assert np.all(np.isfinite(U))
    return nsteps / t, n


def oracle_rhs_threads(cfg, threads):
    """One tendency evaluation of the CPU restatement on all host threads and
    on one thread (the same state): seconds each."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from cgd_b200 import physics as Ph
    z = cfg.levels()
    o = oracle.Oracle(cfg.nPanel, cfg.OrdPoly, cfg.nz, cfg.NumTr, z, H=cfg.H,
                      nu=Ph.hyperdiffusion(cfg.nPanel, cfg.OrdPoly), Up=cfg.Up)
    U = o.init_state(Ph.tracer_centres(cfg.NumTr, cfg.seed_tracer) if cfg.NumTr else None)
    Ph.theta_noise(U, cfg.theta_noise, cfg.seed_theta)
    out = []
    for n in (threads, 1):
        oracle.set_threads(n)
        o.rhs(U)
        t0 = time.perf_counter()
        F = o.rhs(U)
        out.append(time.perf_counter() - t0)
        assert np.all(np.isfinite(F))
    oracle.set_threads(threads)
    return out


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.path = tempfile.mktemp(suffix=".csv")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(dev)], stdout=open(self.path, "w"),
                                      stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peak_hbm():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _units(cfg):
    """S (bytes of one FP64 field over all column-levels), E (one FP64 value
    per element-node-level), S' (one per column interface) and NV."""
    numg = 6 * cfg.nPanel ** 2 * cfg.OrdPoly ** 2 + 2
    S = numg * cfg.nz * 8
    E = 6 * cfg.nPanel ** 2 * (cfg.OrdPoly + 1) ** 2 * cfg.nz * 8
    return S, E, numg * (cfg.nz - 1) * 8, 5 + cfg.NumTr


def phase2_bytes(cfg):
    """Algorithmic bytes of one tendency (phase-2) launch: the phase-2 term of
    the per-stage RHS count with the stage state read once (it arrives
    combined; the combination is counted with the column kernel that forms
    it): stage state NV*S + DSS'd hyperviscosity cache (5+NumTr)*S + the
    lumped-mass sum S + 22 metric values per element-node-level (14 dXdxI,
    2 J, 6 X in the reference layout) + the tendency NV*S."""
    S, E, _, NV = _units(cfg)
    return NV * S + (5 + cfg.NumTr) * S + 22 * E + S + NV * S


def step_bytes(cfg):
    """Algorithmic bytes of one SSP-Knoth Rosenbrock-W step (3 stages, FP64,
    stage combinations counted fused, pressure in register):
      stage i: RHS phase 1 (4+NT)*i*S + 10E + S + (5+NT)*S
               RHS phase 2 NV*i*S + (5+NT)*S + 22E + S + NV*S
               Schur       NV*S + (i-1)*NV*S + 8S' + NV*S
      per step: Jacobian 3S + 8S', final update 5*NV*S.
    13.35 GB at nPanel 30, p 4, nz 45, 2 tracers."""
    S, E, Sp, NV = _units(cfg)
    NT = cfg.NumTr
    tot = 0
    for i in (1, 2, 3):
        tot += (4 + NT) * i * S + 10 * E + S + (5 + NT) * S
        tot += NV * i * S + (5 + NT) * S + 22 * E + S + NV * S
        tot += NV * S + (i - 1) * NV * S + 8 * Sp + NV * S
    return tot + 3 * S + 8 * Sp + 5 * NV * S


def ncu_traffic():
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of
    the phase-2 kernel from the committed ncu summary of the drop-in workload."""
    try:
        for line in open(os.path.join(ROOT, "profiles", "k_phase2_dropin_n30_p4_nz45.md")):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


# ---------------------------------------------------------------------------
def run_reference(args, cfg, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    K = max(1, min(args.steps, 5))
    W = 1 if args.warmup > 0 else 0
    v, n = oracle_steps_per_s(cfg, K, W, threads)
    sample = (f"{K} full-grid Rosenbrock-W steps after {W} warm-up step(s), C++ FP64 restatement of the "
              f"reference CPU path (Julia is not available), OpenMP on {n} threads, {cpu_model()}")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(cfg, "fp64"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": n, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_mixed(args, cfg, rank, ranks, U0, fp64_value, torch):
    """The mixed form on the same workload: device-resident steps/s (timed
    like the FP64 line) and, over args.mixed_days simulated days from the same
    initial state, the lowest-level pressure error against the FP64 path
    and the mass drift of both."""
    from cgd_b200 import setup
    dm, _, mcfg = setup(member_config(cfg, rank), precision="mixed")
    stream = torch.cuda.ExternalStream(dm.stream())
    Ut = torch.from_numpy(np.ascontiguousarray(U0.transpose(2, 1, 0))).cuda()
    dm.time_stepper(Ut, cfg.dt, args.warmup)
    ranks.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dm.time_stepper(Ut, cfg.dt, args.steps)
    e1.record(stream)
    e1.synchronize()
    t = ranks.max(e0.elapsed_time(e1) / 1e3)
    value = aggregate(ranks.world, args.steps, t)
    ktimes = dm.kernel_times()
    dm.close()
    # accuracy: the same initial state through both paths
    nsteps = max(1, int(round(args.mixed_days * 86400.0 / cfg.dt)))
    out = {}
    for prec in ("fp64", "mixed"):
        d, _, _ = setup(member_config(cfg, rank), precision=prec)
        V = torch.from_numpy(np.ascontiguousarray(U0.transpose(2, 1, 0))).cuda()
        m0 = d.mass_integral(V)
        d.time_stepper(V, cfg.dt, nsteps)
        torch.cuda.synchronize()
        out[prec] = (np.asarray(d.fcn_prepare(V))[0].copy(), (d.mass_integral(V) - m0) / m0)
        d.close()
    p64, pm = out["fp64"][0], out["mixed"][0]
    return {"value": value, "unit": UNIT, "ms_per_step": t / args.steps * 1e3, "speedup_vs_fp64": value / fp64_value,
            "kernel_ms_last_step": {k: round(v, 4) for k, v in ktimes[:6]},
            "accuracy": {"simulated_days": nsteps * cfg.dt / 86400.0, "steps": nsteps,
                         "p1_rel_l2": float(np.sqrt(np.sum((pm - p64) ** 2) / np.sum(p64 ** 2))),
                         "p1_rel_linf": float(np.abs(pm - p64).max() / np.abs(p64).max()),
                         "mass_drift_mixed": float(out["mixed"][1]), "mass_drift_fp64": float(out["fp64"][1]),
                         "p1": "pressure of the lowest layer (surface-pressure proxy), against the FP64 path"},
            "form": "FP32 horizontal derivative sums on perturbations from an FP64 per-level reference "
                    "profile; FP64 vertical terms, column Jacobian/Schur solve and reductions"}


def run_mixed_cfg3(args, rank, ranks, torch):
    """The mixed form at its own configuration (physics.CONFIGS['mixed']:
    nPanel 60, p 4, nz 64 quadratic, no tracers): device-resident steps/s of
    both precisions (timed like the headline) and, over args.cfg3_days
    simulated days from the same initial state, the lowest-layer pressure
    (surface-pressure proxy) of the mixed form against the FP64 path of the
    same configuration, and the mass drift of both."""
    from cgd_b200 import grid as G
    from cgd_b200 import setup
    from cgd_b200 import physics as Ph
    cfg = member_config(Ph.CONFIGS["mixed"], rank)
    nsteps = max(1, int(round(args.cfg3_days * 86400.0 / cfg.dt)))
    K = max(3, min(args.steps, 20))
    # the grid set-up at this size: host (numpy) against device (cgd_metric_sphere, cgd_mass_dz)
    t0 = time.perf_counter()
    G.init_grid_sphere(cfg.nPanel, cfg.OrdPoly, cfg.levels(), cfg.H, Ph.PhysParameters().RadEarth)
    t_host = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gd = G.init_grid_sphere_device(cfg.nPanel, cfg.OrdPoly, cfg.levels(), cfg.H, Ph.PhysParameters().RadEarth)
    torch.cuda.synchronize()
    t_dev = time.perf_counter() - t0
    del gd
    out = {}
    for prec in ("fp64", "mixed"):
        d, U0, _ = setup(cfg, precision=prec, check_finite=True, where="device")
        stream = torch.cuda.ExternalStream(d.stream())
        V = torch.from_numpy(np.ascontiguousarray(U0.transpose(2, 1, 0))).cuda()
        m0 = d.mass_integral(V)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        W = min(3, nsteps)
        d.time_stepper(V, cfg.dt, W)
        ranks.barrier()
        e0.record(stream)
        d.time_stepper(V, cfg.dt, min(K, nsteps - W))
        e1.record(stream)
        e1.synchronize()
        t = ranks.max(e0.elapsed_time(e1) / 1e3)
        d.time_stepper(V, cfg.dt, max(0, nsteps - W - K))
        torch.cuda.synchronize()
        out[prec] = {"steps_per_s": ranks.world * min(K, nsteps - W) / t, "p1": np.asarray(d.fcn_prepare(V))[0].copy(),
                     "drift": (d.mass_integral(V) - m0) / m0, "finite": bool(torch.isfinite(V).all().item())}
        d.close()
        del V
        torch.cuda.empty_cache()
    p64, pm = out["fp64"]["p1"], out["mixed"]["p1"]
    return {"config": {"workload": "mixed: cubed sphere nPanel 60 (21600 elements), OrdPoly 4, nz 64 quadratic, "
                                   f"NumTr 0, dt {cfg.dt:g} s", "nPanel": cfg.nPanel, "nz": cfg.nz, "dt": cfg.dt,
                       "dt_note": "dt 150 s (and 60 s, NaN within 60 steps) is beyond the explicit horizontal-acoustics limit of this W-method at "
                                  "nPanel 60 (it halves the grid spacing of nPanel 30, where 150 s already fails); "
                                  "50 s is stable for the simulated day"},
            "grid_setup_s": {"host": t_host, "device": t_dev,
                             "what": "metric, mass and dz of the nPanel-60 grid (topology and Glob numbering on the "
                                     "host in both); the runs below use the device-built grid"},
            "fp64_steps_per_s": out["fp64"]["steps_per_s"], "mixed_steps_per_s": out["mixed"]["steps_per_s"],
            "speedup_vs_fp64": out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"],
            "accuracy": {"simulated_days": nsteps * cfg.dt / 86400.0, "steps": nsteps,
                         "p1_rel_l2": float(np.sqrt(np.sum((pm - p64) ** 2) / np.sum(p64 ** 2))),
                         "p1_rel_linf": float(np.abs(pm - p64).max() / np.abs(p64).max()),
                         "mass_drift_mixed": float(out["mixed"]["drift"]), "mass_drift_fp64": float(out["fp64"]["drift"]),
                         "finite": out["fp64"]["finite"] and out["mixed"]["finite"],
                         "p1": "pressure of the lowest layer (surface-pressure proxy), mixed against the FP64 path "
                               "of the same configuration"}}


def adjoint_fd_entries(d, U, dt, nsteps, rng, per_field=8, rels=(1e-5, 1e-6, 1e-7, 1e-8), tol=1e-6):
    """Entry-wise check of the gradient of L(U0) = <lam, U_n> (U_n after
    nsteps steps, lam seeded Gaussian) through the step adjoints
    (steps_adjoint) against central differences: per field, per_field
    entries at levels spread over the column; each entry's error is the
    best of the step sizes rels (of the field's scale).  The forward is
    deterministic, so entries away from the perturbed one cancel exactly in
    the difference."""
    import torch
    lam = torch.from_numpy(rng.standard_normal(tuple(U.shape))).to(U.device)
    G = d.steps_adjoint(U, lam, dt, nsteps, every=1)
    NV, NumG, nz = U.shape
    wp, wm = U.clone(), U.clone()
    rows = []
    for f in range(NV):
        scale = max(float(U[f].abs().max()), 1.0)
        med = float(G[f].abs().median())
        for i in range(per_field):
            l, g = int((i * nz) // per_field), int(rng.integers(NumG))
            a = float(G[f, g, l])
            fds = []
            for rel in rels:
                h = rel * scale
                wp.copy_(U)
                wp[f, g, l] += h
                d.time_stepper(wp, dt, nsteps)
                wm.copy_(U)
                wm[f, g, l] -= h
                d.time_stepper(wm, dt, nsteps)
                # the difference first: away from the perturbed entry's reach the
                # two runs are identical, so only the affected entries add up
                fds.append(float(torch.sum(lam * (wp - wm))) / (2 * h))
            den = max(abs(a), med, 1e-300)
            rows.append({"err": min(abs(x - a) for x in fds) / den, "spread": (max(fds) - min(fds)) / den})
    errs = np.array([r["err"] for r in rows])
    spread = np.array([r["spread"] for r in rows])
    smooth = spread <= tol
    return {"entries": len(rows), "steps": nsteps, "rel_steps": list(rels), "tol": tol,
            "pass_fraction": float(np.mean(errs <= tol)), "pass_fraction_1e-5": float(np.mean(errs <= 1e-5)),
            "smooth_entries": int(smooth.sum()),
            "pass_fraction_smooth": float(np.mean(errs[smooth] <= tol)) if smooth.any() else None,
            "err_median": float(np.median(errs)), "err_max": float(errs.max()),
            "functional": "L = <lam, U_n>, lam ~ N(0,1) seeded; error = min over step sizes |FD - adjoint| / "
                          "max(|adjoint|, median |gradient| of the field); an entry is smooth when its "
                          "differences at the step sizes agree with each other within tol (no limiter or "
                          "upwind kink within reach)"}


def run_adjoint(args, rank, ranks, torch):
    """The hand-written adjoint on the drop-in grid without tracers
    (physics.CONFIGS['adjoint']), device-resident, timed with CUDA events on
    the library's stream (max over ranks):
      * the forward step, one step adjoint (replay + reverse), the tendency
        and its adjoint, at a state with vertical motion;
      * the sensitivity study (physics.ADJOINT_STUDY): J = mean squared
        lowest-layer pressure anomaly over the 10x10-degree box at 50N 60E
        after args.adjoint_steps steps from the baroclinic-wave state, its
        gradient with a checkpoint every 8 steps, against the forward run of
        the same steps;
      * with args.adjoint_fd, central differences of J along seeded random
        unit directions at several step sizes."""
    from cgd_b200 import setup
    from cgd_b200 import physics as Ph
    from cgd_b200.adjoint import BoxPressureFunctional, box_columns
    acfg = Ph.CONFIGS["adjoint"]
    study = Ph.ADJOINT_STUDY
    # no per-kernel event profile here: every forward step of the
    # checkpointed sweep is one call and should launch the captured graph
    prof = os.environ.get("CGD_PROFILE")
    os.environ["CGD_PROFILE"] = "0"
    try:
        d, U0, _ = setup(member_config(acfg, rank))
    finally:
        if prof is None:
            os.environ.pop("CGD_PROFILE", None)
        else:
            os.environ["CGD_PROFILE"] = prof
    stream = torch.cuda.ExternalStream(d.stream())
    dt = acfg.dt
    Ub = torch.from_numpy(np.ascontiguousarray(U0.transpose(2, 1, 0))).cuda()   # baroclinic-wave state
    U = Ub.clone()
    d.time_stepper(U, dt, max(3, args.warmup))   # a state with vertical motion
    gen = torch.Generator(device=U.device).manual_seed(20261203 + rank)
    L = torch.randn(U.shape, dtype=U.dtype, device=U.device, generator=gen)
    out = torch.empty_like(U)
    V = U.clone()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn, n):
        for _ in range(3):
            fn()
        ranks.barrier()
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        e1.synchronize()
        return ranks.max(e0.elapsed_time(e1) / n)

    n = max(3, min(args.steps, 20))
    fwd = timed(lambda: d.time_stepper(V, dt, n), 1) / n   # captured steps, as in the headline
    adj = timed(lambda: d.ros_step_adjoint(U, L, dt, out), n)
    rhs = timed(lambda: d.fcn(U, out), n)
    rhs_adj = timed(lambda: d.fcn_adjoint(U, L, out), n)

    W = args.adjoint_steps
    box = box_columns(d.grid, study["box_lat"], study["box_lon"])
    Jf = BoxPressureFunctional(d, dt, W, box=box, every=study["every"])
    ranks.barrier()
    e0.record(stream)
    V.copy_(Ub)
    d.time_stepper(V, dt, W)
    e1.record(stream)
    e1.synchronize()
    fwd_w = ranks.max(e0.elapsed_time(e1))
    e0.record(stream)
    J, G = Jf.value_and_grad(Ub)
    e1.record(stream)
    e1.synchronize()
    grad_w = ranks.max(e0.elapsed_time(e1))
    finite = bool(torch.isfinite(G).all().item())
    res = {"config": {"workload": "adjoint", "nPanel": acfg.nPanel, "OrdPoly": acfg.OrdPoly, "nz": acfg.nz,
                      "NumTr": acfg.NumTr, "dt": dt},
           "forward_step_ms": fwd, "step_adjoint_ms": adj, "step_ratio": adj / fwd,
           "tendency_ms": rhs, "tendency_adjoint_ms": rhs_adj, "tendency_ratio": rhs_adj / rhs,
           "sensitivity": {"J": J, "box_columns": int(box.size), "steps": W, "simulated_hours": W * dt / 3600.0,
                           "checkpoint_every": study["every"], "forward_ms": fwd_w, "gradient_ms": grad_w,
                           "ratio": grad_w / fwd_w, "finite": finite,
                           "functional": "mean over the box columns of (p1(U_n) - p1(U_0))^2, p1 the "
                                         "lowest-layer pressure, box 45-55N 55-65E"},
           "step_adjoint": "forward replay of the step keeping stage states, phase-1 caches, pressures and k; "
                           "reverse: transposed column Schur solve with band derivatives, tendency adjoint "
                           "(phase 2 and phase 1 with their transposed DSS), stage combinations"}
    # entry-wise central differences of a 4-step gradient on the drop-in grid
    res["fd_entries"] = adjoint_fd_entries(d, U, dt, 4, np.random.default_rng(20261205 + rank))
    if args.adjoint_fd:
        # central differences along seeded unit directions of the FP64 state space
        rng = np.random.default_rng(study["fd_seed"])
        nrm = float(torch.linalg.norm(Ub))
        work = Ub.clone()
        rels = (1e-7, 1e-8, 1e-9)
        rows = []
        for _ in range(study["fd_dirs"]):
            v = torch.from_numpy(rng.standard_normal(tuple(Ub.shape))).to(Ub.device)
            v /= torch.linalg.norm(v)
            ad = float(torch.sum(G * v))
            errs = []
            for rel in rels:
                eps = rel * nrm
                fd = Jf.diff(Ub + eps * v, Ub - eps * v, work) / (2 * eps)
                errs.append(abs(fd - ad) / abs(fd))
            rows.append({"adjoint": ad, "rel_err": errs})
        res["sensitivity"]["fd_check"] = {"directions": rows, "rel_steps": list(rels),
                                          "step": "eps = rel * |U0|_2 along unit directions of i.i.d. N(0,1)"}
    d.close()
    return res


def ensemble_measure(K, warmup, rank, ranks, torch):
    """The batched ensemble (physics.ENSEMBLE: 48 members, 16 each on
    (nPanel, nz) = (16, 30), (24, 45), (32, 64)), one CUDA graph per
    ensemble step, in FP64 and in the mixed form: K timed steps after warmup
    steps (the first call also runs the autotuner), then the rest of the 6
    simulated hours, and each member's lowest-level pressure, mixed against
    FP64, at the end."""
    from cgd_b200 import Dycore, Ensemble
    from cgd_b200 import physics as Ph
    from cgd_b200.model import _grid_and_state
    E = Ph.ENSEMBLE
    phys = Ph.PhysParameters()
    nsteps = int(round(E["hours"] * 3600.0 / E["dt"]))
    K = max(1, min(K, nsteps - warmup))
    members = []   # (grid, nu, U0)
    for n, nz in E["grids"]:
        rc = Ph.RunConfig(f"ens{n}_{nz}", n, E["OrdPoly"], nz, 0, E["dt"], nsteps, "quadratic")
        grid, base = _grid_and_state(rc)
        for j in range(E["per_grid"]):
            U = base.copy(order="F")
            Ph.member_perturbation(U, E["theta_amp"], E["wind_amp"], E["seed0"] + len(members) + 1000 * rank)
            members.append((grid, Ph.hyperdiffusion(n, E["OrdPoly"]), U))
    dof = sum(int(np.prod(U.shape)) for _, _, U in members)
    res = {}
    for prec in ("fp64", "mixed"):
        dycs = [Dycore(g, 0, nu, phys, precision=prec) for g, nu, _ in members]
        ens = Ensemble(dycs, autotune=True)
        stream = torch.cuda.ExternalStream(ens.stream())
        states = [torch.from_numpy(np.ascontiguousarray(U.transpose(2, 1, 0))).cuda() for _, _, U in members]
        dts = [E["dt"]] * len(members)
        m0 = [d.mass_integral(u) for d, u in zip(dycs, states)]
        ens.step(states, dts, warmup)      # the first call also runs the autotuner
        ranks.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(states, dts, K)
        e1.record(stream)
        e1.synchronize()
        t = ranks.max(e0.elapsed_time(e1) / 1e3)
        ens.step(states, dts, nsteps - warmup - K)
        torch.cuda.synchronize()
        p1 = [np.asarray(d.fcn_prepare(u))[0].copy() for d, u in zip(dycs, states)]
        drift = [(d.mass_integral(u) - a) / a for d, u, a in zip(dycs, states, m0)]
        finite = all(bool(torch.isfinite(u).all().item()) for u in states)
        res[prec] = {"t": t, "p1": p1, "drift": drift, "tuning": ens.tuning(), "finite": finite}
        ens.close()
        for d in dycs:
            d.close()
        del states
        torch.cuda.empty_cache()
    v64 = aggregate(ranks.world, K, res["fp64"]["t"]) * dof
    vm = aggregate(ranks.world, K, res["mixed"]["t"]) * dof
    errs = [float(np.sqrt(np.sum((b - a) ** 2) / np.sum(a ** 2))) for a, b in zip(res["fp64"]["p1"], res["mixed"]["p1"])]
    return {"dof_updates_per_s": v64, "unit": "DOF-updates/s", "steps": K, "warmup": warmup,
            "ms_per_step": res["fp64"]["t"] / K * 1e3, "dof_per_ensemble_step": dof,
            "members": len(members), "grids": E["grids"], "per_grid": E["per_grid"], "dt": E["dt"],
            "hours": E["hours"], "steps_total": nsteps, "tuning_fp64": res["fp64"]["tuning"],
            "chosen_form_fp64": res["fp64"]["tuning"].split("stage=")[1].split(";")[0],
            "mixed": {"dof_updates_per_s": vm, "speedup_vs_fp64": vm / v64,
                      "ms_per_step": res["mixed"]["t"] / K * 1e3, "tuning": res["mixed"]["tuning"],
                      "p1_rel_l2_vs_fp64": {"max": max(errs), "median": float(np.median(errs))},
                      "mass_drift_max": float(max(abs(x) for x in res["mixed"]["drift"]))},
            "mass_drift_fp64_max": float(max(abs(x) for x in res["fp64"]["drift"])),
            "finite": res["fp64"]["finite"] and res["mixed"]["finite"],
            "perturbation": f"theta +-{E['theta_amp']} K, u,v +-{E['wind_amp']} m/s, seed {E['seed0']}+member",
            "gpu_launches": {"fused": 3, "members": 15 * len(members)}.get(
                res["fp64"]["tuning"].split("stage=")[1].split(";")[0], 15) * K}


def run_ensemble(args, rank, world, local):
    """Batched-ensemble workload as its own line: every rank advances its
    own 48-member ensemble (ensemble_measure)."""
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    ranks = Ranks(rank, world, torch.device("cuda", local))
    r = ensemble_measure(args.steps, args.warmup, rank, ranks, torch)
    if rank == 0:
        line = {
            "metric": "ensemble DOF-updates/s (48 members, p4: 16 x (nPanel 16, nz 30), (24, 45), (32, 64))",
            "value": r["dof_updates_per_s"], "unit": "DOF-updates/s", "n_gpus": world, "steps": r["steps"],
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (baroclinic wave + seeded member perturbations)",
            "config": {"workload": "batched ensemble: 48 members on 3 grids, one CUDA graph per ensemble step "
                                   "(15 launches split, or 3 fused persistent stage launches; the autotuner picks "
                                   "the work-list order, the form and the levels per phase-2 CTA)",
                       "grids": r["grids"], "per_grid": r["per_grid"], "dt": r["dt"], "hours": r["hours"],
                       "steps_total": r["steps_total"], "perturbation": r["perturbation"],
                       "dt_note": "one dt below the explicit-acoustics limit of the finest member grid",
                       "parallelism": "one ensemble per GPU"},
            "dof_per_ensemble_step": r["dof_per_ensemble_step"], "tuning_fp64": r["tuning_fp64"],
            "mixed": r["mixed"], "mass_drift_fp64_max": r["mass_drift_fp64_max"], "finite": r["finite"],
            "gpu_launches": r["gpu_launches"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_output(dyc, Ut, cfg, rank, torch, reps=10):
    """The VTK output path on the timed run's state: cgd_output_fields for the
    reference's field list at OrdPrint 1 (device-resident, CUDA events on the
    library's stream), and one VtkOutput.write (interpolation, copy to pinned
    host memory, .vtu file) timed on the wall clock."""
    from cgd_b200 import output
    names = ("Rho", "u", "v", "wB", "Th", "Pres", "Vort") + tuple(f"Tr{q + 1}" for q in range(dyc.NumTr))
    t0 = time.perf_counter()
    w = output.VtkOutput(dyc, names=names, OrdPrint=1)
    t_setup = time.perf_counter() - t0
    out = torch.empty(len(names) * w.ncells, dtype=torch.float64, device=Ut.device)
    stream = torch.cuda.ExternalStream(dyc.stream())
    for _ in range(2):
        dyc.output_fields(Ut, w.codes, w.inter, out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        dyc.output_fields(Ut, w.codes, w.inter, out)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    S = (6 * cfg.nPanel ** 2 * cfg.OrdPoly ** 2 + 2) * cfg.nz * 8   # one (nz, NumG) field in bytes
    NF, nz, DoF = 6 * cfg.nPanel ** 2, cfg.nz, (cfg.OrdPoly + 1) ** 2
    metric_vort = 10 * DoF * nz * NF * 8                           # D11..D22 (both nodes), J of every level
    algo = (5 + dyc.NumTr) * S + metric_vort + len(names) * w.ncells * 8
    res = {"fields": list(names), "OrdPrint": 1, "cells": w.ncells, "ms_per_call": ms,
           "algorithmic_bytes": algo, "achieved_GBs": algo / (ms * 1e-3) / 1e9, "setup_s": t_setup,
           "launches_per_call": len(names)}
    if rank == 0:
        with tempfile.TemporaryDirectory() as tmp:
            t0 = time.perf_counter()
            path = w.write(Ut, os.path.join(tmp, "out"))
            w.wait()
            res["write_s"] = time.perf_counter() - t0
            res["file_bytes"] = os.path.getsize(path)
    return res


def run_ours(args, cfg, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    os.environ.setdefault("CGD_PROFILE", "1")
    from cgd_b200 import setup
    dyc, U0, mcfg = setup(member_config(cfg, rank), precision=args.precision)
    stream = torch.cuda.ExternalStream(dyc.stream())
    Ut = torch.from_numpy(np.ascontiguousarray(U0.transpose(2, 1, 0))).cuda()
    ranks = Ranks(rank, world, torch.device("cuda", local))
    barrier, max_over_ranks = ranks.barrier, ranks.max

    dt = cfg.dt
    dyc.time_stepper(Ut, dt, args.warmup)          # includes the one-time graph capture
    barrier()
    clocks = Clocks(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dyc.time_stepper(Ut, dt, args.steps)
    e1.record(stream)
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    barrier()
    clk = clocks.stop()
    t = max_over_ranks(t)
    value = aggregate(world, args.steps, t)
    ktimes = dyc.kernel_times()
    assert torch.isfinite(Ut).all().item()

    # end to end through the C ABI with a pinned host state
    Uh = torch.from_numpy(np.ascontiguousarray(U0.transpose(2, 1, 0))).pin_memory()
    dyc.time_stepper(Uh, dt, 1)
    barrier()
    Ke = max(1, args.e2e_steps)
    e0.record(stream)
    for _ in range(Ke):
        dyc.time_stepper(Uh, dt, 1)
    e1.record(stream)
    e1.synchronize()
    te = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    state_bytes = int(np.prod(U0.shape)) * 8
    e2e = {"value": aggregate(world, Ke, te), "unit": UNIT, "h2d_bytes_per_step": state_bytes,
           "d2h_bytes_per_step": state_bytes, "steps": Ke,
           "call": "cgd_ros_step(h, host_state, dt, 1) per step (pinned host buffer)"}

    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        mixed = run_mixed(args, cfg, rank, ranks, U0, value, torch)
    adjoint = None
    if args.precision == "fp64" and not args.no_adjoint:
        adjoint = run_adjoint(args, rank, ranks, torch)
    mixed_cfg3 = None
    if args.precision == "fp64" and not args.no_mixed_cfg3:
        mixed_cfg3 = run_mixed_cfg3(args, rank, ranks, torch)
    ensemble = None
    if args.precision == "fp64" and not args.no_ensemble:
        ensemble = ensemble_measure(args.ensemble_steps, 3, rank, ranks, torch)
        ensemble["single_member_dof_updates_per_s"] = value * unique_dof(cfg) / world
        ensemble["vs_single_member"] = ensemble["dof_updates_per_s"] / (value * unique_dof(cfg) / world)
        if adjoint is not None:
            # the members carry no tracers (5 fields per DOF); the same grid
            # without tracers, stepped alone (the adjoint leg's forward step)
            dof5 = unique_dof(cfg) // (5 + cfg.NumTr) * 5
            single5 = dof5 / (adjoint["forward_step_ms"] * 1e-3)
            ensemble["single_member_no_tracers_dof_updates_per_s"] = single5
            ensemble["vs_single_member_no_tracers"] = ensemble["dof_updates_per_s"] / single5

    outp = None
    if args.precision == "fp64" and not args.no_output:
        outp = run_output(dyc, Ut, cfg, rank, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, n = oracle_steps_per_s(cfg, args.cpu_steps, 1, threads)
        cpu = {"value": v, "unit": UNIT, "cores": n, "kind": "port",
               "sample": f"{args.cpu_steps} full-grid Rosenbrock-W steps after 1 warm-up step of the same "
                         f"configuration; C++ FP64 restatement of the reference CPU path, OpenMP on {n} "
                         f"threads ({cpu_model()})"}
        # one thread against all of them, on one tendency evaluation (a step
        # on one thread would take tens of seconds)
        tn, t1 = oracle_rhs_threads(cfg, n)
        cpu["one_thread"] = {"tendency_s": t1, "tendency_s_all_threads": tn, "thread_speedup": t1 / tn,
                             "steps_per_s_estimate": v * tn / t1,
                             "sample": "one full-grid tendency evaluation after one untimed one, on 1 and on "
                                       f"{n} threads; steps/s scaled by their ratio"}

    if rank == 0:
        peak, kind = measured_peak_hbm()
        fam = {}
        for name, ms in ktimes:
            fam.setdefault(name, []).append(ms)
        p2 = fam.get("phase2", [float("nan")])
        t_p2 = float(np.mean(p2)) / 1e3
        b_p2 = phase2_bytes(cfg)
        ach = b_p2 / t_p2 / 1e9
        step_ms = t / args.steps * 1e3
        b_step = step_bytes(cfg)
        shares = {k: round(float(np.sum(v)) / max(1e-12, sum(float(np.sum(x)) for x in fam.values())), 4)
                  for k, v in fam.items()}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (baroclinic wave + seeded noise)",
            "config": workload_config(cfg, args.precision),
            "dof_updates_per_s": value * unique_dof(cfg),
            "roofline": {"bound": "hbm", "kernel": "k_phase2 (fused tendency)", "achieved": ach, "peak": peak,
                         "peak_kind": kind, "unit": "GB/s", "frac": ach / peak, "traffic": ncu_traffic(),
                         "algorithmic_bytes_per_launch": b_p2, "launch_ms": t_p2 * 1e3,
                         "step": {"algorithmic_bytes": b_step, "achieved": b_step / (step_ms * 1e-3) / 1e9,
                                  "frac": b_step / (step_ms * 1e-3) / 1e9 / peak}},
            "kernel_ms_last_step": {k: [round(x, 4) for x in v] for k, v in fam.items()},
            "kernel_share": shares,
            "e2e": e2e,
            "mixed": mixed,
            "mixed_cfg3": mixed_cfg3,
            "adjoint": adjoint,
            "ensemble": ensemble,
            "output": outp,
            "gpu_launches": 15 * args.steps,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    dyc.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def run_shard(args, cfg, rank, world, local):
    """One grid decomposed over the ranks (strong scaling): every rank steps
    its contiguous range of elements; each of the two DSS points of every
    tendency exchanges the boundary element-node contributions with the
    neighbouring ranks (NCCL peer sends/receives through torch.distributed),
    and every rank sums a DOF's contributors in the single-process order.
    value = whole-grid steps/s over the max-over-ranks time."""
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from cgd_b200 import Dycore
    from cgd_b200 import physics as Ph
    from cgd_b200.model import _grid_and_state
    from cgd_b200.parallel import TorchTransport, build_plans, partition_elements
    grid, U0 = _grid_and_state(cfg)
    plans = build_plans(grid, partition_elements(grid.NF, world))
    P = plans[rank]
    d = Dycore(P.local_grid(grid), cfg.NumTr, Ph.hyperdiffusion(cfg.nPanel, cfg.OrdPoly), Ph.PhysParameters(),
               halo=P)
    if world > 1:
        d.set_transport(TorchTransport(P))
    ranks = Ranks(rank, world, torch.device("cuda", local))
    stream = torch.cuda.ExternalStream(d.stream())
    Ut = torch.from_numpy(np.ascontiguousarray(P.restrict(U0).transpose(2, 1, 0))).cuda()
    d.time_stepper(Ut, cfg.dt, args.warmup)
    ranks.barrier()
    clocks = Clocks(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d.time_stepper(Ut, cfg.dt, args.steps)
    e1.record(stream)
    e1.synchronize()
    t = ranks.max(e0.elapsed_time(e1) / 1e3)
    clk = clocks.stop()
    finite = bool(torch.isfinite(Ut).all().item())
    # end to end: the rank's part of the state from and to pinned host memory every step
    Uh = torch.from_numpy(np.ascontiguousarray(P.restrict(U0).transpose(2, 1, 0))).pin_memory()
    d.time_stepper(Uh, cfg.dt, 1)
    ranks.barrier()
    Ke = max(1, args.e2e_steps)
    e0.record(stream)
    for _ in range(Ke):
        d.time_stepper(Uh, cfg.dt, 1)
    e1.record(stream)
    e1.synchronize()
    te = ranks.max(e0.elapsed_time(e1) / 1e3)
    bytes_local = int(Uh.numel()) * 8
    tot_bytes = ranks.max(bytes_local) * world if world > 1 else bytes_local
    if rank == 0:
        c = workload_config(cfg, "fp64")
        c["parallelism"] = f"horizontal decomposition over {world} GPU(s): contiguous element ranges, " \
                           f"halo exchange of DSS contributions (two per tendency)"
        c["ghost_slots_rank0"] = int(P.n_ghost)
        line = {"metric": METRIC, "value": args.steps / t, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (baroclinic wave + seeded noise)", "config": c,
                "dof_updates_per_s": args.steps / t * unique_dof(cfg), "finite": finite,
                "e2e": {"value": Ke / te, "unit": UNIT, "h2d_bytes_per_step": tot_bytes,
                        "d2h_bytes_per_step": tot_bytes, "steps": Ke,
                        "call": "cgd_ros_step(h_rank, host_part, dt, 1) per step on every rank"},
                "gpu_launches": (15 + (12 if world > 1 else 0)) * args.steps, "clocks": clk}
        print(json.dumps(line), flush=True)
    d.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    rank, world, local = dist_env()
    from cgd_b200 import physics as Ph
    if args.config == "ensemble":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the ensemble workload has no CPU "
                                  "reference arm (the CPU restatement takes minutes per step at this size)"}))
            return
        run_ensemble(args, rank, world, local)
        return
    cfg = Ph.CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, cfg, rank)
        return
    if args.parallel == "shard":
        run_shard(args, cfg, rank, world, local)
        return
    run_ours(args, cfg, rank, world, local)


if __name__ == "__main__":
    main()
