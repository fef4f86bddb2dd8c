"""Benchmark: induced-charge solves per second on the 162k-charge conductor system.

One step = one full solve of the workload: right-hand side, flexible GMRES to a true
relative residual of 1e-6, and the bead forces, through the C ABI (cr_compute).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload precision_162k|plain_small|replicas_256|dynamics_420k|mlp|polydisperse_204k]

The headline arm (FP32 operator inside FP64-Arnoldi flexible GMRES with FP64 refinement,
two-level preconditioner, each Arnoldi step a captured CUDA graph) is timed beside, in
the same run on the same B200: the same solver in FP64 (the precision-only ratio), FP64
with the conductor response only, and the plain FP64 method with the reference's
diagonal preconditioner.  Every arm's solution is compared with the oracle's (q, Phi,
F).  Kernel shares and the roofline come from a profiled (uncaptured) pass of the same
steps right after the timed region.  Inputs are resident in HBM for ``value``; ``e2e``
repeats the step through cr_compute_host with host buffers, the copies inside the timed
region.  ``--workload plain_small`` is the 4,200-charge plain-method system (FP64
throughout), with a measured full CPU solve beside it.  Multi-GPU runs are independent
replicas (one system per rank, no collective on the data path).  ``--impl reference``
times the reference method's CPU implementation (the FP64 oracle port) on the host
cores, with inputs from the oracle-side generator.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "precision_162k"
METRIC = "solves/s at 1e-6 residual: learned+FP32 vs plain FP64, same B200; spread GB/s"
UNIT = "solves/s"
RESTART = 50          # headline arm (conductor-response preconditioner)
RESTART_PLAIN = 300   # plain arm: the reference's diagonal preconditioner stagnates with short restarts
TOL = 1e-6
#: GMRES iterations of one plain FP64 solve (the reference's diagonal preconditioner,
#: restart 300, true relative residual 1e-6) of the 162k-charge workload (seed 1),
#: measured on B200; projects the reference arm's sampled CPU iterations to a solve
ITERATIONS_PLAIN_FP64 = {"precision_162k": 3835}

PROFILE_BYTES_DOC = {
    "spread": "N*(16+s) + G*s (positions and charges in, one real mesh written)",
    "contract": "G*s + N*(16+s)",
    "real_space": "4*L_pairs + N*(16+2s) (stored neighbour entries plus per-bead data)",
    "fft": "2*G*s per R2C/C2R transform (real side) + 2*G*s (half-spectrum complex side)",
}


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str):
        self.device_id = device_id
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", self.device_id], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        pw = [num(r[3]) for r in rows if num(r[3]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(n)
        under = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(under) if under else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "samples": len(rows), "reasons": sorted(reasons)}


ROOFLINE_CLASSES = ("spread", "contract", "contract_force", "real_space", "real_space_force", "fft", "scale")


def algorithmic_bytes(kind: str, prec_bytes: int, N: int, G: int, pairs: int, cluster_pairs: int = 0) -> float:
    s = prec_bytes
    pos = 16 if s == 4 else 32
    if kind == "spread":
        return N * (pos + s) + G * s
    if kind == "contract":
        return G * s + N * (pos + s)
    if kind == "contract_force":
        return G * s + N * (pos + s) + N * 3 * s
    if kind == "real_space":
        # packed pair values + 128-byte bit mask and 12-byte index/offset per cluster pair
        # + charges in and potentials out
        return float(s) * pairs + 140.0 * cluster_pairs + N * (4 + 2 * s)
    if kind == "real_space_force":
        return 4.0 * pairs + N * (pos + 2 * s) + N * 3 * 8
    if kind == "fft":
        return 2.0 * G * s + 2.0 * G * s
    if kind == "scale":
        return (G / 2) * (2 * s * 2 + s)
    return float("nan")


def run_op_case(args) -> None:
    """Operator applications on the scaled workload (the case the ncu captures use)."""
    import torch

    from conductorrigid_b200 import _lib, systems
    from conductorrigid_b200.device import Handle

    w = systems.workload(WORKLOAD, scale=args.op_case)
    s, p = w.system, w.params
    full_L = systems.workload(WORKLOAD).system.L[0]
    grid = systems.smooth_at_least(int(np.ceil(p["grid"] * s.L[0] / full_L)), 4096)  # same mesh spacing
    base = dict(xi=p["xi"], errortol=p["errortol"], grid=grid, support=p["support"], rcut=p["rcut"])
    h = Handle(_lib.make_params(field=tuple(s.field), precond="conductor", **base), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_realspace(args.realspace)
    h.set_positions(s.pos, s.body_pos)
    x = torch.randn(s.n_beads + s.n_bodies, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup + args.steps):
        h.apply_operator(x, _lib.CR_FP32)
    torch.cuda.synchronize()
    print(json.dumps({"op_case": args.op_case, "charges": s.n_beads, "mesh": grid, **h.geometry_info()}))
    h.close()


def run_replicas(args) -> None:
    """256 uneven independent replicas, three ways: the lockstep batch (cr_batch_solve: one
    Arnoldi step of every unconverged replica per round, each stage one launch over all
    replicas; the workload's value), the stream batch (cr_batch_compute: the single-system
    solver of each replica on its own stream, tiling policy tuned by batch throughput),
    and the single-system solver looped.  Both batches run on their own streams, so each
    timed region is bracketed by device synchronisation and CUDA events on the default
    stream."""
    import torch

    from conductorrigid_b200 import systems
    from conductorrigid_b200.batch import Replicas

    R = Replicas(systems.replica_specs(256, seed=1), precond=args.precond)
    nt = args.batch_threads

    def timed(fn):
        R.reset()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1), st

    # --arms lockstep: the lockstep arm alone (a launch list of its rounds under ncu)
    only_lockstep = set(args.arms.split(",")) == {"lockstep"}
    # the looped single-system solve: reference solutions and the looped rate
    for h in R.handles:
        h.set_tiling(8, 0)
    if only_lockstep:
        ms_loop, st_loop, ref = None, None, None
    else:
        R.warm()
        ms_loop, st_loop = timed(R.solve_looped)
        ref = [tuple(a.clone() for a in arr[2:]) for arr in R.arrays]
    # lockstep batch (8^3 register-column tiling, the default)
    for _ in range(args.warmup):
        timed(lambda: R.solve_lockstep(nt))
    l0, f0, r0 = R.lockstep_counters()
    ms_lock = [timed(lambda: R.solve_lockstep(nt)) for _ in range(args.steps)]
    l1, f1, r1 = R.lockstep_counters()
    phases = R.lockstep_phases()
    st = ms_lock[-1][1]
    err = None
    if ref is not None:
        err = {"q": 0.0, "phi": 0.0, "force": 0.0}
        for arr, want in zip(R.arrays, ref):
            for key, a, b in zip(("q", "phi", "force"), arr[2:], want):
                err[key] = max(err[key], float((a - b).abs().max() / b.abs().max().clamp_min(1e-300)))
        err = {k: float(f"{v:.3g}") for k, v in err.items()}
    rounds = (r1 - r0) / args.steps
    t_lock = statistics.median(m for m, _ in ms_lock)
    t_batch, st_b, policy_rates = None, None, {}
    if not only_lockstep:
        # stream batch, tiling policy chosen by its own throughput
        policy_rates = R.tune_batch(nt)  # untimed set-up
        for _ in range(args.warmup):
            timed(lambda: R.solve_batched(nt))
        ms = [timed(lambda: R.solve_batched(nt)) for _ in range(args.steps)]
        t_batch = statistics.median(m for m, _ in ms)
        st_b = ms[-1][1]
    groups = len({tuple(h.derived().grid) for h in R.handles})
    line = {
        "metric": "replica solves/s at 1e-6 residual, 256 uneven replicas in one batch",
        "value": round(R.n / (t_lock / 1e3), 2), "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_lock, 2), "higher_is_better": True,
        "stream_batch_solves_per_s": round(R.n / (t_batch / 1e3), 2) if t_batch else None,
        "looped_solves_per_s": round(R.n / (ms_loop / 1e3), 2) if ms_loop else None, "preconditioner": args.precond,
        "iterations_mean": round(float(np.mean([s["iterations"] for s in st])), 1),
        "iterations_max": int(max(s["iterations"] for s in st)),
        "iterations_mean_looped": round(float(np.mean([s["iterations"] for s in st_loop])), 1) if st_loop else None,
        "converged": int(sum(s["converged"] for s in st)),
        "converged_stream_batch": int(sum(s["converged"] for s in st_b)) if st_b else None,
        "max_final_residual": max(s["final_residual"] for s in st),
        "error_vs_looped": err,
        "lockstep": {"phase_ms": {k: round(v, 2) for k, v in phases.items()}, "rounds_per_solve": rounds, "kernel_launches_per_round": round((l1 - l0) / args.steps / rounds, 1),
                     "batched_transforms_per_solve": (f1 - f0) / args.steps, "mesh_size_groups": groups},
        "replicas": R.n, "charges": R.n_charges,
        "host_threads": nt, "tiling_policy_stream_batch": getattr(R, "best_policy", None),
        "tiling_policy_rates": {k: round(v, 1) for k, v in policy_rates.items()},
        "dtype": "f32 operator, f64 Krylov", "data": "synthetic (seeded replica generator)",
        "config": {"workload": "replicas_256: N_body~U[20,400], phi~U[0.05,0.35], |E0|=1, 2 nodes/unit, P=9",
                   "mesh_tiling": "8^3 tiles, register-column spreading (lockstep); stream batch: tuned policy",
                   "arnoldi_steps": "lockstep rounds (stream batch: captured graphs)"},
    }
    R.close()
    print(json.dumps(line), flush=True)


def run_dynamics(args) -> None:
    """Rigid-body Brownian steps of the 420k-charge suspension, three solvers on one
    trajectory: the plain solver warm-started from the previous step (it moves the
    bodies), the learned start (guess directions with the network trained online on the
    first --train-solves solves), and the learned start plus the learned preconditioner
    correction (its network trained online on the same solves, then used by every solve
    whose initial-residual test it passes).  Per-step device time includes, for the learned
    arms, the features, network inference and training."""
    import torch

    from conductorrigid_b200 import _lib, systems
    from conductorrigid_b200.dynamics import paired_run

    w = systems.workload("dynamics_420k", scale=args.scale)
    s, p = w.system, w.params
    grid = p["grid"] if args.scale == 1.0 else systems.smooth_at_least(int(np.ceil(256 * s.L[0] / 49.28)), 4096)
    common = dict(field=tuple(s.field), xi=p["xi"], errortol=p["errortol"], grid=grid, support=p["support"],
                  rcut=p["rcut"], gmres_tol=TOL, restart=RESTART, maxiter=20000, precision="mixed",
                  precond=args.precond)
    steps = args.warmup + args.steps
    train = args.train_solves if args.train_solves > 0 else min(200, max(1, steps // 2))
    out, guess, corr = paired_run(_lib.make_params(**common), _lib.make_params(learned=True, **common), s,
                                  np.ones(s.n_bodies), steps, train_solves=train, seed=1,
                                  coarse=(args.coarse_max_dense, args.coarse_cg), corrected=True)
    tail = out[max(train + 1, args.warmup):]

    def arm(name):
        ms = float(np.mean([o[name]["step_ms"] for o in tail]))
        d = {"iterations": round(float(np.mean([o[name]["iterations"] for o in tail])), 1),
             "ms_per_step": round(ms, 2), "solves_per_s": round(1e3 / ms, 3),
             "ns_per_day": round(1e3 / ms * 86400 * 1e-3, 1),
             "converged": int(sum(o[name]["converged"] for o in tail))}
        if name == "corrected":
            d["solves_using_correction"] = int(sum(o[name]["used_learned_correction"] for o in tail))
            red = [o[name]["correction_reduction"] for o in tail if o[name]["correction_reduction"][0] >= 0]
            if red:
                d["initial_step_reduction_plain_vs_corrected"] = [round(float(np.mean([r[0] for r in red])), 4),
                                                                  round(float(np.mean([r[1] for r in red])), 4)]
        return d

    line = {
        "metric": "dynamics: GMRES iterations per step and solves/s, learned start (+ learned preconditioner "
                  "correction) vs plain warm start",
        "value": arm("learned")["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": len(tail),
        "warmup": len(out) - len(tail), "higher_is_better": True,
        "learned": arm("learned"), "corrected": arm("corrected"), "plain_warm_start": arm("plain"),
        "trained_solves": guess.trained, "correction_trained_solves": corr.trained,
        "preconditioner": args.precond, "coarse_cg": args.coarse_cg,
        "heldout_explained": round(float(np.mean(guess.heldout[-len(tail):])) if guess.heldout else 0.0, 3),
        "correction_heldout_explained": round(float(np.mean(corr.heldout[-20:])) if corr.heldout else 0.0, 3),
        "dtype": "f32 operator, f64 Krylov; bf16 networks", "data": "synthetic (seeded placement, relaxed)",
        "config": {"workload": f"dynamics_420k scale {args.scale}: {s.n_bodies} spheres x 42, phi 0.35, "
                               f"mesh {grid}^3, P=9, dt 1e-3, kT 1, steric repulsion k=1000 gap 0.1, "
                               f"{steps} steps, networks trained on the first {train} solves",
                   "ns_per_day_unit": "reduced time units per day (dt = 1e-3)"},
    }
    print(json.dumps(line), flush=True)


def run_mlp(args) -> None:
    """The learned part's tensor-core kernels at the dynamics size (one row per bead,
    420,000 rows): inference and one training step (forward, backward, weight gradients;
    the Adam update is timed with it).  FLOPs per row: 2 * (48*128 + 128*128 + 128) in the
    forward, and 2 * (128*128) + 2 * (128*128 + 128) + 2 * (48*128 + 48) more in the
    backward (dH1, dW2 with db2, dW1 with db1), the MMA work the kernels issue."""
    import torch

    from conductorrigid_b200.learned import FEATURES, Network

    n = 420_000
    net = Network(seed=1)
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(n, FEATURES, device="cuda", generator=g).to(torch.bfloat16).view(torch.int16).contiguous()
    t = torch.randn(n, device="cuda", generator=g)
    f_fwd = 2.0 * (48 * 128 + 128 * 128 + 128)
    f_bwd = 2.0 * (128 * 128) + 2.0 * (128 * 128 + 128) + 2.0 * (48 * 128 + 48)
    pf = ROOT / "MEASURED_PEAKS.json"
    peak, peak_src = (float(json.loads(pf.read_text())["bf16_tflops"]), "measured bf16 burst") if pf.exists() \
        else (1590.0, "fallback bf16 burst")

    def timed(fn, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    for _ in range(args.warmup):
        net.forward(x)
        net.train_step(x, t)
    c0 = net.counters()["kernel_launches"]
    ms_f = timed(lambda: net.forward(x), args.steps)
    ms_t = timed(lambda: net.train_step(x, t), args.steps)
    launches = net.counters()["kernel_launches"] - c0
    tf_f = n * f_fwd / (ms_f * 1e-3) / 1e12
    tf_t = n * (f_fwd + f_bwd) / (ms_t * 1e-3) / 1e12
    line = {
        "metric": "per-bead network on tcgen05: rows/s and TFLOP/s (inference, training step)",
        "value": round(n / (ms_t * 1e-3), 1), "unit": "training rows/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "dtype": "bf16 operands, f32 accumulate",
        "data": "synthetic normal features", "rows": n,
        "inference": {"ms": round(ms_f, 4), "tflops": round(tf_f, 2)},
        "training_step": {"ms": round(ms_t, 4), "tflops": round(tf_t, 2)},
        "roofline": {"bound": "tensor", "achieved": round(tf_t, 2), "peak": peak, "unit": "TFLOP/s",
                     "frac": round(tf_t / peak, 4), "peak_source": peak_src},
        "gpu_launches": launches,
        "config": {"workload": "mlp_420k: 48-128-128-1 GELU network, one row per bead of the 420k-charge system"},
    }
    print(json.dumps(line), flush=True)


def run_polydisperse(args) -> None:
    """Charged polydisperse mixture (1000 spheres a=1 with 42 charges, 1000 a=2 with 162,
    Q = +-1 summing to zero, phi 0.25, E0 (0.3, 0, 1), mesh 256^3, P = 11): the full stack
    (FP32 operator, FP64 Krylov, conductor preconditioner, captured steps, autotuned
    tiling) against the plain FP64 solve with the reference's preconditioner, both with
    their errors in q, Phi and F against the oracle's solution (the committed oracle
    solution of this system, its residual re-checked, forces from the oracle)."""
    import torch

    from conductorrigid_b200 import _lib, systems
    from conductorrigid_b200.device import Handle

    w = systems.workload("polydisperse_204k", seed=1)
    s, p = w.system, w.params
    base = {k: p[k] for k in ("xi", "errortol", "grid", "support", "rcut")}
    common = dict(field=tuple(s.field), maxiter=40000, **base)
    stream = torch.cuda.Stream()
    # default: the conductor response; at phi = 0.25 the dense induced-dipole coarse level
    # saves 75 -> 57 iterations but costs more than that (136 vs 130 ms per solve)
    h_fast = Handle(_lib.make_params(precision="mixed", precond=args.precond, restart=RESTART, gmres_tol=TOL,
                                     **common), s.L, stream=stream)
    h_fast.set_coarse(args.coarse_max_dense, args.coarse_cg)
    h_plain = Handle(_lib.make_params(precision="fp64", precond="diagonal", restart=RESTART_PLAIN, gmres_tol=TOL,
                                      **common), s.L, stream=stream)
    for h in (h_fast, h_plain):
        h.set_topology(s.body, s.rigid, s.body_charge)
    pos = h_fast.dev(s.pos)
    bpos = h_fast.dev(s.body_pos)
    tiling = h_fast.autotune(pos, bpos, reps=5)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def solve(h, k):
        ms, out = [], None
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                q = torch.zeros(s.n_beads, dtype=torch.float64, device="cuda")
                phi = torch.zeros(s.n_bodies, dtype=torch.float64, device="cuda")
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                F, st = h.compute(pos, bpos, q, phi)
                e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            out = (q, phi, F, st)
        return float(np.median(ms)), out

    solve(h_fast, args.warmup)
    ms_fast, (q, phi, F, st) = solve(h_fast, args.steps)
    ms_plain, (qp, php, Fp, stp) = solve(h_plain, 1)
    errors = None
    if not args.no_oracle:
        ref = oracle_solution("polydisperse_204k", s, p)
        errors = {"reference": ref["how"], "reference_oracle_residual": ref["residual"],
                  "fast": error_vs_oracle(ref, s, q.cpu().numpy(), phi.cpu().numpy(), F.cpu().numpy()),
                  "plain": error_vs_oracle(ref, s, qp.cpu().numpy(), php.cpu().numpy(), Fp.cpu().numpy())}

    line = {
        "metric": "solves/s at 1e-6 residual: full stack vs plain FP64, charged polydisperse mixture",
        "value": round(1e3 / ms_fast, 3), "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_fast, 1), "higher_is_better": True,
        "iterations": st["iterations"], "final_residual": st["final_residual"],
        "preconditioner": args.precond,
        "coarse_level": h_fast.coarse_info() if args.precond == "two_level" else None,
        "plain_fp64": {"value": round(1e3 / ms_plain, 4), "ms_per_step": round(ms_plain, 1),
                       "iterations": stp["iterations"], "converged": stp["converged"],
                       "final_residual": stp["final_residual"]},
        "speedup_vs_plain_fp64": round(ms_plain / ms_fast, 2),
        "error_vs_oracle": errors["fast"] if errors else None,
        "errors_vs_oracle": errors,
        "dtype": "f32 operator / f64 Krylov", "data": "synthetic (seeded placement)",
        "config": {"workload": "polydisperse_204k: 1000 a=1 x 42 + 1000 a=2 x 162 charges, Q=+-1, phi 0.25, "
                               "E0 (0.3,0,1), mesh 256^3, P=11, rc 4", "mesh_tiling": tiling,
                   "l2": "flushed (256 MB write) before every step"},
    }
    for h in (h_fast, h_plain):
        h.close()
    print(json.dumps(line), flush=True)



# ------------------------------------------------------------------ oracle side
def oracle_solution(name: str, s, p) -> dict:
    """The oracle's solution of the workload and the oracle's forces at it.

    precision_162k: the committed oracle solution (tests/golden/make_solutions.py: the
    oracle's operator solved to a true relative residual of 1e-11), its residual
    re-checked here.  plain_small: the oracle's restatement of the reference's solver
    (GMRES with the diagonal preconditioner, restart 300) converged to 1e-12 in this run.
    Forces: the oracle's force pass at those charges (ConductorRigid.cu:1256-1278)."""
    import oracle

    t0 = time.perf_counter()
    orc = oracle.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    fixture = ROOT / "tests" / "golden" / f"solution_{name}.npz"
    if fixture.exists():
        g = np.load(fixture)
        if len(g["q"]) != s.n_beads or len(g["phi"]) != s.n_bodies:
            raise RuntimeError(f"{fixture.name} does not describe this system")
        q, phi = np.array(g["q"]), np.array(g["phi"])
        how = f"committed oracle solution ({fixture.name})"
    else:
        ref = orc.solve(s.field, restart=300, maxiter=20000, tol=1e-12)
        q, phi = ref["q"], ref["phi"]
        how = "oracle GMRES (reference method: diagonal preconditioner, restart 300) to 1e-12 in this run"
    out = {"q": q, "phi": phi, "force": orc.forces(q, s.field), "oracle": orc, "how": how,
           "residual": orc.residual(q, phi, s.field)}
    out["seconds"] = time.perf_counter() - t0
    return out


def error_vs_oracle(ref: dict, s, q, phi, F) -> dict:
    """Max-norm errors relative to the largest entry, and the solution's true relative
    residual under the oracle's operator."""
    def rel(a, b):
        return float(np.abs(np.asarray(a) - b).max() / max(np.abs(b).max(), 1e-300))

    return {"q": rel(q, ref["q"]), "phi": rel(phi, ref["phi"]), "force": rel(F, ref["force"]),
            "oracle_residual": ref["oracle"].residual(q, phi, s.field)}


def cpu_gmres_sample(s, p, iterations: int, cycles: int, restart: int = 10) -> dict:
    """The reference method on the host cores, sampled: the oracle's set-up (tables,
    neighbour list) and `cycles` complete GMRES(restart) cycles of its restatement of the
    reference's solver (diagonal preconditioner, ConductorRigid.cu:1051-1151), continuing
    one solve.  A cycle of `restart` iterations runs restart + 2 operator applications;
    the time per iteration is the cycle time / restart.  One solve is projected as set-up
    + `iterations` x that time (operator-dominated: Gram-Schmidt is a few per cent)."""
    import oracle

    t0 = time.perf_counter()
    orc = oracle.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    setup = time.perf_counter() - t0
    b = orc.objective(s.field)
    x = np.zeros(s.n_beads + s.n_bodies)
    per_iter = []
    for _ in range(cycles):
        t = time.perf_counter()
        x, it, _ = orc.gmres(b, x0=x, restart=restart, maxiter=restart, tol=1e-300)
        per_iter.append((time.perf_counter() - t) / max(it, 1))
    t_it = float(np.median(per_iter))
    cores = oracle.lib().orc_num_threads()
    solve_s = setup + iterations * t_it
    return {"value": 1.0 / solve_s, "unit": UNIT, "cores": cores, "kind": "port", "seconds_per_solve": solve_s,
            "sample": (f"oracle set-up ({setup:.2f} s) + {cycles} complete GMRES({restart}) cycles of the reference "
                       f"method (diagonal preconditioner, FP64) on the {s.n_beads}-charge system, {cores} host "
                       f"threads, {t_it:.3f} s per iteration; projected to the {iterations} iterations the same "
                       f"method needs to reach 1e-6 (measured on the GPU): extrapolated, not a full solve")}


def cpu_full_solve(s, p) -> dict:
    """One complete solve plus forces of the reference method on the host cores: the
    oracle's GMRES (diagonal preconditioner, restart 300, CUSP's stopping rule on the
    left-preconditioned residual, ConductorRigid.cu:1134-1136) to 1e-6, then the force
    pass.  Measured, not projected."""
    import oracle

    t0 = time.perf_counter()
    orc = oracle.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    r = orc.solve(s.field, restart=RESTART_PLAIN, maxiter=20000, tol=TOL)
    dt = time.perf_counter() - t0
    cores = oracle.lib().orc_num_threads()
    return {"value": 1.0 / dt, "unit": UNIT, "cores": cores, "kind": "port", "seconds_per_solve": dt,
            "iterations": r["iterations"], "true_residual": r["true_rel"],
            "sample": (f"one measured full FP64 solve + forces of the {s.n_beads}-charge system by the oracle's "
                       f"reference method (set-up, GMRES({RESTART_PLAIN}) with the diagonal preconditioner to 1e-6, "
                       f"{r['iterations']} iterations, force pass) on {cores} host threads")}


def run_reference(args) -> None:
    """The reference method's CPU implementation (the FP64 oracle port) on the host cores,
    on the headline workload; inputs from the oracle-side generator, so that nothing of
    the CUDA product is loaded.  Each step is one complete GMRES(10) cycle of one
    continuing solve; the line reports the projected solves/s."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    import oracle
    from oracle import systems as osys

    name = args.workload if args.workload in SOLVE_WORKLOADS else WORKLOAD
    s, p = osys.workload(name, seed=1)
    config = {"workload": name, "charges": s.n_beads, "bodies": s.n_bodies, "mesh": p["grid"],
              "support": p["support"], "rcut": p["rcut"], "tol": TOL, "preconditioner": "diagonal (reference)"}
    if name not in ITERATIONS_PLAIN_FP64:  # small enough for complete solves: each step one measured solve
        for _ in range(args.warmup):
            cpu_full_solve(s, p)
        runs = [cpu_full_solve(s, p) for _ in range(args.steps)]
        solve_s = float(np.median([r["seconds_per_solve"] for r in runs]))
        value = 1.0 / solve_s
        cb = dict(runs[-1], value=value)
        cb.pop("seconds_per_solve", None)
        print(json.dumps({"impl": "reference", "metric": SOLVE_WORKLOADS[name][2], "value": value, "unit": UNIT,
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": solve_s * 1e3, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                          "cpu_baseline": cb,
                          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    iterations = ITERATIONS_PLAIN_FP64[name]
    t0 = time.perf_counter()
    orc = oracle.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    setup = time.perf_counter() - t0
    b = orc.objective(s.field)
    x = np.zeros(s.n_beads + s.n_bodies)
    per_iter = []
    for k in range(args.warmup + args.steps):
        t = time.perf_counter()
        x, it, _ = orc.gmres(b, x0=x, restart=10, maxiter=10, tol=1e-300)
        if k >= args.warmup:
            per_iter.append((time.perf_counter() - t) / max(it, 1))
    t_it = float(np.median(per_iter))
    solve_s = setup + iterations * t_it
    value = 1.0 / solve_s
    cores = oracle.lib().orc_num_threads()
    sample = (f"oracle set-up ({setup:.2f} s) + {args.steps} timed complete GMRES(10) cycles ({args.warmup} warm-up) "
              f"of the reference method (diagonal preconditioner, FP64) on the {s.n_beads}-charge system, {cores} "
              f"host threads, {t_it:.3f} s per iteration; projected to the {iterations} iterations the same method "
              f"needs to reach 1e-6 (measured on the GPU): extrapolated, not a full solve")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": solve_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- solve workloads
#: solver arms: precision, preconditioner, restart (None: --restart)
ARMS = {
    "fast": ("mixed", None, None),            # FP32 operator, FP64 Krylov; --precond (two-level by default)
    "f64t": ("fp64", "two_level", RESTART),   # FP64, the same preconditioner: the precision-only ratio
    "f64c": ("fp64", "conductor", RESTART),   # FP64, conductor response only
    "plain": ("fp64", "diagonal", RESTART_PLAIN),  # the reference method in FP64
}
ARM_LABELS = {
    "fast": "FP32 operator in FGMRES, FP64 Arnoldi / constraints / refinement",
    "f64t": "FP64 throughout, same preconditioner as the headline",
    "f64c": "FP64 throughout, conductor-response preconditioner",
    "plain": "FP64 throughout, the reference's diagonal preconditioner (plain method)",
}
#: workload -> (headline arm, arms, metric)
SOLVE_WORKLOADS = {
    "precision_162k": ("fast", ("fast", "f64t", "f64c", "plain"), METRIC),
    "plain_small": ("plain", ("plain", "f64t", "fast"),
                    "solves/s of the plain FP64 method (one solve + forces, 1e-6 residual), 4,200 charges"),
}


def run_solve(args) -> None:
    import torch
    import torch.distributed as dist

    from conductorrigid_b200 import _lib, ranks, systems
    from conductorrigid_b200.device import Handle

    name = args.workload
    head_arm, all_arms, metric = SOLVE_WORKLOADS[name]
    arms = [a for a in all_arms if a in set(args.arms.split(",")) or a == head_arm]
    rank, local, world = ranks.rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    w = systems.workload(name, seed=ranks.replica_seed(1, rank), scale=args.scale)
    s, p = w.system, w.params
    if args.scale != 1.0:  # profiling case: fewer bodies at the same mesh spacing
        full_L = systems.workload(name).system.L[0]
        p = dict(p, grid=systems.smooth_at_least(int(np.ceil(p["grid"] * s.L[0] / full_L)), 4096))
    base = {k: p[k] for k in ("xi", "errortol", "grid", "support", "rcut")}
    common = dict(field=tuple(s.field), gmres_tol=TOL, maxiter=20000, **base)
    stream = torch.cuda.Stream()
    handles = {}
    for a in arms:
        prec, pc, rs = ARMS[a]
        h = Handle(_lib.make_params(precision=prec, precond=pc or args.precond, restart=rs or args.restart,
                                    learned=bool(args.learned) and a == "fast", **common), s.L, stream=stream)
        h.set_coarse(args.coarse_max_dense, args.coarse_cg)
        h.set_realspace(args.realspace)
        h.set_topology(s.body, s.rigid, s.body_charge)
        handles[a] = h
    hh = handles[head_arm]
    pos = hh.dev(s.pos)
    bpos = hh.dev(s.body_pos)
    if args.tiling:  # an explicit tiling (profiling runs: timing-based choices are not valid under a profiler)
        t_edge, t_mode = (int(v) for v in args.tiling.split(","))
        for h in handles.values():
            h.set_tiling(t_edge, t_mode)
        tiling = {"tile_edge": t_edge, "spread_mode": t_mode, "mesh_ms": None}
    else:
        tiling = handles["fast"].autotune(pos, bpos, reps=5) if "fast" in handles else None  # untimed set-up
    q = torch.zeros(s.n_beads, dtype=torch.float64, device="cuda")
    phi = torch.zeros(s.n_bodies, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2
    results = {}

    def timed(a, steps, profile=False):
        """Per-step device time (CUDA events on the solver's stream), L2 flushed before each
        step; the last step's solution is kept for the error check."""
        h = handles[a]
        stats, total_ms = [], 0.0
        if profile:
            h.profile(True)
        c0 = h.counters()
        F = None
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                q.zero_()
                phi.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            F, st = h.compute(pos, bpos, q, phi)
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            stats.append(st)
        c1 = h.counters()
        prof = h.profile_read() if profile else None
        if profile:
            h.profile(False)
        sol = (q.cpu().numpy(), phi.cpu().numpy(), F.cpu().numpy())
        return {"ms": total_ms / steps, "stats": stats, "prof": prof, "sol": sol,
                "launches": c1["kernel_launches"] - c0["kernel_launches"],
                "ffts": c1["fft_execs"] - c0["fft_execs"]}

    def arm_steps(a):
        if a == "plain" and name == "precision_162k":
            return max(1, min(args.steps, 2))  # ~10 s per solve
        return args.steps

    # warm-up (untimed)
    for a in arms:
        timed(a, 1 if (a == "plain" and name == "precision_162k") else args.warmup)
    dev_id = str(local)
    try:
        dev_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(dev_id)
    torch.cuda.synchronize()
    ranks.barrier(world)
    clocks.start()
    results[head_arm] = timed(head_arm, args.steps)
    torch.cuda.synchronize()
    ranks.barrier(world)
    clk = clocks.stop()
    for a in arms:
        if a != head_arm:
            results[a] = timed(a, arm_steps(a))
            torch.cuda.synchronize()
            ranks.barrier(world)
    # per-kernel times: the headline steps again, uncaptured, under the in-library profiler
    prof_run = timed(head_arm, args.steps, profile=True)
    prof = prof_run["prof"]
    torch.cuda.synchronize()
    ranks.barrier(world)
    ms = {a: ranks.max_over_ranks(results[a]["ms"], world, device="cuda") for a in arms}

    # end to end through the public C ABI on host buffers (pinned), the headline arm
    hp = torch.from_numpy(s.pos.copy()).pin_memory()
    hb = torch.from_numpy(s.body_pos.copy()).pin_memory()
    hq = torch.zeros(s.n_beads, dtype=torch.float64).pin_memory()
    hphi = torch.zeros(s.n_bodies, dtype=torch.float64).pin_memory()
    hf = torch.zeros((s.n_beads, 3), dtype=torch.float64).pin_memory()
    e2e_s = []
    hh.compute_host(hp.numpy(), hb.numpy(), hq.numpy(), hphi.numpy(), hf.numpy())  # untimed: host staging
    for _ in range(args.steps):
        hq.zero_()
        hphi.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hh.compute_host(hp.numpy(), hb.numpy(), hq.numpy(), hphi.numpy(), hf.numpy())
        e2e_s.append(time.perf_counter() - t0)
    e2e_ms = ranks.max_over_ranks(1e3 * float(np.mean(e2e_s)), world, device="cuda")
    h2d = 8 * (3 * s.n_beads + 3 * s.n_bodies + s.n_beads + s.n_bodies)
    d2h = 8 * (s.n_beads + s.n_bodies + 3 * s.n_beads)

    # roofline of the dominant kernel class in the profiled headline steps
    prec_bytes = 4 if ARMS[head_arm][0] == "mixed" else 8
    geo = hh.geometry_info()
    G = int(np.prod([p["grid"]] * 3))
    # the roofline kernel: the costliest class with an algorithmic byte count (the Krylov
    # vector operations, preconditioners and body rows have none: their share is reported)
    dominant_class = max(prof, key=lambda k: prof[k]["ms"])
    dom = max((k for k in prof if k in ROOFLINE_CLASSES), key=lambda k: prof[k]["ms"])
    dom_ms = prof[dom]["ms"] / max(prof[dom]["launches"], 1)
    alg = algorithmic_bytes(dom, prec_bytes, s.n_beads, G, geo["real_space_pairs"], geo["cluster_pairs"])
    peak, peak_kind = load_peaks()
    achieved = alg / (dom_ms * 1e-3) / 1e9
    traffic = None
    tpath = ROOT / "profiles" / "ncu_traffic.json"
    if tpath.exists():
        try:
            traffic = json.loads(tpath.read_text()).get(name, {}).get(dom)
        except Exception:
            traffic = None
    total_prof_ms = sum(v["ms"] for v in prof.values())
    shares = {k: round(v["ms"] / total_prof_ms, 4) for k, v in prof.items() if total_prof_ms > 0}

    # errors of every arm's solution against the oracle (rank 0's system, full size only)
    errors = None
    if rank == 0 and args.scale == 1.0 and not args.no_oracle:
        ref = oracle_solution(name, s, p)
        errors = {"reference": ref["how"], "reference_oracle_residual": ref["residual"],
                  "bar": "max-norm error relative to the largest entry; target 1e-5 at residual 1e-6"}
        for a in arms:
            errors[a] = error_vs_oracle(ref, s, *results[a]["sol"])

    def arm_summary(a):
        st = results[a]["stats"][-1]
        d = {"value": ranks.job_throughput(1.0, ms[a], world), "ms_per_step": ms[a], "what": ARM_LABELS[a],
             "precision": ARMS[a][0], "preconditioner": ARMS[a][1] or args.precond,
             "restart": ARMS[a][2] or args.restart, "iterations": st["iterations"],
             "matvecs_fp64": st["matvecs_fp64"], "matvecs_fp32": st["matvecs_fp32"],
             "final_residual": st["final_residual"], "converged": st["converged"]}
        if errors is not None:
            d["error_vs_oracle"] = errors[a]
        return d

    st_h = results[head_arm]["stats"][-1]
    value = ranks.job_throughput(1.0, ms[head_arm], world)
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms[head_arm], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"mixed": "f32 operator / f64 Krylov", "fp64": "f64"}[ARMS[head_arm][0]],
        "data": "synthetic (seeded placement)",
        "config": {"workload": name, "charges": s.n_beads, "bodies": s.n_bodies, "mesh": p["grid"],
                   "support": p["support"], "rcut": p["rcut"], "xi": p["xi"], "tol": TOL,
                   "headline_arm": head_arm, "preconditioner": ARMS[head_arm][1] or args.precond,
                   "restart": ARMS[head_arm][2] or args.restart,
                   "learned": (bool(args.learned) if head_arm == "fast" else False),
                   "learned_note": "n/a for a single static solve: the learned start needs a previous solution "
                                   "(time stepping, dynamics_420k workload)",
                   "mesh_tiling": tiling, "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MB write) before every step"},
        "arms": {a: arm_summary(a) for a in arms},
        "solve": {"iterations": st_h["iterations"], "refinements": st_h["refinements"],
                  "coarse_level": hh.coarse_info() if (ARMS[head_arm][1] or args.precond) == "two_level" else None,
                  "matvecs_fp32": st_h["matvecs_fp32"], "matvecs_fp64": st_h["matvecs_fp64"],
                  "final_residual": st_h["final_residual"]},
        "error_vs_oracle": errors[head_arm] if errors is not None else None,
        "kernel_share": shares,
        "dominant_class": dominant_class,
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "launches": prof[dom]["launches"], "avg_launch_ms": dom_ms,
                     "measured_over": "a profiled pass of the same steps right after the timed region "
                                      f"(uncaptured, {prof_run['ms']:.1f} ms per step): captured graph steps "
                                      "cannot be timed per kernel",
                     "algorithmic_bytes_per_launch": alg},
        "e2e": {"value": world * 1e3 / e2e_ms, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(results[head_arm]["launches"]),
        "captured_arnoldi_steps": hh.graph_launches(),
        "cufft_execs": int(results[head_arm]["ffts"]),
        "clocks": clk,
    }
    if "plain" in arms and head_arm != "plain":
        line["speedup_vs_plain_fp64"] = ms["plain"] / ms[head_arm]
    if "f64t" in arms and head_arm == "fast":
        line["precision_only_speedup"] = ms["f64t"] / ms["fast"]  # same preconditioner, FP64 vs mixed
    if "spread" in prof and prof["spread"]["launches"]:
        sp_ms = prof["spread"]["ms"] / prof["spread"]["launches"]
        sp_alg = algorithmic_bytes("spread", prec_bytes, s.n_beads, G, 0)
        line["spread"] = {"achieved_gbs": sp_alg / (sp_ms * 1e-3) / 1e9, "avg_launch_ms": sp_ms,
                          "frac": sp_alg / (sp_ms * 1e-3) / 1e9 / peak}
    # spread and contract are bound by instruction issue and shared memory, not HBM: their
    # work rate is N P^3 weighted node updates per launch
    updates = float(s.n_beads) * p["support"] ** 3
    for k in ("spread", "contract"):
        if k in prof and prof[k]["launches"]:
            ms_k = prof[k]["ms"] / prof[k]["launches"]
            line.setdefault(k, {"avg_launch_ms": ms_k})["weighted_updates_per_s"] = updates / (ms_k * 1e-3)
    if rank == 0 and world == 1 and not args.no_cpu and args.scale == 1.0:
        if name == "plain_small":
            line["cpu_baseline"] = cpu_full_solve(s, p)
        else:
            it_plain = results["plain"]["stats"][-1]["iterations"] if "plain" in arms else ITERATIONS_PLAIN_FP64[name]
            line["cpu_baseline"] = cpu_gmres_sample(s, p, it_plain, cycles=2)
    if rank == 0:
        print(json.dumps(line), flush=True)
    for h in handles.values():
        h.close()
    if world > 1:
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-oracle", action="store_true", help="skip the errors against the oracle's solution")
    ap.add_argument("--learned", type=int, default=0)
    ap.add_argument("--op-case", type=float, default=0.0,
                    help="profiling case: the workload scaled to this body fraction, --steps operator "
                         "applications in FP32 (small enough for a full ncu capture)")
    ap.add_argument("--arms", default="fast,f64t,f64c,plain",
                    help="arms to run besides the headline one: fast (FP32 operator), f64t (FP64, same "
                         "preconditioner), f64c (FP64, conductor response), plain (FP64, reference preconditioner); "
                         "replicas_256: 'lockstep' runs the lockstep arm alone (no looped or stream-batch arm)")
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=[WORKLOAD, "plain_small", "replicas_256", "dynamics_420k", "mlp", "polydisperse_204k"],
                    help="headline solve (default), the small plain-method system, 256 batched replicas, Brownian "
                         "dynamics, the network kernels, or the charged polydisperse mixture")
    ap.add_argument("--scale", type=float, default=1.0, help="body-count fraction (dynamics; headline profiling cases)")
    ap.add_argument("--tiling", default="", help="T,MODE: fixed mesh tiling of the headline solver instead of "
                                                 "cr_autotune (for runs under a profiler)")
    ap.add_argument("--restart", type=int, default=RESTART, help="FGMRES restart of the headline (fast) arm")
    ap.add_argument("--precond", default=None, choices=["two_level", "conductor"],
                    help="preconditioner of the fast arm (default: two_level; conductor for the polydisperse "
                         "mixture and the dynamics)")
    ap.add_argument("--coarse-max-dense", type=int, default=12288,
                    help="coarse problems above this many unknowns use the sparse form (--coarse-cg steps of CG on "
                         "near-pair blocks + the low-rank wave term) or, with --coarse-cg 0, no coarse level")
    ap.add_argument("--coarse-cg", type=int, default=0, help="CG steps of the sparse coarse form")
    ap.add_argument("--realspace", type=int, default=0,
                    help="real-space kernel values evaluated on the fly: 1 FP32, 2 FP64, 3 both; 4: stored values "
                         "streamed through shared memory; 8: real-space product after the wave-space part instead of beside it "
                         "(default 0: stored, read by one CTA per cluster, concurrent with the wave-space part)")
    ap.add_argument("--batch-threads", type=int, default=16,
                    help="replicas: host threads (one stream each) of the batched solve")
    ap.add_argument("--train-solves", type=int, default=0,
                    help="dynamics: solves the networks are trained on (default min(200, steps/2))")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.precond is None:
        args.precond = "conductor" if args.workload in ("polydisperse_204k", "dynamics_420k") else "two_level"
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "replicas_256":
        run_replicas(args)
    elif args.workload == "dynamics_420k":
        run_dynamics(args)
    elif args.workload == "mlp":
        run_mlp(args)
    elif args.workload == "polydisperse_204k":
        run_polydisperse(args)
    elif args.op_case > 0:
        run_op_case(args)
    else:
        run_solve(args)


if __name__ == "__main__":
    main()
