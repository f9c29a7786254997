"""Benchmark: block load steps/s (forward + adjoint) of the implicit cpGIMP
engine on the batched inverse analysis: 64 self-weight soil blocks of
32x32..128x64 cells (seeded), 2 x 2 particles per cell (1,002,044 particles),
per-particle log Young's modulus from a Gaussian random field, packed into
one engine; the loss is the L2 misfit to the displacements a second field
produces, and every step also runs the hand-written adjoint of the load step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl geowarp|reference]

One "step" is one load step of all 64 blocks: P2G (cell sort, activation,
pattern), the Newton loop (residual + exact element tangent, GMRES on the
block-CSR Jacobian) and G2P, followed by its adjoint (transpose solve with the
converged Jacobian and the adjoint P2G/G2P), in the mixed FP32/FP64 mode.  The
plain FP64 engine runs the same steps for the error check and is reported
beside it.  With N GPUs the job runs N independent replicas (one per rank;
there is no data-path collective) and `value` is the aggregate over ranks.

--workload footing runs the plane-strain Drucker-Prager strip footing (256 x
128 cells, 131,072 particles); --workload consolidation runs the 1 x 200-cell
coupled u-p column (forward load steps with their own time increments; the
adjoint covers the 2D solid solver); --workload bar runs the 4 x 40-cell
self-weight bar.

Before the timed region, --autotune on (the default) searches the library's
launch-shape knobs on the workload's own load step (geowarp_b200.autotune); the
chosen values apply to every arm and are reported in the line.

--impl reference times the CPU restatement of the reference's algorithm (the
reference itself runs only on NVIDIA Warp, not installable here) on a bounded
sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "load steps/s (fwd+adjoint), mixed vs plain FP64 on same B200 at rel err<=1e-6"
WORKLOAD = dict(workload="2D plane-strain rigid strip footing on Drucker-Prager soil",
                cells="256x128 soil cells (260x132 grid), dx=0.05 m", particles=131072, ppc="2x2",
                material="DP E=2e7 Pa nu=0.3 c=10 kPa phi=30 psi=0",
                soil="self-weight rho=2000 kg/m3 g=9.81 from a K0=0.5 geostatic start",
                footing="1 m wide, 0.2 m over 100 steps")
N_STEPS_TOTAL = 100


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="geowarp", choices=["geowarp", "reference"])
    ap.add_argument("--small", action="store_true", help="64x32-cell variant for quick checks")
    ap.add_argument("--workload", default="batched", choices=["footing", "batched", "consolidation", "bar"],
                    help="batched: 64 inverse-analysis blocks in one engine (default); footing: the strip footing; "
                         "consolidation: the 1 x 200-cell u-p column (forward load steps); bar: the 4 x 40-cell "
                         "self-weight bar")
    ap.add_argument("--instances", type=int, default=64, help="blocks of the batched workload")
    ap.add_argument("--profile", action="store_true", help="also time the dominant kernel (instrumented pass)")
    ap.add_argument("--autotune", default="on", choices=["on", "off"],
                    help="search the library's launch-shape knobs on this workload before timing (untimed)")
    ap.add_argument("--ncu", action="store_true",
                    help="run warmup + steps load steps (fwd+adjoint, mixed) with no timing: the command profiled by ncu")
    return ap.parse_args()


def footing_kwargs(small):
    return dict(n_cells_x=64, n_cells_y=32, footing_width=0.25) if small else {}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed
    region: sampling starts (and its first row is awaited) before the region,
    every row carries its timestamp, and only rows inside [mark_start,
    mark_end] are summarised (the nearest row when the region is shorter than
    the sampling interval, flagged as such)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 25

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        if self.proc is not None:
            deadline = time.time() + 5.0
            while time.time() < deadline and not os.path.getsize(self.f.name):
                time.sleep(0.02)
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(2.0 * self.PERIOD_MS / 1e3)  # let the row that covers the end arrive

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    @staticmethod
    def _when(stamp):
        import datetime
        try:
            return datetime.datetime.strptime(stamp.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.f.name).read().strip().split("\n") if l.strip()]
        except OSError:
            rows = []
        os.unlink(self.f.name)
        rows = [r for r in rows if len(r) >= 10]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        timed = [(self._when(r[0]), r) for r in rows]
        note = None
        if self.t0 is not None and self.t1 is not None and all(t is not None for t, _ in timed):
            inside = [r for t, r in timed if self.t0 <= t <= self.t1]
            if not inside:
                mid = 0.5 * (self.t0 + self.t1)
                inside = [min(timed, key=lambda tr: abs(tr[0] - mid))[1]]
                note = "timed region shorter than the sampling interval: nearest sample"
            rows = inside
        sm = [float(r[2]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[6:10]):
                if v.strip() == "Active":
                    reasons.add(name)
        out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][3]), "reasons": sorted(reasons),
               "samples": len(rows), "period_ms": self.PERIOD_MS}
        if note:
            out["note"] = note
        return out


# ------------------------------------------------------------------ workloads
class Workload:
    """A timed unit: step(adj, k) runs load step k forward (checkpointed) and
    then its adjoint seeded by the workload's misfit."""
    adjoint = True

    def step(self, adj, k):
        adj.forward_step(k, self.n_steps, keep=False)
        self.seed(adj, k)
        adj.backward_step()


class FootingWorkload(Workload):
    """The strip footing: one instance per load step."""

    def __init__(self, args):
        self.fk = footing_kwargs(args.small)
        self.units = 1
        self.n_steps = N_STEPS_TOTAL
        self.config = dict(WORKLOAD)
        self.metric = METRIC

    def make(self, precision, dev):
        from geowarp_b200 import problems
        from geowarp_b200.adjoint import LoadStepAdjoint
        s = problems.strip_footing_2d(precision=precision, device=dev, **self.fk)
        return s, LoadStepAdjoint(s)

    def seed(self, adj, k):
        adj.seed_displacement_misfit()

    def errors(self, s_mx, s_64):
        return {"footing_force": abs(s_mx.footing_force - s_64.footing_force) / abs(s_64.footing_force)}


class BatchedWorkload(Workload):
    """Batched inverse analysis: n self-weight blocks (cell counts seeded
    uniformly in 32x32..128x64, per-particle log E a Gaussian random field)
    in one engine; each load step is forward + adjoint of the summed
    displacement misfit to targets made by a second field."""

    def __init__(self, args):
        from geowarp_b200 import batch
        self.n = args.instances
        self.sizes = batch.instance_sizes(self.n, seed=0)
        self.logE = batch.random_fields(self.sizes, seed=1000)
        self.logE_target = batch.random_fields(self.sizes, seed=2000)
        self.units = self.n
        self.n_steps = N_STEPS_TOTAL
        self.targets = None
        npart = sum(a * b * 4 for a, b in self.sizes)
        self.config = dict(workload=f"batched inverse analysis: {self.n} self-weight blocks in one engine",
                           cells="per block uniform (seed 0) in 32x32..128x64, dx=0.05 m, shelf-packed with 4 empty "
                                 "cells between blocks", particles=npart, ppc="2x2",
                           material="Hencky elastic, nu=0.3, log E = Gaussian random field (mean ln 1e7, std 0.3, "
                                    "correlation length 0.5 m, seeds 1000+q); targets from a second field (seeds 2000+q)",
                           load=f"self-weight rho=2000 kg/m3 g=9.81 ramped over {N_STEPS_TOTAL} load steps",
                           units="value counts block load steps (blocks x load steps)")
        self.metric = METRIC.replace("load steps/s", "block load steps/s")

    def make(self, precision, dev):
        from geowarp_b200.adjoint import LoadStepAdjoint
        from geowarp_b200.batch import BatchedBlocks
        bb = BatchedBlocks(self.sizes, logE=self.logE, precision=precision, device=dev)
        return bb.solver, LoadStepAdjoint(bb.solver)

    def prepare(self, n_steps_run, dev):
        """Target displacement after each load step, from the target field."""
        import torch
        from geowarp_b200.batch import BatchedBlocks
        bt = BatchedBlocks(self.sizes, logE=self.logE_target, precision="fp64", device=dev)
        self.targets = []
        for k in range(n_steps_run):
            bt.solver.advance_one_step(k, self.n_steps)
            self.targets.append(bt.displacement().clone())
        del bt
        torch.cuda.empty_cache()

    def seed(self, adj, k):
        # without prepared targets (the ncu target run) the misfit is to zero
        # displacement: the adjoint does the same work
        adj.seed_displacement_misfit(self.targets[k] if self.targets else None)

    def errors(self, s_mx, s_64):
        return {}


class BarWorkload(Workload):
    """Self-weight bar: 4 x 40 cells of 0.25 m, 2 x 2 particles per cell,
    compressible neo-Hookean; forward + adjoint load steps."""

    def __init__(self, args):
        self.units = 1
        self.n_steps = 50
        self.config = dict(workload="2D quasi-static bar compaction under self-weight",
                           cells="4x40 cells (8x44 grid), dx=0.25 m", particles=640, ppc="2x2",
                           material="compressible neo-Hookean E=1e6 Pa nu=0.3 rho=80 kg/m3",
                           load="gravity 9.81 ramped over 50 load steps; roller side walls, fixed base",
                           newton="||R|| < 1e-6 N (1e-8 of one step's load increment)")
        self.metric = METRIC

    def make(self, precision, dev):
        from geowarp_b200 import problems
        from geowarp_b200.adjoint import LoadStepAdjoint
        s = problems.bar_compaction_2d(precision=precision, device=dev)
        return s, LoadStepAdjoint(s)

    def seed(self, adj, k):
        adj.seed_displacement_misfit()

    def errors(self, s_mx, s_64):
        return {}


class ConsolidationStepper:
    """Forward load steps of the consolidation column, each with its own time
    increment."""

    def __init__(self, solver, dts):
        self.solver, self.dts = solver, dts

    def forward_step(self, k, n_steps, keep=False):
        self.solver.dt = float(self.dts[k])
        self.solver.advance_one_step(k, n_steps)


class ConsolidationWorkload(Workload):
    """Coupled u-p 1D consolidation: 1 x 200 cells of 0.05 m, 2 x 2 particles
    per cell, linear elastic skeleton; forward load steps only (the
    hand-written adjoint covers the 2D solid solver)."""
    adjoint = False

    def __init__(self, args):
        from geowarp_b200 import problems
        self.dicts = problems.consolidation_column_dicts()
        self.dts = self.dicts[6]
        self.units = 1
        self.n_steps = len(self.dts)
        self.config = dict(workload="2D coupled u-p 1D consolidation column",
                           cells="1x200 cells (6x202 grid), dx=0.05 m", particles=800, ppc="2x2",
                           material="linear elastic skeleton E=1e7 Pa nu=0.3; permeability 1e-10 m2, fluid viscosity "
                                    "1e-3 Pa.s (mobility 1e-7), porosity 0.4",
                           load="10 kPa surface traction, drained top, undrained fixed base, roller sides",
                           time_steps="200 geometrically growing increments from mesh Fourier number cv dt/dx^2 = 4 "
                                      "to a Terzaghi time factor of 2",
                           solver="flexible GMRES(30) + multigrid V-cycle with Schur-diagonal pressure smoother")
        self.metric = "load steps/s (forward; u-p), mixed vs plain FP64 on same B200"

    def make(self, precision, dev):
        from geowarp_b200 import problems
        s, dts, cv, H = problems.consolidation_column_2d(precision=precision, device=dev)
        return s, ConsolidationStepper(s, dts)

    def step(self, adj, k):
        adj.forward_step(k, self.n_steps)

    def errors(self, s_mx, s_64):
        q = 1e4
        return {"pore_pressure_over_load": float((s_mx.particle_pressure_array - s_64.particle_pressure_array)
                                                 .abs().max() / q)}


def make_workload(args):
    if args.workload == "batched":
        return BatchedWorkload(args)
    if args.workload == "consolidation":
        return ConsolidationWorkload(args)
    if args.workload == "bar":
        return BarWorkload(args)
    return FootingWorkload(args)


# ------------------------------------------------------------------ GPU arm
def run_geowarp(args):
    import torch
    from geowarp_b200 import _lib as L
    from geowarp_b200.replicas import Replicas, aggregate_rate

    rep = Replicas("nccl")  # one independent replica per GPU (no data-path collective)
    world, rank = rep.world, rep.rank
    dev = torch.device("cuda", torch.cuda.current_device())
    wl = make_workload(args)
    W, K = args.warmup, args.steps
    if W + K + 1 > wl.n_steps:
        raise SystemExit(f"--warmup + --steps + 1 (the instrumented step) must not exceed the workload's "
                         f"{wl.n_steps} load steps")
    if hasattr(wl, "prepare"):
        wl.prepare(W + K + 1, dev)
    lib = L.load()
    # written between timed load steps: evicts the 126 MB L2 (256 MB memset, ~0.05 ms)
    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def sync():
        torch.cuda.synchronize(dev)
        rep.barrier()

    def one_step(adj, k):
        # forward load step (checkpointed), then (where the workload has one)
        # its adjoint seeded with the displacement misfit
        wl.step(adj, k)

    # ---- mixed precision, resident (value)
    s_mx, adj_mx = wl.make("mixed", dev)
    for k in range(W):
        one_step(adj_mx, k)
    sync()
    tuned = autotune_workload(wl, s_mx, adj_mx, W) if args.autotune == "on" else None
    sync()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as cs:
        sync()
        n_launch0 = lib.gw_launch_count()
        cs.mark_start()
        ev0.record()
        for k in range(W, W + K):
            l2_flush.zero_()
            one_step(adj_mx, k)
        ev1.record()
        sync()
        cs.mark_end()
        launches = lib.gw_launch_count() - n_launch0
    ms_mx = ev0.elapsed_time(ev1)
    clocks = cs.summary()

    # ---- plain FP64 on the same steps (error reference and its own throughput)
    s_64, adj_64 = wl.make("fp64", dev)
    for k in range(W):
        one_step(adj_64, k)
    sync()
    ev0.record()
    for k in range(W, W + K):
        l2_flush.zero_()
        one_step(adj_64, k)
    ev1.record()
    sync()
    ms_64 = ev0.elapsed_time(ev1)
    disp_mx = (s_mx.x_particles - s_mx.x0)
    disp_64 = (s_64.x_particles - s_64.x0)
    errs = {"displacement": float((disp_mx - disp_64).abs().max() / disp_64.abs().max()),
            "cauchy_stress": float((s_mx.particle_Cauchy_stress_array - s_64.particle_Cauchy_stress_array).abs().max()
                                   / s_64.particle_Cauchy_stress_array.abs().max())}
    errs.update(wl.errors(s_mx, s_64))
    if wl.adjoint:
        errs["grad_E"] = float((adj_mx.grad_E - adj_64.grad_E).abs().max()
                               / adj_64.grad_E.abs().max().clamp_min(1e-300))
    errs["norm"] = "max-abs difference / max-abs FP64 value"
    newton = {"mixed_iters": newton_stats(s_mx.engine), "fp64_iters": newton_stats(s_64.engine)}
    del s_64, adj_64
    torch.cuda.empty_cache()

    # ---- end to end through the public API with the particle state held on the
    # host: every step copies the state in (pinned H2D), runs the load step and
    # its adjoint, and copies the new state, the stress and the gradient out
    s_e2e, adj_e2e = wl.make("mixed", dev)
    e = s_e2e.engine
    state = ("x", "F_old", "b_old", "lp")
    for k in range(W):
        one_step(adj_e2e, k)
    host = {name: torch.empty_like(getattr(e, name), device="cpu").pin_memory() for name in state}
    for name in state:
        host[name].copy_(getattr(e, name))
    sigma_host = torch.empty_like(e.sigma, device="cpu").pin_memory()
    # the step's result: the gradient (fwd+adjoint workloads) or the particle
    # pore pressure (forward u-p workloads)
    out_dev = (lambda: adj_e2e.grad_E) if wl.adjoint else (lambda: e.pressure)
    grad_host = torch.empty(e.N, dtype=torch.float64).pin_memory()
    sync()
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    d2h = h2d + sigma_host.numel() * 8 + grad_host.numel() * 8
    ev0.record()
    for k in range(W, W + K):
        l2_flush.zero_()
        for name in state:
            getattr(e, name).copy_(host[name], non_blocking=True)
        one_step(adj_e2e, k)
        for name in state:
            host[name].copy_(getattr(e, name), non_blocking=True)
        sigma_host.copy_(e.sigma, non_blocking=True)
        grad_host.copy_(out_dev(), non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
    ev1.record()
    sync()
    ms_e2e = ev0.elapsed_time(ev1)
    del s_e2e, adj_e2e
    torch.cuda.empty_cache()

    # ---- dominant kernel, instrumented pass on one more step (not part of value)
    roof = roofline_pass(adj_mx, W + K, wl)

    ms_mx, ms_64, ms_e2e = rep.max_over_ranks([ms_mx, ms_64, ms_e2e], device=dev)
    if rank == 0:
        units = K * world * wl.units
        line = {
            "metric": wl.metric, "value": aggregate_rate([K * wl.units] * world, ms_mx),
            "unit": wl.metric.split(" (")[0],
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms_mx / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic",
            "config": dict(wl.config, parallelism=f"replicas x{world}", global_batch=world * wl.units, seq_len=None,
                           timed_load_steps=f"{W}..{W + K - 1} of {wl.n_steps} (after {W} warm-up steps)",
                           l2="a 256 MB buffer is written before every timed load step (L2 flush, inside the "
                              "timed region)",
                           small=bool(args.small)),
            "plain_fp64": {"value": units / (ms_64 / 1e3), "ms_per_step": ms_64 / K},
            "mixed_over_fp64": ms_64 / ms_mx,
            "rel_err_vs_fp64": errs,
            "e2e": {"value": units / (ms_e2e / 1e3), "unit": wl.metric.split(" (")[0], "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "newton": newton,
            "roofline": roof,
            "clocks": clocks,
            "autotune": tuned,
        }
        line["cpu_baseline"] = cpu_baseline(wl, line)
        print(json.dumps(line))
    rep.close()


def autotune_workload(wl, solver, adj, k):
    """Search the launch-shape knobs (geowarp_b200.autotune) on load step k of
    this workload: every trial restores the particle and adjoint state taken
    after the warm-up and runs the same step, so all candidates do the same
    work.  The state and the Newton log are restored afterwards; the chosen
    knobs stay set for every timed arm."""
    from geowarp_b200 import autotune
    e = solver.engine
    snap = autotune.snapshot(e)
    adj_t = []
    if getattr(adj, "grad_E", None) is not None:
        adj_t = [adj.grad_E] + list(adj.bar.values()) + list(adj.q.values())
    adj_snap = [t.clone() for t in adj_t]
    n_log = len(e.log)

    def reset():
        autotune.restore(e, snap)
        for t, c in zip(adj_t, adj_snap):
            t.copy_(c)

    def trial():
        reset()
        wl.step(adj, k)

    best, table = autotune.tune(trial, reps=2)
    reset()
    del e.log[n_log:]
    return {"config": best, "median_ms": {n: {str(c): round(v, 3) for c, v in t.items()} for n, t in table.items()},
            "trial": f"load step {k} ({'forward + adjoint' if wl.adjoint else 'forward'}) from a restored state; "
                     "median of 2 after an untimed call; coordinate search in the listed order"}


def newton_stats(engine):
    steps = {}
    kry = []
    for (step, it, nrm, kit, relres, rc) in engine.log:
        if rc == "backtrack":
            continue
        steps[step] = steps.get(step, 0) + 1
        kry.append(kit)
    return {"mean_newton_per_step": float(np.mean(list(steps.values()))) if steps else None,
            "mean_krylov_per_newton": float(np.mean(kry)) if kry else None}


def roofline_pass(adj, k, wl):
    """Time the dominant kernel family with CUDA events inside one more step."""
    import json as _json
    from geowarp_b200 import profiling
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = _json.load(open(path)) if os.path.exists(path) else {"hbm_gbs": 6650.0}
    with profiling.kernel_timer() as kt:
        wl.step(adj, k)
    return profiling.roofline_summary(kt, peaks, peak_kind="measured" if "when" in peaks else "fallback")


def host_threads():
    """Host cores this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def oracle_rate(wl, steps=2, budget_s=15.0):
    """The oracle (CPU restatement of the reference's algorithm) on a bounded
    sample of the workload, with every host core on the tangent's
    complex-step passes: (load steps per second in the workload's unit,
    threads, description)."""
    # the tangent of a 2D step is 9 nodes x nf complex-step passes: more
    # threads than passes would sit idle, and are not counted
    nf = 3 if isinstance(wl, ConsolidationWorkload) else 2
    th = max(1, min(host_threads(), 9 * nf))
    if isinstance(wl, ConsolidationWorkload):
        from oracle.bench_sample import oracle_consolidation_sample
        sec, n, sample = oracle_consolidation_sample(wl.dicts[:6], wl.dts, max_steps=max(steps, 3),
                                                     budget_s=budget_s, threads=th)
        return 1.0 / sec, th, sample
    if isinstance(wl, BarWorkload):
        from oracle.bench_sample import oracle_bar_sample
        sec, n, sample = oracle_bar_sample(wl.n_steps, max_steps=max(steps, 3), budget_s=budget_s, threads=th)
        return 1.0 / sec, th, sample + " (forward load steps; the CPU path has no adjoint)"
    if isinstance(wl, BatchedWorkload):
        # whole blocks of the batch, each a complete load step: the blocks are
        # independent, so blocks per second is the metric's own unit.  Its
        # per-particle work runs compiled (oracle/native.py), threads over
        # particles, so every host core counts.
        from oracle import native
        from oracle.bench_sample import oracle_batch_sample
        if native.load() is not None:
            th = host_threads()
        rate, n, sample = oracle_batch_sample(wl.sizes, wl.logE, wl.n_steps, budget_s=budget_s, threads=th)
        return rate, th, sample
    from oracle.bench_sample import oracle_load_step_sample
    times = []
    for k in range(max(1, min(steps, 2))):
        sec, its, sample = oracle_load_step_sample(step=k, threads=th)
        times.append(sec)
    return wl.units / float(np.mean(times)), th, sample + " (forward load step; the CPU path has no adjoint)"


def cpu_baseline(wl, gpu_line):
    """Oracle timing on a bounded sample of the same workload, run on rank 0:
    whole blocks of the batch (one load step each), the first load steps of
    the bar / column, or one load step of the 64x32-cell footing variant
    scaled to the full footing."""
    v, th, sample = oracle_rate(wl, steps=1, budget_s=20.0)
    return {"value": v, "unit": gpu_line["unit"], "cores": th, "kind": "port", "sample": sample}


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    """The reference's algorithm on the host cores: the CPU restatement (the
    reference itself needs NVIDIA Warp, which is not installable here) with
    every host core on its tangent passes, on a bounded sample of the
    workload.  Rank 0 only."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = make_workload(args)
    v, th, sample = oracle_rate(wl, steps=args.steps, budget_s=60.0)
    unit = wl.metric.split(" (")[0]
    print(json.dumps({
        "impl": "reference", "metric": wl.metric, "value": v, "unit": unit, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "dtype": "f64", "data": "synthetic", "config": dict(wl.config, parallelism=f"host cores x{th}"),
        "cpu_baseline": {"value": v, "unit": unit, "cores": th, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ncu_target(args):
    """warmup + steps load steps (forward + adjoint, mixed) with no timing and
    no target run, so the first launches of each kernel are the profiled arm's."""
    import torch
    wl = make_workload(args)
    s, adj = wl.make("mixed", torch.device("cuda"))
    for k in range(args.warmup + args.steps):
        wl.step(adj, k)
    torch.cuda.synchronize()
    print("ncu target done", len(s.engine.log), "Newton iterations")


if __name__ == "__main__":
    a = parse()
    if a.ncu:
        run_ncu_target(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_geowarp(a)
