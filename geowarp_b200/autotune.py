"""Launch-shape autotuner.

The library's launch shapes and the depth of its multigrid hierarchy are
process-wide knobs (gw_tune_set): the CTA size of the assembly and of the
adjoint particle kernels, the warps per CTA of the multigrid row kernels, the
bound of the dense coarsest level.  Which values are fastest depends on
the workload (particle count, material, grid) and on the device, so the
tuner measures them there: a coordinate search over the knobs, each candidate
timed with CUDA events on a caller-supplied trial that repeats the same unit
of work (one load step, forward + adjoint, from a restored particle state).
The first call of every candidate is untimed: it rebuilds the step graphs the
knob invalidates.
"""
import json
import os
import statistics

from . import _lib as L

# knob name -> (gw_tune_set id, candidates searched).  The multigrid smoother
# knobs (GW_TUNE_MG_SWEEPS / _OMEGA / _ONE_SWEEP) are not searched: on the
# workloads here two sweeps at 0.7 on every level were fastest, and damping of
# 0.8 and above makes the block-Jacobi smoother diverge (GMRES then runs to
# its iteration cap).  GW_TUNE_MG_TAIL is not searched either: the fused tail
# measured slower on every workload, and it runs only in FP64 solves, so a
# value picked on a mixed-precision trial would be noise.
KNOBS = {
    "row_warps": (L.TUNE_ROW_WARPS, (2, 4, 8, 16)),
    "mg_coarse": (L.TUNE_MG_COARSE, (40, 80, 160)),
    "particle_block": (L.TUNE_PARTICLE_BLOCK, (64, 128, 256)),
    "adjoint_block": (L.TUNE_ADJOINT_BLOCK, (64, 128, 256)),
}
STATE = ("x", "lp", "F_old", "b_old", "pi_old", "pi_new", "sigma", "pressure")


def current(knobs=KNOBS):
    lib = L.load()
    return {name: int(lib.gw_tune_get(k)) for name, (k, _) in knobs.items()}


def apply(config, knobs=KNOBS):
    """Set the knobs named in config (unknown names are ignored)."""
    for name, value in config.items():
        if name in knobs:
            L.call("gw_tune_set", knobs[name][0], int(value))


def snapshot(engine):
    """Copies of the particle state a load step reads and writes, and of the
    engine's Newton predictor (the previous converged increment and its load
    step), which decides the step's starting iterate."""
    snap = {n: getattr(engine, n).clone() for n in STATE if getattr(engine, n, None) is not None}
    u_prev = getattr(engine, "_u_prev", None)
    snap["_predictor"] = (None if u_prev is None else u_prev.clone(), getattr(engine, "_u_prev_step", None))
    return snap


def restore(engine, snap):
    for n, t in snap.items():
        if n == "_predictor":
            u_prev, step = t
            engine._u_prev = None if u_prev is None else u_prev.clone()
            engine._u_prev_step = step
        else:
            getattr(engine, n).copy_(t)


def cuda_timer(fn):
    """Milliseconds of fn() between CUDA events on the current stream."""
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def tune(trial, reps=3, knobs=KNOBS, timer=cuda_timer, log=None):
    """Coordinate search: for each knob in turn, every candidate is set (the
    other knobs at their best so far), trial() runs once untimed and then reps
    times under timer; the candidate with the smallest median stays set.
    Returns (best config, {knob: {candidate: median ms}})."""
    import time
    best = current(knobs)
    table = {}
    best_ms = None
    for name, (k, cands) in knobs.items():
        times = {}
        for v in cands:
            L.call("gw_tune_set", k, int(v))
            t0 = time.perf_counter()
            trial()
            first_ms = 1e3 * (time.perf_counter() - t0)
            if best_ms is not None and first_ms > 4.0 * best_ms + 50.0:
                times[v] = first_ms  # far slower already untimed: not repeated
            else:
                times[v] = statistics.median(timer(trial) for _ in range(reps))
                best_ms = times[v] if best_ms is None else min(best_ms, times[v])
            if log:
                log(f"autotune {name}={v}: {times[v]:.3f} ms")
        pick = min(times, key=times.get)
        L.call("gw_tune_set", k, int(pick))
        best[name] = pick
        table[name] = times
    return best, table


def device_key():
    """The device the tuned values belong to (name and SM count)."""
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name} ({p.multi_processor_count} SMs)"


def save(path, workload, config, table):
    data = json.load(open(path)) if os.path.exists(path) else {}
    data.setdefault(device_key(), {})[workload] = {"config": config,
                                                  "table": {k: {str(c): v for c, v in t.items()}
                                                            for k, t in table.items()}}
    with open(path, "w") as f:
        json.dump(data, f, indent=1)


def load(path, workload):
    """The saved config for this device and workload, or None."""
    if not os.path.exists(path):
        return None
    entry = json.load(open(path)).get(device_key(), {}).get(workload)
    return entry["config"] if entry else None
