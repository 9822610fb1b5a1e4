"""Benchmark of the DFSPH time step on B200 (one JSON line on rank 0).

Workload (default, --config 3): the 1,000,000-particle sloshing tank (100^3 lattice, r = 0.01 m,
8 x 4 x 4 m box, 400,002 wall particles translating rigidly as x = 0.1 sin(2 pi t / 2) m, CFL 0.4
with dt_max 5 ms, density tolerance 0.01 %, divergence 0.1 %), synthetic seeded input. A step is
one DFSPHCUDA::step() equivalent: the walls' rigid motion (on the device), neighbour search,
divergence solve, XSPH + gravity, CFL dt, pressure solve, position update. `value` is the plain
(reference) warm start; the learned-vs-plain comparison of the metric runs the same workload and the
2,000,000-particle column collapse (0.005 %, dt_max 8 ms) in every mode, and the stiff resting
column where the solver needs many iterations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config 1..5]

With N > 1 (torchrun) every rank runs an independent replica of the workload (one B200 holds the
largest configuration, so the step is not sharded across GPUs) and the reported ms/step is the
maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DFSPH ms/step & solver iters at rho-err<=0.01%, learned vs plain, 1 B200"
UNIT = "ms/step"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons through NVML every few milliseconds while
    the timed region runs. Read-only (never changes a clock or a setting)."""

    def __init__(self, device: int, period_s: float = 0.002):
        self.device = device
        self.period = period_s
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self._nvml = (pynvml, h)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self._sample()
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()
        except Exception:
            self._nvml = None
        return self

    def _sample(self):
        pynvml, h = self._nvml
        self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
        names = {pynvml.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                 pynvml.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                 pynvml.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                 pynvml.nvmlClocksEventReasonSwPowerCap: "sw_power_cap",
                 pynvml.nvmlClocksEventReasonHwPowerBrakeSlowdown: "hw_power_brake_slowdown"}
        for bit, name in names.items():
            if r & bit:
                self.reasons.add(name)

    def _loop(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                break
            time.sleep(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=2)
        if self._nvml:
            try:
                self._sample()
                self._nvml[0].nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "nvml"}


def make_workload(config: int):
    """(scene, wall motion or None) of benchmark configuration `config`. The sloshing tank's walls
    move rigidly (sloshing_wall_motion); motion(d, t) applies their state at simulated time t."""
    from splishsplash_for_cuda_b200.scene import sloshing_wall_motion, synthetic_scene

    scene = synthetic_scene(config, cfl=True)
    if config != 3:
        return scene, None

    def motion(d, t):
        p, v = sloshing_wall_motion(t)
        d.move_boundary_rigid(0, scene.n_boundary, None, p, v, None)

    return scene, motion


def make_scene(config: int):
    return make_workload(config)[0]


# Algorithmic bytes per launch of each kernel (FP32 layout: float4 pos+mass, float4 vel, 4-byte
# scalars, 4-byte neighbour indices, one packed 4-byte count word). Each particle's own data is
# counted once per launch, neighbour data is other particles' own data (perfect reuse), and every
# stored neighbour costs its 4-byte index. nf / nb are the mean fluid / boundary neighbour counts.
def kernel_bytes(name: str, n: int, nb_particles: int, nf: float, nb: float, real: int = 4) -> float:
    """Algorithmic bytes of one launch: every per-particle array read or written once, the neighbour
    lists once, the boundary positions once. real = 4 (FP32 build) or 8 (FP64 build): a position,
    velocity or acceleration record is 4 reals, a scalar field one real; counts and list entries
    are 4 bytes."""
    nn = nf + nb
    v, r = 4 * real, real
    per = {
        "density_alpha": v + v + 4 + r + r + r + r + r + 4 * nn,        # pos, vel, counts, kv r/w, rho, alpha, dadv
        "divergence_jacobi": v + r + 4 + r + r + v + v + 4 * nn,        # pos, k, counts, kv r/w, vel r/w
        "divergence_residual": v + v + 4 + r + r + r + 4 * nn,          # pos, vel, counts, alpha, dadv, k
        "viscosity": v + v + 4 + r + v + 4 * nf,                        # pos, vel, counts, rho, acc
        "pressure_warm_jacobi": v + r + 4 + v + v + 4 * nn,             # pos, kappa, counts, vel r/w
        "pressure_residual": v + v + 4 + r + r + r + r + r + r + 4 * nn,  # pos, vel, counts, rho, alpha, kappa r/w, dadv, k
        "pressure_jacobi": v + r + 4 + v + v + 4 * nn,                  # pos, k, counts, vel r/w
        "neighbor_build": v + 4 + 4 * nn,                               # pos, counts, lists written
        "update_pos": v + v + v,                                        # pos r/w, vel
    }[name]
    extra = v * nb_particles if name not in ("viscosity", "update_pos") else 0  # boundary pos+psi once
    return per * n + extra


def setup_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def reduce_max(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_reference_run(scene, steps: int, warmup: int, time_budget: float | None):
    """Times the CPU reference of the step: the reference TimeStepDFSPH harness when it was built
    (oracle/_ref/dfsph_ref), else the oracle's restatement of the GPU formulation. Returns
    (ms_per_step, steps_timed, threads, kind)."""
    ref_bin = ROOT / "oracle" / "_ref" / "dfsph_ref"
    threads = os.cpu_count() or 1
    if ref_bin.exists():
        from oracle.ref_runner import run_reference

        ms, done = run_reference(ref_bin, scene, steps, warmup, time_budget, threads)
        return ms, done, threads, "reference"
    from oracle import Oracle

    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    o = Oracle(scene, 64)
    for _ in range(warmup):
        o.step()
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        o.step()
        done += 1
        if time_budget is not None and time.perf_counter() - t0 > time_budget and done >= 2:
            break
    ms = (time.perf_counter() - t0) * 1e3 / done
    return ms, done, threads, "port"


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    scene = make_scene(args.config)
    ms, done, threads, kind = cpu_reference_run(scene, args.steps, args.warmup, time_budget=args.ref_budget)
    line = {
        "metric": METRIC, "value": round(ms, 3), "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": done, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": scene.name, "fluid_particles": scene.n_fluid, "boundary_particles": scene.n_boundary,
                   "walls": "static (the reference CPU solver's boundary is a static rigid body; the per-step cost "
                            "of a moving wall is its rebinning)" if args.config == 3 else "static",
                   "parallelism": "cpu"},
        "cpu_baseline": {"value": round(ms, 3), "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{done} steps after {args.warmup} warm-up steps of {scene.name}"},
        "e2e": {"value": round(ms, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


ABLATION_WORKLOADS = ("sloshing_1m", "column_2m", "column_64")


def ablation_scene(workload: str):
    """Scenes of the plain vs learned comparison. column_64: a resting column (64 x 64 x 64 =
    262,144 particles, r = 0.008 m, fixed dt 2 ms) at the reference's default 0.01 % tolerance;
    sloshing_1m: the 1,000,000-particle sloshing tank (walls translating 0.1 sin(2 pi t / 2) m along
    x), CFL; column_2m: the 2,000,000-particle column collapse at 0.005 % with dt_max 8 ms, CFL.
    Returns (scene, wall motion or None)."""
    from splishsplash_for_cuda_b200.scene import column_scene, synthetic_scene

    if workload == "column_64":
        return column_scene(counts=(64, 64, 64), time_step=0.002, max_error=0.01), None
    if workload == "sloshing_1m":
        return make_workload(3)
    if workload == "column_2m":
        return synthetic_scene(4, cfl=True), None
    raise ValueError(workload)


def learned_ablation(local, steps: int, workload: str = "column_64", window: int = 0):
    """Plain vs learned warm start on the same scene from the same state, each for `steps` steps;
    the second half is measured (the flow has developed by then). ms/step is the device time of each
    step (CUDA events inside dfsph_step), online training rounds included. "base" is the learned
    warm start with the network's correction fixed at zero (the needed-coefficient base alone, no
    inference, no training), so "learned" vs "base" is the trained network's own contribution.
    "gated" is the learned warm start behind its cost gate (learned passes only while the plain
    solver needs at least one iteration per step above the minimum counts; plain probe windows
    included in the average). window > 0 adds, per mode, the means over consecutive windows of that
    many steps across the whole run (the full horizon) and the mean over all steps."""
    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    scene, walls = ablation_scene(workload)
    out = {"workload": scene.name if workload == "column_64" else workload, "fluid_particles": scene.n_fluid,
           "steps": steps, "measured_steps": f"{steps // 2}..{steps - 1}",
           "max_error_pct": scene.config.maxError, "moving_walls": walls is not None,
           "cfl": bool(scene.config.cflMethod)}
    for mode in ("plain", "base", "learned", "gated"):
        d = DFSPHCUDA(scene, device=local)
        d.set_param("timing", 1)
        if walls is not None:  # the fluid follows the walls past the initial box: keep every particle
            d.set_param("remove_escaped", 0)
        if mode != "plain":
            d.set_learned_warm_start(True, gate=mode == "gated")
        if mode == "base":
            d.set_param("learned_base_only", 1)
        its, itv, ms, hs, bits, t = [], [], [], [], 0, 0.0
        for _ in range(steps):
            if walls is not None:
                walls(d, t)
            st = d.step()
            t += st.h
            its.append(st.iterations)
            itv.append(st.iterations_v)
            ms.append(st.ms_total)
            hs.append(st.h)
            bits |= st.status
        w = slice(steps // 2, steps)
        rec = {"pressure_iterations": round(float(np.mean(its[w])), 2),
               "divergence_iterations": round(float(np.mean(itv[w])), 2),
               "ms_per_step": round(float(np.mean(ms[w])), 4), "status_bits": int(bits),
               "simulated_s": round(t, 4)}
        if window > 0:
            rec["windows"] = [{"steps": f"{a}..{min(a + window, steps) - 1}",
                               "pressure_iterations": round(float(np.mean(its[a:a + window])), 2),
                               "divergence_iterations": round(float(np.mean(itv[a:a + window])), 2),
                               "ms_per_step": round(float(np.mean(ms[a:a + window])), 3),
                               "dt_ms": round(1e3 * float(np.mean(hs[a:a + window])), 3)}
                              for a in range(0, steps, window)]
            rec["ms_per_step_all"] = round(float(np.mean(ms)), 4)
        if mode == "gated":
            rec.update(learned_steps=int(d.get_param("gate_learned_steps")),
                       plain_steps=int(d.get_param("gate_plain_steps")),
                       last_excess_iterations=round(d.get_param("gate_last_excess"), 3))
        if mode == "learned":
            solves = int(d.get_param("learned_solves_p"))
            kept = int(d.get_param("learned_kept_p"))
            rec.update(network_used_at_end=int(d.get_param("network_used")),
                       heldout_loss_ratio=round(d.get_param("mlp_heldout_ratio"), 4))
            rec.update(trainings=int(d.get_param("mlp_trainings")), kept_pressure=kept, solves_pressure=solves,
                       kept_divergence=int(d.get_param("learned_kept_v")),
                       fallback_rate_pressure=round(1 - kept / solves, 4) if solves else None,
                       damping=d.get_param("warm_start_damping"))
        out[mode] = rec
        d.close()
    out["pressure_iteration_reduction"] = round(1 - out["learned"]["pressure_iterations"]
                                                / out["plain"]["pressure_iterations"], 4)
    out["network_contribution_iterations"] = round(out["base"]["pressure_iterations"]
                                                   - out["learned"]["pressure_iterations"], 3)
    out["ms_per_step_reduction"] = round(1 - out["learned"]["ms_per_step"] / out["plain"]["ms_per_step"], 4)
    out["gated_ms_per_step_reduction"] = round(1 - out["gated"]["ms_per_step"] / out["plain"]["ms_per_step"], 4)
    return out


def run_wave_tank(args, world, rank, local):
    """--config 5: the 4,000,000-particle wave tank (piston, absorbing open boundary, floating box,
    dynamic window; splishsplash_for_cuda_b200/wave_tank.py) for W + K steps. ms_per_step is the
    device time of each whole step, the workload's host-side coupling (piston and body motion, body
    wrench, open boundary, window) included, from CUDA events on the solver's stream."""
    import torch

    from splishsplash_for_cuda_b200.wave_tank import WaveTank, wave_tank_scene

    scene, layout = wave_tank_scene()
    tank = WaveTank(scene, layout, device=local, learned=not args.plain_wave_tank)
    d = tank.d
    d.set_param("timing", 1)
    stream = torch.cuda.ExternalStream(d.stream_handle(), device=torch.device("cuda", local))
    for _ in range(args.warmup):
        tank.step()
    d.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    its, itv, solver_ms, n_max = [], [], [], 0
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                starts[k].record(stream)
            st = tank.step()
            with torch.cuda.stream(stream):
                ends[k].record(stream)
            its.append(st.iterations)
            itv.append(st.iterations_v)
            solver_ms.append(st.ms_total)
            n_max = max(n_max, st.num_fluid)
        torch.cuda.synchronize(local)
    total = sum(starts[k].elapsed_time(ends[k]) for k in range(args.steps))
    ms = reduce_max(total / args.steps, world)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": round(ms, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice + xoshiro256** jitter)",
            "config": {"workload": scene.name, "fluid_particles": scene.n_fluid, "boundary_particles": scene.n_boundary,
                       "warm_start": "plain" if args.plain_wave_tank else "learned (gated)",
                       "lattice_spacing_mm": 18.59, "piston": "0.2 m, 1.5 s", "absorbing_layer_m": 0.3,
                       "window_shift_m": 0.5, "window_check_every_steps": tank.window_every,
                       "window_shift_when": "piston at its furthest advance",
                       "floating_box": "0.403 x 0.199 x 0.199 m, 500 kg/m^3", "dt_max_ms": 1.0,
                       "parallelism": "replicas" if world > 1 else "single"},
            "iterations_per_step": round(float(np.mean(its)), 2), "iterations_v_per_step": round(float(np.mean(itv)), 2),
            "solver_ms_per_step": round(float(np.mean(solver_ms)), 4), "status_bits": int(tank.status),
            "simulated_s": round(tank.t, 4), "window_shifts": tank.shifts, "added": tank.added, "removed": tank.removed,
            "fluid_particles_max": n_max, "fluid_particles_end": d.num_fluid(),
            "body_center": [round(float(c), 4) for c in tank.body.x], "clocks": clk.summary()}), flush=True)
    d.close()


def run_ours(args, world, rank, local):
    import torch

    from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA

    scene, motion = make_workload(args.config)
    n = scene.n_fluid
    d = DFSPHCUDA(scene, device=local, use_graphs=not args.host_loops, precision=args.precision)
    d.set_param("timing", 0)
    if motion is not None:  # the fluid follows the walls past the initial box: keep every particle
        d.set_param("remove_escaped", 0)
    stream = torch.cuda.ExternalStream(d.stream_handle(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    sim_t = [0.0]

    def advance():
        """One step of the workload: the walls' motion at the current simulated time (on the device),
        then the step. With moving walls the step returns its statistics (the next motion needs its
        dt); otherwise it is only enqueued."""
        if motion is None:
            d.step_async()
            return
        motion(d, sim_t[0])
        sim_t[0] += d.step().h

    for _ in range(args.warmup):
        advance()
    d.synchronize()

    def timed_steps(k, e2e=False, host=None):
        """k steps, each bracketed by CUDA events on the solver's stream after a 256 MiB write that
        evicts L2. Without moving walls steps are enqueued without host round trips (the step runs
        on the device, dt included); iterations come from the device counters. e2e: each step also
        uploads its inputs from pinned host memory and reads positions and velocities back
        (readDynamicData, which waits)."""
        tot = 0.0
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        d.set_param("iterations_sum", 0)
        for s in range(k):
            with torch.cuda.stream(stream):
                flush.fill_(float(s))
                starts[s].record(stream)
            if e2e:
                d.update_fluid(host["x"], host["v"])
            advance()
            if e2e:  # DFSPHCData::readDynamicData: positions and velocities, one wait
                d.m_data.readDynamicData(host["x"], host["v"])
            with torch.cuda.stream(stream):
                ends[s].record(stream)
        torch.cuda.synchronize(local)
        for s in range(k):
            tot += starts[s].elapsed_time(ends[s])
        its, itv = d.get_param("iterations_sum"), d.get_param("iterations_v_sum")
        bits = d.status(clear=True)
        return tot, its / k, itv / k, bits

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize(local)
    l0 = d.launch_count()
    with ClockSampler(local) as clk:
        total_ms, mean_it, mean_itv, status_bits = timed_steps(args.steps)
    # the loop bodies inside the solver graphs launch a Jacobi and a residual pass per iteration
    launches = d.launch_count() - l0 + (0 if args.host_loops else int(round(2 * (mean_it + mean_itv) * args.steps)))
    if world > 1:
        dist.barrier()
    ms = reduce_max(total_ms / args.steps, world)
    agg_pps = reduce_sum(n * args.steps / (total_ms / 1e3), world)
    if args.steps_only:  # profiling runs: the warm-up and the timed steps, nothing else
        if rank == 0:
            print(json.dumps({"workload": scene.name, "ms_per_step": round(ms, 4), "iterations_per_step": mean_it,
                              "iterations_v_per_step": mean_itv, "status_bits": int(status_bits)}), flush=True)
        d.close()
        return

    # end-to-end through the public API with host buffers (pinned), copies inside the timed region
    xh = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    vh = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    xh[:] = d.positions()
    vh[:] = d.velocities()
    e2e_total, _, _, _ = timed_steps(args.steps, e2e=True, host={"x": xh, "v": vh})
    e2e_ms = reduce_max(e2e_total / args.steps, world)

    # per-kernel device time with a cold L2 before each launch, for the roofline
    counts = d.field("neighbor_counts")
    nf, nbn = float(counts[:, 0].mean()), float(counts[:, 1].mean())
    kt = {}
    for name in ["pressure_jacobi", "pressure_residual", "divergence_jacobi", "divergence_residual",
                 "density_alpha", "viscosity", "pressure_warm_jacobi", "neighbor_build", "update_pos"]:
        vals = []
        for _ in range(args.kernel_reps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            vals.append(d.time_kernel(name, 1))
        kt[name] = float(np.median(vals))
    per_step_launches = {"pressure_jacobi": mean_it, "pressure_residual": mean_it + 1,
                         "divergence_jacobi": mean_itv + 1, "divergence_residual": mean_itv + 1,
                         "density_alpha": 1, "viscosity": 1, "pressure_warm_jacobi": 1, "neighbor_build": 1,
                         "update_pos": 1}
    share = {k: kt[k] * per_step_launches[k] for k in kt}
    dom = max(share, key=share.get)
    peak, peak_kind = _peaks()
    alg = kernel_bytes(dom, n, scene.n_boundary, nf, nbn, 8 if args.precision == 64 else 4)
    achieved = alg / (kt[dom] * 1e-3) / 1e9
    # The same kernel back to back without the flush: when its working set fits the 126 MB L2 (the
    # 250 k configurations) this is the rate it sustains inside a step, served from L2.
    d.time_kernel(dom, 1)
    warm_ms = float(np.median([d.time_kernel(dom, 1) for _ in range(max(args.kernel_reps, 3))]))
    l2_resident = alg < 0.75 * 126e6
    traffic = None
    tf = ROOT / "profiles" / "ncu_traffic.json"
    if tf.exists() and args.precision == 32:  # the captures are of the FP32 build
        tj = json.loads(tf.read_text())
        rec = tj.get("kernels", {}).get(dom)
        if rec and rec.get("n_particles"):
            traffic = rec["dram_bytes_per_launch"] * n / rec["n_particles"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ms_cpu, done, threads, kind = cpu_reference_run(scene, 10 ** 6, 1, time_budget=args.cpu_budget)
        cpu = {"value": round(ms_cpu, 2), "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{done} steps (after 1 warm-up) of {scene.name}, {args.cpu_budget:.0f} s budget"}

    ablation = None
    if rank == 0 and world == 1 and args.ablation_steps > 0:
        ablation = {w: learned_ablation(local, args.ablation_steps, w, args.ablation_window) for w in args.ablation_workloads}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(ms, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded lattice + xoshiro256** jitter)",
            "config": {"workload": scene.name, "fluid_particles": n, "boundary_particles": scene.n_boundary,
                       "radius": scene.config.particleRadius, "cfl": f"0.4, dt_max {scene.config.cflMaxTimeStepSize * 1e3:g} ms",
                       "max_error_pct": scene.config.maxError, "max_error_v_pct": scene.config.maxErrorV,
                       "warm_start": "plain",
                       "walls": "rigid translation x = 0.1 sin(pi t) m, moved on the device every step"
                       if motion is not None else "static",
                       "l2": "256 MiB write before every timed step"
                       + ("; the step's working set exceeds L2" if n >= 1_000_000 else ""),
                       "parallelism": "replicas" if world > 1 else "single"},
            "iterations_per_step": round(mean_it, 2), "iterations_v_per_step": round(mean_itv, 2),
            "status_bits": int(status_bits),
            "particle_steps_per_s": round(agg_pps, 1),
            "e2e": {"value": round(e2e_ms, 4), "unit": UNIT, "h2d_bytes_per_step": n * 24, "d2h_bytes_per_step": n * 24},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": None if traffic is None else round(traffic),
                         "algorithmic_bytes": round(alg), "ms_per_launch": round(kt[dom], 5),
                         "l2_resident": bool(l2_resident), "ms_per_launch_warm_l2": round(warm_ms, 5),
                         "achieved_warm_l2": round(alg / (warm_ms * 1e-3) / 1e9, 1)},
            "kernel_ms": {k: round(v, 5) for k, v in kt.items()},
            "mean_neighbors": {"fluid": round(nf, 2), "boundary": round(nbn, 2)},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "learned_warm_start": ablation,
        }
        print(json.dumps(line), flush=True)
    d.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--host-loops", action="store_true", help="solver loops driven from the host")
    ap.add_argument("--precision", type=int, choices=[32, 64], default=32,
                    help="64: the FP64 build of the same kernels (the precision comparison of config 2)")
    ap.add_argument("--kernel-reps", type=int, default=5)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-wave-tank", action="store_true", help="--config 5 with the plain warm start")
    ap.add_argument("--steps-only", action="store_true",
                    help="profiling: run the warm-up and the timed steps only and print a short line")
    ap.add_argument("--ablation-steps", type=int, default=300,
                    help="steps per mode of the plain vs learned warm-start comparison (0: skip)")
    ap.add_argument("--ablation-workloads", nargs="*", choices=ABLATION_WORKLOADS, default=list(ABLATION_WORKLOADS))
    ap.add_argument("--ablation-window", type=int, default=0,
                    help="with --ablation-only: also report means over windows of this many steps")
    ap.add_argument("--ablation-only", action="store_true",
                    help="print only the plain vs learned comparison as one JSON line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = setup_dist()
    try:
        if args.ablation_only:
            if rank == 0:
                print(json.dumps({"learned_warm_start": {w: learned_ablation(local, args.ablation_steps, w,
                                                                            args.ablation_window)
                                                         for w in args.ablation_workloads}}), flush=True)
        elif args.impl == "reference":
            run_reference_arm(args, world, rank)
        elif args.config == 5:
            run_wave_tank(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
