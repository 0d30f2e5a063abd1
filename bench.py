"""Benchmark: atom-steps/s of the BEADS per-step MD hot path on B200.

Workload (one replica per GPU, "replicas only" scaling): the 1,048,576-bead
binary LJ mixture in nm_kjmol units (80/20 types, mass 39.95 u, cubic box
37.2 nm, eps 1.0/0.5/0.7, sigma 0.34/0.30/0.32, rc 0.9 shifted, skin 0.1,
max_neighbors 128, Berendsen 120 K / tau 0.1, dt 0.002), seeded uniform start
relaxed by 500 capped steepest-descent steps.  Synthetic data; no dataset.

One bench "step" is one velocity-Verlet MD step of the whole system (pre
half-kick/drift/wrap/rebuild decision, device-decided neighbour rebuild,
LJ forces, post half-kick + Berendsen).  The neighbour list (~360 MB) and the
particle state (~100 MB) exceed the 126 MB L2, so consecutive steps cannot
serve each other from L2.

Arms:
  default            the CUDA engine through its C ABI.
  --impl reference   the reference's algorithm on the host cores (the CPU
                     oracle port: the reference has no CPU implementation of
                     this path) on the same workload, relaxed the same way on
                     the host; its line also carries the reference's own CUDA
                     build timed on the same relaxed input (`reference_cuda`).

`--gpus N` (N > 1) without a launcher re-executes this script under
torch.distributed.run with N local ranks on 127.0.0.1.  The mixture then runs
one replica per GPU ("weak"); `--workload replicas` and `--workload adjoint`
split one replica batch over the ranks by atom count ("strong"), the adjoint
summing its parameter gradients and loss over the ranks (NCCL all-reduce).
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

UNIT = "atom-steps/s"
N_BEADS = 1_048_576
E2E_STEPS = 100  # MD steps per end-to-end call
GRAPH_WARMUP = 31  # untimed steps that instantiate every captured step graph
REF_MIN_STEPS = 60  # fewest timed MD steps of the host-core reference arm
CLOCK_WINDOW_S = 0.6  # shortest stretch of load the clock sampler sees
WORKLOAD = ("binary LJ mixture, 1,048,576 beads per GPU, nm_kjmol, 80/20 types, box 37.2 nm, "
            "rc 0.9 (shifted), skin 0.1, max_neighbors 128, sort every rebuild, Berendsen 120 K "
            "tau 0.1, dt 0.002, seeded uniform start relaxed by 500 capped steepest-descent "
            "steps")
L2_NOTE = "inputs larger than L2 (list ~4*mean_nbr*N bytes + state ~100 B per bead)"


def metric(world: int) -> str:
    return (f"atom-steps/s on {world} B200 (1M-bead binary LJ mixture per GPU, FP32 pair "
            "math, fixed-point totals)")


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _launch_ranks(gpus: int) -> None:
    """Re-executes this command under torch.distributed.run with `gpus` local
    ranks when no launcher set WORLD_SIZE (does not return)."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           str(pathlib.Path(__file__).resolve()), *sys.argv[1:]]
    os.execv(sys.executable, cmd)


def _peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_from_profile():
    """DRAM bytes per launch of the force kernel from the committed ncu summary
    (profiles/lj_force_mixture_1m.txt), or None."""
    path = ROOT / "profiles" / "lj_force_mixture_1m.txt"
    if not path.exists():
        return None
    m = re.search(r"dram_bytes_per_launch_full:\s*([0-9.eE+]+)", path.read_text())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def _load_until(eng, since: float, window_s: float = CLOCK_WINDOW_S, stepping: bool = True) -> int:
    """Keeps the GPU busy (untimed) until `window_s` seconds have passed
    since `since`, so a 200 ms clock sampler sees the kernels under load even
    when the timed steps take a few milliseconds: MD steps, or (stepping =
    False) force evaluations of the current state, which leave the
    trajectory where the timed steps ended.  Returns the extra steps or
    evaluations."""
    import torch

    extra = 0
    while time.perf_counter() - since < window_s:
        if stepping:
            eng.run(16)
        else:
            eng.profile("forces", 16)
        torch.cuda.synchronize()
        extra += 16
    return extra


def _prepare_engine(local_rank: int, n_beads: int = N_BEADS):
    from beads_b200 import workloads
    from beads_b200.engine import Engine

    box = 37.2 * (n_beads / N_BEADS) ** (1 / 3)
    spec = workloads.lj_mixture(n=n_beads, box=box, seed=3 + local_rank)
    # The uniform start has Poisson density fluctuations that overflow the
    # production list capacity (128); relax with a roomier list first.
    capacity = spec.max_neighbors
    spec.max_neighbors = 256
    with Engine(spec) as relax:
        relax.minimize(500, 0.004, 200.0)
        # A wrapped float coordinate can round to the upper bound itself;
        # nudge those onto the last float inside [lo, hi) for the new engine.
        spec.positions = workloads._inside(relax.state()["positions"].astype(np.float64),
                                           np.zeros(3), np.full(3, box))
    spec.max_neighbors = capacity
    eng = Engine(spec)
    eng.run(200)  # settle the list / sort order before timing
    return spec, eng


def _cpu_sim(spec, positions, n_sample: int):
    """CPU oracle state for a bounded sample: the first n_sample beads of a
    cubic sub-box at the workload's density and composition."""
    from oracle import oracle as O

    ff = O.ForceField(epsilon=spec.epsilon.ravel(), sigma=spec.sigma.ravel(), cutoff=spec.cutoff,
                      shift=spec.shift)
    n_all = spec.n
    if n_sample >= n_all:
        pos = np.asarray(positions, np.float32)
        box = spec.box_bound
        sel = np.arange(n_all)
    else:
        side = float(spec.box_bound[1][0] - spec.box_bound[0][0]) * (n_sample / n_all) ** (1 / 3)
        sel = np.nonzero(np.all(np.asarray(positions) < side, axis=1))[0]
        pos = np.asarray(positions, np.float32)[sel]
        box = np.array([[0, 0, 0], [side] * 3], np.float32)
    sim = O.Sim(pos, np.asarray(spec.velocities, np.float64)[sel], np.asarray(spec.masses)[sel],
                np.asarray(spec.types)[sel], box, ff, dt=spec.dt, skin=spec.cutoff_buffer,
                check_every=spec.rebuild_check_every, thermostat=True,
                kt_target=0.00831446261815324 * spec.thermostat[0], tau=spec.thermostat[1])
    return sim, len(sel)


def _cpu_rate(sim, n, steps: int) -> tuple[float, float]:
    t0 = time.perf_counter()
    sim.step(steps)
    wall = time.perf_counter() - t0
    return n * steps / wall, wall


def _cpu_baseline(positions, spec, budget_s: float):
    """Times the CPU oracle port (OpenMP, FP64) on the full system for a
    bounded number of MD steps (about budget_s of host work)."""
    from oracle import oracle as O

    sim, n = _cpu_sim(spec, positions, spec.n)
    rate, wall = _cpu_rate(sim, n, 1)
    steps = max(1, int(budget_s / max(wall, 1e-3)))
    rate, wall = _cpu_rate(sim, n, steps)
    sim.close()
    return {"value": rate, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"{steps} MD steps of the full {n}-bead system (after one untimed step), "
                      f"{wall:.1f} s of host work, FP64 oracle with OpenMP"}


def _cpu_baseline_melt(spec, budget_s: float):
    """Times the CPU oracle port (OpenMP, FP64) on the whole bead-spring melt
    (pairs, bonds, angles, dihedrals, exclusions, Berendsen) for a bounded
    number of MD steps (about budget_s of host work)."""
    from oracle import oracle as O

    ff = O.ForceField(epsilon=np.asarray(spec.epsilon, np.float64).ravel(),
                      sigma=np.asarray(spec.sigma, np.float64).ravel(), cutoff=spec.cutoff,
                      shift=spec.shift, bond_k=spec.bond_k, bond_r0=spec.bond_r0,
                      angle_k=spec.angle_k, angle_theta0=spec.angle_theta0,
                      dihedral_k=spec.dihedral_k, dihedral_d=spec.dihedral_d,
                      dihedral_n=spec.dihedral_n, exclusion_distance=spec.exclusion_distance)
    # reduced units: k_B T is the target temperature itself
    sim = O.Sim(spec.positions, spec.velocities, spec.masses, spec.types, spec.box_bound, ff,
                dt=spec.dt, skin=spec.cutoff_buffer, check_every=spec.rebuild_check_every,
                bonds=spec.bonds, angles=spec.angles, dihedrals=spec.dihedrals,
                thermostat=True, kt_target=spec.thermostat[0], tau=spec.thermostat[1])
    sim.step(1)
    # One step at a time until the budget is spent (at most 100 steps): the
    # melt rebuilds its list every few steps, so the first step's time does
    # not predict the rest, and the melt diverges after a few hundred steps.
    steps, wall = 0, 0.0
    t0 = time.perf_counter()
    while wall < budget_s and steps < 100:
        sim.step(1)
        steps += 1
        wall = time.perf_counter() - t0
    rate = spec.n * steps / wall
    sim.close()
    return {"value": rate, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"{steps} MD steps of the full {spec.n}-bead melt (after one untimed "
                      f"step), {wall:.1f} s of host work, FP64 oracle with OpenMP"}


def _relaxed_on_host(seed: int = 3):
    """The workload's input prepared on the host cores: the same seeded
    uniform start relaxed by the same 500 capped steepest-descent steps
    (x += 0.004 nm F / max(|F|, 200), LJ on r^2 >= 0.49 sigma^2), in the CPU
    oracle's FP64 restatement instead of the GPU engine.  Returns the spec (with
    the relaxed positions) and the oracle state ready to step."""
    from beads_b200 import workloads

    spec = workloads.lj_mixture(n=N_BEADS, box=37.2, seed=seed)
    sim, _ = _cpu_sim(spec, spec.positions, spec.n)
    sim.minimize(500, 0.004, 200.0)
    pos, _, img, _ = sim.state()
    spec.positions = workloads._inside(pos, np.zeros(3), np.full(3, 37.2))
    spec.images = img
    return spec, sim


def run_reference(args) -> None:
    """The reference's algorithm for this path on the host cores: the CPU
    oracle port (FP64, OpenMP on every host thread; the reference itself has
    no CPU implementation) on the whole 1,048,576-bead workload, one MD step
    per bench step with the reference's rebuild policy.  Beside it, the
    reference's own CUDA build on the same relaxed input through its
    execute_simulation, timed by its log (`reference_cuda`; outside `value`)."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    from oracle import oracle as O

    t_prep = time.perf_counter()
    spec, sim = _relaxed_on_host()
    prep_s = time.perf_counter() - t_prep
    for _ in range(args.warmup):
        sim.step(1)
    builds0 = sim.state()[3]
    # At least REF_MIN_STEPS timed steps, so the sample holds list rebuilds
    # (this workload rebuilds every ~25 steps) like the GPU arm's timing.
    n_steps = max(args.steps, REF_MIN_STEPS)
    t0 = time.perf_counter()
    for _ in range(n_steps):
        sim.step(1)
    total = time.perf_counter() - t0
    builds = sim.state()[3] - builds0
    sim.close()
    n = spec.n
    value = n * n_steps / total
    cores = O.num_threads()
    sample = (f"the whole {n}-bead workload, relaxed on the host ({prep_s:.0f} s, untimed), "
              f"{args.warmup} warm-up + {n_steps} timed MD steps, {builds} neighbour "
              "rebuilds in the timed steps; FP64 oracle port with OpenMP")
    reference_cuda = None
    if not args.no_reference_cuda:
        try:
            from oracle import ref_bench

            # The reference's steps_per_second covers its whole run, the
            # initial build included, so it runs long enough for steady state.
            reference_cuda = ref_bench.reference_engine_rate(spec, args.reference_cuda_steps)
            reference_cuda.update(
                unit=UNIT, build="the reference's own sources compiled for sm_100a, float32 "
                "(oracle/build_ref.py), same relaxed spec, its execute_simulation and log timer")
        except Exception as e:  # noqa: BLE001 - reported, not fatal
            reference_cuda = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    line = {
        "impl": "reference",
        "metric": metric(world),
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": n_steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / n_steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "l2": L2_NOTE},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "run": {"neighbor_builds_timed": int(builds), "host_relaxation_s": prep_s},
        "reference_cuda": reference_cuda,
    }
    print(json.dumps(line))


def _energy_drift(spec, eng, steps: int = 2000, every: int = 100, time_unit: str = "ns",
                  state: dict | None = None) -> dict:
    """Energy drift of the workload's dynamics: an NVE copy (Berendsen off,
    which would otherwise add or remove energy) of the engine's current state
    runs `steps` steps with a thermo row every `every` steps; the drift is the
    least-squares slope of the total energy per bead against time (time_unit
    "ns" for nm_kjmol inputs, whose dt is in ps; "tau" for reduced units)."""
    import dataclasses

    from beads_b200 import workloads
    from beads_b200.engine import Engine

    st = eng.state() if state is None else state
    box = np.asarray(spec.box_bound, np.float64)
    nve = dataclasses.replace(
        spec, thermostat=None, images=st["images"],
        positions=workloads._inside(st["positions"].astype(np.float64), box[0], box[1]),
        velocities=st["velocities"])
    with Engine(nve) as e:
        rows = [e.eval()[0]]
        for _ in range(steps // every):
            rows.append(e.run(every, every)[0])
    etot = np.array([r["pe"] + r["ke"] for r in rows], np.float64) / spec.n
    scale = 1.0 / 1000.0 if time_unit == "ns" else 1.0  # dt in ps, or in tau
    t = np.arange(len(rows)) * every * spec.dt * scale
    slope = float(np.polyfit(t, etot, 1)[0])
    unit = "kJ/mol per bead per ns" if time_unit == "ns" else "epsilon per bead per tau"
    return {"value": slope, "unit": unit, "steps": steps,
            "dt": spec.dt, "e_total_per_bead_start": float(etot[0]),
            "e_total_per_bead_end": float(etot[-1]),
            "relative_change": float((etot[-1] - etot[0]) / abs(etot[0])),
            "ensemble": "NVE copy (Berendsen off) of the engine state after the timed steps "
                        "(the relaxed start for the melt), "
                        "float32 pair math, fixed-point totals"}


def run_ours(args) -> None:
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from beads_b200.engine import Engine  # noqa: F401

    spec, eng = _prepare_engine(local, args.beads)
    stream = torch.cuda.ExternalStream(eng.info()["stream"], device=torch.device("cuda", local))

    # L2 flush buffer (not needed: the working set is > L2, kept for hygiene of
    # the kernel-level timing below).
    for _ in range(max(3, args.warmup)):
        eng.run(1)
    # Runs replay captured graphs of 16, 8, ..., 1 steps; one untimed run of
    # 31 steps instantiates each of them outside the timed region.
    eng.run(GRAPH_WARMUP)
    stats = eng.list_stats()
    mean_nbr = stats["entries"] / spec.n

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    c0 = eng.counters()
    profile_region = os.environ.get("BEADS_PROFILE_TIMED") == "1"
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    t_sample = time.perf_counter()
    if profile_region:  # lets a profiler started with capture off see only these steps
        torch.cuda.profiler.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    eng.run(args.steps)
    stop.record(stream)
    stop.synchronize()
    if profile_region:
        torch.cuda.profiler.stop()
    c1 = eng.counters()
    # The clock record covers at least CLOCK_WINDOW_S of the same stepping
    # (untimed steps after the timed ones); the value is the timed steps'.
    clock_extra_steps = 0 if profile_region else _load_until(eng, t_sample)
    barrier()
    clocks = sampler.stop()
    clocks["untimed_steps_after_timed"] = clock_extra_steps
    timed_builds = c1["builds"] - c0["builds"]
    timed_chains = c1["chain_launches"] - c0["chain_launches"]
    elapsed_ms = start.elapsed_time(stop)
    if dist is not None:
        t = torch.tensor([elapsed_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    value = world * spec.n * args.steps / (elapsed_ms / 1e3)

    # Dominant kernel: the LJ pair-force kernel under the engine's schedule,
    # timed alone on the engine stream.
    force_ms = eng.profile("forces", 50)
    step_ms_alone = elapsed_ms / args.steps
    # list entries + own position + count + force write
    bytes_per_atom = 4.0 * mean_nbr + 36.0
    achieved = spec.n * bytes_per_atom / (force_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()
    traffic = _traffic_from_profile()
    # Secondary figure: FP32 work of the pair kernel per atom-step, 9 per
    # listed pair (difference, r^2, test) + 23 per pair inside rc (force,
    # energy, virial); pairs inside rc estimated from the list at uniform
    # density, n_c = n_l (rc / (rc + skin))^3.  Peak: SMs x 128 FP32 lanes x
    # 2 FLOP (FMA) x the SM clock sampled during the timed steps.
    n_inside = mean_nbr * (spec.cutoff / (spec.cutoff + spec.cutoff_buffer)) ** 3
    flop_per_atom = 9.0 * mean_nbr + 23.0 * n_inside
    sms = torch.cuda.get_device_properties(local).multi_processor_count

    # End-to-end through the C ABI with host buffers: upload positions and
    # velocities, run E2E_STEPS steps (the call rebuilds the list and forces
    # first, as a fresh run does), download both.
    e2e_value = None
    if args.no_e2e:
        e2e_calls = 0
    pin_pos = torch.empty((spec.n, 3), dtype=torch.float32, pin_memory=True)
    pin_vel = torch.empty((spec.n, 3), dtype=torch.float32, pin_memory=True)
    eng.download_all(pin_pos.numpy(), pin_vel.numpy())
    if not args.no_e2e:
        e2e_calls = max(2, args.steps // (4 * E2E_STEPS))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        eng.upload_all(pin_pos.numpy(), pin_vel.numpy())
        eng.run(E2E_STEPS)
        eng.download_all(pin_pos.numpy(), pin_vel.numpy())
    barrier()
    e2e_wall = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_wall], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_wall = float(t.item())
    if e2e_calls:
        e2e_value = world * spec.n * E2E_STEPS * e2e_calls / e2e_wall
    # Bytes copied per call (positions + velocities in, the same out), per MD step.
    h2d = 2 * spec.n * 3 * 4 / E2E_STEPS
    d2h = 2 * spec.n * 3 * 4 / E2E_STEPS

    drift = None if args.no_drift else _energy_drift(spec, eng)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        st = eng.state()
        cpu = _cpu_baseline(st["positions"], spec, args.cpu_budget)

    # Every step launches pre, the per-replica rebuild decision, the
    # pair-force kernel, post (unless the schedule fuses the kick into the
    # force kernel) and the per-replica finish kernel; a step that rebuilds
    # also runs the rebuild chain (conditional graph node).  The engine counts
    # both as kernel nodes of a captured step.
    launches = eng.launch_counts()
    gpu_launches = (launches["per_step"] * args.steps
                    + launches["per_rebuild_chain"] * int(timed_chains))
    clock_mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
    flops = None
    if clock_mhz:
        flop_achieved = spec.n * flop_per_atom / (force_ms / 1e3) / 1e12
        flop_peak = sms * 128 * 2 * clock_mhz * 1e6 / 1e12
        flops = {"kernel": "k_lj (pair forces)", "per_atom_step": flop_per_atom,
                 "pairs_inside_rc_per_atom": n_inside, "achieved": flop_achieved,
                 "peak": flop_peak, "unit": "TFLOP/s", "frac": flop_achieved / flop_peak,
                 "peak_kind": f"FP32 FMA pipe, {sms} SMs x 128 lanes x 2 at {clock_mhz:.0f} MHz "
                              "(SM clock sampled during the timed steps)"}
    line = {
        "metric": metric(world),
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_ms_alone,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "l2": L2_NOTE},
        "run": {
            "parallelism": f"replicas x{world}",
            "mean_neighbors": round(mean_nbr, 2),
            "max_neighbors_seen": stats["max"],
            "neighbor_builds_timed": int(timed_builds),
            "rebuild_chain_launches_timed": int(timed_chains),
            "kernels_per_step": launches["per_step"],
            "kernels_per_rebuild_chain": launches["per_rebuild_chain"],
            "graph_warmup_steps": GRAPH_WARMUP,
            "schedule": eng.tuning(),
        },
        "roofline": {
            "bound": "hbm",
            "kernel": "k_lj (pair forces)",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "peak_kind": peak_kind,
            "bytes_per_atom": bytes_per_atom,
            "kernel_ms": force_ms,
        },
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "md_steps_per_call": E2E_STEPS,
                "calls": e2e_calls,
                "call": "beads_upload_all (pinned host positions + velocities) -> "
                        "beads_run(100) -> beads_download_all, per call"},
        "gpu_launches": gpu_launches,
        "clocks": clocks,
    }
    if flops is not None:
        line["flops"] = flops
    if drift is not None:
        line["energy_drift"] = drift
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line))
    eng.close()
    if dist is not None:
        dist.destroy_process_group()


def replica_metric(world: int) -> str:
    return (f"atom-steps/s on {world} B200 (512-replica batch of uneven LJ systems in one launch "
            "per kernel per GPU, FP32 pair math, fixed-point totals)")


def _init_nccl(world: int):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return dist


def run_replicas(args) -> None:
    """The 512-replica batch: uneven single-type LJ replicas (sizes seeded
    log-uniform in [256, 32768], density U[0.7, 0.9], Berendsen target T
    U[0.8, 1.5] tau 1, rc 2.5, dt 0.005) stepped together, beside the same
    replicas run one at a time through the same engine.  With several ranks
    the one batch is split over them by atom count (every rank builds the same
    description and keeps its share); the time is the slowest rank's."""
    import torch

    from beads_b200 import workloads
    from beads_b200.distributed import max_over_ranks, shard_replicas, sum_over_ranks
    from beads_b200.engine import Engine

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = _init_nccl(world)
    dev = torch.device("cuda", local)
    all_specs = workloads.replica_batch(args.replicas, seed=7)
    total_atoms = sum(s.n for s in all_specs)
    _, specs = shard_replicas(all_specs, world, rank)
    atoms = sum(s.n for s in specs)
    eng = Engine(specs)
    stream = torch.cuda.ExternalStream(eng.info()["stream"], device=dev)
    eng.run(max(3, args.warmup))
    eng.run(GRAPH_WARMUP)
    builds_before = sum(eng.counters(r)["builds"] for r in range(len(specs)))
    chains_before = eng.counters()["chain_launches"]
    profile_region = os.environ.get("BEADS_PROFILE_TIMED") == "1"
    sampler = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    t_sample = time.perf_counter()
    if profile_region:  # lets a profiler started with capture off see only these steps
        torch.cuda.profiler.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    eng.run(args.steps)
    stop.record(stream)
    stop.synchronize()
    if profile_region:
        torch.cuda.profiler.stop()
    builds = sum(eng.counters(r)["builds"] for r in range(len(specs))) - builds_before
    chains = eng.counters()["chain_launches"] - chains_before
    extra = 0 if profile_region else _load_until(eng, t_sample)
    clocks = sampler.stop()
    clocks["untimed_steps_after_timed"] = extra
    batch_ms = max_over_ranks(start.elapsed_time(stop), dev)
    builds = int(sum_over_ranks(builds, dev))
    schedule = eng.tuning()
    launches = eng.launch_counts()
    value = total_atoms * args.steps / (batch_ms / 1e3)
    eng.close()

    # The same replicas one at a time (one engine each, same kernels), every
    # replica for `seq_steps` steps after warm-up; the sequential rate is the
    # total atom-steps over the summed device time (slowest rank's sum).
    seq_steps = max(10, min(args.steps, 200))
    seq_ms = 0.0
    for spec in specs:
        with Engine(spec) as one:
            one.run(3)
            s1 = torch.cuda.ExternalStream(one.info()["stream"],
                                           device=torch.device("cuda", local))
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(s1)
            one.run(seq_steps)
            b.record(s1)
            b.synchronize()
            seq_ms += a.elapsed_time(b)
    seq_ms = max_over_ranks(seq_ms, dev)
    seq_value = total_atoms * seq_steps / (seq_ms / 1e3)
    if dist is not None:
        dist.destroy_process_group()
    line = {
        "metric": replica_metric(world),
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": batch_ms / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": f"{len(all_specs)} LJ replicas, {total_atoms} beads in total, sizes "
                        "log-uniform [256, 32768], rho U[0.7, 0.9], Berendsen T U[0.8, 1.5], "
                        "rc 2.5, skin 0.3",
            "parallelism": (f"one batch split over {world} GPUs by atom count"
                            if world > 1 else "replicas in one batch"),
            "beads_per_rank_this_rank": atoms,
            "sequential_value": seq_value,
            "sequential_steps_per_replica": seq_steps,
            "batch_over_sequential": value / seq_value,
            "neighbor_builds_timed": int(builds),
            "rebuild_chain_launches_timed": int(chains),
            "graph_warmup_steps": GRAPH_WARMUP,
            "schedule": schedule,
        },
        "gpu_launches": (launches["per_step"] * args.steps
                         + launches["per_rebuild_chain"] * int(chains)),
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line))


CHAINS_METRIC = ("atom-steps/s on 1 B200 (400,000-bead bead-spring melt: WCA pairs, harmonic "
                 "bonds, angles and dihedrals, 1-2/1-3 exclusions; one system, one GPU)")


def run_chains(args) -> None:
    """The bead-spring melt: 2000 chains of 200 beads grown as seeded
    self-avoiding walks (step 0.97, rejection radius 0.8) at rho 0.85 and
    relaxed by 500 capped steepest-descent steps, reduced units; LJ rc
    2^(1/6) shifted, skin 0.3; bonds k 500 r0 0.97, angles k 5 theta0 150,
    dihedrals k 1 d 1 n 1; pairs within two bonds excluded; Berendsen T 1
    tau 1, dt 0.005.  One engine on one GPU, device-timed."""
    import torch

    from beads_b200 import workloads
    from beads_b200.engine import Engine

    world, rank, local = _dist()
    if world > 1:
        raise SystemExit("--workload chains runs on one GPU")
    torch.cuda.set_device(local)
    spec = workloads.relaxed(workloads.polymer_melt(seed=5, growth="lockstep"))
    eng = Engine(spec)
    stream = torch.cuda.ExternalStream(eng.info()["stream"], device=torch.device("cuda", local))
    # The relaxed start, kept on the host: the end-to-end calls and the drift
    # run start from it.  This melt's dynamics are stable for a few hundred
    # steps only (a bond angle reaching 180 degrees makes the harmonic
    # dihedral force diverge; the reference's float32 build stops at step
    # ~150 on the same input), so every leg stays inside that window.
    pin_pos = torch.empty((spec.n, 3), dtype=torch.float32, pin_memory=True)
    pin_vel = torch.empty((spec.n, 3), dtype=torch.float32, pin_memory=True)
    eng.download_all(pin_pos.numpy(), pin_vel.numpy())
    start_state = eng.state()
    eng.run(max(3, args.warmup))
    eng.run(GRAPH_WARMUP)
    builds_before = eng.counters(0)["builds"]
    chains_before = eng.counters()["chain_launches"]
    sampler = ClockSampler(local)
    torch.cuda.synchronize()
    sampler.start()
    t_sample = time.perf_counter()
    profile_region = os.environ.get("BEADS_PROFILE_TIMED") == "1"
    if profile_region:  # lets a profiler started with capture off see only these steps
        torch.cuda.profiler.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    eng.run(args.steps)
    stop.record(stream)
    stop.synchronize()
    if profile_region:
        torch.cuda.profiler.stop()
    clock_extra = 0 if profile_region else _load_until(eng, t_sample, stepping=False)
    clocks = sampler.stop()
    clocks["untimed_force_evaluations_after_timed"] = clock_extra
    ms = start.elapsed_time(stop)
    builds = eng.counters(0)["builds"] - builds_before
    chains = eng.counters()["chain_launches"] - chains_before
    schedule = eng.tuning()
    launches = eng.launch_counts()
    stats = eng.list_stats()
    mean_nbr = stats["entries"] / spec.n

    # The two force kernels timed alone on the current list; the roofline is
    # the slower one's, against its algorithmic bytes per bead.
    pair_ms = eng.profile("pair", 50)
    bonded_ms = eng.profile("bonded", 50)
    pair_bytes = 4.0 * mean_nbr + 36.0
    bonded_bytes = _bonded_bytes_per_bead(spec)
    if bonded_ms >= pair_ms:
        kname, kms, kbytes = "k_bonded (harmonic bonds, angles, dihedrals)", bonded_ms, bonded_bytes
    else:
        kname, kms, kbytes = "k_lj (pair forces)", pair_ms, pair_bytes
    achieved = spec.n * kbytes / (kms / 1e3) / 1e9
    peak, peak_kind = _peaks()

    # End to end through the C ABI with host buffers, as for the mixture,
    # each call from the relaxed start.
    e2e_calls = 0 if args.no_e2e else max(2, args.steps // (4 * E2E_STEPS))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        eng.upload_all(pin_pos.numpy(), pin_vel.numpy())
        eng.run(E2E_STEPS)
        eng.download_all(pin_pos.numpy(), pin_vel.numpy())
    torch.cuda.synchronize()
    e2e_wall = time.perf_counter() - t0
    e2e_value = spec.n * E2E_STEPS * e2e_calls / e2e_wall if e2e_calls else None
    drift = None
    if not args.no_drift:
        try:
            drift = _energy_drift(spec, None, steps=200, every=20, time_unit="tau",
                                  state=start_state)
        except OverflowError as e:
            # Without the thermostat the relaxed melt's released bending
            # energy heats it until a dihedral diverges.
            drift = {"unavailable": f"the NVE copy of the relaxed melt diverged within 200 "
                                    f"steps: {e}"[:300]}
    eng.close()
    line = {
        "metric": CHAINS_METRIC,
        "value": spec.n * args.steps / (ms / 1e3),
        "unit": UNIT,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": "bead-spring melt, 2000 chains x 200 beads, rho 0.85 (relaxed start), "
                        "WCA rc 2^(1/6), "
                        "skin 0.3, bonds/angles/dihedrals, exclusions within 2 bonds, "
                        "Berendsen T 1 tau 1, dt 0.005",
            "parallelism": "none",
            "neighbor_builds_timed": int(builds),
            "graph_warmup_steps": GRAPH_WARMUP,
            "schedule": schedule,
        },
        # pre, decide, pair forces, bonded terms and their gather (+ half-kick),
        # [post,] post finish per step; the rebuild chain (bin, three scan
        # kernels, scatter, cell sorts, two reorder passes, exclusion
        # projection, list build) per rebuild; counted by the engine.
        "gpu_launches": (launches["per_step"] * args.steps
                         + launches["per_rebuild_chain"] * int(chains)),
        "clocks": clocks,
        "roofline": {
            "bound": "hbm",
            "kernel": kname,
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": None,
            "peak_kind": peak_kind,
            "bytes_per_atom": kbytes,
            "kernel_ms": kms,
            "pair_ms": pair_ms,
            "bonded_ms": bonded_ms,
            "pair_bytes_per_atom": pair_bytes,
            "bonded_bytes_per_atom": bonded_bytes,
            "mean_neighbors": round(mean_nbr, 3),
        },
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": 2 * spec.n * 3 * 4 / E2E_STEPS,
                "d2h_bytes_per_step": 2 * spec.n * 3 * 4 / E2E_STEPS,
                "md_steps_per_call": E2E_STEPS, "calls": e2e_calls,
                "call": "beads_upload_all (pinned host positions + velocities) -> "
                        "beads_run(100) -> beads_download_all, per call"},
    }
    if drift is not None:
        line["energy_drift"] = drift
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = _cpu_baseline_melt(spec, args.cpu_budget)
    print(json.dumps(line))


def _bonded_bytes_per_bead(spec) -> float:
    """Algorithmic bytes per bead of the bonded stage (k_bonded_terms, then
    k_bonded), each array element counted once.  Terms: the 16-byte records
    (and 4-byte dihedral types), one 4-byte membership index per member, the
    tag-to-slot map and positions of the beads, one 16-byte contribution
    written per membership.  Gather: the bead's tag and two term offsets,
    the contributions read back, the force read and written."""
    n = spec.n
    nb = 0 if spec.bonds is None else len(spec.bonds)
    na = 0 if spec.angles is None else len(spec.angles)
    nd = 0 if spec.dihedrals is None else len(spec.dihedrals)
    memberships = 2 * nb + 3 * na + 4 * nd
    per_term = 16.0 * (nb + na + nd) + 4.0 * nd + 4.0 * memberships + 16.0 * memberships
    per_gather = 16.0 * memberships
    return (4 + 16) + (4 + 8 + 32) + (per_term + per_gather) / n


def adjoint_metric(world: int) -> str:
    return (f"differentiated atom-steps/s on {world} B200 (64 x 8192-bead LJ mixture, forward "
            "with checkpoints + adjoint backward, FP32 pair math)")


def run_adjoint(args) -> None:
    """The differentiable fit workload: 64 replicas of an 8192-bead binary LJ
    mixture (reduced units, density 0.8, T 1.0 Berendsen tau 1, dt 0.005),
    1000 steps, loss (<PE> - PE*)^2 + (<P> - P*)^2 over the last 200 steps
    with seeded targets, gradients w.r.t. the 3 eps, 3 sigma and the initial
    positions by the adjoint with a checkpoint every 50 steps.  Reports the
    cost of forward + backward against the plain forward run."""
    import torch

    from beads_b200 import workloads
    from beads_b200.adjoint import trajectory_observables
    from beads_b200.engine import Engine

    from beads_b200.distributed import max_over_ranks, reduce_gradients, shard_replicas

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = _init_nccl(world)
    dev = torch.device("cuda", local)
    steps, every = args.adj_steps, 50
    window = min(200, steps)
    # One 64-replica fit, split over the ranks by atom count; the targets are
    # drawn for the whole batch, each rank keeps its replicas' entries.
    all_specs = workloads.fit_mixture(n_replicas=64, n=8192, seed=21)
    rng = np.random.default_rng(5)
    pe_all = rng.uniform(-6.0, -5.0, len(all_specs)) * 8192
    p_all = rng.uniform(0.5, 1.5, len(all_specs))
    mine, specs = shard_replicas(all_specs, world, rank)
    total_atoms = sum(s.n for s in all_specs)
    vols = torch.tensor([float(np.prod(np.asarray(s.box_bound[1], np.float64) - s.box_bound[0]))
                         for s in specs])
    pe_t = torch.tensor(pe_all[mine])
    p_t = torch.tensor(p_all[mine])
    x0 = torch.tensor(np.concatenate([s.positions for s in specs]), dtype=torch.float64)
    v0 = torch.tensor(np.concatenate([s.velocities for s in specs]), dtype=torch.float64)
    eps = torch.tensor(workloads.MIXTURE_EPS, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(specs[0].sigma, dtype=torch.float64, requires_grad=True)
    x = x0.clone().requires_grad_(True)
    with Engine(specs) as eng:
        stream = torch.cuda.ExternalStream(eng.info()["stream"],
                                           device=torch.device("cuda", local))
        eng.run(max(3, args.warmup))
        autotuned_staged = eng.list_staged()
        # One untimed differentiated run of two segments first: it switches
        # the context to the list layout the adjoint reads (slot rows) and
        # instantiates the segment replay graph, so neither the plain nor the
        # differentiated timing below includes graph capture.
        warm = trajectory_observables(eng, eps.detach(), sig.detach().clone().requires_grad_(True),
                                      x0.clone(), v0.clone(), steps=min(2 * every, steps),
                                      record_from=1, checkpoint_every=every)
        warm.sum().backward()
        eng.run(GRAPH_WARMUP)
        # plain forward of the same length from the same start
        eng.upload_all(x0.numpy().astype(np.float32), v0.numpy().astype(np.float32))
        eng.run(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        eng.run(steps)
        b.record(stream)
        b.synchronize()
        plain_s = a.elapsed_time(b) / 1e3
        schedule = eng.tuning()
        # differentiated run (wall clock: host orchestration included)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        obs = trajectory_observables(eng, eps, sig, x, v0.clone(), steps=steps,
                                     record_from=steps - window + 1, checkpoint_every=every)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        pe = obs[:, :, 0].mean(0)
        press = ((2.0 * obs[:, :, 2] + obs[:, :, 1]) / (3.0 * vols)).mean(0)
        loss = ((pe - pe_t) ** 2 + (press - p_t) ** 2).sum()
        loss.backward()
        # eps and sigma are shared by every replica of every rank: sum the
        # ranks' gradients (and losses) with one all-reduce.
        loss_total = loss.detach().clone().reshape(1)
        reduce_gradients([eps.grad, sig.grad, loss_total], dev)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
    fwd_s = max_over_ranks(t1 - t0, dev)
    bwd_s = max_over_ranks(t2 - t1, dev)
    plain_s = max_over_ranks(plain_s, dev)
    # The same gradient with every step's state kept by the forward pass
    # (checkpoint_every = 0, no replay): the memory-for-compute trade that
    # HBM affords at this size ((steps + 1) x 32 B per particle).
    eps2 = eps.detach().clone().requires_grad_(True)
    sig2 = sig.detach().clone().requires_grad_(True)
    x2 = x0.clone().requires_grad_(True)
    with Engine(specs) as eng2:
        eng2.set_tuning(**{k: v for k, v in schedule.items() if k not in ("autotuned", "staged")})
        eng2.set_list_staged(False)
        eng2.run(max(3, args.warmup))
        eng2.run(GRAPH_WARMUP)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        obs2 = trajectory_observables(eng2, eps2, sig2, x2, v0.clone(), steps=steps,
                                      record_from=steps - window + 1, checkpoint_every=0)
        torch.cuda.synchronize()
        t4 = time.perf_counter()
        pe2 = obs2[:, :, 0].mean(0)
        press2 = ((2.0 * obs2[:, :, 2] + obs2[:, :, 1]) / (3.0 * vols)).mean(0)
        ((pe2 - pe_t) ** 2 + (press2 - p_t) ** 2).sum().backward()
        reduce_gradients([eps2.grad, sig2.grad], dev)
        torch.cuda.synchronize()
        t5 = time.perf_counter()
    stored_fwd = max_over_ranks(t4 - t3, dev)
    stored_bwd = max_over_ranks(t5 - t4, dev)
    x_grad_sq = torch.tensor([float(x.grad.norm()) ** 2], dtype=torch.float64)
    reduce_gradients([x_grad_sq], dev)
    if dist is not None:
        dist.destroy_process_group()
    line = {
        "metric": adjoint_metric(world),
        "value": total_atoms * steps / (fwd_s + bwd_s),
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * (fwd_s + bwd_s) / steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": "64 x 8192-bead binary LJ mixture (reduced, rho 0.8, T 1, Berendsen tau 1, "
                        f"dt 0.005), {steps} steps, loss over the last {window} steps, checkpoint "
                        f"every {every}",
            "parallelism": (f"one batch split over {world} GPUs by atom count, gradients "
                            "all-reduced" if world > 1 else "replicas in one batch"),
            "plain_forward_s": plain_s,
            "plain_forward_layout": "slot rows (the adjoint's; the autotuner had picked "
                                    + ("the staged" if autotuned_staged else "the slot")
                                    + " layout)",
            "adjoint_forward_s": fwd_s,
            "backward_s": bwd_s,
            "backward_over_plain_forward": bwd_s / plain_s,
            "forward_plus_backward_over_plain_forward": (fwd_s + bwd_s) / plain_s,
            "stored_forward_s": stored_fwd,
            "stored_backward_s": stored_bwd,
            "stored_backward_over_plain_forward": stored_bwd / plain_s,
            "loss": float(loss_total.item()),
            "grad_eps": eps.grad.tolist(),
            "grad_sigma": sig.grad.tolist(),
            "grad_eps_stored": eps2.grad.tolist(),
            "grad_sigma_stored": sig2.grad.tolist(),
            "grad_x0_norm": float(x_grad_sq.item()) ** 0.5,
        },
    }
    if rank == 0:
        print(json.dumps(line))


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=200)
    parser.add_argument("--warmup", type=int, default=10)
    parser.add_argument("--impl", default="ours", choices=["ours", "reference"])
    parser.add_argument("--cpu-budget", type=float, default=15.0,
                        help="seconds of host work for the cpu_baseline sample")
    parser.add_argument("--no-reference-cuda", action="store_true",
                        help="reference arm: skip timing the reference's own CUDA build")
    parser.add_argument("--reference-cuda-steps", type=int, default=2000,
                        help="reference arm: MD steps of the reference CUDA build's run")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    parser.add_argument("--no-drift", action="store_true", help="skip the energy-drift run")
    parser.add_argument("--adj-steps", type=int, default=1000)
    parser.add_argument("--workload", default="mixture",
                        choices=["mixture", "replicas", "adjoint", "chains"],
                        help="mixture: the 1M-bead mixture (default); replicas: the "
                             "512-replica batch beside one-at-a-time runs; adjoint: the "
                             "differentiable 64-replica fit; chains: the 400,000-bead "
                             "bead-spring melt")
    parser.add_argument("--replicas", type=int, default=512)
    parser.add_argument("--beads", type=int, default=N_BEADS,
                        help="system size (same density); profiling of small cases only")
    args = parser.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        _launch_ranks(args.gpus)
    world = _dist()[0]
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but the launcher started {world} ranks")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "replicas":
        run_replicas(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "chains":
        run_chains(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
