"""Times one stage of the step on a named workload, for profilers.

    python -m tests.stage_profile --workload fit-mixture --beads 524288 \
        --stage rebuild --reps 1

Builds the workload, runs ``--warm`` MD steps, then calls
``Engine.profile(stage, reps)`` between cudaProfilerStart and
cudaProfilerStop, so a profiler started with ``--profile-from-start off``
sees exactly those launches.  Prints the mean milliseconds per launch.
Stages: forces, forces_kick, rebuild, step, pair, bonded (see
``Engine.profile``).
"""

from __future__ import annotations

import argparse
import json


def _workload(name: str, beads: int):
    from beads_b200 import workloads

    if name == "fit-mixture":
        return workloads.fit_mixture(n_replicas=1, n=beads, seed=3, max_neighbors=192)[0]
    if name == "lattice":
        side = round(beads ** (1.0 / 3.0))
        return workloads.lj_lattice(n_side=side)
    if name == "replicas":
        return workloads.replica_batch(512)
    if name == "mixture":
        # the benchmark mixture (same density and composition) at `beads`
        # beads, relaxed as the benchmark relaxes it
        box = 37.2 * (beads / 1_048_576) ** (1.0 / 3.0)
        return workloads.relaxed(workloads.lj_mixture(n=beads, box=box, seed=3),
                                 iterations=500, dmax=0.004, fref=200.0, capacity=256)
    if name == "melt":
        # the bead-spring melt benchmark's input: chains of 200, grown in
        # lockstep and relaxed (beads // 200 chains)
        return workloads.relaxed(workloads.polymer_melt(n_chains=max(1, beads // 200), seed=5,
                                                        growth="lockstep"))
    raise ValueError(f"unknown workload {name!r}")


def main(argv: list[str] | None = None) -> dict:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--workload", default="fit-mixture",
                        choices=["fit-mixture", "lattice", "replicas", "melt", "mixture"])
    parser.add_argument("--beads", type=int, default=524288)
    parser.add_argument("--stage", default="rebuild",
                        choices=["forces", "forces_kick", "rebuild", "step", "pair",
                                 "bonded"])
    parser.add_argument("--reps", type=int, default=1)
    parser.add_argument("--warm", type=int, default=20)
    parser.add_argument("--schedule", default="2,0,4,1",
                        help="threads per particle, fused kick, depth, list bypass L1")
    parser.add_argument("--layout", default="staged", choices=["staged", "slot"],
                        help="neighbour-list layout (pair forces from shared-memory cell "
                             "tiles, or gathered from global memory)")
    args = parser.parse_args(argv)

    import torch

    from beads_b200.engine import Engine

    tpa, fuse, depth, bypass = (int(x) for x in args.schedule.split(","))
    with Engine(_workload(args.workload, args.beads)) as eng:
        eng.set_tuning(tpa, bool(fuse), depth, bool(bypass))
        eng.set_list_staged(args.layout == "staged")
        eng.run(args.warm)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        ms = eng.profile(args.stage, args.reps)
        torch.cuda.profiler.stop()
    out = {"workload": args.workload, "stage": args.stage, "reps": args.reps, "ms": ms,
           "layout": args.layout}
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
