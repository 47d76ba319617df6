"""Step one synthetic workload through a batch, for profiling and smoke runs.

    PYTHONPATH=teuk-kokkos_b200 python -m teuk_b200.batch_run \
        --workload extremal --solves 24 --steps 3

Workloads (teuk_b200.workloads): ``ringdown`` (Kerr a = 0.7, nr 1025,
ell <= 16, 25 nodes), ``extremal`` (a = 0.99, ell <= 24, 37 nodes; nr 1025
unless --radial-points), ``uneven`` (the seeded draw of uneven solves),
``second_order`` (the quadratic-source self-coupling solve, source on from
t = 0: the solves of the batch are replicas of one nodal pipeline).
The batch is built with the default launch options (no autotuning, so the
launch sequence is fixed: build, initial data, then four stage launches per
streaming or tile group and RK4 step) and stepped from a CUDA graph.  It
prints the stage-kernel groups, the strip lengths and the band values.
"""
from __future__ import annotations

import argparse
from dataclasses import replace

import teuk_b200 as tb
from teuk_b200 import workloads as wl


def build(workload: str, solves: int, radial_points: int):
    if workload == "uneven":
        draw = wl.uneven_batch(solves)
        return ([c for c, _, _ in draw], [p for _, p, _ in draw],
                [d for _, _, d in draw])
    if workload == "second_order":
        config, pulse, dt = wl.second_order_self_coupling(
            radial_points=radial_points)
        return [config] * solves, [pulse] * solves, [dt] * solves
    if workload == "extremal":
        base, pulse, _ = wl.extremal_kerr()
    elif workload == "ringdown":
        base, pulse, _ = wl.kerr_ringdown()
    else:
        raise SystemExit(f"unknown workload {workload!r}")
    config = replace(base, radial_points=radial_points)
    dt = wl.time_step(config, 0.25)
    sigma = min(0.005, 0.9 * wl.dissipation_bound(config.discretization,
                                                  dt / config.spacing))
    config = replace(config, dissipation=sigma)
    return [config] * solves, [pulse] * solves, [dt] * solves


def main() -> None:
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--workload", default="extremal",
                   choices=["ringdown", "extremal", "uneven", "second_order"])
    p.add_argument("--solves", type=int, default=24)
    p.add_argument("--radial-points", type=int, default=1025)
    p.add_argument("--steps", type=int, default=3)
    args = p.parse_args()
    configs, pulses, dts = build(args.workload, args.solves, args.radial_points)
    batch = tb.Batch(configs)
    for i, pulse in enumerate(pulses):
        batch.initialize_gaussian(i, pulse)
    batch.step(dts, args.steps)
    batch.synchronize()
    if args.workload == "second_order":
        print(f"second_order: {len(configs)} replicas of one nodal pipeline, "
              f"{sum(wl.grid_points(c) for c in configs)} grid points")
        return
    values = sum(wl.modal_values(c) for c in configs)
    print(f"{args.workload}: {len(configs)} solves, stage kernel groups "
          f"{batch.stage_kernels()}, strip rows {batch.strip_rows()}, "
          f"{values} band values per buffer")


if __name__ == "__main__":
    main()
