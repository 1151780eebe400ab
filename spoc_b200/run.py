"""Runs RK4 steps of one of the benchmark configurations on the GPU.

    python -m spoc_b200.run --config c2_fs_p6 --steps 2 [--precision fp64|fp64_fma|mixed]
        [--path auto|generic|templated|tensor] [--steps-per-call 1]

Builds the configuration (spoc_b200.workloads.CONFIGS), sets the state, runs
the steps (one spoc_rk4_steps call per --steps-per-call steps) and prints the
kernel launches and the energy diagnostic.  A small, self-contained workload
for profilers: every launch of a step is one of the library's kernels.
"""
from __future__ import annotations

import argparse

from . import workloads as W


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c2_fs_p6", choices=sorted(W.CONFIGS))
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--steps-per-call", type=int, default=1)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp64_fma", "mixed"])
    ap.add_argument("--path", default="auto", choices=["auto", "generic", "templated", "tensor"])
    a = ap.parse_args()
    p = W.build_problem(W.CONFIGS[a.config])
    s = W.make_solver(p, a.precision)
    s.set_kernel_path(a.path)
    s.set_state(p.u, p.v, p.h)
    done = 0
    while done < a.steps:
        k = min(a.steps_per_call, a.steps - done)
        s.rk4_steps(p.dt, k)
        done += k
    ke, pe, mass = s.energy()
    print(f"{a.config}: {done} steps, {s.launches} kernel launches, ke={ke:.9e} pe={pe:.9e} "
          f"mass={mass:.9e}")
    s.close()


if __name__ == "__main__":
    main()
