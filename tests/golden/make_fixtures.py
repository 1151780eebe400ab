"""Generates the full-size oracle trajectories in tests/golden/.

TEST INFRASTRUCTURE: everything here runs the CPU oracle (oracle/), never the
CUDA library.  For each benchmark configuration it builds the mesh (the rmal
split of the square basin, seeded jitter, the oracle's chmal corner fix), the
tables and the initial state (the oracle's calh projection of the seeded
analytic fields) and the checkcfl time step, all from the oracle, then runs
the reference RK4 loop (src/shwwnl.f:233-284) and records, every `every`
steps, the energy diagnostic of src/energy.f:3-96 (KE, PE, mass, the values
src/shwwnl.f:291-298 writes to oc.energ) and a SHA-256 of the state bytes.

The GPU tests rebuild the same configuration with the library's own set-up
code, check the initial state against the recorded digest (so the set-up is
compared at full size too), step it on the device and compare every record:
state digests bit for bit, energies to the fixed-order-sum tolerance.

Usage (hours of CPU at the full lengths; the oracle uses OpenMP):
    python tests/golden/make_fixtures.py c2_fs_p6 [--steps N] [--every K] [--threads T]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle.problems import oracle_problem  # noqa: E402
from spoc_b200 import workloads as W  # noqa: E402  (configurations: plain Python data)

# default run lengths and record spacing per configuration
PLAN = {
    "c1_lin_p3": (1000, 100),
    "c2_fs_p6": (2000, 100),
    "c3_inv_p7": (200, 20),
    "c4_ns_p4": (200, 20),
}


def state_digest(u, v, h) -> str:
    """SHA-256 of the (ne, nm) float64 C-order bytes of u, then v, then h."""
    m = hashlib.sha256()
    for a in (u, v, h):
        m.update(np.ascontiguousarray(a, dtype="<f8").tobytes())
    return m.hexdigest()


def generate(name: str, steps: int, every: int, threads: int | None) -> dict:
    cfg = W.CONFIGS[name]
    P = oracle_problem(cfg)
    u, v, h = P.u.copy(), P.v.copy(), P.h.copy()
    rec = {
        "config": name, "variant": cfg.variant, "nc": cfg.nc, "ng": cfg.ng, "ngf": cfg.ngf,
        "ne": P.M.ne, "nm": P.T.nm, "dt": P.dt, "steps": steps, "every": every,
        "generator": "tests/golden/make_fixtures.py (CPU oracle, -ffp-contract=off)",
        "digest": "sha256 of the (ne, nm) float64 little-endian bytes of u, v, h",
        "initial_sha256": state_digest(u, v, h),
        "records": [],
    }
    ke, pe, mass = P.energy(u, v, h)
    rec["records"].append({"step": 0, "ke": ke, "pe": pe, "mass": mass,
                           "sha256": rec["initial_sha256"]})
    t0 = time.time()
    done = 0
    while done < steps:
        k = min(every, steps - done)
        P.rk4(u, v, h, k, threads)
        done += k
        ke, pe, mass = P.energy(u, v, h)
        if not np.isfinite([ke, pe, mass]).all():
            raise RuntimeError(f"{name}: non-finite energy at step {done}")
        rec["records"].append({"step": done, "ke": ke, "pe": pe, "mass": mass,
                               "sha256": state_digest(u, v, h)})
        print(f"{name}: step {done}/{steps} ke={ke:.6e} pe={pe:.6e} mass={mass:.6e} "
              f"({time.time() - t0:.0f} s)", flush=True)
    return rec


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("configs", nargs="+", choices=sorted(PLAN))
    ap.add_argument("--steps", type=int)
    ap.add_argument("--every", type=int)
    ap.add_argument("--threads", type=int)
    a = ap.parse_args()
    for name in a.configs:
        steps, every = PLAN[name]
        rec = generate(name, a.steps or steps, a.every or every, a.threads)
        out = HERE / f"{name}_trajectory.json"
        out.write_text(json.dumps(rec, indent=1) + "\n")
        print("wrote", out)


if __name__ == "__main__":
    main()
