"""Generates tests/golden/small_rhs.json: known answers of the oracle's
right-hand side on 8-triangle basins.

TEST INFRASTRUCTURE: runs the CPU oracle (oracle/) only.  For every tabulated
degree (3-7) and every variant (lin, fs, ns, inv) it sets up the C2 physics on
a 2 x 2 cell basin with the oracle alone (oracle/problems.py), perturbs the
initial state with seeded noise, and records SHA-256 digests of
  * the face traces of u and v (cal_flu, src/calflu.f:6-71: the first phase
    of every variant's right-hand side), (nf, ngf) float64, and
  * the right-hand side itself (cal_var: u1, then v1, then h1, (ne, nm)),
plus their L2 norms for readable diffs.  tests/test_oracle_small_golden.py
holds the oracle to these digests; the GPU parity tests hold the library's
cal_var to them.

Usage:  python tests/golden/make_small_fixtures.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from oracle.problems import (SMALL_DEGREES, SMALL_VARIANTS, oracle_problem, small_case,  # noqa: E402
                             small_case_state)

OUT = HERE / "small_rhs.json"


def digest(*arrays) -> str:
    m = hashlib.sha256()
    for a in arrays:
        m.update(np.ascontiguousarray(a, dtype="<f8").tobytes())
    return m.hexdigest()


def case(nc: int, ng: int, ngf: int, variant: str) -> dict:
    cfg = small_case(nc, ng, ngf, variant)
    P = oracle_problem(cfg)
    u, v, h = small_case_state(P.u, P.v, P.h, nc, variant)
    fu, fv = O.cal_flu(P.T, P.M, u), O.cal_flu(P.T, P.M, v)
    out = O.cal_var(variant, P.T, P.M, u, v, h, P.M.fc, P.w0, P.z0, P.hb, cfg.mu0, cfg.mb0,
                    cfg.g0)
    return {"ne": int(P.M.ne), "nf": int(P.M.nf), "nm": int(P.T.nm),
            "input_sha256": digest(u, v, h),
            "traces_uv_sha256": digest(fu, fv),
            "rhs_sha256": digest(*out),
            "rhs_l2": [float(np.linalg.norm(a)) for a in out]}


def main() -> None:
    rec = {f"p{nc}_{variant}": case(nc, ng, ngf, variant)
           for nc, ng, ngf in SMALL_DEGREES for variant in SMALL_VARIANTS}
    OUT.write_text(json.dumps(rec, indent=1) + "\n")
    print(f"wrote {OUT} ({len(rec)} cases)")


if __name__ == "__main__":
    main()
