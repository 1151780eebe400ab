"""The oracle against its committed known answers on 8-triangle basins
(tests/golden/small_rhs.json, made by tests/golden/make_small_fixtures.py):
every tabulated degree (3-7) and variant, the perturbed input state, the face
traces of u and v (cal_flu) and the right-hand side (cal_var), bit for bit.
A change of the oracle's arithmetic, of its set-up or of the seeded inputs
shows here first."""
import json
from pathlib import Path

import pytest

from oracle import oracle as O
from oracle.problems import (SMALL_DEGREES, SMALL_VARIANTS, oracle_problem, small_case,
                             small_case_state)

GOLDEN = json.loads((Path(__file__).parent / "golden" / "small_rhs.json").read_text())


def _digest(*arrays):
    import hashlib

    import numpy as np
    m = hashlib.sha256()
    for a in arrays:
        m.update(np.ascontiguousarray(a, dtype="<f8").tobytes())
    return m.hexdigest()


@pytest.mark.parametrize("variant", SMALL_VARIANTS)
@pytest.mark.parametrize("deg", SMALL_DEGREES, ids=[f"p{d[0]}" for d in SMALL_DEGREES])
def test_oracle_matches_small_golden(deg, variant):
    nc, ng, ngf = deg
    rec = GOLDEN[f"p{nc}_{variant}"]
    cfg = small_case(nc, ng, ngf, variant)
    P = oracle_problem(cfg)
    assert (P.M.ne, P.M.nf, P.T.nm) == (rec["ne"], rec["nf"], rec["nm"])
    u, v, h = small_case_state(P.u, P.v, P.h, nc, variant)
    assert _digest(u, v, h) == rec["input_sha256"]
    assert _digest(O.cal_flu(P.T, P.M, u), O.cal_flu(P.T, P.M, v)) == rec["traces_uv_sha256"]
    out = O.cal_var(variant, P.T, P.M, u, v, h, P.M.fc, P.w0, P.z0, P.hb, cfg.mu0, cfg.mb0, cfg.g0)
    assert _digest(*out) == rec["rhs_sha256"]


def test_small_golden_covers_every_case():
    assert sorted(GOLDEN) == sorted(f"p{d[0]}_{v}" for d in SMALL_DEGREES for v in SMALL_VARIANTS)
