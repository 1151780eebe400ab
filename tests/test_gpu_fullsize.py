"""Full-size parity: the benchmark configurations at their full sizes and run
lengths, through the C ABI.

* Trajectories against the committed oracle fixtures (tests/golden/
  *_trajectory.json, written by tests/golden/make_fixtures.py from the CPU
  oracle alone): the library's own set-up must reproduce the oracle's initial
  state bit for bit (digest), then every recorded step of the device run must
  have the oracle's state bit for bit (SHA-256 of the u, v, h bytes) and the
  oracle's energy diagnostic (src/energy.f:3-96, the values src/shwwnl.f:
  291-298 writes) to the fixed-order-sum tolerance: 1e-13 relative for the
  positive KE and PE sums, 1e-13 of the summed term magnitudes for the signed
  mass sum (near zero for C3's zero-mean field).  C2 runs its 2000 steps with
  the energy every 100 steps.
* The C4 assimilation window at full size (32768 triangles, degree 4, 200
  steps, 500 observation points at steps 50/100/150/200, 20 binomial
  snapshots): the dot-product test of the 200-step tangent-linear and adjoint
  models, and the gradient against central differences (eps 1e-6) in 20
  seeded random directions.
"""
import functools
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from spoc_b200 import workloads as W

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(GOLDEN.glob("*_trajectory.json"))


@functools.lru_cache(maxsize=None)
def problem(name):
    """Full-size configurations, set up once per test session (C3's initial
    state alone takes about a minute of host time)."""
    return W.build_problem(W.CONFIGS[name])


def mass_scale(p, h):
    """sum_e |det_e| sum_j |ammo(j,1) h_j|: the size of the terms the signed
    mass sum adds (src/energy.f:327-329), the scale of its rounding."""
    return float(np.sum(np.abs(p.mesh.det)[:, None] * np.abs(p.T.ammo[0, :][None, :] * h[:, :p.T.nm])))


def digest(u, v, h, nm):
    m = hashlib.sha256()
    for a in (u, v, h):
        m.update(np.ascontiguousarray(a[:, :nm], dtype="<f8").tobytes())
    return m.hexdigest()


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[f.name.split("_trajectory")[0] for f in FIXTURES])
def test_trajectory_matches_oracle_fixture(gpu_lib, path):
    rec = json.loads(path.read_text())
    p = problem(rec["config"])
    nm = p.T.nm
    assert (p.mesh.ne, nm, p.dt) == (rec["ne"], rec["nm"], rec["dt"])
    assert digest(p.u, p.v, p.h, nm) == rec["initial_sha256"], "set-up differs from the oracle's"
    s = W.make_solver(p)
    s.set_state(p.u, p.v, p.h)
    prev = 0
    for r in rec["records"]:
        if r["step"] > prev:
            s.rk4_steps(p.dt, r["step"] - prev)
            prev = r["step"]
        u, v, h = s.get_state()
        assert digest(u, v, h, nm) == r["sha256"], f"state differs from the oracle at step {prev}"
        ke, pe, mass = s.energy()
        assert ke == pytest.approx(r["ke"], rel=1e-13), f"ke at step {prev}"
        assert pe == pytest.approx(r["pe"], rel=1e-13), f"pe at step {prev}"
        assert abs(mass - r["mass"]) <= 1e-13 * mass_scale(p, h), f"mass at step {prev}"
    assert prev == rec["steps"]


def dot(a, b):
    return sum(float(np.sum(x * y)) for x, y in zip(a, b))


@pytest.fixture(scope="module")
def c4_window(gpu_lib):
    p = problem("c4_ns_p4")
    s = W.make_solver(p)
    W.assimilation_window(p, s, 500, steps=(50, 100, 150, 200))
    yield p, s
    s.close()


@pytest.mark.gpu
def test_c4_full_window_dot_product(c4_window):
    p, s = c4_window
    assert p.mesh.ne == 32768 and p.T.nm == 15
    rng = np.random.default_rng(31)
    x0 = (p.u, p.v, p.h)
    d = tuple(rng.normal(size=a.shape) for a in x0)
    lam = tuple(rng.normal(size=a.shape) for a in x0)
    md = s.tlm_steps(x0, d, p.dt, 200)
    mtl = s.adj_steps(x0, lam, p.dt, 200)
    lhs, rhs = dot(md, lam), dot(d, mtl)
    scale = sum(float(np.sum(np.abs(a * b))) for a, b in zip(md, lam))
    assert abs(lhs - rhs) <= 1e-10 * scale, (lhs, rhs, scale)


@pytest.mark.gpu
def test_c4_full_window_gradient_20_directions(c4_window):
    p, s = c4_window
    nsteps = 200
    x0 = (p.u, p.v, p.h)
    J, g = s.bwd_window(x0, p.dt, nsteps, snaps=20)
    assert J > 0
    assert J == s.fwd_window(x0, p.dt, nsteps)
    rng = np.random.default_rng(2025)
    eps = 1e-6
    worst = 0.0
    for _ in range(20):
        d = tuple(rng.normal(size=a.shape) * (np.sqrt(np.mean(a * a)) + 1e-12) for a in x0)
        jp = s.fwd_window([a + eps * b for a, b in zip(x0, d)], p.dt, nsteps)
        jm = s.fwd_window([a - eps * b for a, b in zip(x0, d)], p.dt, nsteps)
        fd = (jp - jm) / (2 * eps)
        ad = dot(g, d)
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-300))
    assert worst < 1e-5, worst


@pytest.mark.gpu
def test_c4_full_window_mixed_sweeps(c4_window):
    """The C4 gradient with the forward sweeps in the mixed-precision form
    against the FP64 one (measured 7.2e-5 relative, cost 1.6e-6)."""
    p, s = c4_window
    nsteps = 200
    x0 = (p.u, p.v, p.h)
    J64, g64 = s.bwd_window(x0, p.dt, nsteps, snaps=20)
    s.set_adjoint_sweeps("mixed")
    try:
        Jm, gm = s.bwd_window(x0, p.dt, nsteps, snaps=20)
    finally:
        s.set_adjoint_sweeps("fp64")
    assert abs(Jm - J64) <= 1e-5 * J64
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(gm, g64))
    den = sum(float(np.sum(b * b)) for b in g64)
    assert (num / den) ** 0.5 < 5e-4


# Mixed-precision form against FP64 at full size and full run length: the
# north_star bar is eta <= 1e-5 after 1000 steps (C3); the other configurations
# state their errors (bench.py prints them) and are held here to the bounds
# they were measured under, with margin.
MIXED_BOUNDS = {  # name: (steps, eta bound, u/v bound)
    "c1_lin_p3": (1000, 1e-5, 1e-4),
    "c2_fs_p6": (2000, 1e-4, 1e-3),
    "c3_inv_p7": (1000, 1e-5, 1e-4),
    "c4_ns_p4": (200, 1e-4, 1e-3),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(MIXED_BOUNDS))
def test_mixed_errors_full_size(gpu_lib, name):
    steps, eta_tol, uv_tol = MIXED_BOUNDS[name]
    p = problem(name)
    r = W.precision_errors(p, steps)
    err = r["rel_l2_error_vs_fp64"]
    print(name, r)
    assert err["eta"] <= eta_tol, err
    assert err["u"] <= uv_tol and err["v"] <= uv_tol, err
    drift = r["energy_drift"]
    assert abs(drift["mixed"] - drift["fp64"]) <= 5e-2 * abs(drift["fp64"]) + 1e-7, drift
