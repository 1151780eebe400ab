"""Tangent-linear model, adjoint and gradient on the GPU (through the C ABI).

Checks: the dot-product test <J d, l> = <d, J^T l> for the right-hand side and
for RK4 steps, the tangent-linear model against central differences of the
forward model, the cost of the forward window against the observation
operator applied to the forward trajectory, the gradient against central
finite differences (eps = 1e-6) in 20 seeded random directions, and the
gradient with binomial checkpointing against the gradient that stores every
state (identical kernels, identical arithmetic: bit for bit).
"""
import numpy as np
import pytest

from spoc_b200 import workloads as W

NAMES = ["c4_ns_p4", "c2_fs_p6", "c3_inv_p7", "c1_lin_p3"]


def variant_at(name, variant, n=6):
    """Configuration `name` with another physics variant (same degree and tables)."""
    import dataclasses
    return W.build_problem(dataclasses.replace(W.small(W.CONFIGS[name], n), variant=variant))


def dot(a, b):
    return sum(float(np.sum(x * y)) for x, y in zip(a, b))


def rand_like(rng, x, scale=1.0):
    return tuple(scale * rng.normal(size=a.shape) for a in x)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_rhs_dot_product(name):
    p = W.build_problem(W.small(W.CONFIGS[name], 6))
    s = W.make_solver(p)
    rng = np.random.default_rng(21)
    x = (p.u, p.v, p.h)
    d = rand_like(rng, x)
    lam = rand_like(rng, x)
    jd = s.tlm_rhs(x, d)
    jtl = s.adj_rhs(x, lam)
    lhs, rhs = dot(jd, lam), dot(d, jtl)
    scale = sum(float(np.sum(np.abs(a * b))) for a, b in zip(jd, lam))
    assert abs(lhs - rhs) <= 1e-11 * scale, (lhs, rhs, scale)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c4_ns_p4", "c1_lin_p3"])
@pytest.mark.parametrize("variant", ["fs", "ns", "inv"])
def test_rhs_dot_product_low_degrees(name, variant):
    """Degrees 3 and 4 run the two-elements-per-warp adjoint kernels: every
    nonlinear variant, wall elements included."""
    p = variant_at(name, variant)
    s = W.make_solver(p)
    rng = np.random.default_rng(22)
    x = (p.u, p.v, p.h)
    d = rand_like(rng, x)
    lam = rand_like(rng, x)
    jd = s.tlm_rhs(x, d)
    jtl = s.adj_rhs(x, lam)
    lhs, rhs = dot(jd, lam), dot(d, jtl)
    scale = sum(float(np.sum(np.abs(a * b))) for a, b in zip(jd, lam))
    assert abs(lhs - rhs) <= 1e-11 * scale, (lhs, rhs, scale)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_tlm_matches_central_differences(name):
    p = W.build_problem(W.small(W.CONFIGS[name], 6))
    s = W.make_solver(p)
    rng = np.random.default_rng(5)
    x = (p.u, p.v, p.h)
    d = tuple(a * 0 + rng.normal(size=a.shape) * (np.abs(a).max() + 1e-3) for a in x)
    eps = 1e-6
    fp = s.cal_var(*[a + eps * b for a, b in zip(x, d)])
    fm = s.cal_var(*[a - eps * b for a, b in zip(x, d)])
    fd = [(a - b) / (2 * eps) for a, b in zip(fp, fm)]
    jd = s.tlm_rhs(x, d)
    # central differences carry O(eps^2) truncation and round-off / eps; the
    # round-off of the right-hand side grows with cond(amm) (6.5e9 at degree 7)
    for a, b in zip(jd, fd):
        assert np.abs(a - b).max() <= 1e-5 * max(np.abs(b).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c4_ns_p4", "c2_fs_p6", "c1_lin_p3"])
def test_rk4_steps_dot_product(name):
    p = W.build_problem(W.small(W.CONFIGS[name], 5))
    s = W.make_solver(p)
    rng = np.random.default_rng(8)
    x0 = (p.u, p.v, p.h)
    d = rand_like(rng, x0)
    lam = rand_like(rng, x0)
    md = s.tlm_steps(x0, d, p.dt, 4)
    mtl = s.adj_steps(x0, lam, p.dt, 4)
    lhs, rhs = dot(md, lam), dot(d, mtl)
    scale = sum(float(np.sum(np.abs(a * b))) for a, b in zip(md, lam))
    assert abs(lhs - rhs) <= 1e-10 * scale, (lhs, rhs)


def _assimilation_problem(nsteps=20, nobs=60, n=8):
    """C4 physics (no-slip, p4) on a small basin: truth run from a shifted
    state, eta observed at seeded points every nsteps/4 steps."""
    p = W.build_problem(W.small(W.CONFIGS["c4_ns_p4"], n))
    s = W.make_solver(p)
    elem, basis, _, _ = W.random_observations(p, nobs, seed=44)
    steps = np.array([nsteps // 4 * k for k in range(1, 5)], dtype=np.int32)
    rng = np.random.default_rng(9)
    truth = (p.u * 1.05, p.v * 0.95, p.h + 0.02 * rng.normal(size=p.h.shape) * (np.arange(p.h.shape[1]) < 3))
    s.set_state(*truth)
    vals, t_prev = [], 0
    for st in steps:
        s.rk4_steps(p.dt, int(st - t_prev))
        t_prev = st
        _, _, h = s.get_state()
        vals.append(np.sum(h[elem - 1] * basis, axis=1))
    s.set_observations(elem, basis, steps, np.array(vals))
    return p, s, elem, basis, steps, np.array(vals)


@pytest.mark.gpu
def test_cost_matches_observation_operator():
    nsteps = 20
    p, s, elem, basis, steps, vals = _assimilation_problem(nsteps)
    x0 = (p.u, p.v, p.h)
    J = s.fwd_window(x0, p.dt, nsteps)
    s.set_state(*x0)
    ref, t_prev = 0.0, 0
    for k, st in enumerate(steps):
        s.rk4_steps(p.dt, int(st - t_prev))
        t_prev = st
        _, _, h = s.get_state()
        r = np.sum(h[elem - 1] * basis, axis=1) - vals[k]
        ref += 0.5 * float(np.sum(r * r))
    assert J == pytest.approx(ref, rel=1e-12)
    assert J > 0


@pytest.mark.gpu
def test_gradient_finite_differences_20_directions():
    nsteps = 20
    p, s, *_ = _assimilation_problem(nsteps)
    x0 = (p.u, p.v, p.h)
    J, g = s.bwd_window(x0, p.dt, nsteps, snaps=5)
    rng = np.random.default_rng(2024)
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
def test_checkpointing_gives_the_stored_trajectory_gradient():
    nsteps = 20
    p, s, *_ = _assimilation_problem(nsteps)
    x0 = (p.u, p.v, p.h)
    J1, g1 = s.bwd_window(x0, p.dt, nsteps, snaps=2)
    f1, a1 = s.adjoint_counters()
    J2, g2 = s.bwd_window(x0, p.dt, nsteps, snaps=nsteps)
    f2, a2 = s.adjoint_counters()
    assert J1 == J2
    for a, b in zip(g1, g2):
        assert np.array_equal(a, b)
    assert a1 == a2 == nsteps
    assert f1 > f2  # fewer snapshots, more recomputation


def _rel(a, b):
    num = sum(float(np.sum((x - y) ** 2)) for x, y in zip(a, b))
    return (num / sum(float(np.sum(y * y)) for y in b)) ** 0.5


@pytest.mark.gpu
def test_mixed_precision_sweeps():
    """Forward sweeps of the window in the mixed-precision form: the gradient
    stays within 1e-3 of the FP64-sweep gradient (measured 1.6e-4 on this
    window: the residuals are a few percent of the state, so the mixed form's
    1e-6-level state error shows up enlarged), the tangent-linear / adjoint
    pair about the mixed trajectory still passes the dot-product test, and
    switching back gives the FP64 gradient bit for bit."""
    nsteps = 20
    p, s, *_ = _assimilation_problem(nsteps)
    x0 = (p.u, p.v, p.h)
    J64, g64 = s.bwd_window(x0, p.dt, nsteps, snaps=5)
    s.set_adjoint_sweeps("mixed")
    Jm, gm = s.bwd_window(x0, p.dt, nsteps, snaps=5)
    assert Jm != J64 and abs(Jm - J64) <= 1e-3 * J64
    assert _rel(gm, g64) < 1e-3
    rng = np.random.default_rng(17)
    d = rand_like(rng, x0)
    lam = rand_like(rng, x0)
    md = s.tlm_steps(x0, d, p.dt, nsteps)
    mtl = s.adj_steps(x0, lam, p.dt, nsteps)
    lhs, rhs = dot(md, lam), dot(d, mtl)
    scale = sum(float(np.sum(np.abs(a * b))) for a, b in zip(md, lam))
    assert abs(lhs - rhs) <= 1e-10 * scale, (lhs, rhs)
    s.set_adjoint_sweeps("fp64")
    J2, g2 = s.bwd_window(x0, p.dt, nsteps, snaps=5)
    assert J2 == J64
    assert all(np.array_equal(a, b) for a, b in zip(g2, g64))
