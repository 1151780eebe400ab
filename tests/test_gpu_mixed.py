"""Mixed-precision form (FP32 contractions in the orthonormal basis, FP64 RK4
state) against the FP64 path, which is bit-identical to the CPU oracle.

Accuracy bar: relative L2 (mass norm) error of eta <= 1e-5 after 1000 RK4
steps.  The u, v tendencies carry more FP32 error than eta: the DG pressure
gradient and viscous terms are differences of volume and face terms each
~p^2 larger than their sum (measured ~3e-5 relative at degree 6 with a CPU
model of the same arithmetic), so u, v are held to 1e-4.
"""
import numpy as np
import pytest

from oracle import oracle as O
from spoc_b200 import api
from spoc_b200 import workloads as W

NAMES = ["c1_lin_p3", "c2_fs_p6", "c3_inv_p7", "c4_ns_p4"]
# 'templated': FP32 pipes; 'tensor': tcgen05 volume kernel (nonlinear variants)
PATHS = ["templated", "tensor"]


def mixed(p, path="tensor"):
    s = W.make_solver(p, "mixed")
    if path == "tensor" and p.cfg.variant == "lin":
        pytest.skip("the linear variant has no tensor-core kernel")
    s.set_kernel_path(path)
    return s


def rel(T, M, a, b):
    return O.mass_norm(T, M, a - b) / max(O.mass_norm(T, M, b), 1e-300)


def tables(p):
    c = p.cfg
    OT = O.Tables(c.nc, c.ng, c.ngf, p.T.wi, p.T.xi, p.T.yi, p.T.wif, p.T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, c.nc, c.f0, c.beta)
    return OT, OM


@pytest.mark.gpu
@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name", NAMES)
def test_rhs_matches_fp64(name, path):
    """The initial states are in geostrophic balance, where the u, v
    tendencies are small residuals of large cancelling terms; the comparison
    uses an unbalanced state (u reversed)."""
    p = W.build_problem(W.small(W.CONFIGS[name], 8))
    OT, OM = tables(p)
    x = (-p.u, -p.v, p.h)
    ref = W.make_solver(p, "fp64").cal_var(*x)
    mx = mixed(p, path).cal_var(*x)
    for a, b, tol in zip(mx, ref, (1e-4, 1e-4, 1e-5)):
        if O.mass_norm(OT, OM, b) == 0.0:
            assert np.abs(a).max() == 0.0
        else:
            assert rel(OT, OM, a, b) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_state_round_trip(name):
    p = W.build_problem(W.small(W.CONFIGS[name], 6))
    s = W.make_solver(p, "mixed")
    s.set_state(p.u, p.v, p.h)
    for a, b in zip(s.get_state(), (p.u, p.v, p.h)):
        assert np.abs(a - b).max() <= 1e-9 * max(np.abs(b).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name", NAMES)
def test_rk4_steps_match_fp64(name, path):
    p = W.build_problem(W.small(W.CONFIGS[name], 8))
    OT, OM = tables(p)
    out = []
    for prec in ("fp64", "mixed"):
        s = W.make_solver(p, prec) if prec == "fp64" else mixed(p, path)
        s.set_state(p.u, p.v, p.h)
        s.rk4_steps(p.dt, 100)
        out.append(s.get_state())
    for a, b, tol in zip(out[1], out[0], (1e-4, 1e-4, 1e-5)):
        assert rel(OT, OM, a, b) < tol


@pytest.mark.gpu
def test_c1_1000_steps_eta_error():
    """Configuration C1 in full: 2048 triangles, degree 3, 1000 steps."""
    p = W.build_problem(W.CONFIGS["c1_lin_p3"])
    OT, OM = tables(p)
    out = []
    for prec in ("fp64", "mixed"):
        s = W.make_solver(p, prec)
        s.set_state(p.u, p.v, p.h)
        s.rk4_steps(p.dt, 1000)
        out.append(s.get_state())
    assert rel(OT, OM, out[1][2], out[0][2]) < 1e-5


@pytest.mark.gpu
def test_cal_var_keeps_the_resident_state():
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 6))
    s = W.make_solver(p, "mixed")
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 3)
    a = s.get_state()
    s2 = W.make_solver(p, "mixed")
    s2.set_state(p.u, p.v, p.h)
    s2.rk4_steps(p.dt, 2)
    s2.cal_var(p.u * 2, p.v, p.h)
    s2.rk4_steps(p.dt, 1)
    for x, y in zip(a, s2.get_state()):
        assert np.array_equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name", NAMES)
def test_mass_conserved(name, path):
    p = W.build_problem(W.small(W.CONFIGS[name], 8))
    s = mixed(p, path)
    s.set_state(p.u, p.v, p.h)
    m0 = s.energy()[2]
    s.rk4_steps(p.dt, 50)
    m1 = s.energy()[2]
    # mass = sum_e det_e sum_j ammo(j,1) h_j (src/energy.f:327-329); the face
    # values are shared exactly, so only FP32 rounding of the volume and lift
    # terms moves it
    scale = float(np.sum(np.abs(p.mesh.det[:, None] * p.T.ammo[0, :][None, :] * p.h)))
    assert abs(m1 - m0) <= 1e-5 * scale


@pytest.mark.gpu
def test_nonfinite_flag():
    p = W.build_problem(W.small(W.CONFIGS["c4_ns_p4"], 4))
    s = W.make_solver(p, "mixed")
    h = p.h.copy()
    h[3, 0] = np.nan
    with pytest.raises(api.SpocError) as ei:
        s.cal_var(p.u, p.v, h)
    assert ei.value.code == 3
    # the handle stays usable
    s.cal_var(p.u, p.v, p.h)


@pytest.mark.gpu
def test_untabulated_degree_is_rejected():
    p = W.build_problem(W.small(W.CONFIGS["c1_lin_p3"], 4))
    T2 = api.build_tables(3, 25, 5)  # degree 3 with the degree-4 rules: not instantiated
    with pytest.raises(api.SpocError) as ei:
        api.Solver(T2, p.mesh, "lin", "mixed")
    assert ei.value.code == 7


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fs_p6", "c3_inv_p7", "c4_ns_p4"])
def test_tensor_and_fp32_pipes_agree(name):
    """The tcgen05 kernel (three-term TF32 split) and the FP32-FMA kernel
    compute the same right-hand side to FP32 rounding; mesh of 2 x 12 x 12
    elements spans several 128-element tiles and a partial last tile."""
    p = W.build_problem(W.small(W.CONFIGS[name], 12))
    OT, OM = tables(p)
    x = (-p.u, -p.v, p.h)
    a = mixed(p, "templated").cal_var(*x)
    b = mixed(p, "tensor").cal_var(*x)
    ref = W.make_solver(p, "fp64").cal_var(*x)
    for f in range(3):
        # the two FP32 results differ from each other by no more than each
        # differs from FP64
        d = rel(OT, OM, a[f], b[f])
        assert d <= 2.0 * max(rel(OT, OM, a[f], ref[f]), rel(OT, OM, b[f], ref[f])) + 1e-7, (f, d)


@pytest.mark.gpu
def test_tensor_path_refused_for_fp64():
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 4))
    s = W.make_solver(p, "fp64")
    with pytest.raises(api.SpocError) as ei:
        s.set_kernel_path("tensor")
    assert ei.value.code == 7
