"""How the mass solves amplify contraction error (CPU, oracle study mode).

A mixed-precision form would compute the contractions (cal_b, spectoxy,
xytospec, cal_flu, tri_f) on tensor cores in FP32 (TF32 with a hi/lo split at
best) and keep the solves and RK4 in FP64.  The oracle's study mode rounds the
operands of every contraction to float and accumulates in float; this test
records what that does to eta against the FP64 reference.  The P_k1(x) P_k2(y)
basis has cond(amm) = 2.2e5 at degree 4 and 2.1e8 at degree 6, and the solves
amplify the FP32 load-vector error accordingly: the eta error already exceeds
the 1e-5 budget of a 1000-step run within 10 steps at degree 6, and is still
~2e-5 at degree 4.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from spoc_b200 import workloads as W


def eta_error(name, n, steps):
    p = W.build_problem(W.small(W.CONFIGS[name], n))
    T, c = p.T, p.cfg
    OT = O.Tables(c.nc, c.ng, c.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, c.nc, c.f0, c.beta)
    out = []
    L = O.lib()
    try:
        for bits in (64, 32):
            L.ora_set_contraction_precision(bits)
            u, v, h = p.u.copy(), p.v.copy(), p.h.copy()
            O.rk4(c.variant, OT, OM, u, v, h, OM.fc, p.w0, p.z0, p.hb, c.mu0, c.mb0, c.g0, p.dt, steps)
            out.append(h)
    finally:
        L.ora_set_contraction_precision(64)
    return O.mass_norm(OT, OM, out[1] - out[0]) / O.mass_norm(OT, OM, out[0])


def test_fp32_contractions_miss_the_accuracy_budget_at_degree_6():
    err = eta_error("c2_fs_p6", 10, 10)
    assert err > 1e-4  # measured ~2e-3 after 10 steps


def test_fp32_contractions_at_degree_4():
    err = eta_error("c4_ns_p4", 10, 10)
    assert 1e-6 < err < 1e-3  # measured ~2e-5


def test_default_precision_is_restored():
    # the study mode must not leak into other tests: bit-identical reruns
    a = eta_error("c1_lin_p3", 4, 2)
    assert a > 0
    p = W.build_problem(W.small(W.CONFIGS["c1_lin_p3"], 4))
    T, c = p.T, p.cfg
    OT = O.Tables(c.nc, c.ng, c.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, c.nc)
    r1 = O.cal_var("lin", OT, OM, p.u, p.v, p.h, OM.fc, p.w0, p.z0, p.hb, 0, 0, c.g0)
    r2 = O.cal_var("lin", OT, OM, p.u, p.v, p.h, OM.fc, p.w0, p.z0, p.hb, 0, 0, c.g0)
    assert all(np.array_equal(x, y) for x, y in zip(r1, r2))
