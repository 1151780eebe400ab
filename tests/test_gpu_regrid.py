"""GPU parity of the regridding kernels against the CPU oracle, through the C ABI.

checkconv / cal_conv, interpol, verif_rot and checkcfl2 run every sum in the
reference order with separately rounded products and take their maxima /
minima exactly, so they are compared bit for bit (np.array_equal).
"""
import numpy as np
import pytest

from oracle import oracle as O
from spoc_b200 import api
from spoc_b200 import workloads as W

NAMES = ["c1_lin_p3", "c2_fs_p6", "c4_ns_p4", "c3_inv_p7"]


def setup(name, n=8, frac=0.2, seed=0):
    cfg = W.small(W.CONFIGS[name], n)
    p = W.build_problem(cfg)
    T = p.T
    OT = O.Tables(cfg.nc, cfg.ng, cfg.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, cfg.nc, cfg.f0, cfg.beta)
    return p, OT, OM


def stepped(p, n=3):
    """A state with jumps between elements: a few RK4 steps from the projection."""
    s = W.make_solver(p)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, n)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_checkconv_and_cal_conv_bitwise(gpu_lib, name):
    p, OT, OM = setup(name)
    s = stepped(p)
    u, v, h = s.get_state()
    got = s.checkconv()
    for g, a in zip(got, (u, v, h)):
        assert np.array_equal(g, O.checkconv(OT, OM, a))
    amax = np.maximum.reduce(got)
    fac1 = float(np.quantile(amax, 0.8))
    fac2 = float(np.quantile(amax, 0.1))
    cc = s.cal_conv(fac1, fac2, fac1 * 2)
    ref = O.cal_conv(OT, OM, u, v, h, fac1, fac2, fac1 * 2)
    assert np.array_equal(cc["fconv"], ref["fconv"]) and np.array_equal(cc["fderaff"], ref["fderaff"])
    assert cc["supmax"] == ref["supmax"]
    assert (cc["conv"], cc["deraff"], cc["timedir"]) == (ref["conv"], ref["deraff"], ref["timedir"])
    assert 0 < cc["fconv"].sum() < p.mesh.ne


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_interpol_bitwise(gpu_lib, name):
    p, OT, OM = setup(name)
    s = stepped(p)
    u, v, h = s.get_state()
    marked = np.random.default_rng(1).random(p.mesh.ne) < 0.25
    p1, tinter, loc = W.adapt_problem(p, marked)
    NM = O.Mesh(p1.mesh.inn, p1.mesh.xgr, p1.mesh.ygr, p.cfg.nc, p.cfg.f0, p.cfg.beta)
    d = api.Solver(p1.T, p1.mesh, p.cfg.variant)
    d.set_params(p.cfg.mu0, p.cfg.mb0, p.cfg.g0, p1.hb, p1.fc, p1.w0, p1.z0)
    d.interpol_from(s, tinter, *loc)
    got = d.get_state()
    for g, a in zip(got, (u, v, h)):
        ref, *_ = O.interpol(OT, OM, NM, tinter, a)
        assert np.array_equal(g, ref)


@pytest.mark.gpu
def test_interpol_all_inherited_needs_no_points(gpu_lib):
    p, OT, OM = setup("c2_fs_p6")
    s = stepped(p)
    d = W.make_solver(p)
    d.interpol_from(s, np.arange(1, p.mesh.ne + 1, dtype=np.int32))
    for g, a in zip(d.get_state(), s.get_state()):
        assert np.array_equal(g, a)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fs_p6", "c4_ns_p4", "c3_inv_p7"])
def test_verif_rot_bitwise(gpu_lib, name):
    p, OT, OM = setup(name)
    s = stepped(p)
    u, v, h = s.get_state()
    s.verif_rot()
    gu, gv, gh = s.get_state()
    ru, rv = O.verif_rot(OT, OM, u, v)
    assert np.array_equal(gu, ru) and np.array_equal(gv, rv) and np.array_equal(gh, h)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("ngraph", [10, 4])
def test_cfl2_bitwise(gpu_lib, name, ngraph):
    p, OT, OM = setup(name)
    s = stepped(p)
    u, v, h = s.get_state()
    got = s.cfl2(ngraph, 7.0)
    ref = O.checkcfl2(p.cfg.nc, OM, p.hb, u, v, p.cfg.g0, ngraph, 7.0)
    assert got == ref


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fs_p6", "c4_ns_p4"])
def test_regrid_step_matches_oracle_pipeline(gpu_lib, name):
    p, OT, OM = setup(name)
    s = stepped(p, 5)
    u, v, h = s.get_state()
    amax = np.maximum.reduce(s.checkconv())
    fac1 = float(np.quantile(amax, 0.85))
    p1, s1, info = W.regrid_step(p, s, fac1, 0.0, 10 * fac1)
    assert info["flagged"] > 0 and info["ne_new"] > info["ne_old"]
    NM = O.Mesh(p1.mesh.inn, p1.mesh.xgr, p1.mesh.ygr, p.cfg.nc, p.cfg.f0, p.cfg.beta)
    tinter = O.inter_only_new(p.mesh.inn, p1.mesh.inn)
    ru, *_ = O.interpol(OT, OM, NM, tinter, u)
    rv, *_ = O.interpol(OT, OM, NM, tinter, v)
    rh, *_ = O.interpol(OT, OM, NM, tinter, h)
    ru, rv = O.verif_rot(OT, NM, ru, rv)
    gu, gv, gh = s1.get_state()
    assert np.array_equal(gu, ru) and np.array_equal(gv, rv) and np.array_equal(gh, rh)
    cmin, dt = O.checkcfl2(p.cfg.nc, NM, p1.hb, ru, rv, p.cfg.g0, 10, p.dt)
    assert (info["cflmin"], info["dt_cfl2"]) == (cmin, dt)
    # the refined run steps on
    s1.rk4_steps(p1.dt, 3)
    assert all(np.isfinite(a).all() for a in s1.get_state())


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fs_p6", "c4_ns_p4"])
def test_regrid_coarsening_matches_oracle_pipeline(gpu_lib, name):
    """A refined patch flagged calm by cal_conv's fderaff is coarsened
    (deraffiner through the refinement history) and the device re-projection,
    verif_rot and checkcfl2 equal the oracle's bit for bit."""
    p, OT, OM = setup(name)
    s = stepped(p, 5)
    amax = np.maximum.reduce(s.checkconv())
    fac1 = float(np.quantile(amax, 0.85))
    p1, s1, info = W.regrid_step(p, s, fac1, 0.0, 10 * fac1)
    assert info["refined"] > 0 and info["coarsened"] == 0
    s1.rk4_steps(p1.dt, 2)
    u, v, h = s1.get_state()
    amax1 = np.maximum.reduce(s1.checkconv())
    fac2 = float(np.quantile(amax1, 0.97))
    p2, s2, info2 = W.regrid_step(p1, s1, 1e300, fac2, 1e301)
    assert info2["refined"] == 0 and info2["coarsened"] > 0 and p2.mesh.ne < p1.mesh.ne
    M1 = O.Mesh(p1.mesh.inn, p1.mesh.xgr, p1.mesh.ygr, p.cfg.nc, p.cfg.f0, p.cfg.beta)
    M2 = O.Mesh(p2.mesh.inn, p2.mesh.xgr, p2.mesh.ygr, p.cfg.nc, p.cfg.f0, p.cfg.beta)
    tinter = info2["tinter"]
    assert 0 < (tinter > 0).sum() < p2.mesh.ne
    ru, *_ = O.interpol(OT, M1, M2, tinter, u)
    rv, *_ = O.interpol(OT, M1, M2, tinter, v)
    rh, *_ = O.interpol(OT, M1, M2, tinter, h)
    ru, rv = O.verif_rot(OT, M2, ru, rv)
    gu, gv, gh = s2.get_state()
    assert np.array_equal(gu, ru) and np.array_equal(gv, rv) and np.array_equal(gh, rh)
    cmin, dt = O.checkcfl2(p.cfg.nc, M2, p2.hb, ru, rv, p.cfg.g0, 10, p1.dt)
    assert (info2["cflmin"], info2["dt_cfl2"]) == (cmin, dt)
    s2.rk4_steps(p2.dt, 3)
    assert all(np.isfinite(a).all() for a in s2.get_state())


@pytest.mark.gpu
def test_regrid_mixed_handles(gpu_lib):
    """SPOC_MIXED handles keep their state in their own basis; the regrid moves
    it through FP64 and back (a round trip through the ill-conditioned basis
    change, 1e-12 relative here)."""
    p, OT, OM = setup("c2_fs_p6")
    s = stepped(p)
    m = W.make_solver(p, "mixed")
    m.set_state(*s.get_state())
    amax = np.maximum.reduce(s.checkconv())
    cc = s.cal_conv(float(np.quantile(amax, 0.85)), 0.0, 1.0)
    p1, tinter, loc = W.adapt_problem(p, cc["fconv"])
    NM = O.Mesh(p1.mesh.inn, p1.mesh.xgr, p1.mesh.ygr, p.cfg.nc, p.cfg.f0, p.cfg.beta)
    out = []
    for src, prec in ((s, "fp64"), (m, "mixed")):
        d = api.Solver(p1.T, p1.mesh, p.cfg.variant, prec)
        d.set_params(p.cfg.mu0, p.cfg.mb0, p.cfg.g0, p1.hb, p1.fc, p1.w0, p1.z0)
        d.interpol_from(src, tinter, *loc)
        d.verif_rot()
        out.append(d.get_state())
    for a, b in zip(*out):
        assert O.mass_norm(OT, NM, a - b) <= 1e-10 * O.mass_norm(OT, NM, a)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_eval_points_and_lattice_bitwise(gpu_lib, name):
    p, OT, OM = setup(name)
    s = stepped(p)
    u, v, h = s.get_state()
    rng = np.random.default_rng(4)
    n = 500
    elem = rng.integers(1, p.mesh.ne + 1, n).astype(np.int32)
    a = rng.uniform(-1, 1, n)
    b = rng.uniform(-1, 1, n)
    px, py = np.minimum(a, -b), np.maximum(b, -1.0)  # inside the reference triangle
    got = s.eval_points(elem, px, py)
    assert np.array_equal(got, O.eval_points(p.cfg.nc, u, v, h, elem, px, py))
    for ng in (10, 5):
        assert np.array_equal(s.lattice(ng), O.lattice(p.cfg.nc, OM, u, v, h, ng))


@pytest.mark.gpu
def test_compare_standing_wave(gpu_lib):
    """compare.f's norms: the device evaluation gives the oracle's numbers, and
    the projection of the analytic wave itself is close to it."""
    p, OT, OM = setup("c1_lin_p3", n=16)
    L = p.cfg.length
    pi = 4.0 * np.arctan(1.0)
    uc = np.sin(0.2 * pi) * p.cfg.g0 / np.sqrt(10.0)
    hc = np.cos(0.2 * pi)
    u, _, _ = O.calh(OT, OM, lambda x, y: uc * np.sin(2 * pi * x / L))
    hh, _, _ = O.calh(OT, OM, lambda x, y: hc * np.cos(2 * pi * x / L))
    z = np.zeros_like(u)
    s = W.make_solver(p)
    s.set_state(u, z, hh)
    got = W.compare_standing_wave(p, s, 41, 41)

    class OracleEval:
        def eval_points(self, elem, px, py):
            return O.eval_points(p.cfg.nc, u, z, hh, elem, px, py)

    ref = W.compare_standing_wave(p, OracleEval(), 41, 41)
    assert got == ref
    assert got["inside"] == 40 * 40 and got["outside"] == 0
    assert got["rms_norm"][2] < 1e-3 * hc and got["rms_norm"][1] == 0.0


@pytest.mark.gpu
def test_interpol_dev_rejects_bad_ids(gpu_lib):
    """Device point tables are not validated on the host: ids outside the
    source mesh are skipped by the kernel (never read) and the call returns
    SPOC_E_ARG; the handle stays usable."""
    import torch
    p, OT, OM = setup("c2_fs_p6")
    s = stepped(p)
    d = W.make_solver(p)
    ne, ng = p.mesh.ne, p.T.ng
    tinter = np.zeros(ne, np.int32)
    tinter[0] = ne + 5                                   # out of range
    pel = np.full((ne, ng), 1, np.int32)
    pel[1, 3] = -2                                       # out of range
    xy = np.full((ne, ng), -0.5)
    dev = [torch.from_numpy(a).cuda() for a in (tinter, pel, xy, xy.copy())]
    with pytest.raises(api.SpocError) as ei:
        d.interpol_from_dev(s, *[t.data_ptr() for t in dev])
    assert ei.value.code == 1  # SPOC_E_ARG
    d.interpol_from(s, np.arange(1, ne + 1, dtype=np.int32))
    for g, a in zip(d.get_state(), s.get_state()):
        assert np.array_equal(g, a)
