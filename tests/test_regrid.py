"""Solution-driven regridding on the host and in the oracle (no GPU).

The reference ships no test data for src/adapt.f, so the oracle's regridding
is pinned by properties with exact answers: the re-projection of a field that
is a polynomial of the basis degree is the field's own projection on the new
mesh; on refined elements the children's integrals add up to the parent's;
inherited elements copy their old coefficients bit for bit; the error
indicator of a continuous polynomial vanishes to rounding and flags a planted
jump; verif_rot is a projection (idempotent to rounding); checkcfl2 at rest
is the closed-form bound.  The product's host side (inter_only_new and the
interlin walk) must equal the oracle's bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle as O
from spoc_b200 import api
from spoc_b200 import workloads as W

NAMES = ["c1_lin_p3", "c2_fs_p6", "c4_ns_p4"]


def setup(name, n=8, frac=0.2, seed=0):
    cfg = W.small(W.CONFIGS[name], n)
    p = W.build_problem(cfg)
    T = p.T
    OT = O.Tables(cfg.nc, cfg.ng, cfg.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, cfg.nc, cfg.f0, cfg.beta)
    marked = np.random.default_rng(seed).random(p.mesh.ne) < frac
    p1, tinter, loc = W.adapt_problem(p, marked)
    NM = O.Mesh(p1.mesh.inn, p1.mesh.xgr, p1.mesh.ygr, cfg.nc, cfg.f0, cfg.beta)
    return p, OT, OM, p1, NM, tinter, loc


def integral(OT, OM, a):
    det = OM.vect[:, 0] * OM.vect[:, 3] - OM.vect[:, 2] * OM.vect[:, 1]
    return float(np.sum(det * (a[:, :OT.nm] @ OT.ammo[:, 0])))


@pytest.mark.parametrize("name", NAMES)
def test_host_walk_and_tinter_equal_oracle(name):
    p, OT, OM, p1, NM, tinter, (pe, px, py) = setup(name)
    assert NM.check == 0 and NM.its_rc == 0
    assert np.array_equal(tinter, O.inter_only_new(p.mesh.inn, p1.mesh.inn))
    assert 0 < (tinter > 0).sum() < p1.mesh.ne
    _, le, lx, ly = O.interpol(OT, OM, NM, tinter, p.h)
    m = tinter == 0
    assert np.array_equal(pe[m], le[m])
    assert np.array_equal(px[m], lx[m]) and np.array_equal(py[m], ly[m])
    assert not pe[~m].any()


@pytest.mark.parametrize("name", NAMES)
def test_interpol_inherits_and_conserves(name):
    p, OT, OM, p1, NM, tinter, _ = setup(name)
    un, *_ = O.interpol(OT, OM, NM, tinter, p.h)
    k = tinter > 0
    assert np.array_equal(un[k], p.h[tinter[k] - 1])
    # refinement: children tile their parent, the L2 projection keeps the mean
    i0, i1 = integral(OT, OM, p.h), integral(OT, NM, un)
    assert abs(i1 - i0) <= 1e-13 * abs(i0)


@pytest.mark.parametrize("name", NAMES)
def test_interpol_reproduces_basis_polynomials(name):
    p, OT, OM, p1, NM, tinter, _ = setup(name)
    nc = p.cfg.nc
    L = p.cfg.length

    def f(x, y):
        s, t = x / L, y / L
        return 0.3 + s - 2 * t + s * t + s ** nc - 0.5 * t ** nc

    a_old, _, _ = O.calh(OT, OM, f)
    a_new, _, _ = O.calh(OT, NM, f)
    got, *_ = O.interpol(OT, OM, NM, tinter, a_old)
    err = O.mass_norm(OT, NM, got - a_new) / O.mass_norm(OT, NM, a_new)
    assert err < 1e-11, err


def test_walk_leaves_the_mesh_onto_the_wall():
    """A point outside the basin is moved onto the wall edge the walk crossed."""
    p, OT, OM, *_ = setup("c2_fs_p6")
    L = O.lib()
    import ctypes as C
    tk = C.c_int(1)
    half = 0.5 * p.cfg.length
    x, y = C.c_double(0.3 * half), C.c_double(-1.5 * half)
    lab = np.zeros(3)
    rc = L.ora_interlin(O.i(OM.inn), O.i(OM.itm), O.i(OM.tseg), O.i(OM.pseg), O.d(OM.xgr),
                        O.d(OM.ygr), C.byref(tk), C.byref(x), C.byref(y), O.d(lab), 10000)
    assert rc == 0
    assert abs(y.value + half) < 1e-6 * half and abs(x.value - 0.3 * half) < 1e-6 * half
    assert lab.min() >= 0.0 and abs(lab.sum() - 1.0) < 1e-12


@pytest.mark.parametrize("name", NAMES)
def test_checkconv_polynomial_and_planted_jump(name):
    p, OT, OM, *_ = setup(name)
    L = p.cfg.length
    a, _, _ = O.calh(OT, OM, lambda x, y: 1.0 + x / L + (y / L) ** 2)
    amax = O.checkconv(OT, OM, a)
    assert amax.max() < 1e-9
    b = a.copy()
    e = p.mesh.ne // 2
    b[e, 0] += 0.5
    amax = O.checkconv(OT, OM, b)
    assert amax[e] > 0.1 and np.argmax(amax) in set([e]) | set(
        int(t) - 1 for f in OM.itm[e] for t in OM.tseg[f - 1] if t > 0)
    cc = O.cal_conv(OT, OM, a, a, b, 0.1, 1e-9, 0.4)
    assert cc["fconv"][e] and cc["conv"] and cc["supmax"] == amax.max()
    assert cc["timedir"] == (not (amax.max() > 0.4))


@pytest.mark.parametrize("name", ["c2_fs_p6", "c4_ns_p4"])
def test_verif_rot_is_a_projection(name):
    p, OT, OM, *_ = setup(name)
    u1, v1 = O.verif_rot(OT, OM, p.u, p.v)
    u2, v2 = O.verif_rot(OT, OM, u1, v1)
    nu = O.mass_norm(OT, OM, u1) + O.mass_norm(OT, OM, v1)
    d = O.mass_norm(OT, OM, u2 - u1) + O.mass_norm(OT, OM, v2 - v1)
    assert d <= 1e-9 * nu
    inner = OM.bdl == 0
    assert O.mass_norm(OT, OM, np.where(inner[:, None], u1 - p.u, 0.0)) <= 1e-9 * nu


def test_checkcfl2_at_rest_matches_closed_form():
    p, OT, OM, *_ = setup("c2_fs_p6")
    z = np.zeros_like(p.u)
    cmin, dt = O.checkcfl2(p.cfg.nc, OM, p.hb, z, z, p.cfg.g0)
    x, y, inn = OM.xgr, OM.ygr, OM.inn - 1
    best = 6000.0
    for a, b in ((0, 1), (0, 2), (1, 2)):
        dd = np.hypot(x[inn[:, b]] - x[inn[:, a]], y[inn[:, b]] - y[inn[:, a]]) / p.cfg.nc * 0.35
        best = min(best, float(np.min(dd / np.sqrt(p.cfg.g0 * p.cfg.depth))))
    assert abs(cmin - best) <= 1e-13 * best
    if best >= 100:
        assert dt == float(10 * int(cmin / 10))
    elif best >= 10:
        assert dt == float(2 * int(cmin / 2))
    elif best >= 1:
        assert dt == float(int(cmin))
    else:
        assert dt == 0.0  # the reference's integer division


def test_fortran_e_format():
    from spoc_b200.fortran_io import fortran_e
    cases = {0.0: " 0.000E+00", 1234.5: " 0.123E+04", -1234.5: "-0.123E+04",
             0.00012345: " 0.123E-03", 9999.6: " 0.100E+05", 1e100: " 0.100+101", 1.0: " 0.100E+01"}
    for v, s in cases.items():
        assert fortran_e(v) == s, (v, fortran_e(v))


def test_write_gra_layout(tmp_path):
    from spoc_b200.fortran_io import write_gra, gra_name
    lat = np.zeros((2, 3, 5))
    lat[..., 0] = 1.5e5
    lat[..., 4] = -2.0
    path = tmp_path / gra_name("h", 12)
    write_gra(path, lat, 2)
    lines = path.read_text().splitlines()
    assert path.name == "h12.gra" and len(lines) == 6
    assert lines[0] == " 0.150E+06  0.000E+00 -0.200E+01 "


def test_host_locate_xy_equals_oracle_walk():
    p, OT, OM, *_ = setup("c2_fs_p6")
    rng = np.random.default_rng(3)
    half = 0.5 * p.cfg.length
    px = rng.uniform(-half, half, 300)
    py = rng.uniform(-half, half, 300)
    elem, x1, y1, inside, tk = api.locate_xy(p.mesh, px, py, 1, 1)
    t = 1
    for i in range(px.size):
        t, _, _, lab = O.interlin(OM, t, px[i], py[i])
        assert inside[i] == 1 and elem[i] == t
        assert x1[i] == 2.0 * lab[1] - 1.0 and y1[i] == 2.0 * lab[2] - 1.0
    assert tk == t
