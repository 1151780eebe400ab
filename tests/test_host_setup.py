"""Host set-up of the product library against the oracle (no GPU).

Both restate src/shwwnl.f:127-174 in the reference order with separately
rounded products, so tables, mesh pointers and projections agree bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle as O
from spoc_b200 import api, fortran_io
from spoc_b200 import workloads as W

TABLE_CASES = [(3, 12, 4), (4, 25, 5), (5, 27, 6), (6, 33, 7), (7, 42, 9), (2, 6, 3)]


@pytest.mark.parametrize("nc,ng,ngf", TABLE_CASES)
def test_tables_bitwise(nc, ng, ngf):
    T = api.build_tables(nc, ng, ngf)
    OT = O.Tables(nc, ng, ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    for name in ("pi2", "pico", "amm", "amml", "agx", "agy", "ammo", "ammx", "ammy", "cip"):
        assert np.array_equal(getattr(T, name), getattr(OT, name)), name


def test_singular_tables_rejected_with_dpotrf_info():
    with pytest.raises(api.SpocError) as ei:
        api.build_tables(8, 42, 9)
    assert ei.value.code == 4 and "43" in str(ei.value)


@pytest.mark.parametrize("n,jitter", [(3, 0.0), (8, 0.2), (17, 0.2)])
def test_mesh_pointers_bitwise(n, jitter):
    nn, inn, x, y = W.square_mesh(n, 1e6, jitter, seed=5)
    m = api.build_mesh(inn, x, y, 4, 1e-4, 2e-11)
    om = O.Mesh(inn, x, y, 4, 1e-4, 2e-11)
    assert om.check == 0 and om.its_rc == 0
    for name in ("itm", "its", "tseg", "pseg", "ssit", "norm", "vect", "normt", "bdl", "fc"):
        assert np.array_equal(getattr(m, name), getattr(om, name)), name
    assert m.nf == om.nf


@pytest.mark.parametrize("n", [2, 3, 8, 32])
def test_corner_fix_matches_chmal(n):
    nx = n + 1
    cells = np.arange(n * n)
    ne1 = cells % n + 1 + nx * (cells // n)
    inn = np.empty((2 * n * n, 3), np.int32)
    inn[0::2] = np.stack([ne1, ne1 + 1, ne1 + nx], 1)
    inn[1::2] = np.stack([ne1 + 1, ne1 + 1 + nx, ne1 + nx], 1)
    fixed = api.fix_mesh(inn, nx * nx)
    assert np.array_equal(fixed, O.changemaille(inn, nx * nx))
    # after the fix every wall element has exactly one wall face and it is side 1
    x = np.tile(np.arange(nx, dtype=float), nx)
    y = np.repeat(np.arange(nx, dtype=float), nx)
    om = O.Mesh(fixed, x, y, 3)
    assert om.check == 0
    assert om.nebd == 4 * n


def test_workload_sizes_match_the_configurations():
    c = W.CONFIGS
    assert (c["c1_lin_p3"].ne, c["c1_lin_p3"].nm) == (2048, 10)
    assert (c["c2_fs_p6"].ne, c["c2_fs_p6"].nm) == (32768, 28)
    assert (c["c4_ns_p4"].ne, c["c4_ns_p4"].nm) == (32768, 15)
    assert (c["c3_inv_p7"].ne, c["c3_inv_p7"].nm) == (131072, 36)
    nn, inn, x, y = W.square_mesh(128, 1e6, 0.2, seed=2)
    m = api.build_mesh(inn, x, y, 6)
    assert m.nf == 49408 and int(m.bdl.sum()) == 512
    assert (m.det > 0).all()


def test_c1_time_step_is_the_cfl_value():
    p = W.build_problem(W.CONFIGS["c1_lin_p3"])
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, 3)
    cmin, dt = O.checkcfl(3, OM, p.hb, 9.81)
    assert dt == p.dt == 14.0
    assert 14.0 <= cmin < 16.0


def test_projection_bitwise():
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 5))
    T = p.T
    OT = O.Tables(6, 33, 7, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, 6)
    f = lambda x, y: np.sin(x / 3e4) * np.cos(y / 5e4) + 0.1
    ref, px, py = O.calh(OT, OM, f)
    qx, qy = api.projection_points(p.mesh, T)
    assert np.array_equal(px, qx) and np.array_equal(py, qy)
    assert np.array_equal(api.project(T, f(qx, qy)), ref)


def test_state_file_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    ne, nm = 12, 10
    fields = {k: rng.normal(size=(ne, 45)) for k in fortran_io.FIELDS}
    path = tmp_path / "init.bin"
    fortran_io.write_state(path, 86400.0, nm, **fields)
    raw = path.read_bytes()
    # first record: 4-byte length 8, the time, 4-byte length 8
    assert raw[:4] == (8).to_bytes(4, "little") and raw[12:16] == (8).to_bytes(4, "little")
    assert len(raw) == 16 + 6 * (8 + ne * nm * 8)
    t, back = fortran_io.read_state(path, nm)
    assert t == 86400.0
    for k in fortran_io.FIELDS:
        assert np.array_equal(back[k], fields[k][:, :nm])
