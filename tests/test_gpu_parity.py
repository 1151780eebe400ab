"""GPU parity: the CUDA path against the CPU oracle, through the C ABI.

The FP64 path evaluates every sum in the reference order with separately
rounded products, so the comparison is bit-for-bit (np.array_equal) for the
right-hand side, the RK4 steps and the CFL bound; the energy diagnostic is
summed in a different order (fixed-order tree) and is compared at 1e-13
relative.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from spoc_b200 import api
from spoc_b200 import workloads as W

NAMES = ["c1_lin_p3", "c2_fs_p6", "c4_ns_p4", "c3_inv_p7"]


def oracle_for(p):
    T = p.T
    OT = O.Tables(p.cfg.nc, p.cfg.ng, p.cfg.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(p.mesh.inn, p.mesh.xgr, p.mesh.ygr, p.cfg.nc, p.cfg.f0, p.cfg.beta,
                ld=p.u.shape[1])
    return OT, OM


def oracle_rhs(p, OT, OM, u, v, h):
    c = p.cfg
    return O.cal_var(c.variant, OT, OM, u, v, h, OM.fc, p.w0, p.z0, p.hb, c.mu0, c.mb0, c.g0)


def assert_bitwise(got, ref, nm):
    for g, r in zip(got, ref):
        g, r = g[:, :nm], r[:, :nm]
        bad = ~((g == r) | (np.isnan(g) & np.isnan(r)))
        assert not bad.any(), f"{bad.sum()} coefficients differ; max |d| = {np.abs(g - r).max():.3e}"


PATHS = ["generic", "templated"]


@pytest.mark.gpu
@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("ld", [None, 45])
def test_cal_var_bitwise(gpu_lib, name, ld, path):
    p = W.build_problem(W.small(W.CONFIGS[name], 6), ld=ld)
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    s.set_kernel_path(path)
    got = s.cal_var(p.u, p.v, p.h)
    ref = oracle_rhs(p, OT, OM, p.u, p.v, p.h)
    assert_bitwise(got, ref, p.T.nm)
    assert any(np.abs(r).max() > 0 for r in ref)


@pytest.mark.gpu
@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name", NAMES)
def test_cal_var_random_state_bitwise(gpu_lib, name, path):
    """Rough random state: exercises every branch with O(1) values everywhere."""
    p = W.build_problem(W.small(W.CONFIGS[name], 5))
    rng = np.random.default_rng(7)
    u, v = rng.normal(size=p.u.shape), rng.normal(size=p.v.shape)
    h = rng.normal(size=p.h.shape)
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    s.set_kernel_path(path)
    assert_bitwise(s.cal_var(u, v, h), oracle_rhs(p, OT, OM, u, v, h), p.T.nm)


@pytest.mark.gpu
@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name", NAMES)
def test_rk4_device_resident_bitwise(gpu_lib, name, path):
    p = W.build_problem(W.small(W.CONFIGS[name], 6))
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    s.set_kernel_path(path)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 5)
    got = s.get_state()
    u, v, h = p.u.copy(), p.v.copy(), p.h.copy()
    c = p.cfg
    O.rk4(c.variant, OT, OM, u, v, h, OM.fc, p.w0, p.z0, p.hb, c.mu0, c.mb0, c.g0, p.dt, 5)
    assert_bitwise(got, (u, v, h), p.T.nm)


@pytest.mark.gpu
def test_rk4_host_entry_matches_resident(gpu_lib):
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 8), ld=45)
    s = W.make_solver(p)
    u, v, h = p.u.copy(), p.v.copy(), p.h.copy()
    s.rk4_steps_host(u, v, h, p.dt, 3)
    s2 = W.make_solver(p)
    s2.set_state(p.u, p.v, p.h)
    s2.rk4_steps(p.dt, 3)
    assert_bitwise((u, v, h), s2.get_state(45), p.T.nm)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fs_p6", "c1_lin_p3"])
@pytest.mark.parametrize("ld", [28, 45])
@pytest.mark.parametrize("path", ["templated", "generic"])
def test_rk4_host_entry_pinned_buffers(gpu_lib, ld, path, name):
    """Mapped pinned caller arrays take the direct path (the last stage stores
    the new state into them); the result is the resident run's, bit for bit,
    and the rows past nm of an ld-strided array are left alone."""
    import torch
    p = W.build_problem(W.small(W.CONFIGS[name], 8), ld=ld)
    s = W.make_solver(p)
    s.set_kernel_path(path)
    pin = [torch.from_numpy(a.copy()).pin_memory() for a in (p.u, p.v, p.h)]
    host = [t.numpy() for t in pin]
    for a in host:
        a[:, p.T.nm:] = 7.0
    s.rk4_steps_host(*host, p.dt, 3)
    s2 = W.make_solver(p)
    s2.set_kernel_path(path)
    s2.set_state(p.u, p.v, p.h)
    s2.rk4_steps(p.dt, 3)
    assert_bitwise(host, s2.get_state(ld), p.T.nm)
    assert all((a[:, p.T.nm:] == 7.0).all() for a in host)
    # the handle's resident state is the new state as well
    assert_bitwise(s.get_state(ld), s2.get_state(ld), p.T.nm)
    # zero steps: the arrays come back unchanged
    before = [a.copy() for a in host]
    s.rk4_steps_host(*host, p.dt, 0)
    assert all(np.array_equal(a, b) for a, b in zip(host, before))


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [1, 7])
def test_lin_steps_in_one_launch(gpu_lib, steps):
    """The linear variant's RK4 steps run as one cooperative launch on a mesh
    that one pass of the resident warps covers (grid barriers between the
    stages), bit-identical to one launch per stage (generic kernels)."""
    p = W.build_problem(W.CONFIGS["c1_lin_p3"])
    s = W.make_solver(p)
    s.set_kernel_path("templated")
    s.set_state(p.u, p.v, p.h)
    l0 = s.launches
    s.rk4_steps(p.dt, steps)
    assert s.launches - l0 == 1
    g = W.make_solver(p)
    g.set_kernel_path("generic")
    g.set_state(p.u, p.v, p.h)
    l0 = g.launches
    g.rk4_steps(p.dt, steps)
    assert g.launches - l0 == 4 * steps
    assert_bitwise(s.get_state(), g.get_state(), p.T.nm)


@pytest.mark.gpu
def test_c1_full_1000_steps_bitwise(gpu_lib):
    """Configuration C1 as specified: 2048 triangles, p3, 1000 RK4 steps at the cfl.f step."""
    p = W.build_problem(W.CONFIGS["c1_lin_p3"])
    assert p.mesh.ne == 2048 and p.dt == 14.0
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 1000)
    got = s.get_state()
    u, v, h = p.u.copy(), p.v.copy(), p.h.copy()
    c = p.cfg
    O.rk4(c.variant, OT, OM, u, v, h, OM.fc, p.w0, p.z0, p.hb, c.mu0, c.mb0, c.g0, p.dt, 1000)
    assert_bitwise(got, (u, v, h), p.T.nm)
    # the state moved: this is not a trivially stationary run
    assert O.mass_norm(OT, OM, h - p.h) > 1e-3 * O.mass_norm(OT, OM, p.h)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fs_p6", "c4_ns_p4"])
def test_medium_mesh_steps_bitwise(gpu_lib, name):
    p = W.build_problem(W.small(W.CONFIGS[name], 16))
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 10)
    u, v, h = p.u.copy(), p.v.copy(), p.h.copy()
    c = p.cfg
    O.rk4(c.variant, OT, OM, u, v, h, OM.fc, p.w0, p.z0, p.hb, c.mu0, c.mb0, c.g0, p.dt, 10)
    assert_bitwise(s.get_state(), (u, v, h), p.T.nm)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1_lin_p3", "c2_fs_p6"])
def test_energy_and_cfl(gpu_lib, name):
    p = W.build_problem(W.small(W.CONFIGS[name], 10))
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    s.set_state(p.u, p.v, p.h)
    ke, pe, mass = s.energy()
    rke, rpe, rmass = O.energy(OT, OM, p.u, p.v, p.h, p.hb, p.cfg.g0)
    assert ke == pytest.approx(rke, rel=1e-13, abs=1e-300)
    assert pe == pytest.approx(rpe, rel=1e-13)
    scale = abs(rpe) ** 0.5 + abs(rmass) + 1.0
    assert abs(mass - rmass) <= 1e-13 * scale * p.mesh.ne
    cmin, dt = s.cfl()
    rcmin, rdt = O.checkcfl(p.cfg.nc, OM, p.hb, p.cfg.g0)
    assert cmin == rcmin and dt == rdt == p.dt


@pytest.mark.gpu
def test_fortran_drop_in_cal_var_(gpu_lib):
    """cal_var_ with the reference's 31 by-reference arguments (src/calvarnl_fs.f:9-12)."""
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 6))
    lib = api.load_library()
    ts = p.T.struct()
    assert lib.spoc_register_commons(C.byref(ts), api.FS, api.FP64) == 0
    m, c = p.mesh, p.cfg
    outs = [np.zeros_like(p.u) for _ in range(3)]
    keep = []

    def ints(x):
        keep.append(C.c_int(x))
        return C.c_void_p(C.addressof(keep[-1]))

    def dbl(x):
        keep.append(C.c_double(x))
        return C.c_void_p(C.addressof(keep[-1]))

    ptr = lambda a: C.c_void_p(a.ctypes.data)
    nbdl, nint = int(m.bdl.sum()), int(m.ne - m.bdl.sum())
    pbdl = np.zeros(m.ne, np.int32)
    pint = np.zeros(m.ne, np.int32)
    args = [ints(m.nf), ints(m.ne), ptr(p.u), ptr(p.v), ptr(p.h), *map(ptr, outs), ptr(m.tseg),
            ptr(m.pseg), ptr(m.ssit), ptr(m.itm), ptr(m.its), ptr(m.norm), ints(nbdl), ptr(pbdl),
            ints(nint), ptr(pint), ptr(m.bdl), ptr(p.T.cip), ptr(m.vect), ptr(m.normt),
            dbl(c.mu0), dbl(c.mb0), ptr(p.fc), dbl(c.beta), ptr(p.w0), ptr(p.z0), dbl(c.g0),
            ptr(p.hb), dbl(0.0)]
    for _ in range(2):  # second call reuses the cached handle
        lib.cal_var_(*args)
        assert lib.spoc_cal_var_status()[0] == 0
    OT, OM = oracle_for(p)
    assert_bitwise(outs, oracle_rhs(p, OT, OM, p.u, p.v, p.h), p.T.nm)
    lib.spoc_release_commons()


@pytest.mark.gpu
def test_fortran_drop_in_mesh_rewritten_in_place(gpu_lib):
    """The adaptive driver rewrites its mesh, geometry and depth arrays in place
    at a regrid (src/shwwnl_adap.f:397-433), possibly with the same ne and nf:
    the second cal_var_ call, on a different mesh at the same addresses, must
    use the new mesh."""
    cfg = W.small(W.CONFIGS["c2_fs_p6"], 6)
    p = W.build_problem(cfg)
    q = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 6, seed=9))  # other jitter
    assert (q.mesh.ne, q.mesh.nf) == (p.mesh.ne, p.mesh.nf)
    assert not np.array_equal(q.mesh.vect, p.mesh.vect)
    q.hb[:, 0] = 3500.0
    lib = api.load_library()
    ts = p.T.struct()
    assert lib.spoc_register_commons(C.byref(ts), api.FS, api.FP64) == 0
    m, c = p.mesh, p.cfg
    # the driver's arrays, at fixed addresses for both calls
    arr = {k: getattr(m, k).copy() for k in ("tseg", "pseg", "ssit", "itm", "its", "norm", "bdl",
                                                 "vect", "normt")}
    fc, w0, z0, hb = p.fc.copy(), p.w0.copy(), p.z0.copy(), p.hb.copy()
    outs = [np.zeros_like(p.u) for _ in range(3)]
    keep = []

    def ints(x):
        keep.append(C.c_int(x))
        return C.c_void_p(C.addressof(keep[-1]))

    def dbl(x):
        keep.append(C.c_double(x))
        return C.c_void_p(C.addressof(keep[-1]))

    ptr = lambda a: C.c_void_p(a.ctypes.data)
    pbdl = np.zeros(m.ne, np.int32)
    pint = np.zeros(m.ne, np.int32)
    args = [ints(m.nf), ints(m.ne), ptr(p.u), ptr(p.v), ptr(p.h), *map(ptr, outs),
            ptr(arr["tseg"]), ptr(arr["pseg"]), ptr(arr["ssit"]), ptr(arr["itm"]),
            ptr(arr["its"]), ptr(arr["norm"]), ints(0), ptr(pbdl), ints(0), ptr(pint),
            ptr(arr["bdl"]), ptr(p.T.cip), ptr(arr["vect"]), ptr(arr["normt"]), dbl(c.mu0),
            dbl(c.mb0), ptr(fc), dbl(c.beta), ptr(w0), ptr(z0), dbl(c.g0), ptr(hb), dbl(0.0)]
    lib.cal_var_(*args)
    assert lib.spoc_cal_var_status()[0] == 0
    OT, OM = oracle_for(p)
    assert_bitwise(outs, oracle_rhs(p, OT, OM, p.u, p.v, p.h), p.T.nm)
    # regrid in place: same ne, nf and addresses, new contents
    for k in arr:
        arr[k][...] = getattr(q.mesh, k)
    fc[...], hb[...] = q.fc, q.hb
    lib.cal_var_(*args)
    assert lib.spoc_cal_var_status()[0] == 0
    OTq, OMq = oracle_for(q)
    ref = O.cal_var(c.variant, OTq, OMq, p.u, p.v, p.h, OMq.fc, q.w0, q.z0, q.hb, c.mu0, c.mb0,
                    c.g0)
    assert_bitwise(outs, ref, p.T.nm)
    # depth rewritten in place on the same mesh: announced with spoc_cal_var_refresh
    hb[:, 0] = 3000.0
    lib.spoc_cal_var_refresh()
    lib.cal_var_(*args)
    assert lib.spoc_cal_var_status()[0] == 0
    ref = O.cal_var(c.variant, OTq, OMq, p.u, p.v, p.h, OMq.fc, q.w0, q.z0, hb, c.mu0, c.mb0, c.g0)
    assert_bitwise(outs, ref, p.T.nm)
    lib.spoc_release_commons()


@pytest.mark.gpu
def test_nonfinite_state_is_reported(gpu_lib):
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 4))
    s = W.make_solver(p)
    h = p.h.copy()
    h[3, 0] = np.nan
    s.set_state(p.u, p.v, h)
    with pytest.raises(api.SpocError) as ei:
        s.rk4_steps(p.dt, 1)
    assert ei.value.code == 3
    # the handle stays usable after the error
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 1)


@pytest.mark.gpu
def test_full_c2_deterministic_and_conservative(gpu_lib):
    """C2 at full size: repeatable bit for bit, and mass conserved to round-off."""
    p = W.build_problem(W.CONFIGS["c2_fs_p6"])
    s = W.make_solver(p)
    runs = []
    for _ in range(2):
        s.set_state(p.u, p.v, p.h)
        s.rk4_steps(p.dt, 3)
        runs.append(s.get_state())
    assert_bitwise(runs[0], runs[1], p.T.nm)
    s.set_state(p.u, p.v, p.h)
    _, _, m0 = s.energy()
    s.rk4_steps(p.dt, 3)
    _, _, m1 = s.energy()
    # mass = sum_e det_e sum_j ammo(j,1) h_j (src/energy.f:327-329); walls carry no flux
    scale = float(np.sum(np.abs(p.mesh.det[:, None] * p.T.ammo[0, :][None, :] * p.h)))
    assert abs(m1 - m0) <= 1e-12 * scale


@pytest.mark.gpu
def test_untabulated_degree_runs_generic_kernels(gpu_lib):
    """Degree 2 with the 6-point rule has no compile-time-sized kernels: auto
    selects the generic ones, and asking for the templated ones is refused."""
    cfg = W.small(W.CONFIGS["c2_fs_p6"], 5, nc=2, ng=6, ngf=3)
    p = W.build_problem(cfg)
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    with pytest.raises(api.SpocError) as ei:
        s.set_kernel_path("templated")
    assert ei.value.code == 7
    assert_bitwise(s.cal_var(p.u, p.v, p.h), oracle_rhs(p, OT, OM, p.u, p.v, p.h), p.T.nm)


@pytest.mark.gpu
def test_singular_mass_matrix_rejected(gpu_lib):
    """Degree 8 with the 42-point rule: 45 modes, rank <= 42; dpotrf fails as in the reference."""
    with pytest.raises(api.SpocError) as ei:
        api.build_tables(8, 42, 9)
    assert ei.value.code == 4


def rel_mass_diff(OT, OM, got, ref):
    """max over (u, v, h) of the physical-L2 difference relative to the field."""
    nm = OT.nm
    out = 0.0
    for g, r in zip(got, ref):
        d = np.ascontiguousarray(g[:, :nm] - r[:, :nm])
        rr = np.ascontiguousarray(r[:, :nm])
        out = max(out, O.mass_norm(OT, OM, d) / max(O.mass_norm(OT, OM, rr), 1e-300))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_fma_mode_rhs_and_steps_within_tolerance(gpu_lib, name):
    """SPOC_FP64_FMA: fused multiply-adds, FP64 accuracy but not the reference
    rounding.  The mass solves amplify one-ulp load differences by up to
    sqrt(cond(amm)) (1.5e4 at degree 6, 8e4 at degree 7): the right-hand side
    differs by up to ~1e-9 at degree 7 and one RK4 step by ~2e-12 (physical L2 norm,
    measured 1.9e-12 at degree 6), which is just above the 1e-12-per-step
    parity bar; the bit-exact SPOC_FP64 mode is the one that meets it."""
    p = W.build_problem(W.small(W.CONFIGS[name], 6))
    OT, OM = oracle_for(p)
    s = W.make_solver(p, "fp64_fma")
    got = s.cal_var(p.u, p.v, p.h)
    ref = oracle_rhs(p, OT, OM, p.u, p.v, p.h)
    assert rel_mass_diff(OT, OM, got, ref) < 1e-8
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 1)
    u, v, h = p.u.copy(), p.v.copy(), p.h.copy()
    c = p.cfg
    O.rk4(c.variant, OT, OM, u, v, h, OM.fc, p.w0, p.z0, p.hb, c.mu0, c.mb0, c.g0, p.dt, 1)
    assert rel_mass_diff(OT, OM, s.get_state(), (u, v, h)) < 1e-11


@pytest.mark.gpu
def test_fma_mode_c1_1000_steps_within_1e10(gpu_lib):
    p = W.build_problem(W.CONFIGS["c1_lin_p3"])
    OT, OM = oracle_for(p)
    s = W.make_solver(p, "fp64_fma")
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 1000)
    u, v, h = p.u.copy(), p.v.copy(), p.h.copy()
    c = p.cfg
    O.rk4(c.variant, OT, OM, u, v, h, OM.fc, p.w0, p.z0, p.hb, c.mu0, c.mb0, c.g0, p.dt, 1000)
    assert rel_mass_diff(OT, OM, s.get_state(), (u, v, h)) < 1e-10


# every tabulated degree with every nonlinear variant through the
# compile-time-sized kernels (one and two rows per lane, wall branches)
DEGREES = [(3, 12, 4), (4, 25, 5), (5, 27, 6), (6, 33, 7), (7, 42, 9)]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["lin", "fs", "ns", "inv"])
@pytest.mark.parametrize("deg", DEGREES, ids=[f"p{d[0]}" for d in DEGREES])
def test_every_degree_and_variant_bitwise(gpu_lib, deg, variant):
    import dataclasses
    nc, ng, ngf = deg
    base = W.small(W.CONFIGS["c2_fs_p6"], 5)
    cfg = dataclasses.replace(base, nc=nc, ng=ng, ngf=ngf, variant=variant)
    p = W.build_problem(cfg)
    OT, OM = oracle_for(p)
    s = W.make_solver(p)
    s.set_kernel_path("templated")
    rng = np.random.default_rng(nc)
    u, v = p.u + 0.1 * rng.normal(size=p.u.shape), p.v + 0.1 * rng.normal(size=p.v.shape)
    assert_bitwise(s.cal_var(u, v, p.h), oracle_rhs(p, OT, OM, u, v, p.h), p.T.nm)
    s.set_state(p.u, p.v, p.h)
    s.rk4_steps(p.dt, 3)
    x = [p.u.copy(), p.v.copy(), p.h.copy()]
    O.rk4(variant, OT, OM, *x, OM.fc, p.w0, p.z0, p.hb, cfg.mu0, cfg.mb0, cfg.g0, p.dt, 3)
    assert_bitwise(s.get_state(), x, p.T.nm)


@pytest.mark.gpu
def test_strided_cal_var_leaves_padding_rows(gpu_lib):
    """spoc_cal_var with ld = 45 arrays writes rows 1..nm of the outputs only,
    as the reference's loops do (the rows past nm keep the caller's values)."""
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 6), ld=45)
    s = W.make_solver(p)
    lib = api.load_library()
    outs = [np.full_like(p.u, 7.0) for _ in range(3)]
    rc = lib.spoc_cal_var(s._h, 45, api._d(p.u), api._d(p.v), api._d(p.h), *map(api._d, outs))
    assert rc == 0
    OT, OM = oracle_for(p)
    assert_bitwise(outs, oracle_rhs(p, OT, OM, p.u, p.v, p.h), p.T.nm)
    assert all((o[:, p.T.nm:] == 7.0).all() for o in outs)


@pytest.mark.gpu
@pytest.mark.parametrize("path", PATHS)
def test_small_golden_rhs(gpu_lib, path):
    """The library's right-hand side on the committed 8-triangle known answers
    (tests/golden/small_rhs.json, every tabulated degree and variant), set up
    with the library's own code: input state and cal_var output bit for bit."""
    import hashlib
    import json
    from pathlib import Path

    from oracle.problems import SMALL_DEGREES, SMALL_VARIANTS, small_case, small_case_state

    golden = json.loads((Path(__file__).parent / "golden" / "small_rhs.json").read_text())

    def digest(*arrays):
        m = hashlib.sha256()
        for a in arrays:
            m.update(np.ascontiguousarray(a[:, :nm], dtype="<f8").tobytes())
        return m.hexdigest()

    for nc, ng, ngf in SMALL_DEGREES:
        for variant in SMALL_VARIANTS:
            rec = golden[f"p{nc}_{variant}"]
            p = W.build_problem(small_case(nc, ng, ngf, variant))
            nm = p.T.nm
            u, v, h = small_case_state(p.u, p.v, p.h, nc, variant)
            assert digest(u, v, h) == rec["input_sha256"], (nc, variant)
            s = W.make_solver(p)
            s.set_kernel_path(path)
            assert digest(*s.cal_var(u, v, h)) == rec["rhs_sha256"], (nc, variant, path)
            s.close()
