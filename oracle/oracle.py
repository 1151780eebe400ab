"""Python binding of the CPU oracle (oracle/libspoc_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.

The oracle builds its own tables and mesh pointers from raw inputs (quadrature
points, node coordinates, element-to-node table), so a comparison against the
product checks the product's set-up code as well as its kernels.
Parity status: unpinned against reference output (no golden data ships with
the reference and it cannot be compiled here); pinned by the known-answer
tests in tests/test_oracle_pins.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libspoc_oracle.so"

LIN, FS, NS, INV = 0, 1, 2, 3
VARIANTS = {"lin": LIN, "fs": FS, "ns": NS, "inv": INV}

_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)


class Common(C.Structure):
    _fields_ = [
        ("nc", C.c_int), ("nm", C.c_int), ("ng", C.c_int), ("ngf", C.c_int),
        ("wi", _DP), ("xi", _DP), ("yi", _DP), ("wif", _DP), ("tif", _DP),
        ("pi2", _DP), ("ldq", C.c_int), ("pico", _DP), ("ldg", C.c_int), ("ldp", C.c_int),
        ("amm", _DP), ("amml", _DP), ("agx", _DP), ("agy", _DP), ("ammo", _DP), ("ldm", C.c_int),
        ("cip", _IP),
    ]


class MeshS(C.Structure):
    _fields_ = [
        ("ne", C.c_int), ("nf", C.c_int), ("itm", _IP), ("its", _IP), ("tseg", _IP),
        ("ssit", _IP), ("norm", _DP), ("vect", _DP), ("normt", _DP), ("bdl", _IP),
    ]


def build() -> Path:
    """Compile the oracle with its Makefile if it is missing or stale."""
    src = [HERE / "spoc_oracle.c", HERE / "spoc_oracle.h", HERE / "Makefile"]
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
        L = _lib
        L.ora_po.restype = C.c_double
        L.ora_po.argtypes = [C.c_int, C.c_double]
        L.ora_dpo.restype = C.c_double
        L.ora_dpo.argtypes = [C.c_int, C.c_double]
        L.ora_checkcfl.restype = C.c_double
        L.ora_checkcfl.argtypes = [C.c_int, C.c_int, C.c_int, _DP, _IP, C.c_double, _DP, _DP, _DP]
        for name in ("ora_cal_var",):
            getattr(L, name).argtypes = [C.c_int, C.POINTER(Common), C.POINTER(MeshS), C.c_int,
                                         _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP,
                                         C.c_double, C.c_double, C.c_double, C.c_int]
        L.ora_rk4.argtypes = [C.c_int, C.POINTER(Common), C.POINTER(MeshS), C.c_int, _DP, _DP, _DP,
                              _DP, _DP, _DP, _DP, C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_int, C.c_int]
        L.ora_energy.argtypes = [C.POINTER(Common), C.c_int, C.c_int, _DP, _DP, _DP, C.c_double, _DP,
                                 _DP, _DP, _DP, _IP, _DP, _DP]
    return _lib


def d(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def i(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_IP)


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


class Tables:
    """Oracle restatement of the set-up of src/shwwnl.f:127-156."""

    def __init__(self, nc, ng, ngf, wi, xi, yi, wif, tif):
        L = lib()
        self.nc, self.ng, self.ngf = nc, ng, ngf
        self.nm = nm = (nc + 1) * (nc + 2) // 2
        self.wi, self.xi, self.yi = (np.ascontiguousarray(a, dtype=np.float64) for a in (wi, xi, yi))
        self.wif, self.tif = (np.ascontiguousarray(a, dtype=np.float64) for a in (wif, tif))
        self.pi2 = np.zeros((nm, ng))
        L.ora_cal_p2(nc, ng, d(self.xi), d(self.yi), d(self.pi2), ng)
        self.pico = np.zeros((3, nm, ngf))
        L.ora_cal_pico(nc, ngf, d(self.tif), d(self.pico), ngf, nm)
        self.cip = np.zeros((nc + 1, 2), np.int32)
        L.ora_calip(nc, i(self.cip))
        mats = {}
        for k, name in enumerate(("amm", "ammx", "ammy", "agx", "agy")):
            m = np.zeros((nm, nm))
            L.ora_cal_mat(nc, ng, k, d(self.xi), d(self.yi), d(self.wi), d(m), nm)
            mats[name] = m
        self.ammo = mats["amm"].copy()
        self.amml = np.zeros((nm, nm))
        L.ora_cal_matl(nc, d(self.ammo), d(self.amml), nm)
        self.amml_raw = self.amml.copy()
        self.amm = mats["amm"]
        self.ammx, self.ammy, self.agx, self.agy = mats["ammx"], mats["ammy"], mats["agx"], mats["agy"]
        self.info_amm = L.ora_dpotf2_upper(nm, d(self.amm), nm)
        self.info_amml = L.ora_dpotf2_upper(nm - nc - 1, d(self.amml), nm)
        self.common = Common(nc, nm, ng, ngf, d(self.wi), d(self.xi), d(self.yi), d(self.wif),
                             d(self.tif), d(self.pi2), ng, d(self.pico), ngf, nm, d(self.amm),
                             d(self.amml), d(self.agx), d(self.agy), d(self.ammo), nm, i(self.cip))


class Mesh:
    """Oracle restatement of pointer_mesh / check_mesh / cal_rotnf / cal_its /
    calpre / coriolis (src/shwwnl.f:162-174)."""

    def __init__(self, inn, xgr, ygr, nc, f0=0.0, beta=0.0, ld=None):
        L = lib()
        self.inn = np.ascontiguousarray(inn, dtype=np.int32)
        self.xgr = np.ascontiguousarray(xgr, dtype=np.float64)
        self.ygr = np.ascontiguousarray(ygr, dtype=np.float64)
        self.ne, self.nn = self.inn.shape[0], self.xgr.shape[0]
        nm = (nc + 1) * (nc + 2) // 2
        self.ld = ld or nm
        nfmax = 3 * self.ne
        self.itm = np.zeros((self.ne, 3), np.int32)
        tseg = np.zeros((nfmax, 2), np.int32)
        pseg = np.zeros((nfmax, 2), np.int32)
        nf = L.ora_pointer_mesh(self.nn, self.ne, i(self.inn), i(self.itm), i(tseg), i(pseg), nfmax)
        if nf < 0:
            raise RuntimeError("pointer_mesh overflow")
        self.nf = nf
        self.tseg = np.ascontiguousarray(tseg[:nf])
        self.pseg = np.ascontiguousarray(pseg[:nf])
        self.check = L.ora_check_mesh(self.ne, nf, i(self.itm), i(self.tseg))
        self.norm = np.zeros((nf, 2))
        L.ora_cal_rotnf(nf, d(self.xgr), d(self.ygr), d(self.norm), i(self.pseg))
        self.its = np.zeros((self.ne, 3), np.int32)
        self.ssit = np.zeros((nf, 2), np.int32)
        self.its_rc = L.ora_cal_its(nf, i(self.itm), i(self.its), i(self.tseg), i(self.ssit))
        self.vect = np.zeros((self.ne, 5))
        self.normt = np.zeros((self.ne, 2))
        self.bdl = np.zeros(self.ne, np.int32)
        self.pint = np.zeros(self.ne, np.int32)
        self.pbdl = np.zeros(self.ne, np.int32)
        nint, nbdl, nebd = C.c_int(), C.c_int(), C.c_int()
        L.ora_calpre(self.nn, self.ne, nf, i(self.inn), d(self.xgr), d(self.ygr), d(self.vect),
                     i(self.itm), d(self.norm), d(self.normt), i(self.bdl), C.byref(nint),
                     i(self.pint), C.byref(nbdl), i(self.pbdl), C.byref(nebd), i(self.tseg),
                     i(self.pseg))
        self.nint, self.nbdl, self.nebd = nint.value, nbdl.value, nebd.value
        self.fc = np.zeros((self.ne, self.ld))
        L.ora_coriolis.argtypes = [C.c_int, C.c_int, _IP, _DP, _DP, _DP, C.c_int, C.c_double, C.c_double]
        L.ora_coriolis(nc, self.ne, i(self.inn), d(self.xgr), d(self.ygr), d(self.fc), self.ld, f0, beta)
        self.s = MeshS(self.ne, nf, i(self.itm), i(self.its), i(self.tseg), i(self.ssit),
                       d(self.norm), d(self.vect), d(self.normt), i(self.bdl))


def cal_var(variant, T: Tables, M: Mesh, u0, v0, h0, fc, w0, z0, hb, mu0, mb0, g0, nthreads=None):
    ld = u0.shape[1]
    out = [np.zeros_like(u0) for _ in range(3)]
    rc = lib().ora_cal_var(VARIANTS.get(variant, variant), C.byref(T.common), C.byref(M.s), ld,
                           d(u0), d(v0), d(h0), *map(d, out), d(fc), d(w0), d(z0), d(hb),
                           mu0, mb0, g0, nthreads or default_threads())
    if rc:
        raise RuntimeError(f"ora_cal_var rc={rc}")
    return tuple(out)


def cal_flu(T: Tables, M: Mesh, a0, nthreads=None):
    """Face traces of one field (src/calflu.f:6-71): (nf, ngf), the central
    average of both sides' traces at the ngf edge points (side 1's trace on
    wall faces)."""
    a0 = np.ascontiguousarray(a0, dtype=np.float64)
    out = np.zeros((M.nf, T.ngf))
    L = lib()
    L.ora_cal_flu.argtypes = [C.POINTER(Common), C.c_int, _IP, _DP, C.c_int, _DP, C.c_int, _IP,
                              C.c_int]
    L.ora_cal_flu(C.byref(T.common), M.nf, i(M.tseg), d(out), T.ngf, d(a0), a0.shape[1],
                  i(M.ssit), nthreads or default_threads())
    return out


def rk4(variant, T: Tables, M: Mesh, u, v, h, fc, w0, z0, hb, mu0, mb0, g0, dt, nsteps,
        nthreads=None):
    """nsteps RK4 steps in place on (u, v, h)."""
    rc = lib().ora_rk4(VARIANTS.get(variant, variant), C.byref(T.common), C.byref(M.s), u.shape[1],
                       d(u), d(v), d(h), d(fc), d(w0), d(z0), d(hb), mu0, mb0, g0, dt, nsteps,
                       nthreads or default_threads())
    if rc:
        raise RuntimeError(f"ora_rk4 rc={rc}")


def energy(T: Tables, M: Mesh, u, v, h, hb, g0):
    k, p, m = C.c_double(), C.c_double(), C.c_double()
    lib().ora_energy(C.byref(T.common), M.ne, u.shape[1], d(u), d(v), d(h), g0, d(hb),
                     C.byref(k), C.byref(p), C.byref(m), i(M.inn), d(M.xgr), d(M.ygr))
    return k.value, p.value, m.value


def checkcfl(nc, M: Mesh, hb, g0):
    c = C.c_double()
    dt = lib().ora_checkcfl(nc, M.ne, hb.shape[1], d(hb), i(M.inn), g0, d(M.xgr), d(M.ygr),
                            C.byref(c))
    return c.value, dt


def calh(T: Tables, M: Mesh, f, ld=None):
    """calh of src/init.f:290-344 for a vectorised f(x, y)."""
    L = lib()
    px = np.zeros((M.ne, T.ng))
    py = np.zeros((M.ne, T.ng))
    L.ora_calh_points(C.byref(T.common), M.ne, i(M.inn), d(M.xgr), d(M.ygr), d(px), d(py))
    vals = np.ascontiguousarray(f(px, py), dtype=np.float64)
    out = np.zeros((M.ne, ld or T.nm))
    L.ora_calh(C.byref(T.common), M.ne, d(vals), d(out), out.shape[1])
    return out, px, py


def changemaille(inn, nn):
    """chmal corner fix (src/chmal.f:240-330) on a copy of `in`."""
    L = lib()
    out = np.array(inn, dtype=np.int32, order="C", copy=True)
    ne = out.shape[0]
    nfmax = 3 * ne
    itm = np.zeros((ne, 3), np.int32)
    tseg = np.zeros((nfmax, 2), np.int32)
    pseg = np.zeros((nfmax, 2), np.int32)
    nf = L.ora_pointer_mesh(nn, ne, i(out), i(itm), i(tseg), i(pseg), nfmax)
    rc = L.ora_changemaille(nn, ne, nf, i(out), i(itm), i(tseg), i(pseg))
    if rc:
        raise RuntimeError("changemaille failed")
    return out


def mass_norm(T: Tables, M: Mesh, a):
    """Physical L2 norm sqrt(sum_e det_e a_e^T ammo a_e) of a modal field (ne, ld)."""
    nm = T.nm
    x = a[:, :nm]
    det = M.vect[:, 0] * M.vect[:, 3] - M.vect[:, 2] * M.vect[:, 1]
    G = T.ammo.T  # numpy [j, i] holds ammo(i, j); symmetric anyway
    return float(np.sqrt(np.sum(det * np.einsum("ei,ij,ej->e", x, G, x))))


# ---------------------------------------------------------------------------
# Regridding (src/adapt.f) and the adaptive driver's CFL (src/cfl.f:57-140)
# ---------------------------------------------------------------------------

def checkconv(T: Tables, M: Mesh, a):
    """checkconv of src/adapt.f:1260-1334: normalised trace jump per element."""
    L = lib()
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.zeros(M.ne)
    L.ora_checkconv(C.byref(T.common), M.nf, M.ne, a.shape[1], d(a), i(M.tseg), i(M.ssit), d(out))
    return out


def cal_conv(T: Tables, M: Mesh, u, v, h, fac1, fac2, fac3):
    """cal_conv of src/adapt.f:1122-1193."""
    L = lib()
    u, v, h = (np.ascontiguousarray(x, dtype=np.float64) for x in (u, v, h))
    fconv = np.zeros(M.ne, np.int32)
    fderaff = np.zeros(M.ne, np.int32)
    flags = np.zeros(3, np.int32)
    mx = [np.zeros(M.ne) for _ in range(3)]
    sup = C.c_double()
    L.ora_cal_conv.argtypes = [C.POINTER(Common), C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, _IP,
                               _IP, C.c_double, C.c_double, C.c_double, _IP, _IP, _IP, _DP,
                               _DP, _DP, _DP]
    L.ora_cal_conv(C.byref(T.common), M.nf, M.ne, u.shape[1], d(u), d(v), d(h), i(M.tseg),
                   i(M.ssit), fac1, fac2, fac3, i(fconv), i(fderaff), i(flags), C.byref(sup),
                   *map(d, mx))
    return {"fconv": fconv, "fderaff": fderaff, "conv": bool(flags[0]), "deraff": bool(flags[1]),
            "timedir": bool(flags[2]), "supmax": sup.value, "amax": tuple(mx)}


def inter_only_new(inn, innew):
    """inter_only_new of src/adapt.f:1233-1258 (1-based element tables)."""
    inn = np.ascontiguousarray(inn, dtype=np.int32)
    innew = np.ascontiguousarray(innew, dtype=np.int32)
    out = np.zeros(innew.shape[0], np.int32)
    lib().ora_inter_only_new(inn.shape[0], innew.shape[0], i(inn), i(innew), i(out))
    return out


def interpol(T: Tables, old: Mesh, new: Mesh, tinter, u):
    """interpol of src/adapt.f:1662-1745: u (ne_old, ld) onto the new mesh.
    Returns (unew, loc_elem, loc_x, loc_y); loc_* are (ne_new, ng)."""
    L = lib()
    u = np.ascontiguousarray(u, dtype=np.float64)
    tinter = np.ascontiguousarray(tinter, dtype=np.int32)
    unew = np.zeros((new.ne, u.shape[1]))
    le = np.zeros((new.ne, T.ng), np.int32)
    lx = np.zeros((new.ne, T.ng))
    ly = np.zeros((new.ne, T.ng))
    rc = L.ora_interpol(C.byref(T.common), old.ne, i(old.inn), i(old.itm), i(old.tseg),
                        i(old.pseg), d(old.xgr), d(old.ygr), i(tinter), d(u), u.shape[1],
                        d(unew), new.ne, d(new.xgr), d(new.ygr), i(new.inn), i(le), d(lx), d(ly))
    if rc:
        raise RuntimeError("interlin walk did not end")
    return unew, le, lx, ly


def verif_rot(T: Tables, M: Mesh, u, v):
    """verif_rot of src/shwwnl_adap.f:481-596 on copies of (u, v)."""
    u = np.array(u, dtype=np.float64, order="C", copy=True)
    v = np.array(v, dtype=np.float64, order="C", copy=True)
    lib().ora_verif_rot(C.byref(T.common), M.ne, u.shape[1], d(u), d(v), d(M.normt), i(M.bdl))
    return u, v


def cal_pgraph(nc, n):
    nm = (nc + 1) * (nc + 2) // 2
    out = np.zeros((n, n, nm))
    lib().ora_cal_pgraph(nc, n, d(out))
    return out


def checkcfl2(nc, M: Mesh, hb, u, v, g0, n=10, dt_in=0.0):
    """checkcfl2 of src/cfl.f:57-140 on the n-point lattice; returns (cflmin, dt)."""
    L = lib()
    pg = cal_pgraph(nc, n)
    hb, u, v = (np.ascontiguousarray(x, dtype=np.float64) for x in (hb, u, v))
    L.ora_checkcfl2.restype = C.c_double
    L.ora_checkcfl2.argtypes = [C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, _IP, C.c_double, _DP,
                                _DP, C.c_int, _DP, C.c_double, _DP]
    c = C.c_double()
    dt = L.ora_checkcfl2(nc, M.ne, hb.shape[1], d(hb), d(u), d(v), i(M.inn), g0, d(M.xgr),
                         d(M.ygr), n, d(pg), dt_in, C.byref(c))
    return c.value, dt


def eval_points(nc, u, v, h, elem, px, py):
    """fsol of u, v, h at points given by element (1-based) and reference coordinates."""
    u, v, h = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, h))
    elem = np.ascontiguousarray(elem, dtype=np.int32)
    px = np.ascontiguousarray(px, dtype=np.float64)
    py = np.ascontiguousarray(py, dtype=np.float64)
    out = np.zeros((3, elem.size))
    lib().ora_eval_points(nc, u.shape[1], d(u), d(v), d(h), elem.size, i(elem), d(px), d(py),
                          d(out))
    return out


def lattice(nc, M: Mesh, u, v, h, n=10):
    """write_gra's lattice values: (ne, np, 5) with x, y, u, v, h."""
    u, v, h = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, h))
    pg = cal_pgraph(nc, n)
    out = np.zeros((M.ne, n * (n + 1) // 2, 5))
    lib().ora_lattice(nc, M.ne, u.shape[1], d(u), d(v), d(h), i(M.inn), d(M.xgr), d(M.ygr), n,
                      d(pg), d(out))
    return out


def interlin(M: Mesh, tk, x, y):
    """One interlin walk (src/adapt.f:1747-1830): (tk, x, y, lab)."""
    t, xx, yy = C.c_int(tk), C.c_double(x), C.c_double(y)
    lab = np.zeros(3)
    rc = lib().ora_interlin(i(M.inn), i(M.itm), i(M.tseg), i(M.pseg), d(M.xgr), d(M.ygr),
                            C.byref(t), C.byref(xx), C.byref(yy), d(lab), 16 * M.ne + 64)
    if rc:
        raise RuntimeError("interlin walk did not end")
    return t.value, xx.value, yy.value, lab
