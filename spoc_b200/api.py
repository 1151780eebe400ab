"""ctypes binding of the C ABI in include/spoc_gpu.h (spoc_b200/libspoc_gpu.so).

This is the host-side mirror of the reference's operator interface: the
Fortran driver calls `cal_var` (src/calvarnl_fs.f:9-12) four times per RK4
step (src/shwwnl.f:238-274); here `Solver.cal_var` is that call with host
arrays, `Solver.rk4_steps` keeps the state on the device, and the set-up
helpers restate read_gauss / cal_p2 / cal_pico / calip / cal_mat / cal_matl /
dpotrf / pointer_mesh / calpre / coriolis / calh.

Arrays follow the Fortran layout: a field of `ne` elements with leading
dimension `ld` is a C-contiguous numpy array of shape (ne, ld); connectivity
arrays hold 1-based ids.  Every call raises SpocError on a non-zero status.
The library is required: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libspoc_gpu.so"

LIN, FS, NS, INV = 0, 1, 2, 3
VARIANTS = {"lin": LIN, "fs": FS, "ns": NS, "inv": INV}
FP64 = 0
FP64_FMA = 1
MIXED = 2  # FP32 contractions in the orthonormal basis, FP64 RK4 state
PRECISIONS = {"fp64": FP64, "fp64_fma": FP64_FMA, "mixed": MIXED}

_STATUS = {
    0: "ok", 1: "bad argument", 2: "CUDA error", 3: "non-finite tendency",
    4: "mass matrix not positive definite", 5: "mesh check failed", 6: "out of memory",
    7: "unsupported configuration",
}


class SpocError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        super().__init__(f"{where}: {_STATUS.get(code, code)} ({code}) {detail}".rstrip())


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)


class _Tables(C.Structure):
    _fields_ = [
        ("nc", C.c_int), ("nm", C.c_int), ("ng", C.c_int), ("ngf", C.c_int),
        ("wi", _DP), ("xi", _DP), ("yi", _DP), ("wif", _DP), ("tif", _DP),
        ("pi2", _DP), ("ld_pi2", C.c_int),
        ("pico", _DP), ("ld_pico1", C.c_int), ("ld_pico2", C.c_int),
        ("amm", _DP), ("amml", _DP), ("agx", _DP), ("agy", _DP), ("ammo", _DP), ("ld_mat", C.c_int),
        ("cip", _IP),
    ]


class _Mesh(C.Structure):
    _fields_ = [
        ("ne", C.c_int), ("nf", C.c_int),
        ("itm", _IP), ("its", _IP), ("tseg", _IP), ("ssit", _IP),
        ("norm", _DP), ("vect", _DP), ("normt", _DP), ("bdl", _IP),
    ]


class _Params(C.Structure):
    _fields_ = [
        ("mu0", C.c_double), ("mb0", C.c_double), ("g0", C.c_double),
        ("fc", _DP), ("w0", _DP), ("z0", _DP), ("hb", _DP), ("ld", C.c_int),
    ]


_lib = None


def load_library(path: Path | str | None = None) -> C.CDLL:
    """Load libspoc_gpu.so (build it first with spoc_b200.build.build())."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run `python -m spoc_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(str(p))
    vp = C.c_void_p
    sig = {
        "spoc_create": (C.c_int, [C.POINTER(_Tables), C.POINTER(_Mesh), C.c_int, C.c_int, C.POINTER(vp)]),
        "spoc_destroy": (None, [vp]),
        "spoc_ensemble_create": (C.c_int, [C.c_int, C.POINTER(vp), C.POINTER(vp)]),
        "spoc_ensemble_destroy": (None, [vp]),
        "spoc_ensemble_configure": (C.c_int, [vp, C.c_int, C.c_int]),
        "spoc_ensemble_info": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "spoc_ensemble_steps": (C.c_int, [vp, _DP, C.c_int, C.c_int]),
        "spoc_ensemble_balance": (C.c_int, [vp, _DP, C.c_int]),
        "spoc_set_stream": (C.c_int, [vp, vp]),
        "spoc_set_kernel_path": (C.c_int, [vp, C.c_int]),
        "spoc_set_params": (C.c_int, [vp, C.POINTER(_Params)]),
        "spoc_cal_var": (C.c_int, [vp, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP]),
        "spoc_cal_var_dev": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, vp]),
        "spoc_set_state": (C.c_int, [vp, C.c_int, _DP, _DP, _DP]),
        "spoc_get_state": (C.c_int, [vp, C.c_int, _DP, _DP, _DP]),
        "spoc_rk4_steps": (C.c_int, [vp, C.c_double, C.c_int]),
        "spoc_rk4_steps_host": (C.c_int, [vp, C.c_int, _DP, _DP, _DP, C.c_double, C.c_int]),
        "spoc_energy": (C.c_int, [vp, _DP, _DP, _DP]),
        "spoc_cfl": (C.c_int, [vp, C.c_int, _IP, _DP, _DP, _DP, _DP]),
        "spoc_kernel_launches": (C.c_longlong, [vp]),
        "spoc_checkconv": (C.c_int, [vp, _DP, _DP, _DP]),
        "spoc_cal_conv": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, _IP, _IP, _IP, _DP]),
        "spoc_interpol": (C.c_int, [vp, vp, _IP, _IP, _DP, _DP]),
        "spoc_interpol_dev": (C.c_int, [vp, vp, vp, vp, vp, vp]),
        "spoc_verif_rot": (C.c_int, [vp]),
        "spoc_cfl2": (C.c_int, [vp, C.c_int, C.c_int, _IP, _DP, _DP, C.c_double, _DP, _DP]),
        "spoc_inter_only_new": (C.c_int, [C.c_int, C.c_int, _IP, _IP, _IP]),
        "spoc_eval_points": (C.c_int, [vp, C.c_int, _IP, _DP, _DP, _DP]),
        "spoc_lattice": (C.c_int, [vp, C.c_int, C.c_int, _IP, _DP, _DP, _DP]),
        "spoc_locate_xy": (C.c_int, [C.c_int, _IP, _IP, _IP, _IP, _DP, _DP, C.c_int, _DP, _DP,
                                     _IP, C.c_int, _IP, _DP, _DP, _IP]),
        "spoc_locate_points": (C.c_int, [C.c_int, _IP, _IP, _IP, _IP, _DP, _DP, C.c_int, _IP, _DP,
                                         _DP, _IP, C.c_int, _DP, _DP, _IP, _DP, _DP]),
        "spoc_profile_rk4": (C.c_int, [vp, C.c_double, C.c_int, _DP, _IP]),
        "spoc_fp64_peak": (C.c_int, [C.c_int, _DP]),
        "spoc_tlm_rhs": (C.c_int, [vp, C.c_int] + [_DP] * 9),
        "spoc_adj_rhs": (C.c_int, [vp, C.c_int] + [_DP] * 9),
        "spoc_tlm_steps": (C.c_int, [vp, C.c_int] + [_DP] * 6 + [C.c_double, C.c_int]),
        "spoc_adj_steps": (C.c_int, [vp, C.c_int] + [_DP] * 6 + [C.c_double, C.c_int]),
        "spoc_set_observations": (C.c_int, [vp, C.c_int, _IP, _DP, C.c_int, _IP, _DP]),
        "spoc_fwd_window": (C.c_int, [vp, C.c_int, _DP, _DP, _DP, C.c_double, C.c_int, _DP]),
        "spoc_bwd_window": (C.c_int, [vp, C.c_int, _DP, _DP, _DP, C.c_double, C.c_int, C.c_int,
                                      _DP, _DP, _DP, _DP]),
        "spoc_adjoint_counters": (C.c_int, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
        "spoc_set_adjoint_sweeps": (C.c_int, [vp, C.POINTER(_Tables), C.c_int]),
        "spoc_last_error": (C.c_char_p, []),
        "spoc_register_commons": (C.c_int, [C.POINTER(_Tables), C.c_int, C.c_int]),
        "spoc_cal_var_status": (_IP, []),
        "spoc_release_commons": (None, []),
        "spoc_cal_var_refresh": (None, []),
        "spoc_build_tables": (C.c_int, [C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP,
                                        _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _IP]),
        "spoc_build_mesh": (C.c_int, [C.c_int, C.c_int, _IP, _DP, _DP, C.c_int, C.c_double,
                                      C.c_double, C.c_int, _IP, _IP, _IP, _IP, _IP, _IP, _DP,
                                      _DP, _DP, _IP, _DP, C.c_int]),
        "spoc_fix_mesh": (C.c_int, [C.c_int, C.c_int, _IP]),
        "spoc_projection_points": (C.c_int, [C.c_int, _IP, _DP, _DP, C.c_int, _DP, _DP, _DP, _DP]),
        "spoc_project": (C.c_int, [C.c_int, C.c_int, _DP, _DP, _DP, C.c_int, _DP, _DP, C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    # cal_var_ takes 31 pointers (gfortran by-reference ABI)
    lib.cal_var_.restype = None
    lib.cal_var_.argtypes = [vp] * 31
    if path is None:
        _lib = lib
    return lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _i(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_IP)


def _check(rc: int, where: str) -> None:
    if rc != 0:
        msg = load_library().spoc_last_error()
        raise SpocError(rc, where, msg.decode() if msg else "")


# ---------------------------------------------------------------------------
# quadrature data (src/readgauss.f)
# ---------------------------------------------------------------------------
_QUAD = None


def quadrature(ng: int, ngf: int):
    """(wi, xi, yi, wif, tif) of tri2_<ng>.dat and legen<ngf>.dat."""
    global _QUAD
    if _QUAD is None:
        _QUAD = json.loads((HERE / "data" / "quadrature_tables.json").read_text())
    tri = _QUAD["triangle"].get(str(ng))
    edge = _QUAD["edge"].get(str(ngf))
    if tri is None or edge is None:
        raise ValueError(f"no quadrature table tri2_{ng}.dat / legen{ngf}.dat")
    t = np.array([[float(v) for v in r] for r in tri], dtype=np.float64)
    e = np.array([[float(v) for v in r] for r in edge], dtype=np.float64)
    return (np.ascontiguousarray(t[:, 0]), np.ascontiguousarray(t[:, 1]),
            np.ascontiguousarray(t[:, 2]), np.ascontiguousarray(e[:, 0]),
            np.ascontiguousarray(e[:, 1]))


@dataclass
class Tables:
    """Reference-element tables (the COMMON blocks of src/shwwnl.f:60-71)."""
    nc: int
    ng: int
    ngf: int
    wi: np.ndarray
    xi: np.ndarray
    yi: np.ndarray
    wif: np.ndarray
    tif: np.ndarray
    pi2: np.ndarray   # (nm, ng): pi2(q, n) at [n, q]
    pico: np.ndarray  # (3, nm, ngf): pico(j, n, s) at [s, n, j]
    amm: np.ndarray   # (nm, nm) column-major storage: amm(i, j) at [j, i]; upper Cholesky factor
    amml: np.ndarray
    agx: np.ndarray
    agy: np.ndarray
    ammo: np.ndarray
    ammx: np.ndarray
    ammy: np.ndarray
    cip: np.ndarray   # (nc+1, 2)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nm(self) -> int:
        return (self.nc + 1) * (self.nc + 2) // 2

    def struct(self) -> _Tables:
        nm = self.nm
        t = _Tables(self.nc, nm, self.ng, self.ngf, _d(self.wi), _d(self.xi), _d(self.yi),
                    _d(self.wif), _d(self.tif), _d(self.pi2), self.ng, _d(self.pico), self.ngf,
                    nm, _d(self.amm), _d(self.amml), _d(self.agx), _d(self.agy), _d(self.ammo),
                    nm, _i(self.cip))
        return t


def fp64_peak(mode: int = 0) -> float:
    """Measured TFLOP/s of the current GPU (0: FP64 FMA, 1: FP64 mul + add,
    2: FP32 FMA)."""
    t = C.c_double()
    _check(load_library().spoc_fp64_peak(mode, C.byref(t)), "fp64_peak")
    return t.value


def tc_selftest(A, B, kpad: int, split: int, dinit=None):
    """D = dinit + A B^T on the tensor cores (tcgen05, TF32; split 1 = 3xTF32)."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    n = B.shape[0]
    D = np.zeros((128, n), np.float32)
    fp = C.POINTER(C.c_float)
    di = None if dinit is None else np.ascontiguousarray(dinit, dtype=np.float32)
    lib = load_library()
    lib.spoc_tc_selftest.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, fp, fp, fp, fp]
    _check(lib.spoc_tc_selftest(A.shape[1], kpad, n, split, A.ctypes.data_as(fp), B.ctypes.data_as(fp),
                                None if di is None else di.ctypes.data_as(fp), D.ctypes.data_as(fp)),
           "tc_selftest")
    return D


def build_tables(nc: int, ng: int, ngf: int) -> Tables:
    """Quadrature, basis tables, operators and Cholesky factors for degree nc."""
    lib = load_library()
    wi, xi, yi, wif, tif = quadrature(ng, ngf)
    nm = (nc + 1) * (nc + 2) // 2
    z = lambda *s: np.zeros(s, dtype=np.float64)
    T = Tables(nc, ng, ngf, wi, xi, yi, wif, tif, z(nm, ng), z(3, nm, ngf), z(nm, nm), z(nm, nm),
               z(nm, nm), z(nm, nm), z(nm, nm), z(nm, nm), z(nm, nm),
               np.zeros((nc + 1, 2), dtype=np.int32))
    info = C.c_int(0)
    rc = lib.spoc_build_tables(nc, ng, ngf, _d(wi), _d(xi), _d(yi), _d(wif), _d(tif), _d(T.pi2),
                               _d(T.pico), _d(T.amm), _d(T.amml), _d(T.agx), _d(T.agy),
                               _d(T.ammo), _d(T.ammx), _d(T.ammy), _i(T.cip), C.byref(info))
    if rc:
        raise SpocError(rc, f"build_tables(nc={nc}, ng={ng})", f"dpotrf info {info.value}")
    return T


@dataclass
class Mesh:
    """Mesh pointers of pointer_mesh / cal_its / calpre (1-based ids)."""
    nn: int
    ne: int
    nf: int
    inn: np.ndarray   # (ne, 3) node ids
    xgr: np.ndarray
    ygr: np.ndarray
    itm: np.ndarray   # (ne, 3)
    its: np.ndarray   # (ne, 3)
    tseg: np.ndarray  # (nf, 2)
    pseg: np.ndarray  # (nf, 2)
    ssit: np.ndarray  # (nf, 2)
    norm: np.ndarray  # (nf, 2)
    vect: np.ndarray  # (ne, 5)
    normt: np.ndarray  # (ne, 2)
    bdl: np.ndarray   # (ne,)
    fc: np.ndarray    # (ne, ld)

    def struct(self) -> _Mesh:
        return _Mesh(self.ne, self.nf, _i(self.itm), _i(self.its), _i(self.tseg), _i(self.ssit),
                     _d(self.norm), _d(self.vect), _d(self.normt), _i(self.bdl))

    @property
    def det(self) -> np.ndarray:
        v = self.vect
        return v[:, 0] * v[:, 3] - v[:, 2] * v[:, 1]


def build_mesh(inn: np.ndarray, xgr: np.ndarray, ygr: np.ndarray, nc: int, f0: float = 0.0,
               beta: float = 0.0, ld: int | None = None) -> Mesh:
    lib = load_library()
    inn = np.ascontiguousarray(inn, dtype=np.int32)
    xgr = np.ascontiguousarray(xgr, dtype=np.float64)
    ygr = np.ascontiguousarray(ygr, dtype=np.float64)
    ne, nn = inn.shape[0], xgr.shape[0]
    nm = (nc + 1) * (nc + 2) // 2
    ld = ld or nm
    nfmax = 3 * ne
    nf = C.c_int(0)
    itm = np.zeros((ne, 3), np.int32)
    its = np.zeros((ne, 3), np.int32)
    tseg = np.zeros((nfmax, 2), np.int32)
    pseg = np.zeros((nfmax, 2), np.int32)
    ssit = np.zeros((nfmax, 2), np.int32)
    norm = np.zeros((nfmax, 2))
    vect = np.zeros((ne, 5))
    normt = np.zeros((ne, 2))
    bdl = np.zeros(ne, np.int32)
    fc = np.zeros((ne, ld))
    rc = lib.spoc_build_mesh(nn, ne, _i(inn), _d(xgr), _d(ygr), nc, f0, beta, nfmax,
                             C.byref(nf), _i(itm), _i(its), _i(tseg), _i(pseg), _i(ssit),
                             _d(norm), _d(vect), _d(normt), _i(bdl), _d(fc), ld)
    _check(rc, "build_mesh")
    k = nf.value
    return Mesh(nn, ne, k, inn, xgr, ygr, itm, its, np.ascontiguousarray(tseg[:k]),
                np.ascontiguousarray(pseg[:k]), np.ascontiguousarray(ssit[:k]),
                np.ascontiguousarray(norm[:k]), vect, normt, bdl, fc)


def fix_mesh(inn: np.ndarray, nn: int) -> np.ndarray:
    """Corner fix of src/chmal.f (returns a corrected copy of `in`)."""
    out = np.array(inn, dtype=np.int32, order="C", copy=True)
    _check(load_library().spoc_fix_mesh(nn, out.shape[0], _i(out)), "fix_mesh")
    return out


def inter_only_new(old: Mesh, new_inn: np.ndarray) -> np.ndarray:
    """inter_only_new (src/adapt.f:1233-1258): old element each new one repeats, or 0."""
    new_inn = np.ascontiguousarray(new_inn, dtype=np.int32)
    out = np.zeros(new_inn.shape[0], np.int32)
    _check(load_library().spoc_inter_only_new(old.ne, new_inn.shape[0], _i(old.inn), _i(new_inn),
                                              _i(out)), "inter_only_new")
    return out


def locate_xy(mesh: Mesh, px, py, tk: int, reset_tk: int):
    """compare.f's sequential point location (src/compare.f:118-150):
    (elem, x1, y1, inside, tk after the last point)."""
    px = np.ascontiguousarray(px, dtype=np.float64)
    py = np.ascontiguousarray(py, dtype=np.float64)
    n = px.size
    elem = np.zeros(n, np.int32)
    inside = np.zeros(n, np.int32)
    x1 = np.zeros(n)
    y1 = np.zeros(n)
    t = C.c_int(tk)
    _check(load_library().spoc_locate_xy(mesh.ne, _i(mesh.inn), _i(mesh.itm), _i(mesh.tseg),
                                         _i(mesh.pseg), _d(mesh.xgr), _d(mesh.ygr), n, _d(px),
                                         _d(py), C.byref(t), reset_tk, _i(elem), _d(x1), _d(y1),
                                         _i(inside)), "locate_xy")
    return elem, x1, y1, inside, t.value


def locate_points(old: Mesh, new: Mesh, tinter: np.ndarray, T: Tables):
    """Point location of interpol (src/adapt.f:1690-1718): (pt_elem, pt_x, pt_y), (ne_new, ng)."""
    tinter = np.ascontiguousarray(tinter, dtype=np.int32)
    pe = np.zeros((new.ne, T.ng), np.int32)
    px = np.zeros((new.ne, T.ng))
    py = np.zeros((new.ne, T.ng))
    _check(load_library().spoc_locate_points(
        old.ne, _i(old.inn), _i(old.itm), _i(old.tseg), _i(old.pseg), _d(old.xgr), _d(old.ygr),
        new.ne, _i(new.inn), _d(new.xgr), _d(new.ygr), _i(tinter), T.ng, _d(T.xi), _d(T.yi),
        _i(pe), _d(px), _d(py)), "locate_points")
    return pe, px, py


def projection_points(mesh: Mesh, T: Tables):
    px = np.zeros((mesh.ne, T.ng))
    py = np.zeros((mesh.ne, T.ng))
    _check(load_library().spoc_projection_points(mesh.ne, _i(mesh.inn), _d(mesh.xgr), _d(mesh.ygr),
                                                 T.ng, _d(T.xi), _d(T.yi), _d(px), _d(py)),
           "projection_points")
    return px, py


def project(T: Tables, vals: np.ndarray, ld: int | None = None) -> np.ndarray:
    """calh (src/init.f:290-344): L2 projection of point values (ne, ng)."""
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    ne = vals.shape[0]
    ld = ld or T.nm
    out = np.zeros((ne, ld))
    _check(load_library().spoc_project(T.nc, T.ng, _d(T.wi), _d(T.pi2), _d(T.amm), ne, _d(vals),
                                       _d(out), ld), "project")
    return out


class Solver:
    """One device handle: tables and mesh resident, one CUDA stream."""

    def __init__(self, T: Tables, mesh: Mesh, variant: int | str, precision: int | str = FP64):
        if isinstance(precision, str):
            precision = PRECISIONS[precision]
        self.lib = load_library()
        self.T, self.mesh = T, mesh
        self.variant = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        self.nm = T.nm
        self._h = C.c_void_p()
        ts, ms = T.struct(), mesh.struct()
        _check(self.lib.spoc_create(C.byref(ts), C.byref(ms), self.variant, precision,
                                    C.byref(self._h)), "spoc_create")

    def close(self) -> None:
        if self._h:
            self.lib.spoc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_kernel_path(self, path: str) -> None:
        """'auto', 'generic' (runtime-sized kernels), 'templated' (compile-time
        sized) or, for the mixed precision, 'tensor' (tcgen05 volume kernel)."""
        code = {"auto": 0, "generic": 1, "templated": 2, "tensor": 3}[path]
        _check(self.lib.spoc_set_kernel_path(self._h, code), "set_kernel_path")

    def set_stream(self, stream_ptr: int) -> None:
        _check(self.lib.spoc_set_stream(self._h, C.c_void_p(stream_ptr)), "set_stream")

    def set_params(self, mu0: float, mb0: float, g0: float, hb: np.ndarray, fc=None, w0=None,
                   z0=None) -> None:
        ld = hb.shape[1]
        keep = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (fc, w0, z0, hb)]
        ptr = lambda a: _d(a) if a is not None else _DP()
        p = _Params(mu0, mb0, g0, ptr(keep[0]), ptr(keep[1]), ptr(keep[2]), ptr(keep[3]), ld)
        _check(self.lib.spoc_set_params(self._h, C.byref(p)), "set_params")

    def cal_var(self, u0, v0, h0):
        """One right-hand side with host arrays (ne, ld); returns (u1, v1, h1)."""
        ld = u0.shape[1]
        outs = [np.zeros_like(u0) for _ in range(3)]
        _check(self.lib.spoc_cal_var(self._h, ld, _d(u0), _d(v0), _d(h0), *map(_d, outs)),
               "spoc_cal_var")
        return tuple(outs)

    def cal_var_dev(self, ld: int, ptrs) -> None:
        _check(self.lib.spoc_cal_var_dev(self._h, ld, *[C.c_void_p(p) for p in ptrs]),
               "spoc_cal_var_dev")

    def set_state(self, u, v, h) -> None:
        _check(self.lib.spoc_set_state(self._h, u.shape[1], _d(u), _d(v), _d(h)), "set_state")

    def get_state(self, ld: int | None = None):
        ld = ld or self.nm
        outs = [np.zeros((self.mesh.ne, ld)) for _ in range(3)]
        _check(self.lib.spoc_get_state(self._h, ld, *map(_d, outs)), "get_state")
        return tuple(outs)

    def rk4_steps(self, dt: float, nsteps: int) -> None:
        _check(self.lib.spoc_rk4_steps(self._h, dt, nsteps), "rk4_steps")

    def rk4_steps_host(self, u, v, h, dt: float, nsteps: int) -> None:
        _check(self.lib.spoc_rk4_steps_host(self._h, u.shape[1], _d(u), _d(v), _d(h), dt, nsteps),
               "rk4_steps_host")

    def energy(self):
        k, p, m = C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.spoc_energy(self._h, C.byref(k), C.byref(p), C.byref(m)), "energy")
        return k.value, p.value, m.value

    def cfl(self):
        c, dt = C.c_double(), C.c_double()
        m = self.mesh
        _check(self.lib.spoc_cfl(self._h, m.nn, _i(m.inn), _d(m.xgr), _d(m.ygr), C.byref(c),
                                 C.byref(dt)), "cfl")
        return c.value, dt.value

    # -- solution-driven regridding (src/adapt.f) --
    def checkconv(self):
        """Per-element trace-jump indicators (umax, vmax, hmax) of the resident state."""
        out = [np.zeros(self.mesh.ne) for _ in range(3)]
        _check(self.lib.spoc_checkconv(self._h, *map(_d, out)), "checkconv")
        return tuple(out)

    def cal_conv(self, fac1: float, fac2: float, fac3: float) -> dict:
        """cal_conv flags of the resident state (src/adapt.f:1122-1193)."""
        fconv = np.zeros(self.mesh.ne, np.int32)
        fderaff = np.zeros(self.mesh.ne, np.int32)
        flags = np.zeros(3, np.int32)
        sup = C.c_double()
        _check(self.lib.spoc_cal_conv(self._h, fac1, fac2, fac3, _i(fconv), _i(fderaff), _i(flags),
                                      C.byref(sup)), "cal_conv")
        return {"fconv": fconv, "fderaff": fderaff, "conv": bool(flags[0]),
                "deraff": bool(flags[1]), "timedir": bool(flags[2]), "supmax": sup.value}

    def interpol_from(self, src: "Solver", tinter: np.ndarray, pt_elem=None, pt_x=None,
                      pt_y=None) -> None:
        """This handle's state := src's state re-projected onto this mesh (interpol)."""
        tinter = np.ascontiguousarray(tinter, dtype=np.int32)
        if pt_elem is None:
            args = (None, None, None)
        else:
            args = (_i(np.ascontiguousarray(pt_elem, dtype=np.int32)),
                    _d(np.ascontiguousarray(pt_x, dtype=np.float64)),
                    _d(np.ascontiguousarray(pt_y, dtype=np.float64)))
        _check(self.lib.spoc_interpol(self._h, src._h, _i(tinter), *args), "interpol")

    def interpol_from_dev(self, src: "Solver", tinter: int, pt_elem: int, pt_x: int,
                          pt_y: int) -> None:
        """interpol_from with device pointers (ints), enqueued on this handle's stream."""
        _check(self.lib.spoc_interpol_dev(self._h, src._h, tinter, pt_elem, pt_x, pt_y),
               "interpol_dev")

    def verif_rot(self) -> None:
        _check(self.lib.spoc_verif_rot(self._h), "verif_rot")

    def cfl2(self, ngraph: int = 10, dt_in: float = 0.0):
        """checkcfl2 (src/cfl.f:57-140) of the resident state: (cflmin, dt)."""
        c, dt = C.c_double(), C.c_double()
        m = self.mesh
        _check(self.lib.spoc_cfl2(self._h, ngraph, m.nn, _i(m.inn), _d(m.xgr), _d(m.ygr), dt_in,
                                  C.byref(c), C.byref(dt)), "cfl2")
        return c.value, dt.value

    def eval_points(self, elem, px, py) -> np.ndarray:
        """fsol of the resident u, v, h at (element, reference coordinates): (3, npts)."""
        elem = np.ascontiguousarray(elem, dtype=np.int32)
        px = np.ascontiguousarray(px, dtype=np.float64)
        py = np.ascontiguousarray(py, dtype=np.float64)
        out = np.zeros((3, elem.size))
        _check(self.lib.spoc_eval_points(self._h, elem.size, _i(elem), _d(px), _d(py), _d(out)),
               "eval_points")
        return out

    def lattice(self, ngraph: int = 10) -> np.ndarray:
        """write_gra's lattice values of the resident state: (ne, np, 5) = x, y, u, v, h."""
        m = self.mesh
        out = np.zeros((m.ne, ngraph * (ngraph + 1) // 2, 5))
        _check(self.lib.spoc_lattice(self._h, ngraph, m.nn, _i(m.inn), _d(m.xgr), _d(m.ygr),
                                     _d(out)), "lattice")
        return out

    def profile_rk4(self, dt: float, nsteps: int):
        """Per-kernel-kind milliseconds over nsteps steps (advances the state)."""
        ms = np.zeros(3)
        nk = C.c_int()
        _check(self.lib.spoc_profile_rk4(self._h, dt, nsteps, _d(ms), C.byref(nk)), "profile_rk4")
        return ms[: nk.value]

    # ---- tangent-linear model, adjoint, observation cost ----
    def _c(self, a):
        return np.ascontiguousarray(a, dtype=np.float64)

    def tlm_rhs(self, x, d):
        """J(x) d for x = (u, v, h), d = (du, dv, dh), arrays (ne, ld)."""
        x, d = [self._c(a) for a in x], [self._c(a) for a in d]
        out = [np.zeros_like(x[0]) for _ in range(3)]
        _check(self.lib.spoc_tlm_rhs(self._h, x[0].shape[1], *map(_d, x), *map(_d, d),
                                     *map(_d, out)), "tlm_rhs")
        return tuple(out)

    def adj_rhs(self, x, b):
        """J(x)^T b."""
        x, b = [self._c(a) for a in x], [self._c(a) for a in b]
        out = [np.zeros_like(x[0]) for _ in range(3)]
        _check(self.lib.spoc_adj_rhs(self._h, x[0].shape[1], *map(_d, x), *map(_d, b),
                                     *map(_d, out)), "adj_rhs")
        return tuple(out)

    def tlm_steps(self, x0, d, dt: float, nsteps: int):
        x0, d = [self._c(a) for a in x0], [self._c(a).copy() for a in d]
        _check(self.lib.spoc_tlm_steps(self._h, x0[0].shape[1], *map(_d, x0), *map(_d, d), dt,
                                       nsteps), "tlm_steps")
        return tuple(d)

    def adj_steps(self, x0, b, dt: float, nsteps: int):
        x0, b = [self._c(a) for a in x0], [self._c(a).copy() for a in b]
        _check(self.lib.spoc_adj_steps(self._h, x0[0].shape[1], *map(_d, x0), *map(_d, b), dt,
                                       nsteps), "adj_steps")
        return tuple(b)

    def set_observations(self, elem, basis, steps, values):
        elem = np.ascontiguousarray(elem, dtype=np.int32)
        basis = self._c(basis)
        steps = np.ascontiguousarray(steps, dtype=np.int32)
        values = self._c(values)
        self._obs = (elem, basis, steps, values)
        _check(self.lib.spoc_set_observations(self._h, elem.size, _i(elem), _d(basis), steps.size,
                                              _i(steps), _d(values)), "set_observations")

    def fwd_window(self, x0, dt: float, nsteps: int) -> float:
        x0 = [self._c(a) for a in x0]
        J = C.c_double()
        _check(self.lib.spoc_fwd_window(self._h, x0[0].shape[1], *map(_d, x0), dt, nsteps,
                                        C.byref(J)), "fwd_window")
        return J.value

    def bwd_window(self, x0, dt: float, nsteps: int, snaps: int):
        x0 = [self._c(a) for a in x0]
        g = [np.zeros_like(x0[0]) for _ in range(3)]
        J = C.c_double()
        _check(self.lib.spoc_bwd_window(self._h, x0[0].shape[1], *map(_d, x0), dt, nsteps, snaps,
                                        C.byref(J), *map(_d, g)), "bwd_window")
        return J.value, tuple(g)

    def set_adjoint_sweeps(self, precision: int | str) -> None:
        """Precision of the forward steps of the window and tangent-linear /
        adjoint step functions: 'fp64' (default) or 'mixed'."""
        if isinstance(precision, str):
            precision = PRECISIONS[precision]
        ts = self.T.struct()
        _check(self.lib.spoc_set_adjoint_sweeps(self._h, C.byref(ts), precision),
               "set_adjoint_sweeps")

    def adjoint_counters(self):
        f, a = C.c_longlong(), C.c_longlong()
        _check(self.lib.spoc_adjoint_counters(self._h, C.byref(f), C.byref(a)), "adjoint_counters")
        return f.value, a.value

    @property
    def launches(self) -> int:
        return int(self.lib.spoc_kernel_launches(self._h))


class Ensemble:
    """Members (Solver handles of precision 'mixed', free-slip, degree 3-6)
    stepped together: one cooperative launch per RK4 stage for all members.
    States, parameters and meshes stay in the members; each has its own dt."""

    def __init__(self, members):
        self.lib = load_library()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        self._e = C.c_void_p()
        _check(self.lib.spoc_ensemble_create(len(self.members), arr, C.byref(self._e)), "ensemble_create")

    def close(self) -> None:
        if self._e:
            self.lib.spoc_ensemble_destroy(self._e)
            self._e = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, blocks_per_sm: int, weight: int) -> None:
        _check(self.lib.spoc_ensemble_configure(self._e, blocks_per_sm, weight), "ensemble_configure")

    def info(self) -> dict:
        v = [C.c_int() for _ in range(5)]
        mb = (C.c_int * len(self.members))()
        _check(self.lib.spoc_ensemble_info(self._e, *map(C.byref, v), mb), "ensemble_info")
        return {"blocks_per_sm": v[0].value, "max_blocks_per_sm": v[1].value, "weight": v[2].value,
                "blocks": v[3].value, "graph": bool(v[4].value), "member_blocks": list(mb)}

    def steps(self, dts, nsteps: int, graph: bool = True) -> None:
        d = np.ascontiguousarray(dts, dtype=np.float64)
        _check(self.lib.spoc_ensemble_steps(self._e, _d(d), nsteps, int(graph)), "ensemble_steps")

    def balance(self, dts, rounds: int = 2) -> None:
        """Measured work model (weight 4): `rounds` steps with per-block cycle
        counters, blocks dealt again after each.  Advances the members."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        _check(self.lib.spoc_ensemble_balance(self._e, _d(d), rounds), "ensemble_balance")

    def autotune(self, dts, nsteps: int = 3) -> dict:
        """Times every layout (resident blocks per SM x work model: ne nm^p,
        p = 2, 1, 0.5, 0, or measured block cycles, weight 4) over nsteps
        steps after one warm-up step and keeps the fastest.  Advances the
        members' states: set them again afterwards."""
        import time
        best, table = None, []
        for bps in range(1, self.info()["max_blocks_per_sm"] + 1):
            for weight in (0, 1, 2, 3, 4):
                if weight == 4:
                    self.configure(bps, 2)
                    self.balance(dts, 2)
                else:
                    self.configure(bps, weight)
                self.steps(dts, 1)
                t = time.perf_counter()
                self.steps(dts, nsteps)
                ms = (time.perf_counter() - t) * 1e3 / nsteps
                table.append({"blocks_per_sm": bps, "weight": weight, "ms_per_step": ms})
                if best is None or ms < best["ms_per_step"]:
                    best = table[-1]
        self.configure(best["blocks_per_sm"], best["weight"])
        return {"best": best, "tried": table}
