"""The C-ABI library loads without a GPU and exports every declared symbol."""
import re
import subprocess
from pathlib import Path

import pytest

from spoc_b200 import api

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "spoc_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "for", "while")))


def test_header_declares_the_drop_in_and_handle_api():
    names = declared_functions()
    for n in ("spoc_create", "spoc_destroy", "spoc_cal_var", "spoc_cal_var_dev", "spoc_rk4_steps",
              "spoc_rk4_steps_host", "spoc_energy", "spoc_cfl", "cal_var_",
              "spoc_register_commons", "spoc_build_tables", "spoc_build_mesh"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = api.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", str(api.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert getattr(lib, n) is not None


def test_build_targets_sm100a_only():
    from spoc_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "--fmad=false" in B.NVCC_FLAGS


def test_host_errors_without_gpu_are_status_codes():
    """Argument checks return status codes before any CUDA call."""
    lib = api.load_library()
    import ctypes as C
    h = C.c_void_p()
    assert lib.spoc_create(None, None, 0, 0, C.byref(h)) == 1
    assert lib.spoc_cal_var(None, 45, None, None, None, None, None, None) == 1
    assert b"null" in lib.spoc_last_error() or lib.spoc_last_error()


def test_create_argument_checks_before_any_cuda_call():
    """spoc_create validates its arguments on the host first: unknown variant
    or precision, a table with nm != (nc+1)(nc+2)/2, sizes past the built
    limits, missing pointers, an empty mesh, a non-positive mass factor."""
    import ctypes as C
    from spoc_b200 import workloads as W
    lib = api.load_library()
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 4))

    def create(variant=1, precision=0, tweak_t=None, tweak_m=None):
        ts, ms = p.T.struct(), p.mesh.struct()
        if tweak_t:
            tweak_t(ts)
        if tweak_m:
            tweak_m(ms)
        h = C.c_void_p()
        rc = lib.spoc_create(C.byref(ts), C.byref(ms), variant, precision, C.byref(h))
        assert not h.value
        return rc

    E_ARG, E_MATRIX, E_UNSUPPORTED = 1, 4, 7  # include/spoc_gpu.h
    assert create(variant=4) == E_ARG
    assert create(variant=-1) == E_ARG
    assert create(precision=9) == E_UNSUPPORTED
    assert create(tweak_t=lambda t: setattr(t, "nm", t.nm + 1)) == E_ARG
    assert create(tweak_t=lambda t: setattr(t, "ng", 65)) == E_UNSUPPORTED
    assert create(tweak_t=lambda t: setattr(t, "ngf", 11)) == E_UNSUPPORTED
    assert create(tweak_t=lambda t: setattr(t, "agx", None)) == E_ARG
    assert create(tweak_m=lambda m: setattr(m, "ne", 0)) == E_ARG
    assert create(tweak_m=lambda m: setattr(m, "itm", None)) == E_ARG
    amm = p.T.amm.copy()
    amm[0, 0] = -1.0
    ts = p.T.struct()
    ts.amm = api._d(amm)
    h = C.c_void_p()
    assert lib.spoc_create(C.byref(ts), C.byref(p.mesh.struct()), 1, 0, C.byref(h)) == E_MATRIX
