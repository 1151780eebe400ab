"""spoc_energy_noalloc: the energy diagnostic for callers that cannot allocate.

Some callers may not call cudaMalloc: it and cudaFree are prohibited while a
stream is captured into a CUDA graph and cudaFree synchronises the device, or
their host program owns all device memory.  They pass device arrays they
already own; the entry point keeps its per-element scratch in a static device
array.  Its result must equal the handle entry point spoc_energy (same
kernels, same summation order) and the CPU oracle's energy (1e-13 relative,
the energy tolerance of the other tests), on two calls in a row so that a
stale scratch would show.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from spoc_b200 import api
from spoc_b200 import workloads as W


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")


@pytest.mark.gpu
def test_energy_noalloc_matches_handle_entry_point():
    import torch

    lib = api.load_library()
    lib.spoc_energy_noalloc.restype = C.c_int
    lib.spoc_energy_noalloc.argtypes = [C.c_int] * 4 + [C.c_double] + [C.c_void_p] * 10
    p = W.build_problem(W.small(W.CONFIGS["c2_fs_p6"], 12), ld=45)
    T, m = p.T, p.mesh
    s = W.make_solver(p)
    rng = np.random.default_rng(11)
    states = [(p.u, p.v, p.h),
              (p.u + 0.1 * rng.normal(size=p.u.shape), p.v - 0.05, 2.0 * p.h)]
    vect = _dev(torch, m.vect)
    pi2 = _dev(torch, T.pi2)
    wi = _dev(torch, T.wi)
    ammo1 = _dev(torch, T.ammo[0, :])  # ammo(j, 1)
    hb = _dev(torch, p.hb)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    OT = O.Tables(T.nc, T.ng, T.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    OM = O.Mesh(m.inn, m.xgr, m.ygr, T.nc, p.cfg.f0, p.cfg.beta, ld=45)
    for u, v, h in states:  # two calls in a row through the shared scratch
        s.set_state(u, v, h)
        ref = s.energy()
        ora = O.energy(OT, OM, np.ascontiguousarray(u), np.ascontiguousarray(v),
                       np.ascontiguousarray(h), p.hb, p.cfg.g0)
        du, dv, dh = (_dev(torch, a) for a in (u, v, h))
        torch.cuda.synchronize()
        rc = lib.spoc_energy_noalloc(T.nc, T.ng, m.ne, 45, p.cfg.g0, du.data_ptr(), dv.data_ptr(),
                                     dh.data_ptr(), hb.data_ptr(), vect.data_ptr(),
                                     pi2.data_ptr(), wi.data_ptr(), ammo1.data_ptr(),
                                     out.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        for g, r, o in zip(got, ref, ora):
            assert g == pytest.approx(r, rel=1e-13, abs=1e-300)
            assert g == pytest.approx(o, rel=1e-13, abs=1e-300)


@pytest.mark.gpu
def test_energy_noalloc_rejects_meshes_beyond_its_scratch():
    lib = api.load_library()
    lib.spoc_energy_noalloc.restype = C.c_int
    lib.spoc_energy_noalloc.argtypes = [C.c_int] * 4 + [C.c_double] + [C.c_void_p] * 10
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.spoc_energy_noalloc(3, 12, 131073, 10, 9.81, *([dummy] * 9), None)
    assert rc == 7
