"""B200 (sm_100a) implementation of SPOC's RK4 discontinuous-Galerkin
shallow-water right-hand side (the cal_var plug-in of dupontf/SPOC).

The compute path is the CUDA library spoc_b200/libspoc_gpu.so with the C ABI
of include/spoc_gpu.h; `api` binds it with ctypes, `workloads` generates the
synthetic meshes and initial states, `fortran_io` reads and writes the
reference's init.bin / temp.bin files.
"""
from . import api  # noqa: F401

__all__ = ["api"]
