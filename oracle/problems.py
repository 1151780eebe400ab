"""Benchmark configurations set up by the CPU oracle alone.

TEST INFRASTRUCTURE ONLY (the fixture generator, the tests and the CPU legs
of bench.py): builds a configuration's mesh (the rmal split of the square
basin with its seeded jitter and the oracle's chmal corner fix, after
src/rmal.f:30-46 and src/chmal.f:240-330), the oracle's tables, the initial
state (the oracle's calh projection, src/init.f:290-344, of the seeded
analytic fields) and the checkcfl time step (src/cfl.f:4-52), without
loading the CUDA library.  The configurations, the seeded fields and the
quadrature tables are plain Python data from spoc_b200.workloads / .api.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from oracle import oracle as O
from spoc_b200 import api
from spoc_b200 import workloads as W


@dataclass
class OracleProblem:
    cfg: W.Config
    T: O.Tables
    M: O.Mesh
    u: np.ndarray
    v: np.ndarray
    h: np.ndarray
    hb: np.ndarray
    w0: np.ndarray
    z0: np.ndarray
    dt: float

    def rk4(self, u, v, h, nsteps, threads=None):
        """nsteps reference RK4 steps (src/shwwnl.f:233-284) in place."""
        c = self.cfg
        O.rk4(c.variant, self.T, self.M, u, v, h, self.M.fc, self.w0, self.z0, self.hb, c.mu0,
              c.mb0, c.g0, self.dt, nsteps, threads)

    def energy(self, u, v, h):
        return O.energy(self.T, self.M, u, v, h, self.hb, self.cfg.g0)


def oracle_problem(cfg: W.Config) -> OracleProblem:
    wi, xi, yi, wif, tif = api.quadrature(cfg.ng, cfg.ngf)
    T = O.Tables(cfg.nc, cfg.ng, cfg.ngf, wi, xi, yi, wif, tif)
    nn, inn, x, y = W.square_mesh(cfg.n, cfg.length, cfg.jitter, cfg.seed, fix=O.changemaille)
    M = O.Mesh(inn, x, y, cfg.nc, cfg.f0, cfg.beta)
    rng = np.random.Generator(np.random.PCG64(1000 + cfg.seed))
    state = {"gauss": None, "gauss8": W._gauss8, "kminus3": W._kminus3}[cfg.ic]
    rs = state(cfg, rng) if state else None
    cache = {}

    def field(k):
        def f(px, py):
            if "v" not in cache:
                cache["v"] = W._fields(cfg, px, py, rs)
            return cache["v"][k]
        return f

    h = O.calh(T, M, field(0))[0]
    u = O.calh(T, M, field(1))[0]
    v = O.calh(T, M, field(2))[0]
    hb = np.zeros((M.ne, T.nm))
    hb[:, 0] = cfg.depth
    w0 = np.zeros_like(hb)
    z0 = np.zeros_like(hb)
    dt = W.cfl_dt(cfg.nc, M, cfg.g0, cfg.depth) * cfg.dt_scale
    return OracleProblem(cfg, T, M, u, v, h, hb, w0, z0, dt)


# Small known-answer cases (tests/golden/small_rhs.json): the C2 physics on a
# 2 x 2 cell basin (8 triangles) at every tabulated degree and variant, with a
# seeded perturbation of the initial state so the nonlinear terms are active.
SMALL_DEGREES = [(3, 12, 4), (4, 25, 5), (5, 27, 6), (6, 33, 7), (7, 42, 9)]
SMALL_VARIANTS = ["lin", "fs", "ns", "inv"]


def small_case(nc: int, ng: int, ngf: int, variant: str) -> W.Config:
    import dataclasses
    return dataclasses.replace(W.small(W.CONFIGS["c2_fs_p6"], 2), nc=nc, ng=ng, ngf=ngf,
                               variant=variant)


def small_case_state(u, v, h, nc: int, variant: str):
    """The perturbed state of a small case: u, v, h plus seeded noise."""
    rng = np.random.default_rng(1000 * nc + SMALL_VARIANTS.index(variant))
    return (u + 0.1 * rng.normal(size=u.shape), v + 0.1 * rng.normal(size=v.shape),
            h + 0.05 * rng.normal(size=h.shape))
