"""Synthetic meshes, initial states and the benchmark configurations.

No mesh, initial state or oc.inp ships with the reference, so each
configuration is generated here from seeded inputs:
  * mesh: a square basin cut into n x n cells, each split into two right
    triangles as src/rmal.f:30-46 does, interior vertices optionally jittered
    by U(-j, j) * cell size with numpy's PCG64, then the corner fix of
    src/chmal.f:240-330 (spoc_fix_mesh);
  * state: analytic fields L2-projected onto the modal basis with the calh
    method of src/init.f:290-344 (spoc_project); depth hb = H constant as in
    src/init.f:246-252.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass, field
from types import SimpleNamespace

import numpy as np

from . import api
from .adapt import AdaptiveMesh


@dataclass
class Config:
    name: str
    variant: str
    nc: int
    ng: int
    ngf: int
    n: int                 # cells per side: ne = 2 n^2
    length: float = 1.0e6  # basin side (m), centred on the origin
    jitter: float = 0.0    # interior vertex jitter, fraction of the cell size
    f0: float = 1.0e-4
    beta: float = 0.0
    g0: float = 9.81
    depth: float = 4000.0
    mu0: float = 0.0
    mb0: float = 0.0
    ic: str = "gauss"
    steps: int = 100
    seed: int = 0
    dt_scale: float = 1.0  # fraction of the checkcfl step the workload runs at
    extra: dict = field(default_factory=dict)

    @property
    def nm(self) -> int:
        return (self.nc + 1) * (self.nc + 2) // 2

    @property
    def ne(self) -> int:
        return 2 * self.n * self.n


# The reference's own configuration space (see the survey of the benchmark
# configurations): C1 linear p3, C2 free-slip p6, C3 inviscid, C4 no-slip p4.
# C3 asks for degree 8 with the 42-point rule, whose mass matrix has rank
# <= 42 < 45 (dpotrf fails); C3 here runs degree 7 with the same rules.
# The checkcfl step (edge / nc * 0.3 / sqrt(g H), src/cfl.f:4-52) grows like
# 1/nc while the spectral radius of the degree-nc DG operator grows like nc^2:
# at degree 7 on the 256 x 256 basin the FP64 run at that step (0.5 s) blows
# up within 20 steps, at half of it (0.25 s) it stays bounded over 1000, so C3
# runs at half the checkcfl step.
CONFIGS = {
    "c1_lin_p3": Config("c1_lin_p3", "lin", 3, 12, 4, 32, ic="gauss", steps=1000, seed=1),
    "c2_fs_p6": Config("c2_fs_p6", "fs", 6, 33, 7, 128, jitter=0.2, beta=2.0e-11, mu0=100.0,
                       mb0=1.0e-3, ic="gauss8", steps=2000, seed=2),
    "c3_inv_p7": Config("c3_inv_p7", "inv", 7, 42, 9, 256, jitter=0.2, mu0=0.0, ic="kminus3",
                        steps=1000, seed=3, dt_scale=0.5),
    "c4_ns_p4": Config("c4_ns_p4", "ns", 4, 25, 5, 128, jitter=0.2, beta=2.0e-11, mu0=100.0,
                       mb0=1.0e-3, ic="gauss8", steps=200, seed=4),
}


def small(cfg: Config, n: int, **kw) -> Config:
    """The same physics, discretisation and cell size on an n x n cell basin.

    The initial-condition length scales (Gaussian widths, wavelengths) stay
    those of the full basin, so the fields remain resolved on the small one.
    """
    d = dict(cfg.__dict__)
    d.update(n=n, length=cfg.length * n / cfg.n)
    d.update(**kw)
    d["extra"] = dict(cfg.extra)
    d["extra"].setdefault("ic_length", cfg.length)
    return Config(**d)


def square_mesh(n: int, length: float = 1.0e6, jitter: float = 0.0, seed: int = 0, fix=None):
    """(nn, inn (ne,3) 1-based, xgr, ygr) of the rmal split, jittered, corner-fixed.

    fix(inn, nn) applies the corner fix (default: the library's spoc_fix_mesh)."""
    nx = n + 1
    h = length / n
    xs = -0.5 * length + h * np.arange(nx)
    X, Y = np.meshgrid(xs, xs, indexing="xy")  # node j*nx + i at (xs[i], xs[j])
    x, y = X.ravel().copy(), Y.ravel().copy()
    if jitter > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        d = rng.uniform(-jitter, jitter, size=(x.size, 2)) * h
        ii = np.arange(x.size)
        interior = (ii % nx > 0) & (ii % nx < nx - 1) & (ii // nx > 0) & (ii // nx < nx - 1)
        x[interior] += d[interior, 0]
        y[interior] += d[interior, 1]
    cells = np.arange(n * n)
    ci, cj = cells % n, cells // n
    ne1 = ci + 1 + nx * cj  # 1-based lower-left node (src/rmal.f:174)
    t1 = np.stack([ne1, ne1 + 1, ne1 + nx], axis=1)
    t2 = np.stack([ne1 + 1, ne1 + 1 + nx, ne1 + nx], axis=1)
    inn = np.empty((2 * n * n, 3), dtype=np.int32)
    inn[0::2] = t1
    inn[1::2] = t2
    nn = nx * nx
    inn = (fix or api.fix_mesh)(inn, nn)
    return nn, inn, x, y


def _ic_length(cfg: Config) -> float:
    return cfg.extra.get("ic_length", cfg.length)


def _gauss8(cfg: Config, rng):
    L, Lic = cfg.length, _ic_length(cfg)
    cx = rng.uniform(-0.35 * L, 0.35 * L, 8)
    cy = rng.uniform(-0.35 * L, 0.35 * L, 8)
    amp = rng.uniform(-2.0, 2.0, 8)
    wid = rng.uniform(0.05 * Lic, 0.15 * Lic, 8)  # 50-150 km for the 1000 km basin
    return cx, cy, amp, wid


def _kminus3(cfg: Config, rng, kmax: int = 12):
    k = np.arange(-kmax, kmax + 1)
    KX, KY = np.meshgrid(k, k, indexing="ij")
    kk = np.hypot(KX, KY)
    keep = (kk > 0) & (kk <= kmax)
    kx, ky, kk = KX[keep], KY[keep], kk[keep]
    amp = kk ** -2.0  # |eta_k|^2 ~ k^-4, E(k) ~ k |eta_k|^2 ~ k^-3
    phase = rng.uniform(0.0, 2.0 * np.pi, kx.size)
    return kx, ky, amp, phase


def _fields(cfg: Config, px, py, rng_state):
    """(eta, u, v) at physical points; u, v geostrophic where the IC asks."""
    g, L = cfg.g0, cfg.length
    if cfg.ic == "gauss":  # ftourbh-like Gaussian, 1 m, 100 km e-folding (src/fonc.f:42-50)
        eta = np.exp(-(px ** 2 + py ** 2) / (0.1 * _ic_length(cfg)) ** 2)
        return eta, np.zeros_like(eta), np.zeros_like(eta)
    f = cfg.f0 + cfg.beta * py
    if cfg.ic == "gauss8":
        cx, cy, amp, wid = rng_state
        eta = np.zeros_like(px)
        ex = np.zeros_like(px)
        ey = np.zeros_like(px)
        for a, x0, y0, w in zip(amp, cx, cy, wid):
            gsh = a * np.exp(-((px - x0) ** 2 + (py - y0) ** 2) / w ** 2)
            eta += gsh
            ex += gsh * (-2.0 * (px - x0) / w ** 2)
            ey += gsh * (-2.0 * (py - y0) / w ** 2)
    elif cfg.ic == "kminus3":
        kx, ky, amp, phase = rng_state
        two_pi_l = 2.0 * np.pi / _ic_length(cfg)
        eta = np.zeros_like(px)
        ex = np.zeros_like(px)
        ey = np.zeros_like(px)
        for a, p, qx, qy in zip(amp, phase, kx, ky):
            arg = two_pi_l * (qx * px + qy * py) + p
            eta += a * np.cos(arg)
            ex -= a * two_pi_l * qx * np.sin(arg)
            ey -= a * two_pi_l * qy * np.sin(arg)
        s = 0.5 / np.sqrt(np.mean(eta ** 2))
        eta, ex, ey = eta * s, ex * s, ey * s
    else:
        raise ValueError(cfg.ic)
    return eta, -g / f * ey, g / f * ex


@dataclass
class Problem:
    cfg: Config
    T: api.Tables
    mesh: api.Mesh
    u: np.ndarray
    v: np.ndarray
    h: np.ndarray
    hb: np.ndarray
    fc: np.ndarray
    w0: np.ndarray
    z0: np.ndarray
    dt: float
    # refinement history of an adapted mesh: (AdaptiveMesh, used, leaf, half)
    # as adapt_tree leaves it (None: the mesh is its own base mesh)
    adapt: object = None


def build_problem(cfg: Config, ld: int | None = None, tables: api.Tables | None = None) -> Problem:
    T = tables or api.build_tables(cfg.nc, cfg.ng, cfg.ngf)
    nm = T.nm
    ld = ld or nm
    nn, inn, x, y = square_mesh(cfg.n, cfg.length, cfg.jitter, cfg.seed)
    mesh = api.build_mesh(inn, x, y, cfg.nc, cfg.f0, cfg.beta, ld)
    rng = np.random.Generator(np.random.PCG64(1000 + cfg.seed))
    state = {"gauss": None, "gauss8": _gauss8, "kminus3": _kminus3}[cfg.ic]
    rs = state(cfg, rng) if state else None
    px, py = api.projection_points(mesh, T)
    eta, uu, vv = _fields(cfg, px, py, rs)
    h = api.project(T, eta, ld)
    u = api.project(T, uu, ld)
    v = api.project(T, vv, ld)
    hb = np.zeros((mesh.ne, ld))
    hb[:, 0] = cfg.depth
    w0 = np.zeros((mesh.ne, ld))
    z0 = np.zeros((mesh.ne, ld))
    # time step of checkcfl (src/cfl.f:4-52), evaluated on the host
    dt = cfl_dt(cfg.nc, mesh, cfg.g0, cfg.depth) * cfg.dt_scale
    return Problem(cfg, T, mesh, u, v, h, hb, mesh.fc, w0, z0, dt)


def cfl_dt(nc: int, mesh: api.Mesh, g0: float, depth: float) -> float:
    """checkcfl (src/cfl.f:4-52).  Below 1 s the reference's last branch,
    dfloat(int(cflmin*10)/10), is an integer division and always gives 0;
    the bound rounded down to one decimal is used there instead."""
    x, y, inn = mesh.xgr, mesh.ygr, mesh.inn - 1
    cc0 = np.sqrt(g0 * depth)
    best = 6000.0
    for a, b in ((0, 1), (0, 2), (1, 2)):
        dx = x[inn[:, b]] - x[inn[:, a]]
        dy = y[inn[:, b]] - y[inn[:, a]]
        dd = np.sqrt(dx * dx + dy * dy) / float(nc) * 0.30
        best = min(best, float(np.min(dd / cc0)))
    if best >= 100:
        return float(10 * int(best / 10))
    if best >= 10:
        return float(2 * int(best / 2))
    if best >= 1:
        return float(int(best))
    return float(int(best * 10)) / 10.0


def make_solver(p: Problem, precision: str = "fp64") -> api.Solver:
    s = api.Solver(p.T, p.mesh, p.cfg.variant, precision)
    s.set_params(p.cfg.mu0, p.cfg.mb0, p.cfg.g0, p.hb, p.fc, p.w0, p.z0)
    return s


def mass_norm(p: Problem, a: np.ndarray) -> float:
    """Physical L2 norm sqrt(sum_e det_e a_e^T ammo a_e) of a modal field."""
    x = a[:, :p.T.nm]
    return float(np.sqrt(np.sum(p.mesh.det * np.einsum("ei,ij,ej->e", x, p.T.ammo.T, x))))


def run_steps(p: Problem, precision: str, steps: int, path: str = "auto"):
    """(state, energy at the start, energy at the end) of `steps` RK4 steps
    from the problem's state in the given precision form."""
    s = make_solver(p, precision)
    s.set_kernel_path(path)
    s.set_state(p.u, p.v, p.h)
    e0 = s.energy()
    s.rk4_steps(p.dt, steps)
    e1 = s.energy()
    st = s.get_state()
    s.close()
    return st, e0, e1


def energy_drift(e0, e1) -> float:
    """Relative change of the total energy KE + PE (src/energy.f:3-96)."""
    return ((e1[0] + e1[1]) - (e0[0] + e0[1])) / (e0[0] + e0[1])


def precision_errors(p: Problem, steps: int, precision: str = "mixed", path: str = "auto",
                     ref=None) -> dict:
    """Relative L2 (mass-norm) errors of u, v, eta of a precision form against
    the FP64 form (bit-identical to the CPU oracle) after `steps` steps, and
    both runs' energy drift.  ref: an FP64 run_steps result to reuse."""
    ref = ref or run_steps(p, "fp64", steps)
    got = run_steps(p, precision, steps, path)
    err = {f: mass_norm(p, got[0][i] - ref[0][i]) / max(mass_norm(p, ref[0][i]), 1e-300)
           for i, f in enumerate(("u", "v", "eta"))}
    return {"steps": steps, "rel_l2_error_vs_fp64": err,
            "energy_drift": {"fp64": energy_drift(ref[1], ref[2]),
                             precision: energy_drift(got[1], got[2])}}


def locate(mesh: api.Mesh, px: np.ndarray, py: np.ndarray):
    """Element (1-based) and reference coordinates (xi, eta) of each point.

    The element map is x = x1 + ax (xi + 1) + bx (eta + 1) (src/shwwnl.f:384-397,
    src/init.f:330-331); a point belongs to the first element whose reference
    coordinates lie in the triangle xi, eta >= -1, xi + eta <= 0.
    """
    inn = mesh.inn - 1
    x1, y1 = mesh.xgr[inn[:, 0]], mesh.ygr[inn[:, 0]]
    ax, bx, ay, by, detai = (mesh.vect[:, k] for k in range(5))
    elem = np.zeros(px.size, dtype=np.int32)
    xi = np.zeros(px.size)
    eta = np.zeros(px.size)
    for o, (x, y) in enumerate(zip(px, py)):
        dx, dy = x - x1, y - y1
        s = (by * dx - bx * dy) * detai - 1.0
        t = (-ay * dx + ax * dy) * detai - 1.0
        inside = (s >= -1 - 1e-12) & (t >= -1 - 1e-12) & (s + t <= 1e-12)
        k = int(np.argmax(inside))
        if not inside[k]:
            raise ValueError(f"point {o} ({x}, {y}) is outside the mesh")
        elem[o], xi[o], eta[o] = k + 1, s[k], t[k]
    return elem, xi, eta


def basis_at(nc: int, xi: np.ndarray, eta: np.ndarray) -> np.ndarray:
    """phi_n(xi, eta) = P_k1(xi) P_k2(eta), modes kc1 outer, kc2 inner (src/nonlin.f:325-331)."""
    from numpy.polynomial import legendre as L
    cols = []
    for a in range(nc + 1):
        for b in range(nc + 1 - a):
            ca = np.zeros(a + 1)
            ca[a] = 1
            cb = np.zeros(b + 1)
            cb[b] = 1
            cols.append(L.legval(xi, ca) * L.legval(eta, cb))
    return np.stack(cols, axis=1)


def random_observations(p: Problem, nobs: int, seed: int):
    """nobs points uniform in the basin (seeded), with their elements and basis values."""
    rng = np.random.Generator(np.random.PCG64(seed))
    L = p.cfg.length
    px = rng.uniform(-0.5 * L, 0.5 * L, nobs)
    py = rng.uniform(-0.5 * L, 0.5 * L, nobs)
    elem, xi, eta = locate(p.mesh, px, py)
    return elem, basis_at(p.cfg.nc, xi, eta), px, py


def assimilation_window(p: Problem, s: api.Solver, nobs: int = 500,
                        steps=(50, 100, 150, 200), seed: int | None = None):
    """The C4 assimilation set-up: nobs seeded points uniform in the basin,
    eta observed at the given steps of a truth run that starts from the
    problem's state with seeded noise on the element means of eta; the
    observations are registered on solver s.  Returns (elem, basis, steps,
    values)."""
    seed = p.cfg.seed if seed is None else seed
    elem, basis, _, _ = random_observations(p, nobs, seed=seed)
    steps = np.asarray(steps, dtype=np.int32)
    rng = np.random.Generator(np.random.PCG64(7))
    truth = (p.u, p.v, p.h + 0.05 * rng.normal(size=p.h.shape) * (np.arange(p.h.shape[1]) < 1))
    s.set_state(*truth)
    vals, t_prev = [], 0
    for st in steps:
        s.rk4_steps(p.dt, int(st - t_prev))
        t_prev = st
        vals.append(np.sum(s.get_state()[2][elem - 1] * basis, axis=1))
    vals = np.array(vals)
    s.set_observations(elem, basis, steps, vals)
    return elem, basis, steps, vals


# ---------------------------------------------------------------------------
# Ensemble configuration C5: members on adapt.f-style refined meshes
# ---------------------------------------------------------------------------

def refine(inn: np.ndarray, x: np.ndarray, y: np.ndarray, marked: np.ndarray):
    """One level of red refinement with green closure (src/adapt.f:532-997).

    Marked triangles are split into four by their edge midpoints; a triangle
    with two or three split edges is marked too (until none is left), and a
    triangle with one split edge is bisected from the opposite vertex to the
    midpoint, so the result is conforming and neighbouring levels differ by
    at most one.  Vertex order (counter-clockwise) is kept.  inn is 0-based
    here; returns (inn, x, y)."""
    inn = np.asarray(inn)
    marked = np.array(marked, dtype=bool)
    ne = inn.shape[0]
    edges = [(0, 1), (1, 2), (2, 0)]
    key = lambda a, b: (a, b) if a < b else (b, a)
    while True:
        split = set()
        for t in np.nonzero(marked)[0]:
            for a, b in edges:
                split.add(key(inn[t, a], inn[t, b]))
        grow = []
        for t in np.nonzero(~marked)[0]:
            c = sum(key(inn[t, a], inn[t, b]) in split for a, b in edges)
            if c >= 2:
                grow.append(t)
        if not grow:
            break
        marked[grow] = True
    xs, ys = list(x), list(y)
    mid = {}

    def m(a, b):
        k = key(a, b)
        if k not in mid:
            mid[k] = len(xs)
            xs.append(0.5 * (x[a] + x[b]))
            ys.append(0.5 * (y[a] + y[b]))
        return mid[k]

    out = []
    for t in range(ne):
        a, b, c = (int(v) for v in inn[t])
        if marked[t]:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            out += [(a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)]
            continue
        s = [key(p, q) in split for p, q in ((a, b), (b, c), (c, a))]
        if s[0]:
            k = m(a, b)
            out += [(a, k, c), (k, b, c)]
        elif s[1]:
            k = m(b, c)
            out += [(a, b, k), (a, k, c)]
        elif s[2]:
            k = m(c, a)
            out += [(a, b, k), (k, b, c)]
        else:
            out.append((a, b, c))
    return np.array(out, dtype=np.int32), np.array(xs), np.array(ys)


@dataclass
class Member:
    cfg: Config
    center: tuple
    radius: float
    levels: int
    amplitude: float


def ensemble_members(count: int = 64, seed: int = 5) -> list:
    """Seeded members of configuration C5: degree 3-6, free-slip, a Gaussian
    eta bump of random centre, amplitude and width, and a mesh refined
    around it (1-3 levels on a 48, 64 or 80 square base, 4k-40k triangles)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    tables = {3: (12, 4), 4: (25, 5), 5: (27, 6), 6: (33, 7)}
    out = []
    for i in range(count):
        nc = int(rng.integers(3, 7))
        ng, ngf = tables[nc]
        n = int(rng.choice([48, 64, 80]))
        cfg = Config(f"c5_member{i:02d}", "fs", nc, ng, ngf, n, beta=2.0e-11, mu0=100.0,
                     mb0=1.0e-3, ic="bump", steps=500, seed=100 + i)
        L = cfg.length
        center = (float(rng.uniform(-0.2, 0.2) * L), float(rng.uniform(-0.2, 0.2) * L))
        out.append(Member(cfg, center, float(rng.uniform(0.1, 0.2) * L), int(rng.integers(1, 4)),
                          float(rng.uniform(0.5, 2.0))))
    return out


def amr_mesh(mb: Member):
    """Square basin (rmal split) refined `levels` times around the bump, the
    refinement radius shrinking by 0.7 per level; the refined region stays
    away from the walls, whose elements keep the base mesh's layout."""
    nn, inn, x, y = square_mesh(mb.cfg.n, mb.cfg.length)
    inn = inn - 1
    r = mb.radius
    for _ in range(mb.levels):
        cx = x[inn].mean(axis=1)
        cy = y[inn].mean(axis=1)
        marked = (cx - mb.center[0]) ** 2 + (cy - mb.center[1]) ** 2 < r * r
        inn, x, y = refine(inn, x, y, marked)
        r *= 0.7
    return x.size, (inn + 1).astype(np.int32), x, y


_TABLES = {}


def build_member(mb: Member) -> Problem:
    cfg = mb.cfg
    key = (cfg.nc, cfg.ng, cfg.ngf)
    if key not in _TABLES:
        _TABLES[key] = api.build_tables(*key)
    T = _TABLES[key]
    nn, inn, x, y = amr_mesh(mb)
    mesh = api.build_mesh(inn, x, y, cfg.nc, cfg.f0, cfg.beta)
    px, py = api.projection_points(mesh, T)
    w = 0.5 * mb.radius
    eta = mb.amplitude * np.exp(-((px - mb.center[0]) ** 2 + (py - mb.center[1]) ** 2) / w ** 2)
    ex = eta * (-2.0 * (px - mb.center[0]) / w ** 2)
    ey = eta * (-2.0 * (py - mb.center[1]) / w ** 2)
    f = cfg.f0 + cfg.beta * py
    h = api.project(T, eta)
    u = api.project(T, -cfg.g0 / f * ey)
    v = api.project(T, cfg.g0 / f * ex)
    hb = np.zeros((mesh.ne, T.nm))
    hb[:, 0] = cfg.depth
    z = np.zeros((mesh.ne, T.nm))
    dt = cfl_dt(cfg.nc, mesh, cfg.g0, cfg.depth)
    return Problem(cfg, T, mesh, u, v, h, hb, mesh.fc, z, z.copy(), dt)


# ---------------------------------------------------------------------------
# Solution-driven regridding: the refinement and coarsening pass of the
# adaptive driver (src/shwwnl_adap.f:375-450, src/adapt.f:5-187)
# ---------------------------------------------------------------------------

def adapt_problem(p: Problem, marked: np.ndarray):
    """The mesh of p with the marked elements refined (adapt_tree without
    coarsening): (Problem without state, tinter, (pt_elem, pt_x, pt_y))."""
    p1, tinter, loc, _ = adapt_tree(p, marked)
    return p1, tinter, loc


def calh2(T: api.Tables, mesh: api.Mesh, tinter: np.ndarray, old: np.ndarray, f, ld: int | None = None):
    """calh2 (src/adapt.f:303-373): the L2 projection of f(x, y) on the new
    elements (tinter == 0, by calh's method) and the old coefficients copied
    on the inherited ones."""
    ld = ld or old.shape[1]
    out = np.zeros((mesh.ne, ld))
    k = tinter > 0
    out[k] = old[tinter[k] - 1]
    if (~k).any():
        px, py = api.projection_points(mesh, T)
        out[~k] = api.project(T, f(px[~k], py[~k]), ld)
    return out


def _base_adapt(p: Problem):
    """Refinement history of a mesh that has none: its own elements as the
    base triangles (mesh vertices are the tree's vertices)."""
    tree = AdaptiveMesh(p.mesh.inn - 1, p.mesh.xgr, p.mesh.ygr)
    ne = p.mesh.ne
    return tree, np.arange(p.mesh.xgr.size), np.arange(ne, dtype=np.int64), np.zeros(ne, np.int8)


def _canon(t):
    """A triangle up to the rotation of its vertices (the corner fix rotates
    wall elements)."""
    i = min(range(3), key=lambda j: t[j])
    return (t[i], t[(i + 1) % 3], t[(i + 2) % 3])


def adapt_tree(p: Problem, fconv: np.ndarray, fderaff: np.ndarray | None = None,
               bathymetry=None):
    """One pass of the adaptive mesh (src/adapt.f:5-187): coarsening of the
    nodes whose four children carry fderaff (deraffiner), refinement of the
    leaves under fconv with the level rules (adapmaille, check_level,
    protridouble), the new mesh with its unchanged elements first in their
    old order, inter_only_new's tinter (vertices matched through the tree,
    since the compaction renumbers them) and the located quadrature points of
    the other elements.  Depth on the new mesh: calh2 of `bathymetry(x, y)`,
    or the constant depth of p (newinter, src/adapt.f:238-265); no wind.
    Returns (Problem without state, tinter, (pt_elem, pt_x, pt_y), info)."""
    cfg, T = p.cfg, p.T
    ld = p.hb.shape[1]
    tree0, used0, leaf0, half0 = p.adapt if p.adapt is not None else _base_adapt(p)
    tree = copy.deepcopy(tree0)
    fconv = np.asarray(fconv, dtype=bool)
    fderaff = np.zeros_like(fconv) if fderaff is None else np.asarray(fderaff, dtype=bool)
    ref, coarse = tree.flags_to_leaves(leaf0, half0, fconv, fderaff)
    ncoarse = tree.coarsen(coarse)
    nref = tree.refine(ref)
    inn, x, y, leaf, half, used = tree.mesh()
    # unchanged elements first, in their old order (inter_only_new matches
    # old elements in sequence), then the new ones in tree order
    old_tree = used0[p.mesh.inn - 1]
    old_pos = {_canon(tuple(t)): i for i, t in enumerate(old_tree.tolist())}
    new_tree = used[inn]
    pos = np.array([old_pos.get(_canon(tuple(t)), -1) for t in new_tree.tolist()])
    keep = np.nonzero(pos >= 0)[0]
    keep = keep[np.argsort(pos[keep], kind="stable")]
    order = np.concatenate([keep, np.nonzero(pos < 0)[0]])
    inn, leaf, half = inn[order], leaf[order], half[order]
    inn = api.fix_mesh(inn + 1, x.size)
    mesh = api.build_mesh(inn, x, y, cfg.nc, cfg.f0, cfg.beta, ld)
    # the old elements in the new vertex numbering (removed vertices: 0)
    remap = np.full(max(int(used0.max()), int(used.max())) + 1, -1, dtype=np.int64)
    remap[used] = np.arange(used.size)
    old_in_new = (remap[old_tree] + 1).astype(np.int32)
    tinter = api.inter_only_new(SimpleNamespace(ne=p.mesh.ne, inn=old_in_new), inn)
    loc = api.locate_points(p.mesh, mesh, tinter, T)
    if bathymetry is None:
        hb = np.zeros((mesh.ne, ld))
        hb[:, 0] = p.hb[0, 0]
    else:
        hb = calh2(T, mesh, tinter, p.hb, bathymetry, ld)
    z = np.zeros((mesh.ne, ld))
    dt = cfl_dt(cfg.nc, mesh, cfg.g0, cfg.depth) * cfg.dt_scale
    info = {"refined": nref, "coarsened": ncoarse}
    p1 = Problem(cfg, T, mesh, None, None, None, hb, mesh.fc, z, z.copy(), dt,
                 (tree, used, leaf, half))
    return p1, tinter, loc, info


def regrid_step(p: Problem, s: api.Solver, fac1: float, fac2: float, fac3: float,
                precision: str = "fp64", ngraph: int = 10):
    """One pass of the adaptive driver on the device state of s
    (src/adapt.f:5-187): cal_conv's indicator (src/adapt.f:1122-1193),
    coarsening and refinement of the flagged elements (adapt_tree), interpol
    of u, v, h onto the new mesh (src/adapt.f:1662-1745), verif_rot
    (src/shwwnl_adap.f:481-596) and checkcfl2's time step (src/cfl.f:57-140).
    Returns (new problem, new solver, info); the inputs when the mesh stays
    as it is."""
    cc = s.cal_conv(fac1, fac2, fac3)
    info = {"conv": cc["conv"], "timedir": cc["timedir"], "supmax": cc["supmax"],
            "flagged": int(cc["fconv"].sum()), "flagged_coarsen": int(cc["fderaff"].sum())}
    if not cc["conv"]:
        return p, s, info
    p1, tinter, loc, ainfo = adapt_tree(p, cc["fconv"], cc["fderaff"])
    info.update(ainfo)
    if ainfo["refined"] == 0 and ainfo["coarsened"] == 0:
        return p, s, info
    s1 = api.Solver(p1.T, p1.mesh, p.cfg.variant, precision)
    s1.set_params(p.cfg.mu0, p.cfg.mb0, p.cfg.g0, p1.hb, p1.fc, p1.w0, p1.z0)
    s1.interpol_from(s, tinter, *loc)
    s1.verif_rot()
    cflmin, dt = s1.cfl2(ngraph, p.dt)
    info.update({"ne_old": p.mesh.ne, "ne_new": p1.mesh.ne, "tinter": tinter,
                 "inherited": int((tinter > 0).sum()), "cflmin": cflmin, "dt_cfl2": dt})
    return p1, s1, info


def ensemble_adaptive_run(problems: list, solvers: list, nsteps: int, every: int, thresholds,
                          graph: bool = True, layout=(4, 2), precision: str = "mixed"):
    """An ensemble of adaptive runs: the members are stepped together (one
    cooperative launch per RK4 stage for all of them, api.Ensemble) and every
    `every` steps each member goes through the adaptive pass (regrid_step:
    cal_conv's indicator on the device, coarsening and refinement through its
    refinement history, interpol and verif_rot on the device); a member whose
    mesh changed continues on a new handle with the new mesh's time step and
    the ensemble is set up again for the new meshes.  `thresholds(i, p, s)`
    gives member i's (fac1, fac2, fac3).  Returns (problems, solvers, log)."""
    problems, solvers = list(problems), list(solvers)
    log = []
    done = 0
    while done < nsteps:
        k = min(every, nsteps - done)
        ens = api.Ensemble(solvers)
        ens.configure(*layout)
        ens.steps([p.dt for p in problems], k, graph)
        ens.close()
        done += k
        if done >= nsteps:
            break
        for i, (p, s) in enumerate(zip(problems, solvers)):
            p1, s1, info = regrid_step(p, s, *thresholds(i, p, s), precision=precision)
            if s1 is not s:
                problems[i], solvers[i] = p1, s1
                log.append({"step": done, "member": i, "ne_old": info["ne_old"], "ne_new": info["ne_new"],
                            "refined": info["refined"], "coarsened": info["coarsened"]})
    return problems, solvers, log


# ---------------------------------------------------------------------------
# compare.f: error of a state against the analytic standing wave
# ---------------------------------------------------------------------------

def compare_standing_wave(p: Problem, s: api.Solver, nx: int, ny: int, lx: float | None = None,
                          ly: float | None = None):
    """compare.f (src/compare.f:56-192): the resident state of s evaluated on
    the (nx-1) x (ny-1) points x0 = lx/2 (2i - nx)/(nx - 1), y0 likewise, each
    located by interlin's walk on the host and evaluated (fsol) on the device,
    against u = uc sin(2 pi x0 / lx), v = 0, h = hc cos(2 pi x0 / lx) with
    c0 = sqrt(10), uc = sin(0.2 pi) g0 / c0, hc = cos(0.2 pi).  Returns the
    reference's printed norms; the sums run in the reference's point order."""
    lx = lx or p.cfg.length
    ly = ly or p.cfg.length
    g0 = p.cfg.g0
    c0 = np.sqrt(10.0)
    pi = 4.0 * np.arctan(1.0)
    uc = np.sin(0.2 * pi) * g0 / c0
    hc = np.cos(0.2 * pi) * 1.0
    m = p.mesh
    _, _, _, _, tk1 = api.locate_xy(m, np.array([1.0e6]), np.array([1.0e6]), 1, 1)
    jj, ii = np.meshgrid(np.arange(1, ny), np.arange(1, nx), indexing="ij")
    x0 = 0.5 * lx * (2.0 * ii.ravel() - nx) / float(nx - 1)
    y0 = 0.5 * ly * (2.0 * jj.ravel() - ny) / float(ny - 1)
    elem, x1, y1, inside, _ = api.locate_xy(m, x0, y0, tk1, tk1)
    k = inside.astype(bool)
    vals = s.eval_points(elem[k], x1[k], y1[k])
    ud, vd, hd = vals
    xs = x0[k]
    uref = uc * np.sin(2.0 * pi * xs / lx)
    href = hc * np.cos(2.0 * pi * xs / lx)
    seq = lambda a: float(np.cumsum(a)[-1]) if a.size else 0.0  # left-to-right sum
    e1, e2, e3 = seq(np.abs(uref - ud)), seq(np.abs(vd)), seq(np.abs(href - hd))
    e4, e5, e6 = seq((uref - ud) ** 2), seq(vd ** 2), seq((href - hd) ** 2)
    k1 = int(k.sum())
    ps = m.pseg - 1
    dis = np.sqrt((m.xgr[ps[:, 0]] - m.xgr[ps[:, 1]]) ** 2 + (m.ygr[ps[:, 0]] - m.ygr[ps[:, 1]]) ** 2)
    return {"outside": int((~k).sum()), "inside": k1, "dx_mean": seq(dis) / float(m.nf),
            "abs_norm": (e1 / k1, e2 / k1, e3 / k1),
            "rms_norm": (np.sqrt(e4 / k1), np.sqrt(e5 / k1), np.sqrt(e6 / k1)),
            "rms_norm_v": float(np.sqrt((e4 + e5) / k1))}
