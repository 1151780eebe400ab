"""Ensemble of basins (configuration C5): members with their own refined
meshes, degrees and time steps advanced together, one cooperative launch per
RK4 stage.  Each element is computed by the same kernel code as in a
single-member run, so an ensemble step reproduces the members' own
mixed-precision steps bit for bit, whatever the block layout and whether the
steps run from a CUDA graph."""
import dataclasses

import numpy as np
import pytest

from spoc_b200 import api
from spoc_b200 import workloads as W


def small_members():
    ms = W.ensemble_members(4, seed=11)
    out = []
    for mb, nc in zip(ms, (3, 4, 5, 6)):
        ng, ngf = {3: (12, 4), 4: (25, 5), 5: (27, 6), 6: (33, 7)}[nc]
        cfg = dataclasses.replace(mb.cfg, n=8, nc=nc, ng=ng, ngf=ngf)
        out.append(dataclasses.replace(mb, cfg=cfg, levels=2))
    return [W.build_member(m) for m in out]


def solver(p, prec="mixed"):
    s = W.make_solver(p, prec)
    s.set_state(p.u, p.v, p.h)
    return s


def mass_norm(p, a):
    """Physical L2 norm: sum_e det_e a_e^T ammo a_e (the coefficients of the
    modal basis are too ill-conditioned to compare directly)."""
    A = p.T.ammo.T
    return float(np.sqrt(np.sum(p.mesh.det * np.einsum("ei,ij,ej->e", a, A, a))))


def states(solvers):
    return [s.get_state() for s in solvers]


@pytest.mark.gpu
def test_ensemble_matches_members_run_alone():
    ps = small_members()
    assert len({p.T.nc for p in ps}) == 4
    dts = [p.dt for p in ps]
    alone = []
    for p in ps:
        s = solver(p)
        s.rk4_steps(p.dt, 5)
        alone.append(s.get_state())
    mem = [solver(p) for p in ps]
    ens = api.Ensemble(mem)
    ens.steps(dts, 5)
    for got, ref in zip(states(mem), alone):
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_layouts_and_graph_replay_agree():
    ps = small_members()
    dts = [p.dt for p in ps]
    results = []
    for bps, weight, graph in ((None, None, True), (1, 0, False), (1, 1, True), (2, 0, True)):
        mem = [solver(p) for p in ps]
        ens = api.Ensemble(mem)
        if bps is not None and bps <= ens.info()["max_blocks_per_sm"]:
            ens.configure(bps, weight)
        ens.steps(dts, 4, graph=graph)
        results.append(states(mem))
        info = ens.info()
        assert info["blocks"] == sum(info["member_blocks"])
        assert min(info["member_blocks"]) >= 1
        ens.close()
    for r in results[1:]:
        for x, y in zip(r, results[0]):
            for a, b in zip(x, y):
                assert np.array_equal(a, b)


@pytest.mark.gpu
def test_measured_balance_keeps_results():
    """spoc_ensemble_balance's steps (with block cycle counters) and the steps
    on the re-dealt layout give the same states as plain steps."""
    ps = small_members()
    dts = [p.dt for p in ps]
    ref_mem = [solver(p) for p in ps]
    api.Ensemble(ref_mem).steps(dts, 4)
    mem = [solver(p) for p in ps]
    ens = api.Ensemble(mem)
    with pytest.raises(api.SpocError):
        ens.configure(1, 4)  # no measurement yet
    ens.balance(dts, 2)
    info = ens.info()
    assert info["weight"] == 4 and info["blocks"] == sum(info["member_blocks"])
    ens.steps(dts, 2)
    for x, y in zip(states(mem), states(ref_mem)):
        for a, b in zip(x, y):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_ensemble_error_against_fp64():
    ps = small_members()
    dts = [p.dt for p in ps]
    mem = [solver(p) for p in ps]
    api.Ensemble(mem).steps(dts, 20)
    for p, s in zip(ps, mem):
        f = solver(p, "fp64")
        f.rk4_steps(p.dt, 20)
        a, b = s.get_state()[2], f.get_state()[2]
        assert mass_norm(p, a - b) <= 1e-5 * mass_norm(p, b)


@pytest.mark.gpu
def test_ensemble_rejects_fp64_members():
    p = small_members()[0]
    with pytest.raises(api.SpocError) as ei:
        api.Ensemble([solver(p, "fp64")])
    assert ei.value.code == 7


@pytest.mark.gpu
def test_adaptive_ensemble_matches_members_run_alone():
    """Members regridded inside a batched run (refined where cal_conv flags
    jumps, then coarsened back once every element is flagged calm) end where
    the same adaptive runs end one member at a time."""
    ps = small_members()[1:]

    def thresholds(i, p, s):
        if p.adapt is None:  # first pass: refine the jumpiest 10 %
            amax = np.maximum.reduce(s.checkconv())
            return float(np.quantile(amax, 0.9)), 0.0, 1e300
        return 1e300, 1e300, 1e301  # second pass: everything calm

    runs = []
    for mode in ("ensemble", "alone"):
        mem = [solver(p) for p in ps]
        if mode == "ensemble":
            p2, s2, log = W.ensemble_adaptive_run(ps, mem, 9, 3, thresholds)
        else:
            p2, s2, log = list(ps), mem, []
            for i in range(len(ps)):
                for _ in range(2):
                    s2[i].rk4_steps(p2[i].dt, 3)
                    q, t, info = W.regrid_step(p2[i], s2[i], *thresholds(i, p2[i], s2[i]),
                                               precision="mixed")
                    if t is not s2[i]:
                        log.append({"member": i, "ne_new": info["ne_new"],
                                    "coarsened": info["coarsened"]})
                    p2[i], s2[i] = q, t
                s2[i].rk4_steps(p2[i].dt, 3)
        runs.append((p2, states(s2), log))
    (pe, se, loge), (pa, sa, loga) = runs
    assert len(loge) == 2 * len(ps)
    key = lambda l: (l["member"], l["ne_new"], l["coarsened"])
    assert sorted(map(key, loge)) == sorted(map(key, loga))
    assert all(l["coarsened"] > 0 for l in loge if l["step"] == 6)
    for p, p0 in zip(pe, ps):  # back to the base meshes
        assert p.adapt is not None and p.mesh.ne == p0.mesh.ne
    for got, ref in zip(se, sa):
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
