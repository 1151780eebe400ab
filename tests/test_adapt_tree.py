"""Refinement history, coarsening and calh2 on the host (no GPU).

src/adapt.f ships no test data, so the tree (spoc_b200/adapt.py) is pinned by
properties with exact answers: a fresh tree is its base mesh; every mesh it
gives is conforming with neighbouring levels at most one apart; refining and
then coarsening everything gives back the base mesh, vertex for vertex; the
elements inter_only_new inherits are the same triangles; a field refined and
coarsened back through the oracle's interpol is the field again (the
children carry their parent's polynomial); a coarsening that would leave an
edge split twice is not made; calh2 copies inherited rows and projects the
others bit for bit like the oracle's calh.
"""
import numpy as np

from oracle import oracle as O
from spoc_b200 import workloads as W
from spoc_b200.adapt import AdaptiveMesh


def _problem(n=8):
    cfg = W.small(W.CONFIGS["c2_fs_p6"], n)
    p = W.build_problem(cfg)
    T = p.T
    OT = O.Tables(cfg.nc, cfg.ng, cfg.ngf, T.wi, T.xi, T.yi, T.wif, T.tif)
    return p, OT


def _omesh(p, mesh):
    return O.Mesh(mesh.inn, mesh.xgr, mesh.ygr, p.cfg.nc, p.cfg.f0, p.cfg.beta)


def _centre_flags(p, mesh, r):
    L = p.cfg.length
    cx = mesh.xgr[mesh.inn - 1].mean(axis=1)
    cy = mesh.ygr[mesh.inn - 1].mean(axis=1)
    return cx ** 2 + cy ** 2 < (r * L) ** 2


def _conforming(mesh):
    inn = mesh.inn - 1
    e = np.sort(np.concatenate([inn[:, [0, 1]], inn[:, [1, 2]], inn[:, [2, 0]]]), axis=1)
    _, c = np.unique(e, axis=0, return_counts=True)
    x, y = mesh.xgr, mesh.ygr
    a = (x[inn[:, 1]] - x[inn[:, 0]]) * (y[inn[:, 2]] - y[inn[:, 0]]) - \
        (x[inn[:, 2]] - x[inn[:, 0]]) * (y[inn[:, 1]] - y[inn[:, 0]])
    return c.max() == 2 and (a > 0).all(), int((c == 1).sum())


def _tri_set(mesh):
    return {tuple(sorted(t)) for t in mesh.inn.tolist()}


def test_fresh_tree_is_the_base_mesh():
    p, _ = _problem()
    tree = AdaptiveMesh(p.mesh.inn - 1, p.mesh.xgr, p.mesh.ygr)
    inn, x, y, leaf, half, used = tree.mesh()
    assert np.array_equal(inn + 1, p.mesh.inn)
    assert np.array_equal(x, p.mesh.xgr) and np.array_equal(y, p.mesh.ygr)
    assert np.array_equal(leaf, np.arange(p.mesh.ne)) and not half.any()
    assert np.array_equal(used, np.arange(x.size))


def test_refine_then_coarsen_gives_back_the_base_mesh():
    p, _ = _problem()
    ok, nwall = _conforming(p.mesh)
    assert ok
    p1, t1, _, i1 = W.adapt_tree(p, _centre_flags(p, p.mesh, 0.2))
    p2, t2, _, i2 = W.adapt_tree(p1, _centre_flags(p, p1.mesh, 0.1))
    assert i1["refined"] > 0 and i2["refined"] > 0 and p2.mesh.ne > p1.mesh.ne > p.mesh.ne
    tree = p2.adapt[0]
    assert max(tree.level[t] for t in tree.leaves()) == 2
    for q in (p1, p2):
        assert _conforming(q.mesh) == (True, nwall)   # the walls keep their layout
    q, passes = p2, 0
    while True:
        z = np.zeros(q.mesh.ne, bool)
        q1, tq, _, iq = W.adapt_tree(q, z, ~z)
        if iq["coarsened"] == 0:
            break
        assert _conforming(q1.mesh) == (True, nwall)
        assert iq["refined"] == 0 and 0 < (tq > 0).sum() < q1.mesh.ne
        q, passes = q1, passes + 1
    assert passes == 2
    assert _tri_set(q.mesh) == _tri_set(p.mesh)
    assert np.array_equal(q.mesh.xgr, p.mesh.xgr) and np.array_equal(q.mesh.ygr, p.mesh.ygr)


def test_inherited_elements_are_the_same_triangles():
    p, _ = _problem()
    p1, _, _, _ = W.adapt_tree(p, _centre_flags(p, p.mesh, 0.25))
    p2, _, _, _ = W.adapt_tree(p1, _centre_flags(p, p1.mesh, 0.1))
    z = np.zeros(p2.mesh.ne, bool)
    p3, t3, _, i3 = W.adapt_tree(p2, z, ~z)        # coarsening removes vertices
    assert i3["coarsened"] > 0 and p3.mesh.xgr.size < p2.mesh.xgr.size
    for old, new, tin in ((p2, p3, t3),):
        k = np.nonzero(tin)[0]
        assert k.size > 0 and np.array_equal(k, np.arange(k.size))  # unchanged ones first
        o = old.mesh.inn[tin[k] - 1] - 1
        n = new.mesh.inn[k] - 1
        assert np.array_equal(old.mesh.xgr[o], new.mesh.xgr[n])
        assert np.array_equal(old.mesh.ygr[o], new.mesh.ygr[n])
    # every element that is not inherited really is new
    old_tris = {tuple(np.round(np.c_[p2.mesh.xgr[t - 1], p2.mesh.ygr[t - 1]], 6).ravel())
                for t in p2.mesh.inn}
    for i in np.nonzero(t3 == 0)[0]:
        t = p3.mesh.inn[i]
        key = tuple(np.round(np.c_[p3.mesh.xgr[t - 1], p3.mesh.ygr[t - 1]], 6).ravel())
        assert key not in old_tris


def test_refined_and_coarsened_field_is_the_field_again():
    p, OT = _problem()
    OM = _omesh(p, p.mesh)
    a = p.h
    p1, t1, _, _ = W.adapt_tree(p, _centre_flags(p, p.mesh, 0.2))
    M1 = _omesh(p, p1.mesh)
    a1, *_ = O.interpol(OT, OM, M1, t1, a)
    z = np.zeros(p1.mesh.ne, bool)
    p2, t2, _, i2 = W.adapt_tree(p1, z, ~z)
    assert i2["coarsened"] > 0 and _tri_set(p2.mesh) == _tri_set(p.mesh)
    M2 = _omesh(p, p2.mesh)
    a2, *_ = O.interpol(OT, M1, M2, t2, a1)
    pos = {tuple(t): i for i, t in enumerate(p.mesh.inn.tolist())}
    idx = np.array([pos[tuple(t)] for t in p2.mesh.inn.tolist()])
    ref = a[idx]
    err = O.mass_norm(OT, M2, a2 - ref) / O.mass_norm(OT, M2, ref)
    assert err < 1e-11, err
    inh = t2 > 0
    assert np.array_equal(a2[inh], a1[t2[inh] - 1])


def test_coarsening_that_would_split_an_edge_twice_is_refused():
    p, _ = _problem()
    tree = AdaptiveMesh(p.mesh.inn - 1, p.mesh.xgr, p.mesh.ygr)
    # two neighbouring base triangles A, B
    inn = p.mesh.inn - 1
    A = p.mesh.ne // 2 + 3
    sa = {frozenset(e) for e in ((inn[A, 0], inn[A, 1]), (inn[A, 1], inn[A, 2]), (inn[A, 2], inn[A, 0]))}
    B = next(t for t in range(p.mesh.ne) if t != A and any(
        frozenset(e) in sa for e in ((inn[t, 0], inn[t, 1]), (inn[t, 1], inn[t, 2]), (inn[t, 2], inn[t, 0]))))
    tree.refine([A, B])
    shared = frozenset(set(inn[A]) & set(inn[B]))
    # B's child along the shared edge, split once more
    kb = next(k for k in tree.kids[B] if len(set(tree.tri[k]) & set(shared)) == 1 and any(
        tree.mid.get(tuple(sorted(shared))) == v for v in tree.tri[k]))
    tree.refine([kb])
    tree.mesh()
    before = tree.mesh()[0].copy()
    assert tree.coarsen(tree.kids[A]) == 0                       # A's edge would be split twice
    assert np.array_equal(tree.mesh()[0], before)
    assert tree.coarsen(tree.kids[B][:3]) == 0                   # not all four children flagged
    assert tree.coarsen(tree.kids[kb]) == 1                      # allowed: back to level 1
    assert tree.coarsen(tree.kids[A]) == 1                       # now A's edge is split once
    tree.mesh()


def test_flags_of_bisected_halves():
    p, _ = _problem()
    p1, _, _, _ = W.adapt_tree(p, _centre_flags(p, p.mesh, 0.2))
    tree, used, leaf, half = p1.adapt
    hv = np.nonzero(half > 0)[0]
    assert hv.size > 0
    f = np.zeros(p1.mesh.ne, bool)
    f[hv[0]] = True
    ref, coarse = tree.flags_to_leaves(leaf, half, f, f)
    assert ref == {int(leaf[hv[0]])} and not coarse          # refinement wins
    ref, coarse = tree.flags_to_leaves(leaf, half, np.zeros_like(f), f)
    assert not ref and not coarse                            # halves never coarsen


def test_calh2_copies_and_projects_like_calh():
    p, OT = _problem()
    p1, t1, _, _ = W.adapt_tree(p, _centre_flags(p, p.mesh, 0.2))
    L = p.cfg.length
    f = lambda x, y: 4000.0 - 500.0 * np.cos(np.pi * x / L) * np.sin(np.pi * y / L)
    old, _, _ = O.calh(OT, _omesh(p, p.mesh), f)
    got = W.calh2(p.T, p1.mesh, t1, old, f)
    ref, _, _ = O.calh(OT, _omesh(p, p1.mesh), f)
    k = t1 > 0
    assert np.array_equal(got[k], old[t1[k] - 1])
    assert np.array_equal(got[~k], ref[~k])
    # the hb of a regridded problem follows calh2 when a bathymetry is given
    p2, t2, _, _ = W.adapt_tree(p, _centre_flags(p, p.mesh, 0.2), bathymetry=f)
    assert p2.hb.shape == (p2.mesh.ne, p.hb.shape[1])


def test_refining_next_to_a_coarser_leaf_refines_it_first():
    """check_level: a flagged leaf whose edge is half of a coarser leaf's edge
    splits that leaf too, so no edge is ever split twice."""
    p, _ = _problem()
    tree = AdaptiveMesh(p.mesh.inn - 1, p.mesh.xgr, p.mesh.ygr)
    A = p.mesh.ne // 2 + 3
    tree.refine([A])
    level1 = set(tree.leaves())
    # a child of A on A's boundary: its outer edge is half of a base leaf's edge
    k = tree.kids[A][0]
    n = tree.refine([k])
    assert n > 1                                  # the coarser neighbour(s) went too
    split_base = [t for t in range(p.mesh.ne) if t != A and tree.kids[t] is not None]
    assert split_base and all(t in level1 and tree.level[t] == 0 for t in split_base)
    tree.mesh()                                   # raises if a rule were broken
    levels = [tree.level[t] for t in tree.leaves()]
    assert max(levels) == 2


def test_refinement_at_the_walls_and_back():
    """Refinement that reaches the walls and a corner (wall edges split, the
    corner fix rotating wall elements), then coarsening back: conforming
    meshes, valid mesh pointers, polynomials re-projected exactly, and the
    base mesh again at the end."""
    p, OT = _problem()
    L = p.cfg.length

    def wall_flags(mesh, d):
        cy = mesh.ygr[mesh.inn - 1].mean(axis=1)
        cx = mesh.xgr[mesh.inn - 1].mean(axis=1)
        return (cy < -0.5 * L + d * L) | ((cx > 0.5 * L - d * L) & (cy > 0.5 * L - d * L))

    def f(x, y):
        s, t = x / L, y / L
        return 0.3 + s - 2 * t + s * t + s ** p.cfg.nc - 0.5 * t ** p.cfg.nc

    q, passes = p, []
    for d in (0.15, 0.08):
        q1, t1, _, i1 = W.adapt_tree(q, wall_flags(q.mesh, d))
        assert i1["refined"] > 0
        ok, _ = _conforming(q1.mesh)
        M0, M1 = _omesh(p, q.mesh), _omesh(p, q1.mesh)
        assert ok and M1.check == 0 and M1.its_rc == 0
        a0, _, _ = O.calh(OT, M0, f)
        a1, _, _ = O.calh(OT, M1, f)
        got, *_ = O.interpol(OT, M0, M1, t1, a0)
        assert O.mass_norm(OT, M1, got - a1) < 1e-11 * O.mass_norm(OT, M1, a1)
        q = q1
    assert _conforming(q.mesh)[1] > _conforming(p.mesh)[1]   # wall edges were split
    for _ in range(4):
        z = np.zeros(q.mesh.ne, bool)
        q1, t1, _, i1 = W.adapt_tree(q, z, ~z)
        if i1["coarsened"] == 0:
            break
        M1 = _omesh(p, q1.mesh)
        assert _conforming(q1.mesh)[0] and M1.check == 0 and M1.its_rc == 0
        q = q1
    assert _tri_set(q.mesh) == _tri_set(p.mesh)
