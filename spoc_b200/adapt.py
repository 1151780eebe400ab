"""Adaptive mesh with its refinement history, on the host (src/adapt.f).

The reference keeps every triangle it has made in a tree (COMMON
/adap_int/: `in_ab` vertices, `tlevel` level, `torigi` parent, `tenfan` the
four children; `tabsol` maps the solution's elements to tree nodes) and
rebuilds the solution mesh from the tree's leaves after each adaptive pass:

- refinement (`adapmaille`, src/adapt.f:532-788) splits a flagged leaf into
  four at its edge midpoints;
- the level rules keep the mesh conforming with neighbouring levels at most
  one apart: a flagged leaf next to a coarser leaf flags that leaf too
  (`check_level`, src/adapt.f:1350-1391), a leaf with two or three split
  edges is split as well, and a leaf with one split edge is bisected from the
  opposite vertex (the "double" triangles of `protridouble`,
  src/adapt.f:789-997), which are not tree nodes (their flags go to the leaf
  they came from: `preref`, src/adapt.f:1199-1231);
- coarsening (`deraffiner`, src/adapt.f:1393-1582) gives a node whose four
  children are leaves flagged by `cal_conv`'s `fderaff` (and not by `fconv`)
  back its place as a leaf.

This class restates those rules on its own data structure: node ids are
stable (a coarsened node's children are dropped, nothing is renumbered),
vertices are never removed from the tree (the solution mesh lists only the
vertices its triangles use, in tree order, as `deraffiner`'s compaction
does), and a coarsening that would leave the parent with two split edges or
an edge split twice is not made.  Vertex order stays counter-clockwise.
"""
from __future__ import annotations

import numpy as np

_EDGES = ((0, 1), (1, 2), (2, 0))


def _key(a: int, b: int):
    return (a, b) if a < b else (b, a)


class AdaptiveMesh:
    """Refinement tree over a base mesh (0-based `inn0` (ne, 3), vertex
    coordinates x, y).  `mesh()` gives the current solution mesh and, for
    each of its elements, the leaf it belongs to and whether it is a
    bisected half."""

    def __init__(self, inn0, x, y):
        inn0 = np.asarray(inn0)
        self.x = [float(v) for v in x]
        self.y = [float(v) for v in y]
        self.tri = [tuple(int(v) for v in t) for t in inn0]
        self.level = [0] * len(self.tri)
        self.parent = [-1] * len(self.tri)
        self.kids: list = [None] * len(self.tri)
        self.alive = [True] * len(self.tri)
        self.mid: dict = {}     # edge -> midpoint vertex
        self.edge_of: dict = {}  # midpoint vertex -> edge
        self._count: dict = {}   # leaf edge -> number of leaves using it
        for t in range(len(self.tri)):
            self._add_edges(t, 1)

    # -- leaf edge multiset --------------------------------------------------
    def _add_edges(self, t: int, s: int):
        a = self.tri[t]
        for i, j in _EDGES:
            k = _key(a[i], a[j])
            n = self._count.get(k, 0) + s
            if n:
                self._count[k] = n
            else:
                del self._count[k]

    def _split(self, a: int, b: int):
        """Midpoint of edge (a, b) when leaves on the other side use it."""
        m = self.mid.get(_key(a, b))
        return m if m is not None and _key(a, m) in self._count else None

    def _nsplit(self, t: int) -> int:
        a = self.tri[t]
        return sum(self._split(a[i], a[j]) is not None for i, j in _EDGES)

    def _double_split(self, t: int) -> bool:
        a = self.tri[t]
        for i, j in _EDGES:
            m = self._split(a[i], a[j])
            if m is not None and (self._split(a[i], m) is not None or self._split(m, a[j]) is not None):
                return True
        return False

    def leaves(self) -> list:
        return [t for t in range(len(self.tri)) if self.alive[t] and self.kids[t] is None]

    def _midpoint(self, a: int, b: int) -> int:
        k = _key(a, b)
        m = self.mid.get(k)
        if m is None:
            m = len(self.x)
            self.x.append(0.5 * (self.x[a] + self.x[b]))
            self.y.append(0.5 * (self.y[a] + self.y[b]))
            self.mid[k] = m
            self.edge_of[m] = k
        return m

    # -- refinement ----------------------------------------------------------
    def _coarser_owner_edge(self, p: int, q: int):
        """The edge of which (p, q) is a half, when a leaf uses that edge."""
        for u, v in ((p, q), (q, p)):
            e = self.edge_of.get(v)
            if e is not None and u in e:
                big = e
                if big in self._count:
                    return big
        return None

    def refine(self, marked) -> int:
        """Split the marked leaves into four, with the level and closure
        rules; returns the number of leaves split."""
        leaves = self.leaves()
        owners: dict = {}
        for t in leaves:
            a = self.tri[t]
            for i, j in _EDGES:
                owners.setdefault(_key(a[i], a[j]), []).append(t)
        M = set(int(t) for t in marked)
        while True:
            grow = set()
            for t in M:
                a = self.tri[t]
                for i, j in _EDGES:
                    big = self._coarser_owner_edge(a[i], a[j])
                    if big is not None:
                        grow.update(o for o in owners[big] if o not in M)
            will = set()
            for t in M | grow:
                a = self.tri[t]
                for i, j in _EDGES:
                    will.add(_key(a[i], a[j]))
            for t in leaves:
                if t in M or t in grow:
                    continue
                a = self.tri[t]
                c = sum(self._split(a[i], a[j]) is not None or _key(a[i], a[j]) in will for i, j in _EDGES)
                if c >= 2:
                    grow.add(t)
            if not grow:
                break
            M |= grow
        for t in sorted(M):
            a, b, c = self.tri[t]
            ab, bc, ca = self._midpoint(a, b), self._midpoint(b, c), self._midpoint(c, a)
            self._add_edges(t, -1)
            kids = []
            for tri in ((a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)):
                n = len(self.tri)
                self.tri.append(tri)
                self.level.append(self.level[t] + 1)
                self.parent.append(t)
                self.kids.append(None)
                self.alive.append(True)
                self._add_edges(n, 1)
                kids.append(n)
            self.kids[t] = kids
        return len(M)

    # -- coarsening ----------------------------------------------------------
    def coarsen(self, flagged) -> int:
        """Give back their place to the nodes whose four children are all
        flagged leaves; returns the number of nodes coarsened."""
        F = set(int(t) for t in flagged)
        cand = sorted({self.parent[t] for t in F if self.parent[t] >= 0})
        cand = [p for p in cand if self.kids[p] is not None
                and all(k in F and self.kids[k] is None for k in self.kids[p])]
        # all candidates at once (inside a refined patch every node has
        # refined neighbours until they are coarsened too), then the ones
        # that break the level rules are put back until none does
        kids_of = {}
        for p in cand:
            kids_of[p] = self.kids[p]
            for k in kids_of[p]:
                self._add_edges(k, -1)
            self._add_edges(p, 1)
            self.kids[p] = None
        active = set(cand)
        changed = True
        while changed:
            changed = False
            for p in sorted(active):
                if self._nsplit(p) >= 2 or self._double_split(p):
                    self._add_edges(p, -1)
                    for k in kids_of[p]:
                        self._add_edges(k, 1)
                    self.kids[p] = kids_of[p]
                    active.discard(p)
                    changed = True
        for p in active:
            for k in kids_of[p]:
                self.alive[k] = False
        return len(active)

    # -- the solution mesh ---------------------------------------------------
    def mesh(self):
        """(inn (ne, 3) 0-based over the used vertices, x, y, leaf, half,
        used): leaves in node order, each whole or as its two bisected halves
        (half = 1, 2); used[i] is the tree vertex of mesh vertex i."""
        out, leaf, half = [], [], []
        for t in self.leaves():
            a, b, c = self.tri[t]
            s = [self._split(p, q) for p, q in ((a, b), (b, c), (c, a))]
            n = sum(v is not None for v in s)
            if n > 1 or self._double_split(t):
                raise RuntimeError(f"tree node {t}: {n} split edges; the level rules were broken")
            if s[0] is not None:
                tris = [(a, s[0], c), (s[0], b, c)]
            elif s[1] is not None:
                tris = [(a, b, s[1]), (a, s[1], c)]
            elif s[2] is not None:
                tris = [(a, b, s[2]), (s[2], b, c)]
            else:
                tris = [(a, b, c)]
            for h, tri in enumerate(tris):
                out.append(tri)
                leaf.append(t)
                half.append(0 if len(tris) == 1 else h + 1)
        inn = np.array(out, dtype=np.int64)
        used = np.unique(inn)
        remap = np.full(len(self.x), -1, dtype=np.int64)
        remap[used] = np.arange(used.size)
        xs = np.array(self.x)[used]
        ys = np.array(self.y)[used]
        return (remap[inn].astype(np.int32), xs, ys, np.array(leaf, dtype=np.int64),
                np.array(half, dtype=np.int8), used)

    def flags_to_leaves(self, leaf, half, fconv, fderaff):
        """cal_conv's per-element flags as leaf sets (preref): a bisected
        half flags its leaf for refinement and never for coarsening; an
        element flagged both ways is only refined (deraffiner's first test)."""
        fconv = np.asarray(fconv, dtype=bool)
        fderaff = np.asarray(fderaff, dtype=bool) & ~fconv
        ref = set(leaf[fconv].tolist())
        coarse = set(leaf[fderaff & (half == 0)].tolist()) - ref
        return ref, coarse
