"""Red refinement with green closure for the ensemble meshes (host, no GPU)."""
import numpy as np

from spoc_b200 import workloads as W


def _edges(inn):
    e = np.sort(np.concatenate([inn[:, [0, 1]], inn[:, [1, 2]], inn[:, [2, 0]]]), axis=1)
    u, c = np.unique(e, axis=0, return_counts=True)
    return u, c


def _area(inn, x, y):
    a, b, c = inn[:, 0], inn[:, 1], inn[:, 2]
    return 0.5 * ((x[b] - x[a]) * (y[c] - y[a]) - (x[c] - x[a]) * (y[b] - y[a]))


def test_refinement_is_conforming_and_keeps_area():
    nn, inn, x, y = W.square_mesh(8, 1.0)
    inn = inn - 1
    area0 = _area(inn, x, y).sum()
    cx, cy = x[inn].mean(axis=1), y[inn].mean(axis=1)
    for level in range(3):
        marked = cx ** 2 + cy ** 2 < (0.2 * 0.7 ** level) ** 2
        inn, x, y = W.refine(inn, x, y, marked)
        cx, cy = x[inn].mean(axis=1), y[inn].mean(axis=1)
        a = _area(inn, x, y)
        assert (a > 0).all()                          # orientation kept
        assert abs(a.sum() - area0) < 1e-12
        _, c = _edges(inn)
        assert c.max() == 2                           # no hanging nodes
        assert (c == 1).sum() == 4 * 8                # the boundary is untouched
    assert inn.shape[0] > 2 * 8 * 8


def test_members_fit_the_configuration():
    ms = W.ensemble_members(64, 5)
    assert {m.cfg.nc for m in ms} == {3, 4, 5, 6}
    assert all(m.cfg.variant == "fs" for m in ms)
    sizes = [W.amr_mesh(m)[1].shape[0] for m in ms[:6]]
    assert all(4000 <= s <= 40000 for s in sizes), sizes
