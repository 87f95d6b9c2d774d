"""The oracle's tree records (the definition the GPU tree build matches bit
for bit): nodes inside a walk group (at most 32 particles of one cloud) are
summed directly over their particle range in index order, larger nodes
combine their children left first.  Checked here against NumPy sums over
each node's range, and the direct rule against a Python restatement of the
same order.  No GPU."""
import numpy as np
import pytest

from oracle import oracle as O
from sph_2_b200 import ic


@pytest.fixture(scope="module")
def tree():
    n = 3000
    d = ic.evrard(n, seed=21)
    x, y, z = (d["pos"][:, k].copy() for k in range(3))
    keys = O.morton_keys(x, y, z)
    p = O.sort_perm(keys)
    x, y, z = x[p].copy(), y[p].copy(), z[p].copy()
    m = (d["m"] * (1 + 0.1 * np.cos(np.arange(n))))[p].copy()
    h = d["h"][p].copy()
    child, parent, first, last = O.build_radix_tree(keys[p])
    node, hmax = O.tree_moments(child, first, last, x, y, z, m, h)
    return dict(n=n, x=x, y=y, z=z, m=m, h=h, child=child, first=first, last=last, node=node,
                hmax=hmax)


def test_every_node_matches_its_particle_range(tree):
    t = tree
    pos = np.stack([t["x"], t["y"], t["z"]], 1)
    for nd in range(2 * t["n"] - 1):
        f, l = t["first"][nd], t["last"][nd] + 1
        mm, pp = t["m"][f:l], pos[f:l]
        M = mm.sum()
        c = (mm[:, None] * pp).sum(0) / M
        d = pp - c
        q = [(mm * d[:, a] * d[:, b]).sum() for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))]
        o = t["node"][nd]
        assert abs(o[3] / M - 1) < 1e-14
        assert np.max(np.abs(o[:3] - c)) < 1e-13
        if l - f > 1:  # a leaf's moments are 0 by definition
            scale = max(abs(v) for v in q[:3])
            assert np.max(np.abs(np.array(o[4:10]) - np.array(q))) < 1e-10 * scale
        else:
            assert not np.any(o[4:10])
        assert np.array_equal(o[10:13], pp.min(0)) and np.array_equal(o[13:16], pp.max(0))
        assert t["hmax"][nd] == t["h"][f:l].max()


def test_group_nodes_follow_the_direct_order(tree):
    t = tree
    cnt = t["last"] - t["first"] + 1
    inner = np.nonzero((cnt[: t["n"] - 1] <= 32) & (cnt[: t["n"] - 1] >= 2))[0]
    assert len(inner) > 100
    for nd in inner[:: max(1, len(inner) // 200)]:
        f, l = t["first"][nd], t["last"][nd]
        M = sx = sy = sz = 0.0
        for k in range(f, l + 1):
            M = M + t["m"][k]
            sx = sx + t["m"][k] * t["x"][k]
            sy = sy + t["m"][k] * t["y"][k]
            sz = sz + t["m"][k] * t["z"][k]
        cx, cy, cz = sx / M, sy / M, sz / M
        qxx = qyy = qzz = qxy = qxz = qyz = 0.0
        for k in range(f, l + 1):
            dx, dy, dz = t["x"][k] - cx, t["y"][k] - cy, t["z"][k] - cz
            tx, ty, tz = t["m"][k] * dx, t["m"][k] * dy, t["m"][k] * dz
            qxx = qxx + tx * dx; qxy = qxy + tx * dy; qxz = qxz + tx * dz
            qyy = qyy + ty * dy; qyz = qyz + ty * dz; qzz = qzz + tz * dz
        want = np.array([cx, cy, cz, M, qxx, qyy, qzz, qxy, qxz, qyz])
        assert np.array_equal(t["node"][nd][:10].view(np.uint64), want.view(np.uint64))
