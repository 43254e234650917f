"""The ray tracer's nearest-region-node search (rays.cu nearest_node), which
replaces the reference's scan of every region node (rays2d.f90:966-972,
1118-1127) by a search that widens column by column from the query.  A
restatement of that search over the library's own region tables must return
the node the full scan returns (the first in the reference's node order among
equal distances) for points inside, beside and far outside every region of
two models (CPU)."""
import numpy as np
import pytest

from fmt2d_b200 import synth
from fmt2d_b200.api import Fmt2d


def _tables(g, r):
    i1, i2, i3 = g.region_nodes(r)
    x, z, _ = g.region_geometry(r)
    grid = i1 > 0
    nx, dx, x0 = g.nx, g.dx, g.x0
    r0 = np.full(nx, 0, int)
    r1 = np.full(nx, -1, int)
    for c, row in zip(i1[grid] - 1, i2[grid] - 1):
        if r1[c] < r0[c]:
            r0[c] = r1[c] = row
        else:
            r0[c], r1[c] = min(r0[c], row), max(r1[c], row)
    ng = int(grid.sum())
    ztop, zbot = z[ng:ng + nx], z[ng + nx:ng + 2 * nx]
    xi = x[ng:ng + nx]
    return x, z, r0, r1, ztop, zbot, xi, ng, nx, dx, x0


def _column_search(t, px, pz):
    x, z, r0, r1, ztop, zbot, xi, ng, nx, dx, x0 = t
    best, key, node = 1e300, (3, 0, 0), -1
    # node index: grid nodes by column then row, then top / bottom interface
    base = np.concatenate([[0], np.cumsum(np.maximum(r1 - r0 + 1, 0))])
    c0 = min(nx - 1, max(0, int(np.floor((px - x0) / dx))))
    fr = int(np.floor(pz / dx))
    k = 0
    while True:
        near = False
        for c in ([c0] if k == 0 else [c0 - k, c0 + k]):
            if c < 0 or c >= nx:
                continue
            gx = x0 + c * dx
            if (px - gx) ** 2 > best and (px - xi[c]) ** 2 > best:
                continue
            near = True
            cands = []
            if r0[c] <= r1[c]:
                for q in (-1, 0, 1, 2):
                    row = min(r1[c], max(r0[c], fr + q))
                    cands.append(((px - gx) * (px - gx) + (pz - row * dx) * (pz - row * dx),
                                  (0, c, row), base[c] + row - r0[c]))
            cands.append(((px - xi[c]) * (px - xi[c]) + (pz - ztop[c]) * (pz - ztop[c]),
                          (1, c, 0), ng + c))
            cands.append(((px - xi[c]) * (px - xi[c]) + (pz - zbot[c]) * (pz - zbot[c]),
                          (2, c, 0), ng + nx + c))
            for d, kk, n in cands:
                if d < best or (d == best and kk < key):
                    best, key, node = d, kk, n
        if not near and k > 0:
            break
        k += 1
    return node


@pytest.mark.parametrize("model", ["small", 0])
def test_matches_full_scan(model):
    m = synth.small_model() if model == "small" else synth.config(0)
    g = Fmt2d(-1).upload(m)
    rng = np.random.default_rng(12)
    span_x, span_z = m.xpos[-1] - m.xpos[0], g.nz * g.dx
    for r in range(1, 7):
        t = _tables(g, r)
        x, z = t[0], t[1]
        pts = np.column_stack([rng.uniform(-0.2 * span_x, 1.2 * span_x, 150),
                               rng.uniform(-0.3 * span_z, 1.3 * span_z, 150)])
        # points on grid nodes and interface nodes (exact ties)
        pick = rng.integers(0, x.size, 40)
        pts = np.vstack([pts, np.column_stack([x[pick], z[pick]])])
        for px, pz in pts:
            d = (px - x) * (px - x) + (pz - z) * (pz - z)
            assert _column_search(t, px, pz) == int(np.argmin(d)), (r, px, pz)
