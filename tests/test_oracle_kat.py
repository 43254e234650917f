"""Known-answer tests of the FP64 oracle (CPU).

The reference ships no tests, fixtures or golden vectors and cannot be built
here (no Fortran compiler), so the oracle is pinned against closed-form
traveltimes: a homogeneous medium (T = r/v), a linear gradient
v = v0 + g z (T = acosh(1 + g^2 r^2 / (2 v_s v_r)) / g) and a flat reflector
(image source).  Tolerances are those of the reference's mixed first/second-
order fast-marching stencil on a 0.25 km grid.

The point-source tests seed the four corners of the source cell with the
exact time and run the heap FMM directly (propagate2d), away from region
boundaries: with a source on the seafloor the reference's initialisation sees
the source only through the corners of its cell and the region's top row
marches as a 1-D line, which is the reference's behaviour, not an eikonal
error.
"""
import numpy as np

from fmt2d_b200.synth import SmeshModel


def layered(nx=161, dx=0.25, depth=10.0, v_of_z=lambda z: 5.0 + 0 * z, sea=2.0, moho=8.0,
            vwater=1.5):
    xpos = dx * np.arange(nx, dtype=np.float64)
    topo = np.full(nx, sea)
    zrel = np.linspace(0.0, depth, 81)
    vel = np.repeat(v_of_z(zrel[:, None] + sea), nx, axis=1)
    return SmeshModel(xpos=xpos, topo=topo, zrel=zrel, vel=vel, vwater=vwater,
                      sed_z=np.full(nx, sea + 1.0), moho_z=np.full(nx, moho),
                      obs_x=np.array([xpos[nx // 2]]), name="layered")


def interior_source(oracle_lib, v_of_z, exact, sx, sz):
    m = layered(v_of_z=v_of_z)
    o = oracle_lib.Oracle(m)
    R = o.region(5)
    n = R["nnode"]
    st = -np.ones(n, np.int32)
    T = np.full(n, 1e20)
    gnode = R["i1"] > 0
    x = o.x0 + (R["i1"] - 1) * o.dx
    z = (R["i2"] - 1) * o.dx
    ix0, iz0 = int(np.floor(sx / o.dx)), int(np.floor(sz / o.dx))
    for a in (ix0, ix0 + 1):
        for b in (iz0, iz0 + 1):
            k = np.where(gnode & (R["i1"] == a + 1) & (R["i2"] == b + 1))[0][0]
            T[k] = exact(x[k], z[k])
            st[k] = 1
    st, T, gx, gz = o.propagate(5, st, T, np.zeros(n), np.zeros(n))
    return o, gnode, x, z, T


def _check(o, gnode, x, z, T, ex, sx, sz):
    r = np.hypot(x - sx, z - sz)
    rel = np.abs(T - ex) / np.maximum(ex, 1e-9)
    inside = gnode & (z > 2.5) & (z < 11.0)
    far = inside & (r > 20 * o.dx)
    mid = inside & (r > 10 * o.dx)
    assert rel[far].max() < 0.02 and rel[far].mean() < 0.005, (rel[far].max(), rel[far].mean())
    assert np.quantile(rel[mid], 0.99) < 0.03


def test_homogeneous_r_over_v(oracle_lib):
    sx, sz = 20.1, 6.07
    ex = lambda x, z: np.hypot(x - sx, z - sz) / 5.0
    o, gnode, x, z, T = interior_source(oracle_lib, lambda z: 5.0 + 0 * z, ex, sx, sz)
    _check(o, gnode, x, z, T, ex(x, z), sx, sz)


def test_linear_gradient(oracle_lib):
    v0, grad, sx, sz = 4.0, 0.1, 20.1, 6.07

    def ex(x, z):
        vs, vr = v0 + grad * sz, v0 + grad * z
        r2 = (x - sx) ** 2 + (z - sz) ** 2
        return np.arccosh(1.0 + grad * grad * r2 / (2.0 * vs * vr)) / grad

    o, gnode, x, z, T = interior_source(oracle_lib, lambda z: v0 + grad * z, ex, sx, sz)
    _check(o, gnode, x, z, T, ex(x, z), sx, sz)


def test_flat_reflector_image_source(oracle_lib):
    """PmP of the full phase recipe (seafloor source, down to the Moho,
    reflect, back up) against the image source at the seafloor."""
    m = layered(moho=8.0)
    o = oracle_lib.Oracle(m)
    sx = m.obs_x[0]
    o.forward(0, sx, 0b100)
    T = o.field(0, 5)[0]
    R = o.region(6)
    top = (R["i1"] == 0) & (R["i2"] == 2)     # seafloor interface nodes of region 6
    xs = o.x0 + (R["i3"][top] - 1) * o.dx
    zs = o.source_z(0)
    image = np.hypot(xs - sx, 2 * 8.0 - zs - zs) / 5.0
    off = np.abs(xs - sx)
    sel = (off > 2.0) & (off < 15.0)
    rel = np.abs(T[top][sel] - image[sel]) / image[sel]
    assert rel.max() < 0.012, rel.max()
