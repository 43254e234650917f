"""Bit-exact model tables: region node numbering (propagate2d.f90:1505-1621,
ix outer / iz inner, then top and bottom interface nodes) and inversion
parameter numbering (frechet2d.f90:55-63, iz outer / ix inner) of the product's
host model build against the oracle (CPU, host-only context)."""
import numpy as np
import pytest

from fmt2d_b200 import synth


@pytest.fixture(scope="module")
def native():
    from fmt2d_b200 import build
    build.build()
    from fmt2d_b200.api import Fmt2d
    return Fmt2d


@pytest.mark.parametrize("which", ["small", 0, 1, 4])   # 4: the largest, 4001x601
def test_region_and_parameter_numbering(oracle_lib, native, which):
    m = synth.small_model() if which == "small" else synth.config(which)
    o = oracle_lib.Oracle(m)
    g = native(-1).upload(m)
    assert (g.nx, g.nz) == (o.nx, o.nz)
    assert g.dx == o.dx and g.x0 == o.x0
    for r in range(1, 7):
        R = o.region(r)
        i1, i2, i3 = g.region_nodes(r)
        assert i1.size == R["nnode"]
        np.testing.assert_array_equal(i1, R["i1"])
        np.testing.assert_array_equal(i2, R["i2"])
        np.testing.assert_array_equal(i3, R["i3"])
        # positions and velocities are the doubles the FP64 stencil uses:
        # they must be bit-identical to the restatement's
        x, z, v = g.region_geometry(r)
        np.testing.assert_array_equal(x, R["x"])
        np.testing.assert_array_equal(z, R["z"])
        np.testing.assert_array_equal(v, R["vel"])
    inv_o, nvp_o, np_o = o.inv_idx()
    inv_g, nvp_g, np_g = g.inv_index()
    np.testing.assert_array_equal(inv_g, inv_o)
    assert (nvp_g, np_g) == (nvp_o, np_o)


def test_edge_models(oracle_lib, native):
    """Ragged and degenerate geometry: a seafloor exactly on grid rows, a Moho
    crossing the sediment base, a 3-column model."""
    m = synth.small_model(nx=41, dx=0.25)
    m.topo[:] = 3.0                       # every seafloor node on a grid row
    m.sed_z[::2] = m.moho_z[::2] + 0.3    # sediment base below the Moho in places
    for mm in (m, synth.small_model(nx=3, dx=0.25)):
        o = oracle_lib.Oracle(mm)
        g = native(-1).upload(mm)
        for r in range(1, 7):
            R = o.region(r)
            i1, i2, i3 = g.region_nodes(r)
            np.testing.assert_array_equal(i1, R["i1"])
            np.testing.assert_array_equal(i2, R["i2"])
            np.testing.assert_array_equal(i3, R["i3"])
