"""Model steps of the inversion (fmt2d_update_model: apply_model_step then
rebuild_geometry2d, src/inversion2d.f90:7173-7237, 3661-3816), host-only.

An interface step must give exactly the geometry a fresh model build with
the moved interface gives (region node tables, positions, velocities,
inversion numbering); a velocity step must change the region velocities to
the new grid values and nothing else."""
import dataclasses

import numpy as np
import pytest

from fmt2d_b200 import synth
from fmt2d_b200.api import Fmt2d
from fmt2d_b200._native import Fmt2dError


def _tables(g):
    out = []
    for r in range(1, 7):
        out.append(g.region_nodes(r))
        out.append(g.region_geometry(r))
    out.append(g.inv_index())
    return out


def _same(a, b):
    for x, y in zip(a, b):
        if isinstance(x, tuple):
            assert len(x) == len(y)
            for p, q in zip(x, y):
                if isinstance(p, np.ndarray):
                    assert np.array_equal(p, q)
                else:
                    assert p == q
        else:
            assert np.array_equal(x, y)


def test_interface_step_equals_fresh_build():
    m = synth.small_model()
    g = Fmt2d(-1).upload(m)
    moho = g.interface(4)
    assert np.array_equal(moho, m.moho_z)
    dz = 0.3 * np.sin(np.linspace(0.0, 3.0, m.nx))
    g.update_model(iface_z=moho + dz)
    ref = Fmt2d(-1).upload(dataclasses.replace(m, moho_z=m.moho_z + dz))
    assert np.array_equal(g.interface(4), ref.interface(4))
    _same(_tables(g), _tables(ref))


def test_velocity_step():
    m = synth.small_model()
    g = Fmt2d(-1).upload(m)
    v0 = g.velocity()
    before = _tables(g)
    inv, nvp, npar = g.inv_index()
    v1 = np.where(inv > 0, v0 * 1.02, v0)
    g.update_model(vel=v1)
    assert np.array_equal(g.velocity(), v1)
    after = _tables(g)
    # node tables and numbering unchanged; region velocities follow the grid
    for k in range(6):
        _same([before[2 * k]], [after[2 * k]])
        x0, z0, vel0 = before[2 * k + 1]
        x1, z1, vel1 = after[2 * k + 1]
        assert np.array_equal(x0, x1) and np.array_equal(z0, z1)
        if k >= 1:        # regions below the seafloor hold parameters
            assert not np.array_equal(vel0, vel1)
    _same([before[-1]], [after[-1]])
    g.update_model(vel=v0)
    _same(_tables(g), before)


def test_bad_updates_rejected():
    m = synth.small_model()
    g = Fmt2d(-1).upload(m)
    v = g.velocity()
    with pytest.raises(Fmt2dError):
        g.update_model(vel=np.where(v > 0, -1.0, v))
    with pytest.raises(ValueError):
        g.update_model(iface_z=np.zeros(3))
    assert np.array_equal(g.velocity(), v)
