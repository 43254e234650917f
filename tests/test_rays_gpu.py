"""Device ray backtrace, water-leg entry search and Frechet rows
(fmt2d_trace / fmt2d_frechet_rows) against the oracle's restatement of
trace_ray_from_receiver2d, find_optimal_entry_inv and
compute_frechet_for_ray2d.

Both sides trace on the same time fields (the device's, loaded into the
oracle), so the comparison isolates the tracer: identical valid flags,
receiver times within 1e-9 s, identical row index sets (bit-exact
parameter indexing) and every Frechet value within 1e-4 relative (north-star
tolerance; the two differ only in summation order), with an absolute floor
of 1e-6 grid steps of path length.  End to end (each side
on its own fields) receiver times must agree within 0.5 ms.
"""
import numpy as np
import pytest

from fmt2d_b200 import synth

pytestmark = pytest.mark.gpu


def _setup(oracle_lib, phases, seed=7):
    from fmt2d_b200.api import Fmt2d, fields_of, phase_mask
    m = synth.small_model(phases=phases, seed=seed)
    g = Fmt2d(0).upload(m).forward(m.obs_x, phases)
    o = oracle_lib.Oracle(m)
    mask = phase_mask(phases)
    for s, sx in enumerate(m.obs_x):
        o.forward(s, sx, mask)
    return m, g, o, fields_of(mask)


def _rows(rp, gi, gv, i):
    return gi[rp[i] - 1: rp[i + 1] - 1], gv[rp[i] - 1: rp[i + 1] - 1]


@pytest.mark.parametrize("phases", [(1,), (2,), (3,), (4,), (5,)])
def test_trace_and_rows_on_same_fields(oracle_lib, phases):
    m, g, o, tfs = _setup(oracle_lib, phases)
    pk = m.picks
    src, ph = pk[:, 0].astype(np.int32), pk[:, 1].astype(np.int32)
    t, valid, nnz = g.trace(src, ph, pk[:, 2], pk[:, 3])
    wt, ex, ez = g.trace_entries()
    assert len(pk) > 0
    own = [o.trace(int(p[0]), int(p[1]), p[2], p[3]) for p in pk]
    # same fields: load the device fields into the oracle
    for s in range(len(m.obs_x)):
        for tf in tfs:
            T, gx, gz = g.field(s, tf)
            o.set_field(s, tf, T, gx, gz)
    rp, gi, gv = g.frechet_rows(index_base=1)
    assert rp[0] == 1 and rp[-1] - 1 == nnz
    n_rows = 0
    for i, p in enumerate(pk):
        r = o.trace(int(p[0]), int(p[1]), p[2], p[3])
        assert bool(valid[i]) == r["valid"], (i, p)
        idx, val = _rows(rp, gi, gv, i)
        if not r["valid"]:
            assert idx.size == 0
            continue
        assert abs(t[i] - r["t"]) <= 1e-9, (i, t[i], r["t"])
        # the ray's receiver end (the seafloor entry point of an in-water
        # pick) is a point of the oracle's ray; the water leg runs from the
        # receiver to it at the water velocity
        assert np.hypot(r["pts"][:, 0] - ex[i], r["pts"][:, 1] - ez[i]).min() <= 1e-9
        leg = np.hypot(ex[i] - p[2], ez[i] - p[3]) / m.vwater if wt[i] > 0.0 else 0.0
        assert abs(wt[i] - leg) <= 1e-12
        np.testing.assert_array_equal(idx, r["idx"])
        n_rows += idx.size > 0
        if idx.size:   # a ray that stays in the water has no rows
            # per entry: 1e-4 relative, with an absolute floor of 1e-6 grid
            # steps of path length (entries are path length times bilinear
            # weights; the two sides add the same contributions in a
            # different order)
            err = np.abs(val - r["val"])
            assert np.all(err <= 1e-4 * np.abs(r["val"]) + 1e-6 * m.dx), err.max()
    assert n_rows >= 0.5 * len(pk)
    # end to end (the oracle on its own fields, traced before the fields were
    # replaced).  Valid flags can differ where a ray passes a grid node that
    # the reference seeds at zero distance from an interface node: its NaN
    # gradient survives or not by the heap's acceptance order (about 5% of the
    # PmP picks of this model).
    both = np.array([v and r["valid"] for v, r in zip(valid, own)])
    agree = np.mean([bool(v) == r["valid"] for v, r in zip(valid, own)])
    assert agree >= 0.93, agree
    dt = np.array([abs(t[i] - own[i]["t"]) for i in np.where(both)[0]])
    assert dt.size == 0 or dt.max() <= 0.5e-3, dt.max()


def test_trace_edge_cases(oracle_lib):
    """An empty pick list, a pick on an unsolved phase (invalid), and picks
    out of range (rejected)."""
    from fmt2d_b200 import _native as N
    m, g, o, tfs = _setup(oracle_lib, (1,))
    t, v, nnz = g.trace([], [], [], [])
    assert t.size == 0 and nnz == 0
    t, v, nnz = g.trace([0], [3], [m.obs_x[0] + 10.0], [0.005])   # PmP was not solved
    assert not v[0]
    with pytest.raises(N.Fmt2dError):
        g.trace([5], [1], [1.0], [0.005])
    with pytest.raises(N.Fmt2dError):
        g.trace([0], [6], [1.0], [0.005])


def test_trace_pg_401x121(oracle_lib):
    """Pg picks of three sources of the 401x121 model on shared fields."""
    from fmt2d_b200.api import Fmt2d, fields_of, phase_mask
    m = synth.config(0)
    sel = [0, 4, 9]
    srcs = m.obs_x[sel]
    g = Fmt2d(0).upload(m).forward(srcs, (1,))
    o = oracle_lib.Oracle(m)
    for s, sx in enumerate(srcs):
        o.forward(s, sx, phase_mask((1,)))
        for tf in fields_of(phase_mask((1,))):
            o.set_field(s, tf, *g.field(s, tf))
    pk = m.picks[np.isin(m.picks[:, 0], sel)].copy()
    pk[:, 0] = np.searchsorted(sel, pk[:, 0])
    t, valid, nnz = g.trace(pk[:, 0].astype(np.int32), pk[:, 1].astype(np.int32), pk[:, 2],
                            pk[:, 3])
    rp, gi, gv = g.frechet_rows(index_base=1)
    assert valid.mean() > 0.5
    for i, p in enumerate(pk):
        r = o.trace(int(p[0]), int(p[1]), p[2], p[3])
        assert bool(valid[i]) == r["valid"], (i, p)
        idx, val = _rows(rp, gi, gv, i)
        if not r["valid"]:
            continue
        assert abs(t[i] - r["t"]) <= 1e-9, (i, t[i], r["t"])
        np.testing.assert_array_equal(idx, r["idx"])
        if idx.size:
            assert np.abs(val - r["val"]).max() <= 1e-4 * np.abs(r["val"]).max()


def test_trace_times_only():
    """fmt2d_trace_times (the line search's times-only trace) returns the
    same receiver times and valid flags as fmt2d_trace, bit for bit, and
    leaves no Frechet rows to read."""
    from fmt2d_b200._native import Fmt2dError
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model(phases=(1, 2, 3))
    g = Fmt2d(0).upload(m)
    g.forward(m.obs_x, (1, 2, 3))
    P = m.picks
    args = (P[:, 0].astype(np.int32), P[:, 1].astype(np.int32), P[:, 2].copy(), P[:, 3].copy())
    t, v, _ = g.trace(*args)
    t2, v2 = g.trace_times(*args)
    assert np.array_equal(t.view(np.int64), t2.view(np.int64))
    assert np.array_equal(v, v2)
    with pytest.raises((Fmt2dError, RuntimeError)):
        g.frechet_rows()
    g.close()
