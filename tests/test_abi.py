"""The C-ABI library loads, exports every symbol include/fmt2d_gpu.h
declares, and reports errors through codes and messages (CPU only: no
compute calls)."""
import ctypes as C
import subprocess

import numpy as np
import pytest


@pytest.fixture(scope="module")
def native():
    from fmt2d_b200 import build
    build.build()
    from fmt2d_b200 import _native
    return _native


def test_exports_every_declared_symbol(native):
    syms = native.header_symbols()
    assert "fmt2d_forward" in syms and len(syms) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    L = native.lib()
    for s in syms:
        assert hasattr(L, s)


def test_host_only_context_errors(native):
    from fmt2d_b200 import synth
    from fmt2d_b200.api import Fmt2d
    g = Fmt2d(-1)
    with pytest.raises(native.Fmt2dError, match="no model"):
        g.region_nnode(1)
    g.upload(synth.small_model())
    assert g.region_nnode(5) > 0
    with pytest.raises(native.Fmt2dError, match="host-only"):
        g.forward([10.0], (1,))
    L = native.lib()
    assert L.fmt2d_forward(g.h, np.array([1.0]), 1, 0) == -1     # empty phase mask
    assert L.fmt2d_forward(g.h, np.array([1.0]), 1, 64) == -1    # unknown phase
    assert L.fmt2d_region_nodes(g.h, 7, None, None, None, None) == -1
    h = C.c_void_p()
    assert L.fmt2d_ctx_create(C.byref(h), -5) != 0


def test_bad_model_rejected(native):
    from fmt2d_b200 import synth
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model()
    m.xpos = m.xpos[::-1].copy()
    with pytest.raises(native.Fmt2dError, match="xpos"):
        Fmt2d(-1).upload(m)


def test_argument_checks_of_later_entry_points(native):
    """Bad arguments give FMT2D_ERR_ARG (-1) before anything else; valid ones
    on a host-only context give FMT2D_ERR_STATE (-3) with a message, never a
    crash or a silent success."""
    from fmt2d_b200 import synth
    from fmt2d_b200.api import Fmt2d
    L = native.lib()
    g = Fmt2d(-1).upload(synth.small_model())
    ia, da = np.zeros(4, np.int32), np.zeros(4)
    i1, d1 = native.ptr(ia), native.ptr(da)
    nnz = C.c_longlong()
    # fmt2d_trace: negative count, null arrays with picks
    assert L.fmt2d_trace(g.h, i1, i1, d1, d1, -1, d1, i1, C.byref(nnz)) == -1
    assert L.fmt2d_trace(g.h, None, i1, d1, d1, 1, d1, i1, C.byref(nnz)) == -1
    assert L.fmt2d_trace(g.h, i1, i1, d1, d1, 1, d1, i1, C.byref(nnz)) == -3
    # fmt2d_frechet_rows: index base must be 0 or 1
    assert L.fmt2d_frechet_rows(g.h, i1, i1, d1, 2) == -1
    assert L.fmt2d_frechet_rows(g.h, i1, i1, d1, 1) == -3
    # fmt2d_set_frechet: sizes and base
    rpa = np.array([1, 1], np.int32)
    rp = native.ptr(rpa)
    assert L.fmt2d_set_frechet(g.h, 1, 0, rp, i1, d1, 1) == -1
    assert L.fmt2d_set_frechet(g.h, -1, 5, rp, i1, d1, 1) == -1
    assert L.fmt2d_set_frechet(g.h, 1, 5, rp, i1, d1, 3) == -1
    assert L.fmt2d_set_frechet(g.h, 1, 5, rp, i1, d1, 1) == -3
    # fmt2d_set_schedule: ranges
    assert L.fmt2d_set_schedule(g.h, -1.0, 6, 0) == -1
    assert L.fmt2d_set_schedule(g.h, 2.0e6, 6, 0) == -1
    assert L.fmt2d_set_schedule(g.h, 0.5, 0, 0) == -1
    assert L.fmt2d_set_schedule(g.h, 0.5, 65, 0) == -1
    assert L.fmt2d_set_schedule(g.h, 0.5, 6, -1) == -1
    assert L.fmt2d_set_schedule(g.h, 0.5, 6, 0) == -3
    # products and LSQR need a device
    assert L.fmt2d_spmv(g.h, 0, None, d1) == -1
    assert L.fmt2d_spmv(g.h, 0, d1, d1) == -3
    assert L.fmt2d_gtg_diag(g.h, None) == -1
    p = native.LsqrParams(1, 10, 1.0, 1.0, 1.0, 1.0, 1e-3)
    assert L.fmt2d_lsqr(g.h, None, d1, d1, d1, d1, None, None, None, None) == -1
    assert L.fmt2d_lsqr(g.h, C.byref(p), d1, d1, d1, d1, None, None, None, None) == -3
    buf = C.create_string_buffer(256)
    L.fmt2d_last_error(g.h, buf, 256)
    assert b"host-only" in buf.value
