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
