"""Several models of uneven grid size solved in one fmt2d_forward_batch call
(the uneven multi-model batch): every context's fields must be bit-identical
to the same context solved alone, and a sampled source of the smallest model
must match the FP64 heap oracle (<= 0.5 ms on every reached node, identical
reached sets up to 2 nodes per field), all five phases."""
import numpy as np
import pytest

from fmt2d_b200 import synth
from fmt2d_b200.api import Fmt2d, fields_of, forward_batch, phase_mask

pytestmark = pytest.mark.gpu

PHASES = (1, 2, 3, 4, 5)


def _models():
    ms = [synth.uneven_model(k, max_obs=12) for k in (3, 0, 1)]
    return [(m, np.asarray(m.obs_x[:4], dtype=np.float64)) for m in ms]


def test_batch_equals_single_contexts():
    cases = _models()
    batch = [Fmt2d(0).upload(m) for m, _ in cases]
    forward_batch(batch, [x for _, x in cases], PHASES)
    for (m, x), gb in zip(cases, batch):
        ga = Fmt2d(0).upload(m)
        ga.forward(x, PHASES)
        for s in range(x.size):
            for tf in fields_of(phase_mask(PHASES)):
                Ta, gxa, _ = ga.field(s, tf)
                Tb, gxb, _ = gb.field(s, tf)
                assert np.array_equal(Ta, Tb), (m.name, s, tf)
                assert np.array_equal(gxa, gxb, equal_nan=True)
        ga.close()
    for g in batch:
        g.close()


def test_batch_sample_against_oracle(oracle_lib):
    cases = _models()
    batch = [Fmt2d(0).upload(m) for m, _ in cases]
    forward_batch(batch, [x for _, x in cases], PHASES)
    m, x = cases[0]
    o = oracle_lib.Oracle(m)
    s = 1
    o.forward(0, float(x[s]), phase_mask(PHASES))
    worst = 0.0
    for tf in fields_of(phase_mask(PHASES)):
        To = o.field(0, tf)[0]
        Tg = batch[0].field(s, tf)[0]
        ro, rg = To < 1e19, Tg < 1e19
        assert (ro != rg).sum() <= 2, tf
        both = ro & rg
        if both.any():
            worst = max(worst, float(np.abs(To[both] - Tg[both]).max()))
    assert worst <= 5e-4, worst
