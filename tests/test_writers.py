"""The reference's output files written from a context (CPU, host-only
context): write_model2d's smesh / refl / model_iter files
(src/inversion2d.f90:3842-3962) and write_residuals2d (:3342-3377).  The
smesh must read back through the library's own reader (read_smesh's list
-directed rules) with the grid velocity sampled by write_model2d's rule, the
interface and model_iter values must round to what was written, and the
residual lines must have the reference's fixed columns."""
import numpy as np

from fmt2d_b200 import io, synth
from fmt2d_b200.api import Fmt2d


def test_write_model_reads_back(tmp_path):
    m = synth.small_model()
    g = Fmt2d(-1).upload(m)
    io.write_model(str(tmp_path), g, 3, m.zrel, m.vwater, 0.33)
    r = io.read_smesh(str(tmp_path / "vgrid_1_vtype1.smesh"))
    assert r["vel"].shape == (m.zrel.size, m.nx)
    assert r["vwater"] == m.vwater and abs(r["vair"] - 0.33) < 1e-12
    assert np.abs(r["xpos"] - m.xpos).max() <= 5e-5
    assert np.abs(r["topo"] - m.topo).max() <= 5e-5
    assert np.abs(r["zrel"] - m.zrel).max() <= 5e-5
    inv, _, _ = g.inv_index()
    want = io.smesh_from_grid(m.xpos, g.interface(2), m.zrel, np.arange(g.nz) * g.dx,
                              g.velocity(), inv > 0)
    assert np.abs(r["vel"] - want).max() <= 5e-5
    # away from the velocity jumps the resampling round trip keeps the model
    smooth = synth.small_model(cb_amp=0.0)
    gs = Fmt2d(-1).upload(smooth)
    io.write_model(str(tmp_path), gs, 0, smooth.zrel, smooth.vwater)
    rs = io.read_smesh(str(tmp_path / "vgrid_1_vtype1.smesh"))
    assert np.median(np.abs(rs["vel"] - smooth.vel)) < 1e-3
    x, z = io.read_refl(str(tmp_path / "iface_4.refl"))
    assert np.abs(x - m.xpos).max() <= 5e-4 and np.abs(z - g.interface(4)).max() <= 5e-4


def test_model_iter_file(tmp_path):
    m = synth.small_model()
    g = Fmt2d(-1).upload(m)
    io.write_model(str(tmp_path), g, 7, m.zrel, m.vwater)
    lines = open(tmp_path / "model_iter7.dat").read().splitlines()
    assert lines[0] == "Iteration 7" and lines[1] == "vgrid 1 vtype 1"
    per_col = (g.nz + 9) // 10
    vals = [float(lines[2 + i][10 * k:10 * k + 10]) for i in range(per_col * g.nx)
            for k in range(len(lines[2 + i]) // 10)]
    v = np.array(vals).reshape(g.nx, g.nz)
    assert np.abs(v - g.velocity().T).max() <= 5e-5
    j = 2 + per_col * g.nx
    assert lines[j] == "iface 4"
    z = [float(l[12 * k:12 * k + 12]) for l in lines[j + 1:] for k in range(len(l) // 12)]
    assert np.abs(np.array(z) - g.interface(4)).max() <= 5e-5


def test_residual_lines(tmp_path):
    p = tmp_path / "res.dat"
    n = io.write_residuals(str(p), [0, 1, 2], [10.5, 20.25, 30.0], [0.005] * 3, [1, 3, 1],
                           [2.5, -1.0, 3.0], [2.4, 1.0, 3.0125], [True, True, False])
    lines = open(p).read().splitlines()
    assert n == 1 and len(lines) == 2
    assert lines[1] == "     1      10.500     0.005   1    2.500000    2.400000  1.000000E-01"


def test_arrival_files(tmp_path):
    a, o, e = (str(tmp_path / f) for f in ("arrivals.dat", "obs.dat", "entry_points.dat"))
    n = io.write_arrivals(a, o, e, [0, 4], [2, 2], [1, 3], [3.25, 7.0], [True, False],
                          [0.5, 0.25], [10.0, 0.0], [3.5, 0.0])
    assert n == 1
    assert open(a).read().splitlines() == [
        "       1       3       1       3.250000       2.750000    0.500000",
        "       5       3       3      -1.000000      -1.000000    0.250000"]
    assert open(o).read().splitlines() == ["1", "       1       3       1       3.250000"]
    assert open(e).read().splitlines() == [
        "1", "       1       3       1      10.000000       3.500000    0.500000"]
