"""The reference's input files (read_tomo2d.f90) read by the library
(fmt2d_read_smesh / fmt2d_read_refl / fmt2d_read_geom): round trips of
whole models, Fortran list-directed details (values over several lines,
commas, D exponents, repeat counts, the rest of a line dropped), the
reference's error cases, and a model built from files uploading the same
geometry as the arrays it came from (CPU)."""
import numpy as np
import pytest

from fmt2d_b200 import io, synth


def _write_model(tmp_path, m, t_obs=None):
    p = {k: str(tmp_path / k) for k in ("smesh", "sed", "moho", "geom")}
    io.write_smesh(p["smesh"], m.xpos, m.topo, m.zrel, m.vel, m.vwater)
    io.write_refl(p["sed"], m.xpos, m.sed_z)
    io.write_refl(p["moho"], m.xpos, m.moho_z)
    io.write_geom(p["geom"], m.obs_x, np.interp(m.obs_x, m.xpos, m.topo), m.picks, t_obs)
    return p


@pytest.mark.parametrize("which", ["small", 0])
def test_model_round_trip(tmp_path, which):
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model() if which == "small" else synth.config(0)
    t_obs = np.linspace(1.0, 9.0, len(m.picks))
    p = _write_model(tmp_path, m, t_obs)
    m2, g = io.model_from_files(p["smesh"], p["sed"], p["moho"], p["geom"])
    for k in ("xpos", "topo", "zrel", "vel", "obs_x", "picks"):
        np.testing.assert_array_equal(getattr(m2, k), getattr(m, k), err_msg=k)
    np.testing.assert_allclose(m2.sed_z, m.sed_z, rtol=0, atol=1e-12)
    np.testing.assert_allclose(m2.moho_z, m.moho_z, rtol=0, atol=1e-12)
    np.testing.assert_array_equal(g["t_obs"], t_obs)
    assert m2.vwater == m.vwater
    a, b = Fmt2d(-1).upload(m).inv_index(), Fmt2d(-1).upload(m2).inv_index()
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1:] == b[1:]


def test_list_directed_details(tmp_path):
    f = tmp_path / "m.smesh"
    # header with trailing text, xpos over two lines with commas, D exponents,
    # a repeat count, velocity records with extra values that are dropped
    f.write_text("3 2, 1.5D0 0.33 header comment\n"
                 "0.0, 1.0\n 2.0\n"
                 "3*2.5\n"
                 "0.0 1.0D+0\n"
                 "4.0 5.0 ignored\n"
                 "4.5 5.5\n"
                 "4.75,\n5.75\n")
    d = io.read_smesh(str(f))
    np.testing.assert_array_equal(d["xpos"], [0.0, 1.0, 2.0])
    np.testing.assert_array_equal(d["topo"], [2.5, 2.5, 2.5])
    np.testing.assert_array_equal(d["zrel"], [0.0, 1.0])
    np.testing.assert_array_equal(d["vel"], [[4.0, 4.5, 4.75], [5.0, 5.5, 5.75]])
    assert d["vwater"] == 1.5 and d["vair"] == 0.33


def test_refl_skips_blank_and_malformed_lines(tmp_path):
    f = tmp_path / "moho.dat"
    f.write_text("0.0 20.0\n\n   \n2.0, 20.5\nnot a line\n4.0 21.0 extra\n5.0\n")
    x, z = io.read_refl(str(f))
    np.testing.assert_array_equal(x, [0.0, 2.0, 4.0])
    np.testing.assert_array_equal(z, [20.0, 20.5, 21.0])


def test_reflector_on_its_own_nodes():
    xpos = np.arange(0.0, 20.0001, 0.25)
    xn = np.arange(0.0, 20.0001, 2.0)
    zn = 20.0 + np.sin(xn)
    z = io.iface_on_grid(xn, zn, xpos)
    np.testing.assert_allclose(z, np.interp(xpos, xn, zn), rtol=0, atol=1e-12)
    z2 = io.iface_on_grid(xn, zn, np.array([-3.0, 25.0]))   # clamped at the ends
    np.testing.assert_array_equal(z2, [zn[0], zn[-1]])


def test_errors(tmp_path):
    from fmt2d_b200 import _native as N
    with pytest.raises(N.Fmt2dError, match="cannot open"):
        io.read_smesh(str(tmp_path / "missing"))
    f = tmp_path / "bad.smesh"
    f.write_text("1 2 1.5 0.33\n")
    with pytest.raises(N.Fmt2dError, match="too small"):
        io.read_smesh(str(f))
    f.write_text("3 2 1.5 0.33\n0 1 2\n0 1\n")
    with pytest.raises(N.Fmt2dError, match="topo"):
        io.read_smesh(str(f))
    g = tmp_path / "bad.geom"
    g.write_text("1\ns 5.0 3.0 2\nr 1.0 0.005 1 2.0 0.05\n")
    with pytest.raises(N.Fmt2dError, match="irec = 2"):
        io.read_geom(str(g))
    r = tmp_path / "empty.dat"
    r.write_text("\nabc\n")
    with pytest.raises(N.Fmt2dError, match="no valid data"):
        io.read_refl(str(r))


def test_null_values_are_not_shifted(tmp_path):
    """Two commas with only blanks between them are a null value in
    list-directed input (the variable stays unset), not a wider separator:
    the values after it keep their positions, and the null item is reported
    as unreadable."""
    from fmt2d_b200 import _native as N
    f = tmp_path / "null.smesh"
    f.write_text("3 2 1.5 0.33\n0.0,, 2.0\n2.5 2.5 2.5\n0.0 1.0\n4 4 4\n5 5 5\n")
    with pytest.raises(N.Fmt2dError, match="xpos"):
        io.read_smesh(str(f))
    r = tmp_path / "null.dat"
    r.write_text("0.0 20.0\n1.0,,21.0\n2.0 , 22.0\n")
    x, z = io.read_refl(str(r))
    np.testing.assert_array_equal(x, [0.0, 2.0])
    np.testing.assert_array_equal(z, [20.0, 22.0])


def test_refl_line_limit_counts_every_nonblank_line(tmp_path):
    """read_refl stops at 100000 data lines; a further non-blank line fails
    the read even when it is malformed (read_tomo2d.f90:105-109 counts the
    line before parsing it)."""
    from fmt2d_b200 import _native as N
    r = tmp_path / "long.dat"
    body = "".join(f"{i * 0.01:.2f} 20.0\n" for i in range(100000))
    r.write_text(body + "\n  \n")
    x, _ = io.read_refl(str(r))
    assert x.size == 100000
    r.write_text(body + "not a line\n")
    with pytest.raises(N.Fmt2dError, match="exceeds 100000"):
        io.read_refl(str(r))
