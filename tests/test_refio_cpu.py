"""The reference's field file formats (moons_b200.refio): grid_field
export_primitives / import_primitives dumps and 3-D Tecplot POINT files."""
import io
import os

import numpy as np
import pytest

from moons_b200 import refio as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EXPECTED = np.array([1.0, 2.5, -3.25e-2, 4.0, 5.0, 6.0, 7.0, 8.0, 9.0, 10.0, 11.0, 1.2e20]).reshape((2, 2, 3),
                                                                                                     order="F")


@pytest.mark.parametrize("name", ["grid_field_primitives_2x2x3.txt", "grid_field_primitives_2x2x3_variant.txt"])
def test_import_reference_dumps(name):
    a = R.import_primitives(os.path.join(GOLDEN, name))
    assert a.shape == (2, 2, 3)
    assert np.array_equal(a, EXPECTED)


def test_export_import_is_bit_identical():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((5, 4, 7)) * 10.0 ** rng.uniform(-300, 300, (5, 4, 7))
    a[0, 0, 0] = 0.0
    a[1, 0, 0] = -0.0
    a[2, 0, 0] = 5e-324          # smallest subnormal
    a[3, 0, 0] = np.finfo(np.float64).max
    buf = io.StringIO()
    R.export_primitives(a, buf)
    b = R.import_primitives(io.StringIO(buf.getvalue()))
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_export_layout_matches_the_reference_records():
    buf = io.StringIO()
    R.export_primitives(EXPECTED, buf)
    lines = buf.getvalue().splitlines()
    assert [int(x) for x in lines[0].split()] == [2, 2, 3]
    assert lines[1].strip() == "f     ="
    i = next(k for k, ln in enumerate(lines) if ln.strip() == "s     =")
    assert [int(x) for x in lines[i + 1].split()] == [2, 2, 3]
    assert lines[i + 2].strip() == "s_1D  ="
    assert int(lines[i + 3]) == 12


def test_inconsistent_dump_is_rejected():
    text = open(os.path.join(GOLDEN, "grid_field_primitives_2x2x3.txt")).read().replace("          12", "          13")
    with pytest.raises(ValueError):
        R.import_primitives(io.StringIO(text))


def test_truncated_dump_is_rejected():
    text = "\n".join(open(os.path.join(GOLDEN, "grid_field_primitives_2x2x3.txt")).read().splitlines()[:3])
    with pytest.raises(ValueError):
        R.import_primitives(io.StringIO(text))


def test_location_coordinates():
    hn = [np.array([-0.1, 0.0, 0.4, 1.0, 1.1]), np.array([0.0, 1.0, 2.0]), np.array([0.0, 2.0, 4.0, 6.0])]
    assert R.n_along(0) == (False, False, False)     # CC
    assert R.n_along(1) == (True, False, False)      # Fx
    assert R.n_along(4) == (False, True, True)       # Ex: CC along x, nodes along y and z
    cx, cy, cz = R.location_coords(hn, R.n_along(1))
    assert np.array_equal(cx, hn[0])
    assert np.allclose(cy, [0.5, 1.5]) and np.allclose(cz, [1.0, 3.0, 5.0])


@pytest.mark.parametrize("ncomp", [1, 2, 3])
def test_tecplot_point_file(ncomp):
    rng = np.random.default_rng(ncomp)
    hn = [np.linspace(0, 1, 6), np.linspace(0, 2, 5), np.linspace(0, 3, 7)]
    co = R.location_coords(hn, (False, False, False))        # CC: 5 x 4 x 6
    comps = [rng.standard_normal((5, 4, 6)) for _ in range(ncomp)]
    buf = io.StringIO()
    R.export_tecplot_3d(buf, co, comps, "U", pad=1, dir=3 if ncomp == 2 else 0)
    text = buf.getvalue()
    lines = text.splitlines()
    assert lines[0].strip() == ('TITLE = "3D Scalar Field"' if ncomp == 1 else 'TITLE = "3D Vector Field"')
    want = {1: '"x","y","z","U"', 2: '"x","y","z","U_x","U_y"', 3: '"x","y","z","U_x","U_y","U_z"'}[ncomp]
    assert lines[1].strip() == "VARIABLES = " + want
    assert lines[2].strip() == 'ZONE , T ="1", I =3, J =2, K =4 DATAPACKING = POINT'
    # records: i fastest, then j, then k; the pad layer dropped
    first = [float(x) for x in lines[3].split()]
    assert np.allclose(first[:3], [co[0][1], co[1][1], co[2][1]])
    second = [float(x) for x in lines[4].split()]
    assert np.isclose(second[0], co[0][2]) and np.isclose(second[1], co[1][1])
    (shape, d), = R.import_tecplot_3d(io.StringIO(text))
    assert shape == (3, 2, 4)
    for c in range(ncomp):
        assert np.array_equal(d[..., 3 + c], comps[c][1:-1, 1:-1, 1:-1])


def test_tecplot_needs_the_left_out_direction_for_two_components():
    co = R.location_coords([np.linspace(0, 1, 3)] * 3, (False, False, False))
    with pytest.raises(ValueError):
        R.export_tecplot_3d(io.StringIO(), co, [np.zeros((2, 2, 2))] * 2, "U")


# ---- planes, lines and histories ------------------------------------------------

def _field(rng, shape):
    return rng.standard_normal(shape)


@pytest.mark.parametrize("dir", [1, 2, 3])
@pytest.mark.parametrize("ncomp", [1, 2, 3])
def test_tecplot_plane_file(dir, ncomp):
    rng = np.random.default_rng(10 * dir + ncomp)
    hn = [np.linspace(0, 1, 6), np.linspace(0, 2, 5), np.linspace(0, 3, 7)]
    co = R.location_coords(hn, (False, False, False))        # CC: 5 x 4 x 6
    comps = [_field(rng, (5, 4, 6)) for _ in range(ncomp)]
    plane = 3
    buf = io.StringIO()
    R.export_tecplot_2d(buf, co, comps, "B", dir=dir, plane=plane, pad=1)
    lines = buf.getvalue().splitlines()
    d1, d2 = {1: (2, 3), 2: (1, 3), 3: (1, 2)}[dir]
    xyz = "xyz"
    assert lines[0].strip() == ('TITLE = "2D Scalar Field"' if ncomp == 1 else 'TITLE = "2D Vector Field"')
    if ncomp == 1:
        names = f'"B_{xyz[dir - 1]}"'
    elif ncomp == 2:
        names = f'"B_{xyz[d1 - 1]}","B_{xyz[d2 - 1]}"'
    else:
        names = '"B_x","B_y","B_z"'
    assert lines[1].strip() == f'VARIABLES = "{xyz[d1 - 1]}","{xyz[d2 - 1]}",{names}'
    s = (5, 4, 6)
    assert lines[2].strip() == f'ZONE , T ="1", I ={s[d1 - 1] - 2}, J ={s[d2 - 1] - 2} DATAPACKING = POINT'
    assert lines[3] == f"# Plane direction = {dir}"
    assert lines[4] == f"# Plane index({xyz[dir - 1]})  = {plane}"
    assert lines[5] == f"# Plane location({xyz[dir - 1]})  = {co[dir - 1][plane - 1]:.20f}"
    names_, zones = R.import_tecplot(io.StringIO(buf.getvalue()))
    (shape, d), = zones
    assert shape == (s[d1 - 1] - 2, s[d2 - 1] - 2)
    sl = [slice(1, -1)] * 3
    sl[dir - 1] = plane - 1
    for c in range(ncomp):
        assert np.array_equal(d[..., 2 + c], comps[c][tuple(sl)])
    assert np.array_equal(d[:, 0, 0], co[d1 - 1][1:-1]) and np.array_equal(d[0, :, 1], co[d2 - 1][1:-1])


@pytest.mark.parametrize("dir", [1, 2, 3])
@pytest.mark.parametrize("ncomp", [1, 2, 3])
def test_tecplot_line_file(dir, ncomp):
    rng = np.random.default_rng(20 * dir + ncomp)
    hn = [np.linspace(0, 1, 6), np.linspace(0, 2, 5), np.linspace(0, 3, 7)]
    co = R.location_coords(hn, (True, False, False))          # Fx: 6 x 4 x 6
    comps = [_field(rng, (6, 4, 6)) for _ in range(ncomp)]
    d1, d2 = {1: (2, 3), 2: (1, 3), 3: (1, 2)}[dir]
    line = (2, 3)
    buf = io.StringIO()
    R.export_tecplot_1d(buf, co, comps, "U", dir=dir, line=line)
    lines = buf.getvalue().splitlines()
    xyz = "xyz"
    assert lines[0].strip() == ('TITLE = "1D Scalar Field"' if ncomp == 1 else 'TITLE = "1D Vector Field"')
    names = {1: '"U"', 2: f'"U_{xyz[d1 - 1]}","U_{xyz[d2 - 1]}"', 3: '"U_x","U_y","U_z"'}[ncomp]
    assert lines[1].strip() == f'VARIABLES = "{xyz[dir - 1]}",{names}'
    s = (6, 4, 6)
    assert lines[2].strip() == f'ZONE , T ="1", I ={s[dir - 1]} DATAPACKING = POINT'
    assert lines[3] == f"# Line direction = {dir}"
    assert lines[4] == f"# Line index({xyz[d1 - 1]})  = {line[0]}"
    assert lines[5] == f"# Line index({xyz[d2 - 1]})  = {line[1]}"
    assert lines[6] == f"# Line location({xyz[d1 - 1]})  = {co[d1 - 1][line[0] - 1]:.20f}"
    assert lines[7] == f"# Line location({xyz[d2 - 1]})  = {co[d2 - 1][line[1] - 1]:.20f}"
    _, zones = R.import_tecplot(io.StringIO(buf.getvalue()))
    (shape, d), = zones
    assert shape == (s[dir - 1],)
    idx = [0, 0, 0]
    idx[d1 - 1] = line[0] - 1
    idx[d2 - 1] = line[1] - 1
    idx[dir - 1] = slice(None)
    for c in range(ncomp):
        assert np.array_equal(d[:, 1 + c], comps[c][tuple(idx)])
    assert np.array_equal(d[:, 0], co[dir - 1])


def test_history_file_and_its_reader():
    # the layout of the reference's probe histories (0-D): header, zone, (N, value)
    text = (' TITLE = "0D Field KU"\n VARIABLES = N ,"KU_test"\n ZONE DATAPACKING = POINT\n'
            '    0.300000000000E+001    0.125000000000E-030\n'
            '    0.530000000000E+002    0.250000000000E-027\n')
    names, zones = R.import_tecplot(io.StringIO(text))
    assert names == ["N", "KU_test"]
    (shape, d), = zones
    assert shape == (2,) and d[1, 0] == 53.0 and d[0, 1] == 0.125e-30
    buf = io.StringIO()
    R.export_tecplot_0d(buf, [2, 52, 102], [1e-3, 2.5e-3, -1.0], "KE")
    lines = buf.getvalue().splitlines()
    assert lines[0].strip() == 'TITLE = "0D Scalar Field"'
    assert lines[1].strip() == 'VARIABLES = "N","KE"'
    assert lines[2].strip() == "ZONE DATAPACKING = POINT"
    names, zones = R.import_tecplot(io.StringIO(buf.getvalue()))
    (shape, d), = zones
    assert names == ["N", "KE"] and shape == (3,)
    assert np.array_equal(d[:, 1], [1e-3, 2.5e-3, -1.0])


def test_plane_and_line_errors():
    co = R.location_coords([np.linspace(0, 1, 4)] * 3, (False, False, False))
    f = np.zeros((3, 3, 3))
    with pytest.raises(ValueError):
        R.export_tecplot_2d(io.StringIO(), co, [f], "p", dir=4, plane=1)
    with pytest.raises(ValueError):
        R.export_tecplot_2d(io.StringIO(), co, [f], "p", dir=1, plane=4)
    with pytest.raises(ValueError):
        R.export_tecplot_1d(io.StringIO(), co, [f], "p", dir=2, line=(0, 1))
    assert R.i_midplane(10) == 6
