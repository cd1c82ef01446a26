"""A library field written in the reference's dump format and loaded back
into another field, and a Tecplot file of a face field with its data
location's coordinates."""
import io

import numpy as np
import pytest

from moons_b200 import capi as G
from moons_b200 import refio as R
from tests.common import small_mesh_coords

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dl", [G.CC, G.FX, G.EY, G.NODE])
def test_field_dump_round_trip(dl):
    m = G.Mesh(*small_mesh_coords())
    a, b = m.field(dl), m.field(dl)
    a.upload(np.random.default_rng(dl).standard_normal(a.shape))
    buf = io.StringIO()
    R.export_field(a, buf)
    R.import_field(b, io.StringIO(buf.getvalue()))
    assert np.array_equal(a.download(), b.download())
    c = m.field(G.CC if dl != G.CC else G.FX)
    with pytest.raises(ValueError):
        R.import_field(c, io.StringIO(buf.getvalue()))


def test_tecplot_of_a_face_field():
    hs = small_mesh_coords()
    m = G.Mesh(*hs)
    f = m.field(G.FY)
    f.upload(np.random.default_rng(3).standard_normal(f.shape))
    co = R.location_coords(hs, R.n_along(G.FY))
    buf = io.StringIO()
    R.export_tecplot_3d(buf, co, [f.download()], "B_y", pad=1)
    (shape, d), = R.import_tecplot_3d(io.StringIO(buf.getvalue()))
    assert shape == tuple(s - 2 for s in f.shape)
    assert np.array_equal(d[..., 3], f.download()[1:-1, 1:-1, 1:-1])
    assert np.array_equal(d[:, 0, 0, 1], np.full(shape[0], co[1][1]))
