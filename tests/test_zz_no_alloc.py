"""moons_lap_var_noalloc (the sigma-weighted Laplacian with its face
temporaries in a built-in device array instead of the allocator) against
moons_lap_var, through the C-ABI.  This file is collected last so it also
runs after every other GPU test; it must pass alone as well."""
import numpy as np
import pytest

from moons_b200 import capi as G
from moons_b200 import mesh_gen as mg

pytestmark = pytest.mark.gpu

MOONS_ERR_LIMIT = 7


def _mesh(n, beta=1.05):
    hs = [mg.add_ghost_nodes(mg.roberts_both(0.0, 1.0, n, beta)) for _ in range(3)]
    return G.Mesh(*hs)


def _case(m, seed):
    rng = np.random.default_rng(seed)
    u = m.field(G.CC)
    u.upload(rng.standard_normal(u.shape))
    ks = [m.field(d) for d in (G.FX, G.FY, G.FZ)]
    for k in ks:
        k.upload(10.0 ** rng.uniform(-3, 3, k.shape))
    return u, ks


def test_noalloc_matches_lap_var_twice_in_a_row():
    m = _mesh(20)
    u, ks = _case(m, 11)
    ref = m.field(G.CC)
    G.lap_var(ref, u, ks)
    want = ref.download()
    scale = np.abs(want).max()
    for _ in range(2):  # the second call reuses the scratch set up by the first
        out = m.field(G.CC)
        out.fill(123.0)
        G.lap_var_noalloc(out, u, ks)
        got = out.download()
        assert np.abs(got - want).max() <= 1e-13 * scale
    # a second, different field through the same scratch
    u2, ks2 = _case(m, 12)
    G.lap_var(ref, u2, ks2)
    out = m.field(G.CC)
    G.lap_var_noalloc(out, u2, ks2)
    assert np.abs(out.download() - ref.download()).max() <= 1e-13 * np.abs(ref.download()).max()


def test_noalloc_takes_no_device_memory():
    """Free device memory is the same before and after calls of the no-alloc
    entry point (the library module, and with it the built-in array, is
    loaded by the fields' first kernels, before the first reading)."""
    import torch
    m = _mesh(20)
    u, ks = _case(m, 13)
    out = m.field(G.CC)
    G.lap_var_noalloc(out, u, ks)  # first call: the one-time address lookup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        G.lap_var_noalloc(out, u, ks)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_fields_beyond_the_scratch():
    # 52^3 cells: face temporaries of 55*54*54 = 160380 > 131072 points
    m = _mesh(52)
    u, ks = _case(m, 3)
    out = m.field(G.CC)
    with pytest.raises(G.MoonsError) as e:
        G.lap_var_noalloc(out, u, ks)
    assert e.value.code == MOONS_ERR_LIMIT
    assert "too large" in str(e.value)
