"""The hierarchy cache on disk (b2g_mesh_create_cached): the first build writes the agglomeration's
restriction maps under a content signature of its inputs; a second build with the same inputs loads
them, skips the pairing passes and must give the same hierarchy (every step's maps, coarse
addressing and the direction flag) and the same solve; changed inputs must not use the file.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from brae_b200 import cases  # noqa: E402


@pytest.fixture(scope="module")
def b2g():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import brae_b200.native as n
    return n


def _steps(mesh):
    return [mesh.step(i) for i in range(mesh.n_levels)]


@pytest.mark.parametrize("forward", [True, False])
def test_cache_round_trip(b2g, tmp_path, forward):
    c = cases.box_case(24, 20, 22, (2.0, 1.0, 1.0), 20.0, seed=31)
    path = str(tmp_path / "mesh.b2gh")
    plain = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, forward)
    first = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, forward, cache_path=path)
    assert not first.from_cache
    second = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, forward, cache_path=path)
    assert second.from_cache
    assert plain.n_levels == first.n_levels == second.n_levels
    assert plain.forward == first.forward == second.forward
    for a, b, d in zip(_steps(plain), _steps(first), _steps(second)):
        for key in a:
            assert np.array_equal(a[key], b[key]) and np.array_equal(a[key], d[key]), key
    ctl = b2g.controls_default(tolerance=1e-8, relTol=0.0, reduction="serial")
    x1, x2 = np.zeros(c.n_cells), np.zeros(c.n_cells)
    p1 = b2g.pcg_gamg_solve(plain, c.diag, c.coef, c.source, x1, ctl)[0]
    p2 = b2g.pcg_gamg_solve(second, c.diag, c.coef, c.source, x2, ctl)[0]
    assert tuple(p1) == tuple(p2)
    assert np.array_equal(x1, x2)


def test_cache_rejects_other_inputs(b2g, tmp_path):
    c = cases.box_case(16, 14, 12, (2.0, 1.0, 1.0), 8.0, seed=32)
    path = str(tmp_path / "mesh.b2gh")
    b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True, cache_path=path)
    Sf = c.Sf.copy()
    k = np.flatnonzero(Sf.reshape(-1))[3]
    Sf.reshape(-1)[k] *= 1.000001  # one face area component changed: another agglomeration input
    other = b2g.Mesh(c.lower, c.upper, Sf, c.magSf, c.n_cells, 10, True, cache_path=path)
    assert not other.from_cache
    again = b2g.Mesh(c.lower, c.upper, Sf, c.magSf, c.n_cells, 10, True, cache_path=path)
    assert again.from_cache  # the file now holds the changed mesh's agglomeration
    for flag in (False,):
        flipped = b2g.Mesh(c.lower, c.upper, Sf, c.magSf, c.n_cells, 10, flag, cache_path=path)
        assert not flipped.from_cache  # the direction flag is an input too
