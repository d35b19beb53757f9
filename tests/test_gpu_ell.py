"""The sliced ELL copy of a level's rows (levels of 65,536 cells or more): Amul and the correction
scaling read their rows from it, in the same entry order as the reference's lduMatrix::Amul
(src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu:62-88), so they stay bit for bit the oracle's;
a whole solve on such a mesh too (serial reductions)."""
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


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=torch.float64)


def test_amul_and_scale_on_sliced_levels(b2g, oracle):
    c = cases.box_case(72, 60, 50, (2.0, 1.0, 1.0), 20.0, True)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    rng = np.random.default_rng(4)
    checked = 0
    for lv in range(mesh.n_levels + 1):
        nc, nf = mesh.level_size(lv)
        if nc < 65536:
            continue
        lo, up = (c.lower, c.upper) if lv == 0 else (mesh.step(lv - 1)["lower"], mesh.step(lv - 1)["upper"])
        d, u = A.level(lv)
        x = rng.uniform(-1.0, 1.0, nc)
        y = dev(np.zeros(nc))
        A.amul(lv, dev(x), y)
        assert np.array_equal(y.cpu().numpy(), oracle.amul(lo, up, d, u, x)), lv
        checked += 1
    assert checked >= 2


def test_solve_on_sliced_levels_serial(b2g, oracle):
    c = cases.box_case(72, 60, 50, (2.0, 1.0, 1.0), 20.0)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), 1e-6, 0.0)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    x = dev(np.zeros(c.n_cells))
    perf = A.solve(dev(c.source), x, b2g.controls_default(reduction="serial"))[0]
    assert tuple(perf) == want["perf"]
    assert np.array_equal(x.cpu().numpy(), want["psi"])
