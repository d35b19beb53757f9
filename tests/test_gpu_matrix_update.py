"""New coefficients on an existing matrix (b2g_matrix_set_coeffs, and the matrix b2g_pcg_gamg_solve keeps
per mesh), the per-level profile of a solve, and the sweep's bounded device-side waits.

The reference's pcgGamgSolve builds the Galerkin hierarchy of the matrix it is given in every call
(src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu:1081-1083); a matrix that takes new
coefficients must therefore solve exactly as a matrix created from them, in every form and with every
smoother (their derived layouts are refilled from the new values), while keeping its buffers so that
its captured iteration graphs are replayed.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from brae_b200 import cases  # noqa: E402

FIELD_RTOL = 1e-10


@pytest.fixture(scope="module")
def b2g():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import brae_b200.native as n
    return n


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.fixture(scope="module")
def pair_of_systems():
    # one mesh, two coefficient sets: single-phase and the 1000:1 two-phase one
    a = cases.box_case(20, 18, 24, (2.0, 1.0, 1.0), 20.0, False)
    b = cases.box_case(20, 18, 24, (2.0, 1.0, 1.0), 20.0, True)
    assert np.array_equal(a.lower, b.lower) and np.array_equal(a.magSf, b.magSf)
    return a, b


def _solve(A, c, ctl):
    x = dev(np.zeros(c.n_cells))
    perf, hist, coarse = A.solve(dev(c.source), x, ctl, history_cap=1000, coarsest_cap=4096)
    return perf, hist, coarse, x.cpu().numpy()


@pytest.mark.parametrize("smoother", ["GaussSeidel", "symGaussSeidel", "DIC", "DICGaussSeidel"])
def test_set_coeffs_matches_fresh_matrix_serial(b2g, oracle, pair_of_systems, smoother):
    a, b = pair_of_systems
    mesh = b2g.Mesh(a.lower, a.upper, a.Sf, a.magSf, a.n_cells, 10, True)
    ctl = b2g.controls_default(reduction="serial", smoother=smoother)
    A = b2g.Matrix(mesh, dev(a.diag), dev(a.coef))
    first = _solve(A, a, ctl)
    A.set_coeffs(dev(b.diag), dev(b.coef))
    upd = _solve(A, b, ctl)
    fresh = _solve(b2g.Matrix(mesh, dev(b.diag), dev(b.coef)), b, ctl)
    assert tuple(upd[0]) == tuple(fresh[0])
    assert upd[1] == fresh[1] and upd[2] == fresh[2]
    assert np.array_equal(upd[3], fresh[3])
    # and back: the first coefficients again give the first solve bit for bit
    A.set_coeffs(a.diag, a.coef)  # host arrays
    again = _solve(A, a, ctl)
    assert tuple(again[0]) == tuple(first[0]) and np.array_equal(again[3], first[3])
    # the single-phase system against the oracle
    agg = oracle.agglomerate(a.lower, a.upper, a.Sf, a.magSf, a.n_cells, 10, True)
    from oracle.bindings import controls as oc_controls
    want = oracle.pcg_gamg_solve(agg, a.diag, a.coef, a.source, np.zeros(a.n_cells), 1e-6, 0.0,
                                 ctl=oc_controls(smoother=smoother))
    assert tuple(first[0]) == want["perf"]
    assert np.array_equal(first[3], want["psi"])


@pytest.mark.parametrize("precision", ["fp32_precond", "fp32_precond_multicolour"])
def test_set_coeffs_precision_forms(b2g, pair_of_systems, precision):
    a, b = pair_of_systems
    mesh = b2g.Mesh(a.lower, a.upper, a.Sf, a.magSf, a.n_cells, 10, True)
    ctl = b2g.controls_default(precision=precision)
    A = b2g.Matrix(mesh, dev(a.diag), dev(a.coef))
    _solve(A, a, ctl)
    A.set_coeffs(dev(b.diag), dev(b.coef))
    upd = _solve(A, b, ctl)
    fresh = _solve(b2g.Matrix(mesh, dev(b.diag), dev(b.coef)), b, ctl)
    assert tuple(upd[0]) == tuple(fresh[0])
    assert np.array_equal(upd[3], fresh[3])


def test_pcg_gamg_solve_reuses_the_mesh_matrix(b2g, pair_of_systems):
    a, b = pair_of_systems
    mesh = b2g.Mesh(a.lower, a.upper, a.Sf, a.magSf, a.n_cells, 10, True)
    ctl = b2g.controls_default()
    out = []
    for c in (a, b, a):
        x = np.zeros(c.n_cells)
        perf, hist, _ = b2g.pcg_gamg_solve(mesh, c.diag, c.coef, c.source, x, ctl)
        out.append((tuple(perf), hist, x))
    for c, (perf, hist, x) in zip((a, b), out[:2]):
        want = _solve(b2g.Matrix(mesh, dev(c.diag), dev(c.coef)), c, ctl)
        assert perf == tuple(want[0]) and hist == want[1]
        assert np.array_equal(x, want[3])
    assert out[2][0] == out[0][0] and np.array_equal(out[2][2], out[0][2])


def test_level_timings_profile(b2g):
    c = cases.box_case(40, 40, 40)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    ctl = b2g.controls_default(tolerance=1e-6, relTol=0.0)
    b2g.set_profiling(True)
    try:
        perf = _solve(A, c, ctl)[0]
        ms4, cnt4 = A.timings()
        amul = A.level_timings(0)
        smooth = A.level_timings(1)
        fused = A.level_timings(2)
    finally:
        b2g.set_profiling(False)
    n_levels = mesh.n_levels
    vcycles = 2 * perf.nIterations
    # finest level: two sweeps per V-cycle; coarse level l (1 .. coarsest-1) min(2 + (l - 1), 4)
    assert smooth[0][2] == 2 * vcycles and smooth[0][1] == vcycles
    for lv in range(1, n_levels):
        assert smooth[lv][2] == min(2 + lv - 1, 4) * vcycles, lv
    assert all(ms > 0 for ms, _, _ in smooth[:n_levels])
    # finest Amuls: the initial residual and one per iteration; fused with another step, the residual
    # between the two V-cycles and the correction scaling's of every V-cycle
    assert amul[0][2] == 1 + perf.nIterations
    assert fused[0][2] == perf.nIterations + vcycles
    assert cnt4[1] == smooth[0][2] and abs(ms4[1] - smooth[0][0]) < 1e-9
    assert ms4[3] > sum(ms for ms, _, _ in smooth) > 0


def test_bounded_wait_gives_up(b2g, oracle):
    # a level swept by several parts; no part publishes its progress, so a part that needs another's
    # values waits for a word nothing sets and gives up after a short limit: the call reports a device
    # time-out and the context stays usable
    c = cases.box_case(40, 40, 40)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    x0 = np.sin(np.arange(c.n_cells) * 0.37)
    x = dev(x0)
    status, parts = A.smooth_stall(0, x, dev(c.source), 1 << 14)
    assert parts > 1
    assert status == "DEVICE_TIMEOUT"
    # the next sweep on the same matrix runs normally and is bit for bit the oracle's
    x = dev(x0)
    A.smooth(0, x, dev(c.source), 2)
    want = oracle.smooth(c.lower, c.upper, c.diag, c.coef, x0, c.source, 2)
    assert np.array_equal(x.cpu().numpy(), want)
