"""The coupled (cyclic) pair on the device, held to the oracle (oracle/gamg_oracle.c, itself pinned
bit for bit to the reference's gamgSolve with a coupled patch in tests/test_oracle_pair.py).

Bit for bit: every level's pair (faces keyed on the coarse cell pair, coefficients summed in fine
face order), Amul with the pair on every level, the four smoothers with the pair (Gauss-Seidel
through bPrime, DIC through the residual), and whole standalone GAMG solves with serial-order
reductions. With tree reductions: identical iteration counts, residuals within 1e-12 of the initial
residual, the field within 1e-10 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from brae_b200 import cases  # noqa: E402
from oracle.bindings import controls as oc_controls  # noqa: E402

SMOOTHERS = ("GaussSeidel", "symGaussSeidel", "DIC", "DICGaussSeidel")
BOXES = [
    ("tiny", dict(nx=8, ny=7, nz=6)),
    ("graded", dict(nx=12, ny=10, nz=9, grading_y=5.0)),
    ("two_phase", dict(nx=20, ny=18, nz=24, grading_y=20.0, two_phase=True)),
    # pairs along x and z: the edge cells own two pair faces on the finest level too
    ("two_axes", dict(nx=14, ny=12, nz=10, grading_y=5.0, axes=("x", "z"))),
]


@pytest.fixture(scope="module")
def b2g():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import brae_b200.native as n
    return n


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=torch.float64)


def host(t):
    return t.detach().cpu().numpy()


def _setup(b2g, oracle, kw):
    c, own, nbr, pc = cases.periodic_box(**kw)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    mesh.set_pair(own, nbr)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    return c, own, nbr, pc, mesh, agg


@pytest.mark.parametrize("name,kw", BOXES, ids=[b[0] for b in BOXES])
def test_pair_levels_and_kernels_bitexact(b2g, oracle, name, kw):
    c, own, nbr, pc, mesh, agg = _setup(b2g, oracle, kw)
    H = agg.hierarchy
    pairs = oracle.hierarchy_pairs(agg, c.diag, c.coef, own, nbr, pc)
    A = b2g.Matrix(mesh, c.diag, c.coef, pair_coeffs=pc)
    rng = np.random.default_rng(11)
    for lv in range(H.n_levels + 1):
        po, pn, pcv = pairs[lv]
        o, n = mesh.level_pair(lv)
        assert np.array_equal(o, po) and np.array_equal(n, pn), f"pair faces level {lv}"
        assert np.array_equal(A.pair_coeffs(lv), pcv), f"pair coefficients level {lv}"
        d, u = A.level(lv)
        lo, up = H.lower[lv], H.upper[lv]
        x = rng.standard_normal(H.n_cells[lv])
        y = torch.empty(H.n_cells[lv], dtype=torch.float64, device="cuda")
        A.amul(lv, dev(x), y)
        assert np.array_equal(host(y), oracle.amul_pair(lo, up, d, u, po, pn, pcv, x)), f"Amul level {lv}"
        b = rng.standard_normal(H.n_cells[lv])
        for sm in SMOOTHERS:
            for sweeps in (1, 2):
                psi = dev(x)
                A.smooth(lv, psi, dev(b), sweeps, smoother=sm)
                want = oracle.smooth_pair(lo, up, d, u, po, pn, pcv, x, b, sweeps, sm)
                assert np.array_equal(host(psi), want), f"{sm} level {lv} sweeps {sweeps}"


@pytest.mark.parametrize("name,kw", BOXES, ids=[b[0] for b in BOXES])
def test_pair_gamg_solve_serial_bitexact(b2g, oracle, name, kw):
    c, own, nbr, pc, mesh, agg = _setup(b2g, oracle, kw)
    for sm in SMOOTHERS:
        want = oracle.gamg_solve_pair(agg, c.diag, c.coef, own, nbr, pc, c.source, np.zeros(c.n_cells),
                                      oc_controls(smoother=sm, tolerance=1e-8, relTol=0.0))
        ctl = b2g.controls_default(solver="GAMG", smoother=sm, tolerance=1e-8, relTol=0.0, reduction="serial")
        psi = np.zeros(c.n_cells)
        perf, hist = b2g.gamg_solve_coupled(mesh, c.diag, c.coef, pc, c.source, psi, ctl)
        assert tuple(perf) == want["perf"], sm
        assert np.array_equal(psi, want["psi"]), sm
        assert np.array_equal(np.array(hist), want["history"]), sm


@pytest.mark.parametrize("name,kw", BOXES[1:], ids=[b[0] for b in BOXES[1:]])
def test_pair_gamg_solve_tree(b2g, oracle, name, kw):
    c, own, nbr, pc, mesh, agg = _setup(b2g, oracle, kw)
    A = b2g.Matrix(mesh, c.diag, c.coef, pair_coeffs=pc)
    for sm in ("GaussSeidel", "DIC"):
        want = oracle.gamg_solve_pair(agg, c.diag, c.coef, own, nbr, pc, c.source, np.zeros(c.n_cells),
                                      oc_controls(smoother=sm, tolerance=1e-8, relTol=0.0))
        ctl = b2g.controls_default(solver="GAMG", smoother=sm, tolerance=1e-8, relTol=0.0)
        for _ in range(2):  # the second solve replays the captured iteration graph
            psi = dev(np.zeros(c.n_cells))
            perf, hist = A.gamg_solve(dev(c.source), psi, ctl)
            assert perf.nIterations == want["perf"][2], sm
            init = want["perf"][0]
            assert abs(perf.initialResidual - init) <= 1e-12 * init
            assert np.abs(np.array(hist) - want["history"]).max() <= 1e-12 * init
            err = np.abs(host(psi) - want["psi"]).max() / np.abs(want["psi"]).max()
            assert err < 1e-10, sm


def test_pair_refusals(b2g, oracle):
    c, own, nbr, pc, mesh, agg = _setup(b2g, oracle, BOXES[0][1])
    with pytest.raises(b2g.GamgError, match="already carries"):
        mesh.set_pair(own, nbr)
    A = b2g.Matrix(mesh, c.diag, c.coef, pair_coeffs=pc)
    # the reference's pcgGamgSolve refuses coupled patches (gamg_solver_cpp.cu:1045)
    with pytest.raises(b2g.GamgError, match="refuses coupled patches"):
        A.solve(dev(c.source), dev(np.zeros(c.n_cells)), b2g.controls_default())
    with pytest.raises(b2g.GamgError, match="FP64 form only"):
        A.gamg_solve(dev(c.source), dev(np.zeros(c.n_cells)),
                     b2g.controls_default(solver="GAMG", precision="fp32_precond"))
    with pytest.raises(b2g.GamgError, match="coupled pair"):
        b2g.Batch([A])
    # an uncoupled matrix on the same mesh solves without the pair, as before
    B = b2g.Matrix(mesh, c.diag, c.coef)
    want = oracle.gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells),
                             oc_controls(tolerance=1e-8, relTol=0.0))
    psi = np.zeros(c.n_cells)
    perf, _ = B.gamg_solve(c.source, psi, b2g.controls_default(solver="GAMG", tolerance=1e-8, relTol=0.0,
                                                                 reduction="serial"))
    assert tuple(perf) == want["perf"] and np.array_equal(psi, want["psi"])
    # a face naming a cell outside the mesh
    other = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    bad = own.copy()
    bad[3] = c.n_cells
    with pytest.raises(b2g.GamgError, match="outside the mesh"):
        other.set_pair(bad, nbr)
