"""The FP32-preconditioned forms' direct coarsest solve: a dense FP64 Cholesky factor of the coarsest
level made once per coarse matrix, applied by two triangular substitutions in every V-cycle (the
reference's precision form solves its coarsest level directly, device_amg_coarse.cu:545-700; the FP64
parity form keeps the reference's PCG-DIC)."""
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


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


BOXES = [
    ("graded20", dict(nx=24, ny=20, nz=22, lengths=(2.0, 1.0, 1.0), grading_y=20.0)),
    ("two_phase", dict(nx=20, ny=18, nz=24, lengths=(2.0, 1.0, 1.0), grading_y=20.0, two_phase=True)),
    ("cube40", dict(nx=40, ny=40, nz=40)),
]


@pytest.mark.parametrize("name,kw", BOXES, ids=[b[0] for b in BOXES])
def test_dense_solve_matches_numpy(b2g, name, kw):
    c = cases.box_case(**kw)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    lv = mesh.n_levels
    st = mesh.step(lv - 1)
    d, u = A.level(lv)
    n = d.shape[0]
    M = np.diag(d)
    M[st["lower"], st["upper"]] = u
    M[st["upper"], st["lower"]] = u
    b = np.random.default_rng(3).uniform(-1.0, 1.0, n)
    x = dev(np.zeros(n))
    A.coarsest_dense_solve(x, dev(b))
    want = np.linalg.solve(M, b)
    assert np.abs(x.cpu().numpy() - want).max() <= 1e-11 * np.abs(want).max()


@pytest.mark.parametrize("precision", ["fp32_precond", "fp32_precond_multicolour"])
def test_fp32_forms_with_direct_coarsest(b2g, oracle, precision):
    c = cases.box_case(40, 40, 40, (2.0, 1.0, 1.0), 20.0, True)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), 1e-9, 0.0)
    scale = np.abs(want["psi"]).max()
    its = {}
    for direct in (1, 0):
        A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
        ctl = b2g.controls_default(precision=precision, coarsestDirect=direct, tolerance=1e-9)
        x = dev(np.zeros(c.n_cells))
        perf, hist, _ = A.solve(dev(c.source), x, ctl)
        assert perf.finalResidual < 1e-9
        assert np.abs(x.cpu().numpy() - want["psi"]).max() <= 1e-6 * scale
        its[direct] = perf.nIterations
    # an exact coarsest solve is no worse a preconditioner than the iterative one
    assert its[1] <= its[0] + 1


def test_batch_fp32_direct_coarsest_same_as_single(b2g):
    dims = [(16, 14, 12), (20, 10, 9), (12, 12, 30)]
    mats, srcs, cs = [], [], []
    for k, n in enumerate(dims):
        c = cases.box_case(*n, (2.0, 1.0, 1.0), 5.0 + k, False, k)
        mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
        mats.append(b2g.Matrix(mesh, dev(c.diag), dev(c.coef)))
        srcs.append(dev(c.source))
        cs.append(c)
    batch = b2g.Batch(mats)
    tol = 1e-9
    ctl = b2g.controls_default(precision="fp32_precond", coarsestDirect=1, tolerance=tol)
    psis = [dev(np.zeros(c.n_cells)) for c in cs]
    perfs = batch.solve(srcs, psis, ctl)
    for k, c in enumerate(cs):
        x = dev(np.zeros(c.n_cells))
        p1 = mats[k].solve(srcs[k], x, ctl)[0]
        assert perfs[k].finalResidual < tol and p1.finalResidual < tol
        # the batch's tile reductions are not the single solve's: the same iterations to one, the
        # same field to the FP32 form's accuracy
        assert abs(perfs[k].nIterations - p1.nIterations) <= 1
        assert np.abs(psis[k].cpu().numpy() - x.cpu().numpy()).max() <= 1e-6 * np.abs(x.cpu().numpy()).max()
