"""The batched form (b2g_batch_*): many independent cases solved together, every level step one
launch over all cases that have the level.

Each case's result must be the one its own solve gives: with serial-order reductions bit for bit the
oracle's pcgGamgSolve (psi and SolverPerformance), whatever the other cases in the batch; with tree
reductions the same iteration count, the initial residual within 1e-12 and the field within 1e-10 of
the oracle, and bit for bit the same whether the case is alone in a batch or among others. The FP32
V-cycle form is checked against the FP64 oracle at equal tolerance.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from brae_b200 import cases  # noqa: E402
from oracle.bindings import controls as oc_controls  # noqa: E402

HIST_RTOL = 1e-12
FIELD_RTOL = 1e-10


@pytest.fixture(scope="module")
def b2g():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import brae_b200.native as n
    return n


# uneven sizes, gradings and level counts (the smallest has two coarse levels)
BOXES = [
    dict(nx=6, ny=5, nz=4, seed=21),
    dict(nx=14, ny=12, nz=12, lengths=(2.0, 1.0, 1.0), grading_y=5.0, seed=22),
    dict(nx=30, ny=24, nz=20, lengths=(2.0, 1.0, 1.0), grading_y=20.0, seed=23),
    dict(nx=20, ny=18, nz=24, lengths=(2.0, 1.0, 1.0), grading_y=20.0, two_phase=True, seed=24),
    dict(nx=40, ny=40, nz=40, seed=25),
    dict(nx=9, ny=30, nz=11, lengths=(1.0, 3.0, 1.0), grading_y=3.0, seed=26),
]


def _build(b2g, kws):
    built = [cases.box_case(**kw) for kw in kws]
    meshes = [b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True) for c in built]
    mats = [b2g.Matrix(m, c.diag, c.coef) for m, c in zip(meshes, built)]
    return built, meshes, mats


def _oracle(oracle, c, tol, rel, ctl_kw, psi0=None):
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    x0 = np.zeros(c.n_cells) if psi0 is None else psi0
    return oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, x0, tol, rel, ctl=oc_controls(**ctl_kw))


@pytest.mark.parametrize("ctl_kw", [dict(), dict(nPreSweeps=2, nVcycles=3), dict(scaleCorrection=False),
                                    dict(nFinestSweeps=3, nPostSweeps=1, maxPostSweeps=3)],
                         ids=["defaults", "presweeps", "noscale", "sweeps"])
def test_batch_serial_bitexact(b2g, oracle, ctl_kw):
    built, meshes, mats = _build(b2g, BOXES)
    batch = b2g.Batch(mats)
    tol, rel = 1e-8, 0.0
    ctl = b2g.controls_default(tolerance=tol, relTol=rel, reduction="serial", **ctl_kw)
    psis = [np.zeros(c.n_cells) for c in built]
    perfs = batch.solve([c.source for c in built], psis, ctl)
    its = set()
    for c, psi, perf in zip(built, psis, perfs):
        want = _oracle(oracle, c, tol, rel, ctl_kw)
        assert tuple(perf) == want["perf"]
        assert np.array_equal(psi, want["psi"])
        its.add(perf.nIterations)
    assert len(its) > 1  # the cases converge at different iterations
    assert batch.launches() > 0


def test_batch_destroyed_before_its_meshes(b2g, oracle):
    # a batch builds level-held layouts of its meshes on its stream; the meshes outlive the batch and
    # free them later, and a second batch on the same meshes reuses what the first built
    import gc
    built, meshes, mats = _build(b2g, BOXES[:3])
    ctl = b2g.controls_default(tolerance=1e-8, relTol=0.0, reduction="serial")
    for _ in range(2):
        batch = b2g.Batch(mats)
        psis = [np.zeros(c.n_cells) for c in built]
        perfs = batch.solve([c.source for c in built], psis, ctl)
        del batch
        gc.collect()
        for c, psi, perf in zip(built, psis, perfs):
            want = _oracle(oracle, c, 1e-8, 0.0, {})
            assert tuple(perf) == want["perf"] and np.array_equal(psi, want["psi"])
    del mats
    gc.collect()
    del meshes
    gc.collect()
    torch.cuda.synchronize()


def test_batch_tree_parity_and_alone(b2g, oracle):
    built, meshes, mats = _build(b2g, BOXES)
    tol, rel = 1e-8, 0.0
    ctl = b2g.controls_default(tolerance=tol, relTol=rel)
    batch = b2g.Batch(mats)
    psis = [np.zeros(c.n_cells) for c in built]
    perfs = batch.solve([c.source for c in built], psis, ctl)
    for c, psi, perf in zip(built, psis, perfs):
        want = _oracle(oracle, c, tol, rel, {})
        wi, wf, wn = want["perf"]
        assert perf.nIterations == wn
        assert abs(perf.initialResidual - wi) <= HIST_RTOL * abs(wi)
        assert np.abs(psi - want["psi"]).max() <= FIELD_RTOL * np.abs(want["psi"]).max()
    # each case alone in a batch of one: the same bits
    for k in (0, 2, 4):
        alone = b2g.Batch([mats[k]])
        x = np.zeros(built[k].n_cells)
        p = alone.solve([built[k].source], [x], ctl)[0]
        assert tuple(p) == tuple(perfs[k])
        assert np.array_equal(x, psis[k])
    # a second solve on the same batch (graph replayed) from a nonzero guess
    psi0 = [np.linspace(-1.0, 1.0, c.n_cells) for c in built]
    psis2 = [p.copy() for p in psi0]
    perfs2 = batch.solve([c.source for c in built], psis2, ctl)
    for c, x0, psi, perf in zip(built, psi0, psis2, perfs2):
        want = _oracle(oracle, c, tol, rel, {}, psi0=x0)
        assert perf.nIterations == want["perf"][2]
        assert np.abs(psi - want["psi"]).max() <= FIELD_RTOL * np.abs(want["psi"]).max()


def test_batch_fp32_form(b2g, oracle):
    built, meshes, mats = _build(b2g, BOXES)
    tol = 1e-9
    ctl = b2g.controls_default(tolerance=tol, relTol=0.0, precision="fp32_precond")
    batch = b2g.Batch(mats)
    psis = [np.zeros(c.n_cells) for c in built]
    perfs = batch.solve([c.source for c in built], psis, ctl)
    for c, m, psi, perf in zip(built, meshes, psis, perfs):
        assert perf.finalResidual < tol
        want = _oracle(oracle, c, tol, 0.0, {})
        assert np.abs(psi - want["psi"]).max() / np.abs(want["psi"]).max() < 1e-6
        # the single-case FP32 form reaches the same iteration count
        x = np.zeros(c.n_cells)
        single = b2g.pcg_gamg_solve(m, c.diag, c.coef, c.source, x, ctl)[0]
        assert abs(single.nIterations - perf.nIterations) <= 1


def test_batch_fp32_multicolour_form(b2g, oracle):
    built, meshes, mats = _build(b2g, BOXES)
    tol = 1e-9
    ctl = b2g.controls_default(tolerance=tol, relTol=0.0, precision="fp32_precond_multicolour")
    batch = b2g.Batch(mats)
    for _ in range(2):  # the second solve runs on the prepared layouts and the captured graph
        psis = [np.zeros(c.n_cells) for c in built]
        perfs = batch.solve([c.source for c in built], psis, ctl)
        for c, m, psi, perf in zip(built, meshes, psis, perfs):
            assert perf.finalResidual < tol
            want = _oracle(oracle, c, tol, 0.0, {})
            assert 1 <= perf.nIterations <= want["perf"][2] + 2
            assert np.abs(psi - want["psi"]).max() / np.abs(want["psi"]).max() < 1e-6
    # the same sweeps as the single solve's multicolour form: the same iteration counts (+-1)
    for c, m, perf in zip(built, meshes, perfs):
        x = np.zeros(c.n_cells)
        single = b2g.pcg_gamg_solve(m, c.diag, c.coef, c.source, x, ctl)[0]
        assert abs(single.nIterations - perf.nIterations) <= 1


def test_batch_device_fields_and_refusals(b2g, oracle):
    built, meshes, mats = _build(b2g, BOXES[:3])
    batch = b2g.Batch(mats)
    ctl = b2g.controls_default(tolerance=1e-7, relTol=0.0, reduction="serial")
    src = [torch.as_tensor(c.source).cuda() for c in built]
    psis = [torch.zeros(c.n_cells, dtype=torch.float64, device="cuda") for c in built]
    perfs = batch.solve(src, psis, ctl)
    for c, psi, perf in zip(built, psis, perfs):
        want = _oracle(oracle, c, 1e-7, 0.0, {})
        assert tuple(perf) == want["perf"]
        assert np.array_equal(psi.cpu().numpy(), want["psi"])
    with pytest.raises(b2g.GamgError, match="GaussSeidel only"):
        batch.solve([c.source for c in built], [np.zeros(c.n_cells) for c in built],
                    b2g.controls_default(smoother="DIC"))
    with pytest.raises(b2g.GamgError, match="batched solve is PCG"):
        batch.solve([c.source for c in built], [np.zeros(c.n_cells) for c in built],
                    b2g.controls_default(solver="GAMG"))
    with pytest.raises(b2g.GamgError, match="appears twice"):
        b2g.Batch([mats[0], mats[1], mats[0]])


def test_batch_part_rule(b2g, oracle):
    # meshes built with the batch's part rule (fewer parts per level): the same bits as the oracle
    b2g.set_part_cells(128)
    try:
        built, meshes, mats = _build(b2g, BOXES[2:5])
    finally:
        b2g.set_part_cells(48)
    batch = b2g.Batch(mats)
    ctl = b2g.controls_default(tolerance=1e-8, relTol=0.0, reduction="serial")
    psis = [np.zeros(c.n_cells) for c in built]
    perfs = batch.solve([c.source for c in built], psis, ctl)
    for c, psi, perf in zip(built, psis, perfs):
        want = _oracle(oracle, c, 1e-8, 0.0, {})
        assert tuple(perf) == want["perf"] and np.array_equal(psi, want["psi"])
    with pytest.raises(b2g.GamgError):
        b2g.set_part_cells(0)
