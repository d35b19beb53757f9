"""The pipelined multi-sweep Gauss-Seidel launch (pipe_kernels.cuh) against the oracle, bit for bit.

nSweeps sequential sweeps (gaussSeidelSweeps, src/OpenFOAM/matrices/smooth_solver_cpp.cu:87-166, once
per sweep) run as ONE launch in which sweep s+1 starts on a cell as soon as every value its row reads
is final. Every shape (one CTA; clusters of 2, 4, 8, 16 CTAs holding psi in distributed shared memory;
the grid form, psi in global memory and each CTA waiting for its neighbour ranks) must give the
oracle's sweeps exactly, on every level, and whole solves must not change when the launch is switched
on or off.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from brae_b200 import cases  # noqa: E402
from oracle.bindings import controls as oc_controls  # noqa: E402


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


def _level_system(mesh, A, c, lv):
    if lv == 0:
        lo, up = c.lower, c.upper
    else:
        st = mesh.step(lv - 1)
        lo, up = st["lower"], st["upper"]
    d, u = A.level(lv)
    return lo, up, d, u


@pytest.mark.parametrize("name,kw", BOXES, ids=[b[0] for b in BOXES])
def test_forced_shapes_bitexact(b2g, oracle, name, kw):
    c = cases.box_case(**kw)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    rng = np.random.default_rng(5)
    ran = 0
    for lv in range(mesh.n_levels + 1):
        lo, up, d, u = _level_system(mesh, A, c, lv)
        n = d.shape[0]
        x0 = rng.uniform(-1.0, 1.0, n)
        b = rng.uniform(-1.0, 1.0, n)
        for sweeps in (1, 2, 4):
            want = oracle.smooth(lo, up, d, u, x0, b, sweeps)
            for ranks in (1, 2, 4, 8, 16, -1, 24, 64):
                x = dev(x0)
                try:
                    A.smooth_pipelined(lv, x, dev(b), sweeps, ranks)
                except b2g.GamgError as e:
                    assert e.status == "ARGUMENT"
                    continue
                assert np.array_equal(x.cpu().numpy(), want), (lv, sweeps, ranks)
                ran += 1
    assert ran > 0


@pytest.mark.parametrize("name,kw", BOXES[:2], ids=[b[0] for b in BOXES[:2]])
def test_level_smooth_tuned_bitexact(b2g, oracle, name, kw):
    # the smoothing calls the V-cycle makes (tuned shape per level) against the oracle's sweeps
    c = cases.box_case(**kw)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    rng = np.random.default_rng(7)
    for lv in range(mesh.n_levels + 1):
        lo, up, d, u = _level_system(mesh, A, c, lv)
        x0 = rng.uniform(-1.0, 1.0, d.shape[0])
        b = rng.uniform(-1.0, 1.0, d.shape[0])
        for sweeps in (2, 3, 4):
            x = dev(x0)
            A.smooth(lv, x, dev(b), sweeps)
            assert np.array_equal(x.cpu().numpy(), oracle.smooth(lo, up, d, u, x0, b, sweeps)), (lv, sweeps)
        shape = mesh.pipe_shape(lv, 4)
        assert shape["ms_sweep_by_sweep"] > 0 or d.shape[0] == 0


@pytest.mark.parametrize("smoother", ["GaussSeidel", "DICGaussSeidel"])
@pytest.mark.parametrize("precision", ["fp64", "fp32_precond"])
def test_solve_same_with_and_without_pipeline(b2g, oracle, smoother, precision):
    c = cases.box_case(40, 40, 40)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    reduction = "serial" if precision == "fp64" else "tree"
    ctl = b2g.controls_default(smoother=smoother, precision=precision, reduction=reduction)
    out = {}
    try:
        for on in (False, True):
            b2g.set_sweep_pipeline(on)
            A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
            x = dev(np.zeros(c.n_cells))
            perf, hist, coarse = A.solve(dev(c.source), x, ctl, history_cap=1000, coarsest_cap=4096)
            out[on] = (tuple(perf), hist, coarse, x.cpu().numpy())
    finally:
        b2g.set_sweep_pipeline(True)
    assert out[True][0] == out[False][0]
    assert out[True][1] == out[False][1] and out[True][2] == out[False][2]
    assert np.array_equal(out[True][3], out[False][3])
    if precision == "fp64":
        agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
        want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), 1e-6, 0.0,
                                     ctl=oc_controls(smoother=smoother))
        assert out[True][0] == want["perf"]
        assert np.array_equal(out[True][3], want["psi"])
    # the tuner timed a pipelined shape on the smoothed levels
    timed = [mesh.pipe_shape(lv, s, 8 if precision == "fp64" else 4)["ms_pipelined"]
             for lv in range(mesh.n_levels) for s in (2, 3, 4)]
    assert any(t > 0 for t in timed)


def test_item_schedule_many_parts(b2g, oracle):
    # the multi-part sweep over (sweep, cell) items on levels cut into many parts, which wait for
    # parts after them as well as before: bit for bit the oracle's sequential sweeps
    c = cases.box_case(64, 64, 64, (2.0, 1.0, 1.0), 20.0)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    rng = np.random.default_rng(11)
    ran = 0
    for lv in (0, 1, 2):
        lo, up, d, u = _level_system(mesh, A, c, lv)
        x0 = rng.uniform(-1.0, 1.0, d.shape[0])
        b = rng.uniform(-1.0, 1.0, d.shape[0])
        for sweeps in (2, 4):
            x = dev(x0)
            try:
                A.smooth_pipelined(lv, x, dev(b), sweeps, -1)
            except b2g.GamgError as e:
                assert e.status == "ARGUMENT"
                continue
            assert np.array_equal(x.cpu().numpy(), oracle.smooth(lo, up, d, u, x0, b, sweeps)), (lv, sweeps)
            ran += 1
    assert ran >= 4


def test_grid_form_many_ranks(b2g, oracle):
    # the grid form on the levels of a box cut into many ranks: one per SM and fewer, every sweep count
    c = cases.box_case(64, 64, 64, (2.0, 1.0, 1.0), 20.0)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    rng = np.random.default_rng(13)
    ran = 0
    for lv in (0, 1, 2, 4):
        lo, up, d, u = _level_system(mesh, A, c, lv)
        x0 = rng.uniform(-1.0, 1.0, d.shape[0])
        b = rng.uniform(-1.0, 1.0, d.shape[0])
        for sweeps in (1, 2, 4):
            want = oracle.smooth(lo, up, d, u, x0, b, sweeps)
            for ranks in (sms, sms // 2, 17):
                x = dev(x0)
                A.smooth_pipelined(lv, x, dev(b), sweeps, ranks)
                assert np.array_equal(x.cpu().numpy(), want), (lv, sweeps, ranks)
                ran += 1
    assert ran == 4 * 3 * 3


def test_grid_form_wait_gives_up(b2g, oracle):
    # the grid form with no rank publishing its progress: every rank's wait for its neighbours runs
    # out after a short limit, the kernel ends and the call reports a device time-out; the context
    # stays usable and the next call on the same matrix is bit for bit the oracle's
    c = cases.box_case(64, 64, 64, (2.0, 1.0, 1.0), 20.0)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, dev(c.diag), dev(c.coef))
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    rng = np.random.default_rng(17)
    lo, up, d, u = _level_system(mesh, A, c, 1)
    x0 = rng.uniform(-1.0, 1.0, d.shape[0])
    b = rng.uniform(-1.0, 1.0, d.shape[0])
    assert A.grid_stall(1, dev(x0), dev(b), 2, sms, 1 << 14) == "DEVICE_TIMEOUT"
    x = dev(x0)
    A.smooth_pipelined(1, x, dev(b), 2, sms)
    assert np.array_equal(x.cpu().numpy(), oracle.smooth(lo, up, d, u, x0, b, 2))
