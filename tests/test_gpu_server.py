"""The serving form (b2g_server_*): each result is the same alone and in the mix, and admission by
HBM footprint evicts idle cases least recently used first, or refuses.

A solve in the mix is the same batched solve as a solve alone (a case's reductions are its own, in
a fixed order, whatever group it is solved in), so the bar is bit-for-bit identity between the two,
for both forms (plain FP64 and the FP32 V-cycle) and both reduction orders; the serial-order FP64
results are also checked bit for bit against the oracle's pcgGamgSolve.
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


MIX = [
    dict(nx=14, ny=12, nz=12, lengths=(2.0, 1.0, 1.0), grading_y=5.0, seed=3),
    dict(nx=30, ny=24, nz=20, lengths=(2.0, 1.0, 1.0), grading_y=20.0, seed=4),
    dict(nx=20, ny=18, nz=24, lengths=(2.0, 1.0, 1.0), grading_y=20.0, two_phase=True, seed=5),
    dict(nx=40, ny=40, nz=40, seed=6),
    dict(nx=10, ny=9, nz=8, seed=7),
    dict(nx=48, ny=30, nz=30, lengths=(2.0, 1.0, 1.0), grading_y=12.0, seed=8),
]


def _add(srv, c):
    return srv.add_case(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, c.diag, c.coef)


@pytest.mark.parametrize("precision", ["fp64", "fp32_precond", "fp32_precond_multicolour"])
@pytest.mark.parametrize("reduction", ["serial", "tree"])
def test_same_alone_and_in_the_mix(b2g, oracle, precision, reduction):
    built = [cases.box_case(**kw) for kw in MIX]
    ctl = b2g.controls_default(tolerance=1e-8, relTol=0.0, precision=precision, reduction=reduction)
    srv = b2g.Server(64 << 30, slots=4)
    try:
        ids = [_add(srv, c) for c in built]
        alone = []
        for i, c in enumerate(built):
            psi, perf, lat = srv.wait(srv.submit(ids[i], c.source, ctl))
            assert lat > 0.0 and perf.nIterations > 0
            alone.append((psi.copy(), tuple(perf)))
        # every case three times at once: solves of different cases overlap on the device, solves
        # of one case queue behind each other
        tickets = [(i, srv.submit(ids[i], built[i].source, ctl)) for _ in range(3) for i in range(len(built))]
        for i, t in tickets:
            psi, perf, _ = srv.wait(t)
            assert tuple(perf) == alone[i][1]
            assert np.array_equal(psi, alone[i][0])
    finally:
        srv.close()
    if precision == "fp64" and reduction == "serial":
        for c, (psi, perf) in zip(built, alone):
            agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
            want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), 1e-8, 0.0)
            assert perf == want["perf"]
            assert np.array_equal(psi, want["psi"])


def test_initial_guess_and_standalone_gamg(b2g):
    c = cases.box_case(nx=20, ny=16, nz=14, lengths=(2.0, 1.0, 1.0), grading_y=8.0, seed=9)
    srv = b2g.Server(16 << 30, slots=2)
    try:
        cid = _add(srv, c)
        psi0 = np.linspace(-1.0, 1.0, c.n_cells)
        for solver in ("PCG", "GAMG"):
            ctl = b2g.controls_default(tolerance=1e-7, relTol=0.0, solver=solver)
            got, perf, _ = srv.wait(srv.submit(cid, c.source, ctl, psi0=psi0))
            mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells)
            want = psi0.copy()
            if solver == "PCG":  # served as a batch: the batched solve's result
                A = b2g.Matrix(mesh, c.diag, c.coef)
                wperf = b2g.Batch([A]).solve([c.source], [want], ctl)[0]
            else:                # served alone: the standalone solver's
                wperf = b2g.gamg_solve(mesh, c.diag, c.coef, c.source, want, ctl)[0]
            assert tuple(perf) == tuple(wperf)
            assert np.array_equal(got, want)
    finally:
        srv.close()


def test_admission_evicts_least_recently_used(b2g):
    small = [cases.box_case(nx=16, ny=14, nz=12, seed=s) for s in (11, 12, 13)]
    probe = b2g.Server(1 << 40, slots=1)
    try:
        cs = probe.case_bytes(_add(probe, small[0]))
    finally:
        probe.close()
    assert cs > 0
    ctl = b2g.controls_default(tolerance=1e-6, relTol=0.0)
    srv = b2g.Server(2 * cs + cs // 2, slots=2)
    try:
        a = _add(srv, small[0])
        b = _add(srv, small[1])
        srv.wait(srv.submit(a, small[0].source, ctl))  # a is now the more recently used
        c = _add(srv, small[2])                        # evicts b
        srv.wait(srv.submit(a, small[0].source, ctl))
        srv.wait(srv.submit(c, small[2].source, ctl))
        with pytest.raises(b2g.GamgError, match="evicted"):
            srv.submit(b, small[1].source, ctl)
    finally:
        srv.close()
    tight = b2g.Server(cs // 2, slots=1)
    try:
        with pytest.raises(b2g.GamgError, match="HBM cap"):
            _add(tight, small[0])
    finally:
        tight.close()


def test_wait_timeout_keeps_the_request(b2g):
    c = cases.box_case(nx=60, ny=40, nz=40, lengths=(2.0, 1.0, 1.0), grading_y=20.0, seed=14)
    srv = b2g.Server(32 << 30, slots=1)
    try:
        cid = _add(srv, c)
        ctl = b2g.controls_default(tolerance=1e-10, relTol=0.0)
        t = srv.submit(cid, c.source, ctl)
        try:
            psi, perf, _ = srv.wait(t, timeout_ms=0)
        except b2g.GamgError as e:
            assert "still pending" in str(e)
            psi, perf, _ = srv.wait(t)  # a pending request stays waitable
        assert perf.nIterations > 0 and np.isfinite(psi).all()
        with pytest.raises(b2g.GamgError, match="unknown"):
            srv.wait(t)  # collected already
    finally:
        srv.close()
