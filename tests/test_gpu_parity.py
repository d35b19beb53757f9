"""Parity of the CUDA path with the oracle (oracle/gamg_oracle.c), through the C ABI.

Bit-for-bit: the agglomeration (every map), the Galerkin coarse matrices, Amul, the Gauss-Seidel
sweeps, restriction/prolongation and the coarsest-level PCG-DIC; and, with serial-order
reductions (B2G_REDUCTION_SERIAL), whole solves: psi, every residual and every coarsest-level log.
With the default tree reductions the sums differ from the reference's serial sums in the last bit,
which the PCG recurrence r -= alpha*w amplifies by r0/rk, so the bar there is: identical iteration
counts (solve and every coarsest level), residual history within 1e-12 of the initial residual, and
the field within 1e-10 relative.
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


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def host(t):
    return t.detach().cpu().numpy()


BOXES = [
    ("tiny", dict(nx=8, ny=7, nz=6, lengths=(2.0, 1.0, 1.0))),
    ("graded", dict(nx=12, ny=10, nz=9, lengths=(2.0, 1.0, 1.0), grading_y=5.0)),
    ("graded20", dict(nx=24, ny=20, nz=22, lengths=(2.0, 1.0, 1.0), grading_y=20.0)),
    ("two_phase", dict(nx=20, ny=18, nz=24, lengths=(2.0, 1.0, 1.0), grading_y=20.0, two_phase=True)),
    ("cube40", dict(nx=40, ny=40, nz=40)),
]


def _pair(b2g, oracle, c, forward=True, n_coarsest=10):
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, n_coarsest, forward)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, n_coarsest, forward)
    return mesh, agg


@pytest.mark.parametrize("name,kw", BOXES, ids=[b[0] for b in BOXES])
@pytest.mark.parametrize("forward", [True, False])
def test_hierarchy_bitexact(b2g, oracle, name, kw, forward):
    c = cases.box_case(**kw)
    mesh, agg = _pair(b2g, oracle, c, forward)
    H = agg.hierarchy
    assert mesh.n_levels == H.n_levels
    assert mesh.forward == H.forward
    for lv in range(H.n_levels + 1):
        assert mesh.level_size(lv) == (H.n_cells[lv], H.n_faces[lv])
    for s in range(H.n_levels):
        st = mesh.step(s)
        assert np.array_equal(st["restrict"], H.restrict[s]), s
        assert np.array_equal(st["face_restrict"], H.face_restrict[s]), s
        assert np.array_equal(st["flip"], H.flip[s]), s
        assert np.array_equal(st["lower"], H.lower[s + 1]), s
        assert np.array_equal(st["upper"], H.upper[s + 1]), s


def test_hierarchy_openfoam_case20(b2g, case20):
    c = case20
    mesh = b2g.Mesh(c["lower"], c["upper"], c["Sf"], c["magSf"], int(c["n_cells"]),
                    int(c["n_coarsest"]), True)
    assert mesh.n_levels == 2
    for i in range(2):
        assert np.array_equal(mesh.step(i)["restrict"], c[f"restrict_{i}"])


@pytest.mark.parametrize("name,kw", BOXES[1:], ids=[b[0] for b in BOXES[1:]])
def test_level_kernels_bitexact(b2g, oracle, name, kw):
    c = cases.box_case(**kw)
    mesh, agg = _pair(b2g, oracle, c)
    H = agg.hierarchy
    A = b2g.Matrix(mesh, c.diag, c.coef)
    ref = oracle.coarse_matrices(agg, c.diag, c.coef)
    rng = np.random.default_rng(7)
    for lv in range(H.n_levels + 1):
        d, u = A.level(lv)
        assert np.array_equal(d, ref[lv][0]), f"Galerkin diag level {lv}"
        assert np.array_equal(u, ref[lv][1]), f"Galerkin upper level {lv}"
        lo, up = H.lower[lv], H.upper[lv]
        n = H.n_cells[lv]
        x = rng.standard_normal(n)
        y = torch.empty(n, dtype=torch.float64, device="cuda")
        A.amul(lv, dev(x), y)
        assert np.array_equal(host(y), oracle.amul(lo, up, d, u, x)), f"Amul level {lv}"
        b = rng.standard_normal(n)
        for sweeps in (1, 2, 3):
            psi = dev(x)
            A.smooth(lv, psi, dev(b), sweeps)
            want = oracle.smooth(lo, up, d, u, x, b, sweeps, "GaussSeidel")
            assert np.array_equal(host(psi), want), f"GaussSeidel level {lv} sweeps {sweeps}"
        for sm in ("symGaussSeidel", "DIC", "DICGaussSeidel"):
            for sweeps in (1, 2):
                psi = dev(x)
                A.smooth(lv, psi, dev(b), sweeps, smoother=sm)
                want = oracle.smooth(lo, up, d, u, x, b, sweeps, sm)
                assert np.array_equal(host(psi), want), f"{sm} level {lv} sweeps {sweeps}"
        # scale: dots differ in summation order only
        f = dev(x)
        acf = torch.empty_like(f)
        A.scale(lv, f, acf, dev(b))
        wf, wacf = oracle.scale(lo, up, d, u, x, b)
        assert np.array_equal(host(acf), wacf)
        assert np.allclose(host(f), wf, rtol=1e-12, atol=1e-14 * np.abs(wf).max())
    for s in range(H.n_levels):
        nf, ncoarse = H.n_cells[s], H.n_cells[s + 1]
        ff = rng.standard_normal(nf)
        cf = torch.empty(ncoarse, dtype=torch.float64, device="cuda")
        A.restrict(s, dev(ff), cf)
        want = np.zeros(ncoarse)
        np.add.at(want, H.restrict[s], ff)  # ascending fine cells, as restrictField
        assert np.array_equal(host(cf), want), f"restrict step {s}"
        cc = rng.standard_normal(ncoarse)
        out = torch.empty(nf, dtype=torch.float64, device="cuda")
        A.prolong(s, dev(cc), out)
        assert np.array_equal(host(out), cc[H.restrict[s]]), f"prolong step {s}"


@pytest.mark.parametrize("name,kw", BOXES[1:], ids=[b[0] for b in BOXES[1:]])
def test_coarsest_pcg_dic_bitexact(b2g, oracle, name, kw):
    c = cases.box_case(**kw)
    mesh, agg = _pair(b2g, oracle, c)
    H = agg.hierarchy
    A = b2g.Matrix(mesh, c.diag, c.coef)
    ref = oracle.coarse_matrices(agg, c.diag, c.coef)
    lv = H.n_levels
    d, u = ref[lv]
    rng = np.random.default_rng(11)
    src = rng.standard_normal(H.n_cells[lv])
    psi = torch.zeros(H.n_cells[lv], dtype=torch.float64, device="cuda")
    perf = A.pcg_dic(lv, psi, dev(src), 1e-6, 0.0)
    x, p = oracle.pcg_dic(H.lower[lv], H.upper[lv], d, u, np.zeros(H.n_cells[lv]), src, 1e-6, 0.0)
    assert tuple(perf) == p
    assert np.array_equal(host(psi), x)


def _solve_parity(b2g, oracle, c, tol, rel_tol, ctl_kw=None, psi0=None, reduction="tree"):
    ctl_kw = ctl_kw or {}
    mesh, agg = _pair(b2g, oracle, c)
    psi0 = np.zeros(c.n_cells) if psi0 is None else psi0
    want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, psi0, tol, rel_tol,
                                 ctl=oc_controls(**ctl_kw))
    ctl = b2g.controls_default(tolerance=tol, relTol=rel_tol, reduction=reduction, **ctl_kw)
    psi = psi0.copy()
    perf, hist, coarse = b2g.pcg_gamg_solve(mesh, c.diag, c.coef, c.source, psi, ctl,
                                            coarsest_cap=4096)
    wi, wf, wn = want["perf"]
    if reduction == "serial":
        assert tuple(perf) == want["perf"]
        assert hist == list(want["history"])
        assert coarse == want["coarsest"]
        assert np.array_equal(psi, want["psi"])
        return perf
    assert perf.nIterations == wn
    assert [p[2] for p in coarse] == [p[2] for p in want["coarsest"]]
    assert abs(perf.initialResidual - wi) <= HIST_RTOL * abs(wi)
    assert np.abs(np.asarray(hist) - want["history"]).max() <= HIST_RTOL * wi
    scale = np.abs(want["psi"]).max()
    assert np.abs(psi - want["psi"]).max() <= FIELD_RTOL * scale
    return perf


@pytest.mark.parametrize("reduction", ["serial", "tree"])
@pytest.mark.parametrize("name,kw", BOXES, ids=[b[0] for b in BOXES])
def test_pcg_gamg_solve_parity(b2g, oracle, name, kw, reduction):
    c = cases.box_case(**kw)
    _solve_parity(b2g, oracle, c, 1e-6, 0.0, reduction=reduction)


@pytest.mark.parametrize("reduction", ["serial", "tree"])
def test_pcg_gamg_solve_parity_options(b2g, oracle, reduction):
    c = cases.box_case(16, 14, 12, (2.0, 1.0, 1.0), 8.0)
    _solve_parity(b2g, oracle, c, 1e-9, 0.0, dict(nPreSweeps=2, nVcycles=3), reduction=reduction)
    _solve_parity(b2g, oracle, c, 1e-7, 0.0, dict(nFinestSweeps=3, nPostSweeps=1, maxPostSweeps=3),
                  reduction=reduction)
    _solve_parity(b2g, oracle, c, 1e-6, 0.05, dict(scaleCorrection=False),
                  psi0=np.linspace(-1.0, 1.0, c.n_cells), reduction=reduction)


@pytest.mark.parametrize("reduction", ["serial", "tree"])
@pytest.mark.parametrize("name,kw", BOXES[1:4], ids=[b[0] for b in BOXES[1:4]])
@pytest.mark.parametrize("smoother", ["symGaussSeidel", "DIC", "DICGaussSeidel"])
def test_pcg_gamg_other_smoothers_parity(b2g, oracle, name, kw, reduction, smoother):
    # symGaussSeidel's backward walk and DIC's backward substitution run as forward sweeps of
    # reversed levels, DIC's forward substitution as one of a lower-only level
    c = cases.box_case(**kw)
    _solve_parity(b2g, oracle, c, 1e-8, 0.0, dict(smoother=smoother), reduction=reduction)
    _solve_parity(b2g, oracle, c, 1e-8, 0.0, dict(smoother=smoother, nPreSweeps=1), reduction=reduction)


@pytest.mark.parametrize("smoother", ["DIC", "DICGaussSeidel"])
def test_standalone_gamg_dic_parity(b2g, oracle, smoother):
    # interFoam's p_rghFinal default: solver GAMG; smoother DIC
    c = cases.box_case(16, 14, 12, (2.0, 1.0, 1.0), 8.0)
    mesh, agg = _pair(b2g, oracle, c)
    want = oracle.gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells),
                             oc_controls(tolerance=1e-8, relTol=0.0, smoother=smoother))
    psi = np.zeros(c.n_cells)
    ctl = b2g.controls_default(solver=1, tolerance=1e-8, relTol=0.0, reduction="serial", smoother=smoother)
    perf, hist = b2g.gamg_solve(mesh, c.diag, c.coef, c.source, psi, ctl)
    assert tuple(perf) == want["perf"]
    assert hist == list(want["history"])
    assert np.array_equal(psi, want["psi"])


@pytest.mark.parametrize("precision", ["fp32_precond", "fp32_precond_multicolour"])
def test_sym_gauss_seidel_fp32_forms(b2g, oracle, precision):
    c = cases.box_case(24, 20, 22, (2.0, 1.0, 1.0), 20.0, True)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), 1e-9, 0.0,
                                 ctl=oc_controls(smoother="symGaussSeidel"))
    psi = np.zeros(c.n_cells)
    ctl = b2g.controls_default(tolerance=1e-9, relTol=0.0, precision=precision, smoother="symGaussSeidel")
    perf = b2g.pcg_gamg_solve(mesh, c.diag, c.coef, c.source, psi, ctl)[0]
    assert perf.finalResidual < 1e-9
    assert 1 <= perf.nIterations <= want["perf"][2] + 2
    assert np.abs(psi - want["psi"]).max() / np.abs(want["psi"]).max() < 1e-6


@pytest.mark.parametrize("reduction", ["serial", "tree"])
def test_unit_cube_64_parity(b2g, oracle, reduction):
    # the CPU-sized configuration: 64^3 unit cube, tol 1e-6, relTol 0
    c = cases.unit_cube(64)
    perf = _solve_parity(b2g, oracle, c, 1e-6, 0.0, reduction=reduction)
    assert perf.nIterations == 5


def test_standalone_gamg_pitzdaily_openfoam(b2g, pitzdaily, oracle):
    # validation/matrixDumpGAMG: OpenFOAM's GAMG takes 101 V-cycles to 1e-8
    g = pitzdaily
    n = int(g["n_cells"])
    mesh = b2g.Mesh(g["lower"], g["upper"], g["Sf"], g["magSf"], n, 10, True)
    psi = np.zeros(n)
    agg = oracle.agglomerate(g["lower"], g["upper"], g["Sf"], g["magSf"], n, 10, True)
    want = oracle.gamg_solve(agg, g["diag"], g["coef"], g["source"], np.zeros(n),
                             oc_controls(tolerance=1e-8, relTol=0.0))
    # serial reductions: bit-identical to the reference's host path
    ctl = b2g.controls_default(solver=1, tolerance=1e-8, relTol=0.0, reduction="serial")
    perf, hist = b2g.gamg_solve(mesh, g["diag"], g["coef"], g["source"], psi, ctl)
    assert tuple(perf) == want["perf"]
    assert hist == list(want["history"])
    assert np.array_equal(psi, want["psi"])
    # tree reductions: OpenFOAM's own count and solution
    psi = np.zeros(n)
    ctl = b2g.controls_default(solver=1, tolerance=1e-8, relTol=0.0)
    perf, hist = b2g.gamg_solve(mesh, g["diag"], g["coef"], g["source"], psi, ctl)
    assert perf.nIterations == int(g["gamg_perf"][2]) == 101
    assert np.abs(np.asarray(hist) - want["history"]).max() <= 1e-12
    assert np.abs(psi - g["gamg_psi"]).max() / np.abs(g["gamg_psi"]).max() < 1e-9


def test_pcg_gamg_pitzdaily_parity(b2g, oracle, pitzdaily):
    g = pitzdaily
    n = int(g["n_cells"])

    class C:
        pass
    c = C()
    c.lower, c.upper, c.Sf, c.magSf = g["lower"], g["upper"], g["Sf"], g["magSf"]
    c.n_cells, c.diag, c.coef, c.source = n, g["diag"], g["coef"], g["source"]
    _solve_parity(b2g, oracle, c, 1e-8, 0.0, reduction="serial")
    _solve_parity(b2g, oracle, c, 1e-8, 0.0, reduction="tree")


def test_device_memory_solve(b2g, oracle):
    c = cases.box_case(20, 18, 16, (2.0, 1.0, 1.0), 10.0)
    mesh = b2g.Mesh(dev(c.lower, torch.int32), dev(c.upper, torch.int32), dev(c.Sf.reshape(-1)),
                    dev(c.magSf), c.n_cells, 10, True)
    psi = torch.zeros(c.n_cells, dtype=torch.float64, device="cuda")
    perf, hist, _ = b2g.pcg_gamg_solve(mesh, dev(c.diag), dev(c.coef), dev(c.source), psi,
                                       b2g.controls_default())
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells))
    assert perf.nIterations == want["perf"][2]
    assert np.abs(host(psi) - want["psi"]).max() <= FIELD_RTOL * np.abs(want["psi"]).max()


def test_fp32_preconditioned_form(b2g, oracle):
    c = cases.box_case(32, 30, 28, (2.0, 1.0, 1.0), 20.0)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    psi = np.zeros(c.n_cells)
    ctl = b2g.controls_default(tolerance=1e-9, relTol=0.0, precision=1)
    perf, hist, _ = b2g.pcg_gamg_solve(mesh, c.diag, c.coef, c.source, psi, ctl)
    assert perf.finalResidual < 1e-9
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), 1e-9, 0.0)
    err = np.abs(psi - want["psi"]).max() / np.abs(want["psi"]).max()
    assert err < 1e-6


@pytest.mark.parametrize("kw", [dict(nx=32, ny=30, nz=28, lengths=(2.0, 1.0, 1.0), grading_y=20.0),
                                dict(nx=24, ny=20, nz=22, lengths=(2.0, 1.0, 1.0), grading_y=20.0, two_phase=True),
                                dict(nx=40, ny=40, nz=40)], ids=["graded", "two_phase", "cube40"])
def test_fp32_multicolour_form(b2g, oracle, kw):
    # the FP32 V-cycle sweeping colour by colour: the same GaussSeidel update in another cell order,
    # so not bit-comparable; it must reach the tolerance in at most the FP64 iteration count + 2, with
    # the FP64 oracle's field
    c = cases.box_case(**kw)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    want = oracle.pcg_gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), 1e-9, 0.0)
    for _ in range(2):  # the second solve runs on the layout built by the first
        psi = np.zeros(c.n_cells)
        ctl = b2g.controls_default(tolerance=1e-9, relTol=0.0, precision="fp32_precond_multicolour")
        perf, hist, _ = b2g.pcg_gamg_solve(mesh, c.diag, c.coef, c.source, psi, ctl)
        assert perf.finalResidual < 1e-9
        assert 1 <= perf.nIterations <= want["perf"][2] + 2
        err = np.abs(psi - want["psi"]).max() / np.abs(want["psi"]).max()
        assert err < 1e-6
    # every level's sweep shape was chosen by the autotuner's measurements
    for level in range(mesh.n_levels + 1):
        shape = mesh.sweep_shape(level)
        assert shape["threads"] in (128, 256, 512, 1024) and shape["ms_per_sweep"] > 0.0
        assert len(mesh.colouring(level)) >= 2


@pytest.mark.parametrize("smoother", ["GaussSeidel", "symGaussSeidel"])
@pytest.mark.parametrize("kw", [dict(nx=32, ny=30, nz=28, lengths=(2.0, 1.0, 1.0), grading_y=20.0),
                                dict(nx=24, ny=20, nz=22, lengths=(2.0, 1.0, 1.0), grading_y=20.0, two_phase=True)],
                         ids=["graded", "two_phase"])
def test_fp32_multicolour_pipelined_same_bits(b2g, kw, smoother):
    # the multicolour smoothing calls as one pipelined launch over the colours (psi in shared memory)
    # where the tuner measured that faster: every row the same fused multiply-adds in the same order
    # on the same values as the colour-by-colour launches, so the solve's bits do not change
    c = cases.box_case(**kw)
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    ctl = b2g.controls_default(tolerance=1e-9, relTol=0.0, precision="fp32_precond_multicolour", smoother=smoother)
    out = {}
    try:
        for on in (True, False):
            b2g.set_sweep_pipeline(on)
            psi = np.zeros(c.n_cells)
            perf = b2g.pcg_gamg_solve(mesh, c.diag, c.coef, c.source, psi, ctl)[0]
            out[on] = (psi, tuple(perf))
    finally:
        b2g.set_sweep_pipeline(True)
    assert out[True][1] == out[False][1]
    assert np.array_equal(out[True][0], out[False][0])
    assert out[True][1][1] < 1e-9
    sym = smoother == "symGaussSeidel"
    shapes = [mesh.mc_pipe(lv, 2 if lv == 0 else min(2 + lv - 1, 4), sym) for lv in range(mesh.n_levels + 1)]
    # each smoothed coarse level's calls were timed both ways, and some took the pipelined launch
    assert all(s["ms_colours"] > 0.0 for s in shapes[1:mesh.n_levels])
    assert any(s["ranks"] > 0 for s in shapes)


def test_refusals(b2g):
    # three cells and no faces: no pass reduces the count, so no coarse level exists and the solve
    # refuses by name, as GAMGSolver.C:333 does
    mesh = b2g.Mesh(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 3)), np.zeros(0), 3, 10,
                    True)
    assert mesh.n_levels == 0
    with pytest.raises(b2g.GamgError) as e:
        b2g.pcg_gamg_solve(mesh, np.array([1.0, 2.0, 3.0]), np.zeros(0), np.ones(3), np.zeros(3),
                           b2g.controls_default(tolerance=1e-12))
    assert e.value.status == "REFUSED" and "no coarse levels" in str(e.value)
    c = cases.box_case(4, 3, 2)
    bad_lower = c.lower.copy()
    bad_lower[1] = bad_lower[0] + 100
    with pytest.raises(b2g.GamgError) as e:
        b2g.Mesh(bad_lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    assert e.value.status == "ARGUMENT"
    swapped = c.lower.copy()
    swapped[2], swapped[3] = c.upper[2], c.lower[2]
    with pytest.raises(b2g.GamgError) as e:
        b2g.Mesh(swapped, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    assert "upper-triangular" in str(e.value)
