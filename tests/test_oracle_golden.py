"""Pins the oracle (oracle/gamg_oracle.c) to OpenFOAM's own dumped answers and to the reference's
own host implementation compiled here (oracle/_ref). CPU only."""
import numpy as np
import pytest

from brae_b200 import cases
from oracle.bindings import controls


def test_amul_matches_openfoam_dump(oracle, pitzdaily):
    # tests/test_spmv.cu:32-47 holds lduMatrix::Amul to OpenFOAM's amul.dat at 1e-12
    g = pitzdaily
    y = oracle.amul(g["lower"], g["upper"], g["diag_raw"], g["coef_raw"], g["amul_psi"])
    rel = np.abs(y - g["amul_Apsi"]).max() / np.abs(g["amul_Apsi"]).max()
    assert rel < 1e-12


def test_standalone_gamg_matches_openfoam(oracle, pitzdaily):
    # validation/matrixDumpGAMG: GaussSeidel, tol 1e-8, relTol 0, nCellsInCoarsestLevel 10, 0/2/2
    g = pitzdaily
    n = int(g["n_cells"])
    agg = oracle.agglomerate(g["lower"], g["upper"], g["Sf"], g["magSf"], n, 10, True)
    assert agg.hierarchy.n_cells == [12225, 6109, 3033, 1504, 745, 367, 181, 88, 42, 20]
    out = oracle.gamg_solve(agg, g["diag"], g["coef"], g["source"], np.zeros(n),
                            controls(tolerance=1e-8, relTol=0.0))
    of_init, of_final, of_iters = g["gamg_perf"]
    init, final, iters = out["perf"]
    assert iters == int(of_iters) == 101
    assert abs(init - of_init) < 1e-12
    assert abs(final - of_final) / of_final < 1e-7
    rel = np.abs(out["psi"] - g["gamg_psi"]).max() / np.abs(g["gamg_psi"]).max()
    assert rel < 1e-11


def test_pcg_dic_matches_openfoam(oracle, pitzdaily):
    # validation/matrixDump/solution.dat: OpenFOAM PCG-DIC, tol 1e-8 -> 224 iterations; this pins
    # the recurrence the coarsest-level solve runs (tests/test_pcg.cu:125-127)
    g = pitzdaily
    n = int(g["n_cells"])
    x, (init, final, iters) = oracle.pcg_dic(g["lower"], g["upper"], g["diag"], g["coef"],
                                             np.zeros(n), g["source"], 1e-8, 0.0, 1000)
    assert iters == int(g["pcg_perf"][2]) == 224
    assert abs(init - g["pcg_perf"][0]) < 1e-9
    assert np.abs(x - g["pcg_psi"]).max() / np.abs(g["pcg_psi"]).max() < 1e-6


def test_face_area_pair_hierarchy_matches_openfoam(oracle, case20):
    # demo/amgpcg/case20/trace/of_hierarchy.csv: OpenFOAM's restrict maps, nCellsInCoarsestLevel 4
    c = case20
    agg = oracle.agglomerate(c["lower"], c["upper"], c["Sf"], c["magSf"], int(c["n_cells"]),
                             int(c["n_coarsest"]), True)
    assert agg.hierarchy.n_levels == 2
    for i in range(2):
        assert np.array_equal(agg.hierarchy.restrict[i], c[f"restrict_{i}"])


CASES = [
    ("tiny", dict(nx=8, ny=7, nz=6, lengths=(2.0, 1.0, 1.0), grading_y=1.0)),
    ("graded", dict(nx=12, ny=10, nz=9, lengths=(2.0, 1.0, 1.0), grading_y=5.0)),
    ("graded20", dict(nx=20, ny=20, nz=20, lengths=(2.0, 1.0, 1.0), grading_y=20.0)),
    ("two_phase", dict(nx=16, ny=14, nz=18, lengths=(2.0, 1.0, 1.0), grading_y=20.0,
                       two_phase=True)),
    ("flat", dict(nx=40, ny=3, nz=2, lengths=(1.0, 1.0, 1.0))),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("forward", [True, False])
def test_oracle_equals_reference_bitwise(oracle, reference, name, kw, forward):
    c = cases.box_case(**kw)
    ao = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, forward)
    ar = reference.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, forward)
    assert ao.hierarchy.equal(ar.hierarchy)
    psi0 = np.zeros(c.n_cells)
    for smoother in ("GaussSeidel", "symGaussSeidel", "DIC", "DICGaussSeidel"):
        ctl = controls(smoother=smoother)
        so = oracle.pcg_gamg_solve(ao, c.diag, c.coef, c.source, psi0, 1e-6, 0.0, ctl=ctl)
        sr = reference.pcg_gamg_solve(ar, c.diag, c.coef, c.source, psi0, 1e-6, 0.0, ctl=ctl)
        assert so["perf"] == sr["perf"], smoother
        assert so["coarsest"] == sr["coarsest"], smoother
        assert np.array_equal(so["psi"], sr["psi"]), smoother


def test_oracle_equals_reference_presweeps_and_standalone(oracle, reference):
    c = cases.box_case(14, 12, 10, (2.0, 1.0, 1.0), 8.0)
    ao = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    ar = reference.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    psi0 = np.linspace(-1, 1, c.n_cells)
    ctl = controls(nPreSweeps=2, nVcycles=3, scaleCorrection=True)
    so = oracle.pcg_gamg_solve(ao, c.diag, c.coef, c.source, psi0, 1e-7, 0.0, min_iter=3, ctl=ctl)
    sr = reference.pcg_gamg_solve(ar, c.diag, c.coef, c.source, psi0, 1e-7, 0.0, min_iter=3, ctl=ctl)
    assert so["perf"] == sr["perf"] and np.array_equal(so["psi"], sr["psi"])
    ctl = controls(tolerance=1e-9, relTol=0.0)
    go = oracle.gamg_solve(ao, c.diag, c.coef, c.source, psi0, ctl)
    gr = reference.gamg_solve(ar, c.diag, c.coef, c.source, psi0, ctl)
    assert go["perf"] == gr["perf"] and np.array_equal(go["psi"], gr["psi"])


def test_oracle_gs_and_coarsest_equal_reference(oracle, reference):
    c = cases.box_case(10, 9, 8, (2.0, 1.0, 1.0), 6.0)
    rng = np.random.default_rng(3)
    psi = rng.standard_normal(c.n_cells)
    for sym in (False, True):
        a = oracle.smooth(c.lower, c.upper, c.diag, c.coef, psi, c.source, 3,
                          "symGaussSeidel" if sym else "GaussSeidel")
        b = reference.gs_smooth(c.lower, c.upper, c.diag, c.coef, psi, c.source, 3, sym)
        assert np.array_equal(a, b)
    x1, p1 = oracle.pcg_dic(c.lower, c.upper, c.diag, c.coef, np.zeros(c.n_cells), c.source,
                            1e-6, 0.0)
    x2, p2 = reference.coarsest_pcg_dic(c.lower, c.upper, c.diag, c.coef, np.zeros(c.n_cells),
                                        c.source, 1e-6, 0.0)
    assert p1 == p2 and np.array_equal(x1, x2)


def test_residual_history_equals_reference(oracle, reference):
    # the reference reports only the final residual: rerun it with maxIter = k for each k
    c = cases.box_case(16, 14, 12, (2.0, 1.0, 1.0), 20.0)
    ao = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    ar = reference.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    psi0 = np.zeros(c.n_cells)
    so = oracle.pcg_gamg_solve(ao, c.diag, c.coef, c.source, psi0, 1e-9, 0.0)
    hist = so["history"]
    assert len(hist) == so["perf"][2] >= 4
    for k in range(1, len(hist) + 1):
        sr = reference.pcg_gamg_solve(ar, c.diag, c.coef, c.source, psi0, 1e-9, 0.0, max_iter=k)
        assert sr["perf"][1] == hist[k - 1]


@pytest.mark.slow
def test_unit_cube_64_equals_reference(oracle, reference):
    # the CPU-sized configuration: 64^3 unit cube, PCG + GAMG(GaussSeidel), tol 1e-6, relTol 0
    c = cases.unit_cube(64)
    ao = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    ar = reference.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    assert ao.hierarchy.equal(ar.hierarchy)
    assert len(ao.hierarchy.n_cells) == 15
    psi0 = np.zeros(c.n_cells)
    so = oracle.pcg_gamg_solve(ao, c.diag, c.coef, c.source, psi0, 1e-6, 0.0)
    sr = reference.pcg_gamg_solve(ar, c.diag, c.coef, c.source, psi0, 1e-6, 0.0)
    assert so["perf"] == sr["perf"]
    assert np.array_equal(so["psi"], sr["psi"])
