"""The coupled (cyclic) pair on the standalone GAMG solve, pinned on the CPU: the oracle's restatement
(oracle/gamg_oracle.c, oc_gamg_solve_pair) against the reference's own gamgSolve with one coupled
patch (gamg_solver_cpp.cu:943-959, compiled here into oracle/_ref), bit for bit -- performance and
field -- for the four smoothers, on periodic boxes.

The pair enters every level: Amul subtracts coeff * psi[nbr] (gamg_solver_cpp.cu:82-87), residual adds
it (:110-115), sumA subtracts coeff (:137-145), the Gauss-Seidel smoothers fold it into bPrime once per
smooth() call (:287-305), DIC reaches it through the residual, and each coarse level's pair is
agglomerated on the coarse cell pair (:497-524).
"""
import numpy as np
import pytest

from brae_b200 import cases
from oracle.bindings import controls

CASES = [
    ("tiny", dict(nx=8, ny=7, nz=6)),
    ("graded", dict(nx=12, ny=10, nz=9, grading_y=5.0)),
    ("two_phase", dict(nx=16, ny=14, nz=18, grading_y=20.0, two_phase=True)),
    # pairs along x and z: the edge cells own two pair faces, added in face order
    ("two_axes", dict(nx=10, ny=9, nz=8, grading_y=5.0, axes=("x", "z"))),
    ("two_axes_two_phase", dict(nx=12, ny=10, nz=14, grading_y=20.0, two_phase=True, axes=("z", "x"))),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_pair_gamg_oracle_equals_reference_bitwise(oracle, reference, name, kw):
    c, own, nbr, pc = cases.periodic_box(**kw)
    ao = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    ar = reference.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    psi0 = np.zeros(c.n_cells)
    for smoother in ("GaussSeidel", "symGaussSeidel", "DIC", "DICGaussSeidel"):
        ctl = controls(smoother=smoother, tolerance=1e-8, relTol=0.0)
        so = oracle.gamg_solve_pair(ao, c.diag, c.coef, own, nbr, pc, c.source, psi0, ctl)
        sr = reference.gamg_solve_pair(ar, c.diag, c.coef, own, nbr, pc, c.source, psi0, ctl)
        assert so["perf"] == sr["perf"], smoother
        assert np.array_equal(so["psi"], sr["psi"]), smoother
        assert 1 <= so["perf"][2] < 1000


def test_pair_controls_oracle_equals_reference(oracle, reference):
    # pre-sweeps, no correction scaling, other sweep counts: every branch of the V-cycle with the pair
    c, own, nbr, pc = cases.periodic_box(12, 10, 9, grading_y=5.0, axes=("x", "z"))
    ao = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    ar = reference.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    psi0 = np.zeros(c.n_cells)
    for kw in (dict(nPreSweeps=2), dict(scaleCorrection=False), dict(nPostSweeps=1, maxPostSweeps=2, nFinestSweeps=3),
               dict(nPreSweeps=1, preSweepsLevelMultiplier=2, smoother="DICGaussSeidel")):
        ctl = controls(tolerance=1e-8, relTol=0.0, **kw)
        so = oracle.gamg_solve_pair(ao, c.diag, c.coef, own, nbr, pc, c.source, psi0, ctl)
        sr = reference.gamg_solve_pair(ar, c.diag, c.coef, own, nbr, pc, c.source, psi0, ctl)
        assert so["perf"] == sr["perf"], kw
        assert np.array_equal(so["psi"], sr["psi"]), kw


def test_pair_changes_the_solution(oracle):
    # the pair couples the two ends: the same system without it converges to another field
    c, own, nbr, pc = cases.periodic_box(12, 10, 9)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    ctl = controls(tolerance=1e-10, relTol=0.0)
    with_pair = oracle.gamg_solve_pair(agg, c.diag, c.coef, own, nbr, pc, c.source, np.zeros(c.n_cells), ctl)
    without = oracle.gamg_solve(agg, c.diag, c.coef, c.source, np.zeros(c.n_cells), ctl)
    # with the pair the solution satisfies the coupled equations
    r = c.source - oracle.amul_pair(c.lower, c.upper, c.diag, c.coef, own, nbr, pc, with_pair["psi"])
    assert np.abs(r).sum() < 1e-6 * np.abs(c.source).sum()
    assert np.abs(with_pair["psi"] - without["psi"]).max() > 1e-3 * np.abs(with_pair["psi"]).max()


def test_coarse_pairs_agglomerate_on_cell_pairs(oracle):
    c, own, nbr, pc = cases.periodic_box(16, 12, 10)
    agg = oracle.agglomerate(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    pairs = oracle.hierarchy_pairs(agg, c.diag, c.coef, own, nbr, pc)
    H = agg.hierarchy
    assert np.array_equal(pairs[0][0], own) and np.array_equal(pairs[0][2], pc)
    for lv in range(1, H.n_levels + 1):
        fo, fn, fc = pairs[lv - 1]
        co, cn, cc = pairs[lv]
        r = H.restrict[lv - 1]
        keys = list(zip(r[fo].tolist(), r[fn].tolist()))
        # one coarse face per distinct coarse cell pair, in order of first appearance
        first = list(dict.fromkeys(keys))
        assert list(zip(co.tolist(), cn.tolist())) == first
        # coefficients: the fine ones summed from zero in fine face order
        want = np.zeros(len(first))
        index = {k: n for n, k in enumerate(first)}
        for k, v in zip(keys, fc):
            want[index[k]] += v
        assert np.array_equal(cc, want)
        assert len(co) <= len(fo)
