"""The C ABI library without a GPU: it loads, exports every symbol include/brae_gamg.h declares,
and its host-side logic (controls, the fvSolution reader and its refusals) behaves. No compute."""
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(REPO, "include", "brae_gamg.h")).read()
    return sorted(set(re.findall(r"B2G_API\s+[\w\s\*]+?\b(b2g_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import brae_b200.native as n
    declared = _declared()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(n.lib, name), name
    assert sorted(n.EXPORTED) == declared


def test_controls_defaults():
    import brae_b200 as b
    c = b.controls_default()
    assert (c.tolerance, c.relTol, c.maxIter, c.minIter) == (1e-6, 0.0, 1000, 0)
    assert (c.nPreSweeps, c.preSweepsLevelMultiplier, c.maxPreSweeps) == (0, 1, 4)
    assert (c.nPostSweeps, c.postSweepsLevelMultiplier, c.maxPostSweeps) == (2, 1, 4)
    assert (c.nFinestSweeps, c.scaleCorrection, c.nCellsInCoarsestLevel, c.nVcycles) == (2, 1, 10, 2)
    assert (c.precTolerance, c.precRelTol) == (1e-6, 0.0)


ENTRY = """
    solver          PCG;
    tolerance       1e-06;   // the PCG's
    relTol          0.05;
    maxIter         1000;
    preconditioner
    {
        preconditioner  GAMG;
        smoother        GaussSeidel;
        nPreSweeps      0;
        nPostSweeps     2;
        nCellsInCoarsestLevel 10;
        tolerance       1e-5;
        /* the GAMG's own relTol */
        relTol          0.01;
        nVcycles        3;
    }
"""


def test_read_pcg_gamg_entry():
    import brae_b200 as b
    c = b.read_controls(ENTRY)
    assert c.solver == 0 and c.tolerance == 1e-6 and c.relTol == 0.05 and c.maxIter == 1000
    assert c.smoother == 0 and c.nPostSweeps == 2 and c.nCellsInCoarsestLevel == 10
    assert c.precTolerance == 1e-5 and c.precRelTol == 0.01 and c.nVcycles == 3


def test_read_standalone_gamg_entry():
    import brae_b200 as b
    c = b.read_controls("solver GAMG; smoother DICGaussSeidel; tolerance 1e-8; relTol 0; "
                        "nFinestSweeps 3; scaleCorrection off;")
    assert c.solver == 1 and c.smoother == 3 and c.tolerance == 1e-8 and c.nFinestSweeps == 3
    assert c.scaleCorrection == 0 and c.precTolerance == 1e-8


@pytest.mark.parametrize("entry,needle", [
    ("solver PCG; preconditioner { preconditioner GAMG; }", "names no `smoother`"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother DILU; }", "ASYMMETRIC"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother FDIC; }", "not ported"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother Jacobi; }", "not ported"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; agglomerator algebraicPair; }",
     "agglomerator"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; mergeLevels 2; }", "mergeLevels"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; updateInterval 5; }",
     "updateInterval"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; cacheAgglomeration no; }",
     "cacheAgglomeration"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; interpolateCorrection yes; }",
     "interpolateCorrection"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; directSolveCoarsest yes; }",
     "directSolveCoarsest"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; coarsestLevelCorr { solver PCG; } }",
     "coarsestLevelCorr"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; processorAgglomerator masterCoarsest; }",
     "processorAgglomerator"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; scaleCorrection maybe; }",
     "not a Switch"),
    ("solver PCG; preconditioner DIC;", "sub-dictionary"),
    ("solver PCG; preconditioner { preconditioner DIC; }", "Only the GAMG preconditioner"),
    ("solver PBiCGStab; preconditioner DILU;", "solver PBiCGStab"),
    ("solver PCG; preconditioner { preconditioner GAMG; smoother GaussSeidel; nVcycles 0; }", "nVcycles"),
])
def test_read_refusals(entry, needle):
    import brae_b200 as b
    with pytest.raises(b.GamgError) as e:
        b.read_controls(entry)
    assert e.value.status == "REFUSED"
    assert needle in str(e.value)
