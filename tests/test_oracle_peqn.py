"""The pressure equation's assembly ahead of the solve (the reference's cpu::assemblePEqn,
src/applications/solvers/simpleFoam/pEqn_cpp.cu:209-260): the oracle's restatement against the
reference's own code on the reference's own box mesh (tests/box_mesh.cuh), bit for bit -- the matrix,
the source with div(phiHbyA), the patches' coefficients and setReference."""
import numpy as np
import pytest

CASES = [
    # (n, spacing, patch fixed flags, patch values, pRefCell)
    ((6, 5, 4), (1.0, 1.0, 1.0), (0, 1, 0, 0, 0, 0), (0, 0.0, 0, 0, 0, 0), -1),
    ((9, 7, 5), (0.5, 0.25, 0.125), (0, 1, 0, 0, 0, 0), (0, 0.0, 0, 0, 0, 0), -1),
    ((8, 6, 7), (0.3, 0.7, 0.2), (1, 1, 0, 0, 0, 0), (1.5, -0.25, 0, 0, 0, 0), -1),
    ((7, 7, 7), (0.1, 0.2, 0.3), (0, 0, 0, 0, 0, 0), (0, 0, 0, 0, 0, 0), 17),   # all zeroGradient: a reference
]


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = n
    nC = nx * ny * nz
    nF = 3 * nC - (ny * nz + nx * nz + nx * ny)
    nB = 2 * (ny * nz + nx * nz + nx * ny)
    return rng.uniform(0.5, 2.0, nC), rng.uniform(-1.0, 1.0, nF), rng.uniform(-1.0, 1.0, nB)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_assembly_equals_reference(oracle, reference, case):
    n, spacing, fixed, values, ref_cell = CASES[case]
    rAU, phi, phi_b = _inputs(n, case)
    sys_, want = reference.box_pressure_system(n, spacing, fixed, values, rAU, phi, phi_b, ref_cell, 2.5)
    got = oracle.assemble_pressure(sys_, ref_cell, 2.5)
    for k in ("diag", "coef", "source", "internalCoeffs", "boundaryCoeffs"):
        assert np.array_equal(got[k].view(np.int64), want[k].view(np.int64)), k   # bitwise, signed zeros too
    # the face order is the reference box's: owner ascending, +x, +y, +z
    assert np.all(np.diff(sys_["lower"]) >= 0)


def test_assembly_folds_to_the_solved_system(oracle, reference):
    # folded (foldBoundary: diag += internalCoeffs, source += boundaryCoeffs), the matrix is the
    # pressure system the solver takes: symmetric, diagonally dominant with the fixedValue outlet
    n = (8, 6, 5)
    rAU, phi, phi_b = _inputs(n, 9)
    sys_, m = reference.box_pressure_system(n, (0.2, 0.3, 0.4), (0, 1, 0, 0, 0, 0), (0, 0, 0, 0, 0, 0),
                                            rAU, phi, phi_b)
    diag = m["diag"].copy()
    np.add.at(diag, sys_["bFaceCells"], m["internalCoeffs"])
    off = np.zeros_like(diag)
    np.add.at(off, sys_["lower"], np.abs(m["coef"]))
    np.add.at(off, sys_["upper"], np.abs(m["coef"]))
    assert np.all(diag < 0) and np.all(-diag >= off * (1 - 1e-12))
