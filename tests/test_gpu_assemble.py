"""The pressure equation's assembly on the device (b2g_assemble_pressure) against the reference's own
cpu::assemblePEqn (src/applications/solvers/simpleFoam/pEqn_cpp.cu:209-260, compiled in oracle/_ref) on
the reference's own box mesh, bit for bit; and the chain a simpleFoam step runs -- assemble, fold the
patches (b2g_fold_boundary), solve -- against the oracle's same chain."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from tests.test_oracle_peqn import CASES, _inputs  # noqa: E402


@pytest.fixture(scope="module")
def b2g():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import brae_b200.native as n
    return n


def _mesh(b2g, sys_, n_cells):
    # the assembly reads only the faces' addressing; the face areas along x stand in for Sf
    nF = len(sys_["lower"])
    Sf = np.zeros((nF, 3))
    Sf[:, 0] = sys_["magSf"]
    return b2g.Mesh(sys_["lower"], sys_["upper"], Sf, sys_["magSf"], n_cells, 10, True)


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("device_arrays", [False, True])
def test_assembly_bitexact_vs_reference(b2g, reference, case, device_arrays):
    n, spacing, fixed, values, ref_cell = CASES[case]
    rAU, phi, phi_b = _inputs(n, case)
    sys_, want = reference.box_pressure_system(n, spacing, fixed, values, rAU, phi, phi_b, ref_cell, 2.5)
    mesh = _mesh(b2g, sys_, len(rAU))
    arg = sys_
    if device_arrays:
        arg = {k: torch.as_tensor(v).cuda() for k, v in sys_.items() if k != "patchSizes"}
    got = b2g.assemble_pressure(mesh, arg, ref_cell, 2.5)
    for k in ("diag", "coef", "source", "internalCoeffs", "boundaryCoeffs"):
        g = got[k].cpu().numpy() if device_arrays else got[k]
        assert np.array_equal(g.view(np.int64), want[k].view(np.int64)), k


def test_assemble_fold_solve_chain(b2g, oracle, reference):
    n = (18, 14, 12)
    rAU, phi, phi_b = _inputs(n, 21)
    sys_, want = reference.box_pressure_system(n, (0.2, 0.1, 0.15), (0, 1, 0, 0, 0, 0), (0, 0, 0, 0, 0, 0),
                                               rAU, phi, phi_b)
    nC = len(rAU)
    mesh = _mesh(b2g, sys_, nC)
    m = b2g.assemble_pressure(mesh, sys_)
    coupled = np.zeros(len(sys_["bFaceCells"]), np.uint8)
    diag, source = b2g.fold_boundary(m["diag"], m["source"], sys_["bFaceCells"], m["internalCoeffs"],
                                     m["boundaryCoeffs"], coupled)
    # the oracle's chain: the restated assembly, the reference's foldBoundary sums, the pinned solve
    o = oracle.assemble_pressure(sys_)
    odiag, osrc = o["diag"].copy(), o["source"].copy()
    for b, c in enumerate(sys_["bFaceCells"]):
        odiag[c] += o["internalCoeffs"][b]
        osrc[c] += o["boundaryCoeffs"][b]
    assert np.array_equal(diag, odiag) and np.array_equal(source, osrc)
    ctl = b2g.controls_default(reduction="serial", tolerance=1e-8)
    psi = np.zeros(nC)
    perf = b2g.pcg_gamg_solve(mesh, diag, m["coef"], source, psi, ctl)[0]
    Sf = np.zeros((len(sys_["lower"]), 3))
    Sf[:, 0] = sys_["magSf"]
    agg = oracle.agglomerate(sys_["lower"], sys_["upper"], Sf, sys_["magSf"], nC, 10, True)
    ref = oracle.pcg_gamg_solve(agg, odiag, o["coef"], osrc, np.zeros(nC), 1e-8, 0.0)
    assert tuple(perf) == ref["perf"]
    assert np.array_equal(psi, ref["psi"])
