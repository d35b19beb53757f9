"""The coarsest-level PCG-DIC entry that allocates no device memory (b2g_level_pcg_dic_static).

Callers whose device memory belongs to another allocator, or that cannot take the device-wide
synchronisation a cudaMalloc/cudaFree may bring in the middle of a solve, call this entry instead of
b2g_level_pcg_dic: its scratch vectors live in a static device array of the library. It must give
exactly what the allocating entry gives, on every call (the array keeps the previous call's
contents), so two calls in a row are checked against b2g_level_pcg_dic here.

The file is named to be collected last: if it fails, a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from brae_b200 import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def b2g():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import brae_b200.native as n
    return n


def _static_solve(b2g, A, level, psi, src, tol, rel_tol):
    perf = b2g._Perf()
    status = b2g.lib.b2g_level_pcg_dic_static(A.handle, level, C.c_void_p(psi.data_ptr()),
                                              C.c_void_p(src.data_ptr()), tol, rel_tol, C.byref(perf))
    assert status == 0, b2g.lib.b2g_last_error().decode()
    return (perf.initialResidual, perf.finalResidual, perf.nIterations)


@pytest.mark.parametrize("coarsest", [True, False], ids=["coarsest-level", "a-finer-level"])
def test_static_scratch_pcg_dic_matches_allocating_entry(b2g, coarsest):
    c = cases.box_case(24, 20, 16, (2.0, 1.0, 1.0), 20.0, name="static")
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, c.diag, c.coef)
    level = mesh.n_levels if coarsest else max(mesh.n_levels - 3, 1)
    n = mesh.level_size(level)[0]
    assert n <= 4096
    rng = np.random.default_rng(5)
    for call in range(2):
        src = torch.as_tensor(rng.standard_normal(n), device="cuda")
        want_psi = torch.zeros(n, dtype=torch.float64, device="cuda")
        want = tuple(A.pcg_dic(level, want_psi, src, 1e-9, 0.0))
        psi = torch.zeros(n, dtype=torch.float64, device="cuda")
        got = _static_solve(b2g, A, level, psi, src, 1e-9, 0.0)
        assert got == want, f"call {call}"
        assert torch.equal(psi, want_psi), f"call {call}"


def test_static_scratch_rejects_large_levels(b2g):
    c = cases.box_case(20, 18, 16, (2.0, 1.0, 1.0), 20.0, name="static-large")
    mesh = b2g.Mesh(c.lower, c.upper, c.Sf, c.magSf, c.n_cells, 10, True)
    A = b2g.Matrix(mesh, c.diag, c.coef)
    n = c.n_cells
    assert n > 4096
    psi = torch.zeros(n, dtype=torch.float64, device="cuda")
    src = torch.ones(n, dtype=torch.float64, device="cuda")
    perf = b2g._Perf()
    status = b2g.lib.b2g_level_pcg_dic_static(A.handle, 0, C.c_void_p(psi.data_ptr()), C.c_void_p(src.data_ptr()),
                                              1e-6, 0.0, C.byref(perf))
    assert status == 1  # B2G_ERR_ARGUMENT
    assert b"at most 4096" in b2g.lib.b2g_last_error()
