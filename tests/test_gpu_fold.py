"""foldBoundary on the device (b2g_fold_boundary): the step before the solve, bit for bit.

The reference (gamg_solver_cpp.cu:769-797) walks the patches in order and each patch's faces in
order, adding every internal coefficient to its cell's diagonal and, only where the patch is not
coupled, the boundary coefficient to its source. Cells with several boundary faces (edges and
corners of a box, and faces of several patches) receive their terms in that order; the device fold
must give the same bits.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def b2g():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import brae_b200.native as n
    return n


def _reference_fold(diag, source, patches):
    d, s = diag.copy(), source.copy()
    for cells, ic, bc, coupled in patches:
        for i in range(len(cells)):
            c = cells[i]
            d[c] = d[c] + ic[i]
            if not coupled:
                s[c] = s[c] + bc[i]
    return d, s


def _patches(rng, n):
    out = []
    for size, coupled in ((700, False), (350, True), (900, False), (5, False)):
        cells = rng.integers(0, n, size=size).astype(np.int32)  # repeats within and across patches
        out.append((cells, rng.standard_normal(size), rng.standard_normal(size), coupled))
    return out


def _concat(patches):
    fc = np.concatenate([p[0] for p in patches])
    ic = np.concatenate([p[1] for p in patches])
    bc = np.concatenate([p[2] for p in patches])
    cp = np.concatenate([np.full(len(p[0]), 1 if p[3] else 0, np.uint8) for p in patches])
    return fc, ic, bc, cp


def test_fold_bitexact_host_and_device(b2g):
    rng = np.random.default_rng(3)
    n = 1000
    diag = rng.standard_normal(n) + 10.0
    source = rng.standard_normal(n)
    patches = _patches(rng, n)
    want_d, want_s = _reference_fold(diag, source, patches)
    fc, ic, bc, cp = _concat(patches)
    d, s = b2g.fold_boundary(diag, source, fc, ic, bc, cp)
    assert np.array_equal(d, want_d)
    assert np.array_equal(s, want_s)
    # device memory: the same bits
    dev = lambda a: torch.as_tensor(a).cuda()
    td, ts = dev(diag.copy()), dev(source.copy())
    tfc, tic, tbc, tcp = dev(fc), dev(ic), dev(bc), dev(cp)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    rc = b2g.lib.b2g_fold_boundary(n, len(fc), ptr(tfc), ptr(tic), ptr(tbc), ptr(tcp), ptr(td), ptr(ts),
                                   b2g.B2G_MEM_DEVICE, None)
    assert rc == 0
    assert np.array_equal(td.cpu().numpy(), want_d)
    assert np.array_equal(ts.cpu().numpy(), want_s)


def test_fold_no_boundary_and_refusals(b2g):
    diag = np.arange(5.0) + 1.0
    source = np.ones(5)
    d, s = b2g.fold_boundary(diag, source, np.zeros(0, np.int32), np.zeros(0), np.zeros(0), np.zeros(0, np.uint8))
    assert np.array_equal(d, diag) and np.array_equal(s, source)
    with pytest.raises(b2g.GamgError, match="outside"):
        b2g.fold_boundary(diag, source, np.array([0, 7], np.int32), np.ones(2), np.ones(2), np.zeros(2, np.uint8))
