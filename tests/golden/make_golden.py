"""Regenerates the golden fixtures in this directory from the reference's validation data.

Run here (where the reference tree exists), not on a GPU box:

    make -C oracle fixture REF=/root/reference
    python tests/golden/make_golden.py --ref /root/reference

Inputs, all OpenFOAM v2412 output shipped by the reference (paths relative to its root):

* validation/matrixDump/constant/polyMesh -- the pitzDaily mesh (12,225 cells). Face-area vectors
  come from the reference's own FvGeometry via oracle/_ref/golden_dump, so they are bit-for-bit
  the ones its agglomeration weighs.
* validation/matrixDump/matrix.dat -- OpenFOAM's fvm::laplacian(1,T) LDU (diag, upper, lower,
  source, per-patch internalCoeffs/boundaryCoeffs); format as tests/test_fvm_laplacian.cu:48-75.
* validation/matrixDump/amul.dat -- psi and OpenFOAM's A*psi (tests/test_spmv.cu:32-47).
* validation/matrixDump/solution.dat -- OpenFOAM PCG-DIC, tol 1e-8: 224 iterations.
* validation/matrixDumpGAMG/solution.dat -- OpenFOAM GAMG (GaussSeidel, tol 1e-8, relTol 0,
  nCellsInCoarsestLevel 10, 0/2/2): 101 iterations.
* demo/amgpcg/case20/constant/polyMesh and trace/of_hierarchy.csv -- OpenFOAM's faceAreaPair
  restrict maps for a 4x5x1 mesh at nCellsInCoarsestLevel 4.

The solves use the system as the reference's tests do: the dump negated (tests/test_gamg.cu:31-36)
and the patch coefficients folded in (fvMatrix::solve), from psi = T = 0.
"""
from __future__ import annotations

import argparse
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DUMP = os.path.join(REPO, "oracle", "_ref", "golden_dump")


def read_mesh_bin(path):
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=n, offset=off)
        off += a.nbytes
        return a.copy()

    nC, nIf = take(np.int32, 2)
    lower = take(np.int32, nIf)
    upper = take(np.int32, nIf)
    Sf = take(np.float64, 3 * nIf).reshape(nIf, 3)
    magSf = take(np.float64, nIf)
    (npat,) = take(np.int32, 1)
    patches = []
    for _ in range(npat):
        (ln,) = take(np.int32, 1)
        name = raw[off:off + ln].decode()
        off += ln
        start, size = take(np.int32, 2)
        cells = take(np.int32, size)
        patches.append((name, int(start), cells))
    return int(nC), lower, upper, Sf, magSf, patches


def dump_mesh(poly_mesh_dir, tmp):
    out = os.path.join(tmp, "mesh.bin")
    subprocess.run([DUMP, poly_mesh_dir, out], check=True)
    return read_mesh_bin(out)


def read_matrix_dat(path):
    tok = open(path).read().split()
    nC, nIf, npat = int(tok[0]), int(tok[1]), int(tok[2])
    p = 3
    vals = np.array(tok[p:p + 2 * nC + 2 * nIf], dtype=np.float64)
    p += 2 * nC + 2 * nIf
    diag = vals[:nC]
    upper = vals[nC:nC + nIf]
    lower = vals[nC + nIf:nC + 2 * nIf]
    source = vals[nC + 2 * nIf:]
    patches = {}
    for _ in range(npat):
        name, sz = tok[p], int(tok[p + 1])
        p += 2
        a = np.array(tok[p:p + 2 * sz], dtype=np.float64).reshape(sz, 2) if sz else np.zeros((0, 2))
        p += 2 * sz
        patches[name] = a
    return diag, upper, lower, source, patches


def read_solution(path):
    tok = open(path).read().split()
    nC = int(tok[0])
    init, final, iters = float(tok[1]), float(tok[2]), int(tok[3])
    return init, final, iters, np.array(tok[4:4 + nC], dtype=np.float64)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's source tree")
    args = ap.parse_args()
    ref = args.ref
    tmp = os.path.join(REPO, "oracle", "_ref")
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "fixture", f"REF={ref}"],
                   check=True)

    # ---- pitzDaily ----------------------------------------------------------------------------
    md = os.path.join(ref, "validation", "matrixDump")
    nC, lower, upper, Sf, magSf, mpatches = dump_mesh(os.path.join(md, "constant", "polyMesh"), tmp)
    diag, up, lo, src, pcoef = read_matrix_dat(os.path.join(md, "matrix.dat"))
    assert diag.shape[0] == nC and up.shape[0] == lower.shape[0]
    assert np.array_equal(up, lo), "the pitzDaily laplacian is symmetric"
    # fvMatrix::solve's fold, on the negated system (tests/test_gamg.cu:31-36): diag += iC,
    # source += bC, patch by patch, face by face
    fdiag = -diag
    fsrc = -src
    for name, _start, cells in mpatches:
        a = pcoef.get(name)
        if a is None or a.shape[0] == 0:
            continue
        assert a.shape[0] == cells.shape[0], name
        for i, c in enumerate(cells):
            fdiag[c] += -a[i, 0]
            fsrc[c] += -a[i, 1]
    tok = open(os.path.join(md, "amul.dat")).read().split()
    n = int(tok[0])
    am = np.array(tok[1:1 + 2 * n], dtype=np.float64).reshape(n, 2)
    g_init, g_final, g_iters, g_psi = read_solution(os.path.join(ref, "validation", "matrixDumpGAMG",
                                                                 "solution.dat"))
    p_init, p_final, p_iters, p_psi = read_solution(os.path.join(md, "solution.dat"))
    np.savez_compressed(
        os.path.join(HERE, "pitzdaily.npz"),
        n_cells=np.int32(nC), lower=lower, upper=upper, Sf=Sf, magSf=magSf,
        diag_raw=diag, coef_raw=up, source_raw=src,
        diag=fdiag, coef=-up, source=fsrc,
        amul_psi=am[:, 0], amul_Apsi=am[:, 1],
        gamg_perf=np.array([g_init, g_final, g_iters]), gamg_psi=g_psi,
        pcg_perf=np.array([p_init, p_final, p_iters]), pcg_psi=p_psi)

    # ---- case20: OpenFOAM's own faceAreaPair hierarchy ----------------------------------------
    c20 = os.path.join(ref, "demo", "amgpcg", "case20")
    nC, lower, upper, Sf, magSf, _ = dump_mesh(os.path.join(c20, "constant", "polyMesh"), tmp)
    rows = np.loadtxt(os.path.join(c20, "trace", "of_hierarchy.csv"), delimiter=",", skiprows=1,
                      dtype=np.int64)
    maps = []
    for lv in sorted(set(rows[:, 0].tolist())):
        r = rows[(rows[:, 0] == lv) & (rows[:, 1] >= 0)]
        m = np.full(r[:, 1].max() + 1, -1, np.int32)
        m[r[:, 1]] = r[:, 2]
        maps.append(m)
    np.savez_compressed(
        os.path.join(HERE, "case20.npz"), n_cells=np.int32(nC), lower=lower, upper=upper, Sf=Sf,
        magSf=magSf, n_coarsest=np.int32(4),
        **{f"restrict_{i}": m for i, m in enumerate(maps)})
    print("wrote", os.path.join(HERE, "pitzdaily.npz"), os.path.join(HERE, "case20.npz"))


if __name__ == "__main__":
    main()
