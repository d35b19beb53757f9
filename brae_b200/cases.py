"""Deterministic synthetic pressure systems on structured hex boxes.

These are the benchmark and test inputs: the symmetric 7-point LDU system of a pressure equation
on an Nx x Ny x Nz box, in OpenFOAM's face order (internal faces upper-triangular: for each cell
ascending, its +x, +y, +z neighbour faces -- the order of the reference's tests/box_mesh.cuh:83-92),
with

* off-diagonal (upper == lower) coefficient ``-|Sf|/|d|`` per internal face, ``|d|`` the distance
  between the two cell centres, optionally divided by a face density ``rho_f``;
* diagonal ``-sum(off-diagonals)`` plus ``|Sf|/|C_f - C_P|`` on a fixedValue p=0 patch at x = Lx
  (the boundary coefficient already folded in, as the solver receives it); every other patch is
  zeroGradient and adds nothing;
* source ``b_c = sum_{owned f} phi_f - sum_{neighbour f} phi_f`` with face fluxes ``phi`` drawn
  uniform[-1, 1) from SplitMix64 (a fully specified generator; ``std::uniform_real_distribution``
  is implementation-defined and is not used).

The face-area vectors ``Sf`` (axis aligned) and ``|Sf|`` are returned too: the faceAreaPair
agglomeration weighs faces by them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64_uniform(seed: int, n: int, start: int = 0) -> np.ndarray:
    """Draws ``start .. start+n-1`` of SplitMix64(seed) as doubles in [0, 1) (top 53 bits)."""
    idx = np.arange(start + 1, start + n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + idx * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def graded_spacing(n: int, length: float, grading: float) -> np.ndarray:
    """Cell sizes along one axis, refined geometrically toward BOTH ends.

    ``grading`` is the ratio of the largest (middle) to the smallest (wall) cell in each half; 1 is
    uniform. The two halves mirror each other (an odd middle cell takes the largest size)."""
    if grading == 1.0 or n < 4:
        return np.full(n, length / n)
    half = n // 2
    r = grading ** (1.0 / (half - 1))
    h = r ** np.arange(half, dtype=np.float64)
    if n % 2:
        sizes = np.concatenate([h, [h[-1] * r], h[::-1]])
    else:
        sizes = np.concatenate([h, h[::-1]])
    return sizes * (length / sizes.sum())


@dataclass
class BoxCase:
    """One pressure system: LDU addressing, geometry for the agglomeration, the folded matrix."""

    name: str
    n: tuple
    lengths: tuple
    lower: np.ndarray   # int32 [nFaces] owner side
    upper: np.ndarray   # int32 [nFaces] neighbour side
    Sf: np.ndarray      # float64 [nFaces, 3]
    magSf: np.ndarray   # float64 [nFaces]
    diag: np.ndarray    # float64 [nCells], boundary folded in
    coef: np.ndarray    # float64 [nFaces], upper == lower
    source: np.ndarray  # float64 [nCells]
    max_aspect: float

    @property
    def n_cells(self) -> int:
        return int(self.diag.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.coef.shape[0])


def _rho(z: np.ndarray, dz: float) -> np.ndarray:
    # two-phase density: 1000 below z = 0.5, 1 above, tanh interface 3 cells wide
    return 1.0 + 999.0 * 0.5 * (1.0 - np.tanh((z - 0.5) / (3.0 * dz)))


def box_case(nx: int, ny: int, nz: int, lengths=(1.0, 1.0, 1.0), grading_y: float = 1.0,
             two_phase: bool = False, seed: int = 0, name: str = "box") -> BoxCase:
    lx, ly, lz = lengths
    dx = np.full(nx, lx / nx)
    dy = graded_spacing(ny, ly, grading_y)
    dz = np.full(nz, lz / nz)
    xn = np.concatenate([[0.0], np.cumsum(dx)])
    yn = np.concatenate([[0.0], np.cumsum(dy)])
    zn = np.concatenate([[0.0], np.cumsum(dz)])
    xc = 0.5 * (xn[:-1] + xn[1:])
    yc = 0.5 * (yn[:-1] + yn[1:])
    zc = 0.5 * (zn[:-1] + zn[1:])
    nC = nx * ny * nz
    if nC >= 2**31 - 1:
        raise ValueError("cell count does not fit a 32-bit label")

    k, j, i = np.meshgrid(np.arange(nz, dtype=np.int64), np.arange(ny, dtype=np.int64),
                          np.arange(nx, dtype=np.int64), indexing="ij")
    i = i.ravel(); j = j.ravel(); k = k.ravel()
    c = np.arange(nC, dtype=np.int64)
    nb = np.full((nC, 3), -1, dtype=np.int64)
    nb[:, 0] = np.where(i + 1 < nx, c + 1, -1)
    nb[:, 1] = np.where(j + 1 < ny, c + nx, -1)
    nb[:, 2] = np.where(k + 1 < nz, c + nx * ny, -1)
    mask = nb.ravel() >= 0
    ftype = np.tile(np.arange(3, dtype=np.int8), nC)[mask]
    own = np.repeat(c, 3)[mask]
    nei = nb.ravel()[mask]
    del nb, mask
    fi = i[own]; fj = j[own]; fk = k[own]
    del i, j, k

    area = np.empty(own.shape[0])
    dist = np.empty(own.shape[0])
    zf = np.empty(own.shape[0])
    m = ftype == 0
    area[m] = dy[fj[m]] * dz[fk[m]]
    dist[m] = xc[fi[m] + 1] - xc[fi[m]]
    zf[m] = zc[fk[m]]
    m = ftype == 1
    area[m] = dx[fi[m]] * dz[fk[m]]
    dist[m] = yc[fj[m] + 1] - yc[fj[m]]
    zf[m] = zc[fk[m]]
    m = ftype == 2
    area[m] = dx[fi[m]] * dy[fj[m]]
    dist[m] = zc[fk[m] + 1] - zc[fk[m]]
    zf[m] = zn[fk[m] + 1]
    del m, fi, fj

    Sf = np.zeros((own.shape[0], 3))
    Sf[np.arange(own.shape[0]), ftype.astype(np.int64)] = area
    coef = -area / dist
    if two_phase:
        coef = coef / _rho(zf, lz / nz)
    del zf, dist

    lower = own.astype(np.int32)
    upper = nei.astype(np.int32)
    diag = -(np.bincount(lower, weights=coef, minlength=nC)
             + np.bincount(upper, weights=coef, minlength=nC))
    # fixedValue p = 0 at x = Lx: |Sf| / |C_f - C_P| on the last cell of every x-row
    last = np.arange(nx - 1, nC, nx, dtype=np.int64)
    lj = (last // nx) % ny
    lk = last // (nx * ny)
    bcoef = dy[lj] * dz[lk] / (xn[nx] - xc[nx - 1])
    if two_phase:
        bcoef = bcoef / _rho(zc[lk], lz / nz)
    diag[last] += bcoef

    phi = 2.0 * splitmix64_uniform(seed, own.shape[0]) - 1.0
    source = np.bincount(lower, weights=phi, minlength=nC) - np.bincount(upper, weights=phi,
                                                                         minlength=nC)
    aspect = max(dx.max(), dz.max(), dy.max()) / min(dx.min(), dy.min(), dz.min())
    return BoxCase(name=name, n=(nx, ny, nz), lengths=tuple(lengths), lower=lower, upper=upper,
                   Sf=Sf, magSf=area.copy(), diag=diag, coef=coef, source=source,
                   max_aspect=float(aspect))


def periodic_box(nx: int, ny: int, nz: int, lengths=(2.0, 1.0, 1.0), grading_y: float = 1.0,
                 two_phase: bool = False, seed: int = 0, axes=("z",)):
    """box_case with cyclic pairs: along z (the default) joining the z = 0 and z = Lz faces, and
    along x (axes containing "x") joining x = 0 and x = Lx. Each axis gives two coupled patches, the
    low one first, each listing its cells in face order and its neighbours across the pair face for
    face; the patches follow in the order of `axes`. Returns (case, own, nbr, coeff): the pair in the
    form the coupled patches' faceCells / neighbour faceCells / boundaryCoeffs give it, with the
    matrix's sign convention that Amul subtracts coeff * psi[nbr]. The pair's diagonal share is
    folded into case.diag (the coupled patches' internalCoeffs), so the pair coefficient is the
    off-diagonal's negative. With both axes the box's edge cells own two pair faces."""
    c = box_case(nx, ny, nz, lengths, grading_y, two_phase, seed, name=f"periodic_{nx}x{ny}x{nz}")
    lx, ly, lz = lengths
    dx = lx / nx
    dy = graded_spacing(ny, ly, grading_y)
    dz = lz / nz
    zc = (np.arange(nz) + 0.5) * dz
    owns, nbrs, coefs = [], [], []
    for ax in axes:
        if ax == "z":
            j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
            i = i.ravel(); j = j.ravel()
            low = (j * nx + i).astype(np.int64)
            high = low + (nz - 1) * nx * ny
            coeff = dx * dy[j] / dz  # the two half-cells across the pair face
            if two_phase:
                coeff = coeff / _rho(np.full(coeff.shape, zc[0]), dz)
        elif ax == "x":
            k, j = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
            j = j.ravel(); k = k.ravel()
            low = (k * nx * ny + j * nx).astype(np.int64)
            high = low + (nx - 1)
            coeff = dy[j] * dz / dx
            if two_phase:
                coeff = coeff / _rho(zc[k], dz)
        else:
            raise ValueError(f"periodic axis {ax!r}: x or z")
        owns += [low, high]
        nbrs += [high, low]
        coefs += [coeff, coeff]
    own = np.concatenate(owns).astype(np.int32)
    nbr = np.concatenate(nbrs).astype(np.int32)
    pc = np.concatenate(coefs)
    diag = c.diag.copy()
    np.add.at(diag, own, pc)
    c.diag = diag
    return c, own, nbr, pc


def unit_cube(n: int = 64, seed: int = 0) -> BoxCase:
    """The CPU-sized case: an n^3 uniform unit cube (n = 64: 262,144 cells)."""
    return box_case(n, n, n, (1.0, 1.0, 1.0), 1.0, False, seed, name=f"unit_cube_{n}")


def graded_channel(n: int = 272, seed: int = 0, two_phase: bool = False) -> BoxCase:
    """The 20 M-cell case at n = 272: a 2 x 1 x 1 m box graded 20:1 toward y = 0 and y = 1, outlet
    at x = 2; ``two_phase`` adds the 1000:1 density step at z = 0.5."""
    return box_case(n, n, n, (2.0, 1.0, 1.0), 20.0, two_phase, seed,
                    name=f"graded_channel_{n}" + ("_two_phase" if two_phase else ""))


def mixed_batch_sizes(n_cases: int = 256, lo: int = 4096, hi: int = 1048576, seed: int = 1):
    """Per-case box dimensions for the batched workload: cell counts log-uniform in [lo, hi],
    aspect ratios uniform[1, 8] and y-grading uniform[1, 20] (SplitMix64 stream ``seed``)."""
    u = splitmix64_uniform(seed, 4 * n_cases).reshape(n_cases, 4)
    out = []
    for t in range(n_cases):
        target = math.exp(math.log(lo) + u[t, 0] * (math.log(hi) - math.log(lo)))
        ax = 1.0 + 7.0 * u[t, 1]
        ay = 1.0 + 7.0 * u[t, 2]
        grading = 1.0 + 19.0 * u[t, 3]
        # proportions lx : ly : lz = ax : 1 : ay with cubic cells in the uniform directions
        base = (target / (ax * ay)) ** (1.0 / 3.0)
        nx = max(2, int(round(base * ax)))
        ny = max(4, int(round(base)))
        nz = max(2, int(round(base * ay)))
        out.append(dict(n=(nx, ny, nz), lengths=(ax, 1.0, ay), grading=grading))
    return out


def served_box(target_cells: float, seed: int = 0) -> BoxCase:
    """A served-stream case: the graded channel's construction (2 x 1 x 1 m, 20:1 toward the y
    walls, outlet at x = 2) on a 2m x m x m grid with 2 m^3 nearest ``target_cells``."""
    m = max(4, int(round((target_cells / 2.0) ** (1.0 / 3.0))))
    return box_case(2 * m, m, m, (2.0, 1.0, 1.0), 20.0, False, seed, name=f"served_{2 * m}x{m}x{m}")


# size classes of the served stream: (probability, low cells, high cells), log-uniform within a class
SERVED_CLASSES = ((0.70, 16e3, 128e3), (0.25, 0.5e6, 2e6), (0.05, 8e6, 8e6))


def served_population(per_class=(32, 4, 1), seed: int = 2):
    """Target cell counts of the resident cases the served stream draws from, per size class."""
    u = splitmix64_uniform(seed, sum(per_class))
    out, k = [], 0
    for (p, lo, hi), cnt in zip(SERVED_CLASSES, per_class):
        sizes = []
        for _ in range(cnt):
            sizes.append(math.exp(math.log(lo) + u[k] * (math.log(hi) - math.log(lo))))
            k += 1
        out.append(sizes)
    return out
