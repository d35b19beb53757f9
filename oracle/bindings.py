"""ctypes bindings for the oracle (TEST INFRASTRUCTURE ONLY).

``Oracle`` wraps oracle/_build/liboracle.so, the C restatement of the reference path
(gamg_oracle.c). ``Reference`` wraps oracle/_ref/libref.so, the reference's own host sources
compiled where they lie plus ref_driver.cpp. Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline and reference legs import this module, and only as the checker or as the
timed CPU baseline; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

SMOOTHERS = {"GaussSeidel": 0, "symGaussSeidel": 1, "DIC": 2, "DICGaussSeidel": 3}

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class Controls(C.Structure):
    """oc_controls (gamg_oracle.h): GamgControls + nVcycles with GAMGSolver's defaults."""
    _fields_ = [("smoother", C.c_int), ("tolerance", C.c_double), ("relTol", C.c_double),
                ("maxIter", C.c_int), ("minIter", C.c_int), ("nPreSweeps", C.c_int),
                ("preSweepsLevelMultiplier", C.c_int), ("maxPreSweeps", C.c_int),
                ("nPostSweeps", C.c_int), ("postSweepsLevelMultiplier", C.c_int),
                ("maxPostSweeps", C.c_int), ("nFinestSweeps", C.c_int),
                ("scaleCorrection", C.c_int), ("nCellsInCoarsestLevel", C.c_int),
                ("nVcycles", C.c_int)]


def controls(smoother="GaussSeidel", tolerance=1e-6, relTol=0.0, maxIter=1000, minIter=0,
             nPreSweeps=0, preSweepsLevelMultiplier=1, maxPreSweeps=4, nPostSweeps=2,
             postSweepsLevelMultiplier=1, maxPostSweeps=4, nFinestSweeps=2, scaleCorrection=True,
             nCellsInCoarsestLevel=10, nVcycles=2) -> Controls:
    return Controls(SMOOTHERS[smoother], tolerance, relTol, maxIter, minIter, nPreSweeps,
                    preSweepsLevelMultiplier, maxPreSweeps, nPostSweeps, postSweepsLevelMultiplier,
                    maxPostSweeps, nFinestSweeps, int(bool(scaleCorrection)),
                    nCellsInCoarsestLevel, nVcycles)


class Perf(C.Structure):
    _fields_ = [("initialResidual", C.c_double), ("finalResidual", C.c_double),
                ("nIterations", C.c_int)]

    def as_tuple(self):
        return (self.initialResidual, self.finalResidual, self.nIterations)


def build(reference_root: str | None = None) -> None:
    """Compiles the restatement, and the reference library too when a reference source tree is named
    (reference_root, else the REF environment variable) and present."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref = reference_root or os.environ.get("REF")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={ref}"], check=True)


class Hierarchy:
    """Per-level arrays of an agglomeration: restrict maps, face maps, flips, coarse addressing."""

    def __init__(self, n_cells, n_faces, restrict, face_restrict, flip, lower, upper, forward):
        self.n_cells = n_cells          # [level 0 .. nLevels]
        self.n_faces = n_faces
        self.restrict = restrict        # [step] int32 nCells(step)
        self.face_restrict = face_restrict
        self.flip = flip
        self.lower = lower              # [level] int32 nFaces(level); level 0 = mesh
        self.upper = upper
        self.forward = forward

    @property
    def n_levels(self):
        return len(self.restrict)

    def equal(self, other) -> bool:
        if self.n_cells != other.n_cells or self.n_faces != other.n_faces:
            return False
        for a, b in ((self.restrict, other.restrict), (self.face_restrict, other.face_restrict),
                     (self.flip, other.flip), (self.lower, other.lower), (self.upper, other.upper)):
            for x, y in zip(a, b):
                if not np.array_equal(x, y):
                    return False
        return self.forward == other.forward


def _read_hierarchy(lib, prefix, h, lower0, upper0, forward):
    nlev = getattr(lib, prefix + "agglom_nlevels")(h)
    nc = C.c_int()
    nf = C.c_int()
    n_cells, n_faces = [], []
    for lv in range(nlev + 1):
        getattr(lib, prefix + "agglom_level_size")(h, lv, C.byref(nc), C.byref(nf))
        n_cells.append(nc.value)
        n_faces.append(nf.value)
    restrict, fr, flip, lower, upper = [], [], [], [lower0.copy()], [upper0.copy()]
    for s in range(nlev):
        r = np.empty(n_cells[s], np.int32)
        f = np.empty(n_faces[s], np.int32)
        fl = np.empty(n_faces[s], np.int8)
        lo = np.empty(n_faces[s + 1], np.int32)
        up = np.empty(n_faces[s + 1], np.int32)
        getattr(lib, prefix + "agglom_get")(h, s, r.ctypes.data, f.ctypes.data, fl.ctypes.data,
                                           lo.ctypes.data, up.ctypes.data)
        restrict.append(r); fr.append(f); flip.append(fl); lower.append(lo); upper.append(up)
    return Hierarchy(n_cells, n_faces, restrict, fr, flip, lower, upper, forward)


class _Agglom:
    """Owns a native agglomeration handle."""

    def __init__(self, lib, prefix, handle, hierarchy):
        self._lib = lib
        self._prefix = prefix
        self.handle = handle
        self.hierarchy = hierarchy

    def __del__(self):
        try:
            getattr(self._lib, self._prefix + "agglom_free")(self.handle)
        except Exception:
            pass


class Oracle:
    """The C restatement (gamg_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        self.lib = L
        L.oc_agglomerate.restype = C.c_void_p
        L.oc_agglomerate.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, C.c_int,
                                     C.POINTER(C.c_int)]
        L.oc_agglom_free.argtypes = [C.c_void_p]
        L.oc_agglom_nlevels.argtypes = [C.c_void_p]
        L.oc_agglom_level_size.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                           C.POINTER(C.c_int)]
        L.oc_agglom_get.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 5
        L.oc_agglom_weights.argtypes = [C.c_void_p, C.c_int, _f64p]
        L.oc_hier_build.restype = C.c_void_p
        L.oc_hier_build.argtypes = [C.c_void_p, _f64p, _f64p]
        L.oc_hier_free.argtypes = [C.c_void_p]
        L.oc_hier_level.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p]
        lvl = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p]
        L.oc_amul.argtypes = lvl + [_f64p, _f64p]
        L.oc_norm_factor.restype = C.c_double
        L.oc_norm_factor.argtypes = lvl + [_f64p, _f64p, _f64p]
        L.oc_sum_mag.restype = C.c_double
        L.oc_sum_mag.argtypes = [C.c_int, _f64p]
        L.oc_sum_prod.restype = C.c_double
        L.oc_sum_prod.argtypes = [C.c_int, _f64p, _f64p]
        L.oc_smooth.argtypes = lvl + [_f64p, _f64p, C.c_int, C.c_int]
        L.oc_pcg_dic.restype = Perf
        L.oc_pcg_dic.argtypes = lvl + [_f64p, _f64p, C.c_double, C.c_double, C.c_int]
        L.oc_scale.argtypes = lvl + [_f64p, _f64p, _f64p]
        L.oc_precondition.argtypes = [C.c_void_p, C.POINTER(Controls), _f64p, _f64p, C.c_void_p,
                                      C.c_int, C.POINTER(C.c_int)]
        L.oc_pcg_gamg_solve.restype = Perf
        L.oc_pcg_gamg_solve.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, C.c_double,
                                        C.c_double, C.c_int, C.c_int, C.POINTER(Controls),
                                        C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_int)]
        L.oc_gamg_solve.restype = Perf
        L.oc_gamg_solve.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, C.POINTER(Controls),
                                    C.c_void_p, C.c_int]
        pair = [C.c_int, _i32p, _i32p, _f64p]
        L.oc_hier_build_pair.restype = C.c_void_p
        L.oc_hier_build_pair.argtypes = [C.c_void_p, _f64p, _f64p] + pair
        L.oc_hier_level_pair.restype = C.c_int
        L.oc_hier_level_pair.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_gamg_solve_pair.restype = Perf
        L.oc_gamg_solve_pair.argtypes = [C.c_void_p, _f64p, _f64p] + pair + [
            _f64p, _f64p, C.POINTER(Controls), C.c_void_p, C.c_int]
        L.oc_amul_pair.argtypes = lvl + pair + [_f64p, _f64p]
        L.oc_smooth_pair.argtypes = lvl + pair + [_f64p, _f64p, C.c_int, C.c_int]
        L.oc_assemble_pressure.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                           _f64p, C.c_int, _i32p, _f64p, _f64p, _i32p, _f64p, _f64p, C.c_int,
                                           C.c_double, _f64p, _f64p, _f64p, _f64p, _f64p]

    # -- agglomeration --------------------------------------------------------------------------
    def agglomerate(self, lower, upper, Sf, magSf, n_cells, n_coarsest=10, forward=True):
        lower = np.ascontiguousarray(lower, np.int32)
        upper = np.ascontiguousarray(upper, np.int32)
        fw = C.c_int(1 if forward else 0)
        h = self.lib.oc_agglomerate(n_cells, lower.shape[0], lower, upper,
                                    np.ascontiguousarray(Sf, np.float64).reshape(-1),
                                    np.ascontiguousarray(magSf, np.float64), n_coarsest,
                                    C.byref(fw))
        hier = _read_hierarchy(self.lib, "oc_", h, lower, upper, bool(fw.value))
        return _Agglom(self.lib, "oc_", h, hier)

    def weights(self, agg: _Agglom, step: int) -> np.ndarray:
        w = np.empty(agg.hierarchy.n_faces[step], np.float64)
        self.lib.oc_agglom_weights(agg.handle, step, w)
        return w

    def coarse_matrices(self, agg: _Agglom, diag, coef):
        h = self.lib.oc_hier_build(agg.handle, np.ascontiguousarray(diag, np.float64),
                                   np.ascontiguousarray(coef, np.float64))
        out = []
        H = agg.hierarchy
        for lv in range(H.n_levels + 1):
            d = np.empty(H.n_cells[lv]); u = np.empty(H.n_faces[lv])
            self.lib.oc_hier_level(h, lv, d, u)
            out.append((d, u))
        self.lib.oc_hier_free(h)
        return out

    def precondition(self, agg: _Agglom, diag, coef, r, ctl: Controls, cap=4096):
        h = self.lib.oc_hier_build(agg.handle, np.ascontiguousarray(diag, np.float64),
                                   np.ascontiguousarray(coef, np.float64))
        w = np.zeros_like(r)
        log = (Perf * cap)()
        n = C.c_int()
        self.lib.oc_precondition(h, C.byref(ctl), w, np.ascontiguousarray(r), C.addressof(log),
                                 cap, C.byref(n))
        self.lib.oc_hier_free(h)
        return w, [log[i].as_tuple() for i in range(min(n.value, cap))]

    # -- one level ------------------------------------------------------------------------------
    @staticmethod
    def _lvl(lower, upper, diag, coef):
        return (int(diag.shape[0]), int(coef.shape[0]), np.ascontiguousarray(lower, np.int32),
                np.ascontiguousarray(upper, np.int32), np.ascontiguousarray(diag, np.float64),
                np.ascontiguousarray(coef, np.float64))

    def amul(self, lower, upper, diag, coef, x):
        y = np.empty_like(diag, dtype=np.float64)
        self.lib.oc_amul(*self._lvl(lower, upper, diag, coef), np.ascontiguousarray(x), y)
        return y

    def norm_factor(self, lower, upper, diag, coef, psi, source, Apsi):
        return self.lib.oc_norm_factor(*self._lvl(lower, upper, diag, coef),
                                       np.ascontiguousarray(psi), np.ascontiguousarray(source),
                                       np.ascontiguousarray(Apsi))

    def smooth(self, lower, upper, diag, coef, psi, source, n_sweeps, smoother="GaussSeidel"):
        x = np.array(psi, dtype=np.float64, copy=True)
        self.lib.oc_smooth(*self._lvl(lower, upper, diag, coef), x, np.ascontiguousarray(source),
                           n_sweeps, SMOOTHERS[smoother])
        return x

    def pcg_dic(self, lower, upper, diag, coef, psi, source, tol, rel_tol, max_iter=1000):
        x = np.array(psi, dtype=np.float64, copy=True)
        p = self.lib.oc_pcg_dic(*self._lvl(lower, upper, diag, coef), x,
                                np.ascontiguousarray(source), tol, rel_tol, max_iter)
        return x, p.as_tuple()

    def scale(self, lower, upper, diag, coef, field, source):
        f = np.array(field, dtype=np.float64, copy=True)
        acf = np.empty_like(f)
        self.lib.oc_scale(*self._lvl(lower, upper, diag, coef), f, acf,
                          np.ascontiguousarray(source))
        return f, acf

    # -- whole solves ---------------------------------------------------------------------------
    def pcg_gamg_solve(self, agg: _Agglom, diag, coef, source, psi, tol=1e-6, rel_tol=0.0,
                       max_iter=1000, min_iter=0, ctl: Controls | None = None, cap=4096):
        ctl = ctl or controls()
        x = np.array(psi, dtype=np.float64, copy=True)
        hist = np.zeros(max(1, min(max_iter, cap)))
        log = (Perf * cap)()
        n = C.c_int()
        p = self.lib.oc_pcg_gamg_solve(agg.handle, np.ascontiguousarray(diag, np.float64),
                                       np.ascontiguousarray(coef, np.float64),
                                       np.ascontiguousarray(source, np.float64), x, tol, rel_tol,
                                       max_iter, min_iter, C.byref(ctl), hist.ctypes.data,
                                       hist.shape[0], C.addressof(log), cap, C.byref(n))
        return dict(psi=x, perf=p.as_tuple(), history=hist[:min(p.nIterations, hist.shape[0])],
                    coarsest=[log[i].as_tuple() for i in range(min(n.value, cap))])

    def gamg_solve(self, agg: _Agglom, diag, coef, source, psi, ctl: Controls, cap=100000):
        x = np.array(psi, dtype=np.float64, copy=True)
        hist = np.zeros(cap)
        p = self.lib.oc_gamg_solve(agg.handle, np.ascontiguousarray(diag, np.float64),
                                   np.ascontiguousarray(coef, np.float64),
                                   np.ascontiguousarray(source, np.float64), x, C.byref(ctl),
                                   hist.ctypes.data, cap)
        return dict(psi=x, perf=p.as_tuple(), history=hist[:min(p.nIterations, cap)])

    # -- the pressure equation's assembly ---------------------------------------------------------
    def assemble_pressure(self, sys_: dict, p_ref_cell=-1, p_ref_value=0.0):
        """cpu::assemblePEqn restated (oc_assemble_pressure) on a PressureSystem dict (see
        Reference.box_pressure_system): returns diag, coef, source, internalCoeffs, boundaryCoeffs."""
        nC, nF, nB = len(sys_["V"]), len(sys_["lower"]), len(sys_["bFaceCells"])
        out = {k: np.zeros(n) for k, n in (("diag", nC), ("coef", nF), ("source", nC),
                                            ("internalCoeffs", nB), ("boundaryCoeffs", nB))}
        self.lib.oc_assemble_pressure(nC, nF, *[np.ascontiguousarray(sys_[k]) for k in (
            "lower", "upper", "weights", "deltaCoeffs", "magSf", "V", "rAU", "phi")], nB,
            *[np.ascontiguousarray(sys_[k]) for k in ("bFaceCells", "bMagSf", "bDeltaCoeffs", "bType", "bValue",
                                                        "bPhi")],
            int(p_ref_cell), float(p_ref_value), out["diag"], out["coef"], out["source"], out["internalCoeffs"],
            out["boundaryCoeffs"])
        return out

    # -- the coupled pair -----------------------------------------------------------------------
    @staticmethod
    def _pair(own, nbr, coeff):
        return (int(len(own)), np.ascontiguousarray(own, np.int32), np.ascontiguousarray(nbr, np.int32),
                np.ascontiguousarray(coeff, np.float64))

    def gamg_solve_pair(self, agg: _Agglom, diag, coef, own, nbr, pcoef, source, psi, ctl: Controls,
                        cap=100000):
        x = np.array(psi, dtype=np.float64, copy=True)
        hist = np.zeros(cap)
        p = self.lib.oc_gamg_solve_pair(agg.handle, np.ascontiguousarray(diag, np.float64),
                                        np.ascontiguousarray(coef, np.float64), *self._pair(own, nbr, pcoef),
                                        np.ascontiguousarray(source, np.float64), x, C.byref(ctl),
                                        hist.ctypes.data, cap)
        return dict(psi=x, perf=p.as_tuple(), history=hist[:min(p.nIterations, cap)])

    def hierarchy_pairs(self, agg: _Agglom, diag, coef, own, nbr, pcoef):
        """Every level's pair (own, nbr, coeff) after agglomeration, level 0 first."""
        h = self.lib.oc_hier_build_pair(agg.handle, np.ascontiguousarray(diag, np.float64),
                                        np.ascontiguousarray(coef, np.float64), *self._pair(own, nbr, pcoef))
        out = []
        for lv in range(agg.hierarchy.n_levels + 1 if hasattr(agg.hierarchy, "n_levels")
                        else len(agg.hierarchy.n_cells)):
            m = self.lib.oc_hier_level_pair(h, lv, None, None, None)
            o = np.empty(m, np.int32); nb = np.empty(m, np.int32); c = np.empty(m, np.float64)
            self.lib.oc_hier_level_pair(h, lv, o.ctypes.data, nb.ctypes.data, c.ctypes.data)
            out.append((o, nb, c))
        self.lib.oc_hier_free(h)
        return out

    def amul_pair(self, lower, upper, diag, coef, own, nbr, pcoef, x):
        y = np.empty_like(diag, dtype=np.float64)
        self.lib.oc_amul_pair(*self._lvl(lower, upper, diag, coef), *self._pair(own, nbr, pcoef),
                              np.ascontiguousarray(x), y)
        return y

    def smooth_pair(self, lower, upper, diag, coef, own, nbr, pcoef, psi, source, n_sweeps,
                    smoother="GaussSeidel"):
        x = np.array(psi, dtype=np.float64, copy=True)
        self.lib.oc_smooth_pair(*self._lvl(lower, upper, diag, coef), *self._pair(own, nbr, pcoef), x,
                                np.ascontiguousarray(source), n_sweeps, SMOOTHERS[smoother])
        return x


class Reference:
    """The reference's own host path (oracle/_ref/libref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle ref)")
        L = C.CDLL(path)
        self.lib = L
        L.ref_last_error.restype = C.c_char_p
        L.ref_agglomerate.restype = C.c_void_p
        L.ref_agglomerate.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, C.c_int,
                                      C.POINTER(C.c_int)]
        L.ref_agglom_free.argtypes = [C.c_void_p]
        L.ref_agglom_nlevels.argtypes = [C.c_void_p]
        L.ref_agglom_level_size.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                            C.POINTER(C.c_int)]
        L.ref_agglom_get.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 5
        L.ref_pcg_gamg_solve.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, C.c_double,
                                         C.c_double, C.c_int, C.c_int, C.POINTER(Controls),
                                         C.POINTER(Perf), C.c_void_p, C.c_int,
                                         C.POINTER(C.c_int)]
        L.ref_gamg_solve.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, C.POINTER(Controls),
                                     C.POINTER(Perf)]
        L.ref_gs_smooth.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p,
                                    C.c_int, C.c_int]
        L.ref_gamg_solve_pair.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, C.c_int, _i32p, _i32p,
                                          _f64p, C.POINTER(Controls), C.POINTER(Perf)]
        L.ref_coarsest_pcg_dic.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p,
                                           _f64p, C.c_double, C.c_double, C.POINTER(Perf)]

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    # -- the pressure equation's assembly (ref_peqn.cpp over cpu::assemblePEqn) -----------------
    BOX_PATCHES = ("inlet", "outlet", "wallYmin", "wallYmax", "wallZmin", "wallZmax")

    def box_pressure_system(self, n, spacing, fixed, values, rAU, phi, phi_b, p_ref_cell=-1, p_ref_value=0.0):
        """The reference's own assembly of the pressure equation on its own Nx x Ny x Nz box (cell sizes
        `spacing`), the pressure fixedValue values[i] on patch i where fixed[i], zeroGradient elsewhere
        (patches in BOX_PATCHES order). Returns the inputs and the geometry the assembly read (a
        PressureSystem dict the oracle and the device take) and the reference's matrix."""
        L = self.lib
        if not getattr(self, "_peqn", False):
            L.ref_peqn_last_error.restype = C.c_char_p
            L.ref_box_assemble_peqn.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [_i32p, _f64p, _f64p, _f64p,
                                                                                  _f64p, C.c_int, C.c_double] + \
                [_i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]
            self._peqn = True
        nx, ny, nz = n
        nC = nx * ny * nz
        nF = 3 * nC - (ny * nz + nx * nz + nx * ny)
        sizes = [ny * nz, ny * nz, nx * nz, nx * nz, nx * ny, nx * ny]
        nB = sum(sizes)
        g = {"lower": np.zeros(nF, np.int32), "upper": np.zeros(nF, np.int32), "weights": np.zeros(nF),
             "deltaCoeffs": np.zeros(nF), "magSf": np.zeros(nF), "V": np.zeros(nC),
             "bFaceCells": np.zeros(nB, np.int32), "bMagSf": np.zeros(nB), "bDeltaCoeffs": np.zeros(nB)}
        m = {"diag": np.zeros(nC), "coef": np.zeros(nF), "source": np.zeros(nC), "internalCoeffs": np.zeros(nB),
             "boundaryCoeffs": np.zeros(nB)}
        rc = L.ref_box_assemble_peqn(nx, ny, nz, *[float(x) for x in spacing],
                                     np.ascontiguousarray(fixed, np.int32), np.ascontiguousarray(values, np.float64),
                                     np.ascontiguousarray(rAU, np.float64), np.ascontiguousarray(phi, np.float64),
                                     np.ascontiguousarray(phi_b, np.float64), int(p_ref_cell), float(p_ref_value),
                                     g["lower"], g["upper"], g["weights"], g["deltaCoeffs"], g["magSf"], g["V"],
                                     g["bFaceCells"], g["bMagSf"], g["bDeltaCoeffs"], m["diag"], m["coef"],
                                     m["source"], m["internalCoeffs"], m["boundaryCoeffs"])
        if rc != 0:
            raise RuntimeError(L.ref_peqn_last_error().decode())
        btype = np.concatenate([np.full(sz, 1 if f else 0, np.int32) for sz, f in zip(sizes, fixed)])
        bval = np.concatenate([np.full(sz, float(v) if f else 0.0) for sz, f, v in zip(sizes, fixed, values)])
        g.update(rAU=np.ascontiguousarray(rAU, np.float64), phi=np.ascontiguousarray(phi, np.float64),
                 bPhi=np.ascontiguousarray(phi_b, np.float64), bType=btype, bValue=bval,
                 patchSizes=np.asarray(sizes, np.int32))
        return g, m

    def agglomerate(self, lower, upper, Sf, magSf, n_cells, n_coarsest=10, forward=True):
        lower = np.ascontiguousarray(lower, np.int32)
        upper = np.ascontiguousarray(upper, np.int32)
        fw = C.c_int(1 if forward else 0)
        h = self.lib.ref_agglomerate(n_cells, lower.shape[0], lower, upper,
                                     np.ascontiguousarray(Sf, np.float64).reshape(-1),
                                     np.ascontiguousarray(magSf, np.float64), n_coarsest,
                                     C.byref(fw))
        if not h:
            raise RuntimeError(self.lib.ref_last_error().decode())
        hier = _read_hierarchy(self.lib, "ref_", h, lower, upper, bool(fw.value))
        return _Agglom(self.lib, "ref_", h, hier)

    def pcg_gamg_solve(self, agg: _Agglom, diag, coef, source, psi, tol=1e-6, rel_tol=0.0,
                       max_iter=1000, min_iter=0, ctl: Controls | None = None, cap=4096):
        ctl = ctl or controls()
        x = np.array(psi, dtype=np.float64, copy=True)
        perf = Perf()
        log = (Perf * cap)()
        n = C.c_int()
        self._check(self.lib.ref_pcg_gamg_solve(
            agg.handle, np.ascontiguousarray(diag, np.float64),
            np.ascontiguousarray(coef, np.float64), np.ascontiguousarray(source, np.float64), x,
            tol, rel_tol, max_iter, min_iter, C.byref(ctl), C.byref(perf), C.addressof(log), cap,
            C.byref(n)))
        return dict(psi=x, perf=perf.as_tuple(),
                    coarsest=[log[i].as_tuple() for i in range(min(n.value, cap))])

    def gamg_solve(self, agg: _Agglom, diag, coef, source, psi, ctl: Controls):
        x = np.array(psi, dtype=np.float64, copy=True)
        perf = Perf()
        self._check(self.lib.ref_gamg_solve(agg.handle, np.ascontiguousarray(diag, np.float64),
                                            np.ascontiguousarray(coef, np.float64),
                                            np.ascontiguousarray(source, np.float64), x,
                                            C.byref(ctl), C.byref(perf)))
        return dict(psi=x, perf=perf.as_tuple())

    def gamg_solve_pair(self, agg: _Agglom, diag, coef, own, nbr, pcoef, source, psi, ctl: Controls):
        """gamgSolve with one coupled patch carrying the pair (its internalCoeffs zero)."""
        x = np.array(psi, dtype=np.float64, copy=True)
        perf = Perf()
        self._check(self.lib.ref_gamg_solve_pair(
            agg.handle, np.ascontiguousarray(diag, np.float64), np.ascontiguousarray(coef, np.float64),
            np.ascontiguousarray(source, np.float64), x, int(len(own)), np.ascontiguousarray(own, np.int32),
            np.ascontiguousarray(nbr, np.int32), np.ascontiguousarray(pcoef, np.float64), C.byref(ctl),
            C.byref(perf)))
        return dict(psi=x, perf=perf.as_tuple())

    def gs_smooth(self, lower, upper, diag, coef, psi, b, n_sweeps, symmetric=False):
        x = np.array(psi, dtype=np.float64, copy=True)
        self._check(self.lib.ref_gs_smooth(int(diag.shape[0]), int(coef.shape[0]),
                                           np.ascontiguousarray(lower, np.int32),
                                           np.ascontiguousarray(upper, np.int32),
                                           np.ascontiguousarray(diag, np.float64),
                                           np.ascontiguousarray(coef, np.float64), x,
                                           np.ascontiguousarray(b, np.float64), n_sweeps,
                                           int(symmetric)))
        return x

    def coarsest_pcg_dic(self, lower, upper, diag, coef, psi, source, tol, rel_tol):
        x = np.array(psi, dtype=np.float64, copy=True)
        perf = Perf()
        self._check(self.lib.ref_coarsest_pcg_dic(int(diag.shape[0]), int(coef.shape[0]),
                                                  np.ascontiguousarray(lower, np.int32),
                                                  np.ascontiguousarray(upper, np.int32),
                                                  np.ascontiguousarray(diag, np.float64),
                                                  np.ascontiguousarray(coef, np.float64), x,
                                                  np.ascontiguousarray(source, np.float64), tol,
                                                  rel_tol, C.byref(perf)))
        return x, perf.as_tuple()
