"""ctypes bindings of include/brae_gamg.h.

Array arguments may be numpy arrays (host memory, ``B2G_MEM_HOST``) or CUDA tensors (device memory,
``B2G_MEM_DEVICE``); the two are never mixed in one call. Device work runs on the stream the mesh
was created on (torch's current stream when created from Python), and every call returns after it
completes.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import NamedTuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbrae_gamg.so")

B2G_MEM_HOST = 0
B2G_MEM_DEVICE = 1
SMOOTHERS = {"GaussSeidel": 0, "symGaussSeidel": 1, "DIC": 2, "DICGaussSeidel": 3}
STATUS = {0: "OK", 1: "ARGUMENT", 2: "REFUSED", 3: "CUDA", 4: "NO_MEMORY", 5: "DEVICE_TIMEOUT", 6: "STATE"}


class GamgError(RuntimeError):
    """A failed call: ``status`` is the b2g_status name, the message is b2g_last_error()."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{STATUS.get(status, status)}] {message}")
        self.status = STATUS.get(status, str(status))


class Controls(C.Structure):
    """b2g_controls."""
    _fields_ = [("solver", C.c_int), ("tolerance", C.c_double), ("relTol", C.c_double),
                ("maxIter", C.c_int), ("minIter", C.c_int), ("smoother", C.c_int),
                ("precTolerance", C.c_double), ("precRelTol", C.c_double),
                ("nPreSweeps", C.c_int), ("preSweepsLevelMultiplier", C.c_int),
                ("maxPreSweeps", C.c_int), ("nPostSweeps", C.c_int),
                ("postSweepsLevelMultiplier", C.c_int), ("maxPostSweeps", C.c_int),
                ("nFinestSweeps", C.c_int), ("scaleCorrection", C.c_int),
                ("nCellsInCoarsestLevel", C.c_int), ("nVcycles", C.c_int), ("precision", C.c_int),
                ("reduction", C.c_int), ("coarsestDirect", C.c_int)]


class _Perf(C.Structure):
    _fields_ = [("initialResidual", C.c_double), ("finalResidual", C.c_double),
                ("nIterations", C.c_int)]


class _Log(C.Structure):
    _fields_ = [("history", C.POINTER(C.c_double)), ("historyCapacity", C.c_int),
                ("historyCount", C.c_int), ("coarsest", C.POINTER(_Perf)),
                ("coarsestCapacity", C.c_int), ("coarsestCount", C.c_int)]


class SolverPerformance(NamedTuple):
    """SolverPerformance (src/OpenFOAM/matrices/pcg.cuh:16-21)."""
    initialResidual: float
    finalResidual: float
    nIterations: int


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m brae_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_double
    sig = {
        "b2g_last_error": (C.c_char_p, []),
        "b2g_version": (C.c_char_p, []),
        "b2g_set_profiling": (ip, [ip]),
        "b2g_set_sweep_pipeline": (ip, [ip]),
        "b2g_coarsest_dense_solve": (ip, [vp, vp, vp]),
        "b2g_assemble_pressure": (ip, [vp] + [vp] * 6 + [ip] + [vp] * 6 + [ip, dp] + [vp] * 5 + [ip, vp]),
        "b2g_set_part_cells": (ip, [ip]),
        "b2g_level_grid_stall": (ip, [vp, ip, vp, vp, ip, ip, C.c_longlong]),
        "b2g_level_smooth_pipelined": (ip, [vp, ip, vp, vp, ip, ip]),
        "b2g_level_pipe_shape": (ip, [vp, ip, ip, ip, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float),
                                      C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                      C.POINTER(C.c_float), C.POINTER(C.c_int)]),
        "b2g_controls_default": (ip, [C.POINTER(Controls)]),
        "b2g_controls_read": (ip, [C.c_char_p, C.POINTER(Controls)]),
        "b2g_mesh_create": (ip, [ip, ip, vp, vp, vp, vp, ip, C.POINTER(C.c_int), ip, vp,
                                 C.POINTER(vp)]),
        "b2g_mesh_create_cached": (ip, [ip, ip, vp, vp, vp, vp, ip, C.POINTER(C.c_int), ip, vp, C.c_char_p,
                                        C.POINTER(vp), C.POINTER(C.c_int)]),
        "b2g_mesh_destroy": (ip, [vp]),
        "b2g_mesh_levels": (ip, [vp, C.POINTER(C.c_int)]),
        "b2g_mesh_level_size": (ip, [vp, ip, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "b2g_mesh_get_step": (ip, [vp, ip, vp, vp, vp, vp, vp]),
        "b2g_mesh_build_ms": (ip, [vp, C.POINTER(C.c_float)]),
        "b2g_pcg_gamg_solve": (ip, [vp, vp, vp, vp, vp, C.POINTER(Controls), ip, vp,
                                    C.POINTER(_Perf), C.POINTER(_Log)]),
        "b2g_gamg_solve": (ip, [vp, vp, vp, vp, vp, C.POINTER(Controls), ip, vp, C.POINTER(_Perf),
                                C.POINTER(_Log)]),
        "b2g_matrix_create": (ip, [vp, vp, vp, ip, vp, C.POINTER(vp)]),
        "b2g_matrix_destroy": (ip, [vp]),
        "b2g_matrix_set_coeffs": (ip, [vp, vp, vp, ip]),
        "b2g_matrix_get_level": (ip, [vp, ip, vp, vp]),
        "b2g_level_amul": (ip, [vp, ip, vp, vp]),
        "b2g_level_smooth": (ip, [vp, ip, ip, vp, vp, ip]),
        "b2g_level_scale": (ip, [vp, ip, vp, vp, vp]),
        "b2g_step_restrict": (ip, [vp, ip, vp, vp]),
        "b2g_step_prolong": (ip, [vp, ip, vp, vp]),
        "b2g_level_norm_factor": (ip, [vp, ip, vp, vp, vp, C.POINTER(C.c_double)]),
        "b2g_level_pcg_dic": (ip, [vp, ip, vp, vp, dp, dp, C.POINTER(_Perf)]),
        "b2g_level_pcg_dic_static": (ip, [vp, ip, vp, vp, dp, dp, C.POINTER(_Perf)]),
        "b2g_level_schedule": (ip, [vp, ip, vp, vp]),
        "b2g_level_colouring": (ip, [vp, ip, C.POINTER(C.c_int), vp]),
        "b2g_fold_boundary": (ip, [ip, ip, vp, vp, vp, vp, vp, vp, ip, vp]),
        "b2g_level_sweep_shape": (ip, [vp, ip, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)]),
        "b2g_level_mc_pipe": (ip, [vp, ip, ip, ip, C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "b2g_precondition": (ip, [vp, C.POINTER(Controls), vp, vp, C.POINTER(_Log)]),
        "b2g_matrix_pcg_solve": (ip, [vp, vp, vp, C.POINTER(Controls), ip, C.POINTER(_Perf),
                                      C.POINTER(_Log)]),
        "b2g_matrix_timings": (ip, [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
        "b2g_matrix_level_timings": (ip, [vp, ip, ip, vp, vp, vp, C.POINTER(C.c_int)]),
        "b2g_level_smooth_trace": (ip, [vp, ip, vp, vp, vp, ip, C.POINTER(C.c_int)]),
        "b2g_level_smooth_stall": (ip, [vp, ip, vp, vp, C.c_longlong, C.POINTER(C.c_int)]),
        "b2g_batch_create": (ip, [C.POINTER(vp), ip, C.POINTER(vp)]),
        "b2g_batch_solve": (ip, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(Controls), ip, C.POINTER(_Perf)]),
        "b2g_batch_launches": (ip, [vp, C.POINTER(C.c_longlong)]),
        "b2g_batch_destroy": (ip, [vp]),
        "b2g_server_create": (ip, [C.c_ulonglong, ip, C.POINTER(vp)]),
        "b2g_server_destroy": (ip, [vp]),
        "b2g_server_add_case": (ip, [vp, ip, ip, vp, vp, vp, vp, vp, vp, ip, ip, C.POINTER(C.c_int)]),
        "b2g_server_submit": (ip, [vp, ip, vp, vp, C.POINTER(Controls), C.POINTER(C.c_longlong)]),
        "b2g_server_wait": (ip, [vp, C.c_longlong, C.POINTER(_Perf), C.POINTER(C.c_double), ip]),
        "b2g_server_case_bytes": (ip, [vp, ip, C.POINTER(C.c_ulonglong)]),
        "b2g_mesh_set_pair": (ip, [vp, ip, vp, vp, ip, vp]),
        "b2g_mesh_level_pair": (ip, [vp, ip, C.POINTER(C.c_int), vp, vp]),
        "b2g_gamg_solve_coupled": (ip, [vp, vp, vp, vp, vp, vp, C.POINTER(Controls), ip, vp, C.POINTER(_Perf),
                                        C.POINTER(_Log)]),
        "b2g_matrix_create_coupled": (ip, [vp, vp, vp, vp, ip, vp, C.POINTER(vp)]),
        "b2g_matrix_level_pair_coeffs": (ip, [vp, ip, vp]),
        "b2g_matrix_gamg_solve": (ip, [vp, vp, vp, C.POINTER(Controls), ip, C.POINTER(_Perf), C.POINTER(_Log)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


lib = _load()
EXPORTED = [
    "b2g_last_error", "b2g_version", "b2g_set_profiling", "b2g_controls_default",
    "b2g_controls_read", "b2g_mesh_create", "b2g_mesh_create_cached", "b2g_mesh_destroy", "b2g_mesh_levels",
    "b2g_mesh_level_size", "b2g_mesh_get_step", "b2g_mesh_build_ms", "b2g_pcg_gamg_solve",
    "b2g_gamg_solve", "b2g_matrix_create", "b2g_matrix_destroy", "b2g_matrix_get_level",
    "b2g_level_amul", "b2g_level_smooth", "b2g_level_scale", "b2g_step_restrict",
    "b2g_step_prolong", "b2g_level_norm_factor", "b2g_level_pcg_dic", "b2g_precondition",
    "b2g_matrix_pcg_solve", "b2g_matrix_timings", "b2g_level_smooth_trace", "b2g_level_pcg_dic_static",
    "b2g_level_schedule", "b2g_level_colouring", "b2g_fold_boundary", "b2g_level_sweep_shape", "b2g_level_mc_pipe", "b2g_server_create", "b2g_server_destroy", "b2g_server_add_case",
    "b2g_server_submit", "b2g_server_wait", "b2g_server_case_bytes", "b2g_batch_create", "b2g_batch_solve",
    "b2g_batch_launches", "b2g_batch_destroy", "b2g_mesh_set_pair", "b2g_mesh_level_pair",
    "b2g_gamg_solve_coupled", "b2g_matrix_create_coupled", "b2g_matrix_level_pair_coeffs", "b2g_matrix_gamg_solve",
    "b2g_matrix_set_coeffs", "b2g_matrix_level_timings", "b2g_level_smooth_stall", "b2g_set_sweep_pipeline",
    "b2g_level_smooth_pipelined", "b2g_level_grid_stall", "b2g_set_part_cells", "b2g_level_pipe_shape", "b2g_coarsest_dense_solve", "b2g_assemble_pressure",
]


def _check(rc: int):
    if rc != 0:
        raise GamgError(rc, lib.b2g_last_error().decode())


def controls_default(**overrides) -> Controls:
    c = Controls()
    _check(lib.b2g_controls_default(C.byref(c)))
    for k, v in overrides.items():
        if k == "smoother" and isinstance(v, str):
            v = SMOOTHERS[v]
        if k == "precision" and isinstance(v, str):
            v = {"fp64": 0, "fp32_precond": 1, "fp32_precond_multicolour": 2}[v]
        if k == "reduction" and isinstance(v, str):
            v = {"tree": 0, "serial": 1}[v]
        if k == "solver" and isinstance(v, str):
            v = {"PCG": 0, "GAMG": 1}[v]
        setattr(c, k, v)
    return c


def read_controls(entry_text: str) -> Controls:
    """Reads an fvSolution solver entry (readGamgControls with the reference's refusals)."""
    c = Controls()
    _check(lib.b2g_controls_read(entry_text.encode(), C.byref(c)))
    return c


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x):
    if x is None:
        return None
    if _is_torch(x):
        return C.c_void_p(x.data_ptr())
    return C.c_void_p(x.ctypes.data)


def _memspace(*arrays) -> int:
    dev = [_is_torch(a) and a.is_cuda for a in arrays if a is not None]
    if all(dev):
        return B2G_MEM_DEVICE
    if not any(dev):
        return B2G_MEM_HOST
    raise ValueError("arrays must be all host (numpy) or all CUDA tensors")


def _stream():
    try:
        import torch
        if torch.cuda.is_available():
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    except ImportError:
        pass
    return None


def _as_host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Mesh:
    """The mesh's GAMG hierarchy (GamgAgglomerationCache): built once, on the device."""

    def __init__(self, lower, upper, Sf, magSf, n_cells: int, n_coarsest: int = 10,
                 forward: bool = True, cache_path: str | None = None):
        if not _is_torch(lower):
            lower = _as_host(lower, np.int32)
            upper = _as_host(upper, np.int32)
            Sf = _as_host(Sf, np.float64).reshape(-1)
            magSf = _as_host(magSf, np.float64)
        ms = _memspace(lower, upper, Sf, magSf)
        fw = C.c_int(1 if forward else 0)
        h = C.c_void_p()
        nF = int(lower.shape[0])
        self.from_cache = False
        if cache_path is None:
            _check(lib.b2g_mesh_create(int(n_cells), nF, _ptr(lower), _ptr(upper), _ptr(Sf),
                                       _ptr(magSf), int(n_coarsest), C.byref(fw), ms, _stream(),
                                       C.byref(h)))
        else:
            hit = C.c_int(0)
            _check(lib.b2g_mesh_create_cached(int(n_cells), nF, _ptr(lower), _ptr(upper), _ptr(Sf),
                                              _ptr(magSf), int(n_coarsest), C.byref(fw), ms, _stream(),
                                              str(cache_path).encode(), C.byref(h), C.byref(hit)))
            self.from_cache = bool(hit.value)
        self.handle = h
        self.forward = bool(fw.value)
        self.n_cells = int(n_cells)
        self.n_faces = nF

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and lib is not None:
            lib.b2g_mesh_destroy(h)
            self.handle = None

    @property
    def n_levels(self) -> int:
        n = C.c_int()
        _check(lib.b2g_mesh_levels(self.handle, C.byref(n)))
        return n.value

    def level_size(self, level: int):
        nc, nf = C.c_int(), C.c_int()
        _check(lib.b2g_mesh_level_size(self.handle, level, C.byref(nc), C.byref(nf)))
        return nc.value, nf.value

    @property
    def build_ms(self) -> float:
        v = C.c_float()
        _check(lib.b2g_mesh_build_ms(self.handle, C.byref(v)))
        return v.value

    def schedule(self, level: int, n_parts: int, n_chunks: int):
        """The Gauss-Seidel schedule of a level (diagnostic): (partChunkStart, chunk records [n, 12])."""
        pcs = np.empty(n_parts + 1, np.int32)
        rec = np.empty((n_chunks, 12), np.int32)
        _check(lib.b2g_level_schedule(self.handle, level, pcs.ctypes.data_as(C.c_void_p), rec.ctypes.data_as(C.c_void_p)))
        return pcs, rec

    def colouring(self, level: int):
        """The level's multicolour row ranges (empty before the multicolour form's first solve)."""
        n = C.c_int()
        _check(lib.b2g_level_colouring(self.handle, level, C.byref(n), None))
        starts = np.zeros(n.value + 1, np.int32)
        _check(lib.b2g_level_colouring(self.handle, level, C.byref(n), _ptr(starts)))
        return starts

    def mc_pipe(self, level: int, n_sweeps: int, symmetric: bool = False) -> dict:
        """Whether `level`'s multicolour smoothing calls of n_sweeps sweeps run as one pipelined launch
        over the colours (b2g_level_mc_pipe): its CTAs (0: colour by colour) and both measured times."""
        r, mp, mc = C.c_int(), C.c_float(), C.c_float()
        _check(lib.b2g_level_mc_pipe(self.handle, level, n_sweeps, 1 if symmetric else 0, C.byref(r), C.byref(mp),
                                     C.byref(mc)))
        return {"ranks": r.value, "ms_pipelined": mp.value, "ms_colours": mc.value}

    def sweep_shape(self, level: int) -> dict:
        """The autotuner's multicolour sweep shape for `level` (zeros before the form's first solve):
        one block for the whole level, one cluster of `cluster_ctas` CTAs, or one launch per colour."""
        whole, thr, ms = C.c_int(), C.c_int(), C.c_float()
        _check(lib.b2g_level_sweep_shape(self.handle, level, C.byref(whole), C.byref(thr), C.byref(ms)))
        return {"one_block": whole.value == 1, "cluster_ctas": whole.value if whole.value > 1 else 0,
                "threads": thr.value, "ms_per_sweep": ms.value}

    def pipe_shape(self, level: int, n_sweeps: int, value_bytes: int = 8) -> dict:
        """The tuned choice for `level`'s smoothing calls of n_sweeps sweeps (b2g_level_pipe_shape)."""
        r, st, mp, ms, msh, mit = C.c_int(), C.c_int(), C.c_float(), C.c_float(), C.c_float(), C.c_float()
        mg, gf = C.c_float(), C.c_int()
        _check(lib.b2g_level_pipe_shape(self.handle, level, n_sweeps, value_bytes, C.byref(r), C.byref(st),
                                        C.byref(mp), C.byref(ms), C.byref(msh), C.byref(mit), C.byref(mg),
                                        C.byref(gf)))
        return {"ranks": r.value, "steps": st.value, "ms_pipelined": mp.value, "ms_sweep_by_sweep": ms.value,
                "ms_shared_memory": msh.value, "ms_items": mit.value, "ms_grid": mg.value, "grid": bool(gf.value)}

    def set_pair(self, own, nbr) -> None:
        """The coupled (cyclic) pair: faceCells and neighbour cells of the coupled patches' faces, each
        face once from its own side (b2g_mesh_set_pair); every coarse level's is built from it."""
        o = np.ascontiguousarray(own, np.int32)
        n = np.ascontiguousarray(nbr, np.int32)
        _check(lib.b2g_mesh_set_pair(self.handle, int(o.shape[0]), _ptr(o), _ptr(n), B2G_MEM_HOST, None))

    def level_pair(self, level: int):
        """Level `level`'s pair as (own, nbr) cell arrays of that level."""
        m = C.c_int()
        _check(lib.b2g_mesh_level_pair(self.handle, level, C.byref(m), None, None))
        o = np.empty(m.value, np.int32)
        n = np.empty(m.value, np.int32)
        _check(lib.b2g_mesh_level_pair(self.handle, level, C.byref(m), _ptr(o), _ptr(n)))
        return o, n

    def step(self, i: int) -> dict:
        nc, nf = self.level_size(i)
        cc, cf = self.level_size(i + 1)
        r = np.empty(nc, np.int32)
        fr = np.empty(nf, np.int32)
        fl = np.empty(nf, np.int8)
        lo = np.empty(cf, np.int32)
        up = np.empty(cf, np.int32)
        _check(lib.b2g_mesh_get_step(self.handle, i, _ptr(r), _ptr(fr), _ptr(fl), _ptr(lo),
                                     _ptr(up)))
        return dict(restrict=r, face_restrict=fr, flip=fl, lower=lo, upper=up)


class _LogBuf:
    def __init__(self, history_cap: int, coarsest_cap: int):
        self.hist = (C.c_double * max(history_cap, 1))()
        self.coarse = (_Perf * max(coarsest_cap, 1))()
        self.log = _Log(C.cast(self.hist, C.POINTER(C.c_double)), history_cap, 0,
                        C.cast(self.coarse, C.POINTER(_Perf)), coarsest_cap, 0)

    def history(self):
        return [self.hist[i] for i in range(min(self.log.historyCount, self.log.historyCapacity))]

    def coarsest(self):
        n = min(self.log.coarsestCount, self.log.coarsestCapacity)
        return [(self.coarse[i].initialResidual, self.coarse[i].finalResidual,
                 self.coarse[i].nIterations) for i in range(n)]


class Matrix:
    """One folded matrix on a mesh's hierarchy (GamgHierarchy): Galerkin levels on the device."""

    def __init__(self, mesh: Mesh, diag, upper, pair_coeffs=None):
        if not _is_torch(diag):
            diag = _as_host(diag, np.float64)
            upper = _as_host(upper, np.float64)
            if pair_coeffs is not None:
                pair_coeffs = _as_host(pair_coeffs, np.float64)
        ms = _memspace(diag, upper, pair_coeffs)
        h = C.c_void_p()
        if pair_coeffs is None:
            _check(lib.b2g_matrix_create(mesh.handle, _ptr(diag), _ptr(upper), ms, _stream(), C.byref(h)))
        else:
            _check(lib.b2g_matrix_create_coupled(mesh.handle, _ptr(diag), _ptr(upper), _ptr(pair_coeffs), ms,
                                                 _stream(), C.byref(h)))
        self.handle = h
        self.mesh = mesh

    def set_coeffs(self, diag, upper):
        """New fine-level coefficients on the same mesh; every coarse level is rebuilt in place."""
        if not _is_torch(diag):
            diag = _as_host(diag, np.float64)
            upper = _as_host(upper, np.float64)
        _check(lib.b2g_matrix_set_coeffs(self.handle, _ptr(diag), _ptr(upper), _memspace(diag, upper)))

    def pair_coeffs(self, level: int):
        m = len(self.mesh.level_pair(level)[0])
        c = np.empty(m)
        _check(lib.b2g_matrix_level_pair_coeffs(self.handle, level, _ptr(c)))
        return c

    def gamg_solve(self, source, psi, controls: Controls, history_cap=100000):
        """The standalone GAMG solve on this matrix (b2g_matrix_gamg_solve)."""
        ms = _memspace(source, psi)
        p = _Perf()
        lb = _LogBuf(history_cap, 0)
        _check(lib.b2g_matrix_gamg_solve(self.handle, _ptr(source), _ptr(psi), C.byref(controls), ms, C.byref(p),
                                         C.byref(lb.log)))
        return SolverPerformance(p.initialResidual, p.finalResidual, p.nIterations), lb.history()

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and lib is not None:
            lib.b2g_matrix_destroy(h)
            self.handle = None

    def level(self, level: int):
        nc, nf = self.mesh.level_size(level)
        d = np.empty(nc)
        u = np.empty(nf)
        _check(lib.b2g_matrix_get_level(self.handle, level, _ptr(d), _ptr(u)))
        return d, u

    # device pointers only below (CUDA tensors)
    def amul(self, level, x, y):
        _check(lib.b2g_level_amul(self.handle, level, _ptr(x), _ptr(y)))

    def smooth(self, level, psi, source, n_sweeps, smoother="GaussSeidel"):
        _check(lib.b2g_level_smooth(self.handle, level, SMOOTHERS[smoother], _ptr(psi),
                                    _ptr(source), n_sweeps))

    def smooth_trace(self, level, psi, source, trace=None):
        """One sweep with per-chunk device-clock stamps; returns (schedule, trace tensor)."""
        sched = (C.c_int * 5)()
        _check(lib.b2g_level_smooth_trace(self.handle, level, _ptr(psi), _ptr(source), None, 0, sched))
        info = dict(parts=sched[0], chunks=sched[1], cells=sched[2], entries=sched[3], depth=sched[4])
        if trace is not None:
            _check(lib.b2g_level_smooth_trace(self.handle, level, _ptr(psi), _ptr(source), _ptr(trace),
                                              int(trace.numel()), sched))
        return info

    def smooth_pipelined(self, level, psi, source, n_sweeps, ranks):
        """n_sweeps sweeps in one pipelined launch on `ranks` CTAs (b2g_level_smooth_pipelined)."""
        _check(lib.b2g_level_smooth_pipelined(self.handle, level, _ptr(psi), _ptr(source), n_sweeps, ranks))

    def grid_stall(self, level, psi, source, n_sweeps, ranks, spin_limit):
        """The grid form with no rank publishing its progress (b2g_level_grid_stall): the status name."""
        rc = lib.b2g_level_grid_stall(self.handle, level, _ptr(psi), _ptr(source), n_sweeps, ranks, int(spin_limit))
        return STATUS.get(rc, str(rc))

    def coarsest_dense_solve(self, psi, source):
        """psi = A^-1 source on the coarsest level by its dense Cholesky factor."""
        _check(lib.b2g_coarsest_dense_solve(self.handle, _ptr(psi), _ptr(source)))

    def smooth_stall(self, level, psi, source, spin_limit):
        """One sweep in which no part publishes its progress, waits limited to `spin_limit` polls
        (b2g_level_smooth_stall): returns (status name, the level's part count)."""
        parts = C.c_int()
        rc = lib.b2g_level_smooth_stall(self.handle, level, _ptr(psi), _ptr(source), int(spin_limit),
                                        C.byref(parts))
        return STATUS.get(rc, str(rc)), parts.value

    def scale(self, level, field, Acf, source):
        _check(lib.b2g_level_scale(self.handle, level, _ptr(field), _ptr(Acf), _ptr(source)))

    def restrict(self, step, fine, coarse):
        _check(lib.b2g_step_restrict(self.handle, step, _ptr(fine), _ptr(coarse)))

    def prolong(self, step, coarse, fine):
        _check(lib.b2g_step_prolong(self.handle, step, _ptr(coarse), _ptr(fine)))

    def norm_factor(self, level, psi, source, Apsi) -> float:
        v = C.c_double()
        _check(lib.b2g_level_norm_factor(self.handle, level, _ptr(psi), _ptr(source), _ptr(Apsi),
                                         C.byref(v)))
        return v.value

    def pcg_dic(self, level, psi, source, tol, rel_tol) -> SolverPerformance:
        p = _Perf()
        _check(lib.b2g_level_pcg_dic(self.handle, level, _ptr(psi), _ptr(source), tol, rel_tol,
                                     C.byref(p)))
        return SolverPerformance(p.initialResidual, p.finalResidual, p.nIterations)

    def precondition(self, controls: Controls, w, r, coarsest_cap: int = 0):
        lb = _LogBuf(0, coarsest_cap)
        _check(lib.b2g_precondition(self.handle, C.byref(controls), _ptr(w), _ptr(r),
                                    C.byref(lb.log)))
        return lb.coarsest()

    def solve(self, source, psi, controls: Controls, history_cap=1000, coarsest_cap=0):
        ms = _memspace(source, psi)
        p = _Perf()
        lb = _LogBuf(history_cap, coarsest_cap)
        _check(lib.b2g_matrix_pcg_solve(self.handle, _ptr(source), _ptr(psi), C.byref(controls),
                                        ms, C.byref(p), C.byref(lb.log)))
        return (SolverPerformance(p.initialResidual, p.finalResidual, p.nIterations),
                lb.history(), lb.coarsest())

    def timings(self):
        """(ms, counts) of the last solve: [finest Amuls, finest smoothing (count: sweeps), other
        (count: launches), whole solve (count: all launches)]."""
        ms = (C.c_double * 4)()
        n = (C.c_longlong * 4)()
        _check(lib.b2g_matrix_timings(self.handle, ms, n))
        return list(ms), list(n)

    def level_timings(self, kind: int):
        """Per level of the last profiled solve, kind 0 (Amul), 1 (smoothing) or 2 (Amul fused with the
        residual, the scaling or the prolongation): a list of (ms, timed regions, units) -- units are
        Amuls, or the sweeps of the smoothing calls."""
        cap = self.mesh.n_levels + 1
        ms = (C.c_double * cap)()
        reg = (C.c_longlong * cap)()
        un = (C.c_longlong * cap)()
        have = C.c_int()
        _check(lib.b2g_matrix_level_timings(self.handle, kind, cap, ms, reg, un, C.byref(have)))
        return [(ms[i], reg[i], un[i]) for i in range(min(have.value, cap))]


def set_part_cells(cells: int) -> None:
    """The multi-part sweep's part rule for meshes created from now on (b2g_set_part_cells)."""
    _check(lib.b2g_set_part_cells(int(cells)))


def set_profiling(on: bool) -> None:
    _check(lib.b2g_set_profiling(1 if on else 0))


def set_sweep_pipeline(on: bool) -> None:
    """Whether smoothing calls may run their sweeps in one pipelined launch (the default)."""
    _check(lib.b2g_set_sweep_pipeline(1 if on else 0))


def pcg_gamg_solve(mesh: Mesh, diag, upper, source, psi, controls: Controls | None = None,
                   history_cap: int = 1000, coarsest_cap: int = 0):
    """pcgGamgSolve (src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cuh:217-229) on a folded
    system. ``psi`` is updated in place (numpy or CUDA tensor). Returns (SolverPerformance,
    residual history, coarsest-level performances)."""
    controls = controls or controls_default()
    if not _is_torch(diag):
        diag = _as_host(diag, np.float64)
        upper = _as_host(upper, np.float64)
        source = _as_host(source, np.float64)
    ms = _memspace(diag, upper, source, psi)
    p = _Perf()
    lb = _LogBuf(history_cap, coarsest_cap)
    _check(lib.b2g_pcg_gamg_solve(mesh.handle, _ptr(diag), _ptr(upper), _ptr(source), _ptr(psi),
                                  C.byref(controls), ms, _stream(), C.byref(p), C.byref(lb.log)))
    return (SolverPerformance(p.initialResidual, p.finalResidual, p.nIterations), lb.history(),
            lb.coarsest())


def assemble_pressure(mesh: Mesh, system: dict, p_ref_cell: int = -1, p_ref_value: float = 0.0) -> dict:
    """simpleFoam's pressure equation ahead of the solve on the device (b2g_assemble_pressure). `system`
    holds numpy arrays (host) or CUDA tensors: weights, deltaCoeffs, magSf, phi per internal face; V, rAU
    per cell; bFaceCells, bMagSf, bDeltaCoeffs, bType, bValue, bPhi per boundary face. Returns diag,
    coef, source, internalCoeffs, boundaryCoeffs in the same memory."""
    keys = ("weights", "deltaCoeffs", "magSf", "V", "rAU", "phi", "bFaceCells", "bMagSf", "bDeltaCoeffs", "bType",
            "bValue", "bPhi")
    arr = {}
    for k in keys:
        a = system[k]
        if not _is_torch(a):
            a = np.ascontiguousarray(a, np.int32 if k in ("bFaceCells", "bType") else np.float64)
        arr[k] = a
    ms = _memspace(*arr.values())
    nC, nF, nB = mesh.n_cells, mesh.n_faces, int(arr["bFaceCells"].shape[0])
    if ms == B2G_MEM_HOST:
        out = {k: np.zeros(n) for k, n in (("diag", nC), ("coef", nF), ("source", nC), ("internalCoeffs", nB),
                                            ("boundaryCoeffs", nB))}
    else:
        import torch
        dev = arr["V"].device
        out = {k: torch.zeros(n, dtype=torch.float64, device=dev) for k, n in (
            ("diag", nC), ("coef", nF), ("source", nC), ("internalCoeffs", nB), ("boundaryCoeffs", nB))}
    _check(lib.b2g_assemble_pressure(mesh.handle, *[_ptr(arr[k]) for k in keys[:6]], nB,
                                     *[_ptr(arr[k]) for k in keys[6:]], int(p_ref_cell), float(p_ref_value),
                                     _ptr(out["diag"]), _ptr(out["coef"]), _ptr(out["source"]),
                                     _ptr(out["internalCoeffs"]), _ptr(out["boundaryCoeffs"]), ms, _stream()))
    return out


def gamg_solve(mesh: Mesh, diag, upper, source, psi, controls: Controls,
               history_cap: int = 100000):
    """gamgSolveFolded (gamg_solver_cpp.cuh:185-192): the standalone GAMG solver."""
    if not _is_torch(diag):
        diag = _as_host(diag, np.float64)
        upper = _as_host(upper, np.float64)
        source = _as_host(source, np.float64)
    ms = _memspace(diag, upper, source, psi)
    p = _Perf()
    lb = _LogBuf(history_cap, 0)
    _check(lib.b2g_gamg_solve(mesh.handle, _ptr(diag), _ptr(upper), _ptr(source), _ptr(psi),
                              C.byref(controls), ms, _stream(), C.byref(p), C.byref(lb.log)))
    return SolverPerformance(p.initialResidual, p.finalResidual, p.nIterations), lb.history()


def gamg_solve_coupled(mesh: Mesh, diag, upper, pair_coeffs, source, psi, controls: Controls,
                       history_cap: int = 100000):
    """gamgSolve with coupled patches (gamg_solver_cpp.cuh:174-181) on a folded system: the mesh's
    pair (Mesh.set_pair) with these coefficients, in the sign convention Amul subtracts."""
    if not _is_torch(diag):
        diag = _as_host(diag, np.float64)
        upper = _as_host(upper, np.float64)
        pair_coeffs = _as_host(pair_coeffs, np.float64)
        source = _as_host(source, np.float64)
    ms = _memspace(diag, upper, pair_coeffs, source, psi)
    p = _Perf()
    lb = _LogBuf(history_cap, 0)
    _check(lib.b2g_gamg_solve_coupled(mesh.handle, _ptr(diag), _ptr(upper), _ptr(pair_coeffs), _ptr(source),
                                      _ptr(psi), C.byref(controls), ms, _stream(), C.byref(p), C.byref(lb.log)))
    return SolverPerformance(p.initialResidual, p.finalResidual, p.nIterations), lb.history()


def fold_boundary(diag, source, face_cells, internal_coeffs, boundary_coeffs, coupled):
    """foldBoundary (gamg_solver_cpp.cu:769-797) on the device: returns the folded (diag, source).
    The boundary arrays are all patches' faces concatenated in patch order; `coupled` per face."""
    d = np.array(diag, dtype=np.float64, copy=True)
    s = np.array(source, dtype=np.float64, copy=True)
    fc = np.ascontiguousarray(face_cells, np.int32)
    ic = np.ascontiguousarray(internal_coeffs, np.float64)
    bc = np.ascontiguousarray(boundary_coeffs, np.float64)
    cp = np.ascontiguousarray(coupled, np.uint8)
    _check(lib.b2g_fold_boundary(d.shape[0], fc.shape[0], _ptr(fc), _ptr(ic), _ptr(bc), _ptr(cp), _ptr(d), _ptr(s),
                                 B2G_MEM_HOST, None))
    return d, s


class Server:
    """The serving form (b2g_server_*): cases registered once and kept resident, solves queued as
    they arrive and run on `slots` worker streams side by side. Host arrays in and out."""

    def __init__(self, hbm_cap_bytes: int, slots: int = 4):
        h = C.c_void_p()
        _check(lib.b2g_server_create(int(hbm_cap_bytes), int(slots), C.byref(h)))
        self.handle = h
        self.n_cells = {}
        self._pending = {}

    def add_case(self, lower, upper, Sf, magSf, n_cells, diag, coef, n_coarsest=10) -> int:
        lower = np.ascontiguousarray(lower, np.int32)
        upper = np.ascontiguousarray(upper, np.int32)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (np.asarray(Sf).reshape(-1), magSf, diag, coef)]
        cid = C.c_int()
        _check(lib.b2g_server_add_case(self.handle, int(n_cells), int(lower.shape[0]), _ptr(lower), _ptr(upper),
                                       _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(arrs[3]),
                                       int(n_coarsest), B2G_MEM_HOST, C.byref(cid)))
        self.n_cells[cid.value] = int(n_cells)
        return cid.value

    def submit(self, case_id: int, source, controls: Controls, psi0=None, out=None) -> int:
        """Queues a solve. The server reads `source` and solves into `out` (a float64 array of the
        case's size; a new one if None) in place, starting from psi0 (zero if None). Both arrays
        are held here until wait() hands the solution back."""
        n = self.n_cells[case_id]
        src = np.ascontiguousarray(source, np.float64)
        if out is None:
            out = np.zeros(n, np.float64)
        if psi0 is not None:
            out[:] = psi0
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.shape != (n,) or src.shape != (n,):
            raise ValueError("submit: source and out must be float64 arrays of the case's size")
        t = C.c_longlong()
        _check(lib.b2g_server_submit(self.handle, int(case_id), _ptr(src), _ptr(out), C.byref(controls),
                                     C.byref(t)))
        self._pending[t.value] = (src, out)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(psi, SolverPerformance, latency ms) of a submitted solve."""
        perf = _Perf()
        lat = C.c_double()
        rc = lib.b2g_server_wait(self.handle, int(ticket), C.byref(perf), C.byref(lat), int(timeout_ms))
        if rc != 0:
            msg = lib.b2g_last_error().decode()
            if "still pending" not in msg:  # a pending request keeps its buffers held
                self._pending.pop(ticket, None)
            raise GamgError(rc, msg)
        _, psi = self._pending.pop(ticket)
        return psi, SolverPerformance(perf.initialResidual, perf.finalResidual, perf.nIterations), lat.value

    def case_bytes(self, case_id: int) -> int:
        v = C.c_ulonglong()
        _check(lib.b2g_server_case_bytes(self.handle, int(case_id), C.byref(v)))
        return v.value

    def close(self):
        if self.handle is not None and lib is not None:
            _check(lib.b2g_server_destroy(self.handle))
        self.handle = None
        self._pending.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """The batched form (b2g_batch_*): many matrices, each on its own mesh, solved together with every
    level step one launch over all cases. The matrices are kept alive as long as the batch."""

    def __init__(self, matrices):
        self.matrices = list(matrices)
        arr = (C.c_void_p * len(self.matrices))(*[m.handle.value for m in self.matrices])
        h = C.c_void_p()
        _check(lib.b2g_batch_create(arr, len(self.matrices), C.byref(h)))
        self.handle = h

    def solve(self, sources, psis, controls: Controls):
        """Solves every case: sources[k], psis[k] (numpy arrays or CUDA tensors, all of one kind, natural
        cell order); psis are overwritten. Returns the list of SolverPerformance."""
        K = len(self.matrices)
        if len(sources) != K or len(psis) != K:
            raise ValueError("one source and one psi per case")
        hold = []
        src_p = (C.c_void_p * K)()
        psi_p = (C.c_void_p * K)()
        for k in range(K):
            s, x = sources[k], psis[k]
            if not _is_torch(s):
                s = _as_host(s, np.float64)
                hold.append(s)
            src_p[k] = _ptr(s)
            psi_p[k] = _ptr(x)
        ms = _memspace(*sources, *psis)
        perfs = (_Perf * K)()
        _check(lib.b2g_batch_solve(self.handle, src_p, psi_p, C.byref(controls), ms, perfs))
        return [SolverPerformance(p.initialResidual, p.finalResidual, p.nIterations) for p in perfs]

    def launches(self) -> int:
        v = C.c_longlong()
        _check(lib.b2g_batch_launches(self.handle, C.byref(v)))
        return v.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and lib is not None:
            lib.b2g_batch_destroy(h)
            self.handle = None
