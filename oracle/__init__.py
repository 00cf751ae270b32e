"""ctypes loader for the oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a CPU restatement of the reference CG ``cg_3d_mpi``
(src/mod_solver_3d.f90:485-620); see eaf_oracle.c for the line-by-line
mapping. Only tests, the smoke check and the CPU-baseline legs of bench.py
use it, always as the checker or the timed CPU reference, never as the
product path. Parity is unpinned at the CG boundary: no reference binary or
reference CG golden vector exists to pin it against.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libeaforacle.so")

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        ci, cd = ctypes.c_int, ctypes.c_double
        L.eaf_oracle_cg.argtypes = [ci, ci, ci] + [_dp] * 9 + [ci, cd, _dp,
                                                               ctypes.POINTER(ci)]
        L.eaf_oracle_cg.restype = ci
        L.eaf_oracle_cg_threads.argtypes = (L.eaf_oracle_cg.argtypes + [ci])
        L.eaf_oracle_cg_threads.restype = ci
        L.eaf_oracle_cg_tree.argtypes = (L.eaf_oracle_cg.argtypes + [ci, ci])
        L.eaf_oracle_cg_tree.restype = ci
        L.eaf_oracle_cg_cluster.argtypes = (L.eaf_oracle_cg.argtypes + [ci, ci, ci])
        L.eaf_oracle_cg_cluster.restype = ci
        L.eaf_oracle_cg1.argtypes = (L.eaf_oracle_cg.argtypes + [ci, ci])
        L.eaf_oracle_cg1.restype = ci
        L.eaf_oracle_dot.argtypes = [ci, ci, ci, _dp, _dp, ci, ci]
        L.eaf_oracle_dot.restype = cd
        L.eaf_oracle_dot_cluster.argtypes = [ci, ci, ci, _dp, _dp, ci, ci, ci]
        L.eaf_oracle_dot_cluster.restype = cd
        L.eaf_oracle_matvec.argtypes = [ci, ci, ci] + [_dp] * 9
        L.eaf_oracle_matvec.restype = None
        L.eaf_oracle_theta_wrap.argtypes = [ci, ci, ci, _dp]
        L.eaf_oracle_theta_wrap.restype = None
        L.eaf_oracle_tdma_3d.argtypes = [ci, ci, ci] + [_dp] * 9 + [ci]
        L.eaf_oracle_tdma_3d.restype = ci
        L.eaf_oracle_residual_3d.argtypes = [ci, ci, ci] + [_dp] * 9 + [ci, ci]
        L.eaf_oracle_residual_3d.restype = cd
        L.eaf_oracle_pressure_correct.argtypes = [ci, ci, ci, ctypes.POINTER(_dp),
                                                  ctypes.POINTER(ctypes.POINTER(ci)),
                                                  ci, cd]
        L.eaf_oracle_pressure_correct.restype = ci
        L.eaf_oracle_pressure_assemble.argtypes = [ci, ci, ci, ctypes.POINTER(_dp),
                                                   ctypes.POINTER(ctypes.POINTER(ci)),
                                                   ci, _dp, _dp]
        L.eaf_oracle_pressure_assemble.restype = ci
        L.eaf_oracle_max_threads.argtypes = []
        L.eaf_oracle_max_threads.restype = ci
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def cg(system, phi: np.ndarray, max_iter: int, tol: float, nthreads: int = 1,
       plan: tuple | None = None):
    """Solve in place on ``phi`` (halo layout). Returns (residual, n_iter).

    ``plan=(G, B)`` associates the dot products as the CUDA kernels do for a
    launch of G blocks x B threads (everything else is unchanged);
    ``plan=(G, B, C)`` as the kernels do on a grid of thread-block clusters
    of C blocks. The default is the reference's sequential sum.
    """
    res = ctypes.c_double(0.0)
    nit = ctypes.c_int(0)
    args = [system.nr, system.nth, system.nz] + [_p(a) for a in system.arrays()]
    args += [_p(phi), int(max_iter), float(tol), ctypes.byref(res),
             ctypes.byref(nit)]
    if plan is not None and len(plan) > 2 and int(plan[2]) > 1:
        rc = lib().eaf_oracle_cg_cluster(*args, int(plan[0]), int(plan[1]), int(plan[2]))
    elif plan is not None:
        rc = lib().eaf_oracle_cg_tree(*args, int(plan[0]), int(plan[1]))
    elif nthreads == 1:
        rc = lib().eaf_oracle_cg(*args)
    else:
        rc = lib().eaf_oracle_cg_threads(*args, int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle cg failed with status {rc}")
    return res.value, nit.value


def cg1(system, phi: np.ndarray, max_iter: int, tol: float, plan: tuple | None = None):
    """The single-reduction (Chronopoulos-Gear) form of the same PCG, in
    place on ``phi``; ``plan=(G, B)`` associates its dots as the CUDA
    single-reduction kernel does. Returns (residual, n_iter)."""
    res = ctypes.c_double(0.0)
    nit = ctypes.c_int(0)
    G, B = plan if plan is not None else (0, 0)
    args = [system.nr, system.nth, system.nz] + [_p(a) for a in system.arrays()]
    args += [_p(phi), int(max_iter), float(tol), ctypes.byref(res), ctypes.byref(nit),
             int(G), int(B)]
    rc = lib().eaf_oracle_cg1(*args)
    if rc != 0:
        raise RuntimeError(f"oracle cg1 failed with status {rc}")
    return res.value, nit.value


def matvec(system, x: np.ndarray) -> np.ndarray:
    """Reference matvec: refreshes x's theta halos in place, returns y."""
    y = np.zeros_like(x)
    args = [system.nr, system.nth, system.nz] + [_p(a) for a in system.arrays()[:7]]
    lib().eaf_oracle_matvec(*args, _p(x), _p(y))
    return y


def dot(nr: int, nth: int, nz: int, a: np.ndarray, b: np.ndarray,
        plan: tuple | None = None) -> float:
    """Interior dot in the association of ``plan`` ((G, B) or (G, B, C));
    the reference's sequential sum without one."""
    if plan is not None and len(plan) > 2 and int(plan[2]) > 1:
        G, B, C = plan
        return lib().eaf_oracle_dot_cluster(nr, nth, nz, _p(a), _p(b), int(G), int(B),
                                            int(C))
    G, B = plan[:2] if plan is not None else (0, 0)
    return lib().eaf_oracle_dot(nr, nth, nz, _p(a), _p(b), int(G), int(B))


def theta_wrap(nr: int, nth: int, nz: int, x: np.ndarray) -> None:
    lib().eaf_oracle_theta_wrap(nr, nth, nz, _p(x))


def tdma_3d(system, phi: np.ndarray, n_sweep: int) -> None:
    """Serial tdma_3d_mpi (src/mod_solver_3d.f90:252-366) in place on phi."""
    args = [system.nr, system.nth, system.nz] + [_p(a) for a in system.arrays()]
    rc = lib().eaf_oracle_tdma_3d(*args, _p(phi), int(n_sweep))
    if rc != 0:
        raise RuntimeError(f"oracle tdma failed with status {rc}")


def residual_3d(system, phi: np.ndarray, plan: tuple | None = None) -> float:
    """compute_residual_3d_mpi (src/mod_solver_3d.f90:625-694), serial;
    ``plan=(G, B)`` associates the two sums as the CUDA kernel does."""
    G, B = plan if plan is not None else (0, 0)
    args = [system.nr, system.nth, system.nz] + [_p(a) for a in system.arrays()]
    return lib().eaf_oracle_residual_3d(*args, _p(phi), int(G), int(B))


def pressure_correct(f) -> None:
    """Serial post-CG corrections (src/mod_pressure_3d.f90:333-397, 689-746)
    in place on the arrays of an eafgen.PcorrFields."""
    ci = ctypes.c_int
    dv = f.doubles()
    iv = f.ints()
    for a in dv:
        assert a.dtype == np.float64 and a.flags.c_contiguous
    for a in iv:
        assert a.dtype == np.int32 and a.flags.c_contiguous
    darr = (_dp * len(dv))(*[a.ctypes.data_as(_dp) for a in dv])
    iarr = (ctypes.POINTER(ci) * len(iv))(*[a.ctypes.data_as(ctypes.POINTER(ci)) for a in iv])
    rc = lib().eaf_oracle_pressure_correct(f.nr, f.nth, f.nz, darr, iarr,
                                           1 if f.has_gas else 0, float(f.alpha_p))
    if rc != 0:
        raise RuntimeError(f"oracle pressure_correct failed with status {rc}")


def pressure_assemble(f) -> float:
    """Serial assembly of the pressure-correction equation
    (src/mod_pressure_3d.f90:135-310) in place on the output arrays of an
    eafgen.AssemblyFields; returns the continuity residual."""
    ci = ctypes.c_int
    dv, iv = f.doubles(), f.ints()
    for a in dv:
        assert a.dtype == np.float64 and a.flags.c_contiguous
    for a in iv:
        assert a.dtype == np.int32 and a.flags.c_contiguous
    darr = (_dp * len(dv))(*[a.ctypes.data_as(_dp) for a in dv])
    iarr = (ctypes.POINTER(ci) * len(iv))(*[a.ctypes.data_as(ctypes.POINTER(ci)) for a in iv])
    sc = (ctypes.c_double * 4)(*f.scalars)
    res = ctypes.c_double()
    rc = lib().eaf_oracle_pressure_assemble(f.nr, f.nth, f.nz, darr, iarr, int(f.flags), sc,
                                            ctypes.byref(res))
    if rc != 0:
        raise RuntimeError(f"oracle pressure_assemble failed with status {rc}")
    return res.value


def max_threads() -> int:
    return lib().eaf_oracle_max_threads()
