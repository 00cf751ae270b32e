"""Multi-rank drop-in: an MPI-decomposed run (m%is_parallel) solving its
pressure equation on ONE GPU.

The reference's parallel CG keeps each rank's block and exchanges halos and
dot products every iteration (src/mod_solver_3d.f90:485-620 with
src/mod_mpi_topology.f90:291-417). Here the whole theta x z domain goes to one
GPU instead: every rank packs its block of the eight coefficient arrays and
phi (its interior, plus the halo layers beyond a physical r or z boundary it
touches), the root rank assembles the global arrays, solves them with the
single-GPU solver and sends each rank its block of the solution with every
halo cell that lies inside the domain -- what the closing 26-neighbour
exchange of cg_3d_mpi (:567) would have filled; halos beyond a physical
boundary keep their values. The index work lives in the C library
(eaf_mr_*); the buffers travel through torch.distributed object collectives
(a Fortran caller moves the same buffers with MPI_Gatherv / MPI_Scatterv).

The answer is that of the serial solve of the global system (the reference's
parallel run associates its dot products differently, so it lands elsewhere
in the residual ball, as any two correct FP64 CGs do).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_I3 = ctypes.c_int * 3


def _dp(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("arrays must be C-contiguous float64")
    return ctypes.c_void_p(a.ctypes.data)


def process_grid(nprocs: int, nr: int, nth: int, nz: int) -> tuple:
    """(npr, npth, npz) as factorize_3d (src/mod_mpi_topology.f90:157-204)."""
    g = _I3()
    _lib.check(_lib.load().eaf_mr_grid(nprocs, nr, nth, nz, g), "eaf_mr_grid")
    return tuple(g)


def rank_coords(rank: int, grid: tuple) -> tuple:
    """Cartesian coordinates of a rank, row-major over (r, theta, z) as
    MPI_Cart_coords numbers the ranks of a Cartesian communicator."""
    npr, npth, npz = grid
    return (rank // (npth * npz), (rank // npz) % npth, rank % npz)


def block(nr: int, nth: int, nz: int, grid: tuple, coords: tuple) -> tuple:
    """(loc, start): block extents and 1-based global start
    (decompose_domain, src/mod_mpi_topology.f90:209-250)."""
    loc, start = _I3(), _I3()
    _lib.check(_lib.load().eaf_mr_block(nr, nth, nz, _I3(*grid), _I3(*coords), loc, start),
               "eaf_mr_block")
    return tuple(loc), tuple(start)


def local_shape(loc: tuple) -> tuple:
    return (loc[2] + 4, loc[1] + 4, loc[0] + 4)


def pack(local: np.ndarray, grid, coords, loc) -> np.ndarray:
    lib = _lib.load()
    n = lib.eaf_mr_pack_count(_I3(*grid), _I3(*coords), _I3(*loc))
    buf = np.empty(n)
    _lib.check(lib.eaf_mr_pack(_dp(local), _I3(*grid), _I3(*coords), _I3(*loc), _dp(buf)),
               "eaf_mr_pack")
    return buf


def place(global_: np.ndarray, nr, nth, nz, grid, coords, loc, start, buf) -> None:
    _lib.check(_lib.load().eaf_mr_place(_dp(global_), nr, nth, nz, _I3(*grid), _I3(*coords),
                                        _I3(*loc), _I3(*start), _dp(buf)), "eaf_mr_place")


def extract(global_: np.ndarray, nr, nth, nz, loc, start) -> np.ndarray:
    lib = _lib.load()
    n = lib.eaf_mr_unpack_count(nr, nz, _I3(*start), _I3(*loc))
    buf = np.empty(n)
    _lib.check(lib.eaf_mr_extract(_dp(global_), nr, nth, nz, _I3(*loc), _I3(*start),
                                  _dp(buf)), "eaf_mr_extract")
    return buf


def unpack(local: np.ndarray, nr, nz, loc, start, buf) -> None:
    _lib.check(_lib.load().eaf_mr_unpack(_dp(local), nr, nz, _I3(*loc), _I3(*start),
                                         _dp(buf)), "eaf_mr_unpack")


def _gpu_solve(arrays, phi, max_iter, tol):
    from . import CGSolver
    nr, nth, nz = phi.shape[2] - 4, phi.shape[1] - 4, phi.shape[0] - 4
    with CGSolver(nr, nth, nz) as cg:
        return cg.solve(arrays, phi, max_iter, tol)


class MultirankError(_lib.EafError):
    """The root's gather, solve or scatter preparation failed; raised on
    every rank of the collective, with the root's status and message."""

    def __init__(self, status: int, message: str):
        super().__init__(status, "cg_3d_multirank (root): " + message)


def cg_3d_multirank(local_arrays, phi_local: np.ndarray, nr: int, nth: int, nz: int,
                    max_iter: int, tol: float, group=None, root: int = 0,
                    grid: tuple | None = None, coords: tuple | None = None, solve=None,
                    return_status: bool = False):
    """Collective over `group`: every rank passes its local (aW, aE, aS, aN,
    aB, aT, aP, Su) and phi (numpy, shape (kloc+4, jloc+4, iloc+4)); phi is
    updated in place (interior and in-domain halos). Returns (residual,
    n_iter) on every rank, or (residual, n_iter, status) with
    `return_status`. `root` is a rank of `group`.

    `solve(arrays, phi, max_iter, tol)` replaces the root's GPU solve
    (default: the single-GPU CG on the current device) and returns
    (residual, n_iter) or (residual, n_iter, status). A non-finite result is
    not an error, as in the reference (src/mod_pressure_3d.f90:322): every
    rank gets the NaN residual and status EAF_ENONFINITE. If anything on the
    root fails (placing the blocks, the solve raising, e.g. EAF_ETIMEOUT or
    EAF_ECUDA, or extracting them), every rank still completes the same
    collectives and then raises MultirankError; phi is left as it was."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    # torch takes src/dst of the object collectives as global ranks
    groot = root if group is None else dist.get_global_rank(group, root)
    grid = tuple(grid) if grid is not None else process_grid(world, nr, nth, nz)
    coords = tuple(coords) if coords is not None else rank_coords(rank, grid)
    loc, start = block(nr, nth, nz, grid, coords)
    shp = local_shape(loc)
    for a in list(local_arrays) + [phi_local]:
        if a.shape != shp:
            raise ValueError(f"local array shape {a.shape} != {shp}")
    payload = (coords, loc, start, [pack(a, grid, coords, loc)
                                    for a in list(local_arrays) + [phi_local]])
    gathered = [None] * world if rank == root else None
    dist.gather_object(payload, gathered, dst=groot, group=group)
    outs = None
    # (residual, n_iter, status, error message or None)
    result = [None]
    if rank == root:
        try:
            hshape = (nz + 4, nth + 4, nr + 4)
            G = [np.zeros(hshape) for _ in range(9)]
            for (c, l, s, bufs) in gathered:
                for a, b in zip(G, bufs):
                    place(a, nr, nth, nz, grid, c, l, s, b)
            out = (solve or _gpu_solve)(G[:8], G[8], max_iter, tol)
            res, nit = float(out[0]), int(out[1])
            st = int(out[2]) if len(out) > 2 else (
                _lib.EAF_OK if np.isfinite(res) else _lib.EAF_ENONFINITE)
            if st not in (_lib.EAF_OK, _lib.EAF_ENONFINITE):
                raise _lib.EafError(st, "solve")
            outs = [extract(G[8], nr, nth, nz, l, s) for (_, l, s, _) in gathered]
            result = [(res, nit, st, None)]
        except Exception as exc:  # reported to every rank below
            outs = [None] * world
            status = exc.status if isinstance(exc, _lib.EafError) else _lib.EAF_EINVAL
            result = [(float("nan"), 0, int(status), f"{type(exc).__name__}: {exc}")]
    recv = [None]
    dist.scatter_object_list(recv, outs, src=groot, group=group)
    dist.broadcast_object_list(result, src=groot, group=group)
    res, nit, st, err = result[0]
    if err is not None:
        raise MultirankError(st, err)
    unpack(phi_local, nr, nz, loc, start, recv[0])
    return (res, nit, st) if return_status else (res, nit)
