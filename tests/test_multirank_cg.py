"""Multi-rank drop-in of the CG (gather onto one GPU rank, scatter back), on
the CPU: the index helpers of libeafcg.so against Python restatements of the
reference's decomposition, and the whole collective over gloo ranks with the
oracle standing in for the root's GPU solve."""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT, gen, pkg


def mr():
    import importlib
    return importlib.import_module("hornofusion-full3d_b200.multirank")


def py_factorize(nprocs, nr, nth, nz):
    """factorize_3d (src/mod_mpi_topology.f90:157-204), restated."""
    best, bp, bt, bz = 1.0e20, 1, 1, nprocs
    for tp in range(1, nprocs + 1):
        if nprocs % tp:
            continue
        for tt in range(1, nprocs // tp + 1):
            if (nprocs // tp) % tt or nth % tt:
                continue
            tz = nprocs // (tp * tt)
            cr, ct, cz = nr / tp, nth / tt, nz / tz
            asp = max(cr / ct, ct / cr) * max(cr / cz, cz / cr) * max(ct / cz, cz / ct)
            if asp < best:
                best, bp, bt, bz = asp, tp, tt, tz
    return (bp, bt, bz)


def local_from_global(glob, nr, nth, nz, loc, start):
    """A rank's local halo-layout array cut from a global one: r/z indices map
    straight (the global halos stand in for physical halos), theta wraps."""
    i = np.arange(-1, loc[0] + 3) + start[0] - 1
    j = (np.arange(-1, loc[1] + 3) + start[1] - 2) % nth + 1
    k = np.arange(-1, loc[2] + 3) + start[2] - 1
    return glob[np.ix_(k + 1, j + 1, i + 1)].copy()


@pytest.mark.parametrize("nprocs,dims", [(1, (12, 24, 16)), (2, (12, 24, 16)),
                                         (4, (60, 120, 84)), (6, (20, 30, 40)),
                                         (8, (7, 9, 11)), (12, (35, 70, 50))])
def test_process_grid_matches_factorize_3d(nprocs, dims):
    assert mr().process_grid(nprocs, *dims) == py_factorize(nprocs, *dims)


@pytest.mark.parametrize("nprocs,dims", [(2, (12, 24, 16)), (4, (9, 8, 7)),
                                         (6, (20, 30, 40)), (3, (5, 6, 4))])
def test_blocks_tile_the_domain_and_round_trip(nprocs, dims):
    m = mr()
    nr, nth, nz = dims
    grid = m.process_grid(nprocs, *dims)
    rng = np.random.default_rng(1)
    glob = rng.normal(size=gen().halo_shape(*dims))
    rebuilt = np.full_like(glob, np.nan)
    count = np.zeros((nz, nth, nr), dtype=int)
    for rank in range(nprocs):
        c = m.rank_coords(rank, grid)
        loc, start = m.block(nr, nth, nz, grid, c)
        count[start[2] - 1:start[2] - 1 + loc[2], start[1] - 1:start[1] - 1 + loc[1],
              start[0] - 1:start[0] - 1 + loc[0]] += 1
        local = local_from_global(glob, nr, nth, nz, loc, start)
        m.place(rebuilt, nr, nth, nz, grid, c, loc, start, m.pack(local, grid, c, loc))
    assert (count == 1).all()
    I = gen().interior
    assert np.array_equal(I(rebuilt), I(glob))
    # physical r and z halo layers came back too
    assert np.array_equal(rebuilt[:, 2:-2, :2], glob[:, 2:-2, :2])
    assert np.array_equal(rebuilt[:2, 2:-2, :], glob[:2, 2:-2, :])
    assert np.array_equal(rebuilt[-2:, 2:-2, -2:], glob[-2:, 2:-2, -2:])
    # scatter: interior and in-domain halos from the global array, the rest kept
    for rank in range(nprocs):
        c = m.rank_coords(rank, grid)
        loc, start = m.block(nr, nth, nz, grid, c)
        local = np.full(m.local_shape(loc), -7.0)
        m.unpack(local, nr, nz, loc, start, m.extract(glob, nr, nth, nz, loc, start))
        want = local_from_global(glob, nr, nth, nz, loc, start)
        ig = np.arange(-1, loc[0] + 3) + start[0] - 1
        kg = np.arange(-1, loc[2] + 3) + start[2] - 1
        inside = ((kg >= 1) & (kg <= nz))[:, None, None] & ((ig >= 1) & (ig <= nr))[None, None, :]
        inside = np.broadcast_to(inside, local.shape)
        assert np.array_equal(local[inside], want[inside])
        assert (local[~inside] == -7.0).all()


def test_helpers_reject_bad_blocks():
    m = mr()
    with pytest.raises(pkg().EafError):
        m.block(4, 4, 4, (5, 1, 1), (0, 0, 0))  # more ranks than cells in r
    with pytest.raises(pkg().EafError):
        m.block(4, 4, 4, (2, 1, 1), (2, 0, 0))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_solve(arrays, phi, max_iter, tol):
    import oracle
    g = gen()
    nr, nth, nz = phi.shape[2] - 4, phi.shape[1] - 4, phi.shape[0] - 4
    s = g.System(nr=nr, nth=nth, nz=nz, **dict(zip(g.COEF_NAMES, arrays)))
    return oracle.cg(s, phi, max_iter, tol)


def _worker(rank, world, port, dims, out_dir, use_gpu):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = mr()
        g = gen()
        nr, nth, nz = dims
        s = g.make_system(nr, nth, nz, nsph=4, seed=3)
        phi_g = np.random.default_rng(2).normal(0, 1e-4, size=g.halo_shape(*dims))
        grid = m.process_grid(world, *dims)
        c = m.rank_coords(rank, grid)
        loc, start = m.block(nr, nth, nz, grid, c)
        arrays = [local_from_global(a, nr, nth, nz, loc, start) for a in s.arrays()]
        phi = local_from_global(phi_g, nr, nth, nz, loc, start)
        res, nit = m.cg_3d_multirank(arrays, phi, nr, nth, nz, 5000, 1e-8,
                                     solve=None if use_gpu else _oracle_solve)
        np.save(os.path.join(out_dir, f"phi{rank}.npy"), phi)
        np.save(os.path.join(out_dir, f"res{rank}.npy"), np.array([res, nit]))
    finally:
        dist.destroy_process_group()


def run_ranks(world, dims, out_dir, use_gpu=False):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), dims, str(out_dir), use_gpu),
                       nprocs=world, join=True, start_method="spawn")


def check_against_single(world, dims, out_dir, solve):
    m = mr()
    g = gen()
    nr, nth, nz = dims
    s = g.make_system(nr, nth, nz, nsph=4, seed=3)
    phi_g = np.random.default_rng(2).normal(0, 1e-4, size=g.halo_shape(*dims))
    before = phi_g.copy()
    res, nit = solve(s, phi_g)
    grid = m.process_grid(world, *dims)
    for rank in range(world):
        c = m.rank_coords(rank, grid)
        loc, start = m.block(nr, nth, nz, grid, c)
        got = np.load(os.path.join(out_dir, f"phi{rank}.npy"))
        want = local_from_global(phi_g, nr, nth, nz, loc, start)
        kept = local_from_global(before, nr, nth, nz, loc, start)
        ig = np.arange(-1, loc[0] + 3) + start[0] - 1
        kg = np.arange(-1, loc[2] + 3) + start[2] - 1
        inside = ((kg >= 1) & (kg <= nz))[:, None, None] & ((ig >= 1) & (ig <= nr))[None, None, :]
        inside = np.broadcast_to(inside, got.shape)
        assert np.array_equal(got[inside], want[inside]), rank
        assert np.array_equal(got[~inside], kept[~inside]), rank
        r = np.load(os.path.join(out_dir, f"res{rank}.npy"))
        assert r[0] == res and int(r[1]) == nit


@pytest.mark.parametrize("world,dims", [(2, (12, 24, 16)), (3, (9, 12, 10)),
                                        (4, (8, 12, 10))])
def test_gloo_ranks_match_serial_solve(tmp_path, world, dims):
    import oracle
    run_ranks(world, dims, tmp_path)
    check_against_single(world, dims, tmp_path,
                         lambda s, phi: oracle.cg(s, phi, 5000, 1e-8))


def _raising_solve(arrays, phi, max_iter, tol):
    raise pkg().EafError(pkg()._lib.EAF_ETIMEOUT, "solve")


def _failure_worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        m = mr()
        g = gen()
        dims = (12, 24, 16)
        s = g.make_system(*dims, nsph=4, seed=3)
        grid = m.process_grid(world, *dims)
        c = m.rank_coords(rank, grid)
        loc, start = m.block(*dims, grid, c)
        arrays = [local_from_global(a, *dims, loc, start) for a in s.arrays()]
        phi = local_from_global(g.zeros_phi(*dims), *dims, loc, start)
        before = phi.copy()
        outcome = "returned"
        try:
            m.cg_3d_multirank(arrays, phi, *dims, 100, 1e-8, solve=_raising_solve)
        except m.MultirankError as exc:
            outcome = f"raised {exc.status}"
        # the collective stays usable after the failure
        dist.barrier()
        np.save(os.path.join(out_dir, f"unchanged{rank}.npy"),
                np.array([np.array_equal(phi, before)]))
        with open(os.path.join(out_dir, f"outcome{rank}.txt"), "w") as f:
            f.write(outcome)
    finally:
        dist.destroy_process_group()


def test_gloo_root_solve_failure_raises_on_every_rank(tmp_path):
    """The root's solve raises (as a timed-out or failed GPU solve does):
    every rank completes the collectives and raises MultirankError with the
    root's status, phi untouched, and the process group still works."""
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_failure_worker, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    st = pkg()._lib.EAF_ETIMEOUT
    for rank in range(world):
        assert open(os.path.join(tmp_path, f"outcome{rank}.txt")).read() == f"raised {st}"
        assert bool(np.load(os.path.join(tmp_path, f"unchanged{rank}.npy"))[0])


def _subgroup_worker(rank, world, port, out_dir):
    """Ranks 1 and 2 of 3 form the group; its rank 0 (global rank 1) is the
    root."""
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sub = dist.new_group([1, 2])
        if rank in (1, 2):
            m = mr()
            g = gen()
            dims = (12, 24, 16)
            s = g.make_system(*dims, nsph=4, seed=3)
            phi_g = np.random.default_rng(2).normal(0, 1e-4, size=g.halo_shape(*dims))
            grank = dist.get_rank(sub)
            grid = m.process_grid(2, *dims)
            c = m.rank_coords(grank, grid)
            loc, start = m.block(*dims, grid, c)
            arrays = [local_from_global(a, *dims, loc, start) for a in s.arrays()]
            phi = local_from_global(phi_g, *dims, loc, start)
            res, nit = m.cg_3d_multirank(arrays, phi, *dims, 5000, 1e-8, group=sub,
                                         root=0, solve=_oracle_solve)
            np.save(os.path.join(out_dir, f"phi{grank}.npy"), phi)
            np.save(os.path.join(out_dir, f"res{grank}.npy"), np.array([res, nit]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_subgroup_root_is_mapped_to_its_global_rank(tmp_path):
    import oracle
    import torch.multiprocessing as mp
    mp.start_processes(_subgroup_worker, args=(3, _free_port(), str(tmp_path)),
                       nprocs=3, join=True, start_method="spawn")
    check_against_single(2, (12, 24, 16), tmp_path,
                         lambda s, phi: oracle.cg(s, phi, 5000, 1e-8))
