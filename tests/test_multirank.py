"""Multi-rank host path on CPU (gloo, world_size 2): independent systems are
partitioned across ranks, each rank solves its share (here with the oracle,
standing in for that rank's GPU), and the gathered results and max-over-
ranks timing equal a single-process run."""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT, gen

MIX = [(6, 8, 5, 2), (5, 7, 6, 2), (8, 6, 4, 2), (4, 9, 5, 2), (7, 7, 3, 2),
       (6, 6, 6, 2), (3, 12, 4, 2)]


def mg():
    import importlib
    return importlib.import_module("hornofusion-full3d_b200.multigpu")


def items():
    m = mg()
    return [m.Item(k, d[0] * d[1] * d[2], m.device_footprint(*d[:3]),
                   m.estimated_work(*d[:3])) for k, d in enumerate(MIX)]


def test_partition_complete_disjoint_balanced_and_deterministic():
    m = mg()
    its = items()
    for n in (1, 2, 3, 8):
        parts = m.partition(its, n)
        keys = sorted(i.key for p in parts for i in p)
        assert keys == list(range(len(its)))
        assert m.partition(its, n) == parts
        if n == 2:
            loads = [sum(i.work for i in p) for p in parts]
            assert max(loads) <= 0.75 * sum(loads)


def test_partition_respects_budget():
    m = mg()
    its = items()
    big = max(i.footprint for i in its)
    parts = m.partition(its, 4, budget=2.2 * big)
    for p in parts:
        assert sum(i.footprint for i in p) <= 2.2 * big
    with pytest.raises(RuntimeError):
        m.partition(its, 1, budget=0.5 * big)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import time

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle
        from conftest import gen as _gen
        g = _gen()
        m = mg()
        parts = m.partition(items(), world)
        t0 = time.perf_counter()
        local = {}
        cells = 0
        for it in parts[rank]:
            d = MIX[it.key]
            s = g.make_system(*d, seed=it.key)
            phi = g.zeros_phi(*d[:3])
            res, nit = oracle.cg(s, phi, 10000, 1e-8)
            local[it.key] = (res, nit, float(g.interior(phi).sum()))
            cells += it.cells * nit
        el = time.perf_counter() - t0
        tmax, units = m.reduce_timing(el, float(cells))
        merged = m.gather_results(local)
        if rank == 0:
            import json
            with open(out_path, "w") as f:
                json.dump({"merged": {str(k): v for k, v in merged.items()},
                           "tmax": tmax, "el": el, "units": units}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo_match_single_process(tmp_path):
    import json

    import oracle
    import torch.multiprocessing as mp
    out = str(tmp_path / "res.json")
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True,
                       start_method="spawn")
    got = json.load(open(out))
    g = gen()
    total_units = 0.0
    for k, d in enumerate(MIX):
        s = g.make_system(*d, seed=k)
        phi = g.zeros_phi(*d[:3])
        res, nit = oracle.cg(s, phi, 10000, 1e-8)
        assert got["merged"][str(k)] == [res, nit, float(g.interior(phi).sum())]
        total_units += d[0] * d[1] * d[2] * nit
    assert got["units"] == total_units
    assert got["tmax"] >= got["el"]


def _oracle_share(mine):
    """The CPU stand-in for one rank's batched GPU solve of its share."""
    import time

    import oracle
    from conftest import gen as _gen
    g = _gen()
    t0 = time.perf_counter()
    out = {}
    for it in mine:
        d = MIX[it.key]
        s = g.make_system(*d, seed=it.key)
        phi = g.zeros_phi(*d[:3])
        res, nit = oracle.cg(s, phi, 10000, 1e-8)
        out[it.key] = (res, nit, float(g.interior(phi).sum()))
    return time.perf_counter() - t0, out


def _failing_share(mine):
    import torch.distributed as dist
    if dist.get_rank() == 1:
        raise RuntimeError("device lost")
    return _oracle_share(mine)


def _sharded_worker(rank, world, port, out_dir, fail):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import json

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        m = mg()
        try:
            t, merged, parts = m.solve_sharded(items(), _failing_share if fail else _oracle_share)
            outcome = {"t": t, "merged": {str(k): v for k, v in merged.items()},
                       "parts": [[i.key for i in p] for p in parts]}
        except m.ShardError as exc:
            outcome = {"error": str(exc)}
        dist.barrier()  # the group still works after a failed share
        with open(os.path.join(out_dir, f"out{rank}.json"), "w") as f:
            json.dump(outcome, f)
    finally:
        dist.destroy_process_group()


def test_solve_sharded_two_ranks_equals_single_process(tmp_path):
    """The batch path's sharding driver (multigpu.solve_sharded) on two gloo
    ranks, with the oracle standing in for each rank's GPU batch: every rank
    gets the complete merged results, equal to the single-process run, and
    the slowest rank's time."""
    import json

    import torch.multiprocessing as mp
    mp.start_processes(_sharded_worker, args=(2, _free_port(), str(tmp_path), False),
                       nprocs=2, join=True, start_method="spawn")
    outs = [json.load(open(tmp_path / f"out{r}.json")) for r in range(2)]
    assert outs[0]["merged"] == outs[1]["merged"] and outs[0]["t"] == outs[1]["t"]
    assert sorted(k for p in outs[0]["parts"] for k in p) == list(range(len(MIX)))
    assert all(len(p) > 0 for p in outs[0]["parts"])
    _, single = _oracle_share(items())
    assert outs[0]["merged"] == {str(k): list(v) for k, v in single.items()}


def test_solve_sharded_failure_on_one_rank_raises_everywhere(tmp_path):
    import json

    import torch.multiprocessing as mp
    mp.start_processes(_sharded_worker, args=(2, _free_port(), str(tmp_path), True),
                       nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        out = json.load(open(tmp_path / f"out{r}.json"))
        assert out == {"error": "rank 1: RuntimeError: device lost"}


def test_merge_streams_whole_job_figures():
    """Streams served side by side on two GPUs: solves over the slowest
    rank's wall time, percentiles over every rank's latencies."""
    import importlib
    sc = importlib.import_module("hornofusion-full3d_b200.serve_client")
    a = {"solves": 3, "wall_s": 2.0, "runs": 1, "p99_ms": 9.0,
         "client_latency_ms": [1.0, 2.0, 3.0]}
    b = {"solves": 2, "wall_s": 4.0, "runs": 1, "p99_ms": 30.0,
         "client_latency_ms": [10.0, 30.0]}
    m = sc.merge_streams([a, b])
    assert m["solves"] == 5 and m["wall_s"] == 4.0 and m["solves_per_s"] == 1.25
    assert m["client_p50_ms"] == 3.0 and m["client_p99_ms"] == 30.0
    assert m["server_p99_ms_by_rank"] == [9.0, 30.0] and m["runs"] == 2


def _outcome_worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import json

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        m = mg()
        outs = m.gather_outcomes(lambda: {"rank": rank, "square": rank * rank})
        with open(os.path.join(out_dir, f"g{rank}.json"), "w") as f:
            json.dump(outs, f)
    finally:
        dist.destroy_process_group()


def test_gather_outcomes_three_ranks(tmp_path):
    import json

    import torch.multiprocessing as mp
    mp.start_processes(_outcome_worker, args=(3, _free_port(), str(tmp_path)), nprocs=3,
                       join=True, start_method="spawn")
    want = [{"rank": r, "square": r * r} for r in range(3)]
    for r in range(3):
        assert json.load(open(tmp_path / f"g{r}.json")) == want
