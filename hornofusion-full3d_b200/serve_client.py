"""Campaign-style serving client: concurrent simulated furnace runs.

    python hornofusion-full3d_b200/serve_client.py --rate 5 --duration 10 \
        --solves 50 [--mixed] [--seed 0] [--pool 4] [--budget-gb 150]

In the manner of scripts/run_campaign.py (which launches one `mpirun` per
run and waits for it), but in process and through the C ABI (ctypes): runs
arrive as a Poisson process of rate --rate per second during --duration
seconds; each run draws its mesh from the serving mix {18x36x24: 50 %,
35x70x50: 35 %, 60x120x84: 15 %}, is admitted against the HBM budget (a
refused run retries until admitted), and issues --solves sequential SIMPLE
pressure solves, each warm-started on the device from its previous one.
Every solve uses one of --pool pre-built perturbed systems of its mesh
(abar_P x U[0.9, 1.1], fresh zero-mean RHS, from the seeded generator),
chosen per run and solve, so inputs cost no host time during the stream.
Prints one JSON line: submit-to-completion latency p50/p99, solves/s and
the server's batching counters.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG = "hornofusion-full3d_b200"


def build_pool(g, eaf, mix, pool: int, seed: int):
    """Pinned host copies of `pool` perturbed systems per mesh of the mix."""
    out = {}
    for (dims, _) in mix:
        nr, nth, nz, nsph = dims
        mesh = g.make_mesh(nr, nth, nz, nsph, seed)
        systems = []
        for k in range(pool):
            s = g.make_system(nr, nth, nz, nsph, seed, resolve=k, mesh=mesh)
            pinned = []
            for a in s.arrays():
                h = eaf.host_empty(a.shape)
                h[...] = a
                pinned.append(h)
            systems.append(pinned)
        out[dims] = systems
    return out


def run_stream(srv, g, eaf, pool, mix, rate: float, duration: float, solves: int,
               seed: int, max_wall: float = 600.0) -> dict:
    rng = np.random.default_rng(seed)
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        u = rng.random()
        acc = 0.0
        for dims, share in mix:
            acc += share
            if u <= acc:
                break
        arrivals.append((t, dims, int(rng.integers(1 << 30))))
    srv.reset_stats()
    t0 = time.perf_counter()
    waiting = list(arrivals)  # arrived or future, not yet admitted
    active = {}               # run id -> state
    done_runs = 0
    residuals = []
    latencies = []            # client-observed submit-to-completion, ms
    while waiting or active:
        now = time.perf_counter() - t0
        if now > max_wall:
            raise RuntimeError("serving stream exceeded its wall-clock bound")
        still = []
        for (ta, dims, rseed) in waiting:
            if ta > now:
                still.append((ta, dims, rseed))
                continue
            rid = srv.try_open_run(*dims[:3])
            if rid is None:
                still.append((ta, dims, rseed))
                continue
            phi = eaf.host_empty(g.halo_shape(*dims[:3]))
            phi[...] = 0.0
            st = {"dims": dims, "seed": rseed, "k": 0, "phi": phi}
            st["ticket"] = srv.submit(rid, pool[dims][rseed % len(pool[dims])], phi)
            st["t_sub"] = time.perf_counter()
            active[rid] = st
        waiting = still
        for rid in list(active):
            st = active[rid]
            r = srv.poll(st["ticket"])
            if r is None:
                continue
            residuals.append(r[0])
            latencies.append(1e3 * (time.perf_counter() - st["t_sub"]))
            if r[3] != 0:
                raise RuntimeError(f"run {rid} solve {st['k']} failed with status {r[3]}")
            st["k"] += 1
            if st["k"] < solves:
                systems = pool[st["dims"]]
                st["ticket"] = srv.submit(
                    rid, systems[(st["seed"] + st["k"]) % len(systems)], st["phi"])
                st["t_sub"] = time.perf_counter()
            else:
                srv.close_run(rid)
                del active[rid]
                done_runs += 1
        time.sleep(0.0002)
    wall = time.perf_counter() - t0
    stats = srv.stats()
    stats.update({"runs": done_runs, "wall_s": wall,
                  "max_residual": float(max(residuals)) if residuals else None,
                  "client_latency_ms": latencies})
    return stats


def merge_streams(per_rank: list) -> dict:
    """Whole-job figures of streams served side by side on several GPUs (one
    run_stream result per rank): solves over the slowest rank's wall time,
    and p50/p99 over every rank's client-observed latencies."""
    lat = np.sort(np.concatenate([np.asarray(r["client_latency_ms"], dtype=float)
                                  for r in per_rank if r["client_latency_ms"]]))
    pct = (lambda p: float(lat[min(len(lat) - 1, int(np.floor(p * (len(lat) - 1) + 0.5)))])
           if len(lat) else None)
    wall = max(r["wall_s"] for r in per_rank)
    solves = sum(r["solves"] for r in per_rank)
    return {"solves": solves, "wall_s": wall, "solves_per_s": solves / wall if wall else 0.0,
            "client_p50_ms": pct(0.50), "client_p99_ms": pct(0.99),
            "server_p99_ms_by_rank": [r.get("p99_ms") for r in per_rank],
            "runs": sum(r["runs"] for r in per_rank)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=5.0, help="runs per second")
    ap.add_argument("--duration", type=float, default=10.0, help="arrival window, s")
    ap.add_argument("--solves", type=int, default=50, help="solves per run")
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--pool", type=int, default=4)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--small", action="store_true",
                    help="mix without the 60x120x84 mesh (quick checks)")
    args = ap.parse_args(argv)
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    mix = g.SERVE_MIX
    if args.small:
        mix = [((12, 24, 16, 8), 0.5), ((18, 36, 24, 8), 0.5)]
    pool = build_pool(g, eaf, mix, args.pool, args.seed)
    with eaf.Server(budget_bytes=args.budget_gb * 1e9, mixed=args.mixed,
                    max_iter=4000 if args.mixed else 200000, tol=1e-8) as srv:
        stats = run_stream(srv, g, eaf, pool, mix, args.rate, args.duration,
                           args.solves, args.seed)
    stats.update({"rate_runs_per_s": args.rate, "duration_s": args.duration,
                  "solves_per_run": args.solves, "mixed": args.mixed,
                  "mix": [[list(d[:3]), share] for d, share in mix]})
    print(json.dumps(stats))
    return 0


if __name__ == "__main__":
    sys.exit(main())
