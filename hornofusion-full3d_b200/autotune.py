"""Autotuner for the launch shapes of the pressure-CG kernels (needs a GPU).

    python hornofusion-full3d_b200/autotune.py [--iters 200] [--write]

For every mesh of the named workloads it measures, with fixed iteration
counts (tol 0) and CUDA-event device times from the library:

* single-system solver (eaf_cg_*): the time per iteration of the persistent
  kernel for block sizes 256/512/1024 and grid sizes from one block up to
  the co-resident maximum, with per-thread loads and, where a block's slice
  fits its shared memory, with the update operands kept there; the
  bulk-copy streaming kernel on one block per SM; and, on meshes that fit one cluster's shared
  memory, the cluster-resident kernel on one cluster of 4, 8 or 16 blocks of
  128 to 1024 threads; the fastest (block, grid, cluster) is kept;
* batched/served solver (eaf_batch_*): the time per iteration t(w) of one
  system on a lane of w blocks of 512 threads. A batch is limited by the
  block-time its systems take (t(w) * w per iteration) and by its longest
  solve (t(w) * iterations), so the kept width is the one with the least
  block-time among those within LATENCY_SLACK of the fastest t(w) measured.

With --write it regenerates csrc/tune_table.h (then rebuild the library)
and tune_table.json beside this file; --out-dir DIR writes both into DIR
instead, and --from-json FILE regenerates them from a saved measurement.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

MESHES = [(12, 24, 16, 8), (18, 36, 24, 8), (35, 70, 50, 16), (60, 120, 84, 24),
          (120, 240, 168, 64)]
LATENCY_SLACK = 2.5
RESIDENT_MAX_CELLS = 28000
KEEP_MAX_SLICE_BYTES = 220 * 1024  # kept operands of one block's slice


def select(log):
    """Tables from the measurement log: fastest single-solver shape per mesh,
    and the lane width rule above."""
    single, lanes = [], []
    meshes = []
    for m in log:
        if tuple(m["mesh"]) not in meshes:
            meshes.append(tuple(m["mesh"]))
    for d in meshes:
        sm = [m for m in log if tuple(m["mesh"]) == d and m["solver"] == "single"]
        if sm:
            b = min(sm, key=lambda m: (m["us_per_iter"], m["block"], m["grid"]))
            single.append((d, b["block"], b["grid"], b.get("cluster", 1), b.get("stream", 0),
                           b["us_per_iter"]))
        lm = [m for m in log if tuple(m["mesh"]) == d and m["solver"] == "lane"]
        if lm:
            tmin = min(m["us_per_iter"] for m in lm)
            ok = [m for m in lm if m["us_per_iter"] <= LATENCY_SLACK * tmin]
            b = min(ok, key=lambda m: (m["us_per_iter"] * m["width"], m["width"]))
            lanes.append((d, b["width"], b["us_per_iter"]))
    return single, lanes


# Flat-grid kernel codes of the table: per-thread loads, bulk-copy
# streaming, own cells kept in shared memory.
FLAT_LOADS, FLAT_STREAM, FLAT_KEEP = 0, 1, 2


def time_single(eaf, dev_arrays, phi, dims, block, grid, iters, cluster=1, stream=FLAT_LOADS,
                want_kernel=False):
    with eaf.CGSolver(*dims) as cg:
        cg.set_launch(block, grid)
        cg.set_cluster(cluster)
        cg.set_kernel({FLAT_LOADS: cg.KERNEL_LOADS, FLAT_STREAM: cg.KERNEL_STREAM,
                       FLAT_KEEP: cg.KERNEL_KEEP}[stream])
        best = float("inf")
        for _ in range(2):
            phi.zero_()
            cg.solve(dev_arrays, phi, iters, 0.0, device_ptrs=True)
            best = min(best, cg.last_timing()["kernel_ms"] / iters)
        if want_kernel:
            return best * 1e3, cg.last_launch(), cg.last_kernel() == cg.KERNEL_KEEP
        return best * 1e3, cg.last_launch()


def time_lane(eaf, g, s, dims, width, iters):
    with eaf.Batch([dims]) as b:
        b.set_width(0, width)
        phi = g.zeros_phi(*dims)
        best = float("inf")
        for _ in range(2):
            b.set_system(0, s.arrays(), phi)
            b.solve(max_iter=iters, tol=0.0)
            best = min(best, b.last_ms / iters)
        return best * 1e3


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=200)
    ap.add_argument("--write", action="store_true")
    ap.add_argument("--out-dir", default=None,
                    help="write tune_table.json and tune_table.h there instead")
    ap.add_argument("--from-json", default=None,
                    help="regenerate the header from a saved tune_table.json")
    args = ap.parse_args(argv)
    if args.from_json:
        with open(args.from_json) as f:
            res = json.load(f)
        single, lanes = select(res["measurements"])
        res["single"] = [{"mesh": list(d), "block": b, "grid": gr, "cluster": c, "stream": st,
                          "us_per_iter": u} for d, b, gr, c, st, u in single]
        res["lanes"] = [{"mesh": list(d), "width": w, "us_per_iter": u}
                        for d, w, u in lanes]
        res["lane_rule"] = f"least t(w)*w among t(w) <= {LATENCY_SLACK} x min t"
        with open(os.path.join(HERE, "tune_table.json"), "w") as f:
            json.dump(res, f, indent=1)
        write_header(single, lanes, os.path.join(HERE, "csrc", "tune_table.h"))
        return 0
    import torch
    eaf = importlib.import_module("hornofusion-full3d_b200")
    g = importlib.import_module("hornofusion-full3d_b200.eafgen")
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    log = []
    for (nr, nth, nz, nsph) in MESHES:
        dims = (nr, nth, nz)
        n = nr * nth * nz
        s = g.make_system(nr, nth, nz, nsph, seed=0)
        dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
        phi = torch.zeros(g.halo_shape(*dims), dtype=torch.float64, device="cuda")
        cands = set()
        for block in (256, 512, 1024):
            per_sm = 2048 // block
            cap = per_sm * sms
            grids = {1, 2, 4, 8, 16, 32, 64, sms // 2, sms, 2 * sms, cap}
            for k in (1, 2, 4, 8, 16):
                grids.add(max(1, math.ceil(n / (block * k))))
            for grid in grids:
                if 1 <= grid <= cap and grid * block <= max(n, block):
                    cands.add((block, grid))
        for (block, grid) in sorted(cands):
            us, used = time_single(eaf, dev, phi, dims, block, grid, args.iters)
            log.append({"mesh": dims, "solver": "single", "block": block, "grid": used[0],
                        "us_per_iter": round(us, 3)})
            if 4 * 8 * math.ceil(n / grid) <= KEEP_MAX_SLICE_BYTES:
                us, used, kept = time_single(eaf, dev, phi, dims, block, grid, args.iters,
                                             1, FLAT_KEEP, want_kernel=True)
                if kept:
                    log.append({"mesh": dims, "solver": "single", "block": block,
                                "grid": used[0], "stream": FLAT_KEEP,
                                "us_per_iter": round(us, 3)})
        for block in (512, 1024):  # the bulk-copy streaming kernel, one block per SM
            us, used = time_single(eaf, dev, phi, dims, block, sms, args.iters, 1, FLAT_STREAM)
            log.append({"mesh": dims, "solver": "single", "block": block, "grid": used[0],
                        "stream": FLAT_STREAM, "us_per_iter": round(us, 3)})
        if n <= RESIDENT_MAX_CELLS:  # one cluster holding the system on chip
            for c in (4, 8, 16):
                for block in (128, 256, 288, 512, 1024):
                    us, used = time_single(eaf, dev, phi, dims, block, c, args.iters, c)
                    if len(used) == 3 and used[0] == c:
                        log.append({"mesh": dims, "solver": "single", "block": block,
                                    "grid": c, "cluster": c, "us_per_iter": round(us, 3)})
        if n <= 1_000_000:  # batched/served meshes
            widths = [w for w in (1, 2, 4, 8, 16, 24, 32, 48, 64, 96, 128)
                      if w * 512 <= max(2 * n, 512)]
            for w in widths:
                us = time_lane(eaf, g, s, dims, w, args.iters)
                log.append({"mesh": dims, "solver": "lane", "width": w,
                            "us_per_iter": round(us, 3)})
        del dev, phi
        torch.cuda.empty_cache()
    single, lanes = select(log)
    result = {"gpu": torch.cuda.get_device_name(0), "iters": args.iters,
              "lane_rule": f"least t(w)*w among t(w) <= {LATENCY_SLACK} x min t",
              "single": [{"mesh": d, "block": b, "grid": gr, "cluster": c, "stream": st,
                          "us_per_iter": round(u, 3)} for d, b, gr, c, st, u in single],
              "lanes": [{"mesh": d, "width": w, "us_per_iter": round(u, 3)}
                        for d, w, u in lanes],
              "measurements": log}
    if args.write or args.out_dir:
        out = args.out_dir or HERE
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "tune_table.json"), "w") as f:
            json.dump(result, f, indent=1)
        write_header(single, lanes, os.path.join(out if args.out_dir else
                                                 os.path.join(HERE, "csrc"),
                                                 "tune_table.h"))
    print(json.dumps({k: result[k] for k in ("gpu", "single", "lanes")}))
    return 0


def write_header(single, lanes, path):
    rows_l = "\n".join(f"    {{{d[0]}, {d[1]}, {d[2]}, {w}}}," for d, w, _ in lanes)
    rows_s = "\n".join(f"    {{{d[0]}, {d[1]}, {d[2]}, {b}, {gr}, {c}, {st}}},"
                       for d, b, gr, c, st, _ in single)
    text = f"""// Launch shapes measured on B200 by hornofusion-full3d_b200/autotune.py
// (tune_table.json beside it holds every measurement). Meshes that are not
// in a table fall back to the rules below.
#pragma once

namespace eaf {{

struct TunedWidth {{
  int nr, nth, nz, width;
}};

// Lane width (blocks of 512 threads) of batched and served solves.
static constexpr TunedWidth kTunedWidths[] = {{
{rows_l}
}};

inline int tuned_lane_width(int nr, int nth, int nz) {{
  for (const TunedWidth& t : kTunedWidths)
    if (t.nr == nr && t.nth == nth && t.nz == nz) return t.width;
  const long long n = (long long)nr * nth * nz;
  long long w = (n + 16383) / 16384;  // about 32 cells per thread
  return (int)(w < 1 ? 1 : (w > 64 ? 64 : w));
}}

struct TunedLaunch {{
  int nr, nth, nz, block, grid, cluster, stream;
}};

// (block, grid, blocks per cluster (1 = no clusters), flat-grid kernel:
// per-thread loads (0), bulk-copy streaming (1) or own cells kept in shared
// memory (2)) of the single-system persistent solver.
static constexpr TunedLaunch kTunedLaunches[] = {{
{rows_s}
}};

// Most blocks a tuned launch of a mesh of at most `max_cells` cells can run
// (a grid is raised to one whole cluster at least); 0 if there is none.
constexpr int max_tuned_grid_up_to(long long max_cells) {{
  int g = 0;
  for (const TunedLaunch& t : kTunedLaunches) {{
    const int blocks = t.grid > t.cluster ? t.grid : t.cluster;
    if ((long long)t.nr * t.nth * t.nz <= max_cells && blocks > g) g = blocks;
  }}
  return g;
}}

inline bool tuned_single_launch(int nr, int nth, int nz, int* block, int* grid,
                                int* cluster = nullptr, int* stream = nullptr) {{
  for (const TunedLaunch& t : kTunedLaunches)
    if (t.nr == nr && t.nth == nth && t.nz == nz) {{
      *block = t.block;
      *grid = t.grid;
      if (cluster) *cluster = t.cluster;
      if (stream) *stream = t.stream;
      return true;
    }}
  return false;
}}

}}  // namespace eaf
"""
    with open(path, "w") as f:
        f.write(text)


if __name__ == "__main__":
    sys.exit(main())
