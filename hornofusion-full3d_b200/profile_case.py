"""One solver launch on a chosen mesh, for profiling (ncu) and quick timing.

    python hornofusion-full3d_b200/profile_case.py --mesh 60 120 84 \
        --iters 400 [--mixed] [--launch BLOCK GRID] [--repeat R]

Builds the seeded system, uploads it once, then runs R solves through the
device-pointer C-ABI entry with tol 0 (exactly `--iters` iterations, so the
work per launch is fixed) and prints the per-solve device times.
"""
import argparse
import importlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, nargs=3, default=[60, 120, 84])
    ap.add_argument("--spheres", type=int, default=24)
    ap.add_argument("--iters", type=int, default=400)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--launch", type=int, nargs=2, default=None)
    args = ap.parse_args(argv)
    import torch
    eaf = importlib.import_module("hornofusion-full3d_b200")
    g = importlib.import_module("hornofusion-full3d_b200.eafgen")
    nr, nth, nz = args.mesh
    s = g.make_system(nr, nth, nz, args.spheres, seed=0)
    dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
    phi = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    out = []
    with eaf.CGSolver(nr, nth, nz) as cg:
        if args.launch:
            cg.set_launch(*args.launch)
        block, grid = cg.launch()
        for _ in range(args.repeat):
            phi.zero_()
            torch.cuda.synchronize()
            if args.mixed:
                res, nit, nout, st = cg.solve_mixed(
                    dev, phi, tol=0.0, inner_tol=1e-30, max_outer=1,
                    max_inner=args.iters, device_ptrs=True)
            else:
                res, nit, st = cg.solve(dev, phi, args.iters, 0.0, device_ptrs=True)
            t = cg.last_timing()
            out.append({"iters": nit, "residual": res, "status": st,
                        "kernel_ms": t["kernel_ms"], "solve_ms": t["solve_ms"],
                        "us_per_iter": 1e3 * t["kernel_ms"] / max(nit, 1)})
    print(json.dumps({"mesh": [nr, nth, nz], "launch": [grid, block],
                      "mixed": args.mixed, "runs": out}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
