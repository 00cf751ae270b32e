"""One solver launch on a chosen mesh, for profiling (ncu) and quick timing.

    python hornofusion-full3d_b200/profile_case.py --mesh 60 120 84 \
        --iters 400 [--mixed] [--launch BLOCK GRID] [--repeat R]
        [--form reference|one-reduction]

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
    ap.add_argument("--form", choices=["reference", "one-reduction"], default="reference",
                    help="recurrences of the plain FP64 solve")
    ap.add_argument("--launch", type=int, nargs=2, default=None)
    ap.add_argument("--batch", type=int, default=0,
                    help="solve this many copies of the mixed batch instead "
                         "(12x24x16, 18x36x24, 35x70x50, 60x120x84 round robin)")
    ap.add_argument("--tdma", type=int, default=0,
                    help="time this many line-TDMA sweeps of a transport system "
                         "on the mesh instead of a CG solve")
    args = ap.parse_args(argv)
    if args.batch:
        return batch_case(args)
    if args.tdma:
        return tdma_case(args)
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
        cg.set_form(cg.FORM_ONE_REDUCTION if args.form == "one-reduction"
                    else cg.FORM_REFERENCE)
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


def tdma_case(args):
    import torch
    eaf = importlib.import_module("hornofusion-full3d_b200")
    g = importlib.import_module("hornofusion-full3d_b200.eafgen")
    nr, nth, nz = args.mesh
    s = g.make_transport_system(nr, nth, nz, seed=0)
    dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
    phi = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64, device="cuda")
    out = []
    with eaf.CGSolver(nr, nth, nz) as cg:
        for _ in range(args.repeat):
            phi.zero_()
            torch.cuda.synchronize()
            cg.tdma(dev, phi, args.tdma, device_ptrs=True)
            t = cg.last_timing()
            out.append({"sweeps": args.tdma, "kernel_ms": t["kernel_ms"],
                        "ms_per_sweep": t["kernel_ms"] / args.tdma,
                        "ns_per_cell_sweep": 1e6 * t["kernel_ms"] / args.tdma
                        / (nr * nth * nz)})
        launch = cg.last_launch()
    print(json.dumps({"mesh": [nr, nth, nz], "tdma": True, "launch": launch, "runs": out}))
    return 0


def batch_case(args):
    import torch
    eaf = importlib.import_module("hornofusion-full3d_b200")
    g = importlib.import_module("hornofusion-full3d_b200.eafgen")
    meshes = [d for d, _ in g.BATCH_MIX]
    systems = [g.make_system(*meshes[k % len(meshes)], seed=k) for k in range(args.batch)]
    dims = [(s.nr, s.nth, s.nz) for s in systems]
    dev = [[torch.from_numpy(a).cuda() for a in s.arrays()] for s in systems]
    phis = [torch.zeros(g.halo_shape(*d), dtype=torch.float64, device="cuda") for d in dims]
    out = []
    with eaf.Batch(dims) as b:
        for i in range(len(systems)):
            b.set_system(i, dev[i], phis[i], device_ptrs=True)
        for _ in range(args.repeat):
            for p in phis:
                p.zero_()
            torch.cuda.synchronize()
            b.solve(max_iter=args.iters, tol=0.0)
            cells = sum(d[0] * d[1] * d[2] for d in dims)
            out.append({"batch_ms": b.last_ms,
                        "cell_iters_per_s": cells * args.iters / (b.last_ms / 1e3)})
        plan = b.plan()
    print(json.dumps({"batch": dims, "plan": plan, "runs": out}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
