"""Batched solves: one persistent launch for many uneven systems.

Each system runs on a lane whose width depends only on its mesh size, so:
  * its result is bit-identical alone (a batch of one) and in any mix;
  * in FP64 it is bit-identical to the kernel-order oracle with the plan
    (lane width, 512 threads);
  * a replayed graph gives the same bits, and new inputs are picked up.
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

MIX = [((12, 24, 16, 8), 3), ((18, 36, 24, 8), 2), ((24, 48, 30, 8), 2),
       ((35, 70, 50, 16), 1)]


def systems():
    g = gen()
    out = []
    for (dims, count) in MIX:
        for k in range(count):
            out.append(g.make_system(*dims, seed=100 + 7 * len(out)))
    return out


def run_batch(sys_list, mixed=False, widths=None, tol=1e-8):
    eaf = pkg()
    g = gen()
    dims = [(s.nr, s.nth, s.nz) for s in sys_list]
    phis = [g.zeros_phi(*d) for d in dims]
    with eaf.Batch(dims) as b:
        if widths:
            for i, w in enumerate(widths):
                b.set_width(i, w)
        for i, s in enumerate(sys_list):
            b.set_system(i, s.arrays(), phis[i])
        st = b.solve(mixed=mixed, max_iter=4000 if mixed else 200000, tol=tol,
                     max_outer=60, inner_tol=0.1)
        res = [b.result(i) for i in range(len(sys_list))]
        for i in range(len(sys_list)):
            b.get_phi(i, phis[i])
        lw = [b.lane_width(i) for i in range(len(sys_list))]
    return st, res, phis, lw


def test_batch_fp64_bitwise_vs_kernel_order_oracle_and_alone():
    import oracle
    g = gen()
    sl = systems()
    st, res, phis, lw = run_batch(sl)
    assert st == 0
    for i, s in enumerate(sl):
        r, n, o, sst = res[i]
        assert sst == 0 and r < 1e-8
        ref = g.zeros_phi(s.nr, s.nth, s.nz)
        ro, no = oracle.cg(s, ref, 200000, 1e-8, plan=(lw[i], 512))
        assert (n, r) == (no, ro), (i, n, no)
        assert np.array_equal(phis[i], ref)
    # alone (batches of one) give the same bits
    for i in (0, 3, len(sl) - 1):
        st1, res1, phis1, _ = run_batch([sl[i]])
        assert res1[0] == res[i] and np.array_equal(phis1[0], phis[i])


def test_batch_mixed_same_alone_and_in_mix():
    g = gen()
    sl = systems()[:6]
    st, res, phis, lw = run_batch(sl, mixed=True)
    assert st == 0
    for i, s in enumerate(sl):
        r, n, o, sst = res[i]
        assert sst == 0 and r < 1e-8 and o >= 1
        tr = g.interior(s.Su) - g.apply_operator(s, phis[i])
        assert np.linalg.norm(tr) / np.linalg.norm(g.interior(s.Su)) < 1.001e-8
    for i in (0, 4):
        st1, res1, phis1, _ = run_batch([sl[i]], mixed=True)
        assert res1[0] == res[i] and np.array_equal(phis1[0], phis[i])


def test_batch_width_override_and_replay():
    eaf = pkg()
    g = gen()
    sl = systems()[:4]
    dims = [(s.nr, s.nth, s.nz) for s in sl]
    with eaf.Batch(dims) as b:
        b.set_width(3, 3)
        assert b.lane_width(3) == 3
        grid, block, nlanes = b.plan()
        assert block == 512 and nlanes >= 4 and grid >= 3
        phis = [g.zeros_phi(*d) for d in dims]
        for i, s in enumerate(sl):
            b.set_system(i, s.arrays(), phis[i])
        b.solve()
        first = [b.result(i) for i in range(4)]
        out1 = [b.get_phi(i, g.zeros_phi(*dims[i])) for i in range(4)]
        # replay with the same inputs (phi re-uploaded as zeros)
        for i, s in enumerate(sl):
            b.set_system(i, s.arrays(), g.zeros_phi(*dims[i]))
        b.solve()
        assert [b.result(i) for i in range(4)] == first
        for i in range(4):
            assert np.array_equal(b.get_phi(i, g.zeros_phi(*dims[i])), out1[i])
        # new right-hand side is picked up
        s2 = g.make_system(12, 24, 16, 8, seed=999)
        b.set_system(0, s2.arrays(), g.zeros_phi(12, 24, 16))
        b.solve()
        assert b.result(0)[0] < 1e-8 and b.result(0) != first[0]


def test_large_system_runs_at_full_width_after_the_lanes():
    """A 60x120x84 system (over the large-system threshold) is solved after
    the batched launch with its single-system launch: bit-identical to the
    oracle with that plan, and to the same system alone; the small systems
    of the batch keep their lanes."""
    import oracle
    g = gen()
    big = g.make_system(60, 120, 84, 24, seed=11)
    sl = [big] + systems()[:3]
    eaf = pkg()
    dims = [(s.nr, s.nth, s.nz) for s in sl]
    with eaf.Batch(dims) as b:
        plans = [b.system_plan(i) for i in range(len(sl))]
    with eaf.CGSolver(60, 120, 84) as cg:
        cg.solve(big.arrays(), g.zeros_phi(60, 120, 84), 1, 1e-8)
        single = cg.last_launch()
    assert plans[0] == single and plans[1][1] == 512
    st, res, phis, lw = run_batch(sl)
    assert st == 0
    for i, s in enumerate(sl):
        ref = g.zeros_phi(s.nr, s.nth, s.nz)
        ro, no = oracle.cg(s, ref, 200000, 1e-8, plan=plans[i])
        assert (res[i][1], res[i][0]) == (no, ro), i
        assert np.array_equal(phis[i], ref)
    st1, res1, phis1, _ = run_batch([big])
    assert res1[0] == res[0] and np.array_equal(phis1[0], phis[0])
