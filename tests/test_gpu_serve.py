"""The serving loop: admission, continuous batching, and results that are
the same alone and in the mix (exactly: a run's lane width depends only on
its mesh size, so its arithmetic never depends on the other runs).

The server reads a request's inputs and writes its phi_out until the ticket
completes; the Python wrapper holds references to them until then."""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

MESH_A = (18, 36, 24, 8)
OTHERS = [(12, 24, 16, 8), (24, 48, 30, 8), (12, 24, 16, 8), (35, 70, 50, 16),
          (18, 36, 24, 8)]


def sequence(dims, seed, n):
    g = gen()
    mesh = g.make_mesh(*dims, seed)
    return [g.make_system(*dims, seed, resolve=k, mesh=mesh) for k in range(n)]


def solve_rounds(srv, runs, rounds):
    """runs: list of (run_id, systems, phi). Submits one solve per run per
    round, all concurrently; returns per run the list of phi copies."""
    out = [[] for _ in runs]
    for k in range(rounds):
        tickets = [srv.submit(rid, systems[k].arrays(), phi)
                   for (rid, systems, phi) in runs]
        for i, t in enumerate(tickets):
            res, nit, nout, st = srv.wait(t)
            assert st == 0 and res < 1e-8
            out[i].append(runs[i][2].copy())
    return out


@pytest.mark.parametrize("mixed", [False, True])
def test_same_alone_and_in_the_mix(mixed):
    eaf = pkg()
    g = gen()
    rounds = 3 if not mixed else 2
    seq_a = sequence(MESH_A, 11, rounds)
    kw = dict(mixed=mixed, max_iter=4000 if mixed else 200000)
    with eaf.Server(**kw) as srv:
        ra = srv.open_run(*MESH_A[:3])
        alone = solve_rounds(srv, [(ra, seq_a, g.zeros_phi(*MESH_A[:3]))], rounds)[0]
    with eaf.Server(**kw) as srv:
        runs = [(srv.open_run(*MESH_A[:3]), seq_a, g.zeros_phi(*MESH_A[:3]))]
        for j, d in enumerate(OTHERS):
            runs.append((srv.open_run(*d[:3]), sequence(d, 50 + j, rounds),
                         g.zeros_phi(*d[:3])))
        mix = solve_rounds(srv, runs, rounds)
        st = srv.stats()
    for k in range(rounds):
        assert np.array_equal(alone[k], mix[0][k]), f"round {k} differs"
    assert st["solves"] == rounds * len(runs) and st["batches"] >= rounds


def test_admission_budget_and_busy_rules():
    eaf = pkg()
    g = gen()
    with eaf.Server(budget_bytes=40e6) as srv:
        assert srv.try_open_run(60, 120, 84) is None   # ~120 MB of device state
        r1 = srv.open_run(12, 24, 16)
        s = g.make_system(12, 24, 16, 8, seed=3)
        phi = g.zeros_phi(12, 24, 16)
        t = srv.submit(r1, s.arrays(), phi)
        with pytest.raises(eaf.EafError):
            srv.submit(r1, s.arrays(), phi)              # one outstanding solve
        res, nit, nout, st = srv.wait(t)
        assert st == 0 and res < 1e-8
        srv.close_run(r1)
        st = srv.stats()
        assert st["refused_runs"] == 1 and st["active_runs"] == 0


def test_wait_timeout_then_result():
    eaf = pkg()
    g = gen()
    s = g.make_system(60, 120, 84, 24, seed=5)
    with eaf.Server() as srv:
        r = srv.open_run(60, 120, 84)
        phi = g.zeros_phi(60, 120, 84)
        t = srv.submit(r, s.arrays(), phi)
        with pytest.raises(eaf.EafError) as e:
            srv.wait(t, timeout_ms=0.01)
        assert e.value.status == eaf._lib.EAF_ETIMEOUT
        res, nit, nout, st = srv.wait(t)
        assert st == 0 and res < 1e-8


def test_injected_device_loss_fails_work_and_closes():
    eaf = pkg()
    g = gen()
    s = g.make_system(35, 70, 50, 16, seed=5)
    with eaf.Server() as srv:
        r = srv.open_run(35, 70, 50)
        phi = g.zeros_phi(35, 70, 50)
        t = srv.submit(r, s.arrays(), phi)
        srv.inject_device_lost()
        res, nit, nout, st = srv.wait(t)
        assert st == eaf._lib.EAF_ECUDA
        with pytest.raises(eaf.EafError) as e:
            srv.submit(r, s.arrays(), phi)
        assert e.value.status == eaf._lib.EAF_ECLOSED


def test_campaign_client_stream():
    import importlib
    eaf = pkg()
    g = gen()
    sc = importlib.import_module("hornofusion-full3d_b200.serve_client")
    mix = [((12, 24, 16, 8), 0.5), ((18, 36, 24, 8), 0.5)]
    pool = sc.build_pool(g, eaf, mix, 2, 0)
    with eaf.Server() as srv:
        st = sc.run_stream(srv, g, eaf, pool, mix, rate=20.0, duration=0.5, solves=3,
                           seed=1, max_wall=120.0)
    assert st["solves"] == 3 * st["runs"] and st["runs"] > 0
    assert st["max_residual"] < 1e-8 and st["p99_ms"] >= st["p50_ms"] > 0


def test_large_run_is_solved_at_full_width_and_same_in_the_mix():
    """A 60x120x84 run (over the large-run threshold) is solved over the whole
    device with the single-system launch of its mesh: its warm-started
    sequence equals the single-system solver's bit for bit, alone and beside
    small runs, and the small runs still finish."""
    eaf = pkg()
    g = gen()
    big = (60, 120, 84, 24)
    rounds = 2
    seq = sequence(big, 5, rounds)
    ref = []
    phi = g.zeros_phi(*big[:3])
    with eaf.CGSolver(*big[:3]) as cg:
        for s in seq:
            res, nit, st = cg.solve(s.arrays(), phi, 200000, 1e-8)
            assert st == 0
            ref.append(phi.copy())
    with eaf.Server() as srv:
        runs = [(srv.open_run(*big[:3]), seq, g.zeros_phi(*big[:3]))]
        for j, d in enumerate(OTHERS[:3]):
            runs.append((srv.open_run(*d[:3]), sequence(d, 70 + j, rounds),
                         g.zeros_phi(*d[:3])))
        mix = solve_rounds(srv, runs, rounds)
    for k in range(rounds):
        assert np.array_equal(mix[0][k], ref[k]), f"round {k} differs"
