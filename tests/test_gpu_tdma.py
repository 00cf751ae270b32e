"""Parity of the device line-by-line TDMA and transport residual with the
oracle (tdma_3d_mpi, compute_residual_3d_mpi; src/mod_solver_3d.f90).

The sweeps are integer-order-exact restatements of a sequential algorithm
(no reductions), so the device result must equal the oracle's BIT FOR BIT
over the whole halo-layout phi: interior, refreshed theta halos and the
untouched r/z halos. The residual's two sums are associated as the CG dots;
against the oracle in that association (plan) it is bitwise, against the
reference's sequential sum within 1e-13 relative.
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu


def rand_phi(dims, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, 1.0, size=gen().halo_shape(*dims))


def run_gpu(s, phi, n_sweep, device=False):
    eaf = pkg()
    out = phi.copy()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        if device:
            import torch
            dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
            p = torch.from_numpy(out).cuda()
            cg.tdma(dev, p, n_sweep, device_ptrs=True)
            out = p.cpu().numpy()
        else:
            cg.tdma(s.arrays(), out, n_sweep)
        timing = cg.last_timing()
    return out, timing


def run_oracle(s, phi, n_sweep):
    import oracle
    out = phi.copy()
    oracle.tdma_3d(s, out, n_sweep)
    return out


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 3), (1, 5, 2), (4, 2, 1),
                                  (5, 3, 4), (3, 7, 1), (12, 24, 16)])
@pytest.mark.parametrize("n_sweep", [1, 3])
def test_tdma_bitwise_small(dims, n_sweep):
    g = gen()
    s = g.make_transport_system(*dims, seed=21, trivial_frac=0.1)
    phi0 = rand_phi(dims, 4)
    a, _ = run_gpu(s, phi0, n_sweep)
    b = run_oracle(s, phi0, n_sweep)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("dims,n_sweep", [((18, 36, 24), 2), ((35, 70, 50), 1),
                                          ((60, 120, 84), 1)])
def test_tdma_bitwise_production_meshes(dims, n_sweep):
    g = gen()
    s = g.make_transport_system(*dims, seed=5)
    phi0 = rand_phi(dims, 6)
    a, _ = run_gpu(s, phi0, n_sweep)
    b = run_oracle(s, phi0, n_sweep)
    assert np.array_equal(a, b)


def test_tdma_pressure_operator_bitwise():
    """The symmetric pressure system (identity pin row, folded links)."""
    g = gen()
    s = g.make_system(*g.SMOKE, seed=2)
    phi0 = g.zeros_phi(12, 24, 16)
    a, _ = run_gpu(s, phi0, 4)
    b = run_oracle(s, phi0, 4)
    assert np.array_equal(a, b)


def test_tdma_device_pointers_match_host_path():
    g = gen()
    s = g.make_transport_system(9, 14, 7, seed=3)
    phi0 = rand_phi((9, 14, 7), 1)
    a, _ = run_gpu(s, phi0, 2)
    b, _ = run_gpu(s, phi0, 2, device=True)
    assert np.array_equal(a, b)


def test_tdma_zero_sweeps_leaves_phi():
    g = gen()
    s = g.make_transport_system(4, 5, 3, seed=1)
    phi0 = rand_phi((4, 5, 3), 2)
    a, t = run_gpu(s, phi0, 0)
    assert np.array_equal(a, phi0) and t["kernels"] == 0


def test_tdma_converges_like_the_oracle():
    """Many sweeps of a diagonally dominant system: same bits all the way."""
    g = gen()
    s = g.make_transport_system(8, 12, 6, seed=5, sp_frac=0.3)
    phi0 = g.zeros_phi(8, 12, 6)
    a, _ = run_gpu(s, phi0, 60)
    b = run_oracle(s, phi0, 60)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("dims", [(1, 1, 1), (7, 9, 5), (35, 70, 50)])
def test_residual_matches_oracle(dims):
    import oracle
    eaf = pkg()
    g = gen()
    s = g.make_transport_system(*dims, seed=8, trivial_frac=0.2)
    phi = rand_phi(dims, 9)
    with eaf.CGSolver(*dims) as cg:
        r = cg.residual(s.arrays(), phi)
        plan = cg.last_launch()
    assert r == oracle.residual_3d(s, phi, plan=plan)
    r_seq = oracle.residual_3d(s, phi)
    assert abs(r - r_seq) <= 1e-13 * r_seq


def test_residual_all_identity_rows_is_zero():
    eaf = pkg()
    g = gen()
    s = g.make_transport_system(3, 4, 2, seed=1, trivial_frac=1.0)
    with eaf.CGSolver(3, 4, 2) as cg:
        assert cg.residual(s.arrays(), rand_phi((3, 4, 2), 3)) == 0.0


@pytest.mark.parametrize("seed", [1, 20260101])
def test_sweep_division_matches_ieee_division(seed):
    """The sweeps divide by a precomputed reciprocal plus one FMA correction
    (Markstein's theorem); it must give the bits of `/` on every pair."""
    import ctypes
    lib = pkg()._lib.load()
    bad, fast = ctypes.c_longlong(), ctypes.c_longlong()
    n = 1 << 26
    assert lib.eaf_diag_div_check(0, n, seed, ctypes.byref(bad), ctypes.byref(fast)) == 0
    assert bad.value == 0
    assert fast.value > n // 2
