"""eaf_cg_solve_f64_noalloc: the solve for callers that must not allocate.

Some callers cannot allocate device memory: a simulator whose device memory
belongs entirely to its own pool allocator or budget, or code on a
latency-critical path where cudaMalloc/cudaFree would synchronise the GPU.
This entry point takes the caller's device inputs and phi and keeps all of
its working memory in one static device array (EAF_NOALLOC_MAX_CELLS cells).

The test calls it through the C ABI twice in a row (a cold solve, then a
warm-started re-solve that reuses the array left by the first call) and
compares each result with the handle-based eaf_cg_solve_f64_device on the
same inputs. Both run the same kernels with the same launch shape, so the
tolerance is exact equality: iteration count, residual and every phi value.
Besides the two tuned meshes, two meshes outside the tuned table run the
fallback launch rule for small meshes (one cluster of 8 or 16 blocks that
keeps the system in its shared memory), which this entry shares with the
handle entries.
The file is named to be collected last and also passes on its own.
"""
import ctypes

import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu


def _noalloc(lib, s, dev_arrays, phi_dev, max_iter=100000, tol=1e-8):
    res = ctypes.c_double()
    nit = ctypes.c_int()
    ptrs = [ctypes.c_void_p(t.data_ptr()) for t in dev_arrays]
    st = lib.eaf_cg_solve_f64_noalloc(s.nr, s.nth, s.nz, 0, None, *ptrs,
                                      ctypes.c_void_p(phi_dev.data_ptr()), max_iter,
                                      tol, ctypes.byref(res), ctypes.byref(nit))
    return st, res.value, nit.value


@pytest.mark.parametrize("dims,launch", [((12, 24, 16, 8), None), ((18, 36, 24, 8), None),
                                         ((10, 20, 12, 4), (8, 320, 8)),
                                         ((20, 40, 30, 8), (16, 768, 16))])
def test_noalloc_matches_handle_entry_on_two_calls(dims, launch):
    torch = pytest.importorskip("torch")
    eaf = pkg()
    g = gen()
    lib = eaf.load()
    nr, nth, nz, nsph = dims
    mesh = g.make_mesh(nr, nth, nz, nsph, seed=6)
    systems = [g.make_system(nr, nth, nz, nsph, seed=6, resolve=k, mesh=mesh)
               for k in range(2)]
    phi_a = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64, device="cuda")
    phi_b = torch.zeros_like(phi_a)
    with eaf.CGSolver(nr, nth, nz, device=0) as cg:
        for s in systems:
            dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
            torch.cuda.synchronize()
            st_a, res_a, nit_a = _noalloc(lib, s, dev, phi_a)
            res_b, nit_b, st_b = cg.solve(dev, phi_b, 100000, 1e-8, device_ptrs=True)
            assert st_a == 0 and st_b == 0, (st_a, st_b)
            assert res_a < 1e-8
            assert (nit_a, res_a) == (nit_b, res_b)
            assert torch.equal(phi_a, phi_b)
            if launch is not None:
                assert cg.last_launch() == launch


def test_noalloc_refuses_meshes_above_its_limit():
    torch = pytest.importorskip("torch")
    eaf = pkg()
    lib = eaf.load()
    assert eaf._lib.EAF_NOALLOC_MAX_CELLS == 32768
    nr, nth, nz = 35, 70, 50                      # 122,500 cells
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(t.data_ptr())
    res = ctypes.c_double()
    nit = ctypes.c_int()
    st = lib.eaf_cg_solve_f64_noalloc(nr, nth, nz, 0, None, *([p] * 9), 10, 1e-8,
                                      ctypes.byref(res), ctypes.byref(nit))
    assert st == eaf._lib.EAF_EINVAL
    assert b"exceed" in lib.eaf_last_error()
