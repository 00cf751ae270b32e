"""Parity of the device post-CG corrections (src/mod_pressure_3d.f90:333-397,
correct_velocities :689-746) with the oracle.

No reduction is involved: every output array -- fluxes, link flags (their
theta halos), both phases' velocities and the pressure -- must equal the
oracle's BIT FOR BIT over the whole halo layout.
"""
import ctypes

import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu


def run_gpu(f, device=False):
    eaf = pkg()
    out = f.copy()
    with eaf.CGSolver(f.nr, f.nth, f.nz) as cg:
        if device:
            import torch
            dev = out.copy()
            keep = []
            for k, v in list(dev.__dict__.items()):
                if isinstance(v, np.ndarray):
                    t = torch.from_numpy(v).cuda()
                    keep.append(t)
                    setattr(dev, k, t)
            cg.pressure_correct(dev, device_ptrs=True)
            for k, v in dev.__dict__.items():
                if hasattr(v, "data_ptr"):
                    setattr(out, k, v.cpu().numpy())
        else:
            cg.pressure_correct(out)
        t = cg.last_timing()
    return out, t


def run_oracle(f):
    import oracle
    out = f.copy()
    oracle.pressure_correct(out)
    return out


def assert_same(a, b):
    for name, arr in a.outputs().items():
        assert np.array_equal(arr, b.outputs()[name]), name


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 3), (3, 4, 3), (1, 3, 1),
                                  (12, 24, 16)])
@pytest.mark.parametrize("has_gas", [True, False])
def test_pcorr_bitwise_small(dims, has_gas):
    f = gen().make_pcorr_fields(*dims, seed=17, has_gas=has_gas, sealed_frac=0.2)
    a, t = run_gpu(f)
    assert_same(a, run_oracle(f))
    assert t["kernels"] == 3


def test_pcorr_bitwise_production_mesh():
    f = gen().make_pcorr_fields(60, 120, 84, seed=3)
    a, _ = run_gpu(f)
    assert_same(a, run_oracle(f))


def test_pcorr_device_pointers_match_host_path():
    f = gen().make_pcorr_fields(9, 14, 7, seed=5)
    a, _ = run_gpu(f)
    b, _ = run_gpu(f, device=True)
    assert_same(a, b)


def test_pcorr_missing_gas_fields_are_an_error():
    eaf = pkg()
    f = gen().make_pcorr_fields(3, 4, 2, seed=1, has_gas=True)
    f.gas_ur = None
    with eaf.CGSolver(3, 4, 2) as cg:
        with pytest.raises((eaf.EafError, TypeError)):
            cg.pressure_correct(f)
    lib = eaf._lib.load()
    h = ctypes.c_void_p()
    assert lib.eaf_cg_create(ctypes.byref(h), 3, 4, 2, 0) == 0
    try:
        assert lib.eaf_pressure_correct_f64(h, None) == eaf._lib.EAF_EINVAL
    finally:
        lib.eaf_cg_destroy(h)
