"""Properties of the seeded synthetic pressure systems (eafgen)."""
import numpy as np
import pytest

from conftest import gen


@pytest.mark.parametrize("dims", [(12, 24, 16, 8), (18, 36, 24, 8), (5, 7, 3, 2)])
def test_symmetric_links_and_walls(dims):
    g = gen()
    s = g.make_system(*dims, seed=1)
    I = g.interior
    nr = dims[0]
    aW, aE, aS, aN, aB, aT = (I(a) for a in (s.aW, s.aE, s.aS, s.aN, s.aB, s.aT))
    assert np.array_equal(aW[:, :, 1:], aE[:, :, :-1])
    assert not aW[:, :, 0].any() and not aE[:, :, nr - 1].any()
    assert np.array_equal(aS, np.roll(aN, 1, axis=1))
    assert np.array_equal(aB[1:], aT[:-1])
    assert not aB[0].any() and not aT[-1].any()


def test_pin_is_identity_and_folded():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    I = g.interior
    nr, nth = 12, 24
    assert I(s.aP)[0, 0, nr - 1] == 1.0 and I(s.Su)[0, 0, nr - 1] == 0.0
    for a in (s.aW, s.aE, s.aS, s.aN, s.aB, s.aT):
        assert I(a)[0, 0, nr - 1] == 0.0
    assert I(s.aE)[0, 0, nr - 2] == 0.0
    assert I(s.aN)[0, nth - 1, nr - 1] == 0.0
    assert I(s.aS)[0, 1, nr - 1] == 0.0
    assert I(s.aB)[1, 0, nr - 1] == 0.0
    # neighbours keep the folded term in aP: strictly diagonally dominant
    nb = I(s.aW) + I(s.aE) + I(s.aS) + I(s.aN) + I(s.aB) + I(s.aT)
    assert I(s.aP)[0, 0, nr - 2] > nb[0, 0, nr - 2]


def test_rhs_zero_mean_and_halos_zero():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    assert abs(g.interior(s.Su).sum()) < 1e-15
    for a in s.arrays():
        h = a.copy()
        g.interior(h)[...] = 0
        assert not h.any()


def test_deterministic_and_resolves_differ():
    g = gen()
    a = g.make_system(*g.SMOKE, seed=0)
    b = g.make_system(*g.SMOKE, seed=0)
    c = g.make_system(*g.SMOKE, seed=0, resolve=0)
    for x, y in zip(a.arrays(), b.arrays()):
        assert np.array_equal(x, y)
    assert not np.array_equal(a.aP, c.aP) and not np.array_equal(a.Su, c.Su)
    ratio = g.interior(c.aP)[5:, 5:, 2:-2] / g.interior(a.aP)[5:, 5:, 2:-2]
    assert ratio.min() > 0.85 and ratio.max() < 1.2


def test_density_fields():
    g = gen()
    m = g.make_mesh(*g.SMOKE, seed=0)
    vals = set(np.unique(m.rho).tolist())
    assert vals <= {g.RHO_STEEL, g.RHO_GAS, g.RHO_SCRAP}
    assert g.RHO_STEEL in vals and g.RHO_GAS in vals
    assert m.abar.min() >= 1e2 and m.abar.max() <= 1e4


def test_fastdiv_model():
    """Host model of the device FastDiv (cg_common.cuh) against //."""
    rng = np.random.default_rng(0)
    for d in list(range(1, 300)) + [1023, 4096, 7200, 60 * 120, 2**20 + 7]:
        s = 0
        while (1 << s) < d:
            s += 1
        m = ((1 << 32) * ((1 << s) - d)) // d + 1
        assert m < (1 << 32)
        ns = np.concatenate([np.arange(0, 5000), rng.integers(0, 2**31 - 1, 4000),
                             np.array([2**31 - 1, 2**31 - 2])]).astype(np.uint64)
        q = (((ns * np.uint64(m)) >> np.uint64(32)) + ns) >> np.uint64(s)
        assert np.array_equal(q, ns // np.uint64(d)), d
