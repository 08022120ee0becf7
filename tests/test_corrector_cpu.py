"""CPU: host-side helpers of the learned-corrector pipeline (no GPU): the
coarse site is the block average of the fine one, sources are seeded and in
their stated ranges, and the error metric counts the cells wet in either
map."""
import numpy as np

from tsuner_b200 import corrector as K


def test_block_mean_and_site():
    a = np.arange(16, dtype=np.float64).reshape(4, 4)
    m = K.block_mean(a, 2)
    assert m.shape == (2, 2)
    assert np.array_equal(m, np.array([[2.5, 4.5], [10.5, 12.5]]))
    site = K.make_site(n=64, factor=4, dx=10.0, slr=0.5, seed=5)
    assert site.H.shape == (64, 64) and site.Hc.shape == (16, 16)
    assert np.allclose(site.Hc, K.block_mean(site.H, 4))
    # coarse mask: a coarse cell is erodible only if all its fine cells are
    fine_min = site.mask.reshape(16, 4, 16, 4).min(axis=(1, 3))
    assert np.array_equal(site.maskc, fine_min)
    # the shelf is partly dry above the raised sea level
    assert 0.05 < np.mean(site.H + site.slr < 0) < 0.5


def test_sources_are_seeded_and_in_range():
    a = K.make_sources(50, seed=11)
    b = K.make_sources(50, seed=11)
    c = K.make_sources(50, seed=12)
    assert a == b and a != c
    amp = np.array([s[0] for s in a])
    per = np.array([s[1] for s in a])
    assert amp.min() >= 1.0 and amp.max() <= 5.0
    assert per.min() >= 200.0 and per.max() <= 600.0


def test_error_metric():
    truth = np.zeros((1, 2, 4, 4), np.float32)
    truth[0, 0, :2] = 1.0  # wet half
    ph = truth[:, 0].copy()
    ph[0, 0, 0] += 0.5      # one wet cell off by 0.5
    ph[0, 3, 3] = 0.25      # a cell the truth keeps dry
    pb = np.full((1, 4, 4), 0.1, np.float32)
    e = K.errors((ph, pb), truth)
    wet = 9  # 8 wet in the truth + 1 wet only in the prediction
    assert np.isclose(e["hmax_rmse_m"], np.sqrt((0.25 + 0.0625) / wet))
    assert np.isclose(e["hmax_linf_m"], 0.5)
    assert np.isclose(e["db_rmse_m"], 0.1)
    ph[0, 3, 0] = -0.5      # a negative maximum depth counts as an error
    e = K.errors((ph, pb), truth)
    assert np.isclose(e["hmax_rmse_m"], np.sqrt((0.25 + 0.0625 + 0.25) / 10))
    region = truth[:, 0] > 0  # an explicit region sets the denominator
    e = K.errors((ph, pb), truth, region)
    assert np.isclose(e["hmax_rmse_m"], np.sqrt(0.25 / 8)) and np.isclose(e["hmax_linf_m"], 0.5)
