"""CPU tests of the oracle: known answers of the scheme's algebra.

The reference ships no tests or expected outputs; these properties follow
from the scheme itself and hold exactly (bit for bit) or to round-off:
  * lake at rest stays at rest (hydrostatic reconstruction,
    GPU/VolumeSolver.cu:37-40, with the pressure source
    GPU/Reconstructor.cu:197,274);
  * with walls, sum(h) is conserved to round-off on a fully wet grid
    (Dm + Dp = F0 - F1 + df = 0, GPU/VolumeSolver.cu:122-126);
  * transpose and mirror symmetry of symmetric data are exact;
  * a 1 x N run equals the transposed N x 1 run (x and y code paths);
  * dt follows MinReduction: float-rounded above 4096 cells.
"""
import numpy as np
import pytest

import oracle
from tsuner_b200 import workloads as W
from tsuner_b200.abi import make_params, make_switches


def flat_hump(n, dx=10.0, depth=10.0, amp=1.0, sigma=60.0, nx=None):
    nx = nx or n
    x = W.centres(nx, dx)[None, :]
    y = W.centres(n, dx)[:, None]
    V = np.zeros((5, n, nx))
    V[3] = depth
    eta = amp * np.exp(-((x - 0.5 * nx * dx) ** 2 + (y - 0.5 * n * dx) ** 2) / (2 * sigma ** 2))
    V[0] = depth + eta
    return make_params(nx, n, dx, dx), V


@pytest.mark.parametrize("order", [1, 2])
def test_lake_at_rest_exact(order):
    w = W.hump(48, 40, 10.0, amp=0.0)
    sw = make_switches(order=order, wbc=1)
    r = oracle.OracleRun(w.p, sw, w.V, w.mask)
    V0 = r.V.copy()
    r.run(40)
    assert np.array_equal(r.V[0], V0[0])
    assert np.array_equal(r.V[3], V0[3])
    assert np.abs(r.V[1:3]).max() == 0.0


def test_mass_conservation_walls():
    p, V = flat_hump(48)
    r = oracle.OracleRun(p, make_switches(order=2, wbc=1), V)
    m0 = r.V[0].sum()
    r.run(150)
    assert abs(r.V[0].sum() - m0) / m0 < 1e-13
    assert np.isfinite(r.V).all()


def test_transpose_symmetry_exact():
    p, V = flat_hump(40)
    r = oracle.OracleRun(p, make_switches(order=2, wbc=1), V)
    r.run(60)
    assert np.array_equal(r.V[0], r.V[0].T)
    assert np.array_equal(r.V[1], r.V[2].T)


def test_mirror_symmetry_exact():
    p, V = flat_hump(40)
    r = oracle.OracleRun(p, make_switches(order=2, wbc=1), V)
    r.run(60)
    assert np.array_equal(r.V[0], r.V[0][::-1, :])
    assert np.array_equal(r.V[0], r.V[0][:, ::-1])


@pytest.mark.parametrize("order", [1, 2])
def test_1d_x_equals_1d_y(order):
    n = 64
    x = W.centres(n, 10.0)
    H = 5.0 + 0.02 * x
    h = np.maximum(H + 1.5 * np.exp(-((x - 200.0) ** 2) / (2 * 40.0 ** 2)), 0.0)
    sw = make_switches(order=order, wbc=1)
    Vx = np.zeros((5, 1, n))
    Vx[0, 0], Vx[3, 0] = h, H
    Vy = np.zeros((5, n, 1))
    Vy[0, :, 0], Vy[3, :, 0] = h, H
    rx = oracle.OracleRun(make_params(n, 1, 10.0, 10.0), sw, Vx)
    ry = oracle.OracleRun(make_params(1, n, 10.0, 10.0), sw, Vy)
    rx.run(80)
    ry.run(80)
    assert np.array_equal(rx.V[0, 0], ry.V[0, :, 0])
    assert np.array_equal(rx.V[1, 0], ry.V[2, :, 0])
    assert np.array_equal(rx.V[3, 0], ry.V[3, :, 0])


def test_dt_float_rounding_above_4096_cells():
    w = W.hump(65, 64, 10.0)  # 4160 cells > 4096
    dt = oracle.initial_dt(w.p, w.sw, w.V)
    assert dt == float(np.float32(dt))
    w2 = W.hump(64, 64, 10.0)  # exactly 4096: exact double min
    dt2 = oracle.initial_dt(w2.p, w2.sw, w2.V)
    h = w2.V[0]
    c = np.sqrt(9.81 * h)
    with np.errstate(divide="ignore"):
        ref = np.min(0.9 * 0.5 * np.minimum(10.0 / c, 10.0 / c))
    assert dt2 == ref


@pytest.mark.parametrize("variant", [
    dict(order=1, wbc=1), dict(order=2, wbc=0), dict(order=2, wbc=2),
    dict(order=2, wbc=1, bedload=0, suspension=0), dict(order=2, wbc=1, bedload_law=1, grass_ag=1e-3),
    dict(order=2, wbc=1, rk=0), dict(order=1, wbc=1, rk=0), dict(order=2, wbc=1, manning=1),
])
def test_switch_variants_run(variant):
    w = W.hump(40, 32, 10.0, sigma=80.0)
    r = oracle.OracleRun(w.p, make_switches(**variant), w.V, w.mask)
    r.run(30)
    assert np.isfinite(r.V).all()
    assert (r.V[0] >= 0).all()


def test_muscl_hancock_state_carried_across_runs():
    """MUSCL-Hancock keeps the reference's unfiltered working state Vk from
    step to step (GPU/Volume_kernel.cu:283-299): runs split over several calls
    equal one run, and the result differs from the RK2 scheme's."""
    w = W.nwave_shelf(40, 30, 40.0, slr=0.5, amp=2.0, period=200.0, t_series=150.0)
    sw = make_switches(order=2, wbc=1, read_files=1, rk=0)
    one = oracle.OracleRun(w.p, sw, w.V, w.mask, w.CC, w.tCC)
    one.run(25)
    parts = oracle.OracleRun(w.p, sw, w.V, w.mask, w.CC, w.tCC)
    for n in (3, 10, 12):
        parts.run(n)
    assert np.array_equal(one.V, parts.V) and one.t.value == parts.t.value
    assert not np.array_equal(one.Vk, one.V)  # the filter rounds; Vk keeps the unfiltered values
    rk2 = oracle.OracleRun(w.p, make_switches(order=2, wbc=1, read_files=1), w.V, w.mask, w.CC, w.tCC)
    rk2.run(25)
    assert not np.array_equal(one.V, rk2.V)


def test_manning_branch_multiplies_momentum():
    """GPU/Reconstructor.cu:47-50 as written: q *= dt FR^2 |u| / h^(4/3), so on
    a wet grid every step scales the carried momentum by that (small) factor
    before the fluxes act, and momentum does not build up as with Chezy."""
    w = W.hump(30, 24, 10.0, sigma=60.0)
    sw = make_switches(order=1, wbc=1, manning=1, bedload=0, suspension=0)
    r = oracle.OracleRun(w.p, sw, w.V, w.mask)
    r.run(5)
    rc = oracle.OracleRun(w.p, make_switches(order=1, wbc=1, bedload=0, suspension=0), w.V, w.mask)
    rc.run(5)
    assert np.isfinite(r.V).all()
    assert np.abs(r.V[1]).max() < 0.5 * np.abs(rc.V[1]).max()


def test_boundary_series_nwave_enters():
    w = W.nwave_shelf(64, 48, 50.0, slr=0.5, amp=2.0, period=300.0, t_series=400.0)
    r = oracle.OracleRun(w.p, w.sw, w.V, w.mask, w.CC, w.tCC)
    r.run(60)
    assert np.isfinite(r.V).all()
    eta = r.V[0] - r.V[3]
    wet = r.V[0] > 1e-3
    assert eta[:, :4][wet[:, :4]].max() > 0.6  # the crest has entered from the west


def test_generators_are_deterministic():
    a = W.gaussian_noise(1, 10)
    assert np.allclose(a[:4], W.gaussian_noise(1, 4))
    w1 = W.nwave_shelf(64, 64, 5.0)
    w2 = W.nwave_shelf(64, 64, 5.0)
    assert np.array_equal(w1.V, w2.V) and np.array_equal(w1.mask, w2.mask)
    assert (w1.mask == 0).any()
    dry = (w1.V[0] == 0).mean()
    assert 0.15 < dry < 0.25
