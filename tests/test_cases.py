"""Synthetic case builder: derived parameters follow the reference's rounding
(PhaseFieldCpu.cpp:141-172) and the initial state follows initField."""
import numpy as np

from cupf_b200 import cases


def test_derived_parameters_line_constants():
    c = cases.line_case(64, 64, 64, num_pf=5, num_grains=20)
    p = c.params
    # tau0 = beta0*lamd*W0/0.8839, dt = cfl*dx*beta0*W0/tau0 with cfl doubled (R < 0.3 m/s)
    assert abs(p.tau0 - 1.328e-7) / 1.328e-7 < 1e-3
    assert abs(p.dt - 0.03637) < 1e-5
    assert abs(p.lamd - 58.3323) < 1e-3
    assert p.hi == np.float32(1.25)
    assert (p.fnx, p.fny, p.fnz) == (66, 66, 66)
    # UC = G*R: 1 K/um * 0.05 m/s = 0.05 K/us
    assert abs(p.underCoolingRate - 0.05) < 1e-7


def test_float_rounding_matches_reference_formulas():
    d = cases.derive_params(dict(cases.LINE_CONSTANTS, R=0.05))
    f = np.float32
    d0 = f(f(0.347) / f(229.0))
    beta0 = f(1.0 / np.float64(f(f(0.217e6) * f(229.0))))
    lamd = f(0.8839 * np.float64(f(0.1)) / np.float64(d0))
    assert d["d0"] == d0 and d["beta0"] == beta0 and d["lamd"] == lamd
    assert d["cfl"] == f(3.0)


def test_initial_state_and_substrate():
    c = cases.line_case(32, 24, 40, num_pf=6, num_grains=15, seed=4, bc="110")
    p = c.params
    assert c.substrate.shape == (24, 32)
    assert set(np.unique(c.substrate)) <= set(range(1, 16))
    ph, ids = c.initial_slots()
    L = c.length
    # slots 1.. empty, slot 0 holds the substrate grain where phi > LS
    assert np.all(ids[L:] == -1) and np.all(ph[L:] == -1.0)
    solid = ids[:L] > 0
    assert solid.any() and (~solid).any()
    assert np.all(ph[:L][solid] > -0.995)
    # liquid above z0: no ids in the top interior layer
    top = ids[:L].reshape(p.fnz, p.fny, p.fnx)[p.fnz - 2, 1:-1, 1:-1]
    assert np.all(top == -1)


def test_orientation_angles_in_range():
    th = cases.grain_angles(100, 3)
    assert th[0] == 0.0
    assert np.all((th[1:] >= 0) & (th[1:] <= np.pi))


def test_periodic_voronoi_wraps():
    a = cases.voronoi_substrate(40, 40, 12, 2, periodic=True)
    assert a.min() >= 1 and a.max() <= 12
    # periodic: the grain touching the left edge continues across the right edge
    assert len(set(a[:, 0]) & set(a[:, -1])) > 0
