"""Known-answer properties of the library's 3D APT step on a B200 (the cases are
described in tests/known_answers.py): a flat front against a 1-D FP64
integration of the equation, bit-exact mirror symmetry of a two-grain boundary,
bit-exact translation invariance under periodic x, the slot invariants of every
cell after a long run, and the moving frame's bookkeeping (the lost area is the
archived layers' count)."""
import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.solver import APTSolver
from tests import known_answers as ka

pytestmark = pytest.mark.gpu


def _run(c, ph, ids, n, prec="fp32"):
    with APTSolver(c, precision=prec) as s:
        s.set_slots(ph, ids, 0)
        s.step(n)
        return s.get_slots()


@pytest.mark.parametrize("prec,tol_phi,tol_front", [("fp32", 2e-5, 2e-4), ("fp16", 5e-3, 5e-2)])
def test_flat_front_matches_1d_solution(built, prec, tol_phi, tol_front):
    c = ka.flat_front_case(nz_int=64, R=0.2)
    p = c.params
    ph, ids = c.initial_slots()
    n = 400
    a_ph, a_id = _run(c, ph, ids, n, prec)
    ref = ka.front_1d(c, n)[-1]
    cols = [ka.column_of(p, a_ph, a_id, 0, i, j) for i in range(1, p.fnx - 1) for j in range(1, p.fny - 1)]
    if prec == "fp32":
        # round to nearest: every column is the same column bit for bit (16-bit
        # storage rounds stochastically per cell, so its columns differ slightly)
        assert all(np.array_equal(cols[0], col) for col in cols[1:])
    moved = ka.front_position(ref) - ka.front_position(c.phi.reshape(p.fnz, p.fny, p.fnx)[:, 1, 1])
    assert moved > 0.5
    for col in cols:
        assert np.max(np.abs(col[1:-1] - ref[1:-1])) < tol_phi
        assert abs(ka.front_position(col) - ka.front_position(ref)) < tol_front


def test_two_grain_boundary_mirror_symmetry(built):
    c, ph, ids = ka.mirror_case(nx_int=70, ny_int=12, nz_int=20)
    p = c.params
    a_ph, a_id = _run(c, ph, ids, 300)
    m_ph, m_id = ka.mirrored(p, a_ph, a_id)
    assert np.array_equal(m_id, a_id)
    assert np.array_equal(m_ph.view(np.int32), a_ph.view(np.int32))
    L = p.fnx * p.fny * p.fnz
    mid = p.fnx // 2
    lane = a_id[:L].reshape(p.fnz, p.fny, p.fnx)[1:-1, 1:-1, :]
    assert np.all(lane[:, :, mid - 1] == 1) and np.all(lane[:, :, mid] == 2)


def test_translation_invariance_periodic_x(built):
    c = cases.line_case(70, 20, 40, num_pf=5, num_grains=14, seed=9, bc="110", z0_frac=0.4)
    p = c.params
    ph, ids = c.initial_slots()
    s = 13  # not a multiple of the 32-cell tile width
    r_ph, r_id = ka.roll_x(p, ph, s), ka.roll_x(p, ids, s)
    cases.fill_bc(p, r_ph, r_id)
    a_ph, a_id = _run(c, ph, ids, 100)
    b_ph, b_id = _run(c, r_ph, r_id, 100)
    x_ph, x_id = ka.roll_x(p, a_ph, s), ka.roll_x(p, a_id, s)
    cases.fill_bc(p, x_ph, x_id)
    assert np.array_equal(x_id, b_id)
    assert np.array_equal(x_ph.view(np.int32), b_ph.view(np.int32))


def test_slot_invariants_after_long_run(built):
    """Every cell holds at most NUM_PF distinct non-negative ids, ids only from
    the substrate, phi within [-1, 1] where an id is held."""
    c = cases.line_case(64, 64, 64, num_pf=5, num_grains=20, seed=0, bc="110")
    p = c.params
    ph, ids = c.initial_slots()
    a_ph, a_id = _run(c, ph, ids, 1000)
    L = p.fnx * p.fny * p.fnz
    d = a_id.reshape(p.num_pf, L).T
    v = a_ph.reshape(p.num_pf, L).T
    held = d >= 0
    assert np.all((d == -1) | ((d >= 1) & (d <= p.num_theta)))
    srt = np.sort(np.where(held, d, -np.arange(1, p.num_pf + 1)), axis=1)
    assert np.all(srt[:, 1:] != srt[:, :-1])  # no id twice in a cell
    assert np.all(np.abs(v[held]) <= 1.0)
    assert held.any(axis=1).sum() > L // 4


def test_lost_area_is_the_archived_layers(built):
    c = cases.line_case(40, 24, 48, num_pf=5, num_grains=9, seed=1, bc="110", z0_frac=0.86)
    p = c.params
    ph, ids = c.initial_slots()
    with APTSolver(c) as s:
        s.set_slots(ph, ids, 0)
        tip, mc = 1, 0
        for _ in range(30):
            s.step(20)
            tip, mc, _ = s.move_domain(tip, int(0.8 * p.fnz), mc)
        af, loss = s.get_archive(p.fnz * 4 + 8)
    assert mc > 0
    plane = p.fnx * p.fny
    layers = af[plane:plane * (mc + 1)]  # archived layer m sits at (m + 1) * plane
    counts = np.bincount(layers[(layers >= 1) & (layers <= p.num_theta)], minlength=p.num_theta + 1)
    assert np.array_equal(counts[1:], loss)
    assert loss.sum() > 0
