"""Known-answer properties of the 3D APT step on the CPU oracle: the flat front
of one grain against a 1-D FP64 integration of the same equation, the mirror
symmetry of a two-grain boundary, and translation invariance under periodic x
(the cases are described in tests/known_answers.py)."""
import numpy as np

from cupf_b200 import cases
from oracle import CpuOracle
from tests import known_answers as ka


def test_flat_front_matches_1d_solution():
    c = ka.flat_front_case(nz_int=48)
    p = c.params
    o = CpuOracle()
    ph, ids = c.initial_slots()
    n = 150
    a_ph, a_id = o.run_f64(c, ph, ids, n)
    ref = ka.front_1d(c, n)[-1]
    # every column of the 3D state is the same column
    cols = [ka.column_of(p, a_ph, a_id, 0, i, j) for i in range(1, p.fnx - 1) for j in range(1, p.fny - 1)]
    assert all(np.array_equal(cols[0], col) for col in cols[1:])
    assert np.max(np.abs(cols[0][1:-1] - ref[1:-1])) < 1e-9
    assert abs(ka.front_position(cols[0]) - ka.front_position(ref)) < 1e-8
    # slot 1 never receives an id (one grain)
    L = p.fnx * p.fny * p.fnz
    assert np.all(a_id[L:2 * L] == -1)


def test_two_grain_boundary_mirror_symmetry():
    c, ph, ids = ka.mirror_case()
    p = c.params
    o = CpuOracle()
    a_ph, a_id, _, _ = o.run_f32(c, ph, ids, 40)
    m_ph, m_id = ka.mirrored(p, a_ph, a_id)
    assert np.array_equal(m_id, a_id)
    assert np.array_equal(m_ph.view(np.int32), a_ph.view(np.int32))
    # the boundary has not moved: the middle columns still belong to their own grains
    L = p.fnx * p.fny * p.fnz
    mid = p.fnx // 2
    lane = a_id[:L].reshape(p.fnz, p.fny, p.fnx)[1:-1, 1:-1, :]
    assert np.all(lane[:, :, mid - 1] == 1) and np.all(lane[:, :, mid] == 2)


def test_translation_invariance_periodic_x():
    c = cases.line_case(24, 8, 16, num_pf=4, num_grains=5, seed=2, bc="110", z0_frac=0.4)
    p = c.params
    o = CpuOracle()
    ph, ids = c.initial_slots()
    s = 7
    r_ph, r_id = ka.roll_x(p, ph, s), ka.roll_x(p, ids, s)
    cases.fill_bc(p, r_ph, r_id)
    a_ph, a_id, _, _ = o.run_f32(c, ph, ids, 30)
    b_ph, b_id, _, _ = o.run_f32(c, r_ph, r_id, 30)
    x_ph, x_id = ka.roll_x(p, a_ph, s), ka.roll_x(p, a_id, s)
    cases.fill_bc(p, x_ph, x_id)
    assert np.array_equal(x_id, b_id)
    assert np.array_equal(x_ph.view(np.int32), b_ph.view(np.int32))
