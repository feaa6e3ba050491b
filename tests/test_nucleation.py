"""Nucleation with a counter-based Philox4x32-10 draw.

CPU: the Philox restatement reproduces the generator's published known-answer
values.  GPU: a liquid-start run (the reference's initial-undercooling phase,
APTPhaseField.cu:779-816) alternating step, nucleation pass, step, is bit-exact
between the CUDA library and the CPU oracle: same nuclei, same grain ids, same
phi, and stepping on from them stays exact.
"""
import numpy as np
import pytest

from cupf_b200 import cases
from oracle import CpuOracle
from tests.helpers import compare_states


def test_philox_known_answers():
    o = CpuOracle()
    assert o.philox((0, 0, 0, 0), (0, 0)) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert o.philox((0xffffffff,) * 4, (0xffffffff,) * 2) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert o.philox((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0)) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def nucl_case(np_=5):
    c = cases.line_case(40, 40, 40, num_pf=np_, num_grains=8, seed=7, bc="111", z0_frac=0.2)
    p = c.params
    p.nuc_rad = np.float32(0.16)
    p.pts_cell = int(np.float32(0.16) / np.float32(np.float32(0.8) * np.float32(0.1)))
    p.nuc_Nmax0 = np.float32(0.1)
    p.nuc_Nmax = np.float32(0.1)
    p.seed = 11
    return c


def test_nucleation_oracle_consistency():
    """CPU only: the status init and a nucleation pass behave as specified."""
    c = nucl_case()
    o = CpuOracle()
    ph, ids = c.initial_slots()
    st = o.nucl_status_init(c.params, ph)
    cd = o.nucl_dims(c.params)
    assert st.size == cd[0] * cd[1] * cd[2] and st.sum() > 0 and st.sum() < st.size
    sph = o.nucleus_table(c.params)
    n = 0
    for it in range(30):
        n += o.nucleate(c, ph, ids, st, sph, 2 * it + 1, use_iuc=True)
    assert n > 0
    assert ids.max() > c.params.num_theta  # new grains got fresh ids


@pytest.mark.gpu
@pytest.mark.parametrize("np_", [5, 8])
def test_nucleation_bit_exact_vs_oracle(built, np_):
    from cupf_b200.solver import APTSolver
    c = nucl_case(np_)
    p = c.params
    o = CpuOracle()
    ph0, id0 = c.initial_slots()
    iters = 40
    with APTSolver(c) as s:
        s.set_slots(ph0, id0, 0)
        s.nucl_init()
        for it in range(iters):
            s.step(1, True)
            total = s.nucleate(True)
            s.step(1, True)
        m_ph, m_id = s.get_slots()
    a_ph, a_id = ph0.copy(), id0.copy()
    b_ph, b_id = ph0.copy(), id0.copy()
    st = o.nucl_status_init(p, a_ph)
    sph = o.nucleus_table(p)
    n = 0
    step = 0
    for it in range(iters):
        for half in range(2):
            step += 1
            t = float(np.float32(np.float32(step) * np.float32(p.dt)) * np.float32(p.tau0))
            o.set_bc(p, a_ph, a_id)
            o.rhs_psi_f32(c, t, a_ph, a_id, b_ph, b_id, use_iuc=True)
            a_ph, b_ph = b_ph, a_ph
            a_id, b_id = b_id, a_id
            if half == 0:
                n += o.nucleate(c, a_ph, a_id, st, sph, step, use_iuc=True)
    o.set_bc(p, a_ph, a_id)
    assert total == n and n > 0
    n_id, n_ph, d = compare_states(p, m_ph, m_id, a_ph, a_id)
    assert (n_id, n_ph) == (0, 0), (n_id, n_ph, d)
