"""Moving-domain shift against the reference's own kernels on a B200.

Reference sequence (APTPhaseField::moveDomain, APTPhaseField.cu:678-697):
tip_mvf on PFs_old (ave_x + host scan, PhaseField.cu:382-399); while the tip is at
or above tip_thres: APTcollect_PF (no clear), APTmove_frame, APTcopy_frame;
then APTsetBC3D.  The library does the same in cupf_apt_move_domain.  The
shifted slot state, the z coordinates, the archived alpha layers, the lost area
and the counters must match; stepping on from the shifted state must stay
bit-exact.
"""
import ctypes as C

import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.solver import APTSolver
from tests.helpers import compare_states

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("np_,bc", [(5, "110"), (8, "000")])
def test_move_domain_matches_reference(built, np_, bc):
    import torch
    from oracle import RefGPU
    # front near the top of the window so the shift triggers
    c = cases.line_case(32, 24, 40, num_pf=np_, num_grains=14, seed=5, bc=bc, z0_frac=0.86)
    p = c.params
    ph0, id0 = c.initial_slots()
    pre = 12
    ref = RefGPU(np_)
    ref.check(ref.L.ref_set_params(p))
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    x, y, z, sint, cost = (dev(a) for a in (c.x, c.y, c.z, c.sint, c.cost))
    old_ph, old_id, new_ph, new_id = dev(ph0), dev(id0), dev(ph0), dev(id0)

    def ref_step(n, a_ph, a_id, b_ph, b_id):
        t = np.float32(np.float32(n) * np.float32(p.dt)) * np.float32(p.tau0)
        ref.check(ref.L.ref_set_bc(a_ph.data_ptr(), a_id.data_ptr()))
        ref.check(ref.L.ref_rhs_psi(float(t), x.data_ptr(), y.data_ptr(), z.data_ptr(),
                                    a_ph.data_ptr(), b_ph.data_ptr(), a_id.data_ptr(),
                                    b_id.data_ptr(), sint.data_ptr(), cost.data_ptr(), None, None,
                                    None, None, None, None, 0))

    for n in range(1, pre + 1):  # even count: state back in "old"
        if n % 2:
            ref_step(n, old_ph, old_id, new_ph, new_id)
        else:
            ref_step(n, new_ph, new_id, old_ph, old_id)
    ref.check(ref.L.ref_set_bc(old_ph.data_ptr(), old_id.data_ptr()))
    # moveDomain
    fnz_f = p.fnz + 16
    L = c.length
    z2 = z.clone()
    phi_m = dev(np.zeros(L, np.float32))
    alpha_m = dev(np.zeros(L, np.int32))
    afull = dev(np.zeros(p.fnx * p.fny * fnz_f, np.int32))
    loss = dev(np.zeros(p.num_theta + 64, np.int32))  # padded: the reference may write [-1]
    meanx_d = dev(np.zeros(p.fnz, np.float32))
    meanx_h = np.zeros(p.fnz, np.float32)
    tip = np.array([1], np.int32)
    tip_thres = int(0.8 * p.fnz)
    ref.check(ref.L.ref_tip_mvf(tip.ctypes.data_as(C.POINTER(C.c_int32)), old_ph.data_ptr(),
                                meanx_d.data_ptr(), meanx_h.ctypes.data_as(C.POINTER(C.c_float))))
    move_count = 0
    while tip[0] >= tip_thres:
        ref.check(ref.L.ref_collect(old_ph.data_ptr(), phi_m.data_ptr(), alpha_m.data_ptr(),
                                    old_id.data_ptr()))
        ref.check(ref.L.ref_move_frame(new_ph.data_ptr(), new_id.data_ptr(), z2.data_ptr(),
                                       old_ph.data_ptr(), old_id.data_ptr(), z.data_ptr(),
                                       alpha_m.data_ptr(), afull.data_ptr(),
                                       loss.data_ptr() + 32 * 4, move_count))
        ref.check(ref.L.ref_copy_frame(new_ph.data_ptr(), new_id.data_ptr(), z2.data_ptr(),
                                       old_ph.data_ptr(), old_id.data_ptr(), z.data_ptr()))
        move_count += 1
        tip[0] -= 1
    ref.check(ref.L.ref_set_bc(old_ph.data_ptr(), old_id.data_ptr()))
    torch.cuda.synchronize()
    assert move_count >= 1, "case must trigger at least one shift"
    r_ph, r_id = old_ph.cpu().numpy(), old_id.cpu().numpy()

    with APTSolver(c) as s:
        s.set_slots(ph0, id0, 0)
        s.step(pre)
        tf, mc, moved = s.move_domain(1, tip_thres, 0)
        assert (tf, mc, moved) == (int(tip[0]), move_count, move_count)
        m_ph, m_id = s.get_slots()
        n_id, n_ph, _ = compare_states(p, m_ph, m_id, r_ph, r_id)
        assert (n_id, n_ph) == (0, 0)
        assert np.array_equal(s.get_z().view(np.int32), z.cpu().numpy().view(np.int32))
        af, lo = s.get_archive(fnz_f)
        assert np.array_equal(lo, loss.cpu().numpy()[32:32 + p.num_theta])
        assert np.array_equal(af[:(move_count + 1) * p.fnx * p.fny],
                              afull.cpu().numpy()[:(move_count + 1) * p.fnx * p.fny])
        # keep stepping from the shifted window
        s.step(6)
        m_ph, m_id = s.get_slots()
    for n in range(pre + 1, pre + 7):
        if n % 2:
            ref_step(n, old_ph, old_id, new_ph, new_id)
        else:
            ref_step(n, new_ph, new_id, old_ph, old_id)
    ref.check(ref.L.ref_set_bc(old_ph.data_ptr(), old_id.data_ptr()))
    torch.cuda.synchronize()
    n_id, n_ph, _ = compare_states(p, m_ph, m_id, old_ph.cpu().numpy(), old_id.cpu().numpy())
    assert (n_id, n_ph) == (0, 0)
