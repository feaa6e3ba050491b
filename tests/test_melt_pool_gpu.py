"""The moving-domain melt-pool configuration with nucleation, in miniature, on a
B200 against the CPU oracle.

The reference's evolve for a line run with nucleation (APTPhaseField.cu:843-946)
alternates: step, nucleation pass (:866-870), every TIPP steps the moving-domain
check and shift (:884-899, moveDomain :678-697), step.  Here the undercooling is
the paraboloid table of thermalType 4 (:308-325) shifted by V t, nuclei come from
the 4-D temperature table (a uniformly cooling melt), and the front sits high
enough in the window for the frame to move.  Every piece is checked bit for bit:
slot state, z coordinates, archived layers, lost area, nuclei, counters.
"""
import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.solver import APTSolver
from tests.helpers import compare_states

pytestmark = pytest.mark.gpu

F32 = np.float32
TIPP = 20


def melt_pool_case():
    c = cases.paraboloid_case(32, 24, 80, num_pf=8, num_grains=12, seed=4, V=0.5, z0_frac=0.8)
    p = c.params
    p.nuc_rad = F32(0.16)
    p.pts_cell = int(F32(0.16) / F32(F32(0.8) * F32(0.1)))
    p.nuc_Nmax0 = F32(5.0)
    p.nuc_Nmax = F32(5.0)
    p.seed = 3
    # uniform melt cooling at 4.3e6 K/s on the psi table's macro grid, two time points
    p.Nt = 2
    c.t_mac = np.array([0.0, 1e-6], F32)
    T = -4.3e6 * c.t_mac.astype(np.float64)
    c.T_3D = np.repeat(T, p.Nx * p.Ny * p.Nz).astype(F32)
    return c


def test_melt_pool_moving_domain_with_nucleation(built):
    from oracle import CpuOracle
    c = melt_pool_case()
    p = c.params
    L = p.fnx * p.fny * p.fnz
    thres = int(0.8 * p.fnz)
    iters = 60
    ph0, id0 = c.initial_slots()

    with APTSolver(c) as s:
        s.set_slots(ph0, id0, 0)
        s.nucl_init()
        tip, mc, moved_total, total = 1, 0, 0, 0
        for it in range(iters):
            s.step(1)
            total = s.nucleate(False)
            if (2 * it + 2) % TIPP == 0:
                tip, mc, moved = s.move_domain(tip, thres, mc)
                moved_total += moved
            s.step(1)
        m_ph, m_id = s.get_slots()
        m_z = s.get_z()
        m_af, m_loss = s.get_archive(p.fnz + 8)

    o = CpuOracle()
    a_ph, a_id = ph0.copy(), id0.copy()
    b_ph, b_id = ph0.copy(), id0.copy()
    st = o.nucl_status_init(p, a_ph)
    sph = o.nucleus_table(p)
    phi_m, alpha_m = np.zeros(L, F32), np.zeros(L, np.int32)
    z = c.z.copy()
    afull = np.zeros(p.fnx * p.fny * (p.fnz + 8), np.int32)
    loss = np.zeros(p.num_theta, np.int32)
    o_tip, o_mc, n, step = 1, 0, 0, 0

    def ostep():
        nonlocal a_ph, a_id, b_ph, b_id, step
        step += 1
        t = float(F32(F32(step) * F32(p.dt)) * F32(p.tau0))
        o.set_bc(p, a_ph, a_id)
        o.rhs_psi_f32(c, t, a_ph, a_id, b_ph, b_id)
        a_ph, b_ph = b_ph, a_ph
        a_id, b_id = b_id, a_id

    for it in range(iters):
        ostep()
        n += o.nucleate(c, a_ph, a_id, st, sph, step, use_iuc=False)
        if (2 * it + 2) % TIPP == 0:
            o.set_bc(p, a_ph, a_id)
            o_tip, _ = o.tip_scan(p, a_ph, o_tip)
            while o_tip >= thres:
                o.collect(p, a_ph, a_id, phi_m, alpha_m)
                o.move_frame(p, a_ph, a_id, z, alpha_m, afull, loss, o_mc)
                b_ph[:], b_id[:] = a_ph, a_id  # both buffers hold the shifted state
                c.z = z.copy()                 # the thermal model reads the moved z
                o_tip -= 1
                o_mc += 1
        ostep()
    o.set_bc(p, a_ph, a_id)

    assert total == n and n > 0
    assert (tip, mc) == (o_tip, o_mc) and mc == moved_total and mc > 0
    assert np.array_equal(m_z, z)
    assert np.array_equal(m_loss, loss)
    plane = p.fnx * p.fny
    assert np.array_equal(m_af[:plane * (mc + 2)], afull[:plane * (mc + 2)])
    n_id, n_ph, d = compare_states(p, m_ph, m_id, a_ph, a_id)
    assert (n_id, n_ph) == (0, 0), (n_id, n_ph, d)
