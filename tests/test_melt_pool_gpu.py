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


def analytic_melt_pool_case():
    """The analytic paraboloid pool (thermalType 5) in miniature, with the same
    uniformly cooling nucleation table and nucleus size as melt_pool_case."""
    c = cases.meltpool_case(32, 24, 80, num_pf=8, num_grains=12, seed=4, r0=8.0, V=0.5,
                            mp_len=12.0, G=2.0, front_frac=0.8)
    p = c.params
    p.nuc_rad = F32(0.16)
    p.pts_cell = int(F32(0.16) / F32(F32(0.8) * F32(0.1)))
    p.nuc_Nmax0 = F32(5.0)
    p.nuc_Nmax = F32(5.0)
    p.undcool_mean = F32(2.0)
    p.undcool_std = F32(0.5)
    p.seed = 3
    p.Nt = 2
    c.t_mac = np.array([0.0, 1e-6], F32)
    T = -4.3e6 * c.t_mac.astype(np.float64)
    c.T_3D = np.repeat(T, p.Nx * p.Ny * p.Nz).astype(F32)
    return c


def test_melt_pool_moving_domain_with_nucleation(built):
    run_and_compare(melt_pool_case())


def test_analytic_melt_pool_moving_domain_with_nucleation(built):
    run_and_compare(analytic_melt_pool_case())


def run_and_compare(c):
    from oracle import CpuOracle
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


def test_analytic_paraboloid_step_bit_exact_vs_oracle(built):
    """thermalType 5 (the library's analytic paraboloid pool, no counterpart in
    the reference) on a larger window: the device step against the oracle's
    restatement of the same operations, bit for bit, 40 steps."""
    from oracle import CpuOracle
    c = cases.meltpool_case(48, 40, 72, num_pf=8, num_grains=25, seed=9, r0=6.0, V=0.8,
                            mp_len=10.0, G=3.0, front_frac=0.6)
    ph0, id0 = c.initial_slots()
    with APTSolver(c) as s:
        s.set_slots(ph0, id0, 0)
        s.step(40)
        m_ph, m_id = s.get_slots()
    o_ph, o_id, _, _ = CpuOracle().run_f32(c, ph0, id0, 40)
    n_id, n_ph, d = compare_states(c.params, m_ph, m_id, o_ph, o_id)
    assert (n_id, n_ph) == (0, 0), (n_id, n_ph, d)


def test_analytic_paraboloid_fp16_against_fp64(built):
    """16-bit storage under the analytic pool (FP64 time and heights in the
    thermal model) against the FP64 oracle: the solid volume and interface area
    within 1e-3 relative after 300 steps."""
    from oracle import CpuOracle, interface_qois
    c = cases.meltpool_case(40, 32, 64, num_pf=8, num_grains=20, seed=2, r0=5.0, V=0.6,
                            mp_len=8.0, G=3.0, front_frac=0.6)
    ph0, id0 = c.initial_slots()
    ref = CpuOracle().run_f64(c, ph0.astype(np.float64), id0, 300)
    q64 = interface_qois(c.params, ref[0])
    with APTSolver(c, precision="fp16") as s:
        s.set_slots(ph0, id0, 0)
        s.step(300)
        q = s.qoi_sums()
    assert abs(q[0] - q64[0]) / q64[0] < 1e-3, (q, q64)
    assert abs(q[1] - q64[1]) / q64[1] < 1e-3, (q, q64)


def test_full_window_paraboloid_table_bit_exact_vs_reference(built):
    """The melt-pool configuration's full window, 256 x 256 x 768 interior, 400
    grains, NUM_PF = 8, under the reference's own pool model (the paraboloid
    table of thermalType 4, APTPhaseField.cu:308-325, moving at 0.5 m/s) with
    nucleation off: 200 steps of the library against the reference kernels,
    grain ids and phi bit for bit on every interior and face-halo cell."""
    from tests.helpers import face_mask, run_cupf, run_reference_gpu
    c = cases.paraboloid_case(256, 256, 768, num_pf=8, num_grains=400, seed=0, V=0.5,
                              z0_frac=0.75)
    p = c.params
    ref_ph, ref_id = run_reference_gpu(c, 200)
    my_ph, my_id = run_cupf(c, 200)
    m = face_mask(p)
    L = c.length
    n_id = n_ph = 0
    for q in range(p.num_pf):
        sl = slice(q * L, (q + 1) * L)
        n_id += int(np.count_nonzero(my_id[sl][m] != ref_id[sl][m]))
        n_ph += int(np.count_nonzero(my_ph[sl][m].view(np.int32) != ref_ph[sl][m].view(np.int32)))
    assert (n_id, n_ph) == (0, 0), (n_id, n_ph)
