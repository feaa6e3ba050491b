"""Full (non-APT, -a) phase-field mode on the GPU: the library's dense step against
the reference's own PhaseField.cu kernels compiled for sm_100a (RefDenseGPU) and
against the CPU restatement (DenseOracle).

The values are floats; with the contraction sites pinned against dumps of the
reference's full-PF kernels (tests/golden/dense) the library and the oracle
reproduce them bit for bit, which the one-step and run tests assert (with the
absolute difference, bounded by 2e-6, recorded beside it); grain ids of the
argmax map and the moving-domain bookkeeping are compared exactly.
"""
import json
import os

import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.dense import DenseSolver
from oracle import DenseOracle, RefDenseGPU

pytestmark = pytest.mark.gpu

OUT = os.environ.get("CUPF_RECORD_DIR", "")  # measured numbers are written here when set
TOL = 2e-6


def _record(name, rec):
    if os.path.isdir(OUT):
        with open(os.path.join(OUT, name), "w") as f:
            json.dump(rec, f, indent=1)


def _case(n=(32, 32, 40), grains=8, seed=0):
    return cases.line_case(*n, num_pf=5, num_grains=grains, seed=seed, bc="110")


def _interior(c, ph):
    p = c.params
    return ph.reshape(p.num_theta, p.fnz, p.fny, p.fnx)[:, 1:-1, 1:-1, 1:-1]


def _faces(c):
    """Cells with at most one halo coordinate (interior and halo faces)."""
    p = c.params
    k, j, i = np.meshgrid(np.arange(p.fnz), np.arange(p.fny), np.arange(p.fnx), indexing="ij")
    nh = ((i == 0) | (i == p.fnx - 1)).astype(int) + ((j == 0) | (j == p.fny - 1)) + \
        ((k == 0) | (k == p.fnz - 1))
    return (nh <= 1).reshape(-1)


def _t(p, n):
    return float(np.float32(np.float32(n) * np.float32(p.dt)) * np.float32(p.tau0))


def _developed(c, steps=60):
    o = DenseOracle()
    ph = o.ini(c.params, c.phi, c.alpha)
    a, _ = o.run(c, c.meta["R"], ph, steps, prestep=True)
    return a


def _dev(a, torch, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _compare(c, got, ref):
    g = _interior(c, got).astype(np.float64)
    r = _interior(c, ref).astype(np.float64)
    d = np.abs(g - r)
    return {"max_abs": float(d.max()), "identical_frac": float((g == r).mean())}


def test_one_step_matches_reference_kernel(built):
    import torch
    c = _case()
    p, R = c.params, c.meta["R"]
    ph = _developed(c)
    n = 61
    ref = RefDenseGPU()
    ref.check(ref.L.refd_set_params(p, R))
    d_in, d_out = _dev(ph, torch), _dev(ph, torch)
    x, y, z = (_dev(np.asarray(v, np.float32), torch) for v in (c.x, c.y, c.z))
    sint, cost = _dev(np.asarray(c.sint, np.float32), torch), _dev(np.asarray(c.cost, np.float32), torch)
    ref.check(ref.L.refd_set_bc(d_in.data_ptr()))
    ref.check(ref.L.refd_rhs_psi(_t(p, n), x.data_ptr(), y.data_ptr(), z.data_ptr(), d_in.data_ptr(),
                                 d_out.data_ptr(), sint.data_ptr(), cost.data_ptr()))
    ref.check(ref.L.refd_sync())
    r = d_out.cpu().numpy()
    with DenseSolver(c) as s:
        s.set_slots(ph, steps_done=n - 1)
        s.step(1)
        lib = s.get_slots()
    ora = DenseOracle().rhs(c, R, _t(p, n), ph)
    rec = {"library": _compare(c, lib, r), "oracle": _compare(c, ora, r),
           "active_frac": float((_interior(c, ph) != -1).mean())}
    _record("dense_one_step.json", rec)
    print(rec)
    assert rec["library"]["max_abs"] < TOL, rec
    assert rec["oracle"]["max_abs"] < TOL, rec
    # with the contraction sites pinned against the reference's full-PF kernels
    # (tests/golden/dense) both reproduce its step bit for bit
    assert rec["library"]["identical_frac"] == 1.0, rec
    assert rec["oracle"]["identical_frac"] == 1.0, rec


def _ref_evolve_start(ref, torch, c):
    """set_minus1 / ini_PF / set_BC_3D on both buffers and the pre-loop rhs_psi
    at t = 0, as PhaseField::evolve (PhaseField.cu:545-556)."""
    p = c.params
    L = p.fnx * p.fny * p.fnz
    n = L * p.num_theta
    old = torch.empty(n, dtype=torch.float32, device="cuda")
    new = torch.empty(n, dtype=torch.float32, device="cuda")
    phi = _dev(np.asarray(c.phi, np.float32), torch)
    alpha = _dev(np.asarray(c.alpha, np.int32), torch)
    for b in (old, new):
        ref.check(ref.L.refd_set_minus1(b.data_ptr(), n))
    for b in (old, new):
        ref.check(ref.L.refd_ini(b.data_ptr(), phi.data_ptr(), alpha.data_ptr()))
    ref.check(ref.L.refd_set_minus1(phi.data_ptr(), L))
    for b in (new, old):
        ref.check(ref.L.refd_set_bc(b.data_ptr()))
    return old, new, phi, alpha


def test_run_matches_reference(built):
    import torch
    c = _case(grains=10, seed=3)
    p, R = c.params, c.meta["R"]
    ref = RefDenseGPU()
    ref.check(ref.L.refd_set_params(p, R))
    x, y, z = (_dev(np.asarray(v, np.float32), torch) for v in (c.x, c.y, c.z))
    sint, cost = _dev(np.asarray(c.sint, np.float32), torch), _dev(np.asarray(c.cost, np.float32), torch)
    old, new, phi, alpha = _ref_evolve_start(ref, torch, c)
    ref.check(ref.L.refd_rhs_psi(0.0, x.data_ptr(), y.data_ptr(), z.data_ptr(), old.data_ptr(),
                                 new.data_ptr(), sint.data_ptr(), cost.data_ptr()))
    import ctypes as C
    ms = C.c_float()
    nsteps = 120
    ref.check(ref.L.refd_run_steps(nsteps, 0, x.data_ptr(), y.data_ptr(), z.data_ptr(), new.data_ptr(),
                                   old.data_ptr(), sint.data_ptr(), cost.data_ptr(), C.byref(ms)))
    last = new if nsteps % 2 == 0 else old
    ref.check(ref.L.refd_set_bc(last.data_ptr()))
    # collect_PF after the QoI memset (PhaseField.cu:573-574)
    alpha.zero_()
    argmax = torch.zeros(p.fnx * p.fny * p.fnz, dtype=torch.int32, device="cuda")
    ref.check(ref.L.refd_collect(last.data_ptr(), phi.data_ptr(), alpha.data_ptr(), argmax.data_ptr()))
    ref.check(ref.L.refd_sync())
    r = last.cpu().numpy()
    with DenseSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.prestep()
        s.step(nsteps)
        lib = s.get_slots()
        lphi, lalpha = s.collect(clear=True)
    # set_BC_3D fills halo edges and corners with racing threads (PhaseField.cu:111-166);
    # the argmax fields are compared on the interior and the halo faces
    m = _faces(c)
    rec = {"steps": nsteps, "state": _compare(c, lib, r),
           "alpha_equal_frac": float((lalpha[m] == alpha.cpu().numpy()[m]).mean()),
           "phi_max_abs": float(np.abs(lphi[m] - phi.cpu().numpy()[m]).max())}
    _record("dense_run_vs_reference.json", rec)
    print(rec)
    assert rec["state"]["identical_frac"] == 1.0, rec
    assert rec["phi_max_abs"] == 0.0, rec
    assert rec["alpha_equal_frac"] == 1.0, rec


def test_collect_keeps_previous_argmax_on_ties(built):
    # two grains equal at a cell: collect_PF keeps the earlier winner, not the
    # first grain (PhaseField.cu:69-74)
    c = _case(n=(8, 8, 8), grains=4)
    p = c.params
    L = p.fnx * p.fny * p.fnz
    ph = np.full((p.num_theta, L), -1.0, np.float32)
    ph[2, :] = 0.5
    cells = np.array([3 + d + p.fnx * (3 + p.fny * 3) for d in range(4)])  # interior cells
    rest = np.setdiff1d(np.arange(L), cells)
    with DenseSolver(c) as s:
        s.set_slots(ph.reshape(-1))
        _, a1 = s.collect(clear=True)
        ph[0, :] = 0.5  # tie with grain 2 everywhere
        ph[3, cells] = 0.9  # strictly larger at a few cells
        s.set_slots(ph.reshape(-1))
        phi2, a2 = s.collect(clear=True)
    assert (a1 == 3).all()
    assert (a2[rest] == 3).all() and (a2[cells] == 4).all()
    assert np.allclose(phi2[cells], 0.9)


def test_moving_domain_matches_reference(built):
    import ctypes as C
    import torch
    c = _case(n=(24, 24, 40), grains=6, seed=1)
    p, R = c.params, c.meta["R"]
    ph = _developed(c, steps=40)
    o = DenseOracle()
    tip0 = o.tip_scan(p, ph, 1)
    thres = tip0 - 3
    # reference: tip_mvf, collect_PF, then per layer collect_PF + move_frame + copy_frame
    ref = RefDenseGPU()
    ref.check(ref.L.refd_set_params(p, R))
    L = p.fnx * p.fny * p.fnz
    d_old, d_new = _dev(ph, torch), _dev(ph, torch)
    zf = np.asarray(c.z, np.float32)
    d_z, d_z2 = _dev(zf, torch), _dev(zf, torch)
    phi = torch.full((L,), -1.0, dtype=torch.float32, device="cuda")
    alpha = torch.zeros(L, dtype=torch.int32, device="cuda")
    argmax = torch.zeros(L, dtype=torch.int32, device="cuda")
    fnz_f = 4 * p.fnz
    afull = torch.zeros(p.fnx * p.fny * fnz_f, dtype=torch.int32, device="cuda")
    loss = torch.zeros(p.num_theta, dtype=torch.int32, device="cuda")
    meanx = torch.zeros(p.fnz, dtype=torch.float32, device="cuda")
    meanx_h = np.zeros(p.fnz, np.float32)
    tip = C.c_int32(1)
    ref.check(ref.L.refd_tip_mvf(C.byref(tip), d_old.data_ptr(), meanx.data_ptr(),
                                 meanx_h.ctypes.data_as(C.POINTER(C.c_float))))
    ref.check(ref.L.refd_collect(d_old.data_ptr(), phi.data_ptr(), alpha.data_ptr(), argmax.data_ptr()))
    tip_ref, mc = tip.value, 0
    while tip_ref >= thres:
        ref.check(ref.L.refd_collect(d_old.data_ptr(), phi.data_ptr(), alpha.data_ptr(), argmax.data_ptr()))
        ref.check(ref.L.refd_move_frame(d_new.data_ptr(), d_z2.data_ptr(), d_old.data_ptr(), d_z.data_ptr(),
                                        alpha.data_ptr(), afull.data_ptr(), loss.data_ptr(), mc))
        ref.check(ref.L.refd_copy_frame(d_new.data_ptr(), d_z2.data_ptr(), d_old.data_ptr(), d_z.data_ptr()))
        mc += 1
        tip_ref -= 1
    ref.check(ref.L.refd_set_bc(d_old.data_ptr()))
    ref.check(ref.L.refd_sync())
    with DenseSolver(c) as s:
        s.set_slots(ph, steps_done=40)
        tf, mcl, moved = s.move_domain(1, thres, 0)
        lib = s.get_slots()
        full, lloss = s.get_archive(fnz_f)
        z = s.get_z()
    rec = {"tip0": tip0, "thres": thres, "tip_ref": tip_ref, "tip_lib": tf, "moves_ref": mc,
           "moves_lib": moved, "state": _compare(c, lib, d_old.cpu().numpy())}
    _record("dense_moving_domain.json", rec)
    print(rec)
    assert moved == mc > 0 and tf == tip_ref and mcl == mc, rec
    assert np.array_equal(_interior(c, lib), _interior(c, d_old.cpu().numpy())), rec
    assert np.array_equal(z[1:-1], d_z.cpu().numpy()[1:-1])
    assert np.array_equal(lloss, loss.cpu().numpy())
    assert np.array_equal(full, afull.cpu().numpy())


def test_list_overflow_path_gives_the_same_bits(built):
    # the evaluation over every grain (lists past capacity) and the list path
    # compute the same floats
    c = _case(grains=8, seed=2)
    ph = _developed(c, steps=30)
    with DenseSolver(c) as a, DenseSolver(c) as b:
        a.set_slots(ph, steps_done=30)
        b.set_slots(ph, steps_done=30)
        b.set_tuning(2)
        a.step(5)
        b.step(5)
        over = b.overflow_cells()
        assert a.overflow_cells() == 0
        assert over > 0
        assert np.array_equal(a.get_slots(), b.get_slots())


def test_carried_lists_equal_rebuilt_lists(built):
    # the lists each step writes for the next, and lists rebuilt from the state
    # (after set_slots), drive the same arithmetic; a capacity change mid-run too
    c = _case(grains=8, seed=5)
    ph = _developed(c, steps=20)
    with DenseSolver(c) as a, DenseSolver(c) as b:
        a.set_slots(ph, steps_done=20)
        a.step(12)
        mid = a.get_slots()
        b.set_slots(mid, steps_done=32)
        a.step(9)
        b.step(4)
        b.set_tuning(3)
        b.step(2)
        b.set_tuning(16)
        b.step(3)
        assert np.array_equal(a.get_slots(), b.get_slots())


def test_matches_oracle_over_many_steps(built):
    c = _case(grains=8, seed=4)
    o = DenseOracle()
    ph0 = o.ini(c.params, c.phi, c.alpha)
    a, _ = o.run(c, c.meta["R"], ph0, 150, prestep=True)
    with DenseSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.prestep()
        s.step(150)
        lib = s.get_slots()
    rec = _compare(c, lib, a)
    _record("dense_vs_oracle.json", rec)
    assert rec["max_abs"] < 1e-5, rec


def test_speed_vs_reference_kernels(built):
    # device time per step: the reference's set_BC_3D + rhs_psi pair against the
    # library's two-launch step, 64^3 interior, 20 grains (the C1 line case)
    import ctypes as C
    import torch
    c = cases.line_case(64, 64, 64, num_pf=5, num_grains=20, seed=0, bc="110")
    p, R = c.params, c.meta["R"]
    o = DenseOracle()
    ph = o.ini(p, c.phi, c.alpha)
    ref = RefDenseGPU()
    ref.check(ref.L.refd_set_params(p, R))
    a, b = _dev(ph, torch), _dev(ph, torch)
    x, y, z = (_dev(np.asarray(v, np.float32), torch) for v in (c.x, c.y, c.z))
    sint, cost = _dev(np.asarray(c.sint, np.float32), torch), _dev(np.asarray(c.cost, np.float32), torch)
    ms = C.c_float()
    args = (x.data_ptr(), y.data_ptr(), z.data_ptr(), a.data_ptr(), b.data_ptr(), sint.data_ptr(),
            cost.data_ptr(), C.byref(ms))
    ref.check(ref.L.refd_run_steps(40, 0, *args))  # warm-up, develops the tails
    ref.check(ref.L.refd_run_steps(100, 40, *args))
    ref_ms = ms.value / 100
    with DenseSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.prestep()
        s.step(40)
        lib_ms = s.time_steps(100) / 100
    rec = {"grid": [64, 64, 64], "grains": 20, "reference_ms_per_step": ref_ms,
           "library_ms_per_step": lib_ms, "speedup": ref_ms / lib_ms}
    _record("dense_perf_vs_reference.json", rec)
    print(rec)
    assert rec["speedup"] > 1.0, rec


def test_phase_field_cli_full_pf_mode(tmp_path, built):
    # the driver with -a: the full-PF solver behind the same input file, forcing
    # folder and QoI archive as the APT run (main.cpp:39-47)
    import subprocess
    from cupf_b200 import preprocess
    Lx = 2.48
    folder = tmp_path / "forcing" / "case0"
    preprocess.write_line_forcing(str(folder), Lx, Lx, 2 * Lx, num_grains=10, seed=0, G=1.0,
                                  R=0.05, z0=0.6, top=0.3, t_end=5e-7)
    preprocess.write_input_file(str(tmp_path / "line.py"), Lx, nts=2, asp_ratio_zx=2.0,
                                moving_ratio=1.0, num_pf=8)
    out = tmp_path / "out"
    out.mkdir()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "cupf_b200", "phase_field")
    r = subprocess.run([exe, "line.py", "-s", "0", "-b", "110", "-l", "1", "-a", "-d", "0", "-o",
                        str(out)], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    files = sorted(os.listdir(out))
    assert len(files) == 1 and files[0].endswith(".h5")
    from tests.h5read import H5File
    d = H5File(str(out / files[0]))
    for key in ("fractions", "tip_y", "cross_sec", "total_area", "node_region"):
        assert key in d, key
    assert d["tip_y"].shape == (3,)
    assert d["total_area"].reshape(3, 10)[0].sum() > 0
