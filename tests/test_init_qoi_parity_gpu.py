"""Parity of the entry points the benchmark, the server and the phase_field
driver start from and report through, on a B200:

* cupf_apt_init_from_argmax (set_minus1 x2 + APTini_PF x2 + setBC x2 of
  APTPhaseField::evolve, 3DgrainMPI/APTPhaseField.cu:727-728,771-772,817-818;
  APTini_PF :78-89; set_minus1 PhaseField.cu:51-57; the ids start at -1 from
  cudaSetup's memset, APTPhaseField.cu:599-600) against the reference kernels
  run on the same phi/alpha and against Case.initial_slots(), bit for bit;
* cupf_apt_grain_volumes and cupf_grain_volumes_noalloc against the reference's
  compiled QOI::calculateQoIs (3DgrainMPI/QOI.cpp:198-231) and a numpy bincount
  of the same argmax map;
* cupf_apt_qoi_sums (FP64 solid volume, interface area, mean interface height)
  against an FP64 numpy evaluation of the same slot state.
"""
import ctypes as C

import numpy as np
import pytest

from cupf_b200 import abi, cases
from cupf_b200.solver import APTSolver
from tests.helpers import face_mask

pytestmark = pytest.mark.gpu

INIT_CASES = [
    # interior, num_pf, grains, seed, bc
    ((64, 64, 64), 5, 20, 0, "110"),     # C1
    ((37, 21, 29), 4, 15, 4, "101"),     # partial tiles
    ((24, 24, 40), 8, 60, 1, "000"),
    ((20, 20, 20), 1, 3, 9, "111"),
]


def reference_init(case):
    """The reference's initial slot state on the GPU: ids -1 (cudaSetup's memset),
    phi -1 (set_minus1), APTini_PF from (phi, alpha), then APTsetBC3D."""
    import torch
    from oracle import RefGPU
    p = case.params
    ref = RefGPU(p.num_pf)
    ref.check(ref.L.ref_set_params(p))
    L = case.length
    ph = torch.empty(p.num_pf * L, dtype=torch.float32, device="cuda")
    ids = torch.full((p.num_pf * L,), -1, dtype=torch.int32, device="cuda")
    phi = torch.from_numpy(np.ascontiguousarray(case.phi, np.float32)).cuda()
    alpha = torch.from_numpy(np.ascontiguousarray(case.alpha, np.int32)).cuda()
    ref.check(ref.L.ref_set_minus1(ph.data_ptr(), p.num_pf * L))
    ref.check(ref.L.ref_ini(ph.data_ptr(), phi.data_ptr(), alpha.data_ptr(), ids.data_ptr()))
    ref.check(ref.L.ref_set_bc(ph.data_ptr(), ids.data_ptr()))
    ref.check(ref.L.ref_sync())
    return ph.cpu().numpy(), ids.cpu().numpy()


@pytest.mark.parametrize("spec", INIT_CASES, ids=lambda s: "%dx%dx%d_np%d_%s" % (*s[0], s[1], s[4]))
def test_init_from_argmax_matches_reference_and_case(built, spec):
    interior, npf, grains, seed, bc = spec
    c = cases.line_case(*interior, num_pf=npf, num_grains=grains, seed=seed, bc=bc)
    p = c.params
    with APTSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        ph, ids = s.get_slots()
    # Case.initial_slots is the state every set_slots parity test starts from:
    # equal everywhere, halo edges included (both map each halo coordinate)
    ph0, id0 = c.initial_slots()
    assert np.array_equal(ids, id0)
    assert np.array_equal(ph.view(np.int32), ph0.view(np.int32))
    # the reference kernels: interior and face-halo cells (edges and corners are
    # filled by racing threads in APTsetBC3D)
    rph, rid = reference_init(c)
    m = np.tile(face_mask(p), p.num_pf)
    assert np.array_equal(ids[m], rid[m])
    assert np.array_equal(ph[m].view(np.int32), rph[m].view(np.int32))


def test_init_from_argmax_liquid_start_field(built):
    """phi > LS on cells with alpha == 0 (a liquid-start field): APTini_PF puts
    id 0 there; the library must too."""
    c = cases.line_case(32, 24, 40, num_pf=5, num_grains=12, seed=5, bc="110",
                        substrate_everywhere=False)
    assert np.any((c.phi.astype(np.float64) > -0.995) & (c.alpha == 0))
    p = c.params
    with APTSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        ph, ids = s.get_slots()
    rph, rid = reference_init(c)
    m = np.tile(face_mask(p), p.num_pf)
    assert np.array_equal(ids[m], rid[m])
    assert np.array_equal(ph[m].view(np.int32), rph[m].view(np.int32))


def _bincount(p, alpha, ng):
    a = alpha.reshape(p.fnz, p.fny, p.fnx)[1:-1, 1:-1, 1:-1].ravel()
    ok = (a >= 1) & (a <= ng)
    counts = np.bincount(a[ok], minlength=ng + 1).astype(np.int64)
    counts[0] = int(np.count_nonzero(~ok))
    return counts


@pytest.mark.parametrize("which", ["c1", "c2"])
def test_grain_volumes_match_reference_qoi(built, which):
    import torch
    from oracle import RefHost
    if which == "c1":
        c = cases.line_case(64, 64, 64, num_pf=5, num_grains=20, seed=0, bc="110")
        steps = 200
    else:
        c = cases.line_case(256, 256, 512, num_pf=8, num_grains=600, seed=0, bc="110")
        steps = 50
    p = c.params
    ng = p.num_theta
    with APTSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.step(steps)
        _, alpha = s.collect(clear=True)
        vols = s.grain_volumes(ng)
    assert vols[1:].sum() > 0
    assert np.array_equal(vols, _bincount(p, alpha, ng))
    g2pf, rv = RefHost().calculate_qois(p.fnx, p.fny, p.fnz, ng, alpha)
    # the reference lists grains in first-seen order with their voxel counts
    assert len(g2pf) == int(np.count_nonzero(vols[1:]))
    assert np.array_equal(vols[g2pf], rv.astype(np.int64))
    # the allocation-free variant on the same device map
    d_alpha = torch.from_numpy(np.ascontiguousarray(alpha)).cuda()
    counts = np.zeros(ng + 1, np.int64)
    abi.check(abi.lib().cupf_grain_volumes_noalloc(C.c_void_p(d_alpha.data_ptr()), p.fnx, p.fny,
                                                    p.fnz, ng,
                                                    counts.ctypes.data_as(C.POINTER(C.c_int64)),
                                                    None))
    assert np.array_equal(counts, vols)


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_qoi_sums_match_fp64_numpy(built, prec):
    from oracle import interface_qois
    c = cases.line_case(48, 40, 64, num_pf=6, num_grains=25, seed=3, bc="110")
    p = c.params
    with APTSolver(c, precision=prec) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.step(120)
        ph, ids = s.get_slots()
        q = s.qoi_sums()
    ref = interface_qois(p, ph)
    # same FP64 formulas over the same values; only the summation order differs
    for got, want in zip(q, ref):
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (q, ref)


def test_collect_into_caller_arrays(built):
    """collect(out=...) reads the argmax fields into caller-owned arrays (here
    page-locked ones) with the same values as the default path, and rejects
    arrays of the wrong type or length."""
    import torch
    c = cases.line_case(40, 36, 48, num_pf=5, num_grains=20, seed=4, bc="110")
    out = (torch.empty(c.length, dtype=torch.float32, pin_memory=True).numpy(),
           torch.empty(c.length, dtype=torch.int32, pin_memory=True).numpy())
    with APTSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.step(20)
        phi0, alpha0 = s.collect(clear=True)
        phi1, alpha1 = s.collect(clear=True, out=out)
        with pytest.raises(ValueError):
            s.collect(out=(np.empty(c.length, np.float64), out[1]))
        with pytest.raises(ValueError):
            s.collect(out=(out[0][:-1], out[1]))
    assert phi1 is out[0] and alpha1 is out[1]
    assert np.array_equal(phi0.view(np.uint32), phi1.view(np.uint32))
    assert np.array_equal(alpha0, alpha1)
