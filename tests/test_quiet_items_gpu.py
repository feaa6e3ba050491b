"""Quiet work items: the step leaves alone the items whose cells stay all-empty.

An item is left alone only when its cells already hold empty slots in the buffer
the step writes, and its cells and their face neighbours hold empty slots in the
buffer it reads, so every cell would be written empty again (APTrhs_psi on a
cell whose 7 stencil points hold no id, APTPhaseField.cu:198-233).  Results must
therefore be bit-identical with the skip on and off, for every boundary mapping,
ragged tile and z-chunk edge, in every storage format, and the skip must
actually leave the liquid above the front alone.
"""
import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.solver import APTSolver

pytestmark = pytest.mark.gpu


def _run(c, prec, skip, zc, nsteps):
    ph0, id0 = c.initial_slots()
    with APTSolver(c, precision=prec) as s:
        s.set_slots(ph0, id0, 0)
        s.set_tuning(zc)
        s.set_skip_quiet(skip)
        s.active_cells()
        s.step(nsteps)
        cells = s.active_cells()
        ph, ids = s.get_slots()
        s.collect()
    return ph, ids, cells


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
@pytest.mark.parametrize("shape,bc,zc,frac", [
    ((45, 21, 37), "110", 4, 0.3),   # ragged x and y tiles, periodic x/y
    ((40, 17, 50), "000", 3, 0.25),  # mirror everywhere, ragged last z chunk
    ((33, 9, 30), "111", 2, 0.4),    # periodic z: the top chunk borders the bottom one
    ((64, 16, 48), "010", 4, 0.2),   # two tiles in x, one in y, mirror x and z
])
def test_skip_is_bit_identical(built, prec, shape, bc, zc, frac):
    c = cases.line_case(*shape, num_pf=5, num_grains=7, seed=3, bc=bc, z0_frac=frac)
    nsteps = 80
    a_ph, a_id, a_cells = _run(c, prec, True, zc, nsteps)
    b_ph, b_id, b_cells = _run(c, prec, False, zc, nsteps)
    assert np.array_equal(a_id, b_id)
    assert np.array_equal(a_ph.view(np.int32), b_ph.view(np.int32))
    total = shape[0] * shape[1] * shape[2] * nsteps
    assert b_cells == total  # the full sweep computes every cell of every step
    if bc[2] == "1":
        # periodic z: the solid at the bottom borders the top plane, which keeps
        # the top chunk busy; only the middle of the liquid is left alone
        assert a_cells < total
    else:
        assert a_cells < 0.9 * total


def test_skip_follows_the_front(built):
    """A front that grows into the liquid wakes the items it reaches: run long
    enough at a high undercooling rate for the front to cross z-chunk edges, then
    compare with the full sweep."""
    c = cases.line_case(32, 16, 48, num_pf=5, num_grains=6, seed=1, bc="110", z0_frac=0.3,
                        R=0.5)
    a_ph, a_id, a_cells = _run(c, "fp32", True, 2, 400)
    b_ph, b_id, _ = _run(c, "fp32", False, 2, 400)
    assert np.array_equal(a_id, b_id)
    assert np.array_equal(a_ph.view(np.int32), b_ph.view(np.int32))
    assert a_cells < 32 * 16 * 48 * 400


def test_skip_across_nucleation_and_domain_shifts(built):
    """Nucleation marks the items a nucleus reaches, and a domain shift moves the
    flags down with the planes; both paths keep the skip exact: a liquid-start
    run with nuclei landing in quiet melt, then moving-domain steps, agrees bit
    for bit with the full sweep."""
    c = cases.line_case(40, 24, 64, num_pf=5, num_grains=8, seed=7, bc="110", z0_frac=0.8)
    p = c.params
    p.nuc_rad = np.float32(0.16)
    p.pts_cell = int(np.float32(0.16) / np.float32(np.float32(0.8) * np.float32(0.1)))
    p.nuc_Nmax0 = np.float32(5.0)
    p.nuc_Nmax = np.float32(5.0)
    p.seed = 5
    ph0, id0 = c.initial_slots()
    out = []
    for skip in (True, False):
        with APTSolver(c) as s:
            s.set_slots(ph0, id0, 0)
            s.set_tuning(2)
            s.set_skip_quiet(skip)
            s.nucl_init()
            total = 0
            for _ in range(30):
                s.step(1, True)
                total = s.nucleate(True)
                s.step(1, True)
            tip, mc, moved_total = 1, 0, 0
            for _ in range(20):
                s.step(10)
                tip, mc, moved = s.move_domain(tip, int(0.8 * p.fnz), mc)
                moved_total += moved
            s.step(20)
            ph, ids = s.get_slots()
            out.append((ph, ids, total, moved_total, s.active_cells()))
    (a_ph, a_id, a_n, a_m, a_cells), (b_ph, b_id, b_n, b_m, b_cells) = out
    assert a_n == b_n and a_n > 0
    assert a_m == b_m and a_m > 0
    assert np.array_equal(a_id, b_id)
    assert np.array_equal(a_ph.view(np.int32), b_ph.view(np.int32))
    assert a_cells < b_cells


def test_skip_matches_full_sweep_on_the_benchmark_workload(built):
    """The benchmark's own case (256x256x512, 600 grains, NUM_PF = 8, FP32) over a
    whole 2000-step run: argmax map, phi and the FP64 interface sums are the same
    with quiet items left alone and with every item computed."""
    c = cases.line_case(256, 256, 512, num_pf=8, num_grains=600, seed=0, bc="110")
    out = []
    for skip in (True, False):
        with APTSolver(c) as s:
            s.init_from_argmax(c.phi, c.alpha)
            s.set_skip_quiet(skip)
            s.active_cells()
            s.step(2000)
            cells = s.active_cells()
            phi, alpha = s.collect(clear=True)
            out.append((phi, alpha, s.qoi_sums(), cells))
    (pa, aa, qa, ca), (pb, ab, qb, cb) = out
    assert np.array_equal(aa, ab)
    assert np.array_equal(pa.view(np.int32), pb.view(np.int32))
    assert tuple(qa) == tuple(qb)
    assert ca < 0.4 * cb
