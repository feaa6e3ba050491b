"""3D junction search (QOI3D::searchJunctionsOnImage, QOI.cpp:233-311) through
the device's candidate list.

The device marks candidate cells and counts each cell's distinct neighbourhood
values (cupf_apt_junction_candidates); the host then builds the records of the
candidates only.  The reference lists each junction's grain ids in the
iteration order of a std::unordered_map that it reuses across cells, so the
host must grow that map as the full scan would before each record.  Here the
candidates and counts come from an independent numpy computation (CPU), and on
the GPU from the device; either way the records must equal the full host
scan's, bit for bit and in order.
"""
import ctypes as C

import numpy as np
import pytest

from cupf_b200 import abi

OFFS = [(dk, dj, di) for dk in (-1, 0, 1) for dj in (-1, 0, 1) for di in (-1, 0, 1)
        if di * di + dj * dj + dk * dk <= 2]


def voronoi_map(n, grains, seed, liquid_from=None):
    """A 3D Voronoi grain map (ids 1..grains) with halo, liquid (0) above
    `liquid_from` planes."""
    rng = np.random.default_rng(seed)
    pts = rng.random((grains, 3)) * n
    z, y, x = np.meshgrid(np.arange(n + 2), np.arange(n + 2), np.arange(n + 2), indexing="ij")
    d = ((x[..., None] - pts[:, 0]) ** 2 + (y[..., None] - pts[:, 1]) ** 2 +
         (z[..., None] - pts[:, 2]) ** 2)
    a = (np.argmin(d, axis=-1) + 1).astype(np.int32)
    if liquid_from is not None:
        a[liquid_from:] = 0
    return np.ascontiguousarray(a)


def numpy_candidates(a):
    """Candidate cells and distinct counts, computed without the library."""
    fnz, fny, fnx = a.shape
    inner = a[1:-1, 1:-1, 1:-1]
    nb = np.stack([a[1 + dk:fnz - 1 + dk, 1 + dj:fny - 1 + dj, 1 + di:fnx - 1 + di]
                   for dk, dj, di in OFFS])
    s = np.sort(nb, axis=0)
    new = np.concatenate([np.ones((1,) + s.shape[1:], bool), s[1:] != s[:-1]])
    distinct = new.sum(axis=0)
    # longest run of equal values = max occurrence
    run = np.ones(s.shape, np.int32)
    for q in range(1, s.shape[0]):
        run[q] = np.where(s[q] == s[q - 1], run[q - 1] + 1, 1)
    maxc = run.max(axis=0)
    zero = (nb == 0).any(axis=0)
    distinct = np.where(inner != 0, distinct, 0).astype(np.uint8)
    cand = (inner != 0) & ~zero & (distinct == 4) & (maxc <= 10)
    kk, jj, ii = np.nonzero(cand)
    cells = ((kk + 1) * fny * fnx + (jj + 1) * fnx + (ii + 1)).astype(np.int64)
    return np.sort(cells), np.ascontiguousarray(distinct.reshape(-1))


def host_full(a):
    fnz, fny, fnx = a.shape
    cap = 1 << 22
    out = np.zeros(cap, np.int32)
    n = abi.lib().cupf_host_junctions_3d(fnx, fny, fnz, a.ctypes.data_as(C.POINTER(C.c_int32)),
                                         out.ctypes.data_as(C.POINTER(C.c_int32)), cap)
    return out[:n].copy()


def host_cells(a, cells, distinct):
    fnz, fny, fnx = a.shape
    cap = 1 << 22
    out = np.zeros(cap, np.int32)
    cells = np.ascontiguousarray(cells, np.int64)
    n = abi.lib().cupf_host_junctions_3d_cells(
        fnx, fny, fnz, a.ctypes.data_as(C.POINTER(C.c_int32)),
        cells.ctypes.data_as(C.POINTER(C.c_int64)), len(cells),
        distinct.ctypes.data_as(C.POINTER(C.c_uint8)), out.ctypes.data_as(C.POINTER(C.c_int32)), cap)
    return out[:n].copy()


@pytest.mark.parametrize("n,grains,seed,liquid", [(28, 90, 0, None), (32, 140, 3, 22),
                                                  (24, 40, 7, 12)])
def test_candidate_records_equal_full_scan(n, grains, seed, liquid):
    a = voronoi_map(n, grains, seed, liquid)
    cells, distinct = numpy_candidates(a)
    full = host_full(a)
    rec = full.reshape(-1, 9)
    found = rec[rec[:, 0] >= 0]
    assert len(found) == len(cells) and len(found) > 0
    assert np.array_equal(host_cells(a, cells, distinct), full)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_device_candidates_equal_full_scan(built, precision):
    from cupf_b200 import cases
    from cupf_b200.solver import APTSolver
    c = cases.line_case(40, 40, 48, num_pf=8, num_grains=60, seed=5, bc="110")
    with APTSolver(c, precision=precision) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.step(60)
        _, alpha = s.collect(clear=True)
        a = np.ascontiguousarray(alpha.reshape(c.params.fnz, c.params.fny, c.params.fnx), np.int32)
        ni = (c.params.fnx - 2) * (c.params.fny - 2) * (c.params.fnz - 2)
        distinct = np.zeros(ni, np.uint8)
        cap = 4
        while True:
            cells = np.zeros(cap, np.int64)
            count = C.c_int64()
            abi.check(abi.lib().cupf_apt_junction_candidates(
                C.c_void_p(s.h.value if hasattr(s.h, "value") else s.h),
                cells.ctypes.data_as(C.POINTER(C.c_int64)), cap, C.byref(count),
                distinct.ctypes.data_as(C.POINTER(C.c_uint8))))
            if count.value <= cap:
                cells = cells[:count.value]
                break
            cap = count.value
    want_cells, want_distinct = numpy_candidates(a)
    assert np.array_equal(cells, want_cells)
    assert np.array_equal(distinct, want_distinct)
    assert np.array_equal(host_cells(a, cells, distinct), host_full(a))


# ---- line configuration (QOILine::searchJunctionsOnImage, QOI.cpp:103-160) ----

def line_map(fnx, fny, fnz, grains, seed):
    """A full line-configuration map: columnar 2D Voronoi grains (ids 1..grains,
    halo included) whose layout changes with height, liquid (0) in the top
    planes."""
    rng = np.random.default_rng(seed)
    a = np.zeros((fnz, fny, fnx), np.int32)
    y, x = np.meshgrid(np.arange(fny), np.arange(fnx), indexing="ij")
    pts = rng.random((grains, 2)) * (fny, fnx)
    for k in range(fnz - 3):
        pts += rng.normal(0, 0.4, pts.shape)  # grains drift with height
        d = (y[..., None] - pts[:, 0]) ** 2 + (x[..., None] - pts[:, 1]) ** 2
        a[k] = np.argmin(d, axis=-1) + 1
    return np.ascontiguousarray(a)


def numpy_line_candidates(a, tip_y):
    """Candidates over the stacked tip layers, computed without the library."""
    fnz, fny, fnx = a.shape
    cells = []
    for kt, t in enumerate(tip_y):
        L = a[t]
        nb = np.stack([L[1 + dj:fny - 1 + dj, 1 + di:fnx - 1 + di]
                       for dj in (-1, 0, 1) for di in (-1, 0, 1)])
        s = np.sort(nb, axis=0)
        distinct = np.concatenate([np.ones((1,) + s.shape[1:], bool), s[1:] != s[:-1]]).sum(0)
        run = np.ones(s.shape, np.int32)
        for q in range(1, 9):
            run[q] = np.where(s[q] == s[q - 1], run[q - 1] + 1, 1)
        cand = (distinct >= 3) & (run.max(axis=0) <= 5)
        jj, ii = np.nonzero(cand)
        cells.append(kt * fny * fnx + (jj + 1) * fnx + (ii + 1))
        assert distinct[cand].max(initial=0) <= 5  # the reference writes past a record beyond 5 ids
    return np.concatenate(cells).astype(np.int64)


LINE_CASES = [  # fnx, fny, fnz, grains, seed, tip_y
    (34, 30, 24, 25, 0, [3, 7, 7, 12, 20]),
    (20, 41, 16, 12, 4, [1, 5, 9]),
    (50, 12, 10, 30, 9, [2, 6]),
]


@pytest.mark.parametrize("spec", LINE_CASES, ids=lambda s: "%dx%dx%d" % s[:3])
def test_line_junctions_match_reference_and_candidates(built, spec):
    from cupf_b200 import host_api
    from oracle import RefHost
    fnx, fny, fnz, grains, seed, tip_y = spec
    a = line_map(fnx, fny, fnz, grains, seed)
    nts, nn = len(tip_y) - 1, 40
    full, cross = host_api.line_junctions(fnx, fny, nts, nn, tip_y, a.reshape(-1))
    rnodes, rcross = RefHost().line_junctions(fnx, fny, nts, nn, tip_y, a.reshape(-1))
    assert np.array_equal(full, rnodes) and np.array_equal(cross, rcross)
    cells = numpy_line_candidates(a, tip_y)
    assert len(cells) > 0
    got, gcross = host_api.line_junctions(fnx, fny, nts, nn, tip_y, a.reshape(-1), cells=cells)
    assert np.array_equal(got, full) and np.array_equal(gcross, cross)


@pytest.mark.gpu
@pytest.mark.parametrize("spec", LINE_CASES, ids=lambda s: "%dx%dx%d" % s[:3])
def test_line_junction_device_candidates(built, spec):
    from cupf_b200 import host_api
    fnx, fny, fnz, grains, seed, tip_y = spec
    a = line_map(fnx, fny, fnz, grains, seed)
    layers = np.stack([a[t] for t in tip_y])
    cells = host_api.line_junction_candidates(fnx, fny, layers)
    assert np.array_equal(cells, numpy_line_candidates(a, tip_y))
    nts = len(tip_y) - 1
    got, _ = host_api.line_junctions(fnx, fny, nts, 40, tip_y, a.reshape(-1), cells=cells)
    full, _ = host_api.line_junctions(fnx, fny, nts, 40, tip_y, a.reshape(-1))
    assert np.array_equal(got, full)
