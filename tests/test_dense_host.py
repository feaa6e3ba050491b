"""The full-PF (-a) restatement in the oracle (apt_oracle.c, full-PF section)
against an independent numpy restatement of PhaseField.cu (no GPU).

With every contraction switch off, both evaluate the same float operations in the
same order, so the step is compared bit for bit; the pinned switches are restored
afterwards.  Also: the boundary fill, ini_PF, collect_PF's persistent argmax,
move_frame / copy_frame, and the property the library's dense step is built on (a
grain that is -1 at all seven stencil points stays exactly -1).
"""
import os

import numpy as np
import pytest

from cupf_b200 import cases
from oracle import DENSE_PINNED_CONTRACTION, DenseOracle

F = np.float32
LS = -0.995


def _case(n=(10, 9, 12), grains=5, seed=0):
    return cases.line_case(*n, num_pf=5, num_grains=grains, seed=seed, bc="110")


def _state(c, steps=6):
    o = DenseOracle()
    ph = o.ini(c.params, c.phi, c.alpha)
    a, _ = o.run(c, c.meta["R"], ph, steps, prestep=True)
    return a


def numpy_rhs(c, R, t, ph):
    """rhs_psi (PhaseField.cu:168-301) in float32 numpy, one operation at a time."""
    p = c.params
    ng, nz, ny, nx = p.num_theta, p.fnz, p.fny, p.fnx
    P = ph.reshape(ng, nz, ny, nx)
    out = P.copy()
    C = P[:, 1:-1, 1:-1, 1:-1]
    R_ = P[:, 1:-1, 1:-1, 2:]
    L_ = P[:, 1:-1, 1:-1, :-2]
    T_ = P[:, 1:-1, 2:, 1:-1]
    B_ = P[:, 1:-1, :-2, 1:-1]
    U_ = P[:, 2:, 1:-1, 1:-1]
    D_ = P[:, :-2, 1:-1, 1:-1]
    h = F(0.5)
    ux, uy, uz = (R_ - L_) * h, (T_ - B_) * h, (U_ - D_) * h
    g = np.arange(ng)
    act = C.astype(np.float64) > LS
    sint, cost = np.asarray(c.sint, F), np.asarray(c.cost, F)
    sa = np.where(act, sint[g + 1][:, None, None, None], F(0))
    ca = np.where(act, cost[g + 1][:, None, None, None], F(1))
    sb = np.where(act, sint[g + 1 + ng][:, None, None, None], F(0))
    cb = np.where(act, cost[g + 1 + ng][:, None, None, None], F(1))
    kd = F(p.kin_delta)
    a_s = F(1) + F(3) * kd
    eps_ = F(-4) * kd / a_s
    rx = (ca * cb) * ux + sa * uy + (ca * sb) * uz
    ry = ((-sa) * cb) * ux + ca * uy - (sa * sb) * uz
    rz = ((-sb) * ux + F(0)) + cb * uz
    x2, y2, z2 = rx * rx, ry * ry, rz * rz
    mag = x2 + y2 + z2
    q = x2 * x2 + y2 * y2 + z2 * z2
    with np.errstate(divide="ignore", invalid="ignore"):
        A2 = np.where(mag > F(p.eps), a_s * (F(1) + eps_ * q / (mag * mag)), F(1)).astype(F)
    s6 = R_ + L_ + T_ + B_ + U_ + D_
    diff = s6 - F(6) * C
    zk = np.asarray(c.z, F)[1:-1].astype(np.float64)
    Tz = (F(p.G) * ((zk - (np.float64(F(R)) * 1e6) * np.float64(t)) - 2.0)).astype(F)
    Up = (Tz / F(p.L_cp))[None, :, None, None]
    q1 = C + F(1)
    term = (F(0.25) * q1) * q1
    repul = np.zeros_like(C)
    out_c = np.empty_like(C)
    for a in range(ng):
        r = np.zeros_like(C[0])
        for b in range(ng):
            if b != a:
                r = r + term[b]
        repul[a] = r
    w = F(1) - C * C
    E1 = (diff * F(p.hi)) * F(p.hi) + w * C
    inner = w * w - (F(6) * (C + F(1))) * repul
    rhs = E1 - (F(p.lamd) * Up) * inner
    out_c = C + F(p.dt) * (rhs / A2)
    out[:, 1:-1, 1:-1, 1:-1] = out_c
    return out.reshape(-1)


def test_dense_rhs_matches_numpy_bit_for_bit():
    c = _case()
    ph = _state(c)
    p = c.params
    t = float(F(F(7) * F(p.dt)) * F(p.tau0))
    o = DenseOracle()  # (constructing an oracle re-applies the pinned switches)
    o.set_contraction([0] * 24)
    try:
        got = o.rhs(c, c.meta["R"], t, ph)
    finally:
        o.set_contraction(DENSE_PINNED_CONTRACTION)
    want = numpy_rhs(c, c.meta["R"], t, ph)
    Pi = lambda a: a.reshape(p.num_theta, p.fnz, p.fny, p.fnx)[:, 1:-1, 1:-1, 1:-1]
    assert np.array_equal(Pi(got), Pi(want))


def test_set_bc_mirrors_every_face():
    c = _case()
    p = c.params
    rng = np.random.default_rng(0)
    ph = rng.uniform(-1, 1, p.num_theta * p.fnx * p.fny * p.fnz).astype(F)
    DenseOracle().set_bc(p, ph)
    P = ph.reshape(p.num_theta, p.fnz, p.fny, p.fnx)
    m = lambda i, n: 2 if i == 0 else (n - 3 if i == n - 1 else i)
    for k in range(p.fnz):
        for j in range(p.fny):
            for i in range(p.fnx):
                assert np.array_equal(P[:, k, j, i], P[:, m(k, p.fnz), m(j, p.fny), m(i, p.fnx)])


def test_ini_places_phi_in_its_grain():
    c = _case()
    p = c.params
    ph = DenseOracle().ini(p, c.phi, c.alpha).reshape(p.num_theta, -1)
    placed = (c.phi.astype(np.float64) > LS) & (c.alpha >= 1) & (c.alpha <= p.num_theta)
    assert placed.sum() > 100
    for C in np.flatnonzero(placed)[:300]:
        g = c.alpha[C] - 1
        assert ph[g, C] == c.phi[C]
        assert (np.delete(ph[:, C], g) == -1).all()
    assert (ph[:, ~placed] == -1).all()  # liquid, or no grain id (ini_PF matches no grain)


def test_untouched_grain_stays_exactly_minus_one():
    # the dense step's list path relies on this (PhaseField.cu:195-297 with all
    # seven values -1: diff 0, (1-phi^2) 0, repulsion factor 6*(phi+1) = 0)
    c = _case(grains=6)
    p = c.params
    ph = _state(c, steps=3)
    out = DenseOracle().rhs(c, c.meta["R"], 1e-6, ph)
    P = ph.reshape(p.num_theta, p.fnz, p.fny, p.fnx)
    O = out.reshape(P.shape)
    for g in range(p.num_theta):
        st = np.ones(P.shape[1:], bool)[1:-1, 1:-1, 1:-1]
        for dz, dy, dx in ((0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1),
                           (0, 0, -1)):
            st &= P[g, 1 + dz:p.fnz - 1 + dz, 1 + dy:p.fny - 1 + dy, 1 + dx:p.fnx - 1 + dx] == -1
        assert st.any()
        assert (O[g, 1:-1, 1:-1, 1:-1][st] == -1).all()


def test_collect_persistent_argmax():
    c = _case()
    p = c.params
    L = p.fnx * p.fny * p.fnz
    rng = np.random.default_rng(1)
    ph = rng.choice(np.array([-1.0, -0.5, 0.25, 0.5], F), size=p.num_theta * L).astype(F)
    am = rng.integers(0, p.num_theta, L).astype(np.int32)
    phi = np.full(L, -1, F)
    alpha = np.zeros(L, np.int32)
    want_am = am.copy()
    want_phi, want_alpha = phi.copy(), alpha.copy()
    P = ph.reshape(p.num_theta, L)
    for C in range(L):
        a = want_am[C]
        for g in range(p.num_theta):
            if P[g, C] > P[a, C]:
                a = g
        want_am[C] = a
        if float(P[a, C]) > LS:
            want_phi[C] = P[a, C]
            want_alpha[C] = a + 1
    DenseOracle().collect(p, ph, phi, alpha, am)
    assert np.array_equal(am, want_am)
    assert np.array_equal(alpha, want_alpha)
    assert np.array_equal(phi, want_phi)


def test_move_frame_shifts_and_extrapolates():
    c = _case()
    p = c.params
    L = p.fnx * p.fny * p.fnz
    plane = p.fnx * p.fny
    rng = np.random.default_rng(2)
    ph = rng.uniform(-1, 1, p.num_theta * L).astype(F)
    before = ph.reshape(p.num_theta, p.fnz, p.fny, p.fnx).copy()
    z = np.asarray(c.z, F).copy()
    z0 = z.copy()
    alpha = rng.integers(0, p.num_theta + 1, L).astype(np.int32)
    full = np.zeros(plane * 4 * p.fnz, np.int32)
    loss = np.zeros(p.num_theta, np.int32)
    DenseOracle().move_frame(p, ph, z, alpha, full, loss, 2)
    A = ph.reshape(before.shape)
    assert np.array_equal(A[:, 1:-2, 1:-1, 1:-1], before[:, 2:-1, 1:-1, 1:-1])
    top = F(2) * before[:, -2, 1:-1, 1:-1] - before[:, -3, 1:-1, 1:-1]
    assert np.array_equal(A[:, -2, 1:-1, 1:-1], top)
    assert np.array_equal(A[:, :, 0, :], before[:, :, 0, :])  # halo untouched
    assert np.array_equal(z[1:-2], z0[2:-1]) and z[-2] == F(2) * z0[-2] - z0[-3]
    layer = alpha[plane:2 * plane]
    assert np.array_equal(full[3 * plane:4 * plane], layer)
    assert np.array_equal(loss, np.bincount(layer[(layer >= 1)] - 1, minlength=p.num_theta))


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dense")


def _golden_files():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.mark.parametrize("name", _golden_files())
def test_dense_oracle_reproduces_reference_dumps(name):
    """Every saved transition of the reference's full-PF kernels (tests/golden/dense,
    made by tests/golden/make_dense_golden.py on a B200) is reproduced bit for bit by the
    oracle's restatement with its pinned contraction switches."""
    d = np.load(os.path.join(GOLDEN, name))
    meta = eval(str(d["meta"]))
    c = cases.line_case(*meta["interior"], num_pf=5, num_grains=meta["grains"], seed=meta["seed"],
                        bc="110")
    p = c.params
    o = DenseOracle()
    Pi = lambda a: a.reshape(p.num_theta, p.fnz, p.fny, p.fnx)[:, 1:-1, 1:-1, 1:-1]
    ph0 = o.ini(p, c.phi, c.alpha)
    o.set_bc(p, ph0)
    # set_BC_3D fills halo edges and corners with racing threads: compare the
    # interior and the halo faces, the cells the 7-point stencil reads
    k3, j3, i3 = np.meshgrid(np.arange(p.fnz), np.arange(p.fny), np.arange(p.fnx), indexing="ij")
    nh = (((i3 == 0) | (i3 == p.fnx - 1)).astype(int) + ((j3 == 0) | (j3 == p.fny - 1)) +
          ((k3 == 0) | (k3 == p.fnz - 1)))
    faces = np.tile((nh <= 1).reshape(-1), p.num_theta)
    assert np.array_equal(ph0[faces], d["ph_0"][faces])
    saves = meta["saves"]
    checked = 0
    for k in saves:
        if k + 1 not in saves:
            continue
        # update k+1 runs at t = k*dt*tau0 (update 1 is the pre-loop one at t = 0)
        t = float(F(F(k) * F(p.dt)) * F(p.tau0)) if k > 0 else 0.0
        got = o.rhs(c, meta["R"], t, d["ph_%d" % k].copy())
        assert np.array_equal(Pi(got), Pi(d["ph_%d" % (k + 1)])), (name, k)
        checked += 1
    assert checked >= 2
    last = d["ph_%d" % max(saves)].copy()
    L = p.fnx * p.fny * p.fnz
    phi = np.full(L, -1.0, F)
    alpha = np.zeros(L, np.int32)
    am = np.zeros(L, np.int32)
    o.collect(p, last, phi, alpha, am)
    inner = ((i3 > 0) & (i3 < p.fnx - 1) & (j3 > 0) & (j3 < p.fny - 1) & (k3 > 0) &
             (k3 < p.fnz - 1)).reshape(-1)
    assert np.array_equal(alpha[inner], d["alpha_last"][inner])
    assert np.array_equal(phi[inner], d["phi_last"][inner])
