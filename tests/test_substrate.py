"""Seeded Voronoi substrate of the forcing folder.

* The library's generator (cupf_host_voronoi_substrate) against a plain-Python
  restatement of its stated algorithm (splitmix64 points and Box-Muller normals,
  nearest point with minimum-image distances, the reference's angle formula
  from graph_datastruct.py:256-269): identical ids, angles to float rounding.
* Its files (cupf_host_write_substrate) in the reference's savetxt formats.
* Orientations given as unit quaternions map to the reference's two angles
  (those of the crystal [001] axis; the rotation about it is dropped), and the
  driver reads quaternions.txt where theta.txt is absent.
* Substrates made by the reference's own graph() (fixtures from
  tests/golden/substrate/make_graph_substrate.py) and by the library's generator
  load through the driver's forcing-folder reader exactly as through the
  reference's PhaseFieldCpu.cpp set-up (parseInputParams + cpuSetup + initField,
  compiled unmodified into oracle/_ref), bit for bit.
"""
import ctypes as C
import glob
import math
import os

import numpy as np
import pytest

from cupf_b200 import abi, host_api, preprocess

HERE = os.path.dirname(os.path.abspath(__file__))
M64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & M64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def uniform(self):
        return (self.next() >> 11) * 2.0 ** -53


def python_substrate(nxp, nyp, ng, seed, periodic):
    r = SplitMix64(seed)
    pts = [(r.uniform() * nxp, r.uniform() * nyp) for _ in range(ng)]
    px = np.array([p[0] for p in pts])
    py = np.array([p[1] for p in pts])
    cx = np.arange(nxp) + 0.5
    cy = np.arange(nyp) + 0.5
    best = np.full((nyp, nxp), np.inf)
    alpha = np.ones((nyp, nxp), np.int32)
    for g in range(ng):
        dx = np.abs(cx - px[g])
        dy = np.abs(cy - py[g])
        if periodic:
            dx = np.minimum(dx, nxp - dx)
            dy = np.minimum(dy, nyp - dy)
        d = dy[:, None] * dy[:, None] + dx[None, :] * dx[None, :]
        m = d < best
        best[m] = d[m]
        alpha[m] = g + 1
    a = SplitMix64(seed ^ 0x5DEECE66D)
    tx, tz = [], []
    for g in range(ng):
        u1, u2, u3, u4 = 1.0 - a.uniform(), a.uniform(), 1.0 - a.uniform(), a.uniform()
        s1, s3 = math.sqrt(-2.0 * math.log(u1)), math.sqrt(-2.0 * math.log(u3))
        ux, uy, uz = s1 * math.cos(2 * math.pi * u2), s1 * math.sin(2 * math.pi * u2), \
            s3 * math.cos(2 * math.pi * u4)
        tx.append(math.atan2(uy, ux) % math.pi)
        tz.append(math.atan2(math.sqrt(ux * ux + uy * uy), uz) % math.pi)
    return alpha, np.array([0.0] + tx + tz)


@pytest.mark.parametrize("nxp,nyp,ng,seed,periodic", [(40, 30, 12, 5, True), (33, 57, 40, 123, False),
                                                      (64, 64, 1, 9, True), (20, 20, 90, 2**40 + 3, True)])
def test_generator_matches_stated_algorithm(built, nxp, nyp, ng, seed, periodic):
    alpha, theta = preprocess.native_substrate(nxp, nyp, ng, seed, periodic)
    ra, rt = python_substrate(nxp, nyp, ng, seed, periodic)
    assert np.array_equal(alpha, ra)
    assert np.allclose(theta, rt, rtol=0, atol=4e-7)
    assert theta[0] == 0 and np.all((theta >= 0) & (theta < np.float32(math.pi)))
    if ng <= (nxp * nyp) // 50:
        assert np.unique(alpha).size == ng  # every grain owns pixels at this density
    # the same seed gives the same substrate; another seed another
    assert np.array_equal(preprocess.native_substrate(nxp, nyp, ng, seed, periodic)[0], alpha)
    if ng > 1:
        assert not np.array_equal(preprocess.native_substrate(nxp, nyp, ng, seed + 1, periodic)[0],
                                  alpha)


def test_files_in_reference_format(built, tmp_path):
    alpha, theta = preprocess.native_substrate(17, 11, 6, 4)
    r = abi.lib().cupf_host_write_substrate(str(tmp_path).encode(), 17, 11,
                                            alpha.ctypes.data_as(C.POINTER(C.c_int32)), 6,
                                            theta.ctypes.data_as(C.POINTER(C.c_float)))
    assert r == 0
    a_lines = (tmp_path / "alpha.txt").read_text().splitlines()
    assert a_lines == ["%d" % v for v in alpha.reshape(-1)]
    t_lines = (tmp_path / "theta.txt").read_text().splitlines()
    assert t_lines == ["%1.4e" % v for v in theta.astype(np.float64)]  # numpy.savetxt's form
    assert (tmp_path / "NG.txt").read_text() == "6\n"


def _setup_both(tmp_path, monkeypatch, substrate, ng, seed, Lx):
    from oracle import RefSetup
    ref = RefSetup()
    folder = tmp_path / "forcing" / ("case%d" % seed)
    # a window of 16 planes (moving_ratio * nx with nx = Lx / 0.08) in a column of
    # 32 (asp_ratio_zx * nx); the macro grid spans twice the column
    nx = int(round(Lx / 0.08))
    Lz = 32 * 0.08
    preprocess.write_line_forcing(str(folder), Lx, Lx, 2 * Lz, num_grains=ng, seed=seed, G=2.0, R=0.4,
                                  z0=0.5, top=0.4, t_end=1e-6, substrate=substrate)
    preprocess.write_input_file(str(tmp_path / "line.py"), Lx, nts=2, asp_ratio_yx=1.0,
                                asp_ratio_zx=32 / nx, moving_ratio=16 / nx, num_pf=8)
    monkeypatch.chdir(tmp_path)
    kw = dict(bc=(1, 1, 0), line_config=True, cap=1 << 21)
    return host_api.setup_state("line.py", str(folder), **kw), ref.setup("line.py", str(folder), **kw)


def _assert_same(mine, theirs):
    assert mine.keys() == theirs.keys()
    for k, v in theirs.items():
        if isinstance(v, np.ndarray):
            assert v.dtype == mine[k].dtype and v.shape == mine[k].shape, k
            assert np.array_equal(mine[k].view(np.int32), v.view(np.int32)), k


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(HERE, "golden", "substrate",
                                                               "graph_*.npz"))),
                         ids=os.path.basename)
def test_reference_graph_substrate_loads_like_reference(built, tmp_path, monkeypatch, path):
    try:
        from oracle import RefSetup  # noqa: F401
        RefSetup()
    except (FileNotFoundError, OSError) as e:
        pytest.skip("reference host code not built: %s" % e)
    f = np.load(path)
    alpha, theta, ng = f["alpha"].astype(np.int32), f["theta"], int(f["ng"])
    mine, theirs = _setup_both(tmp_path, monkeypatch, (alpha, theta), ng, int(f["seed"]),
                               float(f["lxd"]))
    _assert_same(mine, theirs)
    # the solid cells carry the graph's ids (initField reads alpha_mac[(j-1)*(nx+1)+(i-1)])
    fnx, fny = alpha.shape[1] + 2, alpha.shape[0] + 2
    a = mine["alpha"].reshape(-1, fny, fnx)
    solid = a[1:-1] > 0
    assert solid.sum() > 0
    expect = np.broadcast_to(alpha, a[1:-1, 1:-1, 1:-1].shape)
    assert np.array_equal(a[1:-1, 1:-1, 1:-1][solid[:, 1:-1, 1:-1]],
                          expect[solid[:, 1:-1, 1:-1]])


def test_native_substrate_loads_like_reference(built, tmp_path, monkeypatch):
    try:
        from oracle import RefSetup  # noqa: F401
        RefSetup()
    except (FileNotFoundError, OSError) as e:
        pytest.skip("reference host code not built: %s" % e)
    mine, theirs = _setup_both(tmp_path, monkeypatch, "native", 23, 11, 2.48)
    _assert_same(mine, theirs)


# ---- orientations as unit quaternions ----

def quat_mul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])


def quat_z_to(u):
    """A unit quaternion rotating the z axis onto the unit vector u (shortest arc)."""
    u = np.asarray(u, np.float64) / np.linalg.norm(u)
    ax = np.cross([0.0, 0.0, 1.0], u)
    s = np.linalg.norm(ax)
    ang = math.atan2(s, u[2])
    if s < 1e-15:
        ax = np.array([1.0, 0.0, 0.0])
    else:
        ax = ax / s
    return np.concatenate([[math.cos(ang / 2)], math.sin(ang / 2) * ax])


def reference_angles(u):
    """graph_datastruct.py:256-269 for one direction u."""
    return math.atan2(u[1], u[0]) % math.pi, math.atan2(math.hypot(u[0], u[1]), u[2]) % math.pi


def test_quaternions_map_to_the_reference_angles(built):
    rng = np.random.default_rng(5)
    us = rng.standard_normal((60, 3))
    us /= np.linalg.norm(us, axis=1)[:, None]
    q = np.stack([quat_z_to(u) for u in us])
    q[::7] *= -2.5  # scale and sign do not matter
    theta = preprocess.quaternion_angles(q)
    want = np.array([reference_angles(u) for u in us])
    assert theta[0] == 0
    assert np.allclose(theta[1:61], want[:, 0], atol=2e-6) and np.allclose(theta[61:], want[:, 1], atol=2e-6)
    # the rotation about the crystal [001] axis is the dropped third angle
    spun = np.stack([quat_mul(qq, [math.cos(g / 2), 0.0, 0.0, math.sin(g / 2)])
                     for qq, g in zip(q, rng.uniform(0, 2 * math.pi, 60))])
    assert np.allclose(preprocess.quaternion_angles(spun), theta, atol=2e-6)
    with pytest.raises(ValueError):
        preprocess.quaternion_angles(np.zeros((2, 4)))


def test_driver_reads_quaternions_in_place_of_angles(built, tmp_path, monkeypatch):
    ng = 9
    rng = np.random.default_rng(2)
    us = rng.standard_normal((ng, 3))
    q = np.stack([quat_z_to(u) for u in us])
    folder = tmp_path / "forcing" / "case3"
    preprocess.write_line_forcing(str(folder), 2.48, 2.48, 4.96, num_grains=ng, seed=3, G=1.0,
                                  R=0.05, z0=0.6, top=0.3, t_end=5e-7, quaternions=q)
    assert not (folder / "theta.txt").exists()
    preprocess.write_input_file(str(tmp_path / "line.py"), 2.48, nts=2, asp_ratio_zx=2.0, num_pf=5)
    monkeypatch.chdir(tmp_path)
    st = host_api.setup_state("line.py", str(folder), bc=(1, 1, 0), line_config=True, cap=1 << 20)
    # the file holds the quaternions to 9 digits; the driver converts them itself
    qf = np.loadtxt(folder / "quaternions.txt").reshape(-1, 4).astype(np.float32).astype(np.float64)
    theta = preprocess.quaternion_angles(qf)
    assert np.allclose(st["sint"][:2 * ng + 1], np.sin(theta), atol=1e-6)
    assert np.allclose(st["cost"][:2 * ng + 1], np.cos(theta), atol=1e-6)
