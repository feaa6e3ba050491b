"""Host side of the driver against the reference's own host code.

The reference's QOI.cpp, helper.cpp and DesignSettingData.cpp are compiled
unmodified into oracle/_ref/libref_host.so; the library's C++ restatements
(cupf_b200/host) must give identical results on the same inputs.
"""
import numpy as np
import pytest

from cupf_b200 import host_api
from oracle import RefHost


@pytest.fixture(scope="module")
def ref():
    return RefHost()


def random_alpha(shape, ngrains, seed, liquid_top=0.3, zero_frac=0.0):
    """Columnar grain map (fnz, fny, fnx): a Voronoi-like base extruded in z
    with a ragged liquid (0) top."""
    rng = np.random.default_rng(seed)
    fnz, fny, fnx = shape
    base = rng.integers(1, ngrains + 1, size=(fny, fnx)).astype(np.int32)
    # blocky grains
    base = np.repeat(np.repeat(base[::3, ::3], 3, 0), 3, 1)[:fny, :fnx]
    a = np.broadcast_to(base, shape).copy()
    h = (fnz * (1 - liquid_top) + rng.integers(-2, 3, size=(fny, fnx))).astype(int)
    kk = np.arange(fnz)[:, None, None]
    a[kk >= h[None]] = 0
    if zero_frac:
        a[rng.random(shape) < zero_frac] = 0
    return np.ascontiguousarray(a.reshape(-1).astype(np.int32))


@pytest.mark.parametrize("seed", range(4))
def test_grain_volumes_first_seen_order(ref, built, seed):
    shape = (20, 17, 23)
    a = random_alpha(shape, 40, seed, zero_frac=0.05)
    g_ref, v_ref = ref.calculate_qois(shape[2], shape[1], shape[0], 40, a)
    g, v = host_api.grain_volumes(shape[2], shape[1], shape[0], a)
    assert np.array_equal(g, g_ref) and np.array_equal(v, v_ref)


@pytest.mark.parametrize("seed", range(4))
def test_line_qois_and_sample_heights(ref, built, seed):
    shape = (30, 14, 18)
    ng = 25
    a = random_alpha(shape, ng, seed)
    loss = np.random.default_rng(seed).integers(0, 50, ng).astype(np.int32)
    z = np.arange(shape[0], dtype=np.float32)
    r = ref.calculate_line_qois(shape[2], shape[1], shape[0], ng, 0, a, z, loss, move_count=3)
    m = host_api.line_qois(shape[2], shape[1], shape[0], ng, 0, a, loss, 3)
    assert r[0] == m[0] and r[1] == m[1]
    assert np.array_equal(r[2], m[2]) and np.array_equal(r[3], m[3])
    assert ref.sample_heights(1, a, shape[2], shape[1], shape[0]) == \
        host_api.sample_heights(1, a, shape[2], shape[1], shape[0])


@pytest.mark.parametrize("seed", range(3))
def test_junctions_3d(ref, built, seed):
    # 3-D Voronoi map of 10 grains: quadruple junctions stay well below the
    # reference's preallocated 40 records per grain (it writes past them otherwise)
    shape = (14, 16, 16)
    rng = np.random.default_rng(seed)
    pts = rng.uniform(0, 1, (10, 3)) * np.array(shape)
    kk, jj, ii = np.meshgrid(*[np.arange(n) + 0.5 for n in shape], indexing="ij")
    d = [(kk - p[0]) ** 2 + (jj - p[1]) ** 2 + (ii - p[2]) ** 2 for p in pts]
    a = (np.argmin(np.stack(d), axis=0) + 1).astype(np.int32)
    a = np.ascontiguousarray(a.reshape(-1))
    r = ref.junctions_3d(16, 16, 14, a)
    m = host_api.junctions_3d(16, 16, 14, a)
    assert len(r) == len(m)
    assert np.array_equal(r, m)


LINES = [
    "dx = 0.8                            # mesh width",
    "kin_delta = 0.11",
    "delta = 0.01                    # strength",
    "  nts = 120          # number snapshots",
    "dx=0.5",
    "cfl = 1.5 dx = 0.3",
    "W0 = 1e-1 ",
    "# dx = 9",
    "nx = 13.7",
]


@pytest.mark.parametrize("line", LINES)
@pytest.mark.parametrize("key", ["dx", "delta", "kin_delta", "nts", "cfl", "W0", "nx"])
def test_get_param_matches_reference(ref, built, line, key):
    assert host_api.get_param(line, key, float, -7.0) == ref.get_param(line, key, float, -7.0)
    assert host_api.get_param(line, key, int, -7) == ref.get_param(line, key, int, -7)


def test_get_param_ignores_missing_value(built):
    """`key = ` with no value: the reference's stof throws an uncaught exception
    (aborting the driver); the library leaves the parameter unchanged."""
    assert host_api.get_param("dx = ", "dx", float, 3.5) == 3.5


ARGVS = [
    ["phase_field", "line.py"],
    ["phase_field", "line.py", "-s", "12", "-b", "110", "-l", "1", "-o", "out"],
    ["phase_field", "paraboloid.py", "-s", "3", "-b", "001", "-n", "2", "-f", "forcing/x"],
    ["phase_field", "cone.py", "-n", "1", "-m", "2", "-a", "1"],
    ["phase_field", "line.py", "--seed", "7", "--boundaryCondition", "111", "--lineConfig", "1"],
]


@pytest.mark.parametrize("argv", ARGVS, ids=range(len(ARGVS)))
def test_cli_options_match_reference(ref, built, argv):
    assert host_api.get_options(list(argv))[0].tolist() == ref.get_options(list(argv))[0].tolist()
    assert host_api.get_options(list(argv))[1:] == ref.get_options(list(argv))[1:]
