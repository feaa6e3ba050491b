"""2D Echebarria–Karma line model: host code and the oracle, on the CPU.

- input parsing and parameter derivation follow the reference's main.cpp
  (2DdendriteMPI/line_model/main.cpp:37-52, 95-185), restated here in numpy
  with float32 where the reference keeps floats;
- the initial fields follow main.cpp:225-271;
- the oracle's boundary fill, frame move and time loop keep the properties the
  reference's kernels have (x-periodic / y-mirror halos, mirror symmetry of a
  symmetric front, FP32 close to FP64 over short runs);
- the quantities of interest agree with an independent numpy computation.
"""
import ctypes as C
import os

import numpy as np
import pytest

from cupf_b200 import abi, ek2d
from oracle import Ek2dOracle

f32 = np.float32

INPUT_TEXT = """\
## key = value lines in the reference line model's format
    G = 0.05                        # thermal gradient        K/um
    R = 2000                        # pulling speed           um/s
    delta = 0.02
    k = 0.14
    c_infm = 7.8
    Dl = 3000
    d0 = 0.005
    W0 = 0.14
    lT = c_infm*( 1.0/k-1 )/G       # must not be read as G
    R_tilde = R*tau0/W0             # must not be read as R
    eps = 1e-8
    alpha0 = 10
    dx = 0.8
    asp_ratio = 3
   # nx = 128                       # not a key of main.cpp
    lxd = 30
    eta = 0.0
    seed_val = 7
    noi_period = 20
    U0 = -1
    Ny = 40
    Nt = 5
    ztip0 = 12.5
    cfl = 0.25
"""


def test_parse_input(tmp_path):
    path = tmp_path / "input_file"
    path.write_text(INPUT_TEXT)
    p = abi.cupf_ek2d_params()
    ny, nt, zt = C.c_int32(), C.c_int32(), C.c_float()
    abi.check(abi.lib().cupf_ek2d_parse_input(str(path).encode(), C.byref(p), C.byref(ny),
                                              C.byref(nt), C.byref(zt)))
    assert (p.G, p.R, p.delta, p.alpha0, p.lxd, p.asp_ratio) == (f32(0.05), 2000, f32(0.02), 10, 30, 3)
    assert (p.seed_val, p.noi_period, ny.value, nt.value, zt.value) == (7, 20, 40, 5, 12.5)
    assert p.cfl == f32(0.25) and p.eps == f32(1e-8) and p.U0 == -1


def _derive_numpy(v, t_last):
    """main.cpp:158-185 with numpy scalars typed as the reference types them."""
    k, G, W0, d0, Dl, R = (f32(v[n]) for n in ("k", "G", "W0", "d0", "Dl", "R"))
    c_infm, dx, cfl, lxd, asp, delta, alpha0 = (f32(v[n]) for n in (
        "c_infm", "dx", "cfl", "lxd", "asp_ratio", "delta", "alpha0"))
    o = {}
    o["lT"] = f32(float(c_infm) * (1.0 / float(k) - 1) / float(G))
    o["lamd"] = f32(5 * np.sqrt(2.0) / 8 * float(W0) / float(d0))
    o["tau0"] = f32(0.6267 * float(o["lamd"]) * float(W0) * float(W0) / float(Dl))
    o["R_tilde"] = f32(R * o["tau0"] / W0)
    o["Dl_tilde"] = f32(float(Dl * o["tau0"]) / float(W0) ** 2)
    o["lT_tilde"] = f32(o["lT"] / W0)
    o["dt"] = f32(float(cfl) * float(dx) ** 2 / (4 * float(o["Dl_tilde"])))
    o["nx"] = int(f32(lxd / f32(dx * W0)))
    o["ny"] = int(f32(asp * f32(o["nx"])))
    mt = int(f32(f32(f32(t_last) / o["tau0"]) / o["dt"]))
    o["Mt"] = (mt // 2) * 2
    o["hi"] = f32(1.0 / float(dx))
    o["cosa"] = f32(np.cos(float(f32(alpha0 / f32(180))) * np.pi))
    o["a_s"] = f32(1 - 3.0 * float(delta))
    o["epsilon"] = f32(4.0 * float(delta) / float(o["a_s"]))
    o["a_12"] = f32(4.0 * float(o["a_s"]) * float(o["epsilon"]))
    o["dt_sqrt"] = f32(np.sqrt(o["dt"]))
    return o


@pytest.mark.parametrize("over", [{}, dict(G=0.1, R=1e4, cfl=0.2, lxd=50.0, alpha0=15.0)])
def test_derive_matches_main_cpp(over):
    v = dict(ek2d.LINE_MODEL_INPUT)
    v.update(over)
    p = ek2d.make_params(**v)
    ek2d.derive(p, 0.0125)
    want = _derive_numpy(v, 0.0125)
    for k, w in want.items():
        assert getattr(p, k) == w, (k, getattr(p, k), w)
    assert (p.tipp, p.blank, p.ls) == (100, f32(0.3), f32(-0.995))


def test_initial_fields_follow_main_cpp():
    p = ek2d.make_params(lxd=(20 + 0.5) * 0.112, asp_ratio=3.0)
    ek2d.derive(p, 1e-3)
    assert (p.nx, p.ny) == (20, 60)
    ymac = (np.arange(90, dtype=np.float32) * f32(0.09) - f32(1.3)).astype(np.float32)
    psim = np.linspace(8, -30, 90).astype(np.float32)
    um = np.linspace(-0.2, -1.0, 90).astype(np.float32)
    x, y, psi, phi, U = ek2d.initial_fields(p, ymac, psim, um)
    dxd = f32(p.dx * p.W0)
    assert np.array_equal(x, ((np.arange(p.nx + 2) - 1) * dxd).astype(np.float32))
    yy = ((np.arange(p.ny + 3) - 1).astype(np.float32) * dxd + ymac[0]).astype(np.float32)
    assert np.array_equal(y, yy)
    Dy = f32(ymac[1] - ymac[0])
    for j in range(1, p.ny + 2):
        s = f32(f32(y[j] - ymac[0]) / Dy)
        ky = int(s)
        d = f32(s - f32(ky))
        ps = f32(f32(f32(1) - d) * psim[ky] + f32(d * psim[ky + 1]))
        assert psi[j, 1] == ps and np.all(psi[j, 1:-1] == ps)
        assert np.all(U[j, 1:-1] == f32(f32(f32(1) - d) * um[ky] + f32(d * um[ky + 1])))
    assert np.all(psi[0] == 0) and np.all(psi[:, 0] == 0)
    assert np.allclose(phi[1:-1, 1:-1], np.tanh(psi[1:-1, 1:-1] / np.sqrt(2.0)), atol=1e-6)


def test_directional_case_geometry():
    c = ek2d.directional_case(64, 192, 300, sites=4, amp=0.3)
    p = c.params
    assert (p.nx, p.ny, p.Mt) == (64, 192, 300)
    # the planar front sits at the solidus (y = 0, Up = 0) at row j_front
    q = ek2d.qois(c.phi, c.y64(), float(p.dx) * float(p.W0))
    assert abs(q["front_mean_y"]) < 0.3 * float(p.W0)
    j = c.info["j_front"]
    assert abs(c.y64()[j]) < 1e-6
    # U = 0 in the solid, the boundary layer -1 + exp(-y/lD) ahead, U0 far away
    lD = float(p.Dl) / float(c.Rt[0])
    y = c.y64()
    ahead = (y > 0.5) & (y < 3 * lD)
    assert np.allclose(c.U[ahead, 5], -1.0 + np.exp(-y[ahead] / lD), atol=2e-3)
    assert np.all(c.U[1:j - 2, 1:-1] == 0) and np.all(c.U[-2, 1:-1] == f32(-1))
    # the seeded bumps move the front by at most amp W0
    assert abs(q["tip_y"]) <= 0.31 * float(p.W0)


def test_oracle_bc_is_periodic_x_mirror_y():
    o = Ek2dOracle()
    a = np.random.default_rng(1).standard_normal((9, 7))
    b = o.bc(a.copy())
    assert np.array_equal(b[1:-1, 1:-1], a[1:-1, 1:-1])
    assert np.array_equal(b[0, 1:-1], a[2, 1:-1]) and np.array_equal(b[-1, 1:-1], a[-3, 1:-1])
    assert np.array_equal(b[:, 0], b[:, -2]) and np.array_equal(b[:, -1], b[:, 1])
    assert b[0, 0] == a[2, -2] and b[-1, -1] == a[-3, 1]


def _mirror(a):
    """x -> nx+1-x on the interior columns."""
    m = a.copy()
    m[:, 1:-1] = a[:, -2:0:-1]
    return m


def test_oracle_keeps_mirror_symmetry():
    # a front symmetric about the domain centre stays symmetric under the
    # isotropic-in-x (alpha0 = 0) equations with periodic x
    c = ek2d.directional_case(48, 128, 200, sites=0, amp=0.0)
    x = np.arange(c.fnx) - 0.5 - c.params.nx / 2
    bump = 0.8 * np.exp(-(x / 6.0) ** 2)
    c.psi[1:-1, 1:-1] += bump[1:-1][None, :].astype(np.float32)
    c.phi[:] = np.tanh(c.psi / np.sqrt(2.0)).astype(np.float32)
    o = Ek2dOracle()
    s = o.new_state(c, np.float64)
    o.run(c, s, 200, prestep=True)
    for k in ("psi", "U", "dpsi"):
        a = s[k][1:-1]
        assert np.abs(a - _mirror(s[k])[1:-1]).max() <= 1e-9 * (1 + np.abs(a).max()), k
    assert np.abs(s["psi"] - c.psi).max() > 1e-3  # it moved


def test_oracle_f32_tracks_f64():
    c = ek2d.directional_case(48, 160, 300, sites=3, amp=0.5)
    o = Ek2dOracle()
    a = o.new_state(c, np.float64)
    b = o.new_state(c, np.float32)
    o.run(c, a, 300, prestep=True)
    o.run(c, b, 300, prestep=True)
    band = np.abs(a["phi"]) < 0.99
    assert np.abs(a["phi"] - b["phi"]).max() < 1e-4
    assert np.abs(a["U"] - b["U"]).max() < 1e-4
    assert np.abs(a["psi"] - b["psi"])[band].max() < 1e-4
    assert abs(a["info"].intR - b["info"].intR) < 1e-5 * a["info"].intR


def test_oracle_frame_moves_with_front():
    # front above the tip threshold: the first tip search moves the frame until
    # the tip row is below it, keeping the profile (rows shift, y follows)
    c = ek2d.directional_case(32, 120, 200, front_frac=0.8, sites=0, amp=0.0)
    o = Ek2dOracle()
    s = o.new_state(c, np.float64)
    psi0 = s["psi"].copy()
    o.run(c, s, 100)
    info = s["info"]
    fny = c.fny
    assert info.shifts > 0 and info.cur_tip < int(0.7 * fny)
    k = info.shifts
    # y moved by k rows exactly (uniform grid, linear extrapolation)
    assert np.allclose(s["y"][1:-1], c.y64()[1:-1] + k * float(c.params.dx) * float(c.params.W0),
                       rtol=0, atol=1e-9)
    # far below the front the solid moved down by k rows and barely changed
    j = 5
    assert abs(s["psi"][j, 5] - psi0[j + k, 5]) < 0.05 * abs(psi0[j + k, 5])


def test_qois_against_numpy():
    fnx, fny, nx = 130, 90, 128
    dxd = 0.112
    y = 3.0 + (np.arange(fny) - 1) * dxd
    xi = np.arange(nx)
    h = 40 + 10 * (0.5 + 0.5 * np.cos(2 * np.pi * 8 * xi / nx))  # 8 cells of height 40..50 rows
    jj = np.arange(fny)[:, None]
    phi = np.tanh((h[None, :] - jj) / 1.5).astype(np.float32)
    full = np.zeros((fny, fnx), np.float32)
    full[:, 1:-1] = phi
    q = ek2d.qois(full, y, dxd)
    # numpy: each column's highest crossing, interpolated
    tips = []
    for i in range(nx):
        col = full[:, i + 1].astype(np.float64)
        js = [j for j in range(1, fny - 2) if col[j] >= 0 and col[j + 1] < 0]
        j = max(js)
        tips.append(y[j] + dxd * col[j] / (col[j] - col[j + 1]))
    assert abs(q["tip_y"] - max(tips)) < 1e-9 and abs(q["front_mean_y"] - np.mean(tips)) < 1e-9
    assert q["spacing_k"] == 8 and abs(q["spacing"] - nx * dxd / 8) < 1e-9
    frac = (full[:, 1:-1] > 0).mean(axis=1)
    ok = (frac > 0.05) & (frac < 0.95)
    ok[0] = ok[-1] = False
    assert q["mushy_row"] == int(np.flatnonzero(ok)[np.argmin(np.abs(frac[ok] - 0.5))])
    # a planar front has no cells
    flat = np.zeros_like(full)
    flat[:, 1:-1] = np.tanh((45 - jj) / 1.5)
    assert ek2d.qois(flat, y, dxd)["spacing"] == 0.0


def test_library_loads_2d_symbols():
    L = abi.lib()
    for name in ("cupf_ek2d_create", "cupf_ek2d_destroy", "cupf_ek2d_set_thermal",
                 "cupf_ek2d_set_state", "cupf_ek2d_prestep", "cupf_ek2d_step",
                 "cupf_ek2d_get_state", "cupf_ek2d_get_state_f64", "cupf_ek2d_get_y", "cupf_ek2d_info_get",
                 "cupf_ek2d_row_means", "cupf_ek2d_time_steps", "cupf_ek2d_stream",
                 "cupf_ek2d_derive", "cupf_ek2d_parse_input", "cupf_host_ek2d_initial_fields",
                 "cupf_host_ek2d_perturb", "cupf_host_ek2d_qois"):
        assert hasattr(L, name), name
    exe = os.path.join(os.path.dirname(abi.LIB_PATH), "phase_field_2d")
    assert os.access(exe, os.X_OK)


def test_line_model_inputs_round_trip(tmp_path):
    # a case written as the reference's input_file + macro folder and read back
    # the way main.cpp reads it gives the same parameters and initial fields
    c = ek2d.directional_case(64, 256, 300, sites=4, amp=1.0)
    inp = ek2d.write_line_model_inputs(c, str(tmp_path))
    r = ek2d.line_model_case(inp, str(tmp_path))
    for k in ("nx", "ny", "Mt", "dt", "tau0", "lamd", "Dl_tilde", "lT_tilde", "hi", "y0", "seed_val"):
        assert getattr(r.params, k) == getattr(c.params, k), k
    for k in ("psi", "phi", "U", "x", "y"):
        assert np.array_equal(getattr(r, k), getattr(c, k)), k
