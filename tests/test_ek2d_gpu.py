"""2D Echebarria–Karma line model on the GPU: parity of the library's kernel
with the reference's own kernels (2DdendriteMPI/line_model/PF.cu compiled for
sm_100a), with the CPU oracle, and the split-precision error against FP64.

FP32 results are compared with a tolerance, not bit for bit: the library
evaluates each edge flux once for both cells that share it (the reference
evaluates it from each side, in a different operand order), computes phi from
psi on the device, and forms Up in FP64; every difference is a few float ulps
per step.
"""
import json
import os

import numpy as np
import pytest

from cupf_b200 import ek2d
from cupf_b200.ek2d import EK2DSolver
from oracle import Ek2dOracle, RefEK2D

pytestmark = pytest.mark.gpu

OUT = os.environ.get("CUPF_RECORD_DIR", "")  # measured numbers are written here when set


def _record(name, rec):
    if os.path.isdir(OUT):
        with open(os.path.join(OUT, name), "w") as f:
            json.dump(rec, f, indent=1)


def _interior(a):
    return a[1:-1, 1:-1]


def _developed(steps=150, nx=96, ny=256):
    """A case and an FP32 oracle state with a curved front and nonzero dpsi."""
    c = ek2d.directional_case(nx, ny, 400, sites=4, amp=2.0)
    o = Ek2dOracle()
    s = o.new_state(c, np.float32)
    o.run(c, s, steps, prestep=True)
    return c, s


def _step_args(c):
    """intR and lT of the first fused step, as the library forms them (FP64)."""
    p = c.params
    intR = float(c.Rt[0]) * float(p.tau0) / float(p.W0) * float(p.dt)
    lT = (float(p.c_infm) * (1.0 / float(p.k) - 1.0) / float(c.Gt[0])) / float(p.W0)
    return intR, lT


@pytest.mark.parametrize("prestep", [0, 1])
def test_one_step_matches_reference_kernels(built, prestep):
    c, s = _developed()
    intR, lT = _step_args(c)
    if prestep:
        intR = 0.0
    ref = RefEK2D().step(c.params, s["psi"], s["phi"], s["U"], s["dpsi"], c.y, intR, lT, prestep)
    ora = Ek2dOracle().step(c.params, s["psi"], s["phi"], s["U"], s["dpsi"], c.y, np.float32(intR),
                            np.float32(lT), prestep, 1)
    with EK2DSolver(c) as sv:
        sv.set_state(s["psi"], s["U"], s["dpsi"])
        if prestep:
            sv.prestep()
        else:
            sv.step(1)
        lib = sv.get_state()
    rec = {"prestep": prestep}
    for name, got in (("library", lib), ("oracle_f32", ora)):
        for k in ("psi", "phi", "U", "dpsi"):
            d = np.abs(_interior(got[k]).astype(np.float64) - _interior(ref[k]))
            scale = 1.0 + np.abs(_interior(ref[k]))
            rec["%s_%s_max_rel" % (name, k)] = float((d / scale).max())
            rec["%s_%s_normwise" % (name, k)] = float(d.max() / np.abs(_interior(ref[k])).max())
    _record("ek2d_one_step_%d.json" % prestep, rec)
    for name in ("library", "oracle_f32"):
        # psi, phi, U per cell within a few float ulps
        assert rec[name + "_psi_max_rel"] < 2e-6, rec
        assert rec[name + "_phi_max_rel"] < 2e-6, rec
        assert rec[name + "_U_max_rel"] < 2e-6, rec
        # dpsi/dt is a small difference of O(1) flux terms in places, and the
        # anisotropy switches at |grad phi|^2 = eps: bound it against its own scale
        assert rec[name + "_dpsi_normwise"] < 1e-4, rec


def test_run_matches_reference_setup(built):
    # the reference's whole time loop: pre-step, 250 fused steps, tip searches at
    # 100 and 200 with frame moves (front above the 70 % threshold)
    c = ek2d.directional_case(64, 256, 250, front_frac=0.72, sites=4, amp=1.0)
    ref = RefEK2D().setup(c)
    with EK2DSolver(c) as sv:
        sv.set_state(c.psi, c.U)
        sv.prestep()
        sv.step(249)
        a = sv.get_state()       # setup() copies psi/phi of step Mt-1 ...
        sv.step(1)
        b = sv.get_state()       # ... and U of step Mt
        info = sv.info()
        y = sv.get_y()
    rec = {"shifts": info["shifts"], "cur_tip": info["cur_tip"],
           "psi_max_abs": float(np.abs(_interior(a["psi"]) - _interior(ref["psi"])).max()),
           "phi_max_abs": float(np.abs(_interior(a["phi"]) - _interior(ref["phi"])).max()),
           "U_max_abs": float(np.abs(_interior(b["U"]) - _interior(ref["U"])).max()),
           "y_max_abs": float(np.abs(y[1:-1] - ref["y"][1:-1]).max())}
    _record("ek2d_vs_reference_setup.json", rec)
    assert info["shifts"] > 0, rec
    assert rec["phi_max_abs"] < 1e-4 and rec["U_max_abs"] < 1e-4, rec
    assert rec["y_max_abs"] < 1e-3, rec


def test_fp64_device_matches_fp64_oracle(built):
    c = ek2d.directional_case(64, 256, 300, front_frac=0.72, sites=4, amp=1.0)
    o = Ek2dOracle()
    s = o.new_state(c, np.float64)
    o.run(c, s, 300, prestep=True)
    with EK2DSolver(c, precision="fp64") as sv:
        # the oracle starts from phi = tanh(psi/sqrt2) of the float psi, as the device
        sv.set_state(c.psi, c.U)
        sv.prestep()
        sv.step(300)
        d = sv.get_state_f64()
        info = sv.info()
    assert info["shifts"] == s["info"].shifts > 0
    rec = {k: float(np.abs(_interior(d[k]) - _interior(s[k])).max()) for k in ("psi", "phi", "U", "dpsi")}
    _record("ek2d_fp64_vs_oracle.json", rec)
    # both in double; they differ in operand order (shared edge fluxes), and the
    # growing front amplifies those 1e-16 differences over 300 steps
    assert rec["phi"] < 1e-7 and rec["U"] < 1e-7, rec
    assert rec["psi"] < 1e-8 * np.abs(s["psi"]).max(), rec


@pytest.fixture(scope="module")
def split_reference():
    """A reduced directional-solidification run in the FP64 CPU oracle."""
    c = ek2d.directional_case(128, 512, 3000, front_frac=0.3, sites=8, amp=0.5)
    o = Ek2dOracle()
    s = o.new_state(c, np.float64)
    o.run(c, s, 3000, prestep=True)
    dxd = float(c.params.dx) * float(c.params.W0)
    q0 = ek2d.qois(c.phi, c.y64(), dxd)
    q = ek2d.qois(s["phi"].astype(np.float32), s["y"], dxd)
    return c, s, q0, q


@pytest.mark.parametrize("prec", ["fp32", "fp16", "bf16", "fp64"])
def test_split_precision_error_2d(built, split_reference, prec):
    c, s, q0, q64 = split_reference
    dxd = float(c.params.dx) * float(c.params.W0)
    with EK2DSolver(c, precision=prec) as sv:
        sv.set_state(c.psi, c.U)
        sv.prestep()
        sv.step(3000)
        st = sv.get_state()
        y = sv.get_y()
    q = ek2d.qois(st["phi"], y, dxd)
    adv = q64["tip_y"] - q0["tip_y"]
    band = np.abs(_interior(s["phi"])) < 0.9
    rec = {"precision": prec, "steps": 3000, "grid": [128, 512],
           "tip_y": q["tip_y"], "tip_y_fp64": q64["tip_y"], "tip_advance_fp64_um": adv,
           "tip_advance_rel_err": abs(q["tip_y"] - q64["tip_y"]) / abs(adv),
           "tip_position_err_cells": abs(q["tip_y"] - q64["tip_y"]) / dxd,
           "front_mean_rel_err": abs(q["front_mean_y"] - q64["front_mean_y"]) /
                                 abs(q64["front_mean_y"] - q0["front_mean_y"]),
           "spacing": q["spacing"], "spacing_fp64": q64["spacing"],
           "phi_max_abs_err": float(np.abs(_interior(st["phi"]) - _interior(s["phi"])).max()),
           "U_max_abs_err_band": float(np.abs(_interior(st["U"]) - _interior(s["U"]))[band].max())}
    _record("ek2d_split_precision_%s.json" % prec, rec)
    print(rec)
    assert adv > 0.5 * dxd, rec  # the front moved
    if prec in ("fp32", "fp64"):
        assert rec["tip_advance_rel_err"] < 1e-3, rec
    else:
        # 16-bit storage: the tip within a quarter of a cell of FP64 after 3000 steps
        assert rec["tip_position_err_cells"] < 0.25, rec


def test_phase_field_2d_executable(built, tmp_path):
    # the command-line driver on a written input folder gives the Python API's run
    import subprocess
    c = ek2d.directional_case(64, 256, 300, front_frac=0.72, sites=4, amp=1.0)
    inp = ek2d.write_line_model_inputs(c, str(tmp_path), ztip0=5.0)
    exe = os.path.join(os.path.dirname(ek2d.abi.LIB_PATH), "phase_field_2d")
    r = subprocess.run([exe, inp, str(tmp_path), "-o", str(tmp_path)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    from tests.h5read import H5File
    out = H5File(os.path.join(str(tmp_path), "line_nx64_ny256_Mt300_seed0.h5"))
    with EK2DSolver(c) as sv:
        sv.set_state(c.psi, c.U)
        sv.prestep()
        sv.step(300)
        st = sv.get_state()
        y = sv.get_y()
        info = sv.info()
    assert info["shifts"] > 0
    assert np.array_equal(out["phi"].reshape(c.fny, c.fnx), st["phi"])
    assert np.allclose(out["y_coordinates"], (y - 5.0).astype(np.float32))
    k = float(c.params.k)
    cl = (1 + (1 - k) * st["U"]) * (k * (1 + st["phi"]) / 2 + (1 - st["phi"]) / 2) / (1 + (1 - k) * -1.0)
    assert np.allclose(out["Uc"].reshape(c.fny, c.fnx), cl, rtol=1e-6, atol=1e-6)
    assert "primary spacing" in r.stdout


def test_speed_vs_reference_kernel(built):
    # device time per step of the library's FP32 / FP16 step against the
    # reference's set_BC + merge_PF pair on the same 1024x4096 state
    c = ek2d.directional_case(1024, 4096, 2000, sites=16, amp=0.5)
    ref = RefEK2D()
    intR, lT = _step_args(c)
    d = np.zeros_like(c.psi)
    ref_ms = ref.time_steps(c.params, c.psi, c.phi, c.U, d, c.y, intR, lT, 200)
    rec = {"grid": [1024, 4096], "reference_ms_per_step": ref_ms / 200}
    for prec in ("fp32", "fp16"):
        with EK2DSolver(c, precision=prec) as sv:
            sv.set_state(c.psi, c.U)
            sv.prestep()
            sv.time_steps(20)
            rec[prec + "_ms_per_step"] = sv.time_steps(200) / 200
    rec["speedup_fp32"] = rec["reference_ms_per_step"] / rec["fp32_ms_per_step"]
    _record("ek2d_perf_vs_reference.json", rec)
    print(rec)
    assert rec["speedup_fp32"] > 1.0, rec
