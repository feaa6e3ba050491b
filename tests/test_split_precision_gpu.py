"""Split precision (16-bit phi + int16 id storage, FP32 arithmetic) against the
FP64 transcription of the reference step.

C1 (64^3 interior, 20 grains, NUM_PF=5) is advanced 1000 steps in FP32, FP16 and
BF16 storage on the GPU and in FP64 on the CPU (the oracle).  Compared:
  * grain volume fractions of the argmax map (voxels of grain g / solid voxels),
    as the volume-weighted L1 relative error sum|V_g - V64_g| / sum V64_g;
  * the mean interface height (FP64 solid volume / base area);
  * the FP64 interface area.
Tolerance: 1e-3 relative on volume fractions and interface position.
The measured errors are written to $CUPF_RECORD_DIR/split_precision_*.json when that
directory exists.
"""
import json
import os

import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.solver import APTSolver
from oracle import CpuOracle, interface_qois

pytestmark = pytest.mark.gpu

NSTEPS = 1000
TOL = 1e-3


def grain_volumes(p, ph, ids):
    """argmax grain map of a reference-layout state -> voxel counts per id."""
    o = CpuOracle()
    phi, alpha = o.collect(p, ph, ids)
    a = alpha.reshape(p.fnz, p.fny, p.fnx)[1:-1, 1:-1, 1:-1]
    return np.bincount(a[a > 0].ravel(), minlength=p.num_theta + 1)[1:]


@pytest.fixture(scope="module")
def fp64_reference():
    c = cases.line_case(64, 64, 64, num_pf=5, num_grains=20, seed=0, bc="110")
    ph0, id0 = c.initial_slots()
    o = CpuOracle()
    ph, ids = o.run_f64(c, ph0.astype(np.float64), id0, NSTEPS)
    return c, ph0, id0, grain_volumes(c.params, ph, ids), interface_qois(c.params, ph)


@pytest.mark.parametrize("prec", ["fp32", "fp16", "bf16"])
def test_split_precision_error(built, fp64_reference, prec):
    c, ph0, id0, v64, q64 = fp64_reference
    with APTSolver(c, precision=prec) as s:
        s.set_slots(ph0, id0, 0)
        s.step(NSTEPS)
        ph, ids = s.get_slots()
        qs = s.qoi_sums()
    v = grain_volumes(c.params, ph.astype(np.float32), ids)
    vol_err = float(np.abs(v - v64).sum() / v64.sum())
    pos_err = abs(qs[2] - q64[2]) / q64[2]
    area_err = abs(qs[1] - q64[1]) / q64[1]
    rec = {"precision": prec, "steps": NSTEPS, "volume_fraction_l1_rel_err": vol_err,
           "interface_height_rel_err": pos_err, "interface_area_rel_err": area_err,
           "interface_height_cells": qs[2], "interface_height_fp64": q64[2]}
    out = os.environ.get("CUPF_RECORD_DIR", "")
    if os.path.isdir(out):
        with open(os.path.join(out, "split_precision_%s.json" % prec), "w") as f:
            json.dump(rec, f)
    print(rec)
    if prec in ("fp32", "fp16"):
        assert vol_err <= TOL and pos_err <= TOL, rec
    else:
        assert np.isfinite(vol_err) and np.isfinite(pos_err)
