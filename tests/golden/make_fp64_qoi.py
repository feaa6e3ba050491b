"""Generate the FP64 QoIs that split-precision and served results are measured
against (CPU only; the oracle's FP64 transcription of the reference step).

Writes tests/golden/fp64/qoi.npz with, for each case, the per-grain voxel
counts of the argmax map after the case's steps (interior cells, ids 1..NG) and
the FP64 (solid volume, interface area, mean interface height), and the same
two of the oracle's FP32 restatement (the reference's own precision, keys
*_f32_*), so that a result's error can be read beside the error single
precision itself makes on the same case:

  c1_*        the 64^3 line case (20 grains, seed 0, NUM_PF = 5), 1000 steps
  srv<i>_*    request i of the served stream poisson_stream(40, seed=0) for every
              request with a 48^3 grid (NUM_PF = 8), 1000 steps each

Usage:  python tests/golden/make_fp64_qoi.py [OUT]
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cupf_b200 import cases  # noqa: E402
from cupf_b200.server import poisson_stream  # noqa: E402
from oracle import CpuOracle, interface_qois  # noqa: E402

STEPS = 1000
SERVED_REQUESTS = 40
SMALL_GRID = (48, 48, 48)


def qois_of(p, o, ph, ids):
    _, alpha = o.collect(p, ph, ids)
    a = alpha.reshape(p.fnz, p.fny, p.fnx)[1:-1, 1:-1, 1:-1]
    vols = np.bincount(a[a > 0].ravel(), minlength=p.num_theta + 1)[1:].astype(np.int64)
    return vols, np.array(interface_qois(p, ph), np.float64)


def fp64_qois(case, nsteps):
    """(volumes, qoi) of the FP64 oracle and of the FP32 oracle after nsteps."""
    o = CpuOracle()
    ph0, id0 = case.initial_slots()
    ph, ids = o.run_f64(case, ph0.astype(np.float64), id0, nsteps)
    r64 = qois_of(case.params, o, ph, ids)
    ph, ids, _, _ = o.run_f32(case, ph0, id0, nsteps)
    r32 = qois_of(case.params, o, ph, ids)
    return r64, r32


def main(out):
    rec = {"steps": np.int64(STEPS)}
    t0 = time.time()
    c1 = cases.line_case(64, 64, 64, num_pf=5, num_grains=20, seed=0, bc="110")
    (rec["c1_volumes"], rec["c1_qoi"]), (rec["c1_f32_volumes"], rec["c1_f32_qoi"]) = \
        fp64_qois(c1, STEPS)
    print("c1 done %.1f s" % (time.time() - t0), flush=True)
    idx = []
    for i, (_, c) in enumerate(poisson_stream(SERVED_REQUESTS, seed=0)):
        if c.meta["interior"] != SMALL_GRID:
            continue
        (rec["srv%d_volumes" % i], rec["srv%d_qoi" % i]), \
            (rec["srv%d_f32_volumes" % i], rec["srv%d_f32_qoi" % i]) = fp64_qois(c, STEPS)
        idx.append(i)
        print("request %d done %.1f s" % (i, time.time() - t0), flush=True)
    rec["served_index"] = np.array(idx, np.int64)
    np.savez_compressed(out, **rec)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "fp64", "qoi.npz"))
