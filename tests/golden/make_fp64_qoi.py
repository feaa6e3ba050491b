"""Generate the FP64 QoIs that split-precision and served results are measured
against (CPU only; the oracle's FP64 transcription of the reference step).

Writes tests/golden/fp64/qoi.npz with, for each case, the per-grain voxel
counts of the argmax map after the case's steps (interior cells, ids 1..NG) and
the FP64 (solid volume, interface area, mean interface height), and the same
two of the oracle's FP32 restatement (the reference's own precision, keys
*_f32_*) and of the FP64 oracle started from the initial state with one
single-precision rounding step of noise on it (keys *_p64_*: every occupied
interface slot of a seeded half of the cells moved by one float ulp up or down),
so that a result's error can be read beside the error single precision itself
makes on the same case and beside how far the case's own dynamics carry a
perturbation of that size:

  c1_*        the 64^3 line case (20 grains, seed 0, NUM_PF = 5), 1000 steps
  srv<i>_*    request i of the served stream poisson_stream(40, seed=0) for every
              request with a 48^3 or 96^3 grid (NUM_PF = 8), 1000 steps each (the
              oracle's cost, about 4 minutes of 8 cores per 96^3 request and several
              times that per larger one, bounds the rest)

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
SMALL_GRIDS = ((48, 48, 48), (96, 96, 96))


def qois_of(p, o, ph, ids):
    _, alpha = o.collect(p, ph, ids)
    a = alpha.reshape(p.fnz, p.fny, p.fnx)[1:-1, 1:-1, 1:-1]
    vols = np.bincount(a[a > 0].ravel(), minlength=p.num_theta + 1)[1:].astype(np.int64)
    return vols, np.array(interface_qois(p, ph), np.float64)


def ulp_perturbed(ph0, id0, seed):
    """The initial slot phi with every occupied slot of a seeded half of the
    cells whose phi lies strictly inside (-1, 1) moved by one float ulp, up or
    down at random."""
    rng = np.random.default_rng(seed)
    move = (id0 >= 0) & (np.abs(ph0) < 1) & (rng.random(ph0.shape) < 0.5)
    up = rng.random(ph0.shape) < 0.5
    out = ph0.copy()
    out[move & up] = np.nextafter(ph0[move & up], np.float32(2))
    out[move & ~up] = np.nextafter(ph0[move & ~up], np.float32(-2))
    return out


def fp64_qois(case, nsteps):
    """(volumes, qoi) of the FP64 oracle, of the FP32 oracle and of the FP64
    oracle from the ulp-perturbed initial state after nsteps."""
    o = CpuOracle()
    ph0, id0 = case.initial_slots()
    ph, ids = o.run_f64(case, ph0.astype(np.float64), id0, nsteps)
    r64 = qois_of(case.params, o, ph, ids)
    ph, ids, _, _ = o.run_f32(case, ph0, id0, nsteps)
    r32 = qois_of(case.params, o, ph, ids)
    ph, ids = o.run_f64(case, ulp_perturbed(ph0, id0, 7).astype(np.float64), id0, nsteps)
    rp = qois_of(case.params, o, ph, ids)
    return r64, r32, rp


def main(out):
    rec = {"steps": np.int64(STEPS)}
    t0 = time.time()
    c1 = cases.line_case(64, 64, 64, num_pf=5, num_grains=20, seed=0, bc="110")
    (rec["c1_volumes"], rec["c1_qoi"]), (rec["c1_f32_volumes"], rec["c1_f32_qoi"]), \
        (rec["c1_p64_volumes"], rec["c1_p64_qoi"]) = fp64_qois(c1, STEPS)
    print("c1 done %.1f s" % (time.time() - t0), flush=True)
    idx = []
    for i, (_, c) in enumerate(poisson_stream(SERVED_REQUESTS, seed=0)):
        if tuple(c.meta["interior"]) not in SMALL_GRIDS:
            continue
        (rec["srv%d_volumes" % i], rec["srv%d_qoi" % i]), \
            (rec["srv%d_f32_volumes" % i], rec["srv%d_f32_qoi" % i]), \
            (rec["srv%d_p64_volumes" % i], rec["srv%d_p64_qoi" % i]) = fp64_qois(c, STEPS)
        idx.append(i)
        print("request %d done %.1f s" % (i, time.time() - t0), flush=True)
    rec["served_index"] = np.array(idx, np.int64)
    np.savez_compressed(out, **rec)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "fp64", "qoi.npz"))
