"""Pin the CPU oracle against the reference kernels' own outputs.

tests/golden/*.npz hold states produced by the reference kernels compiled for
sm_100a (tests/golden/make_golden.py, run on a B200).  The oracle's single
precision mode must reproduce every saved step bit for bit, from one saved step
to the next and over the whole saved horizon, and its argmax, tip scan and
moving-frame shift must reproduce the reference's.
"""
import ast
import glob
import os

import numpy as np
import pytest

from cupf_b200 import cases
from oracle import CpuOracle
from tests.helpers import compare_states, face_mask

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load(path):
    d = np.load(path)
    meta = ast.literal_eval(str(d["meta"]))
    build = {3: cases.cone_case, 4: cases.paraboloid_case}.get(meta["thermal"], cases.line_case)
    c = build(*meta["interior"], num_pf=meta["num_pf"], num_grains=meta["grains"],
              seed=meta["seed"], bc=meta["bc"])
    if meta["thermal"] == 2:
        c.params.thermalType = 2
        c.params.r0 = np.float32(meta["r0"])
        c.params.G = np.float32(meta["G"])
    return d, meta, c


def tstep(p, n):
    return float(np.float32(np.float32(n) * np.float32(p.dt)) * np.float32(p.tau0))


@pytest.fixture(scope="module")
def oracle():
    return CpuOracle()


def test_golden_files_present():
    assert len(GOLDEN) >= 4, "golden fixtures missing"


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_initial_state_reproduced(path):
    d, meta, c = load(path)
    ph0, id0 = c.initial_slots()
    assert np.array_equal(ph0.view(np.int32), d["ph_0"].view(np.int32))
    assert np.array_equal(id0, d["id_0"])


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_single_steps_bit_exact(oracle, path):
    d, meta, c = load(path)
    p = c.params
    saves = meta["saves"]
    if not any(n + 1 in saves for n in saves):
        pytest.skip("fixture holds no consecutive steps")
    checked = 0
    for n in saves:
        if n + 1 not in saves:
            continue
        ph, ids = d["ph_%d" % n].copy(), d["id_%d" % n].copy()
        # the output buffer before the step: what the reference's skipped cells keep
        # (thermalType 3 / 4 leave cells outside the heat source unwritten)
        if n > 0 and "bph_%d" % n in d.files:
            out0 = d["bph_%d" % n].copy(), d["bid_%d" % n].copy()
        else:
            out0 = ph.copy(), ids.copy()
        out_ph, out_id = oracle.rhs_psi_f32(c, tstep(p, n + 1), ph, ids, *out0, use_iuc=meta["iuc"])
        oracle.set_bc(p, out_ph, out_id)
        n_id, n_ph, dmax = compare_states(p, out_ph, out_id, d["ph_%d" % (n + 1)],
                                          d["id_%d" % (n + 1)])
        assert (n_id, n_ph) == (0, 0), (n, n_id, n_ph, dmax)
        checked += 1
    assert checked >= 1


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_trajectory_bit_exact(oracle, path):
    d, meta, c = load(path)
    p = c.params
    last = max(meta["saves"])
    ph, ids, _, _ = oracle.run_f32(c, d["ph_0"], d["id_0"], last, use_iuc=meta["iuc"])
    n_id, n_ph, dmax = compare_states(p, ph, ids, d["ph_%d" % last], d["id_%d" % last])
    assert (n_id, n_ph) == (0, 0), (n_id, n_ph, dmax)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_collect_tip_and_shift(oracle, path):
    d, meta, c = load(path)
    p = c.params
    last = max(meta["saves"])
    ph, ids = d["ph_%d" % last].copy(), d["id_%d" % last].copy()
    phi, alpha = oracle.collect(p, ph, ids)
    m = face_mask(p)
    assert np.array_equal(alpha[m], d["collect_alpha"][m])
    assert np.array_equal(phi[m].view(np.int32), d["collect_phi"][m].view(np.int32))
    tip, meanx = oracle.tip_scan(p, ph, 1)
    assert tip == int(d["tip"][0])
    # the reference sums each layer (fnx*fny*NUM_PF floats) with float atomics in
    # an unspecified order; the oracle sums in double: agree to float accumulation
    # error (~n*eps), the tip layer itself must be identical
    np.testing.assert_allclose(meanx, d["meanx"], rtol=2e-4)
    fnz_f = p.fnz + 4
    afull = np.zeros(p.fnx * p.fny * fnz_f, np.int32)
    loss = np.zeros(p.num_theta, np.int32)
    z = c.z.copy()
    oracle.move_frame(p, ph, ids, z, d["collect_alpha"].copy(), afull, loss, 1)
    assert np.array_equal(z, d["move_z"])
    assert np.array_equal(loss, d["move_loss"])
    assert np.array_equal(afull, d["move_afull"])
    # the shift touches interior cells only; compare those
    from tests.helpers import interior_mask
    n_id, n_ph, _ = compare_states(p, ph, ids, d["move_ph"], d["move_id"], interior_mask(p))
    assert (n_id, n_ph) == (0, 0)
