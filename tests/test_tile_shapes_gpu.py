"""Column-tile heights of the step (32x8, the default, and 32x4; the server's
autotuner picks one per grid shape with the z chunk): results are identical
bit for bit whichever tile shape steps a simulation.

* single handle, 32x4 against 32x8: partial tiles in y, every boundary code,
  FP32, FP16 and BF16 (the 16-bit 32x8 kernel decodes each centre plane once,
  the 32x4 one per use), merge overflows, z chunks of 1 to 16, quiet items on;
* 32x4 against the reference kernels on a parity case;
* the server with every request on 32x4, on 32x8, and with the two mixed in one
  round (one batched launch per tile height), against the single handle.
"""
import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.server import Server
from cupf_b200.solver import APTSolver

pytestmark = pytest.mark.gpu

CASES = [
    # interior, num_pf, grains, seed, bc, steps, zc, precision
    ((37, 21, 29), 4, 15, 4, "101", 25, 2, "fp32"),
    ((70, 9, 40), 6, 30, 5, "010", 20, 1, "fp32"),
    ((33, 30, 17), 3, 8, 6, "111", 30, 4, "fp32"),
    ((40, 42, 48), 8, 90, 7, "110", 60, 16, "fp32"),
    ((24, 26, 40), 8, 60, 1, "000", 30, 8, "fp16"),
    ((48, 44, 56), 8, 70, 3, "110", 80, 4, "bf16"),
    # few slots, many grains: merge overflows, whose aliased values the 16-bit
    # 32x8 kernel reads through its decoded centre plane and the 32x4 one per use
    ((36, 30, 40), 3, 60, 3, "110", 25, 4, "fp16"),
    ((48, 40, 32), 4, 120, 4, "011", 25, 2, "bf16"),
]


def run(c, steps, ty, zc, precision):
    with APTSolver(c, precision=precision) as s:
        s.set_tile(ty)
        s.set_tuning(zc)
        s.init_from_argmax(c.phi, c.alpha)
        s.step(steps)
        return s.get_slots()


@pytest.mark.parametrize("spec", CASES, ids=lambda s: "%dx%dx%d_np%d_%s_%s" % (*s[0], s[1], s[4], s[7]))
def test_tile4_equals_tile8(built, spec):
    interior, npf, grains, seed, bc, steps, zc, precision = spec
    c = cases.line_case(*interior, num_pf=npf, num_grains=grains, seed=seed, bc=bc)
    ph8, id8 = run(c, steps, 8, zc, precision)
    ph4, id4 = run(c, steps, 4, zc, precision)
    assert np.array_equal(id4, id8)
    assert np.array_equal(ph4.view(np.uint32), ph8.view(np.uint32))


def test_tile4_bit_exact_vs_reference(built):
    from tests.helpers import compare_states, run_reference_gpu
    c = cases.line_case(40, 27, 36, num_pf=8, num_grains=40, seed=21, bc="110")
    ref_ph, ref_id = run_reference_gpu(c, 40)
    ph0, id0 = c.initial_slots()
    with APTSolver(c) as s:
        s.set_tile(4)
        s.set_slots(ph0, id0, 0)
        s.step(40)
        my_ph, my_id = s.get_slots()
    n_id, n_ph, d = compare_states(c.params, my_ph, my_id, ref_ph, ref_id)
    assert (n_id, n_ph) == (0, 0), (n_id, n_ph, d)


def test_server_tile_heights(built):
    reqs = [cases.line_case(48, 44, 40, num_pf=8, num_grains=20, seed=1),
            cases.line_case(64, 36, 56, num_pf=8, num_grains=30, seed=2, G=3.0, R=0.2)]
    steps = [60, 45]
    out = {}
    for ty in (8, 4):
        with Server(steps_per_round=16, autotune=False, tile_y=ty) as srv:
            ids = [srv.submit(c, n) for c, n in zip(reqs, steps)]
            srv.run_until_done(ids)
            out[ty] = [srv.result(i) for i in ids]
    for a, b in zip(out[8], out[4]):
        assert np.array_equal(a["alpha"], b["alpha"]) and a["qoi"] == b["qoi"]
    # the autotuner's picks, whatever they are, give the same results
    with Server(steps_per_round=16, autotune=True) as srv:
        ids = [srv.submit(c, n) for c, n in zip(reqs, steps)]
        srv.run_until_done(ids)
        auto = [srv.result(i) for i in ids]
    for a, b in zip(out[8], auto):
        assert np.array_equal(a["alpha"], b["alpha"]) and a["qoi"] == b["qoi"]
    for c, n, r in zip(reqs, steps, out[8]):
        with APTSolver(c) as s:
            s.init_from_argmax(c.phi, c.alpha)
            s.step(n)
            _, alpha = s.collect(clear=True)
        assert np.array_equal(r["alpha"], alpha)


def test_server_mixed_tile_heights_in_one_round(built):
    """Requests of both tile heights resident together: the round runs one
    batched launch per height; each result equals the same request alone."""
    c8 = cases.line_case(48, 40, 44, num_pf=8, num_grains=20, seed=5)
    c4 = cases.line_case(36, 52, 40, num_pf=8, num_grains=25, seed=6)
    with Server(steps_per_round=8, autotune=False, tile_y=4) as srv:
        r4 = srv.submit(c4, 50)
        srv.run_until_done([r4])
        alone4 = srv.result(r4)
    with Server(steps_per_round=8, autotune=False, tile_y=8) as srv:
        r8 = srv.submit(c8, 50)
        srv.run_until_done([r8])
        alone8 = srv.result(r8)
    srv = Server(steps_per_round=8, autotune=False, tile_y=8)
    try:
        r8 = srv.submit(c8, 50)
        srv.pump()
        # switch the tile height for requests admitted from now on
        srv.set_tile_height(4)
        r4 = srv.submit(c4, 50)
        srv.run_until_done([r8, r4])
        assert srv.tile_height(r8) == 8 and srv.tile_height(r4) == 4
        m8, m4 = srv.result(r8), srv.result(r4)
    finally:
        srv.close()
    assert np.array_equal(m8["alpha"], alone8["alpha"]) and m8["qoi"] == alone8["qoi"]
    assert np.array_equal(m4["alpha"], alone4["alpha"]) and m4["qoi"] == alone4["qoi"]
