"""Continuous-batching server: each result is the same alone and in the mix.

The server advances every resident simulation in one persistent batched kernel
per step (replayed from a CUDA graph).  A request's argmax map, grain volumes and
FP64 interface sums must be bit-identical whether it runs alone, batched with
requests of other grid shapes, admitted late under a tight memory budget, or
through the single-simulation handle; and every request must stop at exactly
its own step target.
"""
import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.server import DONE, Server
from cupf_b200.solver import APTSolver

pytestmark = pytest.mark.gpu


def req(shape, grains, seed, np_=8, G=1.0, R=0.05, bc="110"):
    return cases.line_case(*shape, num_pf=np_, num_grains=grains, seed=seed, G=G, R=R, bc=bc)


A = dict(shape=(48, 48, 48), grains=12, seed=1)
B = dict(shape=(96, 64, 80), grains=40, seed=2, G=3.0, R=0.2)
C = dict(shape=(40, 72, 56), grains=25, seed=3, G=0.5, R=0.01, bc="000")


def single(case, nsteps, precision="fp32"):
    with APTSolver(case, precision=precision) as s:
        s.init_from_argmax(case.phi, case.alpha)
        s.step(nsteps)
        _, alpha = s.collect(clear=True)
        vols = s.grain_volumes(case.params.num_theta)
        q = s.qoi_sums()
    return alpha, vols, q


def same(r1, r2):
    assert np.array_equal(r1["alpha"], r2["alpha"])
    assert np.array_equal(r1["volumes"], r2["volumes"])
    assert r1["qoi"] == r2["qoi"]


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_alone_equals_mixed_equals_single(built, precision):
    ca = req(**A)
    with Server(precision=precision, steps_per_round=16, autotune=False) as srv:
        ra = srv.submit(ca, 90)
        srv.run_until_done([ra])
        alone = srv.result(ra)
    with Server(precision=precision, steps_per_round=16, autotune=True) as srv:
        rb = srv.submit(req(**B), 70)
        srv.pump()  # B resident first, A and C join later (continuous batching)
        ra = srv.submit(ca, 90)
        rc = srv.submit(req(**C), 130)
        srv.run_until_done([ra, rb, rc])
        mixed = srv.result(ra)
        assert srv.result(rb) is not None and srv.result(rc) is not None
    same(alone, mixed)
    alpha, vols, q = single(ca, 90, precision)
    assert np.array_equal(alone["alpha"], alpha)
    assert np.array_equal(alone["volumes"], vols)
    assert alone["qoi"] == q


def test_memory_budget_serialises_admission(built):
    ca, cb = req(**A), req(**B)
    # room for one request at a time: B waits until A retires
    with Server(steps_per_round=8, autotune=False, hbm_budget_bytes=80 << 20) as srv:
        ra = srv.submit(ca, 33)
        rb = srv.submit(cb, 21)
        running, pending, _ = srv.pump()
        assert running == 1 and pending == 1
        srv.run_until_done([ra, rb])
        res_a, res_b = srv.result(ra), srv.result(rb)
        assert res_a["times"][2] <= res_b["times"][1] + 1e-3  # B admitted after A finished
    alpha, vols, q = single(cb, 21)
    assert np.array_equal(res_b["alpha"], alpha) and res_b["qoi"] == q


def test_exact_step_targets(built):
    """Targets that are not multiples of the round length stop exactly."""
    ca = req(**A)
    outs = {}
    with Server(steps_per_round=10, autotune=False) as srv:
        ids = {n: srv.submit(ca, n) for n in (1, 7, 10, 23)}
        srv.run_until_done(list(ids.values()))
        for n, rid in ids.items():
            outs[n] = srv.result(rid)
            assert srv.status(rid) == DONE
    for n, r in outs.items():
        alpha, vols, q = single(ca, n)
        assert r["qoi"] == q, n
        assert np.array_equal(r["alpha"], alpha), n


def test_pool_reuse_across_bursts(built):
    """Retired requests' device memory goes back to the server's pool and serves
    the next admissions: a second burst of the same requests (in the other order)
    gives the same results without the server holding more memory, and destroying
    the server returns what the pool held."""
    import torch
    torch.cuda.init()
    free0, _ = torch.cuda.mem_get_info()
    ca, cb = req(**A), req(**B)
    with Server(precision="fp32", steps_per_round=16, autotune=False) as srv:
        r1 = [srv.submit(ca, 40), srv.submit(cb, 30)]
        srv.run_until_done(r1)
        first = [srv.result(r) for r in r1]
        for r in r1:
            srv.release(r)
        free1, _ = torch.cuda.mem_get_info()
        r2 = [srv.submit(cb, 30), srv.submit(ca, 40)]
        srv.run_until_done(r2)
        second = [srv.result(r) for r in r2]
        free2, _ = torch.cuda.mem_get_info()
    free3, _ = torch.cuda.mem_get_info()
    same(first[0], second[1])
    same(first[1], second[0])
    assert free1 < free0  # the pool kept the retired requests' memory
    assert abs(free2 - free1) <= 32 << 20, (free1, free2)
    assert free3 >= free0 - (64 << 20), (free0, free3)
