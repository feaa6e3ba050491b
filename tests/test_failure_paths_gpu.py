"""Failure paths of the step on a B200, made to happen without a GPU fault:

* the step kernel's bounded wait for its plane loads (TMA completion on an
  mbarrier) runs out: with a bound of one SM cycle the first wait of every
  work item gives up before its load lands.  The kernel then stops loading,
  waits with the default bound for the loads in flight, records its error word
  and finishes; the host reports CUPF_ERR_TIMEOUT, and after a new initial
  state the next steps are exact again;
* the host-side watchdog of cupf_apt_sync: a deadline shorter than the queued
  work returns CUPF_ERR_TIMEOUT without touching the device, and a later wait
  without deadline completes normally.
"""
import numpy as np
import pytest

from cupf_b200 import abi, cases
from cupf_b200.solver import APTSolver

pytestmark = pytest.mark.gpu

TIMEOUT = 5  # CUPF_ERR_TIMEOUT


def test_step_wait_bound_runs_out_then_recovers(built):
    c = cases.line_case(48, 40, 56, num_pf=5, num_grains=20, seed=2, bc="110")
    with APTSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.set_wait_limit(1)
        s.step(3)
        with pytest.raises(abi.CupfError) as e:
            s.sync()
        assert e.value.status == TIMEOUT
        # the error stays reported until a new state is loaded
        with pytest.raises(abi.CupfError):
            s.sync()
        s.set_wait_limit(0)
        s.init_from_argmax(c.phi, c.alpha)
        s.step(12)
        s.sync()
        ph, ids = s.get_slots()
    with APTSolver(c) as s2:
        s2.init_from_argmax(c.phi, c.alpha)
        s2.step(12)
        ph2, ids2 = s2.get_slots()
    assert np.array_equal(ids, ids2)
    assert np.array_equal(ph.view(np.int32), ph2.view(np.int32))


def test_sync_deadline_then_completion(built):
    c = cases.line_case(128, 128, 256, num_pf=8, num_grains=150, seed=0, bc="110")
    with APTSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.set_skip_quiet(False)
        s.sync()
        s.step(3000)  # far more than a millisecond of queued work
        with pytest.raises(abi.CupfError) as e:
            s.sync(1)
        assert e.value.status == TIMEOUT
        s.sync(0)
        assert s.steps_done() == 3000
        q = s.qoi_sums()
        assert np.isfinite(q).all() and q[0] > 0
