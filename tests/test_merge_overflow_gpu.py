"""Hazard H1 of the reference's merge (APTPhaseField.cu:222-231): when a 7-point
stencil holds more than NUM_PF distinct grain ids, the reference writes
local_phs[s][NUM_PF], which aliases the next point's slot 0 for s < 6 and lands
past the array at the last point.  The library reproduces the aliasing, drops
the last point's extra entries, and counts both (cupf_apt_merge_overflows); the
oracle counts the same entries.  On few-slot cases with many grains the counts
and the states must agree exactly."""
import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.solver import APTSolver
from tests.helpers import compare_states

pytestmark = pytest.mark.gpu

CASES = [((32, 28, 24), 1, 12, 1), ((40, 36, 32), 2, 40, 2), ((36, 30, 40), 3, 60, 3),
         ((48, 40, 32), 4, 120, 4)]


@pytest.mark.parametrize("spec", CASES, ids=lambda s: "np%d_%dgrains" % (s[1], s[2]))
def test_overflow_counts_and_states_match_oracle(built, spec):
    from oracle import CpuOracle
    interior, npf, grains, seed = spec
    c = cases.line_case(*interior, num_pf=npf, num_grains=grains, seed=seed, bc="110")
    ph0, id0 = c.initial_slots()
    steps = 25
    stats = np.zeros(2, np.int64)
    o_ph, o_id, _, _ = CpuOracle().run_f32(c, ph0, id0, steps, stats=stats)
    with APTSolver(c) as s:
        s.set_slots(ph0, id0, 0)
        s.merge_overflows()  # reset
        s.step(steps)
        aliased, dropped = s.merge_overflows()
        ph, ids = s.get_slots()
    assert aliased + dropped > 0, "case produced no merge overflow"
    assert (aliased, dropped) == (int(stats[0]), int(stats[1]))
    n_id, n_ph, d = compare_states(c.params, ph, ids, o_ph, o_id)
    assert (n_id, n_ph) == (0, 0), (n_id, n_ph, d)
