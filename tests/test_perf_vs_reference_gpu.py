"""Device time of the reference step (APTsetBC3D + APTrhs_psi as its evolve loop
launches them, compiled for sm_100a) against the library's fused step, on the
C2 throughput configuration (256x256x512 interior, 600 grains, NUM_PF=8).
Records both in perf_vs_reference.json (in $CUPF_RECORD_DIR) and checks that the library
is faster.
"""
import json
import os

import numpy as np
import pytest

from cupf_b200 import cases
from cupf_b200.solver import APTSolver

pytestmark = pytest.mark.gpu

STEPS = 40


def test_step_faster_than_reference_c2(built):
    import ctypes as C

    import torch
    from oracle import RefGPU
    c = cases.line_case(256, 256, 512, num_pf=8, num_grains=600, seed=0, bc="110")
    p = c.params
    cells = (p.fnx - 2) * (p.fny - 2) * (p.fnz - 2)
    ph0, id0 = c.initial_slots()
    ref = RefGPU(8)
    ref.check(ref.L.ref_set_params(p))
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    x, y, z, sint, cost = (dev(a) for a in (c.x, c.y, c.z, c.sint, c.cost))
    a_ph, a_id, b_ph, b_id = dev(ph0), dev(id0), dev(ph0), dev(id0)
    ms = C.c_float()
    args = [x.data_ptr(), y.data_ptr(), z.data_ptr(), a_ph.data_ptr(), b_ph.data_ptr(),
            a_id.data_ptr(), b_id.data_ptr(), sint.data_ptr(), cost.data_ptr()]
    ref.check(ref.L.ref_run_steps(4, 0, *args, C.byref(ms)))  # warm-up (even count)
    ref.check(ref.L.ref_run_steps(STEPS, 4, *args, C.byref(ms)))
    ref_ms = ms.value / STEPS
    del a_ph, a_id, b_ph, b_id
    torch.cuda.empty_cache()
    with APTSolver(c) as s:
        s.set_slots(ph0, id0, 0)
        s.step(4)
        my_ms = s.time_steps(STEPS) / STEPS
    rec = {"workload": "C2 256x256x512 NUM_PF=8 600 grains", "steps": STEPS,
           "reference_ms_per_step": ref_ms, "cupf_ms_per_step": my_ms,
           "reference_mcell_per_s": cells / ref_ms / 1e3, "cupf_mcell_per_s": cells / my_ms / 1e3,
           "speedup": ref_ms / my_ms}
    out = os.environ.get("CUPF_RECORD_DIR", "")
    if os.path.isdir(out):
        with open(os.path.join(out, "perf_vs_reference.json"), "w") as f:
            json.dump(rec, f, indent=1)
    print(rec)
    assert my_ms < ref_ms, rec
