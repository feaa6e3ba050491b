"""The allocation-free grain-volume entry point (cupf_grain_volumes_noalloc).

For callers that cannot let a library allocate device memory (codes that give
all device memory to their own pool allocator, services whose device footprint
must stay fixed): the caller passes the argmax map already on the device, and
the reduction's scratch is a fixed device array inside the library.  Its counts
must equal those of the allocating entry point (cupf_apt_grain_volumes) exactly
(integer counts), on two calls in a row (the shared scratch keeps the previous
call's contents and must be cleared), and sizes beyond its fixed maximum must be
rejected.  Collected last so that a failure here leaves the rest of a
stop-at-first-failure run intact.
"""
import ctypes as C

import numpy as np
import pytest

from cupf_b200 import abi, cases
from cupf_b200.solver import APTSolver

pytestmark = pytest.mark.gpu


def test_noalloc_volumes_equal_allocating_entry_point(built):
    import torch
    torch.cuda.set_device(0)
    c = cases.line_case(48, 40, 56, num_pf=6, num_grains=30, seed=12, bc="110")
    p = c.params
    with APTSolver(c) as s:
        s.init_from_argmax(c.phi, c.alpha)
        s.step(30)
        _, alpha = s.collect(clear=True)
        expected = s.grain_volumes(p.num_theta)
    assert expected[1:].sum() > 0
    # independent count on the host: ids 1..num_grains over the interior, the
    # rest in counts[0]
    a = alpha.reshape(p.fnz, p.fny, p.fnx)[1:-1, 1:-1, 1:-1].ravel()
    ok = (a >= 1) & (a <= p.num_theta)
    host = np.bincount(a[ok], minlength=p.num_theta + 1).astype(np.int64)
    host[0] = int(np.count_nonzero(~ok))
    assert np.array_equal(expected, host)
    d_alpha = torch.from_numpy(np.ascontiguousarray(alpha)).cuda()
    torch.cuda.synchronize()
    L = abi.lib()
    free = []
    for call in range(2):
        counts = np.full(p.num_theta + 1, -7, np.int64)
        abi.check(L.cupf_grain_volumes_noalloc(C.c_void_p(d_alpha.data_ptr()), p.fnx, p.fny,
                                               p.fnz, p.num_theta,
                                               counts.ctypes.data_as(C.POINTER(C.c_int64)), None))
        free.append(torch.cuda.mem_get_info()[0])
        assert np.array_equal(counts, expected), "call %d" % call
    # the second call allocates nothing: free device memory is unchanged
    assert free[0] == free[1], free
    # beyond the fixed scratch: rejected with a clear error, nothing launched
    counts = np.zeros(2, np.int64)
    st = L.cupf_grain_volumes_noalloc(C.c_void_p(d_alpha.data_ptr()), p.fnx, p.fny, p.fnz,
                                      65536, counts.ctypes.data_as(C.POINTER(C.c_int64)), None)
    assert st == 1 and b"65535" in L.cupf_last_error()
