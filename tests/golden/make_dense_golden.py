"""Generate the golden fixtures of the reference's full-PF kernels (needs a B200).

Runs the reference's own PhaseField.cu kernels (oracle/_ref/libref_dense.so:
set_minus1, ini_PF, set_BC_3D, rhs_psi, collect_PF, compiled unmodified for
sm_100a by oracle/build.py) on seeded synthetic line cases, as
PhaseField::evolve issues them (PhaseField.cu:545-566): initial state, the
pre-loop update at t = 0, then set_BC_3D + rhs_psi steps.  Saves selected states
(halo filled) and the argmax map after the last one as compressed .npz files; the
CPU tests pin the oracle's full-PF restatement against them bit for bit.

Usage:  python tests/golden/make_dense_golden.py [OUT_DIR]   (default tests/golden/dense)
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

from cupf_b200 import cases  # noqa: E402
from oracle import RefDenseGPU  # noqa: E402

CASES = {
    # name: (interior, grains, seed, states saved after n updates (0 = initial, 1 = pre-loop))
    "d1_g8": ((24, 24, 32), 8, 0, [0, 1, 2, 30, 31]),
    "d2_g12": ((20, 28, 24), 12, 5, [0, 1, 20, 21]),
}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_case(name, spec, out_dir):
    interior, grains, seed, saves = spec
    c = cases.line_case(*interior, num_pf=5, num_grains=grains, seed=seed, bc="110")
    p = c.params
    R = float(c.meta["R"])
    ref = RefDenseGPU()
    ref.check(ref.L.refd_set_params(p, R))
    L = p.fnx * p.fny * p.fnz
    n = L * p.num_theta
    a = torch.empty(n, dtype=torch.float32, device="cuda")
    b = torch.empty(n, dtype=torch.float32, device="cuda")
    phi, alpha = dev(np.asarray(c.phi, np.float32)), dev(np.asarray(c.alpha, np.int32))
    x, y, z = (dev(np.asarray(v, np.float32)) for v in (c.x, c.y, c.z))
    sint, cost = dev(np.asarray(c.sint, np.float32)), dev(np.asarray(c.cost, np.float32))
    for t_ in (a, b):
        ref.check(ref.L.refd_set_minus1(t_.data_ptr(), n))
    for t_ in (a, b):
        ref.check(ref.L.refd_ini(t_.data_ptr(), phi.data_ptr(), alpha.data_ptr()))
    ref.check(ref.L.refd_set_minus1(phi.data_ptr(), L))
    for t_ in (b, a):
        ref.check(ref.L.refd_set_bc(t_.data_ptr()))
    rec = {}
    if 0 in saves:
        rec["ph_0"] = a.cpu().numpy()
    ref.check(ref.L.refd_rhs_psi(0.0, x.data_ptr(), y.data_ptr(), z.data_ptr(), a.data_ptr(),
                                 b.data_ptr(), sint.data_ptr(), cost.data_ptr()))
    cur, oth = b, a
    ref.check(ref.L.refd_set_bc(cur.data_ptr()))
    if 1 in saves:
        rec["ph_1"] = cur.cpu().numpy()
    ms = C.c_float()
    for k in range(2, max(saves) + 1):
        # update k is loop step k-1 (t = (k-1)*dt*tau0)
        ref.check(ref.L.refd_run_steps(1, k - 2, x.data_ptr(), y.data_ptr(), z.data_ptr(),
                                       cur.data_ptr(), oth.data_ptr(), sint.data_ptr(),
                                       cost.data_ptr(), C.byref(ms)))
        cur, oth = oth, cur
        ref.check(ref.L.refd_set_bc(cur.data_ptr()))
        if k in saves:
            ref.check(ref.L.refd_sync())
            rec["ph_%d" % k] = cur.cpu().numpy()
    am = torch.zeros(L, dtype=torch.int32, device="cuda")
    alpha.zero_()
    ref.check(ref.L.refd_collect(cur.data_ptr(), phi.data_ptr(), alpha.data_ptr(), am.data_ptr()))
    ref.check(ref.L.refd_sync())
    rec["phi_last"], rec["alpha_last"], rec["argmax_last"] = (
        phi.cpu().numpy(), alpha.cpu().numpy(), am.cpu().numpy())
    meta = {"interior": interior, "grains": grains, "seed": seed, "R": R, "saves": saves}
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), meta=repr(meta), **rec)
    print(name, sorted(rec))


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                            "dense")
    os.makedirs(out, exist_ok=True)
    for name, spec in CASES.items():
        run_case(name, spec, out)


if __name__ == "__main__":
    main()
