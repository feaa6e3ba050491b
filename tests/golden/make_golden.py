"""Generate the golden fixtures of the reference APT kernels (needs a B200).

Runs the reference's own kernels (oracle/_ref/libref_apt{5,8}.so: APTrhs_psi,
APTsetBC3D, APTcollect_PF, APTini_PF, APTmove_frame/APTcopy_frame and the tip
scan, compiled for sm_100a by oracle/build.py with the slot count set and
one padding row on the merge's local array) on seeded synthetic cases and writes
their states as compressed .npz files.  The CPU tests pin the oracle against
these files bit-for-bit.

Usage:  python tests/golden/make_golden.py OUT_DIR [CASE ...]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

from cupf_b200 import cases  # noqa: E402
from oracle import RefGPU  # noqa: E402

CASES = {
    # name: (interior, num_pf, grains, seed, bc, steps saved, options)
    "g1_np5_110": ((32, 32, 32), 5, 20, 0, "110", [0, 1, 2, 20, 21, 40], {}),
    "g2_np8_000": ((24, 24, 40), 8, 60, 1, "000", [0, 1, 30, 31], {}),
    "g3_np5_111_iuc": ((24, 24, 24), 5, 40, 2, "111", [0, 1, 10, 11], {"iuc": True}),
    "g4_np5_cyl": ((24, 24, 32), 5, 20, 3, "110", [0, 1, 12, 13], {"thermal": 2}),
    "c1_64_np5": ((64, 64, 64), 5, 20, 0, "110", [0, 200], {"final_only": True}),
    "g5_np5_cone": ((40, 24, 32), 5, 20, 10, "110", [0, 1, 12, 13], {"thermal": 3}),
    "g6_np8_parab": ((36, 28, 32), 8, 30, 11, "110", [0, 1, 12, 13], {"thermal": 4}),
}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t):
    return t.data_ptr() if t is not None else None


def run_case(name, spec, out_dir):
    interior, num_pf, grains, seed, bc, saves, opt = spec
    build = {3: cases.cone_case, 4: cases.paraboloid_case}.get(opt.get("thermal"), cases.line_case)
    c = build(*interior, num_pf=num_pf, num_grains=grains, seed=seed, bc=bc)
    p = c.params
    if opt.get("thermal") == 2:
        p.thermalType = 2
        p.r0 = np.float32(0.5) * p.lzd
        p.G = np.float32(0.5)
    iuc = bool(opt.get("iuc", False))
    ref = RefGPU(num_pf)
    ref.check(ref.L.ref_set_params(p))
    ph0, id0 = c.initial_slots()
    x, y, z, sint, cost = (dev(a) for a in (c.x, c.y, c.z, c.sint, c.cost))
    # macro tables of thermalType 4 (None: the harness passes a zeroed buffer)
    mac = [getattr(c, n, None) for n in ("X_mac", "Y_mac", "Z_mac", "t_mac", "psi_mac", "T_3D")]
    mac = [dev(np.asarray(m, np.float32)) if m is not None else None for m in mac]
    a_ph, a_id = dev(ph0), dev(id0)
    b_ph, b_id = dev(ph0), dev(id0)
    rec = {}
    if 0 in saves:
        rec["ph_0"], rec["id_0"] = ph0, id0
    nmax = max(saves)
    for n in range(1, nmax + 1):
        t = np.float32(np.float32(n) * np.float32(p.dt)) * np.float32(p.tau0)
        ref.check(ref.L.ref_set_bc(ptr(a_ph), ptr(a_id)))
        ref.check(ref.L.ref_rhs_psi(float(t), ptr(x), ptr(y), ptr(z), ptr(a_ph), ptr(b_ph),
                                    ptr(a_id), ptr(b_id), ptr(sint), ptr(cost),
                                    *(ptr(m) for m in mac), int(iuc)))
        a_ph, b_ph = b_ph, a_ph
        a_id, b_id = b_id, a_id
        if n in saves:
            # the state as the next step reads it: boundary-filled
            ref.check(ref.L.ref_set_bc(ptr(a_ph), ptr(a_id)))
            torch.cuda.synchronize()
            rec["ph_%d" % n] = a_ph.cpu().numpy()
            rec["id_%d" % n] = a_id.cpu().numpy()
            # the other buffer: its content is what skipped writes leave behind
            rec["bph_%d" % n] = b_ph.cpu().numpy()
            rec["bid_%d" % n] = b_id.cpu().numpy()
    # argmax of the last state, with and without a cleared output
    L = c.length
    phi = dev(np.zeros(L, np.float32))
    alpha = dev(np.zeros(L, np.int32))
    ref.check(ref.L.ref_collect(ptr(a_ph), ptr(phi), ptr(alpha), ptr(a_id)))
    torch.cuda.synchronize()
    rec["collect_phi"] = phi.cpu().numpy()
    rec["collect_alpha"] = alpha.cpu().numpy()
    # tip scan + one moving-frame shift of the last state
    meanx_d = dev(np.zeros(p.fnz, np.float32))
    meanx_h = np.zeros(p.fnz, np.float32)
    tip = np.array([1], np.int32)
    import ctypes as C
    ref.check(ref.L.ref_tip_mvf(tip.ctypes.data_as(C.POINTER(C.c_int32)), ptr(a_ph), ptr(meanx_d),
                                meanx_h.ctypes.data_as(C.POINTER(C.c_float))))
    rec["tip"] = tip.copy()
    rec["meanx"] = meanx_h.copy()
    fnz_f = p.fnz + 4
    afull = dev(np.zeros(p.fnx * p.fny * fnz_f, np.int32))
    # the reference indexes loss_area[alpha-1], i.e. [-1] for alpha 0: pad both sides
    loss = dev(np.zeros(p.num_theta + 64, np.int32))
    loss_p = ptr(loss) + 32 * 4
    z2 = z.clone()
    ref.check(ref.L.ref_move_frame(ptr(b_ph), ptr(b_id), ptr(z2), ptr(a_ph), ptr(a_id), ptr(z),
                                   ptr(alpha), ptr(afull), loss_p, 1))
    ref.check(ref.L.ref_copy_frame(ptr(b_ph), ptr(b_id), ptr(z2), ptr(a_ph), ptr(a_id), ptr(z)))
    torch.cuda.synchronize()
    rec["move_ph"] = a_ph.cpu().numpy()
    rec["move_id"] = a_id.cpu().numpy()
    rec["move_z"] = z.cpu().numpy()
    rec["move_afull"] = afull.cpu().numpy()
    rec["move_loss"] = loss.cpu().numpy()[32:32 + p.num_theta]
    if opt.get("final_only"):
        keep = {k: v for k, v in rec.items() if not k.startswith("b")}
        rec = keep
    meta = dict(interior=interior, num_pf=num_pf, grains=grains, seed=seed, bc=bc, saves=saves,
                iuc=iuc, thermal=int(p.thermalType), r0=float(p.r0), G=float(p.G))
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), meta=repr(meta), **rec)
    print(name, "saved", sorted(rec))


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    os.makedirs(out_dir, exist_ok=True)
    only = set(sys.argv[2:])
    for name, spec in CASES.items():
        if not only or name in only:
            run_case(name, spec, out_dir)


if __name__ == "__main__":
    main()
