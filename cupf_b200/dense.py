"""Python handle over the C ABI of the full (non-APT) phase-field mode
(include/cupf_dense.h).

`DenseSolver` owns one simulation with one phi field per grain.  Method names
follow the reference's PhaseField (3DgrainMPI/PhaseField.cu): the constructor is
cudaSetup, `init_from_argmax` the set_minus1 / ini_PF / set_BC_3D start of
evolve, `prestep` its pre-loop rhs_psi at t = 0, `step` the set_BC_3D + rhs_psi
pair, `collect` collect_PF, `move_domain` the tip_mvf / move_frame / copy_frame
branch.  Arrays are numpy arrays in the reference layout (grain-major).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .solver import _f, _i


class DenseSolver:
    def __init__(self, case, R=None, device: int = 0):
        """case: a cases.Case; R: pulling speed Rmax in m/s (default: the case's
        meta["R"])."""
        self.L = abi.lib()
        self.params = case.params
        self._keep = []
        inp = abi.cupf_apt_inputs()
        for n in ("x", "y", "z", "sint", "cost"):
            a = np.ascontiguousarray(getattr(case, n), dtype=np.float32)
            self._keep.append(a)
            setattr(inp, n, _f(a))
        if R is None:
            R = case.meta["R"]
        self.R = float(R)
        h = C.c_void_p()
        abi.check(self.L.cupf_dense_create(C.byref(self.params), C.byref(inp), C.c_float(self.R),
                                           device, C.byref(h)))
        self.h = h
        p = self.params
        self.length = p.fnx * p.fny * p.fnz
        self.num_grains = p.num_theta

    def close(self):
        if self.h:
            abi.check(self.L.cupf_dense_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init_from_argmax(self, phi, alpha):
        phi = np.ascontiguousarray(phi, dtype=np.float32)
        alpha = np.ascontiguousarray(alpha, dtype=np.int32)
        abi.check(self.L.cupf_dense_init_from_argmax(self.h, _f(phi), _i(alpha)))

    def prestep(self):
        abi.check(self.L.cupf_dense_prestep(self.h))

    def step(self, nsteps=1):
        abi.check(self.L.cupf_dense_step(self.h, int(nsteps)))

    def steps_done(self):
        n = C.c_int64()
        abi.check(self.L.cupf_dense_steps_done(self.h, C.byref(n)))
        return n.value

    def collect(self, clear=True, out=None):
        """Argmax phi and grain-id fields; `out` = (phi, alpha), caller-owned
        contiguous float32 / int32 arrays of the field's length to read into."""
        if out is None:
            phi = np.empty(self.length, np.float32)
            alpha = np.empty(self.length, np.int32)
        else:
            phi, alpha = out
            for a, dt in ((phi, np.float32), (alpha, np.int32)):
                if a.dtype != dt or a.size != self.length or not a.flags.c_contiguous:
                    raise ValueError("collect out: contiguous %s arrays of %d values"
                                     % (np.dtype(dt).name, self.length))
        abi.check(self.L.cupf_dense_collect(self.h, int(bool(clear)), _f(phi), _i(alpha)))
        return phi, alpha

    def get_slots(self):
        ph = np.empty(self.length * self.num_grains, np.float32)
        abi.check(self.L.cupf_dense_get_slots(self.h, _f(ph)))
        return ph

    def set_slots(self, ph, steps_done=0):
        ph = np.ascontiguousarray(ph, dtype=np.float32)
        abi.check(self.L.cupf_dense_set_slots(self.h, _f(ph), int(steps_done)))

    def move_domain(self, tip_front, tip_thres, move_count):
        tf, mc, moved = C.c_int32(tip_front), C.c_int32(move_count), C.c_int32()
        abi.check(self.L.cupf_dense_move_domain(self.h, C.byref(tf), int(tip_thres), C.byref(mc),
                                                C.byref(moved)))
        return tf.value, mc.value, moved.value

    def get_archive(self, fnz_f):
        p = self.params
        full = np.empty(p.fnx * p.fny * fnz_f, np.int32)
        loss = np.empty(p.num_theta, np.int32)
        abi.check(self.L.cupf_dense_get_archive(self.h, int(fnz_f), _i(full), _i(loss)))
        return full, loss

    def get_z(self):
        z = np.empty(self.params.fnz, np.float32)
        abi.check(self.L.cupf_dense_get_z(self.h, _f(z)))
        return z

    def sync(self, timeout_ms=0):
        abi.check(self.L.cupf_dense_sync(self.h, int(timeout_ms)))

    def time_steps(self, nsteps):
        ms = C.c_float()
        abi.check(self.L.cupf_dense_time_steps(self.h, int(nsteps), C.byref(ms)))
        return ms.value

    def set_tuning(self, list_cap):
        abi.check(self.L.cupf_dense_set_tuning(self.h, int(list_cap)))

    def overflow_cells(self):
        n = C.c_int64()
        abi.check(self.L.cupf_dense_overflow_cells(self.h, C.byref(n)))
        return n.value
