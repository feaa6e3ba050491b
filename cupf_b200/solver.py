"""Python handle over the C ABI (include/cupf.h) of the APT solver.

`APTSolver` owns one simulation on one GPU.  Method names follow the device-side
methods of the reference's APTPhaseField (3DgrainMPI/APTPhaseField.cu): the
constructor is cudaSetup, `step` is the APTsetBC3D + APTrhs_psi pair of evolve,
`collect` is APTcollect_PF, `move_domain` is moveDomain.  All arrays crossing
this API are numpy arrays in the reference layout.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int32)


def _f(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


def _i(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_IP)


class APTSolver:
    def __init__(self, case, device: int = 0, precision: str = "fp32"):
        self.L = abi.lib()
        self.params = case.params
        self._keep = []
        inp = abi.cupf_apt_inputs()
        for n in ("x", "y", "z", "sint", "cost", "X_mac", "Y_mac", "Z_mac", "t_mac", "psi_mac",
                  "T_3D"):
            a = getattr(case, n, None)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float32)
                self._keep.append(a)
                setattr(inp, n, _f(a))
        h = C.c_void_p()
        abi.check(self.L.cupf_apt_create(C.byref(self.params), C.byref(inp), device,
                                         abi.PREC[precision], C.byref(h)))
        self.h = h
        p = self.params
        self.length = p.fnx * p.fny * p.fnz
        self.num_pf = p.num_pf

    # -- lifecycle
    def close(self):
        if self.h:
            abi.check(self.L.cupf_apt_destroy(self.h))
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

    # -- state
    def init_from_argmax(self, phi, alpha):
        phi = np.ascontiguousarray(phi, dtype=np.float32)
        alpha = np.ascontiguousarray(alpha, dtype=np.int32)
        abi.check(self.L.cupf_apt_init_from_argmax(self.h, _f(phi), _i(alpha)))

    def set_slots(self, ph, ids, steps_done=0):
        ph = np.ascontiguousarray(ph, dtype=np.float32)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        abi.check(self.L.cupf_apt_set_slots(self.h, _f(ph), _i(ids), int(steps_done)))

    def get_slots(self):
        n = self.length * self.num_pf
        ph = np.empty(n, np.float32)
        ids = np.empty(n, np.int32)
        abi.check(self.L.cupf_apt_get_slots(self.h, _f(ph), _i(ids)))
        return ph, ids

    def step(self, nsteps=1, use_initial_undercooling=False):
        abi.check(self.L.cupf_apt_step(self.h, int(nsteps), int(bool(use_initial_undercooling))))

    def steps_done(self):
        v = C.c_int64()
        abi.check(self.L.cupf_apt_steps_done(self.h, C.byref(v)))
        return v.value

    def collect(self, clear=True, out=None):
        """Argmax phi and grain-id fields (cupf_apt_collect).  `out` = (phi, alpha):
        caller-owned contiguous float32 / int32 arrays of the field's length to
        read into (page-locked ones make the copy a direct transfer)."""
        if out is None:
            phi = np.empty(self.length, np.float32)
            alpha = np.empty(self.length, np.int32)
        else:
            phi, alpha = out
            for a, dt in ((phi, np.float32), (alpha, np.int32)):
                if a.dtype != dt or a.size != self.length or not a.flags.c_contiguous:
                    raise ValueError("collect out: contiguous %s arrays of %d values"
                                     % (np.dtype(dt).name, self.length))
        abi.check(self.L.cupf_apt_collect(self.h, int(bool(clear)), _f(phi), _i(alpha)))
        return phi, alpha

    def grain_volumes(self, num_grains):
        c = np.zeros(num_grains + 1, np.int64)
        abi.check(self.L.cupf_apt_grain_volumes(self.h, int(num_grains),
                                                c.ctypes.data_as(C.POINTER(C.c_int64))))
        return c

    def qoi_sums(self):
        """(solid volume, interface area, mean interface height) in FP64, cell units."""
        out = (C.c_double * 3)()
        abi.check(self.L.cupf_apt_qoi_sums(self.h, out))
        return tuple(out)

    def move_domain(self, tip_front, tip_thres, move_count):
        tf = C.c_int32(tip_front)
        mc = C.c_int32(move_count)
        moved = C.c_int32(0)
        abi.check(self.L.cupf_apt_move_domain(self.h, C.byref(tf), int(tip_thres), C.byref(mc),
                                              C.byref(moved)))
        return tf.value, mc.value, moved.value

    def get_archive(self, fnz_f):
        p = self.params
        af = np.zeros(p.fnx * p.fny * fnz_f, np.int32)
        loss = np.zeros(p.num_theta, np.int32)
        abi.check(self.L.cupf_apt_get_archive(self.h, int(fnz_f), _i(af), _i(loss)))
        return af, loss

    def get_z(self):
        z = np.empty(self.params.fnz, np.float32)
        abi.check(self.L.cupf_apt_get_z(self.h, _f(z)))
        return z

    def sync(self, timeout_ms=0):
        abi.check(self.L.cupf_apt_sync(self.h, int(timeout_ms)))

    def time_steps(self, nsteps):
        ms = C.c_float()
        abi.check(self.L.cupf_apt_time_steps(self.h, int(nsteps), C.byref(ms)))
        return ms.value

    def nucl_init(self):
        abi.check(self.L.cupf_apt_nucl_init(self.h))

    def nucleate(self, use_initial_undercooling=False, count=True):
        """One nucleation pass; returns the number of nuclei so far (reading it
        waits for the pass; count=False queues the pass and returns None)."""
        if not count:
            abi.check(self.L.cupf_apt_nucleate(self.h, int(bool(use_initial_undercooling)), None))
            return None
        n = C.c_int32()
        abi.check(self.L.cupf_apt_nucleate(self.h, int(bool(use_initial_undercooling)), C.byref(n)))
        return n.value

    def nucl_reset(self):
        abi.check(self.L.cupf_apt_nucl_reset(self.h))

    def set_tuning(self, z_chunk):
        abi.check(self.L.cupf_apt_set_tuning(self.h, int(z_chunk)))

    def set_tile(self, tile_y):
        """Column-tile height of the step's work items: 8 (default) or 4."""
        abi.check(self.L.cupf_apt_set_tile(self.h, int(tile_y)))

    def set_wait_limit(self, cycles):
        """Bound of the step's plane-load waits in SM cycles (0 = default, ~1 s)."""
        abi.check(self.L.cupf_apt_set_wait_limit(self.h, int(cycles)))

    def set_skip_quiet(self, enable):
        """Leave work items whose cells stay all-empty alone (default on)."""
        abi.check(self.L.cupf_apt_set_skip_quiet(self.h, int(bool(enable))))

    def merge_overflows(self):
        """(aliased, dropped) merge-overflow entries since the last call."""
        v = (C.c_uint64 * 2)()
        abi.check(self.L.cupf_apt_merge_overflows(self.h, v))
        return int(v[0]), int(v[1])

    def active_cells(self):
        """Cells of the computed (not quiet) work items since the last call."""
        v = C.c_uint64()
        abi.check(self.L.cupf_apt_active_cells(self.h, C.byref(v)))
        return v.value

    @property
    def stream(self):
        return self.L.cupf_apt_stream(self.h)
