"""Python handle over the continuous-batching server of include/cupf.h."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int32)

PENDING, RUNNING, DONE, FAILED = 0, 1, 2, 3

# Grid shapes of the served request stream (interior cells).
SERVE_GRIDS = [(48, 48, 48), (96, 96, 96), (128, 128, 256), (192, 192, 192)]


def poisson_stream(n, seed=0, num_pf=8, rate=4.0):
    """Seeded stream of 3D grain requests: list of (arrival time in s, Case).

    Arrivals are Poisson at `rate` per second; each request draws its interior
    grid uniformly from SERVE_GRIDS, 10-300 grains, a substrate seed in 0-9999,
    G uniform in 0.1-10 K/um (1e5-1e7 K/m) and R uniform in 0.01-0.5 m/s (the
    time step follows R through the reference's cfl rule)."""
    from . import cases
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += rng.exponential(1.0 / rate)
        g = SERVE_GRIDS[rng.integers(len(SERVE_GRIDS))]
        c = cases.line_case(*g, num_pf=num_pf, num_grains=int(rng.integers(10, 301)),
                            seed=int(rng.integers(0, 10000)), G=float(rng.uniform(0.1, 10.0)),
                            R=float(rng.uniform(0.01, 0.5)), bc="110")
        out.append((t, c))
    return out


class Server:
    def __init__(self, device=0, precision="fp32", num_pf=8, max_active=64, steps_per_round=50,
                 autotune=True, hbm_budget_bytes=0, tile_y=0):
        """tile_y: 0 lets the autotuner pick each grid shape's column-tile height
        with its z chunk (8 without autotune); 4 or 8 fixes it."""
        self.L = abi.lib()
        cfg = abi.cupf_server_config(device, abi.PREC[precision], num_pf, max_active,
                                     steps_per_round, int(bool(autotune)), int(hbm_budget_bytes),
                                     int(tile_y))
        h = C.c_void_p()
        abi.check(self.L.cupf_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.meta = {}

    def close(self):
        if self.h:
            abi.check(self.L.cupf_server_destroy(self.h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, case, nsteps):
        keep = []
        inp = abi.cupf_apt_inputs()
        for n in ("x", "y", "z", "sint", "cost"):
            a = np.ascontiguousarray(getattr(case, n), dtype=np.float32)
            keep.append(a)
            setattr(inp, n, a.ctypes.data_as(_FP))
        phi = np.ascontiguousarray(case.phi, dtype=np.float32)
        alpha = np.ascontiguousarray(case.alpha, dtype=np.int32)
        rid = C.c_int64()
        abi.check(self.L.cupf_server_submit(self.h, C.byref(case.params), C.byref(inp),
                                            phi.ctypes.data_as(_FP), alpha.ctypes.data_as(_IP),
                                            int(nsteps), C.byref(rid)))
        p = case.params
        self.meta[rid.value] = (p.fnx * p.fny * p.fnz, p.num_theta)
        return rid.value

    def pump(self):
        r, q, d = C.c_int32(), C.c_int32(), C.c_int32()
        abi.check(self.L.cupf_server_pump(self.h, C.byref(r), C.byref(q), C.byref(d)))
        return r.value, q.value, d.value

    def status(self, rid):
        st = C.c_int32()
        abi.check(self.L.cupf_server_result(self.h, rid, C.byref(st), None, None, 0, None, None))
        return st.value

    def result(self, rid):
        """dict(alpha, volumes, qoi, times) of a finished request, else None."""
        length, ng = self.meta[rid]
        st = C.c_int32()
        alpha = np.zeros(length, np.int32)
        vols = np.zeros(ng + 1, np.int64)
        qoi = (C.c_double * 3)()
        times = (C.c_double * 3)()
        abi.check(self.L.cupf_server_result(self.h, rid, C.byref(st), alpha.ctypes.data_as(_IP),
                                            vols.ctypes.data_as(C.POINTER(C.c_int64)), ng, qoi,
                                            times))
        if st.value != DONE:
            return None
        return {"alpha": alpha, "volumes": vols, "qoi": tuple(qoi), "times": tuple(times)}

    def stats(self):
        """(device ms of the rounds waited for so far, rounds launched)."""
        ms = C.c_double()
        n = C.c_int64()
        abi.check(self.L.cupf_server_stats(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def tile(self, rid):
        """(column-tile height, z chunk) of an admitted request ((0, 0) before)."""
        ty, zc = C.c_int32(), C.c_int32()
        abi.check(self.L.cupf_server_request_tile(self.h, rid, C.byref(ty), C.byref(zc)))
        return ty.value, zc.value

    def tile_height(self, rid):
        return self.tile(rid)[0]

    def set_tile_height(self, tile_y):
        """Tile height of requests admitted from now on (0 = autotuned)."""
        abi.check(self.L.cupf_server_set_tile(self.h, int(tile_y)))

    def release(self, rid):
        abi.check(self.L.cupf_server_release(self.h, rid))
        self.meta.pop(rid, None)

    def run_until_done(self, rids, max_pumps=100000):
        for _ in range(max_pumps):
            self.pump()
            if all(self.status(r) in (DONE, FAILED) for r in rids):
                return
        raise RuntimeError("requests not finished")
