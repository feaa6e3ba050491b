"""2D Echebarria–Karma directional solidification (psi/U line model) on the B200.

Python face of include/cupf_ek2d.h: `EK2DSolver` wraps one device simulation,
`line_model_case` builds a run the way the reference's line-model main.cpp does
(input-file parameters, macro tables, 1-D initial profiles), and
`directional_case` is the synthetic directional-solidification setup used for
the benchmark: a planar front in its steady state (at the solidus, with the
solute boundary layer ahead), seeded perturbation sites, frozen gradient G and
pulling speed R.

Reference: cuPF 2DdendriteMPI/line_model/main.cpp (parameters :82-205, initial
fields :225-271) and PF.cu (setup() time loop :699-842).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# Input-file values of the reference line model (line_model/input_file:11-63),
# with the keys main.cpp reads.
LINE_MODEL_INPUT = dict(G=0.02, R=50.0, delta=0.01, k=0.14, c_infm=7.8, Dl=3000.0, d0=0.005,
                        W0=0.14, c_infty=3.0, eps=1e-8, alpha0=0.0, dx=0.8, asp_ratio=4.0,
                        lxd=80.0, eta=0.04, U0=-1.0, seed_val=400, noi_period=20, cfl=0.8)


@dataclass
class EK2DCase:
    params: abi.cupf_ek2d_params
    t_mac: np.ndarray
    Gt: np.ndarray
    Rt: np.ndarray
    x: np.ndarray
    y: np.ndarray          # float32 row coordinates as main.cpp builds them
    psi: np.ndarray        # reference layout (fny, fnx), float32
    phi: np.ndarray
    U: np.ndarray
    info: dict = field(default_factory=dict)

    @property
    def fnx(self):
        return self.params.nx + 2

    @property
    def fny(self):
        return self.params.ny + 3

    def y64(self):
        """Row coordinates in FP64 (um): y0 + (j-1) dx W0."""
        p = self.params
        return p.y0 + (np.arange(self.fny, dtype=np.float64) - 1.0) * (float(p.dx) * float(p.W0))


def make_params(**kw):
    """cupf_ek2d_params with the input-file fields set (reference defaults for
    the keys not given) and tipp/blank/ls at the reference's compile-time
    values; call derive() afterwards."""
    p = abi.cupf_ek2d_params()
    vals = dict(LINE_MODEL_INPUT)
    vals.update(kw)
    for k, v in vals.items():
        setattr(p, k, v)
    p.tipp = kw.get("tipp", 100)
    p.blank = kw.get("blank", 0.3)
    p.ls = kw.get("ls", -0.995)
    return p


def derive(p, t_last):
    abi.check(abi.lib().cupf_ek2d_derive(C.byref(p), C.c_float(t_last)))
    return p


def initial_fields(p, y_mac, psi_mac, U_mac):
    """x, y, psi, phi, U of main.cpp:225-271 (reference layout, halos zero)."""
    fnx, fny = p.nx + 2, p.ny + 3
    y_mac = np.ascontiguousarray(y_mac, np.float32)
    psi_mac = np.ascontiguousarray(psi_mac, np.float32)
    U_mac = np.ascontiguousarray(U_mac, np.float32)
    x = np.zeros(fnx, np.float32)
    y = np.zeros(fny, np.float32)
    psi = np.zeros((fny, fnx), np.float32)
    phi = np.zeros_like(psi)
    U = np.zeros_like(psi)
    r = abi.lib().cupf_host_ek2d_initial_fields(C.byref(p), len(y_mac), _fp(y_mac), _fp(psi_mac),
                                                _fp(U_mac), _fp(x), _fp(y), _fp(psi), _fp(phi),
                                                _fp(U))
    if r != 0:
        raise ValueError("initial fields: bad tables")
    return x, y, psi, phi, U


def perturb(p, psi, phi, sites, amp):
    r = abi.lib().cupf_host_ek2d_perturb(C.byref(p), int(sites), C.c_float(amp), _fp(psi), _fp(phi))
    if r != 0:
        raise ValueError("perturb failed")


def qois(phi, y, dxd):
    """(tip height um, mean front height um, primary spacing um, wavenumber
    index, mushy row) of one phi frame, from the library's host code."""
    phi = np.ascontiguousarray(phi, np.float32)
    y = np.ascontiguousarray(y, np.float64)
    out = np.zeros(5, np.float64)
    fny, fnx = phi.shape
    r = abi.lib().cupf_host_ek2d_qois(_fp(phi), fnx, fny, _dp(y), C.c_double(dxd), _dp(out))
    if r != 0:
        raise ValueError("qois failed")
    return {"tip_y": out[0], "front_mean_y": out[1], "spacing": out[2], "spacing_k": int(out[3]),
            "mushy_row": int(out[4])}


def directional_case(nx, ny, steps, G=0.1, R=1.0e4, front_frac=0.3, sites=32, amp=0.01,
                     seed=0, eta=0.0, dx=0.8, cfl=0.2, tipp=100, **extra):
    """Directional solidification in a frozen gradient (the split-precision
    benchmark): nx x ny interior cells of dx*W0, G in K/um, pulling speed R in
    um/s, `steps` time steps.  The interface starts planar at the row
    `front_frac` of the height in the steady state of a planar front: at the
    solidus (Up = 0, y = 0 at t = 0) with U = 0 in the solid and the solute
    boundary layer U = -1 + exp(-(y - y_front)/lD), lD = Dl/R, ahead of it;
    `sites` seeded perturbations of amplitude `amp` (in W0) and no noise unless
    eta > 0."""
    W0 = extra.get("W0", LINE_MODEL_INPUT["W0"])
    dxd = np.float32(np.float32(dx) * np.float32(W0))
    kw = dict(G=G, R=R, dx=dx, cfl=cfl, eta=eta, seed_val=seed, tipp=tipp,
              lxd=float((nx + 0.5) * dxd), asp_ratio=float(ny) / nx)
    kw.update(extra)
    p = make_params(**kw)
    derive(p, 1.0)  # tau0 and dt do not depend on t_last
    t_last = np.float32((steps + 0.5) * float(p.tau0) * float(p.dt))
    derive(p, t_last)
    if p.nx != nx or p.ny != ny or p.Mt != steps - (steps % 2):
        raise ValueError("derived grid %dx%d Mt=%d, wanted %dx%d Mt=%d" % (p.nx, p.ny, p.Mt, nx, ny,
                                                                          steps))
    fny = ny + 3
    j_front = int(front_frac * fny)
    n_mac = fny + 8
    # row j of the grid sits at table index j - 1 (main.cpp:244-246); row j_front at y = 0
    y_mac = ((np.arange(n_mac) - (j_front - 1)) * float(dxd)).astype(np.float32)
    lD = float(p.Dl) / float(R)
    yy = y_mac.astype(np.float64)
    psi_mac = (-yy / W0).astype(np.float32)
    U_mac = np.where(yy > 0, -1.0 + np.exp(-np.maximum(yy, 0.0) / lD), 0.0).astype(np.float32)
    p.y0 = float(y_mac[0])
    x, y, psi, phi, U = initial_fields(p, y_mac, psi_mac, U_mac)
    perturb(p, psi, phi, sites, amp)
    t_mac = np.array([0.0, t_last], np.float32)  # main.cpp derives Mt from the last time
    Gt = np.full(2, G, np.float32)
    Rt = np.full(2, R, np.float32)
    return EK2DCase(p, t_mac, Gt, Rt, x, y, psi, phi, U,
                    info={"j_front": j_front, "sites": sites, "amp": amp, "steps": steps,
                          "y_mac": y_mac, "psi_mac": psi_mac, "U_mac": U_mac})


INPUT_KEYS = ("G", "R", "delta", "k", "c_infm", "Dl", "d0", "W0", "c_infty", "eps", "alpha0", "dx",
              "asp_ratio", "lxd", "eta", "U0", "cfl")


def write_line_model_inputs(case: EK2DCase, folder, ztip0=0.0):
    """Write `case` as the reference line model's inputs: an `input_file` of
    `key = value` lines and the macro tables t.txt, Gt.txt, Rt.txt, y.txt,
    psi.txt, U.txt (one value per line, as line_model/thermal.py writes them,
    with nine significant digits so float values survive).  The 1-D profiles
    are the case's initial column; the seeded perturbation is written as the
    keys perturb_sites / perturb_amp."""
    import os
    p = case.params
    os.makedirs(folder, exist_ok=True)
    lines = ["%s = %.9g" % (k, getattr(p, k)) for k in INPUT_KEYS]
    lines += ["seed_val = %d" % p.seed_val, "noi_period = %d" % p.noi_period,
              "Ny = %d" % len(case.info["y_mac"]), "Nt = %d" % len(case.t_mac), "ztip0 = %.9g" % ztip0,
              "perturb_sites = %d" % case.info.get("sites", 0),
              "perturb_amp = %.9g" % case.info.get("amp", 0.0)]
    with open(os.path.join(folder, "input_file"), "w") as f:
        f.write("\n".join("    " + x for x in lines) + "\n")
    for name, arr in (("t.txt", case.t_mac), ("Gt.txt", case.Gt), ("Rt.txt", case.Rt),
                      ("y.txt", case.info["y_mac"]), ("psi.txt", case.info["psi_mac"]),
                      ("U.txt", case.info["U_mac"])):
        np.savetxt(os.path.join(folder, name), np.asarray(arr, np.float32), fmt="%.9e")
    return os.path.join(folder, "input_file")


def line_model_case(input_path, mac_folder):
    """A case built as the reference's line-model main.cpp builds its run:
    parameters from `input_path`, macro tables from `mac_folder`, the initial
    psi/U interpolated from the 1-D profiles (main.cpp:82-271), plus the
    seeded perturbation when the input file has perturb_sites / perturb_amp."""
    import os
    L = abi.lib()
    p = make_params()
    p.cfl = 0.8
    ny, nt, zt = C.c_int32(), C.c_int32(), C.c_float()
    abi.check(L.cupf_ek2d_parse_input(str(input_path).encode(), C.byref(p), C.byref(ny),
                                      C.byref(nt), C.byref(zt)))
    sites, amp = 0, 0.0
    for line in open(input_path):
        w = line.split()
        for i in range(len(w) - 2):
            if w[i + 1] == "=" and w[i] == "perturb_sites":
                sites = int(float(w[i + 2]))
            if w[i + 1] == "=" and w[i] == "perturb_amp":
                amp = float(w[i + 2])

    def col(name, n):
        a = np.loadtxt(os.path.join(mac_folder, name), dtype=np.float64, ndmin=1)[:n]
        return a.astype(np.float32)

    t_mac, Gt, Rt = col("t.txt", nt.value), col("Gt.txt", nt.value), col("Rt.txt", nt.value)
    y_mac, psi_mac, U_mac = col("y.txt", ny.value), col("psi.txt", ny.value), col("U.txt", ny.value)
    derive(p, float(t_mac[-1]))
    p.y0 = float(y_mac[0])
    x, y, psi, phi, U = initial_fields(p, y_mac, psi_mac, U_mac)
    perturb(p, psi, phi, sites, amp)
    return EK2DCase(p, t_mac, Gt, Rt, x, y, psi, phi, U,
                    info={"sites": sites, "amp": amp, "ztip0": zt.value, "y_mac": y_mac,
                          "psi_mac": psi_mac, "U_mac": U_mac})


class EK2DSolver:
    """One device simulation (reference layout in and out)."""

    def __init__(self, case: EK2DCase, precision="fp32", device=0):
        self.case = case
        self.L = abi.lib()
        self.h = C.c_void_p()
        self.params = case.params
        abi.check(self.L.cupf_ek2d_create(C.byref(self.params), abi.PREC_EK2D[precision], device,
                                          C.byref(self.h)))
        t, G, R = (np.ascontiguousarray(a, np.float32) for a in (case.t_mac, case.Gt, case.Rt))
        abi.check(self.L.cupf_ek2d_set_thermal(self.h, len(t), _fp(t), _fp(G), _fp(R)))

    def close(self):
        if self.h:
            self.L.cupf_ek2d_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, psi, U, dpsi=None):
        psi = np.ascontiguousarray(psi, np.float32)
        U = np.ascontiguousarray(U, np.float32)
        d = None if dpsi is None else np.ascontiguousarray(dpsi, np.float32)
        abi.check(self.L.cupf_ek2d_set_state(self.h, _fp(psi), _fp(U),
                                             None if d is None else _fp(d)))

    def prestep(self):
        abi.check(self.L.cupf_ek2d_prestep(self.h))

    def step(self, n):
        abi.check(self.L.cupf_ek2d_step(self.h, int(n)))

    def time_steps(self, n):
        ms = C.c_float()
        abi.check(self.L.cupf_ek2d_time_steps(self.h, int(n), C.byref(ms)))
        return ms.value

    def get_state(self, out=None):
        """psi, phi, U and dpsi (float32, fny x fnx); `out` = four caller-owned
        contiguous float32 arrays of that size to read into."""
        shape = (self.case.fny, self.case.fnx)
        if out is None:
            out = [np.zeros(shape, np.float32) for _ in range(4)]
        else:
            out = [a.reshape(shape) for a in out]
            if any(a.dtype != np.float32 or not a.flags.c_contiguous for a in out):
                raise ValueError("get_state out: four contiguous float32 arrays of %dx%d" % shape)
        abi.check(self.L.cupf_ek2d_get_state(self.h, *[_fp(a) for a in out]))
        return dict(zip(("psi", "phi", "U", "dpsi"), out))

    def get_state_f64(self):
        shape = (self.case.fny, self.case.fnx)
        out = [np.zeros(shape, np.float64) for _ in range(4)]
        abi.check(self.L.cupf_ek2d_get_state_f64(self.h, *[_dp(a) for a in out]))
        return dict(zip(("psi", "phi", "U", "dpsi"), out))

    def get_y(self):
        y = np.zeros(self.case.fny, np.float64)
        abi.check(self.L.cupf_ek2d_get_y(self.h, _dp(y)))
        return y

    def info(self):
        i = abi.cupf_ek2d_info()
        abi.check(self.L.cupf_ek2d_info_get(self.h, C.byref(i)))
        return {n: getattr(i, n) for n, _ in i._fields_}

    def row_means(self):
        m = np.zeros(self.case.fny, np.float64)
        abi.check(self.L.cupf_ek2d_row_means(self.h, _dp(m)))
        return m

    def stream(self):
        s = C.c_void_p()
        abi.check(self.L.cupf_ek2d_stream(self.h, C.byref(s)))
        return s.value
