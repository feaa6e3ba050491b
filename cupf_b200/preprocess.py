"""Writers of the reference's driver inputs: the `forcing/case<seed>/` folder and
the `line.py`-style input file read by `phase_field`.

File names, formats and meanings follow the reference's pre-processing
(3DgrainMPI/grains3D.py:337-378: one value per line, "%1.4e" for reals, "%d" for
integers) and its line input file (3DgrainMPI/line.py); the thermal model is the
line profile psi = z0 - z on a coarse macro grid spanning [-BC, L+BC]
(grains3D.py:258-260, TemperatureProfile3DAnalytic.py).
"""
from __future__ import annotations

import os

import numpy as np

from .cases import LINE_CONSTANTS, grain_angles, voronoi_substrate

INPUT_KEYS = ["Tmelt", "Dh", "L_cp", "GT", "beta0", "mu_k", "delta", "kin_delta",
              "undcool_mean", "undcool_std", "nuc_Nmax", "nuc_rad", "eps", "dx", "W0", "cfl"]


def write_input_file(path, Lx, nts=2, asp_ratio_yx=1.0, asp_ratio_zx=2.0, moving_ratio=1.0,
                     macro=(13, 13, 23, 11), num_pf=8, extra=None, pre_mt=0):
    """A line.py-style parameter file (`key = value` per line).  pre_mt is the
    number of liquid-start steps a nucleation run takes first (preMt)."""
    vals = dict(LINE_CONSTANTS)
    if extra:
        vals.update(extra)
    lines = ["# parameters of a line (frozen-gradient) run"]
    for k in INPUT_KEYS:
        lines.append("%s = %r" % (k, vals[k]))
    lines += ["underCoolingRate0 = %r" % vals["underCoolingRate0"], "nuc_Nmax0 = 0.01",
              "nx = %d" % macro[0], "ny = %d" % macro[1], "nz = %d" % macro[2],
              "nt = %d" % macro[3], "haloWidth = 1", "xmin = 0", "ymin = 0", "zmin = 0",
              "eta = 0.0", "noi_period = 200", "ictype = 0", "asp_ratio_yx = %r" % asp_ratio_yx,
              "asp_ratio_zx = %r" % asp_ratio_zx, "moving_ratio = %r" % moving_ratio,
              "nts = %d" % nts, "Lx = %r" % Lx, "preMt = %d" % pre_mt, "NUM_PF = %d" % num_pf]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def native_substrate(nxp, nyp, num_grains, seed, periodic=True):
    """(alpha (nyp, nxp) int32, theta (2*num_grains+1,) float32) from the
    library's seeded Voronoi generator (cupf_host_voronoi_substrate)."""
    from . import abi
    import ctypes as C
    alpha = np.zeros((nyp, nxp), np.int32)
    theta = np.zeros(2 * num_grains + 1, np.float32)
    r = abi.lib().cupf_host_voronoi_substrate(nxp, nyp, num_grains, C.c_uint64(seed),
                                              1 if periodic else 0,
                                              alpha.ctypes.data_as(C.POINTER(C.c_int32)),
                                              theta.ctypes.data_as(C.POINTER(C.c_float)))
    if r != 0:
        raise ValueError("bad substrate arguments")
    return alpha, theta


def quaternion_angles(q):
    """Unit quaternions (w, x, y, z) per grain, shape (NG, 4), in the reference's
    two-angle form [0, theta_x[1..NG], theta_z[1..NG]] (float32): the angles of
    each grain's crystal [001] axis (cupf_host_quaternions_to_angles; the rotation
    about that axis is dropped)."""
    from . import abi
    import ctypes as C
    q = np.ascontiguousarray(q, np.float64).reshape(-1, 4)
    theta = np.zeros(2 * len(q) + 1, np.float32)
    if abi.lib().cupf_host_quaternions_to_angles(len(q), q.ctypes.data_as(C.POINTER(C.c_double)),
                                                 theta.ctypes.data_as(C.POINTER(C.c_float))) != 0:
        raise ValueError("zero or non-finite quaternion")
    return theta


def write_line_forcing(folder, Lx, Ly, Lz, num_grains, seed, G, R, z0, top, t_end,
                       periodic=True, macro=(13, 13, 23, 11), dxd=0.08, nmax=0.01,
                       cooling_rate=None, substrate="cases", quaternions=None):
    """The forcing folder of a line run: macro grid, psi = z0 - z, substrate ids
    (alpha.txt, (nx+1)x(ny+1) values), orientations, scalars.  nmax is the
    nucleation density (Nmax.txt).  With cooling_rate (K/s) the folder also holds
    the 4-D temperature table Temp.txt (the reference's Temp.h5:/Temp, x fastest,
    t slowest) of a uniform melt cooling from the melting point,
    T - Tmelt = -cooling_rate * t, which nucleation reads.

    substrate: "cases" (the numpy generator the in-memory test cases use),
    "native" (the library's C++ generator), or an (alpha, theta) pair made
    elsewhere, e.g. by the reference's own graph() (alpha (ny+1, nx+1)).
    quaternions: orientations as unit quaternions (NG, 4) written to
    quaternions.txt in place of theta.txt (the drivers convert them)."""
    os.makedirs(folder, exist_ok=True)
    nxm, nym, nzm, ntm = macro
    BC = Lx / (nxm - 3)
    x = np.linspace(0 - BC, Lx + BC, nxm)
    y = np.linspace(0 - BC, Ly + BC, nym)
    z = np.linspace(0 - BC, Lz + BC, nzm)
    t = np.linspace(0, t_end, ntm)
    xx, yy, zz = np.meshgrid(x, y, z, indexing="ij")
    psi = (z0 - zz).reshape(-1, order="F")
    nx = int(round(Lx / dxd))
    ny = int(round(Ly / dxd))
    if isinstance(substrate, str) and substrate == "native":
        alpha, theta = native_substrate(nx + 1, ny + 1, num_grains, seed, periodic)
    elif isinstance(substrate, str):
        alpha = voronoi_substrate(nx + 1, ny + 1, num_grains, seed, periodic)
        theta = grain_angles(num_grains, seed)
    else:
        alpha, theta = (np.asarray(a) for a in substrate)
        if alpha.shape != (ny + 1, nx + 1) or len(theta) != 2 * num_grains + 1:
            raise ValueError("substrate shape %s / %d angles do not fit a %dx%d map of %d grains"
                             % (alpha.shape, len(theta), nx + 1, ny + 1, num_grains))
    uc = G * R * 1e6 * 1e-6  # K/us

    def put(name, arr, fmt="%1.4e"):
        np.savetxt(os.path.join(folder, name), np.asarray(arr).reshape(-1), fmt=fmt, delimiter="\n")

    put("x.txt", x)
    put("y.txt", y)
    put("z.txt", z)
    put("t.txt", t)
    put("psi.txt", psi)
    put("alpha.txt", alpha.reshape(-1), "%d")
    if quaternions is None:
        put("theta.txt", theta)
    else:
        put("quaternions.txt", np.asarray(quaternions, np.float64).reshape(-1), "%1.8e")
    put("G.txt", [G])
    put("Rmax.txt", [R])
    put("V.txt", [0.0])
    put("Nmax.txt", [nmax])
    if cooling_rate is not None:
        temp = np.broadcast_to(-cooling_rate * t[:, None, None, None], (ntm, nzm, nym, nxm))
        put("Temp.txt", temp)
    put("UC.txt", [uc])
    put("NG.txt", [num_grains], "%d")
    put("NN.txt", [2 * num_grains], "%d")
    put("z0.txt", [z0])
    put("r0.txt", [0.9 * Lz])
    put("x0.txt", [0.0])
    put("top.txt", [top])
    put("angle.txt", [0.0])
    put("min_angle.txt", [0.0])
    put("order.txt", [1.0])
    return dict(nx=nx, ny=ny, alpha=alpha, theta=theta)
