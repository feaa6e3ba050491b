"""Synthetic directional-solidification cases for the 3D APT solver.

This is the library's stand-in for the reference's Python pre-processing
(3DgrainMPI/grains3D.py, graph_datastruct.py, line.py): it builds the parameter
block, grid coordinates, seeded grain substrate, grain orientations and initial
phase field of a "line" (frozen-gradient) case directly in memory.

Parameter derivation follows PhaseField::parseInputParams
(3DgrainMPI/PhaseFieldCpu.cpp:141-195) with the same float32/float64 rounding
(the reference stores every parameter as float but evaluates several formulas
in double); coordinates follow PhaseField::cpuSetup (:336-355); the initial
field follows PhaseField::initField (:377-449) for the line profile
psi = z0 - z, phi = tanh(psi / W0 / sqrt2), substrate ids where phi > LS.

The substrate is a seeded Voronoi tessellation of the (nx+1) x (ny+1) base with
a given number of grains (periodic or not); orientations use the reference's
two-angle form from a Gaussian random unit vector
(graph_datastruct.py:256-269): theta_x = atan2(uy, ux) mod pi,
theta_z = atan2(sqrt(ux^2+uy^2), uz) mod pi, stored as
theta = [0, theta_x[1..NG], theta_z[1..NG]] (grains3D.py:262).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

F32 = np.float32
LS = -0.995

# Physical constants of the reference's line profile input (3DgrainMPI/line.py).
LINE_CONSTANTS = dict(Tmelt=933.3, Dh=8.43e7, L_cp=229.0, GT=0.347, beta0=1e-7, mu_k=0.217e6,
                      delta=0.01, kin_delta=0.11, undcool_mean=2.0, undcool_std=0.5,
                      nuc_Nmax=0.01, nuc_rad=0.4, eps=1e-8, dx=0.8, W0=0.1, cfl=1.5,
                      underCoolingRate0=20.0)


def derive_params(c: dict) -> dict:
    """Derived parameters with the reference's rounding (PhaseFieldCpu.cpp:141-172)."""
    f = {k: F32(v) for k, v in c.items() if isinstance(v, float)}
    R = np.float64(F32(c["R"]))  # m/s: a float compared with double literals
    cfl = f["cfl"]
    uc0 = f["underCoolingRate0"]
    if R < 0.3:
        cfl = F32(cfl * F32(2))
        uc0 = F32(uc0 / F32(2))
    if R > 0.3 and R < 1.0:
        cfl = F32(np.float64(cfl) * 1.5)
        uc0 = F32(np.float64(uc0) / 1.5)
    d0 = F32(f["GT"] / f["L_cp"])
    beta0 = F32(1.0 / np.float64(F32(f["mu_k"] * f["L_cp"])))
    lamd = F32(0.8839 * np.float64(f["W0"]) / np.float64(d0))
    tau0 = F32(np.float64(F32(F32(beta0 * lamd) * f["W0"])) / 0.8839)
    beta0_tilde = F32(F32(beta0 * f["W0"]) / tau0)
    dt = F32(F32(cfl * f["dx"]) * beta0_tilde)
    hi = F32(1.0 / np.float64(f["dx"]))
    return dict(cfl=cfl, underCoolingRate0=uc0, d0=d0, beta0=beta0, lamd=lamd, tau0=tau0,
                dt=dt, hi=hi, sqrt2=F32(math.sqrt(2.0)))


def voronoi_substrate(nxp: int, nyp: int, num_grains: int, seed: int, periodic: bool) -> np.ndarray:
    """Grain id map (1..num_grains) of shape (nyp, nxp): nearest of num_grains
    seeded points, with periodic wrap when periodic is True."""
    rng = np.random.default_rng(seed)
    px = rng.uniform(0, nxp, num_grains)
    py = rng.uniform(0, nyp, num_grains)
    xs = np.arange(nxp) + 0.5
    ys = np.arange(nyp) + 0.5
    best = np.full((nyp, nxp), np.inf)
    alpha = np.zeros((nyp, nxp), dtype=np.int32)
    for g in range(num_grains):
        dx = np.abs(xs - px[g])
        dy = np.abs(ys - py[g])
        if periodic:
            dx = np.minimum(dx, nxp - dx)
            dy = np.minimum(dy, nyp - dy)
        d = dy[:, None] ** 2 + dx[None, :] ** 2
        m = d < best
        best[m] = d[m]
        alpha[m] = g + 1
    return alpha


def grain_angles(num_grains: int, seed: int) -> np.ndarray:
    """theta = [0, theta_x[1..NG], theta_z[1..NG]] from Gaussian unit vectors."""
    rng = np.random.default_rng(seed + 7919)
    ux, uy, uz = rng.standard_normal((3, num_grains))
    tx = np.arctan2(uy, ux) % math.pi
    tz = np.arctan2(np.sqrt(ux ** 2 + uy ** 2), uz) % math.pi
    return np.concatenate([[0.0], tx, tz]).astype(F32)


@dataclass
class Case:
    """Everything the solver needs for one simulation, in reference layout."""
    params: abi.cupf_apt_params
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    theta: np.ndarray
    sint: np.ndarray
    cost: np.ndarray
    substrate: np.ndarray  # (ny+1, nx+1) grain ids
    phi: np.ndarray        # [length] initial phi (argmax field)
    alpha: np.ndarray      # [length] initial grain ids
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        p = self.params
        return (p.fnz, p.fny, p.fnx)

    @property
    def length(self):
        p = self.params
        return p.fnx * p.fny * p.fnz

    def initial_slots(self):
        """Slot state after set_minus1 + APTini_PF + setBC (reference layout)."""
        p = self.params
        L = self.length
        ph = np.full(p.num_pf * L, -1.0, dtype=F32)
        ids = np.full(p.num_pf * L, -1, dtype=np.int32)
        m = self.phi.astype(np.float64) > LS
        ph[:L][m] = self.phi[m]
        ids[:L][m] = self.alpha[m]
        fill_bc(p, ph, ids)
        return ph, ids


def fill_bc(p, ph: np.ndarray, ids: np.ndarray) -> None:
    """Boundary fill of a reference-layout state: every halo coordinate maps to
    its source independently (mirror: 2 / fn-3, periodic: fn-2 / 1), which is
    what sequential z, y, x face fills of APTsetBC3D give
    (3DgrainMPI/APTPhaseField.cu:93-174)."""
    def src(n, bc):
        s = np.arange(n)
        s[0] = 2 if bc == 0 else n - 2
        s[n - 1] = n - 3 if bc == 0 else 1
        return s
    sx, sy, sz = src(p.fnx, p.bcX), src(p.fny, p.bcY), src(p.fnz, p.bcZ)
    shp = (p.num_pf, p.fnz, p.fny, p.fnx)
    for a in (ph, ids):
        v = a.reshape(shp)
        v[:] = v[:, sz][:, :, sy][:, :, :, sx]


def line_case(nx_int: int, ny_int: int, nz_int: int, num_pf: int = 5, num_grains: int = 20,
              seed: int = 0, G: float = 1.0, R: float = 0.05, kin_delta: float = 0.05,
              bc: str = "110", z0_frac: float = 0.25, substrate_everywhere: bool = True) -> Case:
    """Frozen-gradient line case with nx_int x ny_int x nz_int interior cells.

    G in K/um, R in m/s (UC = G * R * 1e6 * 1e-6 K/us).  bc is the reference's
    -b digits (x, y, z; 1 = periodic).  The substrate fills every solid cell
    (what the reference does under its line configuration, initField :430-437)."""
    c = dict(LINE_CONSTANTS)
    c["kin_delta"] = kin_delta
    c["R"] = R
    d = derive_params({**c})
    dxd = F32(F32(c["dx"]) * F32(c["W0"]))
    nx, ny, nz = nx_int - 1, ny_int - 1, nz_int - 1
    fnx, fny, fnz = nx + 3, ny + 3, nz + 3
    bcX, bcY, bcZ = (int(ch) for ch in bc)

    p = abi.cupf_apt_params()
    p.fnx, p.fny, p.fnz = fnx, fny, fnz
    p.num_pf = num_pf
    p.num_theta = num_grains
    p.bcX, p.bcY, p.bcZ = bcX, bcY, bcZ
    p.thermalType = 1
    p.Nx = p.Ny = p.Nz = p.Nt = 2
    p.kin_delta = F32(kin_delta)
    p.eps = F32(c["eps"])
    p.G = F32(G)
    uc = F32(F32(G) * F32(R * 1e6) * F32(1e-6))
    p.underCoolingRate = uc
    p.underCoolingRate0 = d["underCoolingRate0"]
    p.L_cp = F32(c["L_cp"])
    p.hi = d["hi"]
    p.lamd = d["lamd"]
    p.dt = d["dt"]
    p.tau0 = d["tau0"]
    lxd, lyd, lzd = F32(nx * dxd), F32(ny * dxd), F32(nz * dxd)
    p.lyd, p.lzd = lyd, lzd
    p.z0 = F32(F32(z0_frac) * lzd)
    p.r0 = F32(0.9) * lzd
    p.x0 = F32(0)
    p.angle = F32(0)
    p.V = F32(0)
    p.mp_len = F32(0)
    p.order = F32(1)
    p.dx = F32(c["dx"])
    p.W0 = F32(c["W0"])
    p.undcool_mean = F32(c["undcool_mean"])
    p.undcool_std = F32(c["undcool_std"])
    p.nuc_Nmax = F32(c["nuc_Nmax"])
    p.nuc_Nmax0 = F32(c["nuc_Nmax"])
    p.nuc_rad = F32(c["nuc_rad"])
    p.sqrt2 = d["sqrt2"]
    p.pts_cell = int(F32(c["nuc_rad"]) / dxd)
    p.seed = seed
    p.haloWidth = 1

    x = ((np.arange(fnx) - 1).astype(F32) * dxd).astype(F32)
    y = ((np.arange(fny) - 1).astype(F32) * dxd).astype(F32)
    z = ((np.arange(fnz) - 1).astype(F32) * dxd).astype(F32)
    theta = grain_angles(num_grains, seed)
    sint = np.sin(theta.astype(np.float64)).astype(F32)
    cost = np.cos(theta.astype(np.float64)).astype(F32)
    sub = voronoi_substrate(nx + 1, ny + 1, num_grains, seed, periodic=(bcX == 1 and bcY == 1))

    psi = ((F32(p.z0) - z) / p.W0).astype(F32)
    phz = np.tanh((psi / p.sqrt2).astype(np.float64)).astype(F32)
    phi = np.zeros((fnz, fny, fnx), dtype=F32)
    alpha = np.zeros((fnz, fny, fnx), dtype=np.int32)
    phi[1:-1, 1:-1, 1:-1] = phz[1:-1, None, None]
    solid = phi.astype(np.float64) > LS
    if substrate_everywhere:
        full = np.zeros((fny, fnx), dtype=np.int32)
        full[1:-1, 1:-1] = sub
        alpha[:] = np.where(solid, full[None], 0)
    return Case(params=p, x=x, y=y, z=z, theta=theta, sint=sint, cost=cost, substrate=sub,
                phi=phi.reshape(-1), alpha=alpha.reshape(-1),
                meta=dict(kind="line", interior=(nx_int, ny_int, nz_int), num_grains=num_grains,
                          seed=seed, G=G, R=R, bc=bc))


def cone_case(nx_int: int, ny_int: int, nz_int: int, num_pf: int = 5, num_grains: int = 20,
              seed: int = 0, angle: float = 1.0, V: float = 0.2, bc: str = "110", **kw) -> Case:
    """The line case's grains and initial field under the cone undercooling of
    thermalType 3 (APTPhaseField.cu:292-307): dist = cos(angle) * (sqrt((y -
    lyd/2)^2 + (z0 + lzd - z)^2) - r0(x)), r0(x) = z0 + (r0 - z0) x / lm, lm =
    (r0 - z0) / tan(angle), T = -G dist - UC 1e6 t; cells with x > lm + V 1e6 t
    are not updated.  angle in rad, V in m/s."""
    c = line_case(nx_int, ny_int, nz_int, num_pf, num_grains, seed, bc=bc, **kw)
    p = c.params
    p.thermalType = 3
    p.angle = F32(angle)
    p.V = F32(V)
    c.meta.update(kind="cone", angle=angle, V=V)
    return c


def paraboloid_case(nx_int: int, ny_int: int, nz_int: int, num_pf: int = 5, num_grains: int = 20,
                    seed: int = 0, V: float = 0.5, mp_frac: float = 0.75, curvature: float = 0.15,
                    order: float = 1.0, bc: str = "110", **kw) -> Case:
    """The line case's grains and initial field under the table undercooling of
    thermalType 4 (APTPhaseField.cu:308-325, interp3Dtemperature
    devicefunc.cu_inl:85-125): T = -G * psi(x - V 1e6 t, y, z) (order != 100)
    interpolated trilinearly from a table on a grid of spacing 2 dx W0, with psi a
    paraboloid melt-pool distance psi = z0 - z + curvature * ((x - xc)^2 + (y -
    yc)^2) / lz.  Cells whose shifted x leaves [0, mp_len + x0] are not updated;
    mp_len = mp_frac * lxd, x0 = 0.  The table covers every query the interior
    can make (the reference does not bound its index), with two spare points."""
    c = line_case(nx_int, ny_int, nz_int, num_pf, num_grains, seed, bc=bc, **kw)
    p = c.params
    dxd = F32(F32(p.dx) * F32(p.W0))
    lxd = F32((p.fnx - 3) * dxd)
    p.thermalType = 4
    p.V = F32(V)
    p.x0 = F32(0)
    p.mp_len = F32(F32(mp_frac) * lxd)
    p.order = F32(order)
    D = float(F32(2 * dxd))
    nx = int(math.ceil((float(p.mp_len) + float(p.x0)) / D)) + 3
    ny = int(math.ceil((float(p.lyd) + 4 * float(dxd)) / D)) + 3
    nz = int(math.ceil((float(p.lzd) + 4 * float(dxd)) / D)) + 3
    X = (np.arange(nx) * D).astype(F32)
    Y = (-2 * float(dxd) + np.arange(ny) * D).astype(F32)
    Z = (-2 * float(dxd) + np.arange(nz) * D).astype(F32)
    xc, yc = 0.5 * float(p.mp_len), 0.5 * float(p.lyd)
    lz = float(p.lzd)
    zz, yy, xx = np.meshgrid(Z.astype(np.float64), Y.astype(np.float64), X.astype(np.float64),
                             indexing="ij")
    psi = float(p.z0) - zz + curvature * ((xx - xc) ** 2 + (yy - yc) ** 2) / lz
    p.Nx, p.Ny, p.Nz = nx, ny, nz
    c.X_mac, c.Y_mac, c.Z_mac = X, Y, Z
    c.psi_mac = psi.astype(F32).reshape(-1)  # x fastest (index kx + ky*Nx + kz*Nx*Ny)
    c.meta.update(kind="paraboloid", V=V, mp_len=float(p.mp_len), curvature=curvature, order=order)
    return c


def paraboloid_dist(p, x, y, z, t):
    """Distance field of the analytic paraboloid melt pool (thermalType 5) in
    FP64: the beam at x_b = x0 + V 1e6 t moves in +x along the axis y = lyd/2,
    z = z0 + lzd; at distance xi behind it the pool's radius about the axis is
    R = r0 sqrt(1 - xi/mp_len); ahead of it the pool ends in a hemisphere of
    radius r0; past the tail (xi >= mp_len) the distance is to the axis.
    Positive outside the pool (solid side); T = -G dist - UC 1e6 t."""
    xi = float(p.x0) + float(p.V) * 1e6 * t - np.asarray(x, np.float64)
    u = np.asarray(y, np.float64) - 0.5 * float(p.lyd)
    w = float(p.z0) + float(p.lzd) - np.asarray(z, np.float64)
    rr = u * u + w * w
    mp = float(p.mp_len)
    R = float(p.r0) * np.sqrt(np.clip(1.0 - xi / mp, 0.0, None))
    return np.where(xi <= 0, np.sqrt(rr + xi * xi) - float(p.r0),
                    np.where(xi < mp, np.sqrt(rr) - R, np.sqrt(rr)))


def meltpool_case(nx_int: int, ny_int: int, nz_int: int, num_pf: int = 8, num_grains: int = 400,
                  seed: int = 0, r0: float = 60.0, V: float = 0.5, mp_len: float = 120.0,
                  G: float = 1.0, front_frac: float = 0.75, t_end: float = 1e-4,
                  undcool_mean: float = 10.0, undcool_std: float = 2.0, nuc_nmax: float = 0.01,
                  bc: str = "110", **kw) -> Case:
    """Moving-domain melt-pool configuration with the analytic paraboloid
    undercooling (thermalType 5; the reference tabulates its pool instead,
    thermalType 4): pool radius r0 (um) at the beam, length mp_len (um) behind it,
    scan speed V (m/s) in +x, gradient G (K/um) normal to the pool surface, no
    uniform cooling.  The beam starts at the window's far x edge with the pool
    surface there at front_frac of the window height, so the front rises through
    the window's moving threshold as the pool passes.  The initial phase field is
    tanh(dist / (W0 sqrt2)) with the substrate's grain ids in the solid; the 4-D
    temperature table that nucleation reads (Temp.h5's role) samples the same
    field on a 9 x 9 x Nz x 6 grid up to t_end (the window's z range after the
    largest shift the run can make), with nucleation at undercooling N(mean, std)
    K and density nuc_nmax per um^3."""
    c = line_case(nx_int, ny_int, nz_int, num_pf, num_grains, seed, G=G, R=V, bc=bc, **kw)
    p = c.params
    dxd = F32(F32(p.dx) * F32(p.W0))
    lxd = F32((p.fnx - 3) * dxd)
    p.thermalType = 5
    p.V = F32(V)
    p.r0 = F32(r0)
    p.mp_len = F32(mp_len)
    p.x0 = lxd
    p.z0 = F32(F32(front_frac) * p.lzd + F32(r0) - p.lzd)  # axis at z0 + lzd
    p.underCoolingRate = F32(0.0)
    p.undcool_mean = F32(undcool_mean)
    p.undcool_std = F32(undcool_std)
    p.nuc_Nmax = F32(nuc_nmax)
    p.nuc_Nmax0 = F32(nuc_nmax)
    fnz, fny, fnx = c.shape
    zz, yy, xx = np.meshgrid(c.z.astype(np.float64), c.y.astype(np.float64),
                             c.x.astype(np.float64), indexing="ij")
    dist = paraboloid_dist(p, xx, yy, zz, 0.0)
    phi = np.zeros((fnz, fny, fnx), F32)
    inner = np.tanh(dist / (float(p.W0) * math.sqrt(2.0))).astype(F32)
    phi[1:-1, 1:-1, 1:-1] = inner[1:-1, 1:-1, 1:-1]
    full = np.zeros((fny, fnx), np.int32)
    full[1:-1, 1:-1] = c.substrate
    solid = phi.astype(np.float64) > LS
    alpha = np.where(solid, full[None], 0).astype(np.int32)
    c.phi = phi.reshape(-1)
    c.alpha = alpha.reshape(-1)
    # 4-D temperature table for nucleation
    Nx = Ny = 9
    rise = float(V) * 1e6 * t_end  # the pool passes by this much: bound on the window's shift
    zmax = float(c.z[-1]) + rise + 2 * float(dxd)
    Nz = max(9, int(math.ceil((zmax - float(c.z[0])) / float(4 * dxd))) + 1)
    Nt = 6
    X = np.linspace(float(c.x[0]), float(c.x[-1]), Nx).astype(F32)
    Y = np.linspace(float(c.y[0]), float(c.y[-1]), Ny).astype(F32)
    Z = np.linspace(float(c.z[0]), zmax, Nz).astype(F32)
    tm = np.linspace(0.0, t_end, Nt).astype(F32)
    T = np.empty((Nt, Nz, Ny, Nx), np.float64)
    zg, yg, xg = np.meshgrid(Z.astype(np.float64), Y.astype(np.float64), X.astype(np.float64),
                             indexing="ij")
    for it in range(Nt):
        T[it] = -float(p.G) * paraboloid_dist(p, xg, yg, zg, float(tm[it]))
    p.Nx, p.Ny, p.Nz, p.Nt = Nx, Ny, Nz, Nt
    c.X_mac, c.Y_mac, c.Z_mac, c.t_mac = X, Y, Z, tm
    c.T_3D = T.astype(F32).reshape(-1)  # x fastest, t slowest
    c.meta.update(kind="meltpool", r0=r0, V=V, mp_len=mp_len, G=G, front_frac=front_frac,
                  t_end=t_end)
    return c
