"""Known-answer cases of the 3D APT step, shared by the oracle (CPU) and the
library (GPU) tests.

* A single grain with a flat front and periodic x/y reduces the 3D step to one
  column: `front_1d` integrates that column in FP64 straight from the equation of
  APTrhs_psi (3DgrainMPI/APTPhaseField.cu:254-348: one active slot, no
  repulsion, the line undercooling G (z - z0) - UC 1e6 t, kine_ani of the normal
  (0, 0, dphi/dz) rotated by the grain's angles, ids dropped below -0.9999).
* Two grains of the same orientation meeting on a plane x = const under zero
  undercooling, with no-flux x boundaries, are mirror images of each other: every
  operation of the step is symmetric under x -> -x (sums are commutative,
  differences change sign exactly, the rotation by zero angles keeps each
  component), so grain 1 at x and grain 2 at the mirrored x stay equal bit for
  bit and the boundary stays where it is.
* With periodic x the step commutes with a shift in x (`roll_x`).
"""
import numpy as np

from cupf_b200 import cases

LS = -0.995
DROP = -0.9999


def flat_front_case(nz_int=64, num_pf=2, z0_frac=0.3, theta=(0.4, 0.9), G=1.0, R=0.05):
    """One grain filling the solid below a flat front; periodic x and y."""
    c = cases.line_case(8, 8, nz_int, num_pf=num_pf, num_grains=1, seed=0, G=G, R=R, bc="110",
                        z0_frac=z0_frac)
    c.theta = np.array([0.0, theta[0], theta[1]], np.float32)
    c.sint = np.sin(c.theta.astype(np.float64)).astype(np.float32)
    c.cost = np.cos(c.theta.astype(np.float64)).astype(np.float32)
    return c


def front_1d(c, nsteps):
    """FP64 integration of the flat-front column; returns phi per z (halo
    included, -1 where the slot is empty) after each of nsteps steps."""
    p = c.params
    fnz = p.fnz
    col = c.phi.reshape(fnz, p.fny, p.fnx)[:, 1, 1].astype(np.float64)
    ph = np.where(col > LS, col, -1.0)
    occ = col > LS
    ph[0], ph[-1] = -1.0, -1.0
    occ[0] = occ[-1] = False
    z = c.z.astype(np.float64)
    kd = float(p.kin_delta)
    a_s = 1.0 + 3.0 * kd
    epsilon = -4.0 * kd / a_s
    sa, ca = float(c.sint[1]), float(c.cost[1])
    sb, cb = float(c.sint[2]), float(c.cost[2])
    dt, hi, lamd, L_cp = float(p.dt), float(p.hi), float(p.lamd), float(p.L_cp)
    G, z0, uc, eps = float(p.G), float(p.z0), float(p.underCoolingRate), float(p.eps)
    out = []
    for n in range(1, nsteps + 1):
        t = float(np.float32(np.float32(n) * np.float32(p.dt)) * np.float32(p.tau0))
        # no-flux z: halo planes mirror about the first / last interior plane
        ph[0], occ[0] = ph[2], occ[2]
        ph[-1], occ[-1] = ph[-3], occ[-3]
        new = np.full(fnz, -1.0)
        new_occ = np.zeros(fnz, bool)
        for k in range(1, fnz - 1):
            if not (occ[k - 1] or occ[k] or occ[k + 1]):
                continue
            phC = ph[k] if occ[k] else -1.0
            phU = ph[k + 1] if occ[k + 1] else -1.0
            phD = ph[k - 1] if occ[k - 1] else -1.0
            uz = (phU - phD) * 0.5
            if phC > LS:
                rx, ry, rz = -sb * uz, 0.0, cb * uz
            else:
                rx, ry, rz = 0.0, 0.0, uz
            mag = rx * rx + ry * ry + rz * rz
            if mag > eps:
                q = rx ** 4 + ry ** 4 + rz ** 4
                A2 = a_s * (1.0 + epsilon * q / (mag * mag))
            else:
                A2 = 1.0
            diff = phU + phD - 2.0 * phC
            w = 1.0 - phC * phC
            E1 = diff * hi * hi + w * phC
            T = G * (z[k] - z0) - uc * 1e6 * t
            rhs = E1 - lamd * (T / L_cp) * (w * w)
            nv = phC + dt * rhs / A2
            if nv >= DROP:
                new[k], new_occ[k] = nv, True
        ph, occ = new, new_occ
        out.append(ph.copy())
    return out


def front_position(col):
    """Height (in cells, fractional) of the last phi = 0 crossing of a column."""
    s = np.nonzero((col[:-1] > 0) & (col[1:] <= 0))[0]
    if not len(s):
        return float("nan")
    k = s[-1]
    return k + col[k] / (col[k] - col[k + 1])


def column_of(p, ph, ids, slot=0, i=1, j=1):
    """phi of one slot along z at (i, j), -1 where the slot holds no id."""
    L = p.fnx * p.fny * p.fnz
    v = ph[slot * L:(slot + 1) * L].reshape(p.fnz, p.fny, p.fnx)[:, j, i].astype(np.float64)
    d = ids[slot * L:(slot + 1) * L].reshape(p.fnz, p.fny, p.fnx)[:, j, i]
    return np.where(d >= 0, v, -1.0)


def mirror_case(nx_int=24, ny_int=6, nz_int=6, num_pf=3):
    """Two grains (ids 1, 2, zero angles) split by the plane between the middle
    interior columns, no-flux x, periodic y and z, no undercooling.  Returns the
    case and its initial slots (own grain in slot 0, the other in slot 1)."""
    c = cases.line_case(nx_int, ny_int, nz_int, num_pf=num_pf, num_grains=2, seed=0, bc="011",
                        z0_frac=0.5)
    p = c.params
    p.G = np.float32(0.0)
    p.underCoolingRate = np.float32(0.0)
    c.theta = np.zeros(5, np.float32)
    c.sint = np.zeros(5, np.float32)
    c.cost = np.ones(5, np.float32)
    L = p.fnx * p.fny * p.fnz
    ph = np.full(num_pf * L, -1.0, np.float32)
    ids = np.full(num_pf * L, -1, np.int32)
    xm = (p.fnx - 1) / 2.0  # between the middle interior columns
    sq2 = float(p.sqrt2)
    for k in range(1, p.fnz - 1):
        for j in range(1, p.fny - 1):
            for i in range(1, p.fnx - 1):
                d = (i - xm) * float(p.dx)
                own, other = (1, 2) if i < xm else (2, 1)
                a = np.float32(np.tanh(abs(d) / sq2))
                b = np.float32(np.tanh(-abs(d) / sq2))
                C = (k * p.fny + j) * p.fnx + i
                ph[C], ids[C] = a, own
                if b > DROP:
                    ph[L + C], ids[L + C] = b, other
    cases.fill_bc(p, ph, ids)
    return c, ph, ids


def mirrored(p, ph, ids):
    """The state reflected in x with grain ids 1 and 2 exchanged."""
    npf = len(ph) // (p.fnx * p.fny * p.fnz)
    a = ph.reshape(npf, p.fnz, p.fny, p.fnx)[:, :, :, ::-1]
    d = ids.reshape(npf, p.fnz, p.fny, p.fnx)[:, :, :, ::-1]
    d = np.where(d == 1, 2, np.where(d == 2, 1, d))
    return np.ascontiguousarray(a).reshape(-1), np.ascontiguousarray(d).reshape(-1)


def roll_x(p, a, s):
    """Shift the interior of a reference-layout array by s cells in x
    (periodic); the halo columns are left for the boundary fill."""
    npf = len(a) // (p.fnx * p.fny * p.fnz)
    v = a.reshape(npf, p.fnz, p.fny, p.fnx).copy()
    v[:, :, :, 1:-1] = np.roll(v[:, :, :, 1:-1], s, axis=3)
    return v.reshape(-1)
