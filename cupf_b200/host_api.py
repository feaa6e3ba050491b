"""ctypes binding of include/cupf_host.h (host side of the APT driver)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int32)

_bound = False


def _lib():
    global _bound
    L = abi.lib()
    if not _bound:
        L.cupf_host_grain_volumes.argtypes = [C.c_int] * 3 + [_IP, _IP, _IP, C.c_int]
        L.cupf_host_line_qois.argtypes = [C.c_int] * 4 + [_IP, _IP, _IP, C.c_int, _IP, _IP, _IP]
        L.cupf_host_sample_heights.argtypes = [_IP, _IP, C.c_int, C.c_int, C.c_int]
        L.cupf_host_junctions_3d.argtypes = [C.c_int] * 3 + [_IP, _IP, C.c_int]
        L.cupf_host_get_param_float.argtypes = [C.c_char_p, C.c_char_p, _FP]
        L.cupf_host_get_param_int.argtypes = [C.c_char_p, C.c_char_p, _IP]
        L.cupf_host_get_options.argtypes = [C.c_int, C.POINTER(C.c_char_p), _IP, C.c_char_p,
                                            C.c_char_p, C.c_char_p, C.c_int]
        L.cupf_host_setup.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                      _IP, _FP, _FP, _IP, C.c_int64, C.c_char_p, C.c_int]
        L.cupf_host_setup_state.argtypes = [C.c_char_p, C.c_char_p] + [C.c_int] * 4 + [
            _IP, _FP] + [_FP] * 6 + [_IP, _FP, _FP, C.c_int64, C.c_char_p, C.c_int]
        L.cupf_host_h5_write.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), C.c_char_p,
                                         _IP, C.POINTER(C.c_int64), C.POINTER(C.c_void_p)]
        _bound = True
    return L


def _i(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_IP)


def h5_write(path, arrays):
    """Write {name: 1-D numpy array} (signed integers or float32/float64) as an
    HDF5 file through the drivers' writer (cupf_host_h5_write)."""
    names = list(arrays)
    arrs = [np.ascontiguousarray(arrays[k]).reshape(-1) for k in names]
    for a in arrs:
        if a.dtype.kind not in "if" or a.dtype.byteorder == ">":
            raise TypeError("unsupported dtype %s" % a.dtype)
    n = len(names)
    cn = (C.c_char_p * n)(*[k.encode() for k in names])
    kinds = "".join(a.dtype.kind for a in arrs).encode()
    elem = np.array([a.dtype.itemsize for a in arrs], np.int32)
    counts = (C.c_int64 * n)(*[a.size for a in arrs])
    data = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
    r = _lib().cupf_host_h5_write(path.encode(), n, cn, kinds, _i(elem), counts, data)
    if r != 0:
        raise IOError("cupf_host_h5_write failed for %s" % path)


def grain_volumes(fnx, fny, fnz, alpha, cap=1 << 20):
    g = np.zeros(cap, np.int32)
    v = np.zeros(cap, np.int32)
    n = _lib().cupf_host_grain_volumes(fnx, fny, fnz, _i(alpha), _i(g), _i(v), cap)
    if n < 0:
        raise ValueError("too many grains")
    return g[:n].copy(), v[:n].copy()


def line_qois(fnx, fny, fnz, num_theta, cur_tip, alpha, loss_area, move_count):
    tip = C.c_int(cur_tip)
    tip_y = np.zeros(1, np.int32)
    tot = np.zeros(num_theta, np.int32)
    ext = np.zeros(num_theta, np.int32)
    _lib().cupf_host_line_qois(fnx, fny, fnz, num_theta, C.byref(tip), _i(alpha), _i(loss_area),
                               move_count, _i(tip_y), _i(tot), _i(ext))
    return tip.value, int(tip_y[0]), tot, ext


def sample_heights(cur_tip, alpha, fnx, fny, fnz):
    t = np.array([cur_tip], np.int32)
    _lib().cupf_host_sample_heights(_i(t), _i(alpha), fnx, fny, fnz)
    return int(t[0])


def junctions_3d(fnx, fny, fnz, alpha, cap=1 << 22):
    out = np.zeros(cap, np.int32)
    n = _lib().cupf_host_junctions_3d(fnx, fny, fnz, _i(alpha), _i(out), cap)
    return out[:n].copy()


def line_junctions(fnx, fny, nts, num_nodes, tip_y, alpha, cells=None):
    """QOILine::searchJunctionsOnImage on a full map (frame kt's tip layer at
    tip_y[kt]): (node_region, cross_sec).  With `cells` (ascending candidate
    indices into the stacked tip layers, as cupf_line_junction_candidates gives
    them) the records are built for those cells only."""
    cap = (nts + 1) * 5 * num_nodes * 8
    out = np.zeros(max(cap, 1), np.int32)
    cross = np.zeros((nts + 1) * fnx * fny, np.int32)
    tip = np.ascontiguousarray(tip_y, np.int32)
    a = np.ascontiguousarray(alpha, np.int32)
    if cells is None:
        n = _lib().cupf_host_line_junctions(fnx, fny, nts, num_nodes, _i(tip), _i(a), _i(out),
                                            cap, _i(cross), C.c_int64(len(cross)))
    else:
        c = np.ascontiguousarray(cells, np.int64)
        n = _lib().cupf_host_line_junctions_cells(
            fnx, fny, nts, num_nodes, _i(tip), _i(a), c.ctypes.data_as(C.POINTER(C.c_int64)),
            C.c_int64(len(c)), _i(out), cap, _i(cross), C.c_int64(len(cross)))
    if n < 0:
        raise ValueError("bad argument")
    return out[:n].copy(), cross


def line_junction_candidates(fnx, fny, layers, device=0):
    """Device candidates of the line junction search over stacked tip layers
    (nlayers x fny x fnx int32): ascending indices into the stack."""
    layers = np.ascontiguousarray(layers, np.int32)
    nl = layers.size // (fnx * fny)
    cap = 1 << 12
    while True:
        cells = np.zeros(cap, np.int64)
        count = C.c_int64()
        abi.check(_lib().cupf_line_junction_candidates(
            device, fnx, fny, _i(layers), nl, cells.ctypes.data_as(C.POINTER(C.c_int64)),
            C.c_int64(cap), C.byref(count)))
        if count.value <= cap:
            return cells[:count.value].copy()
        cap = count.value


def get_param(line, key, kind=float, init=0):
    if kind is float:
        v = C.c_float(init)
        _lib().cupf_host_get_param_float(line.encode(), key.encode(), C.byref(v))
    else:
        v = C.c_int32(init)
        _lib().cupf_host_get_param_int(line.encode(), key.encode(), C.byref(v))
    return v.value


def get_options(argv):
    arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
    out = np.zeros(10, np.int32)
    b1, b2, b3 = (C.create_string_buffer(512) for _ in range(3))
    _lib().cupf_host_get_options(len(argv), arr, _i(out), b1, b2, b3, 511)
    return out, b1.value.decode(), b2.value.decode(), b3.value.decode()


SETUP_FPARAMS = ("dt", "tau0", "lamd", "hi", "G", "underCoolingRate", "z0", "kin_delta", "lxd",
                 "lyd", "lzd", "R", "V", "top", "r0", "x0", "cfl", "underCoolingRate0", "W0",
                 "dx")
SETUP_DIMS = ("fnx", "fny", "fnz", "num_theta", "Mt", "nts", "thermalType", "fnz_f")


def setup_state(input_file, folder, bc=(0, 0, 0), line_config=False, pure_nucleation=False,
                nucleation=False, cap=1 << 26):
    """The driver's parseInputParams + cpuSetup + initField with the state the
    reference's PhaseField holds afterwards: dict of SETUP_DIMS, SETUP_FPARAMS and
    arrays x, y, z, z_full, phi, psi, alpha, sint, cost."""
    dims = np.zeros(8, np.int32)
    fp = np.zeros(20, np.float32)
    arr = {k: np.zeros(cap, np.float32) for k in ("x", "y", "z", "z_full", "phi", "psi", "sint",
                                                     "cost")}
    alpha = np.zeros(cap, np.int32)
    err = C.create_string_buffer(512)
    flags = (1 if line_config else 0) | (2 if pure_nucleation else 0) | (4 if nucleation else 0)
    f = lambda k: arr[k].ctypes.data_as(_FP)
    r = _lib().cupf_host_setup_state(input_file.encode(), folder.encode(), bc[0], bc[1], bc[2],
                                     flags, _i(dims), fp.ctypes.data_as(_FP), f("x"), f("y"),
                                     f("z"), f("z_full"), f("phi"), f("psi"), _i(alpha), f("sint"),
                                     f("cost"), cap, err, 511)
    if r != 0:
        raise RuntimeError(err.value.decode() or "capacity too small")
    return setup_dict(dims, fp, arr, alpha)


def setup_dict(dims, fp, arr, alpha):
    d = dict(zip(SETUP_DIMS, (int(v) for v in dims)))
    d.update(zip(SETUP_FPARAMS, (np.float32(v) for v in fp)))
    L = d["fnx"] * d["fny"] * d["fnz"]
    nt = 2 * d["num_theta"] + 1
    for k, n in (("x", d["fnx"]), ("y", d["fny"]), ("z", d["fnz"]), ("z_full", d["fnz_f"]),
                 ("phi", L), ("psi", L), ("sint", nt), ("cost", nt)):
        d[k] = arr[k][:n].copy()
    d["alpha"] = alpha[:L].copy()
    return d


def setup(input_file, folder, bc=(0, 0, 0), line_config=False, pure_nucleation=False,
          length_cap=1 << 26):
    """parseInputParams + cpuSetup + initField; returns (dims, fparams, phi, alpha)."""
    dims = np.zeros(4, np.int32)
    fp = np.zeros(8, np.float32)
    phi = np.zeros(length_cap, np.float32)
    alpha = np.zeros(length_cap, np.int32)
    err = C.create_string_buffer(512)
    flags = (1 if line_config else 0) | (2 if pure_nucleation else 0)
    r = _lib().cupf_host_setup(input_file.encode(), folder.encode(), bc[0], bc[1], bc[2], flags,
                               _i(dims), fp.ctypes.data_as(_FP), phi.ctypes.data_as(_FP),
                               _i(alpha), length_cap, err, 511)
    if r != 0:
        raise RuntimeError(err.value.decode())
    L = int(dims[0]) * int(dims[1]) * int(dims[2])
    return dims, fp, phi[:L].copy(), alpha[:L].copy()
