"""The C++ driver reads a forcing folder and input file the way the reference
does (parseInputParams + cpuSetup + initField, PhaseFieldCpu.cpp:17-459) and
arrives at the same parameters and initial state as the in-memory case builder
(which restates the same derivation), up to the 5 significant digits the
forcing files store."""
import numpy as np
import pytest

from cupf_b200 import cases, host_api, preprocess


def test_setup_from_forcing_folder(tmp_path, monkeypatch, built):
    Lx, Ly, Lz = 2.48, 1.92, 2.48   # 32 x 25 x 32 interior points at dx*W0 = 0.08 um
    z0 = 0.62
    folder = tmp_path / "forcing" / "case3"
    info = preprocess.write_line_forcing(str(folder), Lx, Ly, Lz, num_grains=9, seed=3, G=1.0,
                                         R=0.05, z0=z0, top=0.4, t_end=1e-6)
    preprocess.write_input_file(str(tmp_path / "line.py"), Lx, nts=2, asp_ratio_yx=Ly / Lx,
                                asp_ratio_zx=2.0, moving_ratio=1.0, num_pf=5,
                                extra={"kin_delta": 0.05})
    monkeypatch.chdir(tmp_path)
    dims, fp, phi, alpha = host_api.setup("line.py", str(folder), bc=(1, 1, 0), line_config=True)
    assert tuple(dims) == (34, 27, 34, 9)
    c = cases.line_case(32, 25, 32, num_pf=5, num_grains=9, seed=3, bc="110", z0_frac=z0 / Lz)
    p = c.params
    dt, tau0, lamd, hi, G, uc, z0r, kd = fp
    assert dt == p.dt and tau0 == p.tau0 and lamd == p.lamd and hi == p.hi
    assert abs(uc - 0.05) < 1e-6 and G == np.float32(1.0) and kd == np.float32(0.05)
    # phi interpolated from the 5-digit macro grid vs the exact profile
    inner = np.zeros((34, 27, 34), bool)
    inner[1:-1, 1:-1, 1:-1] = True
    inner = inner.reshape(-1)
    assert np.max(np.abs(phi[inner] - c.phi[inner])) < 2e-3
    # substrate ids where both are clearly solid
    solid = inner & (c.phi > -0.99) & (phi > -0.99)
    assert solid.sum() > 1000
    assert np.array_equal(alpha[solid], c.alpha[solid])
    assert np.all(alpha[inner & (phi <= -0.995)] == 0)


def test_setup_reads_alpha3d_field(tmp_path, monkeypatch, built):
    """A 3-D run (not line, not pure nucleation) takes its initial grain ids from
    alpha3D.txt when the forcing folder has one (the additive-manufacturing
    driver's alpha3D.h5, AdditiveManufacturing/PhaseFieldCpu.cpp:430-447), else
    all ids are 0; a short file is an error."""
    Lx = 2.48
    folder = tmp_path / "forcing" / "case0"
    preprocess.write_line_forcing(str(folder), Lx, Lx, 2 * Lx, num_grains=9, seed=0, G=1.0,
                                  R=0.05, z0=0.6, top=0.3, t_end=5e-7)
    preprocess.write_input_file(str(tmp_path / "line.py"), Lx, nts=2, asp_ratio_zx=2.0, num_pf=8)
    monkeypatch.chdir(tmp_path)
    dims, _, _, alpha = host_api.setup("line.py", str(folder), bc=(1, 1, 0))
    assert not alpha.any()
    L = int(dims[0]) * int(dims[1]) * int(dims[2])
    ids = np.random.default_rng(1).integers(0, 10, L).astype(np.int32)
    np.savetxt(folder / "alpha3D.txt", ids, fmt="%d")
    _, _, _, alpha = host_api.setup("line.py", str(folder), bc=(1, 1, 0))
    assert np.array_equal(alpha, ids)
    # the line configuration and pure nucleation do not read it
    _, _, _, alpha = host_api.setup("line.py", str(folder), bc=(1, 1, 0), pure_nucleation=True)
    assert not alpha.any()
    np.savetxt(folder / "alpha3D.txt", ids[:-1], fmt="%d")
    with pytest.raises(RuntimeError, match="alpha3D"):
        host_api.setup("line.py", str(folder), bc=(1, 1, 0))


CASES = [
    # input file name (sets thermalType), line configuration, pure nucleation, bc, extra files
    ("line.py", True, False, (1, 1, 0), {}),
    ("line.py", False, False, (0, 0, 0), {}),
    ("line.py", True, True, (1, 0, 0), {}),
    ("cylinder.py", False, False, (1, 1, 0), {}),
    ("cone.py", True, False, (0, 1, 1), {"angle.txt": "0.7\n", "V.txt": "0.2\n"}),
    ("paraboloid.py", True, False, (1, 1, 0), {"mp_len.txt": "1.6\n", "V.txt": "0.5\n"}),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "%s_line%d_pure%d_bc%d%d%d" % (
    c[0][:-3], c[1], c[2], *c[3]))
def test_setup_matches_reference_host_code(tmp_path, monkeypatch, built, case):
    """The driver's parseInputParams + cpuSetup + initField against the
    reference's own PhaseFieldCpu.cpp:17-459 (compiled unmodified, with a stub
    hdf5.h whose reads return zeros, into oracle/_ref) on the same input file and
    forcing folder: every derived parameter, coordinate array, the interpolated
    psi and phi, the substrate ids and the orientation sines and cosines, bit for
    bit."""
    try:
        from oracle import RefSetup
        ref = RefSetup()
    except (FileNotFoundError, OSError) as e:
        pytest.skip("reference host code not built: %s" % e)
    name, line, pure, bc, extra = case
    Lx, Ly, Lz = 2.48, 1.92, 4.96  # the macro grid covers asp_ratio_zx = 2
    folder = tmp_path / "forcing" / "case5"
    preprocess.write_line_forcing(str(folder), Lx, Ly, Lz, num_grains=11, seed=5, G=2.0,
                                  R=0.4, z0=0.55, top=0.4, t_end=1e-6)
    for fname, text in extra.items():
        (folder / fname).write_text(text)
    preprocess.write_input_file(str(tmp_path / name), Lx, nts=3, asp_ratio_yx=Ly / Lx,
                                asp_ratio_zx=2.0, moving_ratio=0.75 if line else 1.0, num_pf=6,
                                extra={"kin_delta": 0.07})
    monkeypatch.chdir(tmp_path)
    kw = dict(bc=bc, line_config=line, pure_nucleation=pure, cap=1 << 20)
    mine = host_api.setup_state(name, str(folder), **kw)
    theirs = ref.setup(name, str(folder), **kw)
    assert mine.keys() == theirs.keys()
    for k, v in theirs.items():
        if isinstance(v, np.ndarray):
            assert v.dtype == mine[k].dtype and v.shape == mine[k].shape, k
            assert np.array_equal(mine[k].view(np.int32), v.view(np.int32)), k
        else:
            assert np.array_equal(np.float32(mine[k]).view(np.int32),
                                  np.float32(v).view(np.int32)) if isinstance(v, np.floating) \
                else mine[k] == v, (k, mine[k], v)
