"""The phase_field executable runs a line configuration end to end on a B200:
forcing folder + input file in, an HDF5 file of QoIs out with the reference's
dataset names (PhaseFieldCpu.cpp:493-519, QOI.cpp:19-34), read back with the
tests' own HDF5 reader (tests/h5read.py); CUPF_OUTPUT_FORMAT=npz gives the same
datasets as a NumPy archive."""
import os
import subprocess

import numpy as np
import pytest

from cupf_b200 import preprocess
from tests.h5read import H5File

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_phase_field_cli_line_run(tmp_path, built):
    Lx = 2.48
    folder = tmp_path / "forcing" / "case0"
    preprocess.write_line_forcing(str(folder), Lx, Lx, 2 * Lx, num_grains=10, seed=0, G=1.0,
                                  R=0.05, z0=0.6, top=0.3, t_end=5e-7)
    preprocess.write_input_file(str(tmp_path / "line.py"), Lx, nts=2, asp_ratio_zx=2.0,
                                moving_ratio=1.0, num_pf=8)
    exe = os.path.join(ROOT, "cupf_b200", "phase_field")
    runs = {}
    for fmt in ("h5", "npz"):
        out = tmp_path / ("out_" + fmt)
        out.mkdir()
        env = dict(os.environ)
        if fmt == "npz":
            env["CUPF_OUTPUT_FORMAT"] = "npz"
        r = subprocess.run([exe, "line.py", "-s", "0", "-b", "110", "-l", "1", "-d", "0", "-o",
                            str(out)], cwd=tmp_path, capture_output=True, text=True, timeout=600,
                           env=env)
        assert r.returncode == 0, r.stderr + r.stdout
        files = sorted(os.listdir(out))
        assert len(files) == 1 and files[0].startswith("lineseed0_"), files
        assert files[0].endswith("." + fmt)
        runs[fmt] = H5File(str(out / files[0])) if fmt == "h5" else np.load(out / files[0])
    d, z = runs["h5"], runs["npz"]
    keys = ("x_coordinates", "y_coordinates", "z_coordinates", "angles", "r0", "z0", "x0",
            "top", "angle", "V", "fractions", "tip_y", "cross_sec", "extra_area",
            "total_area", "tip_final", "node_region")
    assert sorted(d.keys()) == sorted(keys) == sorted(z.files)
    for key in keys:
        assert d[key].dtype == z[key].dtype and np.array_equal(d[key], z[key]), key
    assert d["tip_y"].shape == (3,)
    assert d["total_area"].reshape(3, 10)[0].sum() > 0


def _nucleation_run(tmp_path, tag, n_flag, pre_mt):
    """A 3-D (non-line) nucleation run of the executable: a uniform melt cooling
    at 5e6 K/s (Temp.txt), nucleation density 1/um^3."""
    Lx = 2.48
    work = tmp_path / tag
    folder = work / "forcing" / "case0"
    preprocess.write_line_forcing(str(folder), Lx, Lx, 2 * Lx, num_grains=9, seed=0, G=1.0,
                                  R=0.05, z0=0.6, top=0.3, t_end=5e-7, nmax=1.0,
                                  cooling_rate=5e6)
    preprocess.write_input_file(str(work / "line.py"), Lx, nts=2, asp_ratio_zx=2.0, num_pf=8,
                                pre_mt=pre_mt)
    out = work / "out"
    out.mkdir()
    exe = os.path.join(ROOT, "cupf_b200", "phase_field")
    r = subprocess.run([exe, "line.py", "-s", "0", "-b", "110", "-n", str(n_flag), "-d", "0",
                        "-o", str(out)], cwd=work, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    files = sorted(os.listdir(out))
    assert len(files) == 1 and "Mixed_density1.000000_grains" in files[0], files
    return H5File(str(out / files[0])), files[0]


def test_phase_field_cli_liquid_start_nucleation(tmp_path, built):
    """-n 1 with preMt = 60: the liquid-start phase nucleates grains in an
    all-liquid domain (APTPhaseField.cu:779-816), their ids label the initial
    solid, and the main loop nucleates from the temperature table.  The draw is
    keyed on (seed, coarse cell, step), so a second run is identical."""
    d, name = _nucleation_run(tmp_path, "a", 1, 60)
    g2p, vol = d["grainToPF"], d["volume"]
    assert len(g2p) == len(vol) and len(g2p) > 0
    assert np.all(g2p > 9)            # every grain was nucleated (ids past num_theta)
    assert np.all(vol > 0)
    assert name.split("_grains")[1].startswith(str(len(np.unique(g2p))) + "_")
    d2, name2 = _nucleation_run(tmp_path, "b", 1, 60)
    assert name2 == name
    for k in d.keys():
        assert np.array_equal(d[k], d2[k]), k


def test_phase_field_cli_nucleation_from_temperature_table(tmp_path, built):
    """-n 2 without a liquid start: the initial solid keeps id 0 (no substrate
    ids outside the line configuration) and grains nucleate in the melt as the
    temperature table cools it (APTPhaseField.cu:866-870)."""
    d, _ = _nucleation_run(tmp_path, "c", 2, 0)
    g2p = d["grainToPF"]
    assert len(g2p) > 0 and np.all(g2p > 9)


def test_reference_main_runs_on_the_library(tmp_path, built):
    """The reference's own driver (3DgrainMPI/main.cpp, unmodified), compiled
    against the library's headers of the reference's names and linked to
    libcupf.so (oracle/_ref/ref_main_on_cupf, built where the reference tree
    exists), runs the line case and writes the same file, dataset for dataset,
    as the library's phase_field."""
    ref_exe = os.path.join(ROOT, "oracle", "_ref", "ref_main_on_cupf")
    if not os.path.exists(ref_exe):
        pytest.skip("reference main not built")
    Lx = 2.48
    folder = tmp_path / "forcing" / "case0"
    preprocess.write_line_forcing(str(folder), Lx, Lx, 2 * Lx, num_grains=10, seed=0, G=1.0,
                                  R=0.05, z0=0.6, top=0.3, t_end=5e-7)
    preprocess.write_input_file(str(tmp_path / "line.py"), Lx, nts=2, asp_ratio_zx=2.0,
                                moving_ratio=1.0, num_pf=8)
    outs = []
    for exe in (os.path.join(ROOT, "cupf_b200", "phase_field"), ref_exe):
        out = tmp_path / ("out_" + os.path.basename(exe))
        out.mkdir()
        r = subprocess.run([exe, "line.py", "-s", "0", "-b", "110", "-l", "1", "-o", str(out)],
                           cwd=tmp_path, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr + r.stdout
        assert "cupf PhaseField" not in r.stderr, r.stderr
        files = sorted(os.listdir(out))
        assert len(files) == 1 and files[0].endswith(".h5"), files
        outs.append((files[0], H5File(str(out / files[0]))))
    (na, a), (nb, b) = outs
    assert na == nb
    assert a.keys() == b.keys() and "tip_y" in a.keys()
    for k in a.keys():
        assert np.array_equal(a[k], b[k]), k
