"""The phase_field executable runs a line configuration end to end on a B200:
forcing folder + input file in, QoI archive out with the reference's dataset
names (PhaseFieldCpu.cpp:493-519, QOI.cpp:19-34)."""
import os
import subprocess

import numpy as np
import pytest

from cupf_b200 import preprocess

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_phase_field_cli_line_run(tmp_path, built):
    Lx = 2.48
    folder = tmp_path / "forcing" / "case0"
    preprocess.write_line_forcing(str(folder), Lx, Lx, 2 * Lx, num_grains=10, seed=0, G=1.0,
                                  R=0.05, z0=0.6, top=0.3, t_end=5e-7)
    preprocess.write_input_file(str(tmp_path / "line.py"), Lx, nts=2, asp_ratio_zx=2.0,
                                moving_ratio=1.0, num_pf=8)
    out = tmp_path / "out"
    out.mkdir()
    exe = os.path.join(ROOT, "cupf_b200", "phase_field")
    r = subprocess.run([exe, "line.py", "-s", "0", "-b", "110", "-l", "1", "-d", "0", "-o", str(out)],
                       cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    files = sorted(os.listdir(out))
    assert len(files) == 1 and files[0].startswith("lineseed0_") and files[0].endswith(".npz")
    d = np.load(out / files[0])
    for key in ("x_coordinates", "y_coordinates", "z_coordinates", "angles", "r0", "z0", "x0",
                "top", "angle", "V", "fractions", "tip_y", "cross_sec", "extra_area",
                "total_area", "tip_final", "node_region"):
        assert key in d.files, key
    assert d["tip_y"].shape == (3,)
    assert d["total_area"].reshape(3, 10)[0].sum() > 0
