"""The reference's own mixed-precision solver on the CPU (the QXS backend,
built from the reference's sources by oracle/Makefile.qxs): the harness the
bench times as the mixed-precision CPU baseline runs its operators and a
bounded Fprop_alt_Standard_eo_Richardson solve on a small lattice (Nx / 2 a
multiple of the backend's x vector length, 4)."""
import os
import subprocess

import numpy as np
import pytest

from b200dwf import synth

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "..", "oracle", "_ref", "qxs", "qxs_harness")


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="oracle/_ref/qxs not built here")
def test_qxs_mixed_solver_runs(tmp_path):
    lat, ls = [8, 8, 4, 4], 4
    synth.gauge_field(lat, 5, "near", eps=0.3).tofile(tmp_path / "gauge.bin")
    synth.spinor_field(lat, ls, 6).tofile(tmp_path / "src.bin")
    (tmp_path / "params.txt").write_text("lattice 8 8 4 4\nLs 4\nmq 0.05\nM0 1.8\nthreads 2\nreps 1\n")
    r = subprocess.run([HARNESS, str(tmp_path / "params.txt"), str(tmp_path)],
                       capture_output=True, text=True, timeout=120, check=True)
    got = dict(line.split() for line in r.stdout.splitlines()
               if len(line.split()) == 2 and line.split()[0].endswith("seconds"))
    for key in ("ddagd_f64_seconds", "ddagd_f32_seconds", "solve_1x1_seconds"):
        assert np.isfinite(float(got[key])) and float(got[key]) > 0.0, key
