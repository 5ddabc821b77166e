"""The C++ shells of include/b200dwf.hpp (AFopr / AField / ASolver_CG /
AShiftsolver_CG stand-ins): they compile against the header on any machine,
and on a GPU the compiled driver's DdagD, CG and multishift results match the
CPU oracle (itself pinned to the reference corelib)."""
import os
import subprocess

import numpy as np
import pytest

from b200dwf import synth

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "shell_check.cpp")
LIBDIR = os.path.join(REPO, "lqcd-dwf-hmc_b200")
CUDA = "/usr/local/cuda"


def compile_shell(out):
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(REPO, "include"), "-I", CUDA + "/include",
           SRC, "-o", out, "-L", LIBDIR, "-lb200dwf", "-L", CUDA + "/lib64", "-lcudart",
           "-Wl,-rpath," + LIBDIR, "-Wl,-rpath," + CUDA + "/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_shell_compiles(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libb200dwf.so")):
        pytest.skip("library not built")
    compile_shell(str(tmp_path / "shell_check"))
    assert (tmp_path / "shell_check").exists()


@pytest.mark.gpu
def test_shell_matches_oracle(tmp_path):
    from oracle.oracle import OracleDWF
    lat, ls, mq, m0 = [4, 4, 4, 8], 8, 0.05, 1.8
    exe = str(tmp_path / "shell_check")
    compile_shell(exe)
    u = synth.gauge_field(lat, 910, "hot")
    b = synth.spinor_field(lat, ls, 911)
    (tmp_path / "params.txt").write_text("%d %d %d %d %d %r %r\n" % (*lat, ls, mq, m0))
    u.tofile(str(tmp_path / "gauge.bin"))
    b.tofile(str(tmp_path / "src.bin"))
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ora = OracleDWF(lat, ls, mq, m0)
    ora.set_links(u)
    n = b.size

    def load(name):
        return np.fromfile(str(tmp_path / name), dtype=np.float64, count=n)

    ref = ora.mult("DdagD", b)
    assert np.linalg.norm(load("ddagd.bin") - ref) <= 1e-13 * np.linalg.norm(ref)
    x_ref = ora.cg(b, 1e-24, 10000)[0]
    assert np.linalg.norm(load("cg.bin") - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    xs_ref = ora.shiftcg(b, [0.05, 0.2, 1.0], 1e-24, 10000)[0]
    assert np.linalg.norm(load("shift1.bin") - xs_ref[1]) <= 1e-8 * np.linalg.norm(xs_ref[1])
