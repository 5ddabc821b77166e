"""The reference's own templates on the B200 field: the overlay
(lqcd-dwf-hmc_b200/overlay/lib_alt_B200: AField<REAL, B200> and
AFopr_Domainwall_5din_eo<AField<REAL, B200>> registered as
"Domainwall_5din_eo") compiled against the reference sources with the
reference corelib by lqcd-dwf-hmc_b200/overlay/Makefile into
oracle/_ref/overlay/overlay_check, which runs

* AFopr<AField<double,B200>>::New("Domainwall_5din_eo") mult / mult_dag,
* ASolver<AField<double,B200>>::New("CG") (src/lib_alt/Solver/asolver_CG-tmpl.h),
* AShiftsolver_CG<AField<double,B200>, AFopr<...>> (src/lib/Solver/ashiftsolver_CG-tmpl.h),
* Fprop_alt_Standard_eo_Richardson<AField<double,B200>, AField<float,B200>>
  ::invert_DdagD_even (FP64 Richardson over the FP32 inner CG,
  src/lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson-tmpl.h)

on the device, checked against the CPU oracle."""
import os
import subprocess

import numpy as np
import pytest

from b200dwf import synth

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
BIN = os.path.join(REPO, "oracle", "_ref", "overlay", "overlay_check")

CASES = {
    "shamir": ([4, 4, 4, 8], 8, 0.04, 1.8, 1.0, 0.0, (1, 1, 1, -1), "hot"),
    "mobius": ([8, 4, 4, 4], 12, 0.02, 1.0, 1.5, 0.5, (1, -1, 1, -1), "near"),
}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run(tmp_path, case, cmd, **extra):
    lat, ls, mq, m0, b, c, bc, kind = CASES[case]
    u = synth.gauge_field(lat, 51, kind)
    src = synth.spinor_field(lat, ls, 52)
    u.tofile(tmp_path / "gauge.bin")
    src.tofile(tmp_path / "src.bin")
    lines = ["lattice %s" % " ".join(map(str, lat)), "Ls %d" % ls, "mq %r" % mq, "M0 %r" % m0,
             "b %r" % b, "c %r" % c, "bc %s" % " ".join(map(str, bc)), "cmd %s" % cmd, "threads 2"]
    for k, v in extra.items():
        lines.append("%s %s" % (k, " ".join(map(str, v)) if isinstance(v, (list, tuple)) else v))
    (tmp_path / "params.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([BIN, str(tmp_path / "params.txt"), str(tmp_path), str(tmp_path)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    info = {}
    if (tmp_path / "info.txt").exists():
        for line in (tmp_path / "info.txt").read_text().splitlines():
            k, v = line.split()
            info[k] = float(v)
    from oracle.oracle import OracleDWF
    ora = OracleDWF(lat, ls, mq, m0, b, c, 1.0, bc)
    ora.set_links(u)
    return ora, src, info


def test_overlay_binary_is_built():
    """The overlay driver exists and links this repository's library."""
    assert os.path.exists(BIN), "oracle/_ref/overlay/overlay_check not built (make -C lqcd-dwf-hmc_b200/overlay)"
    out = subprocess.run(["ldd", BIN], capture_output=True, text=True).stdout
    assert "libb200dwf.so" in out and "not found" not in out.split("libb200dwf.so")[1].splitlines()[0]


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_factory_operator_modes(tmp_path, case):
    modes = ["Deo", "dag_Deo", "Doe", "D", "dag_D", "DdagD", "H", "Dee_inv"]
    ora, src, _ = run(tmp_path, case, "modes", modes=modes)
    for m in modes:
        got = np.fromfile(tmp_path / (m + ".bin"))
        dag = m.startswith("dag_")
        ref = ora.mult(m[4:] if dag else m, src, dag)
        assert rel(got, ref) < 1e-13, (case, m, rel(got, ref))


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_asolver_cg(tmp_path, case):
    ora, src, info = run(tmp_path, case, "cg", tol=1e-24, maxiter=5000)
    x = np.fromfile(tmp_path / "cg_x.bin")
    xr, nr, _, rcr = ora.cg(src, 1e-24, 5000)
    assert rcr == 0
    assert abs(info["nconv"] - nr) <= 2, (info, nr)
    assert rel(x, xr) < 1e-10
    assert rel(ora.mult("DdagD", x), src) < 1e-11


@pytest.mark.gpu
def test_reference_ashiftsolver_cg(tmp_path):
    sigma = [0.01, 0.1, 1.0]
    ora, src, info = run(tmp_path, "shamir", "shiftcg", tol=1e-24, maxiter=5000, sigma=sigma)
    xr, nr, _, rcr = ora.shiftcg(src, sigma, 1e-24, 5000)
    assert rcr == 0
    for i in range(len(sigma)):
        x = np.fromfile(tmp_path / ("shift_%d.bin" % i))
        assert rel(x, xr[i]) < 1e-10, (i, rel(x, xr[i]))
    assert abs(info["nconv"] - nr) <= 2


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_fprop_mixed_richardson(tmp_path, case):
    ora, src, info = run(tmp_path, case, "fprop", tol=1e-24, maxiter=1000)
    x = np.fromfile(tmp_path / "fprop_x.bin")
    assert rel(ora.mult("DdagD", x), src) < 1e-11
    xr, _, _, _ = ora.cg(src, 1e-24, 5000)
    assert rel(x, xr) < 1e-9
