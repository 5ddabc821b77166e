"""Generate the golden fixtures in this directory from the reference itself.

Runs ``oracle/_ref/ref_harness`` (the reference Bridge++ corelib CPU path,
built from the reference sources by ``make -f oracle/Makefile.ref``) on seeded
synthetic inputs and stores its outputs.  Inputs are not stored: they are
regenerated bit-for-bit from the recorded seeds by ``b200dwf.synth``.

    python tests/golden/make_golden.py            # operator, solver, force ...
    python tests/golden/make_golden.py traj       # one 2+1-flavour trajectory
    python tests/golden/make_golden.py rng        # the Mseries_parallel generator
    python tests/golden/make_golden.py io         # gauge-configuration files
    python tests/golden/make_golden.py sample [REF]   # the published 8^4 trajectory

Needs the reference tree (to build the harness); the committed .npz files are
what the tests read, so the tests themselves run without it.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "lqcd-dwf-hmc_b200"))
from b200dwf import synth  # noqa: E402

HARNESS = os.path.join(REPO, "oracle", "_ref", "ref_harness")

# Operator cases.  Ls=4 keeps every fixture small while exercising the s=0
# wall, the bulk and the s=Ls-1 wall of M5 and of the LU factors.
CASES = {
    "shamir": dict(lattice=[4, 4, 4, 4], Ls=4, mq=0.01, M0=1.8, b=1.0, c=0.0,
                   alpha=1.0, bc=[1, 1, 1, -1], gauge=("hot", 11), src=12,
                   modes=["Deo", "Doe", "dag_Deo", "dag_Doe", "Dee", "dag_Dee",
                          "Dee_inv", "dag_Dee_inv", "D", "dag_D", "DdagD",
                          "H", "dag_H", "gm5R", "R"]),
    "mobius_alpha": dict(lattice=[4, 4, 4, 4], Ls=4, mq=0.02, M0=1.0, b=1.5,
                         c=0.5, alpha=1.3, bc=[1, -1, 1, -1],
                         gauge=("near", 21), src=22,
                         modes=["Deo", "dag_Deo", "Dee", "dag_Dee", "Dee_inv",
                                "dag_Dee_inv", "DdagD", "H"]),
}
SOLVE = dict(case="shamir", tol=1e-24, sigma=[0.05, 0.2, 1.0], maxiter=5000)
# stout smearing (rho, 2 levels) and its Jacobian chain on a random force
SMEAR = dict(lattice=[4, 4, 4, 4], Ls=4, mq=0.01, M0=1.8, b=1.0, c=0.0, alpha=1.0,
             bc=[1, 1, 1, -1], gauge=("near", 71), src=72, rho=0.1, nsmear=2, sigma=73)
# Iwasaki (rectangle) gauge force, gauge Hamiltonian and the link update
# W = exp(alpha iP) U (Taylor order nprec + reunitarisation), non-cubic lattice
GAUGE = dict(lattice=[4, 6, 4, 8], Ls=4, mq=0.01, M0=1.8, b=1.0, c=0.0, alpha=1.0,
             bc=[1, 1, 1, -1], gauge=("near", 81), src=82, beta=2.13, c_plaq=3.648,
             c_rect=-0.331, step=0.1, nprec=8, mom=83)
# force: Moebius (alpha must be 1 for Force_F_Domainwall_eo), antiperiodic t
FORCE = dict(lattice=[4, 4, 4, 4], Ls=4, mq=0.02, M0=1.4, b=1.5, c=0.5, alpha=1.0,
             bc=[1, 1, 1, -1], gauge=("near", 31), src=32, src2=33)
# one 2+1-flavour trajectory of the benchmark driver's action set on the
# 4^3x8 Ls=8 Shamir hot start: light 0.01 over Hasenbusch 0.1 over PV 1.0,
# strange 0.04 as a PV rational ratio with 10-pole approximations, Iwasaki
# beta 2.13, 2 stout levels rho 0.1, Omelyan [2,1,3], length 1.  The momenta
# and pseudofermion noise of the reference's M-series generator (seed
# 1234567) are stored with the results.
TRAJ = dict(lattice=[4, 4, 4, 8], Ls=8, mq=0.01, M0=1.8, b=1.0, c=0.0, alpha=1.0,
            bc=[1, 1, 1, -1], gauge=("hot", 101), src=102,
            mq_l=0.01, mq_h=0.1, mq_s=0.04, mq_pv=1.0, beta=2.13, c_plaq=3.648,
            c_rect=-0.331, rho=0.1, nsmear=2, tau=1.0, nstep=[2, 1, 3], level=[0, 0, 1, 2],
            integrator="Omelyan", lambda_=0.1931833275, nprec=8, np_md=10, np_h=10,
            rat_lo=0.01, rat_hi=3.16227766, tol_md=1e-24, tol_h=1e-24, seed=1234567)


def write_params(path, case, extra=None):
    with open(path, "w") as f:
        f.write("lattice %s\n" % " ".join(map(str, case["lattice"])))
        for k in ("Ls", "mq", "M0", "b", "c", "alpha"):
            f.write("%s %r\n" % (k, case[k]))
        f.write("bc %s\n" % " ".join(map(str, case["bc"])))
        for k, v in (extra or {}).items():
            if isinstance(v, (list, tuple)):
                f.write("%s %s\n" % (k, " ".join(map(repr, v))))
            else:
                f.write("%s %s\n" % (k, v))


def inputs(case):
    kind, gseed = case["gauge"]
    u = synth.gauge_field(case["lattice"], gseed, kind)
    src = synth.spinor_field(case["lattice"], case["Ls"], case["src"])
    return u, src


def run(cmd, case, extra, tmp):
    u, src = inputs(case)
    u.tofile(os.path.join(tmp, "gauge.bin"))
    src.tofile(os.path.join(tmp, "src.bin"))
    write_params(os.path.join(tmp, "params.txt"), case, extra)
    subprocess.run([HARNESS, cmd, os.path.join(tmp, "params.txt"), tmp, tmp],
                   check=True, stdout=subprocess.DEVNULL)


def traj():
    import shutil
    from b200dwf.rational import TABLE_DIR
    keys = ("mq_l", "mq_h", "mq_s", "mq_pv", "beta", "c_plaq", "c_rect", "rho", "nsmear",
            "tau", "nstep", "level", "integrator", "nprec", "np_md", "np_h", "rat_lo",
            "rat_hi", "tol_md", "tol_h", "seed")
    extra = {k: TRAJ[k] for k in keys}
    extra["lambda"] = TRAJ["lambda_"]
    with tempfile.TemporaryDirectory() as tmp:
        for name in os.listdir(TABLE_DIR):
            shutil.copy(os.path.join(TABLE_DIR, name), tmp)
        run("traj", TRAJ, extra, tmp)
        out = {k: np.fromfile(os.path.join(tmp, k + ".bin"))
               for k in ("mom", "xi_0", "xi_1", "xi_2", "u_end", "mom_end",
                         "force_0", "force_1", "force_2", "force_3")}
        for line in open(os.path.join(tmp, "traj.txt")):
            key, *vals = line.split()
            out[key] = np.array([float(v) for v in vals])
    np.savez_compressed(os.path.join(HERE, "traj_nf2p1.npz"), meta=json.dumps(TRAJ), **out)
    print("wrote traj_nf2p1.npz: H0 %.10f dH %.10f" % (out["H0"][0], out["dH"][0]))


# the benchmark driver's generator (Mseries_parallel): a non-cubic lattice so
# that x, y, z and t cannot be confused
RNG = dict(lattice=[4, 6, 2, 4], Ls=4, seed=1234567)


def mseries_rng():
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "params.txt"), "w") as f:
            f.write("lattice %s\nLs %d\nseed %d\n"
                    % (" ".join(map(str, RNG["lattice"])), RNG["Ls"], RNG["seed"]))
        subprocess.run([HARNESS, "rng", os.path.join(tmp, "params.txt"), tmp, tmp],
                       check=True, stdout=subprocess.DEVNULL)
        out = {k: np.fromfile(os.path.join(tmp, k + ".bin")) for k in ("u", "h", "x", "h2")}
    np.savez_compressed(os.path.join(HERE, "mseries_parallel.npz"), meta=json.dumps(RNG), **out)
    print("wrote mseries_parallel.npz")


# gauge-configuration files: a synthetic 4x4x4x8 text configuration (hot
# links, seed 77, one "%.14e" number per line as the reference's
# conf_04040408.txt) read by the reference onto 8x4x4x8 and written as Binary
IO = dict(text_lattice=[4, 4, 4, 8], lattice=[8, 4, 4, 8], gauge=("hot", 77), fmt="%.14e")


def io_text(case):
    kind, seed = case["gauge"]
    u = synth.gauge_field(case["text_lattice"], seed, kind)
    n = int(np.prod(case["text_lattice"]))
    t = u.reshape(4, n, 18).transpose(1, 0, 2).reshape(-1)
    return "".join((case["fmt"] + "\n") % v for v in t)


def gauge_io():
    import hashlib
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "conf.txt"), "w") as f:
            f.write(io_text(IO))
        with open(os.path.join(tmp, "params.txt"), "w") as f:
            f.write("lattice %s\n" % " ".join(map(str, IO["lattice"])))
        subprocess.run([HARNESS, "io", os.path.join(tmp, "params.txt"), tmp, tmp],
                       check=True, stdout=subprocess.DEVNULL)
        digest = {}
        for name in ("text_read.bin", "conf.bin", "bin_read.bin"):
            with open(os.path.join(tmp, name), "rb") as f:
                digest[name] = hashlib.sha256(f.read()).hexdigest()
    np.savez_compressed(os.path.join(HERE, "gauge_io.npz"), meta=json.dumps(IO),
                        digest=json.dumps(digest))
    print("wrote gauge_io.npz")


# The reference's published single-GPU trajectory (sample_1gpu/): 8^4 lattice
# from conf_04040408.txt tiled, Moebius DWF b=1.5 c=0.5 M0=1.0 Ls=12, masses
# Nf1 0.02 (rational), Nf2 0.0005 over Nf2_prec 0.002 over PV 1.0, tree-level
# Symanzik beta 4.17, 3 stout steps rho 0.1, Omelyan [2,1,3] on levels
# [0,0,1,2], length 0.1, Mseries_parallel reset to i_conf = 200000, solver
# tolerances |r|^2/|b|^2 1e-28 (CG), 1e-26 / 1e-28 (MD / calcH multishift),
# shipped 16- and 24-pole tables on [1e-4, 10]
# (sample_1gpu/HMC_DWF_Nf2p1_eo.yaml, main.yaml).  Stored: the configuration
# file's numbers, the table files' text, and the published log values with
# the log line each comes from.
SAMPLE = dict(lattice=[8, 8, 8, 8], Ls=12, M0=1.0, b=1.5, c=0.5, mq_l=0.0005, mq_h=0.002,
              mq_s=0.02, mq_pv=1.0, beta=4.17, c_plaq=5.0 / 3.0, c_rect=-1.0 / 12.0, rho=0.1,
              nsmear=3, nstep=[2, 1, 3], level=[0, 0, 1, 2], tau=0.1, lam=0.1931833275, nprec=8,
              np_md=16, np_h=24, rat_lo=1.0e-2, rat_hi=3.16227766, tol_cg=1e-28,
              tol_ms_md=1e-26, tol_ms_h=1e-28, seed=200000)
SAMPLE_TABLES = ["parameter_rational.%s_%d_0.00010000_010.000" % (k, n)
                 for n in (16, 24) for k in ("1_4", "1_4inv", "1_2inv")]
# (key, log file, label printed in the log, occurrence)
SAMPLE_LOG = [("H_total_init", "sample_1gpu/run.log", "H_total(init)", 0),
              ("H_Frational_init", "sample_1gpu/run.log", "H_Frational", 0),
              ("H_Fratio_Nf2_init", "sample_1gpu/run.log", "H_Fratio", 0),
              ("H_Fratio_Nf2prec_init", "sample_1gpu/run.log", "H_Fratio", 2),
              ("H_Grectangle_init", "sample_1gpu/run.log", "H_Grectangle", 0),
              ("plaq_init", "sample_1gpu/run.log", "plaq(init)", 0),
              ("H_total_final", "sample_1gpu/run.log", "H_total(trial)", 0),
              ("H_diff", "sample_1gpu/run.log", "H(diff)", 0),
              ("plaq_final", "sample_1gpu/run.log", "plaq(final)", 0),
              ("H_total_init_corelib", "sample_x86_corelib/run.log", "H_total(init)", 0),
              ("H_total_final_corelib", "sample_x86_corelib/run.log", "H_total(trial)", 0),
              ("H_total_init_qxs", "sample_x86/run.log", "H_total(init)", 0),
              ("H_total_final_qxs", "sample_x86/run.log", "H_total(trial)", 0)]


def sample(ref):
    import re
    vals = np.loadtxt(os.path.join(ref, "conf_04040408.txt"), dtype=np.float64)
    tables = {}
    for name in SAMPLE_TABLES:
        with open(os.path.join(ref, "sample_1gpu", name)) as f:
            tables[name] = f.read()
    published, where = {}, {}
    for key, log, label, nth in SAMPLE_LOG:
        hits = []
        with open(os.path.join(ref, log)) as f:
            for i, line in enumerate(f, 1):
                m = re.match(r"\s*%s\s*=\s*([-+0-9.eE]+)" % re.escape(label), line)
                if m:
                    hits.append((float(m.group(1)), i))
        published[key], line_no = hits[nth]
        where[key] = "%s:%d" % (log, line_no)
    with open(os.path.join(ref, "sample_1gpu", "run.log")) as f:
        for i, line in enumerate(f, 1):
            m = re.match(r"Elapsed time: each trajectory: total\s+([0-9.]+) sec", line)
            if m:
                published["sec_per_trajectory"] = float(m.group(1))
                where["sec_per_trajectory"] = "sample_1gpu/run.log:%d" % i
    np.savez_compressed(os.path.join(HERE, "sample_8x8x8x8.npz"), meta=json.dumps(SAMPLE),
                        conf_04040408=vals, tables=json.dumps(tables),
                        published=json.dumps(published), where=json.dumps(where))
    print("wrote sample_8x8x8x8.npz", published)


def main():
    if sys.argv[1:2] == ["sample"]:
        ref = sys.argv[2] if len(sys.argv) > 2 else os.environ.get("B200_REFERENCE_DIR", "/root/reference")
        sample(ref)
        return
    if sys.argv[1:] == ["io"]:
        gauge_io()
        return
    if sys.argv[1:] == ["traj"]:
        traj()
        return
    if sys.argv[1:] == ["rng"]:
        mseries_rng()
        return
    for name, case in CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            run("modes", case, {"modes": " ".join(case["modes"])}, tmp)
            out = {m: np.fromfile(os.path.join(tmp, m + ".bin")) for m in case["modes"]}
        meta = {k: v for k, v in case.items() if k != "modes"}
        meta["modes"] = case["modes"]
        np.savez_compressed(os.path.join(HERE, "dwf_%s.npz" % name),
                            meta=json.dumps(meta), **out)
        print("wrote dwf_%s.npz" % name)

    case = CASES[SOLVE["case"]]
    with tempfile.TemporaryDirectory() as tmp:
        run("cg", case, {"tol": SOLVE["tol"], "maxiter": SOLVE["maxiter"]}, tmp)
        x = np.fromfile(os.path.join(tmp, "cg_x.bin"))
        info = open(os.path.join(tmp, "cg_info.txt")).read()
        run("shiftcg", case, {"tol": SOLVE["tol"], "maxiter": SOLVE["maxiter"],
                              "sigma": SOLVE["sigma"]}, tmp)
        xs = [np.fromfile(os.path.join(tmp, "shift_%d.bin" % i))
              for i in range(len(SOLVE["sigma"]))]
        sinfo = open(os.path.join(tmp, "shift_info.txt")).read()
    meta = dict(SOLVE, cg_info=info, shift_info=sinfo)
    with tempfile.TemporaryDirectory() as tmp:
        synth.spinor_field(FORCE["lattice"], FORCE["Ls"], FORCE["src2"]).tofile(
            os.path.join(tmp, "src2.bin"))
        run("force", FORCE, {}, tmp)
        forces = {k: np.fromfile(os.path.join(tmp, "force_%s.bin" % k))
                  for k in ("H", "Hdag", "udiv")}
    np.savez_compressed(os.path.join(HERE, "force_mobius.npz"), meta=json.dumps(FORCE),
                        **forces)
    print("wrote force_mobius.npz")
    with tempfile.TemporaryDirectory() as tmp:
        rng = np.random.default_rng(SMEAR["sigma"])
        rng.standard_normal(18 * 4 * int(np.prod(SMEAR["lattice"]))).tofile(
            os.path.join(tmp, "sigma.bin"))
        run("smear", SMEAR, {"rho": SMEAR["rho"], "nsmear": SMEAR["nsmear"]}, tmp)
        out = {"smear_%d" % i: np.fromfile(os.path.join(tmp, "smear_%d.bin" % i))
               for i in range(1, SMEAR["nsmear"] + 1)}
        out["jacobian"] = np.fromfile(os.path.join(tmp, "jacobian.bin"))
    np.savez_compressed(os.path.join(HERE, "smear_stout.npz"), meta=json.dumps(SMEAR), **out)
    print("wrote smear_stout.npz")
    with tempfile.TemporaryDirectory() as tmp:
        synth.algebra_field(GAUGE["lattice"], GAUGE["mom"]).tofile(os.path.join(tmp, "mom.bin"))
        run("gauge", GAUGE, {"beta": GAUGE["beta"], "c_plaq": GAUGE["c_plaq"],
                             "c_rect": GAUGE["c_rect"], "alpha": GAUGE["step"],
                             "nprec": GAUGE["nprec"]}, tmp)
        out = {"gforce": np.fromfile(os.path.join(tmp, "gforce.bin")),
               "update": np.fromfile(os.path.join(tmp, "update.bin")),
               "H": np.array(float(open(os.path.join(tmp, "gauge_H.txt")).read()))}
    np.savez_compressed(os.path.join(HERE, "gauge_rect.npz"), meta=json.dumps(GAUGE), **out)
    print("wrote gauge_rect.npz")
    np.savez_compressed(os.path.join(HERE, "solve_shamir.npz"),
                        meta=json.dumps(meta), cg_x=x,
                        **{"shift_%d" % i: v for i, v in enumerate(xs)})
    print("wrote solve_shamir.npz", info.strip().replace("\n", " "),
          sinfo.strip().replace("\n", " "))
    traj()


if __name__ == "__main__":
    main()
