#!/usr/bin/env python
"""Benchmark of the B200 even/odd domain-wall hot path.

Workload (the lattice the metric is quoted on): 24^3x48, Ls=16, Shamir DWF
M0=1.8, m=0.01, seeded near-unit SU(3) links exp(i*0.3*H) followed by 2 stout
steps rho=0.1 (smeared on the device by the library's stout kernels), Gaussian
RHS, FP64.

A step is one even/odd Dslash apply and its dagger through the reference
operator interface: mult(v, w, "Deo") then mult_dag(v', w, "Deo").  Its
algorithmic traffic is the fused D_eo byte count per 4D half-site
    B = Ls*24*(8 + 8) + 8*18*8 = 7296 bytes  (Ls=16, FP64, 18-real links)
counted once per apply (two applies per step); one apply at 24^3x48
(Vh = 331,776) is 2.42 GB, more than L2.

The JSON line also carries the dominant kernel's roofline (the fused hop
kernel timed alone with CUDA events), an end-to-end number through the C ABI
with host buffers, the 2+1-flavour trajectory on the same lattice in its
three forms (plain FP64, mixed+batched, mixed+batched+learned) as short
top-level keys, the solver timings, and the reference corelib CPU path timed
on this host as the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import gc
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "lqcd-dwf-hmc_b200"))

LATTICE = [24, 24, 24, 48]
LEARN_LATTICE = [16, 16, 16, 32]   # the learned preconditioner's configuration
LS = 16
MQ, M0 = 0.01, 1.8
MS = 0.04                   # strange-quark mass of the 2+1-flavour trajectory
SEED_U, SEED_B = 1234567, 7654321
BYTES_PER_HALF_SITE = LS * 24 * (8 + 8) + 8 * 18 * 8
# flops of one fused D_eo per 4D half-site: the reference's count for the
# Wilson hop and the M5 pre-factor on every slice, halved for one parity
# (afopr_Domainwall_5din_eo-tmpl.h:1445-1448, 1476, 1492)
FLOPS_PER_HALF_SITE = 1488 * LS
REF_HARNESS = os.path.join(REPO, "oracle", "_ref", "ref_harness")
WORKLOAD = "dwf_eo_dslash_24x24x24x48_Ls16_f64"
METRIC = "sec/trajectory 24^3x48 Ls=16: mixed+learned vs plain FP64 on B200; Dslash GB/s"
VALUE_IS = "Dslash HBM GB/s: D_eo + D_eo^dag, FP64, algorithmic bytes / device time"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cg", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-solvers", action="store_true",
                    help="skip the mixed-precision Richardson and multishift timings")
    ap.add_argument("--lattice", type=int, nargs=4, default=LATTICE)
    ap.add_argument("--no-learned", action="store_true",
                    help="skip training and timing the learned preconditioner")
    ap.add_argument("--no-trajectory", action="store_true",
                    help="skip the molecular-dynamics trajectory timing")
    ap.add_argument("--traj-nstep", type=int, nargs=3, default=[2, 1, 3],
                    help="Omelyan steps per level (rational + light ratio, Hasenbusch, gauge)")
    ap.add_argument("--traj-length", type=float, default=0.1,
                    help="trajectory length (0.1 as in the reference's published runs)")
    ap.add_argument("--traj-all-forms", action="store_true",
                    help="also time FP64 CG with the windowed multishift")
    ap.add_argument("--traj-lattice", type=int, nargs=4, default=[24, 24, 24, 48],
                    help="lattice of the 2+1-flavour trajectory timing")
    ap.add_argument("--traj-ls", type=int, default=LS, help="Ls of the trajectory timing")
    ap.add_argument("--traj-mass-l", type=float, default=MQ,
                    help="light quark mass of the trajectory timing")
    ap.add_argument("--traj-inner", default="f16", choices=["f32", "f16", "bf16"],
                    help="storage of the mixed-precision Richardson's inner solve")
    ap.add_argument("--traj-np-h", type=int, default=24,
                    help="poles of the heatbath and Hamiltonian rationals (16 or 24)")
    ap.add_argument("--traj-window", type=int, default=16,
                    help="residual window of the batched forms' multishift")
    ap.add_argument("--traj-chrono", type=int, default=4,
                    help="MD solves of the mixed forms start from the minimal residual "
                         "extrapolation of this many previous solutions (1: the previous one; "
                         "each more costs one FP64 field per solver)")
    ap.add_argument("--traj-force-pool", default="paired", choices=["paired", "streamed"],
                    help="the rational force's solution fields: two sets side by side, or "
                         "one set at a time (np_md fewer fields, one more multishift)")
    ap.add_argument("--traj-seed", type=int, default=SEED_U + 11,
                    help="seed of the driver's generator (Mseries_parallel) for the trajectory; "
                         "(seed + 1) * Lz * Lt must stay below 2^31")
    ap.add_argument("--traj-only", action="store_true",
                    help="time only the trajectory forms (a fresh process holds only their "
                         "fields) and print their JSON; not the benchmark line")
    ap.add_argument("--traj-forms", nargs="+", default=["fp64_plain", "mixed_batched"],
                    help="trajectory forms to time (add mixed_batched_learned for the learned "
                         "light solves; about 5 minutes more at 24^3x48)")
    return ap.parse_args()


def workload_inputs(lattice, ls, device_smear=False):
    """Seeded links exp(i*0.3*H) smeared by 2 stout steps rho=0.1, and the
    Gaussian RHS.  device_smear: the smearing runs in the library's stout
    kernels (equal to the numpy restatement to ~1e-14; used where the numpy
    form would take most of a minute, 24^3x48)."""
    from b200dwf import synth
    u = synth.gauge_field(lattice, SEED_U, "near", eps=0.3)
    if device_smear:
        import b200dwf
        sm = b200dwf.StoutSmear(lattice, 0.1, 2)
        sm.set_config(u)
        u = np.ascontiguousarray(sm.config(2))
        del sm
    else:
        u = synth.stout_smear(u, lattice, 0.1, 2)
    b = synth.spinor_field(lattice, ls, SEED_B)
    return u, b


def vh_of(lattice):
    return int(np.prod(lattice)) // 2


# kernel template of each FP64 hop variant (the autotuner's variant numbers)
HOP_KERNEL_OF_VARIANT = {0: "dwf_hop_kernel", 4: "dwf_hop_kernel", 1: "dwf_hop_tma_kernel",
                         2: "dwf_hop_tma_kernel", 3: "dwf_hop_tma_kernel", 7: "dwf_hop_tma_kernel"}


def dagger_hop_kernel(vh):
    """Name of the FP64 dagger-hop kernel the autotuner kept at this Vh
    (epilogue EPI_DDAGEO), from the library's tuning table."""
    import b200dwf
    for ln in b200dwf.tuning_table().splitlines():
        f = dict(kv.split("=", 1) for kv in ln.split())
        if (f.get("vh") == str(vh) and f.get("ls") == str(LS) and f.get("prec") == "f64"
                and f.get("epi") == "1" and f.get("fk") == "0"):
            v = int(f["variant"])
            return "%s<16,f64,EPI_DDAGEO> (mult_dag Deo, autotuned variant %d)" % (
                HOP_KERNEL_OF_VARIANT.get(v, "hop variant"), v)
    return "fused FP64 dagger hop (mult_dag Deo, EPI_DDAGEO)"


def read_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


TRAFFIC_PROFILE = os.path.join(REPO, "profiles", "hop_kernel_f64_16x16x16x32_Ls16.md")


def read_traffic(vh):
    """DRAM bytes per launch of the FP64 hop kernel: the committed ncu
    summary's capture (a 16^3x32 launch, small enough for a full capture),
    scaled to vh sites.  Each site reads its column, its 8 neighbours'
    columns (7 of them shared with other sites of the launch) and 8 links,
    and writes its column, so the traffic grows in proportion to the sites."""
    got = {}
    try:
        for line in open(TRAFFIC_PROFILE):
            for key in ("dram_bytes_per_launch:", "vh_per_launch:"):
                if line.startswith(key):
                    got[key] = float(line.split(":")[1])
    except OSError:
        return None
    if len(got) < 2:
        return None
    return got["dram_bytes_per_launch:"] * vh / got["vh_per_launch:"]


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        cmd = ["nvidia-smi", "-i", str(self.device),
               "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
               "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
               "clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "100"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thr = threading.Thread(target=self._read, daemon=True)
            self.thr.start()
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        time.sleep(0.15)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ reference (CPU) arm
def run_reference_cpu(lattice, ls, steps, warmup, budget_s=60.0, threads=None, inputs=None,
                      ddagd=False):
    """Time the reference corelib Fopr_Domainwall_eo (oracle/_ref, built from
    the reference sources) on this host: one step = mult(v,w,"Deo") +
    mult_dag(v,w,"Deo") on the same workload (inputs = (u, b) when the caller
    has them).  Returns a dict: GB/s, seconds/step, reps, threads, and with
    ddagd the seconds of one mult(v,w,"DdagD")."""
    if not os.path.exists(REF_HARNESS):
        raise RuntimeError("oracle/_ref/ref_harness not built")
    threads = threads or os.cpu_count() or 1
    u, b = inputs if inputs is not None else workload_inputs(lattice, ls)
    vh = vh_of(lattice)
    modes = "Deo dag_Deo" + (" DdagD" if ddagd else "")
    with tempfile.TemporaryDirectory() as d:
        u.tofile(os.path.join(d, "gauge.bin"))
        b.tofile(os.path.join(d, "src.bin"))

        def timed(reps, warm):
            with open(os.path.join(d, "params.txt"), "w") as f:
                f.write("lattice %s\nLs %d\nmq %r\nM0 %r\nthreads %d\nreps %d\nwarmup %d\n"
                        "modes %s\n"
                        % (" ".join(map(str, lattice)), ls, MQ, M0, threads, reps, warm, modes))
            r = subprocess.run([REF_HARNESS, "time", os.path.join(d, "params.txt"), d, d],
                               capture_output=True, text=True, check=True)
            t = {}
            for line in r.stdout.splitlines():
                p = line.split()
                if len(p) == 2 and p[0] in ("Deo", "dag_Deo", "DdagD"):
                    t[p[0]] = float(p[1])
            return t

        probe = timed(1, 0)
        per_rep = sum(probe.values())
        reps = int(max(1, min(steps, budget_s / max(per_rep, 1e-6))))
        t = timed(reps, max(0, min(warmup, 1)))
    t_step = t["Deo"] + t["dag_Deo"]
    out = {"gbs": 2 * BYTES_PER_HALF_SITE * vh / t_step / 1e9, "t_step": t_step, "reps": reps,
           "threads": threads}
    if ddagd:
        out["t_ddagd"] = t["DdagD"]
    return out


QXS_HARNESS = os.path.join(REPO, "oracle", "_ref", "qxs", "qxs_harness")


def run_reference_qxs_mixed(lattice, ls, inputs, threads=None):
    """The reference's own mixed-precision solver on this host's cores:
    Fprop_alt_Standard_eo_Richardson<AField<double,QXS>, AField<float,QXS>>
    (the QXS backend, compiled from the reference's sources by
    oracle/Makefile.qxs; FP64 Richardson, FP32 CG inner solves on DdagD) on
    the workload: one FP64 and one FP32 DdagD of its operators, and one
    bounded solve (1 outer x 1 inner iteration).  Returns the harness's
    figures."""
    if not os.path.exists(QXS_HARNESS):
        raise RuntimeError("oracle/_ref/qxs/qxs_harness not built")
    threads = threads or os.cpu_count() or 1
    u, b = inputs
    with tempfile.TemporaryDirectory() as d:
        u.tofile(os.path.join(d, "gauge.bin"))
        b.tofile(os.path.join(d, "src.bin"))
        with open(os.path.join(d, "params.txt"), "w") as f:
            f.write("lattice %s\nLs %d\nmq %r\nM0 %r\nb 1.0\nc 0.0\nbc 1 1 1 -1\nthreads %d\n"
                    "reps 1\n" % (" ".join(map(str, lattice)), ls, MQ, M0, threads))
        r = subprocess.run([QXS_HARNESS, os.path.join(d, "params.txt"), d],
                           capture_output=True, text=True, check=True)
    out = {}
    for line in r.stdout.splitlines():
        p = line.split()
        if len(p) == 2 and p[0] in ("ddagd_f64_seconds", "ddagd_f32_seconds", "solve_1x1_seconds",
                                    "threads"):
            out[p[0]] = float(p[1])
    return out


# The configuration the reference runs on its CPU path (4^3x8, Ls=8 Shamir
# M0=1.8, hot start, light 0.01 / Hasenbusch 0.1 / strange 0.04 / PV 1.0,
# Iwasaki beta 2.13, 2 stout rho 0.1, Omelyan [2,1,3], length 1, 10-pole
# rationals, solves to |r|^2/|b|^2 < 1e-24).
SMALL_TRAJ = dict(lattice=[4, 4, 4, 8], Ls=8, M0=1.8, gauge_seed=101, mq_l=0.01, mq_h=0.1,
                  mq_s=0.04, mq_pv=1.0, beta=2.13, c_plaq=3.648, c_rect=-0.331, rho=0.1,
                  nsmear=2, tau=1.0, nstep=[2, 1, 3], level=[0, 0, 1, 2],
                  lam=0.1931833275, nprec=8, np_md=10, np_h=10, rat_lo=0.01,
                  rat_hi=3.16227766, tol=1e-24, seed=1234567)


def small_trajectory_beside_reference(threads=None):
    """One 2+1-flavour trajectory of the reference corelib (oracle/_ref
    ref_harness traj, built from the reference sources) on this host's cores,
    and the same trajectory on the device driven by the momenta and noise the
    reference's generator handed out: both times and both H(diff)."""
    import shutil
    import torch
    from b200dwf import synth
    from b200dwf.hmc import build_dwf_nf2p1, HostNoise
    from b200dwf.rational import TABLE_DIR
    if not os.path.exists(REF_HARNESS):
        return {"unavailable": "oracle/_ref/ref_harness not built"}
    c = SMALL_TRAJ
    threads = threads or os.cpu_count() or 1
    u = synth.gauge_field(c["lattice"], c["gauge_seed"], "hot")
    with tempfile.TemporaryDirectory() as d:
        for name in os.listdir(TABLE_DIR):
            shutil.copy(os.path.join(TABLE_DIR, name), d)
        u.tofile(os.path.join(d, "gauge.bin"))
        with open(os.path.join(d, "params.txt"), "w") as f:
            f.write("lattice %s\nLs %d\nM0 %r\nb 1.0\nc 0.0\nalpha 1.0\nbc 1 1 1 -1\n"
                    % (" ".join(map(str, c["lattice"])), c["Ls"], c["M0"]))
            for k in ("mq_l", "mq_h", "mq_s", "mq_pv", "beta", "c_plaq", "c_rect", "rho",
                      "nsmear", "tau", "nprec", "np_md", "np_h", "rat_lo", "rat_hi", "seed"):
                f.write("%s %r\n" % (k, c[k]))
            f.write("nstep %s\nlevel %s\nlambda %r\ntol_md %r\ntol_h %r\nthreads %d\n"
                    % (" ".join(map(str, c["nstep"])), " ".join(map(str, c["level"])), c["lam"],
                       c["tol"], c["tol"], threads))
        t0 = time.perf_counter()
        subprocess.run([REF_HARNESS, "traj", os.path.join(d, "params.txt"), d, d],
                       capture_output=True, text=True, check=True)
        t_ref = time.perf_counter() - t0
        mom = np.fromfile(os.path.join(d, "mom.bin"))
        xis = [np.fromfile(os.path.join(d, "xi_%d.bin" % k)) for k in range(3)]
        ref = {}
        for line in open(os.path.join(d, "traj.txt")):
            key, *vals = line.split()
            ref[key] = [float(v) for v in vals]

    def device_run():
        hmc = build_dwf_nf2p1(c["lattice"], c["Ls"], c["M0"],
                              dict(l=c["mq_l"], h=c["mq_h"], s=c["mq_s"], pv=c["mq_pv"]),
                              c["beta"], c["c_plaq"], c["c_rect"], c["rho"], c["nsmear"],
                              c["nstep"], c["level"], c["tau"], c["lam"], c["nprec"], c["np_md"],
                              c["np_h"], (c["rat_lo"], c["rat_hi"]), c["tol"], c["tol"])
        ud = torch.from_numpy(u.copy()).cuda()
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = hmc.trajectory(ud, HostNoise(mom, xis))
        torch.cuda.synchronize()
        return time.perf_counter() - t, r["dH"]

    device_run()                     # untimed: autotuning and workspace
    t_dev, dh = device_run()
    return {"config": "4^3x8 Ls=8 Shamir M0=1.8, hot start, masses 0.01/0.1/0.04/PV 1.0, "
                      "Iwasaki 2.13, 2 stout, Omelyan [2,1,3], length 1, 10 poles, tol2 1e-24",
            "reference_cpu_sec": t_ref, "reference_cpu_cores": threads,
            "device_sec": t_dev, "dH_reference": ref["dH"][0], "dH_device": dh,
            "dH_abs_diff": abs(dh - ref["dH"][0]),
            "noise": "the reference's recorded M-series momenta and pseudofermion noise"}


def published_trajectory():
    """The reference's published single-GPU run (sample_1gpu: 8^4 from
    conf_04040408.txt, Moebius Ls=12, 2+1 flavours, Symanzik 4.17, 3 stout,
    the shipped rational tables, Mseries_parallel reset to 200000) on the
    device, from the committed fixture tests/golden/sample_8x8x8x8.npz: the
    device seconds and H(diff) beside the published 21.44 s and 0.00083995
    (sample_1gpu/run.log:1994-2000)."""
    import torch
    from b200dwf.gauge_io import tile_text_4x4x4x8
    from b200dwf.hmc import build_dwf_nf2p1, MseriesNoise
    z = np.load(os.path.join(REPO, "tests", "golden", "sample_8x8x8x8.npz"))
    c = json.loads(str(z["meta"]))
    pub = json.loads(str(z["published"]))
    tables = json.loads(str(z["tables"]))
    with tempfile.TemporaryDirectory() as d:
        for name, text in tables.items():
            with open(os.path.join(d, name), "w") as f:
                f.write(text)

        def run():
            hmc = build_dwf_nf2p1(c["lattice"], c["Ls"], c["M0"],
                                  dict(l=c["mq_l"], h=c["mq_h"], s=c["mq_s"], pv=c["mq_pv"]),
                                  c["beta"], c["c_plaq"], c["c_rect"], c["rho"], c["nsmear"],
                                  c["nstep"], c["level"], c["tau"], c["lam"], c["nprec"],
                                  c["np_md"], c["np_h"], (c["rat_lo"], c["rat_hi"]), c["tol_cg"],
                                  c["tol_cg"], b=c["b"], c=c["c"], rational_dir=d,
                                  tol2_rat_md=c["tol_ms_md"], tol2_rat_h=c["tol_ms_h"])
            ud = torch.from_numpy(tile_text_4x4x4x8(z["conf_04040408"], c["lattice"])).cuda()
            torch.cuda.synchronize()
            t = time.perf_counter()
            r = hmc.trajectory(ud, MseriesNoise(c["lattice"], c["seed"]))
            torch.cuda.synchronize()
            return time.perf_counter() - t, r

        run()                            # untimed: autotuning, workspaces, graphs
        sec, r = run()
    return {"config": "sample_1gpu: 8^4, Moebius b=1.5 c=0.5 M0=1.0 Ls=12, masses 0.0005/0.002/"
                      "0.02/PV 1.0, Symanzik beta 4.17, 3 stout, Omelyan [2,1,3], length 0.1, "
                      "tol2 1e-28, the reference's rational tables, Mseries_parallel 200000",
            "device_sec": sec, "published_sec": pub["sec_per_trajectory"],
            "H0_device": r["H0"], "H0_published": pub["H_total_init"],
            "dH_device": r["dH"], "dH_published": pub["H_total_final"] - pub["H_total_init"],
            "dH_published_log": pub["H_diff"]}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    try:
        r = run_reference_cpu(args.lattice, LS, args.steps, args.warmup, budget_s=60.0)
        gbs, t_step, reps, threads = r["gbs"], r["t_step"], r["reps"], r["threads"]
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": "reference corelib harness failed: %s" % e}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value_is": VALUE_IS, "value": gbs, "unit": "GB/s",
        "n_gpus": args.gpus,
        "steps": reps, "warmup": max(1, args.warmup), "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "dslash_gflops": 2 * FLOPS_PER_HALF_SITE * vh_of(args.lattice) / t_step / 1e9,
        "config": {"workload": WORKLOAD, "lattice": args.lattice, "Ls": LS, "M0": M0, "mq": MQ,
                   "links": "near-unit exp(i*0.3*H) + 2 stout rho=0.1", "parallelism": "replicas"},
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": "%d steps of corelib Fopr_Domainwall_eo mult Deo + mult_dag Deo on "
                                   "the full workload lattice (bounded to ~60 s)" % reps},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------ learned preconditioner
LEARNED_WEIGHTS = os.path.join(REPO, "lqcd-dwf-hmc_b200", "b200dwf", "learned_weights",
                               "hmc_16x16x16x32_Ls16.npz")


def learned_section(args):
    """On the learned preconditioner's configuration (16^3x32, Ls=16,
    m=0.01): the network trained on the plain HMC's own configurations
    (b200dwf.learned_train: 20 trajectories from conf_04040408.txt tiled,
    100 CG (residual, error) pairs each; the committed weights and their
    training record), evaluated on the tiled start after 2 stout steps --
    a configuration it never saw -- with the workload's RHS: flexible CG with
    it against plain FP64 CG, both to |r|/|b| < 1e-10.  One network
    application is timed with CUDA events with both convolution kernels
    (tensor cores, and packed FFMA2)."""
    import torch
    import b200dwf
    from b200dwf import learned_train
    from b200dwf.hopbench import learned_flops
    lattice = list(LEARN_LATTICE)
    z = np.load(LEARNED_WEIGHTS)
    record = json.loads(str(z["record"]))
    hidden = int(z["hidden"])
    _, b_host = workload_inputs(lattice, LS)
    op = b200dwf.DomainWall(lattice, LS, MQ, M0, 1.0, 0.0, 1.0, (1, 1, 1, -1))
    op.set_config(learned_train.smeared(learned_train.tiled_start(lattice), lattice))
    w = op.new_field(0)
    op.convert(w, b_host)
    lp = b200dwf.LearnedPrecond(op, hidden=hidden, seed=11)
    lp.set_weights(z["weights"])
    # one network application, CUDA events, each convolution kernel
    r32 = op.new_field(1)
    z32 = op.new_field(1)
    op.copy_convert(r32, w)
    apply_ms = {}
    old = os.environ.get("B200_LP_CONV")
    try:
        for kernel in ("ffma2", "tc1", "tc"):
            os.environ["B200_LP_CONV"] = kernel
            lp.apply(z32, r32)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            for _ in range(10):
                lp.apply(z32, r32)
            ev1.record()
            torch.cuda.synchronize()
            apply_ms[kernel] = ev0.elapsed_time(ev1) / 10
    finally:
        if old is None:
            os.environ.pop("B200_LP_CONV", None)
        else:
            os.environ["B200_LP_CONV"] = old
    op.check_error()
    flops = learned_flops(vh_of(lattice), LS, hidden)
    op.fcg(op.new_field(0), w, lp, 1.0, 20000, 8)     # untimed: flexible-CG buffers
    res = {}
    for name, fn in (("cg_f64", lambda x: op.cg(x, w, 1e-20, 20000)),
                     ("fcg_learned", lambda x: op.fcg(x, w, lp, 1e-20, 20000, 8)),
                     ("fcg_learned_m2", lambda x: op.fcg(x, w, lp, 1e-20, 20000, 2))):
        x = op.new_field(0)
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        out = fn(x)
        torch.cuda.synchronize()
        c1 = time.perf_counter()
        if name == "cg_f64":
            res[name] = {"iterations": out[0], "true_rel_residual": out[1], "seconds": c1 - c0,
                         "converged": out[2] == 0}
        else:
            res[name] = {"iterations": out[0], "fallback_cg_iterations": out[1],
                         "true_rel_residual": out[2], "seconds": c1 - c0, "converged": out[3] == 0,
                         "orthogonalised_against": 8 if name == "fcg_learned" else 2}
    train = record.get("train", [])
    return {"network": "3 layers, 4->%d->4 channels per color, 11 paths, BF16 weights, "
                       "channel mixing on tcgen05 (BF16 hi+lo inputs, FP32 accumulation)" % hidden,
            "lattice": lattice, "evaluated_on": "conf_04040408.txt tiled, 2 stout rho 0.1",
            "trained_on": "%d HMC configurations, %d CG pairs (b200dwf.learned_train)"
                          % (len(train), record.get("pairs", 0)),
            "train_loss_first_last_config": [train[0]["loss_first"], train[-1]["loss_last"]]
                                            if train else None,
            "apply_ms": apply_ms["tc"], "apply_ms_tc1": apply_ms["tc1"],
            "apply_ms_ffma2": apply_ms["ffma2"],
            "apply_tflops": flops / (apply_ms["tc"] * 1e-3) / 1e12,
            "tol_rel_residual": 1e-10, **res,
            "iteration_ratio": res["cg_f64"]["iterations"] / max(1, res["fcg_learned"]["iterations"]
                                                                 + res["fcg_learned"]["fallback_cg_iterations"]),
            "time_ratio": res["cg_f64"]["seconds"] / res["fcg_learned"]["seconds"]}, lp


# ------------------------------------------------------------------ trajectory
TRAJ_MASSES = dict(l=MQ, h=0.1, s=MS, pv=1.0)


def trajectory_section(op, lattice, u_workload, args, lp=None):
    """One 2+1-flavour HMC trajectory with the reference benchmark driver's
    action set (benchmark_hmc_dwf_corelib/hmc_dwf_eo.cpp): strange quark as
    a rational ratio over Pauli-Villars (16 poles in the force, 24 in the
    heatbath and Hamiltonian, FP64 multishift), the light pair as two
    Hasenbusch ratios (light 0.01 / 0.1 / PV 1.0), Iwasaki beta 2.13, stout
    smeared fermion links (2 x rho 0.1), nested Omelyan [2,1,3], length 0.1,
    momenta and pseudofermion noise from the reference driver's generator
    (Mseries_parallel) run on the device, the same seed for every form.  Timed per form, all solves to |r|/|b| < 1e-10:
    plain = FP64 CG and the multishift updating every shift every iteration;
    batched = the multishift's windowed shift updates, with mixed-precision
    Richardson (f16 storage, FP32 inner, FP64 outer) for the light,
    Hasenbusch and PV solves, each MD solve starting from the action's
    previous solution (use_initial_guess) and, when a trained network is
    given, the learned flexible CG for the light solves."""
    import torch
    import b200dwf
    from b200dwf import synth
    from b200dwf.hmc import build_dwf_nf2p1, Solver
    from b200dwf.gauge_io import tile_text_4x4x4x8
    lattice = list(args.traj_lattice or lattice)
    # the reference benchmark's start: conf_04040408.txt tiled onto the
    # lattice (GaugeConfig("Text_4x4x4x8"), src/lib/IO/fieldIO_Text_4x4x4x8.cpp)
    fx = np.load(os.path.join(REPO, "tests", "golden", "sample_8x8x8x8.npz"))
    u0 = tile_text_4x4x4x8(fx["conf_04040408"], lattice)
    table_dir = tempfile.mkdtemp()
    for name, text in json.loads(str(fx["tables"])).items():
        with open(os.path.join(table_dir, name), "w") as f:
            f.write(text)
    cg = {k: "cg" for k in ("l_md", "l_h", "h_md", "h_h", "pv_h")}
    mixed = {k: "mixed+" for k in ("l_md", "l_h", "h_md", "h_h", "pv_h")}
    # (name, solver kinds, multishift window): the plain form is FP64 CG with
    # every shift updated every iteration; the optimised forms use the
    # mixed-precision solves and the windowed (batched) multishift
    forms = []
    if "fp64_plain" in args.traj_forms:
        forms.append(("fp64_plain", cg, 0))
    if args.traj_all_forms:
        forms.append(("fp64_batched", cg, 16))
    if "mixed_batched" in args.traj_forms:
        forms.append(("mixed_batched", mixed, args.traj_window))
    if lp is not None and "mixed_batched_learned" in args.traj_forms:
        forms.append(("mixed_batched_learned",
                      dict({k: "mixed+" for k in ("h_md", "h_h", "pv_h")}, l_md="learned",
                           l_h="learned"), args.traj_window))
    tol2 = 1e-20
    res = {}
    for name, kinds, window in forms:
        try:
            res[name] = _trajectory_form(lattice, u0, args, lp, kinds, window, tol2, table_dir)
        except Exception as e:  # noqa: BLE001  (one form's failure keeps the others)
            res[name] = {"error": str(e)}
    import shutil
    shutil.rmtree(table_dir, ignore_errors=True)
    gc.collect()
    torch.cuda.empty_cache()
    out = {"lattice": lattice, "Ls": args.traj_ls, "M0": M0,
           "masses": dict(TRAJ_MASSES, l=args.traj_mass_l), "inner_storage": args.traj_inner,
           "actions": "rational ratio (strange / PV, 16|24 poles, FP64 multishift), "
                      "Hasenbusch ratios light/0.1 and 0.1/PV, Iwasaki beta 2.13, "
                      "2 stout rho 0.1 on the fermion links",
           "integrator": "Omelyan %s, lambda 0.1931833275" % list(args.traj_nstep),
           "length": args.traj_length, "solver_tol_rel_residual": 1e-10,
           "links": "conf_04040408.txt tiled (the reference benchmark's start configuration)",
           "rational_tables": "the reference's shipped 16-pole (MD) and %d-pole (heatbath, H) "
                              "tables on [1e-4, 10]" % args.traj_np_h,
           "rational_force_pool": args.traj_force_pool, **res}
    for name in res:
        if "sec_per_trajectory" in res[name] and "sec_per_trajectory" in res.get("fp64_plain", {}):
            out["speedup_" + name] = (res["fp64_plain"]["sec_per_trajectory"]
                                      / res[name]["sec_per_trajectory"])
    return out


def _trajectory_form(lattice, u0, args, lp, kinds, window, tol2, table_dir=None):
    import torch
    import b200dwf
    from b200dwf.hmc import build_dwf_nf2p1, MseriesNoise, Solver
    gc.collect()
    torch.cuda.empty_cache()
    # "mixed+": mixed-precision Richardson whose MD solves start from the
    # action's previous solution (use_initial_guess)
    inner = {"f32": 1, "f16": 2, "bf16": 3}[args.traj_inner]
    sv = {k: Solver(v.rstrip("+"), tol2, chrono=v.endswith("+"), inner_prec=inner,
                    chrono_depth=args.traj_chrono)
          for k, v in kinds.items()}
    torch.cuda.reset_peak_memory_stats()
    free0, total = torch.cuda.mem_get_info()
    hmc = build_dwf_nf2p1(lattice, args.traj_ls, M0, dict(TRAJ_MASSES, l=args.traj_mass_l), 2.13,
                          nstep=args.traj_nstep,
                          tau=args.traj_length, np_md=16, np_h=args.traj_np_h, tol2_md=tol2,
                          tol2_h=tol2, solvers=sv, shift_window=window, rational_dir=table_dir,
                          rational_force_pool=args.traj_force_pool)
    if "learned" in kinds.values():
        # the trained weights are independent of volume and Ls; the network
        # runs on the light operator's own (smeared) links
        lp_form = b200dwf.LearnedPrecond(hmc.fermions["nf2"].f.op, hidden=lp.hidden, seed=1)
        lp_form.set_weights(lp.weights(deployed=False))
        for v in sv.values():
            v.lp = lp_form
    ud = torch.from_numpy(u0.copy()).cuda()
    hmc.set_config(ud)
    hmc.warmup()
    for v in sv.values():
        v.iterations, v.seconds, v.calls = 0, 0.0, 0
    for r in hmc.fermions["nf1"].rationals.values():
        r.iterations, r.seconds, r.calls = 0, 0.0, 0
    # the benchmark driver's generator (Mseries_parallel) on the device; its
    # streams are seeded here, outside the timed trajectory
    noise = MseriesNoise(lattice, args.traj_seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = hmc.trajectory(ud, noise)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    out = {"sec_per_trajectory": time.perf_counter() - t0, "dH": r["dH"],
           "H0": r["H0"], "multishift_window": window,
           "device_memory_gb": {"in_use_after": (total - free1) / 1e9,
                                "added_by_this_form": (free0 - free1) / 1e9,
                                "torch_peak_allocated": torch.cuda.max_memory_allocated() / 1e9},
           **hmc.stats()}
    del hmc, ud, r, sv
    gc.collect()
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------ B200 arm
class _Weights:
    """The committed network weights in the shape _trajectory_form reads."""

    def __init__(self, path):
        z = np.load(path)
        self.hidden = int(z["hidden"])
        self._w = z["weights"]

    def weights(self, deployed=False):
        return self._w


def trajectory_only(args):
    """--traj-only: the trajectory forms alone, with the peak device memory
    the process reached (torch's allocator and the library's own
    allocations alike, from cudaMemGetInfo polled during the run)."""
    import faulthandler
    import torch
    faulthandler.enable()        # a native crash prints every thread's Python stack
    torch.cuda.init()
    lp = _Weights(LEARNED_WEIGHTS) if "mixed_batched_learned" in args.traj_forms else None
    free_min = [torch.cuda.mem_get_info()[0]]
    stop = threading.Event()

    def poll():
        while not stop.wait(0.5):
            free_min[0] = min(free_min[0], torch.cuda.mem_get_info()[0])

    total = torch.cuda.mem_get_info()[1]
    thr = threading.Thread(target=poll, daemon=True)
    thr.start()
    try:
        out = trajectory_section(None, args.traj_lattice, None, args, lp)
    finally:
        stop.set()
        thr.join()
    out["device_memory_high_water_gb"] = (total - free_min[0]) / 1e9
    out["device_memory_total_gb"] = total / 1e9
    print(json.dumps(out))


def b200_arm(args, rank, world, local_rank):
    import torch
    import b200dwf
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    b200dwf.check(b200dwf.lib().b200_init(local_rank, 0))
    lattice = args.lattice
    vh = vh_of(lattice)
    u, b = workload_inputs(lattice, LS, device_smear=True)
    op = b200dwf.DomainWall(lattice, LS, MQ, M0, 1.0, 0.0, 1.0, (1, 1, 1, -1))
    op.set_config(u)
    w = op.new_field(0)
    v1 = op.new_field(0)
    v2 = op.new_field(0)
    op.convert(w, b)
    step_bytes = 2 * BYTES_PER_HALF_SITE * vh
    # the timed loops queue their launches without a host round trip per call;
    # the plan's error word is checked after each loop
    op.set_async(True)

    def step():
        op.mult(v1, w, "Deo")
        op.mult_dag(v2, w, "Deo")

    from b200dwf import replicas

    def barrier():
        replicas.barrier(dist)

    for _ in range(args.warmup):
        step()
    op.check_error()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    op.check_error()
    barrier()
    torch.cuda.synchronize()
    t_total = replicas.max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, "cuda")
    value = replicas.whole_job_rate(step_bytes * args.steps, t_total, world) / 1e9

    # dominant kernel: mult_dag("Deo") is exactly one launch of the fused hop kernel
    nk = max(20, min(args.steps, 200))
    for _ in range(5):
        op.mult_dag(v2, w, "Deo")
    torch.cuda.synchronize()
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record()
    for _ in range(nk):
        op.mult_dag(v2, w, "Deo")
    k1.record()
    torch.cuda.synchronize()
    op.check_error()
    t_hop = k0.elapsed_time(k1) / 1e3 / nk
    peak, peak_kind = read_peaks()
    achieved = BYTES_PER_HALF_SITE * vh / t_hop / 1e9
    traffic = read_traffic(vh)
    op.set_async(False)

    # End to end through the C ABI with page-locked host buffers: every step
    # uploads its input field (reference layout, host) and downloads both
    # results.  Pipelined form: the asynchronous convert / reverse entry
    # points on an upload and a download stream, the two hops on a third, two
    # sets of device fields, so step k+1's upload overlaps step k's download
    # (the two PCIe directions).  Synchronous form: convert, mult, mult_dag,
    # reverse, reverse, as a reference shell would call them.
    nbytes = 24 * vh * LS * 8
    h_in = torch.from_numpy(b).pin_memory()
    h_outs = [[torch.empty(24 * vh * LS, dtype=torch.float64).pin_memory() for _ in range(2)]
              for _ in range(2)]
    ne = max(3, min(args.steps, 10))
    ws = [w, op.new_field(0)]
    v1s, v2s = [v1, op.new_field(0)], [v2, op.new_field(0)]
    s_in, s_cmp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev = {k: [torch.cuda.Event(), torch.cuda.Event()] for k in ("in", "cmp", "out")}
    h_in_np = h_in.numpy()
    h_out_np = [[t.numpy() for t in pair] for pair in h_outs]
    op.set_async(True)

    def e2e_pipeline(n):
        for k in range(n):
            j = k % 2
            if k >= 2:
                s_in.wait_event(ev["cmp"][j])        # ws[j]: its hops of step k-2 are done
            op.convert_async(ws[j], h_in_np, s_in)
            ev["in"][j].record(s_in)
            s_cmp.wait_event(ev["in"][j])
            if k >= 2:
                s_cmp.wait_event(ev["out"][j])       # v1s[j], v2s[j]: downloaded by step k-2
            op.mult(v1s[j], ws[j], "Deo", stream=s_cmp)
            op.mult_dag(v2s[j], ws[j], "Deo", stream=s_cmp)
            ev["cmp"][j].record(s_cmp)
            s_out.wait_event(ev["cmp"][j])
            op.reverse_async(v1s[j], h_out_np[j][0], s_out)
            op.reverse_async(v2s[j], h_out_np[j][1], s_out)
            ev["out"][j].record(s_out)

    e2e_pipeline(2)
    torch.cuda.synchronize()
    op.check_error()
    barrier()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(s_in)
    e2e_pipeline(ne)
    s_out.wait_stream(s_in)
    s_out.wait_stream(s_cmp)
    q1.record(s_out)
    torch.cuda.synchronize()
    op.check_error()
    op.set_async(False)
    t_e2e = replicas.max_over_ranks(q0.elapsed_time(q1) / 1e3, dist, "cuda")
    e2e_value = replicas.whole_job_rate(step_bytes * ne, t_e2e, world) / 1e9
    # the result of the last step equals the device-only result
    assert np.array_equal(h_out_np[(ne - 1) % 2][1], op.reverse(v2))

    def e2e_sync_step():
        op.convert(w, h_in_np)
        op.mult(v1, w, "Deo")
        op.mult_dag(v2, w, "Deo")
        op.reverse(v1, out=h_out_np[0][0])
        op.reverse(v2, out=h_out_np[0][1])

    e2e_sync_step()
    torch.cuda.synchronize()
    q2, q3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q2.record()
    for _ in range(ne):
        e2e_sync_step()
    q3.record()
    torch.cuda.synchronize()
    t_sync = replicas.max_over_ranks(q2.elapsed_time(q3) / 1e3, dist, "cuda")
    e2e_sync_value = replicas.whole_job_rate(step_bytes * ne, t_sync, world) / 1e9

    # The host link the end-to-end step runs on: pinned copies of one field
    # each way alone and both ways at once (CUDA events), and the step's
    # lower bound on it (its download beside its upload).
    d_scr = torch.empty(h_in.numel(), dtype=torch.float64, device="cuda")
    d_scr2 = torch.empty_like(d_scr)
    h_dn = h_outs[0][0]

    def timed_copies(pairs, reps=3):
        starts, ends = [], []
        for st, fn in pairs:
            with torch.cuda.stream(st):
                fn()                                   # warm
        torch.cuda.synchronize()
        for st, _ in pairs:
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            starts.append(a)
            ends.append(z)
        for st, fn in pairs:
            with torch.cuda.stream(st):
                for _ in range(reps):
                    fn()
        for (st, _), z in zip(pairs, ends):
            z.record(st)
        torch.cuda.synchronize()
        return [reps * nbytes / (a.elapsed_time(z) * 1e-3) / 1e9 for a, z in zip(starts, ends)]

    up = (s_in, lambda: d_scr.copy_(h_in, non_blocking=True))
    dn = (s_out, lambda: h_dn.copy_(d_scr2, non_blocking=True))
    h2d_alone = timed_copies([up])[0]
    d2h_alone = timed_copies([dn])[0]
    h2d_both, d2h_both = timed_copies([up, dn])
    step_bound_s = max(nbytes / (h2d_both * 1e9), 2 * nbytes / (d2h_both * 1e9))
    host_link = {"h2d_gbs": h2d_alone, "d2h_gbs": d2h_alone, "h2d_gbs_both_ways": h2d_both,
                 "d2h_gbs_both_ways": d2h_both, "step_bound_ms": step_bound_s * 1e3,
                 "step_ms": t_e2e * 1e3 / ne, "frac_of_link_bound": step_bound_s / (t_e2e / ne)}
    del d_scr, d_scr2, h_dn
    del h_in, h_outs, h_in_np, h_out_np, ws, v1s, v2s

    # FP64 CG time to solution, |r|/|b| < 1e-10
    cg = None
    if not args.no_cg:
        x = op.new_field(0)
        op.cg(x, w, 1e-20, 3)          # untimed: work buffers + autotuning of the CG kernels
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        n, diff, rc = op.cg(x, w, 1e-20, 20000)
        torch.cuda.synchronize()
        c1 = time.perf_counter()
        cg = {"tol_rel_residual": 1e-10, "iterations": n, "true_rel_residual": diff,
              "seconds": c1 - c0, "converged": rc == 0,
              "ms_per_iteration": (c1 - c0) * 1e3 / max(n, 1)}

    # mixed-precision Richardson (FP64 outer, inner CG in f32/f16/bf16) and the
    # 16-pole multishift CG (shifts log-spaced 1e-4..64), same lattice and RHS
    solvers = None
    if not args.no_solvers and world == 1:
        solvers = {"richardson": {}, "multishift": None}
        from b200dwf.hmc import INNER_TOL2
        for name, prec in (("f32", 1), ("f16", 2), ("bf16", 3)):
            tin = INNER_TOL2[prec]
            x = op.new_field(0)
            op.richardson(x, w, prec, 1e-20, 1, tin, 3)   # untimed warm-up (buffers, autotuning)
            torch.cuda.synchronize()
            c0 = time.perf_counter()
            nout, nin, diff, rc = op.richardson(x, w, prec, 1e-20, 100, tin, 20000)
            torch.cuda.synchronize()
            c1 = time.perf_counter()
            solvers["richardson"][name] = {"outer_iterations": nout, "inner_iterations": nin,
                                           "inner_tol2": tin, "true_rel_residual": diff,
                                           "seconds": c1 - c0, "converged": rc == 0}
            del x
        sigma = list(np.logspace(-4, np.log10(64.0), 16))
        xs = [op.new_field(0) for _ in sigma]
        ms = {}
        for window in (0, 8, 16):
            # window 0: every shift's x_i, p_i updated every iteration (the
            # reference's form); 8 / 16: deferred updates from stored residuals
            op.set_shift_window(window)
            op.shiftcg(xs, sigma, w, 1e-20, 20)               # untimed warm-up
            torch.cuda.synchronize()
            c0 = time.perf_counter()
            n, diff, rc = op.shiftcg(xs, sigma, w, 1e-20, 20000)
            torch.cuda.synchronize()
            c1 = time.perf_counter()
            ms["window_%d" % window] = {"iterations": n, "max_true_rel_residual": diff,
                                        "seconds": c1 - c0,
                                        "ms_per_iteration": (c1 - c0) * 1e3 / max(n, 1),
                                        "converged": rc == 0}
        op.set_shift_window(16)
        solvers["multishift"] = {"shifts": len(sigma), "sigma": "log-spaced 1e-4..64",
                                 **ms["window_16"], "by_window": ms}
        del xs

    learned, lp = None, None
    # the solver, learned-network and trajectory sections are one-GPU
    # workloads; under torchrun (replicas) only the Dslash metric is timed
    if not args.no_learned and world == 1:
        learned, lp = learned_section(args)
    trajectory = None
    if not args.no_trajectory and world == 1:
        trajectory = trajectory_section(op, lattice, u, args, lp)

    published = None
    if world == 1 and not args.no_trajectory:
        try:
            published = published_trajectory()
        except Exception as e:  # noqa: BLE001
            published = {"unavailable": str(e)}
    small = None
    if world == 1 and not args.no_cpu and not args.no_trajectory:
        try:
            small = small_trajectory_beside_reference()
        except Exception as e:  # noqa: BLE001
            small = {"unavailable": str(e)}
    if rank != 0:
        return
    cpu, cpu_traj = None, None
    if world == 1 and not args.no_cpu:
        try:
            r = run_reference_cpu(lattice, LS, 100, 1, budget_s=20.0, inputs=(u, b), ddagd=True)
            cpu = {"value": r["gbs"], "unit": "GB/s", "cores": r["threads"], "kind": "reference",
                   "sample": "%d steps (Deo + Ddag_eo, plus one DdagD each) of the reference corelib "
                             "Fopr_Domainwall_eo on the full %s Ls=16 workload, bounded to ~20 s"
                             % (r["reps"], "x".join(map(str, lattice))),
                   "ddagd_seconds": r["t_ddagd"]}
            plain = (trajectory or {}).get("fp64_plain", {})
            n_ddagd = sum(v.get("iterations", 0) for k, v in plain.items()
                          if isinstance(v, dict) and (k.startswith("solver_") or k.startswith("multishift_")))
            if n_ddagd:
                cpu_traj = {"sec_per_trajectory": n_ddagd * r["t_ddagd"], "kind": "extrapolated",
                            "how": "reference corelib DdagD seconds on %d host cores x the %d DdagD "
                                   "applications (CG + multishift iterations) of the plain FP64 "
                                   "device trajectory; a lower bound (forces, smearing and vector "
                                   "updates left out)" % (r["threads"], n_ddagd)}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                   "sample": "unavailable: %s" % e}
    # the reference's own mixed-precision solver (QXS backend) on the host
    # cores, a bounded sample, extrapolated with the device solve's
    # iteration counts (same algorithm: FP64 Richardson, FP32 CG inner)
    cpu_mixed = None
    if world == 1 and not args.no_cpu and solvers and "f32" in solvers["richardson"]:
        try:
            q = run_reference_qxs_mixed(lattice, LS, (u, b))
            rf = solvers["richardson"]["f32"]
            est = (rf["outer_iterations"] * q["ddagd_f64_seconds"]
                   + rf["inner_iterations"] * q["ddagd_f32_seconds"])
            cpu_mixed = {"kind": "reference", "cores": int(q.get("threads", 0)),
                         "what": "Fprop_alt_Standard_eo_Richardson<AField<double,QXS>, "
                                 "AField<float,QXS>>::invert_DdagD_even (QXS general backend, "
                                 "oracle/Makefile.qxs), FP64 Richardson with FP32 CG inner solves",
                         "sample": "one FP64 and one FP32 DdagD, and one 1 x 1 (outer x inner) "
                                   "bounded solve, on the full %s Ls=16 workload"
                                   % "x".join(map(str, lattice)),
                         **q,
                         "extrapolated_solve_seconds": est,
                         "device_solve_seconds": rf["seconds"],
                         "how": "a lower bound: the device's f32-inner Richardson iteration "
                                "counts (%d outer, %d inner) x the reference's measured seconds per "
                                "FP64 and per FP32 DdagD (vector updates, conversions and solver "
                                "setup left out)" % (rf["outer_iterations"], rf["inner_iterations"])}
        except Exception as e:  # noqa: BLE001
            cpu_mixed = {"unavailable": str(e)}
    line = {
        "metric": METRIC, "value_is": VALUE_IS, "value": value, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_total * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "dslash_gflops": replicas.whole_job_rate(2 * FLOPS_PER_HALF_SITE * vh * args.steps, t_total,
                                                 world) / 1e9,
        "config": {"workload": WORKLOAD, "lattice": lattice, "Ls": LS, "M0": M0, "mq": MQ,
                   "links": "near-unit exp(i*0.3*H) + 2 stout rho=0.1", "parallelism": "replicas",
                   "l2": "inputs larger than L2 (%.0f MB per field)" % (nbytes / 1e6)},
        "clocks": clk.summary(),
        # Shamir b=1, c=0, alpha=1: the D_eo pre-factor is the identity, so a
        # step is two hop launches (mult Deo, mult_dag Deo)
        "gpu_launches": 2 * args.steps,
        "roofline": {"kernel": dagger_hop_kernel(vh),
                     "bound": "hbm",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_note": "ncu DRAM bytes of a 16^3x32 launch scaled by sites",
                     "algorithmic_bytes_per_launch": BYTES_PER_HALF_SITE * vh,
                     "gflops": FLOPS_PER_HALF_SITE * vh / t_hop / 1e9,
                     "launch_us": t_hop * 1e6, "target_frac": 0.7},
        "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": 2 * nbytes, "steps": ne,
                "how": "pipelined: convert_async / 2 hops / 2 reverse_async on three streams, "
                       "double-buffered, step k+1's upload overlapping step k's download",
                "synchronous_calls_value": e2e_sync_value, "host_link": host_link},
    }
    # the trajectory's headline numbers as short top-level keys
    if trajectory:
        for form in ("fp64_plain", "mixed_batched", "mixed_batched_learned"):
            f = trajectory.get(form, {})
            if "sec_per_trajectory" in f:
                line["sec_traj_" + form] = round(f["sec_per_trajectory"], 3)
                line["dH_" + form] = f.get("dH")
            if "speedup_" + form in trajectory:
                line["speedup_" + form] = round(trajectory["speedup_" + form], 3)
        line["speedup_target"] = 3.0
    if learned:
        # one network application (tensor-core and FFMA2 convolutions), and
        # CG / flexible-CG iterations and seconds on an unseen configuration
        line["learned_apply_ms"] = round(learned["apply_ms"], 3)
        line["learned_apply_ms_tc1"] = round(learned["apply_ms_tc1"], 3)
        line["learned_apply_ms_ffma2"] = round(learned["apply_ms_ffma2"], 3)
        line["learned_iteration_ratio"] = round(learned["iteration_ratio"], 3)
        line["learned_time_ratio"] = round(learned["time_ratio"], 3)
    if cpu_traj:
        line["sec_traj_cpu_reference_extrapolated"] = round(cpu_traj["sec_per_trajectory"], 1)
    if cpu_mixed and "extrapolated_solve_seconds" in cpu_mixed:
        line["sec_mixed_solve_cpu_reference_extrapolated"] = round(cpu_mixed["extrapolated_solve_seconds"], 1)
        line["sec_mixed_solve_device"] = round(cpu_mixed["device_solve_seconds"], 3)
    if published and "device_sec" in published:
        line["sec_traj_published_8x8x8x8_device"] = round(published["device_sec"], 3)
        line["sec_traj_published_8x8x8x8_reference_gpu"] = published["published_sec"]
        line["dH_published_8x8x8x8_device"] = published["dH_device"]
    line.update({
        "cpu_baseline": cpu,
        "cpu_trajectory": cpu_traj,
        "cpu_mixed_precision": cpu_mixed,
        "cg_f64": cg,
        "solvers": solvers,
        "learned_preconditioner": learned,
        "trajectory": trajectory,
        "trajectory_4x4x4x8_beside_reference": small,
        "trajectory_published_8x8x8x8": published,
        "autotune": b200dwf.tuning_table().strip().splitlines(),
    })
    print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.traj_only:
        trajectory_only(args)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        b200_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
