"""Time one operator mode of the even/odd domain-wall operator.

    python -m b200dwf.hopbench --lattice 16 16 16 32 --ls 16 --prec f16 \
        --mode Deo --dag --reps 50 [--variant N] [--warmup 5]

Builds the operator on seeded near-unit links (exp(i*0.3*H), no smearing:
timing does not depend on it), converts a Gaussian field into the chosen
storage precision, and times `reps` calls of mult / mult_dag with CUDA events
on the stream they run on.  Prints one JSON line: microseconds per call, and
for the single-hop modes (Deo, Doe) the fused hop's algorithmic bytes per
call and GB/s,
    B = Vh * (Ls * 2 * s_spinor + 8 * s_link)
with s_spinor the stored bytes of one (site, s) spinor (f64 192, f32 96,
f16/bf16 48 + a 4-byte scale) and s_link the bytes of one link record (f64
144, f32 80, f16/bf16 48).  --variant pins the hop kernel variant
(B200_HOP_VARIANT) instead of the autotuner's choice.

    python -m b200dwf.hopbench --learned [--hidden 8] [--lp-conv ffma2] ...

times one application of the learned preconditioner instead (five
convolution launches on FP32 fields) and reports its FP32 work: per
(site, s, color) row and path, 8 flops per complex multiply-add of the
channel mixing, and per row and hop path 72 flops per channel of the SU(3)
transport.  --lp-conv selects the convolution kernel (B200_LP_CONV): tc,
the tensor-core form on BF16 hi + lo inputs (default); tc1, the
tensor-core form on BF16 inputs; ffma2, the packed-FFMA2 form.

    python -m b200dwf.hopbench --richardson f16 --inner-iters 20 ...

runs one bounded mixed-precision Richardson solve instead (one outer
iteration of at most --inner-iters inner CG iterations in the given
storage, inner tolerance b200dwf.hmc.INNER_TOL2, after one untimed solve
for the autotuner) and reports its iterations and seconds: the command
whose launch list shows what one inner iteration launches."""
import argparse
import json
import os

import numpy as np

SPINOR_BYTES = {0: 192, 1: 96, 2: 52, 3: 52}
LINK_BYTES = {0: 144, 1: 80, 2: 48, 3: 48}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", type=int, nargs=4, default=[16, 16, 16, 32])
    ap.add_argument("--ls", type=int, default=16)
    ap.add_argument("--prec", default="f64", choices=["f64", "f32", "f16", "bf16"])
    ap.add_argument("--mode", default="Deo")
    ap.add_argument("--dag", action="store_true")
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--mq", type=float, default=0.01)
    ap.add_argument("--m0", type=float, default=1.8)
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--hidden", type=int, default=8)
    ap.add_argument("--lp-conv", default=None, choices=["tc", "tc1", "ffma2"])
    ap.add_argument("--richardson", default=None, choices=["f32", "f16", "bf16"])
    ap.add_argument("--inner-iters", type=int, default=20)
    a = ap.parse_args(argv)
    if a.variant is not None:
        os.environ["B200_HOP_VARIANT"] = str(a.variant)
    if a.lp_conv is not None:
        os.environ["B200_LP_CONV"] = a.lp_conv
    if a.learned:
        return learned(a)
    if a.richardson:
        return richardson(a)
    import torch
    import b200dwf
    from b200dwf import synth
    prec = b200dwf.PREC_NAMES[a.prec]
    op = b200dwf.DomainWall(a.lattice, a.ls, a.mq, a.m0)
    op.set_config(synth.gauge_field(a.lattice, 1234567, "near", eps=0.3))
    w, v = op.new_field(prec), op.new_field(prec)
    op.convert(w, synth.spinor_field(a.lattice, a.ls, 7654321))
    call = op.mult_dag if a.dag else op.mult
    op.set_async(True)
    for _ in range(a.warmup):
        call(v, w, a.mode)
    op.check_error()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        call(v, w, a.mode)
    e1.record()
    torch.cuda.synchronize()
    op.check_error()
    us = e0.elapsed_time(e1) * 1e3 / a.reps
    out = {"lattice": a.lattice, "Ls": a.ls, "prec": a.prec, "mode": a.mode, "dag": a.dag,
           "variant": a.variant, "us_per_call": us}
    if a.mode in ("Deo", "Doe"):
        vh = int(np.prod(a.lattice)) // 2
        nbytes = vh * (a.ls * 2 * SPINOR_BYTES[prec] + 8 * LINK_BYTES[prec])
        out.update(bytes_per_call=nbytes, gbs=nbytes / (us * 1e-6) / 1e9)
    print(json.dumps(out))


def richardson(a):
    import time
    import torch
    import b200dwf
    from b200dwf import synth
    from b200dwf.hmc import INNER_TOL2
    prec = b200dwf.PREC_NAMES[a.richardson]
    op = b200dwf.DomainWall(a.lattice, a.ls, a.mq, a.m0)
    op.set_config(synth.gauge_field(a.lattice, 1234567, "near", eps=0.3))
    b, x = op.new_field(0), op.new_field(0)
    op.convert(b, synth.spinor_field(a.lattice, a.ls, 7654321))
    op.richardson(x, b, prec, 1e-20, 1, INNER_TOL2[prec], 30)    # untimed: buffers, autotuner
    x.zero()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nout, nin, diff, rc = op.richardson(x, b, prec, 1e-20, 1, INNER_TOL2[prec], a.inner_iters)
    sec = time.perf_counter() - t0
    print(json.dumps({"lattice": a.lattice, "Ls": a.ls, "richardson": a.richardson,
                      "inner_tol2": INNER_TOL2[prec], "outer": nout, "inner": nin,
                      "seconds": sec, "ms_per_inner": sec * 1e3 / max(nin, 1)}))


def learned_flops(vh, ls, hidden):
    """FP32 flops of one network application (five launches)."""
    rows = vh * ls
    f = 0
    for npath, nhop, cin, cout in ((3, 0, 4, hidden), (8, 8, 4, hidden), (11, 8, hidden, hidden),
                                   (11, 8, hidden, hidden), (11, 8, hidden, 4)):
        f += rows * (3 * npath * cin * cout * 8 + nhop * cin * 72)
    return f


def learned(a):
    import torch
    import b200dwf
    from b200dwf import synth
    op = b200dwf.DomainWall(a.lattice, a.ls, a.mq, a.m0)
    op.set_config(synth.gauge_field(a.lattice, 1234567, "near", eps=0.3))
    lp = b200dwf.LearnedPrecond(op, hidden=a.hidden, seed=3, init_noise=0.1)
    f64 = op.new_field(0)
    op.convert(f64, synth.spinor_field(a.lattice, a.ls, 7654321))
    r, z = op.new_field(1), op.new_field(1)
    op.copy_convert(r, f64)
    for _ in range(a.warmup):
        lp.apply(z, r)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        lp.apply(z, r)
    e1.record()
    torch.cuda.synchronize()
    op.check_error()
    us = e0.elapsed_time(e1) * 1e3 / a.reps
    vh = int(np.prod(a.lattice)) // 2
    fl = learned_flops(vh, a.ls, a.hidden)
    print(json.dumps({"lattice": a.lattice, "Ls": a.ls, "learned": True, "hidden": a.hidden,
                      "lp_conv": os.environ.get("B200_LP_CONV", "tc"), "us_per_apply": us,
                      "flops_per_apply": fl, "tflops": fl / (us * 1e-6) / 1e12}))


if __name__ == "__main__":
    main()
