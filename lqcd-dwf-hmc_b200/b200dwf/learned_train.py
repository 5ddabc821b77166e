"""Train the learned preconditioner on configurations of the HMC itself.

    python -m b200dwf.learned_train --out weights.npz [--lattice 16 16 16 32]
        [--ls 16] [--configs 20] [--pairs 100] [--epochs 1] [--seed 1234567]

1. Configurations: the plain HMC (the reference benchmark driver's 2+1-flavour
   action set, b200dwf.hmc.build_dwf_nf2p1: Shamir M0 = 1.8, light 0.01 /
   Hasenbusch 0.1 / strange 0.04 / PV 1.0, Iwasaki beta 2.13, 2 stout rho 0.1,
   Omelyan [2,1,3], FP64 CG and multishift to |r|/|b| < 1e-10, Metropolis on)
   run from conf_04040408.txt tiled onto the lattice, the driver's generator
   (Mseries_parallel) reset to seed + k before trajectory k as the driver
   does; every configuration after a trajectory is kept.
2. Pairs: on each configuration, the fermion operator on its stout-smeared
   links, a Gaussian source, and `pairs` (residual, error) pairs of plain CG
   spread over its iterations (b200dwf.cg_training_pairs).
3. Training: the library's own forward / adjoint / Adam kernels
   (b200_lp_train), `epochs` passes over each configuration's pairs.
4. Evaluation on a configuration the network never saw (the tiled start):
   plain FP64 CG against the learned flexible CG to |r|/|b| < 1e-10.

The weights (FP32 master copy) and a record of every step go to `out`."""
import argparse
import json
import os
import time

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
SAMPLE = os.path.join(REPO, "tests", "golden", "sample_8x8x8x8.npz")


def tiled_start(lattice):
    from .gauge_io import tile_text_4x4x4x8
    return tile_text_4x4x4x8(np.load(SAMPLE)["conf_04040408"], lattice)


def generate_configs(lattice, ls, n, seed, tau, log):
    """n configurations of the plain HMC from the tiled start (host arrays)."""
    import torch
    from .hmc import build_dwf_nf2p1, MseriesNoise
    hmc = build_dwf_nf2p1(lattice, ls, 1.8, dict(l=0.01, h=0.1, s=0.04, pv=1.0), 2.13,
                          nstep=(2, 1, 3), tau=tau, np_md=16, np_h=24, tol2_md=1e-20,
                          tol2_h=1e-20, shift_window=0)
    u = torch.from_numpy(tiled_start(lattice)).cuda()
    rng = np.random.default_rng(seed)
    noise = MseriesNoise(lattice, seed)
    out = []
    for k in range(n):
        noise.reset(seed + k)
        t = time.perf_counter()
        r = hmc.update(u, noise, rng)
        torch.cuda.synchronize()
        log.append({"trajectory": k, "dH": r["dH"], "accepted": r["accepted"],
                    "seconds": time.perf_counter() - t})
        out.append(u.cpu().numpy().copy())
    return out


def smeared(u, lattice):
    from . import StoutSmear
    sm = StoutSmear(lattice, 0.1, 2)
    sm.set_config(u)
    return np.ascontiguousarray(sm.config(2))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--lattice", type=int, nargs=4, default=[16, 16, 16, 32])
    ap.add_argument("--ls", type=int, default=16)
    ap.add_argument("--configs", type=int, default=20)
    ap.add_argument("--pairs", type=int, default=100)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--hidden", type=int, default=8)
    ap.add_argument("--tau", type=float, default=0.2)
    ap.add_argument("--seed", type=int, default=1234567)
    a = ap.parse_args(argv)
    import torch
    import b200dwf
    from . import synth
    lattice = list(a.lattice)
    record = {"lattice": lattice, "Ls": a.ls, "mq": 0.01, "M0": 1.8, "hmc": [], "train": []}
    t0 = time.perf_counter()
    configs = generate_configs(lattice, a.ls, a.configs, a.seed, a.tau, record["hmc"])
    record["hmc_seconds"] = time.perf_counter() - t0

    op = b200dwf.DomainWall(lattice, a.ls, 0.01, 1.8)
    op.set_config(smeared(configs[0], lattice))
    lp = b200dwf.LearnedPrecond(op, hidden=a.hidden, seed=11)
    t0 = time.perf_counter()
    npairs = 0
    for c, u in enumerate(configs):
        op.set_config(smeared(u, lattice))
        b = op.new_field(0)
        op.convert(b, synth.spinor_field(lattice, a.ls, a.seed + 1000 + c))
        n_ref, _, _ = op.cg(op.new_field(0), b, 1e-20, 100000)
        iters = sorted(set(int(v) for v in np.linspace(2, max(3, n_ref - 2), a.pairs)))
        rs, es = b200dwf.cg_training_pairs(op, b, iters)
        l0, l1 = lp.train(rs, es, a.epochs, a.lr, seed=c + 1)
        npairs += len(rs)
        record["train"].append({"config": c, "cg_iterations": n_ref, "pairs": len(rs),
                                "loss_first": l0, "loss_last": l1})
        del rs, es
        torch.cuda.empty_cache()
    torch.cuda.synchronize()
    record["train_seconds"] = time.perf_counter() - t0
    record["pairs"] = npairs

    # evaluation on the tiled start, which no training configuration is
    op.set_config(smeared(tiled_start(lattice), lattice))
    w = op.new_field(0)
    op.convert(w, synth.spinor_field(lattice, a.ls, a.seed + 7))
    res = {}
    for name, fn in (("cg_f64", lambda x: op.cg(x, w, 1e-20, 100000)),
                     ("fcg_learned", lambda x: op.fcg(x, w, lp, 1e-20, 100000, 8))):
        x = op.new_field(0)
        fn(x)                                   # untimed: buffers
        x = op.new_field(0)
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        out = fn(x)
        torch.cuda.synchronize()
        res[name] = {"iterations": out[0], "seconds": time.perf_counter() - c0}
    record["evaluation"] = res
    np.savez_compressed(a.out, weights=lp.weights(deployed=False), hidden=a.hidden,
                        record=json.dumps(record))
    print(json.dumps({k: v for k, v in record.items() if k not in ("hmc", "train")}))


if __name__ == "__main__":
    main()
