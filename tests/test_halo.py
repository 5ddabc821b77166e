"""Host logic of the halo exchange for a lattice split along t
(b200dwf.halo), on the CPU: the slab geometry and the t boundary phase, the
ghost exchange and global sums over gloo process groups of 2 and 3 ranks,
the extended links each rank assembles from its own slices alone, and the
thread transport the one-GPU tests use.  The operator on the split lattice
against the whole-lattice operator is tests/test_halo_gpu.py."""
import datetime
import os
import sys
import threading

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from b200dwf import synth
from b200dwf.halo import (TSplit, ThreadComm, ThreadHub, TorchComm, _slices, assemble_links,
                          assemble_spinor)

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LAT = [4, 2, 2, 12]


def _pattern(split, nbytes_slice):
    """An extended field whose interior slice i holds bytes (10 * rank + i),
    ghosts 255."""
    buf = torch.full(((split.nt + 2) * nbytes_slice,), 255, dtype=torch.uint8)
    for i in range(split.nt):
        buf[i * nbytes_slice:(i + 1) * nbytes_slice] = 10 * split.rank + i
    return buf


def test_split_geometry_and_boundary_phase():
    u = synth.gauge_field(LAT, 3, "hot")
    T, v3 = LAT[3], LAT[0] * LAT[1] * LAT[2]
    parts = []
    for r, nts in enumerate([[4, 8], [4, 8]]):
        s = TSplit(LAT, nts, r)
        assert s.ext == LAT[:3] + [s.nt + 2]
        assert s.ext_t[:s.nt] == list(range(s.t0, s.t0 + s.nt))
        assert s.ext_t[s.nt:] == [(s.t0 + s.nt) % T, (s.t0 - 1) % T]
        ext = s.gauge(u, -1).reshape(4, s.nt + 2, v3, 18)
        ref = u.reshape(4, T, v3, 18)
        for k, t in enumerate(s.ext_t):
            sign = np.where(np.arange(4)[:, None, None] == 3, -1.0, 1.0) if t == T - 1 else 1.0
            assert np.array_equal(ext[:, k], ref[:, t] * sign)
        parts.append(s.interior_links(ext.reshape(-1)))
    phased = u.reshape(4, T, v3, 18).copy()
    phased[3, T - 1] *= -1
    assert np.array_equal(assemble_links(parts), phased.reshape(-1))
    ls = 4
    w = synth.spinor_field(LAT, ls, 5)
    sparts = [TSplit(LAT, [6, 6], r) for r in range(2)]
    got = assemble_spinor([s.interior_spinor(s.spinor(w, ls), ls) for s in sparts], ls)
    assert np.array_equal(got, w)


@pytest.mark.parametrize("bad", [[5, 7], [12, 0], [4, 4]])
def test_split_refuses_bad_slabs(bad):
    with pytest.raises(ValueError):
        TSplit(LAT, bad, 0)


def _gloo_worker(rank, world, port, nts, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.join(REPO, "lqcd-dwf-hmc_b200"))
    from b200dwf import synth as sy
    from b200dwf.halo import TSplit as TS, TorchComm as TC, _slices as sl, extend_links as el
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        split = TS(LAT, nts, rank)
        comm = TC()
        nb = 48
        buf = _pattern(split, nb)
        comm.exchange(split, *sl(buf, split.nt))
        front = int(buf[(split.nt + 1) * nb])
        back = int(buf[split.nt * nb])
        total = comm.sum(rank + 0.5)
        u = sy.gauge_field(LAT, 11, "hot")
        T, v3 = LAT[3], LAT[0] * LAT[1] * LAT[2]
        loc = u.reshape(4, T, v3 * 18)[:, split.t0:split.t0 + split.nt].reshape(-1)
        ext = el(split, comm, loc, -1, device="cpu").numpy()
        ok_links = bool(np.array_equal(ext, split.gauge(u, -1)))
        out.put((rank, front, back, total, ok_links))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("nts", [[6, 6], [2, 4, 6]])
def test_exchange_sum_and_links_over_gloo(nts):
    world = len(nts)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, nts, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, front, back, total, ok_links in res:
        prev, nxt = (rank - 1) % world, (rank + 1) % world
        assert front == 10 * prev + nts[prev] - 1          # previous rank's last slice
        assert back == 10 * nxt                              # next rank's first slice
        assert total == pytest.approx(sum(r + 0.5 for r in range(world)))
        assert ok_links                                      # equal to the cut of the global links


def test_thread_transport_matches():
    nts = [2, 4, 6]
    hub = ThreadHub(len(nts), timeout=30)
    res = {}

    def run(rank):
        split = TSplit(LAT, nts, rank)
        comm = ThreadComm(hub, rank)
        buf = _pattern(split, 16)
        comm.exchange(split, *_slices(buf, split.nt))
        res[rank] = (int(buf[(split.nt + 1) * 16]), int(buf[split.nt * 16]), comm.sum(2.0 ** rank))

    ths = [threading.Thread(target=run, args=(r,)) for r in range(len(nts))]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=60)
    assert len(res) == 3
    for rank, (front, back, total) in res.items():
        prev, nxt = (rank - 1) % 3, (rank + 1) % 3
        assert front == 10 * prev + nts[prev] - 1
        assert back == 10 * nxt
        assert total == 7.0


def test_single_rank_wraps_onto_itself():
    dist_ok = False
    try:
        if not dist.is_initialized():
            dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0,
                                    world_size=1, timeout=datetime.timedelta(seconds=30))
            dist_ok = True
        split = TSplit(LAT, [12], 0)
        buf = _pattern(split, 8)
        TorchComm().exchange(split, *_slices(buf, split.nt))
        assert int(buf[(split.nt + 1) * 8]) == 11 and int(buf[split.nt * 8]) == 0
    finally:
        if dist_ok:
            dist.destroy_process_group()
