"""The domain-wall operator on a lattice split along t (b200dwf.halo) against
the same operator on the whole lattice, on one GPU.

The ranks run as threads of this process (ThreadComm): each owns a plan on
its extended slab, and the plan's exchange hook fills the ghost slices of
every field a stencil reads, meeting the other ranks at a host barrier, so
no kernel waits for another.  The slabs have different t extents, so no two
plans share a geometry (plans of one geometry share their work fields).
The inputs' ghost slices are filled with garbage first: every neighbour
value a rank uses must come through the hook.  Checked: all 13 modes x dag,
the force (force_udiv, force_udiv1 H / Hdag), with the exchange whole before
each hop and split around the interior sites (overlap), reduced-precision
storage, and the distributed CG against the plan's CG on the whole lattice."""
import threading

import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu

LAT, LS, MQ, M0 = [4, 4, 4, 12], 8, 0.04, 1.8
MODES = ["D", "Ddag", "DdagD", "H", "Hdag", "Deo", "Doe", "Dee", "Doo", "Dee_inv", "Doo_inv",
         "gm5R", "R"]
# (slab t extents, Moebius b, c)
SPLITS = [([4, 8], 1.0, 0.0), ([2, 4, 6], 1.5, 0.5)]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def run_ranks(nts, b, c, u, work, ls=LS, bc=(1, 1, 1, -1), overlap=False):
    """work(rank, split, hop) in one thread per rank; returns the results in
    rank order (re-raises the first failure)."""
    from b200dwf.halo import HaloDomainWall, ThreadComm, ThreadHub, TSplit
    hub = ThreadHub(len(nts), timeout=120)
    res, errs = {}, []

    def body(rank):
        try:
            split = TSplit(LAT, nts, rank)
            hop = HaloDomainWall(split, ThreadComm(hub, rank), ls, MQ, M0, b, c, bc=bc,
                                 overlap=overlap)
            hop.set_config(split.gauge(u, bc[3]))
            res[rank] = work(rank, split, hop)
            hop.close()
        except BaseException as e:
            errs.append(e)
            hub.barrier.abort()

    ths = [threading.Thread(target=body, args=(r,)) for r in range(len(nts))]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=600)
    if errs:
        raise errs[0]
    assert len(res) == len(nts)
    return [res[r] for r in range(len(nts))]


def spoiled(split, w, ls=LS):
    """The rank's extended input with garbage on its ghost slices."""
    ext = split.spinor(w, ls).reshape(ls, split.nt + 2, -1)
    rng = np.random.default_rng(99 + split.rank)
    ext[:, split.nt:] = 1e3 * rng.standard_normal(ext[:, split.nt:].shape)
    return ext.reshape(-1)


def whole(b, c, u):
    import b200dwf
    op = b200dwf.DomainWall(LAT, LS, MQ, M0, b, c)
    op.set_config(u)
    return op


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("nts,b,c", SPLITS)
def test_all_modes_match_the_whole_lattice(nts, b, c, overlap, monkeypatch):
    from b200dwf.halo import assemble_spinor
    monkeypatch.setenv("B200_HOP_VARIANT", "0")
    u = synth.gauge_field(LAT, 41, "hot")
    w = synth.spinor_field(LAT, LS, 42)
    op = whole(b, c, u)
    fw, fv = op.new_field(0), op.new_field(0)
    op.convert(fw, w)
    ref = {}
    for mode in MODES:
        for dag in (False, True):
            (op.mult_dag if dag else op.mult)(fv, fw, mode)
            ref[(mode, dag)] = op.reverse(fv)

    def work(rank, split, hop):
        out = {}
        gw, gv = hop.new_field(0), hop.new_field(0)
        for mode in MODES:
            for dag in (False, True):
                hop.convert(gw, spoiled(split, w))
                (hop.mult_dag if dag else hop.mult)(gv, gw, mode)
                out[(mode, dag)] = hop.reverse(gv)
        return out

    parts = run_ranks(nts, b, c, u, work, overlap=overlap)
    for key, r in ref.items():
        got = assemble_spinor([p[key] for p in parts], LS)
        assert rel(got, r) < 1e-14, (key, rel(got, r))


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("nts,b,c", SPLITS)
def test_force_matches_the_whole_lattice(nts, b, c, overlap):
    from b200dwf.halo import assemble_links
    u = synth.gauge_field(LAT, 43, "hot")
    eta = synth.spinor_field(LAT, LS, 44)
    zeta = synth.spinor_field(LAT, LS, 45)
    op = whole(b, c, u)
    fe, fz = op.new_field(0), op.new_field(0)
    op.convert(fe, eta)
    op.convert(fz, zeta)
    ref = [op.force_udiv(fe), op.force_udiv1("H", fz, fe), op.force_udiv1("Hdag", fe, fz)]

    def work(rank, split, hop):
        ge, gz = hop.new_field(0), hop.new_field(0)
        hop.convert(ge, spoiled(split, eta))
        hop.convert(gz, spoiled(split, zeta))
        return [hop.force_udiv(ge), hop.force_udiv1("H", gz, ge), hop.force_udiv1("Hdag", ge, gz)]

    parts = run_ranks(nts, b, c, u, work, overlap=overlap)
    for k in range(3):
        got = assemble_links([p[k] for p in parts])
        assert rel(got, ref[k]) < 1e-13, (k, rel(got, ref[k]))


@pytest.mark.parametrize("prec,tol", [(1, 1e-6), (2, 1e-3), (3, 1e-2)])
def test_reduced_precision_hop(prec, tol):
    """Deo and Deo^dag on f32 / f16 / bf16 storage: the split result against
    the whole-lattice result of the same storage (the same kernels on the
    same stored values)."""
    from b200dwf.halo import assemble_spinor
    nts, b, c = SPLITS[0]
    u = synth.gauge_field(LAT, 46, "hot")
    w = synth.spinor_field(LAT, LS, 47)
    op = whole(b, c, u)
    fw, fv = op.new_field(prec), op.new_field(prec)
    op.convert(fw, w)
    ref = []
    for dag in (False, True):
        (op.mult_dag if dag else op.mult)(fv, fw, "Deo")
        ref.append(op.reverse(fv))

    def work(rank, split, hop):
        gw, gv = hop.new_field(prec), hop.new_field(prec)
        hop.convert(gw, spoiled(split, w))
        out = []
        for dag in (False, True):
            (hop.mult_dag if dag else hop.mult)(gv, gw, "Deo")
            out.append(hop.reverse(gv))
        return out

    parts = run_ranks(nts, b, c, u, work)
    for k in range(2):
        got = assemble_spinor([p[k] for p in parts], LS)
        assert rel(got, ref[k]) < tol, (prec, k, rel(got, ref[k]))


def test_distributed_cg_matches_the_plan_cg():
    import b200dwf
    from b200dwf.halo import assemble_spinor
    nts, b, c = SPLITS[0]
    u = synth.gauge_field(LAT, 48, "near")
    rhs = synth.spinor_field(LAT, LS, 49)
    op = whole(b, c, u)
    fb, fx = op.new_field(0), op.new_field(0)
    op.convert(fb, rhs)
    n_ref, diff_ref, rc_ref = op.cg(fx, fb, 1e-20, 5000)
    assert rc_ref == 0
    x_ref = op.reverse(fx)

    def work(rank, split, hop):
        gb, gx = hop.new_field(0), hop.new_field(0)
        hop.convert(gb, spoiled(split, rhs))
        with pytest.raises(b200dwf.B200Error, match="halo exchange hook"):
            hop.op.cg(gx, gb, 1e-20, 10)              # the plan's own solver refuses
        with pytest.raises(b200dwf.B200Error, match="halo exchange hook"):
            b200dwf.LearnedPrecond(hop.op)            # and so does the learned preconditioner
        n, diff, rc = hop.cg(gx, gb, 1e-20, 5000)
        return n, diff, rc, hop.reverse(gx)

    parts = run_ranks(nts, b, c, u, work)
    for n, diff, rc, _ in parts:
        assert rc == 0 and abs(n - n_ref) <= 2, (n, n_ref)
        assert diff < 1e-9
    x = assemble_spinor([p[3] for p in parts], LS)
    assert rel(x, x_ref) < 1e-8


def test_ls12_and_antiperiodic_y():
    """Ls = 12 (the packed kernels leave lanes idle) with an antiperiodic y
    boundary, which the split passes through unchanged: hop, Schur operator
    and DdagD against the whole lattice."""
    import b200dwf
    from b200dwf.halo import assemble_spinor
    ls, bc = 12, (1, -1, 1, -1)
    nts, b, c = SPLITS[0]
    u = synth.gauge_field(LAT, 51, "hot")
    w = synth.spinor_field(LAT, ls, 52)
    op = b200dwf.DomainWall(LAT, ls, MQ, M0, b, c, bc=bc)
    op.set_config(u)
    fw, fv = op.new_field(0), op.new_field(0)
    op.convert(fw, w)
    modes = ("Deo", "Doe", "D", "DdagD")
    ref = {}
    for mode in modes:
        for dag in (False, True):
            (op.mult_dag if dag else op.mult)(fv, fw, mode)
            ref[(mode, dag)] = op.reverse(fv)

    def work(rank, split, hop):
        out = {}
        gw, gv = hop.new_field(0), hop.new_field(0)
        for mode in modes:
            for dag in (False, True):
                hop.convert(gw, spoiled(split, w, ls))
                (hop.mult_dag if dag else hop.mult)(gv, gw, mode)
                out[(mode, dag)] = hop.reverse(gv)
        return out

    parts = run_ranks(nts, b, c, u, work, ls=ls, bc=bc)
    for key, r in ref.items():
        got = assemble_spinor([p[key] for p in parts], ls)
        assert rel(got, r) < 1e-13, (key, rel(got, r))
