"""Halo exchange: the domain-wall operator on a lattice split along t.

Replaces the reference's multi-rank path of AFopr_Domainwall_5din_eo: each
D_eo / D_eo^dag packs the spin-projected faces of its input, exchanges them
with the neighbouring ranks over persistent MPI channels from host buffers
and finishes the boundary sites after the bulk
(src/lib_alt_Accel/Fopr/afopr_Domainwall_5din_eo-tmpl.h:998-1101 and
1126-1228; channels: src/lib/Communicator/MPI/channel.cpp:36-150), and the
fermion force reads the shifted fields across the same boundaries.

Design: one process per GPU owns nt consecutive t-slices (nt even, so its
first global t is even and every site keeps its global parity).  Its plan
is an ordinary DomainWall on the periodic lattice {Lx, Ly, Lz, nt + 2}
whose slices are its own nt slices, then the next rank's first slice (the
back ghost), then the previous rank's last slice (the front ghost).  The
kernels then read the previous rank's slice through their t wrap; a hop
launch covers only the rank's own slices (the two ghost slices of its
output stay unwritten).  The global t
boundary phase is folded into the global last slice's t links (the force
kernels apply the phase themselves to their link-free outer products, so
the rank owning that slice applies it to those links' forces).  Before each
hop and before the force kernels the plan calls this module's exchange hook
(b200_dwf_set_halo_exchange) for every field they read at neighbouring
sites.  Since t is the slowest site index, each ghost slice is one
contiguous range of (Lx Ly Lz / 2) site columns: the hook sends the field's
first and last interior slices as they lie, with no pack kernel, through
torch.distributed point-to-point calls (NCCL between GPUs, ordered on the
plan's stream).  With overlap=True the hook comes in two halves
(b200_dwf_set_halo_exchange_split): the transfer starts, the hop runs the
sites whose t neighbours are the rank's own (t = 1 .. nt-2), the plan's
stream waits for the transfer, and the two edge slices run last, as the
reference overlaps its bulk hop with the face exchange.  A face carries full
24 Ls-real columns, twice the reference's spin-projected half spinors; at
24^3 x 48 x 16 one FP64 face is 21 MB (about 27 us over NVLink beside a
700 us hop).

The solvers and reductions of the plan would cover only the rank's
extended lattice, so the plan refuses them; HaloDomainWall supplies the
global reductions and a distributed CG (ASolver_CG,
src/lib/Solver/asolver_CG-tmpl.h) on its own kernels.

ThreadComm runs several ranks as threads of one process on one GPU, for the
tests: each exchange synchronises the device, meets the other ranks at a
host barrier, copies the neighbours' edge slices and meets them again, so no
kernel ever waits for another.
"""
import ctypes
import threading

import numpy as np

from . import F64, HALO_FN, B200Error, DomainWall, check, lib


class TSplit:
    """Rank `rank` of a lattice split along t into consecutive slabs of
    nts[r] slices (each even, at least 2; sum(nts) = Lt)."""

    def __init__(self, lattice, nts, rank):
        lattice = [int(v) for v in lattice]
        nts = [int(v) for v in nts]
        if sum(nts) != lattice[3]:
            raise ValueError("the slabs' t extents must add up to Lt = %d" % lattice[3])
        if any(n < 2 or n % 2 for n in nts):
            raise ValueError("every slab needs an even number (>= 2) of t slices")
        if not 0 <= rank < len(nts):
            raise ValueError("rank %d outside 0..%d" % (rank, len(nts) - 1))
        self.lattice = lattice
        self.nts = nts
        self.rank = rank
        self.nranks = len(nts)
        self.nt = nts[rank]
        self.t0 = sum(nts[:rank])
        self.ext = lattice[:3] + [self.nt + 2]
        self.vol3 = lattice[0] * lattice[1] * lattice[2]
        self.prev = (rank - 1) % self.nranks
        self.next = (rank + 1) % self.nranks
        T = lattice[3]
        # global t of each extended slice: interior, back ghost, front ghost
        self.ext_t = [self.t0 + i for i in range(self.nt)] + [(self.t0 + self.nt) % T,
                                                              (self.t0 - 1) % T]

    @classmethod
    def even(cls, lattice, nranks, rank):
        """Equal slabs of Lt / nranks slices."""
        if lattice[3] % nranks:
            raise ValueError("Lt = %d is not a multiple of %d ranks" % (lattice[3], nranks))
        return cls(lattice, [lattice[3] // nranks] * nranks, rank)

    @property
    def nvol_half(self):
        """Interior sites of one parity."""
        return self.vol3 * self.nt // 2

    def gauge(self, u_global, bc_t):
        """This rank's extended lexical links (Field_G(Nvol_ext, 4)) cut from
        the global ones, the t boundary phase bc_t folded into the global
        last slice's t links."""
        T = self.lattice[3]
        u = np.array(u_global, dtype=np.float64).reshape(4, T, self.vol3, 18)
        u[3, T - 1] *= bc_t
        return np.ascontiguousarray(u[:, self.ext_t]).reshape(-1)

    def spinor(self, w_global, Ls):
        """This rank's extended half-lattice spinor (Field(24, Nvol_ext/2, Ls))
        cut from a global one; its ghost slices already hold the neighbours'
        edge slices."""
        w = np.asarray(w_global, dtype=np.float64).reshape(Ls, self.lattice[3], self.vol3 // 2, 24)
        return np.ascontiguousarray(w[:, self.ext_t]).reshape(-1)

    def interior_spinor(self, w_ext, Ls):
        """The interior slices of an extended spinor, as (Ls, nt, Lx Ly Lz / 2, 24)."""
        return np.asarray(w_ext).reshape(Ls, self.nt + 2, self.vol3 // 2, 24)[:, :self.nt]

    def interior_links(self, f_ext):
        """The interior slices of an extended lexical link field, as (4, nt, Lx Ly Lz, 18)."""
        return np.asarray(f_ext).reshape(4, self.nt + 2, self.vol3, 18)[:, :self.nt]


def assemble_spinor(parts, Ls):
    """Global half-lattice spinor from the ranks' interior_spinor parts (rank order)."""
    return np.ascontiguousarray(np.concatenate(parts, axis=1)).reshape(-1)


def assemble_links(parts):
    """Global lexical link field from the ranks' interior_links parts (rank order)."""
    return np.ascontiguousarray(np.concatenate(parts, axis=1)).reshape(-1)


def _slices(buf, nt):
    """first, last interior slice and back, front ghost of an extended field
    held as a flat tensor whose t slices are equal consecutive ranges."""
    sb = buf.numel() // (nt + 2)
    return (buf[:sb], buf[(nt - 1) * sb:nt * sb], buf[nt * sb:(nt + 1) * sb],
            buf[(nt + 1) * sb:(nt + 2) * sb])


class TorchComm:
    """Ghost exchange and global sums over torch.distributed: NCCL for CUDA
    tensors between GPUs, gloo for CPU tensors.  The split's ranks are the
    group's ranks."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.nccl = dist.get_backend(group) == "nccl"

    def start(self, split, first, last, back, front):
        """Begin: front <- previous rank's last slice, back <- next rank's
        first slice (every rank calls this with tensors of its own extended
        field), ordered after the work on the current stream; returns what
        finish() waits for."""
        if split.nranks != self.size or split.rank != self.rank:
            raise B200Error("the split's ranks are not this group's ranks")
        if self.size == 1:
            front.copy_(last)
            back.copy_(first)
            return []
        d = self.dist
        ops = [d.P2POp(d.isend, last, split.next, self.group, 0),
               d.P2POp(d.irecv, front, split.prev, self.group, 0),
               d.P2POp(d.isend, first, split.prev, self.group, 1),
               d.P2POp(d.irecv, back, split.next, self.group, 1)]
        return d.batch_isend_irecv(ops)

    def finish(self, reqs):
        """The current stream (NCCL) or the host (gloo) waits for start()'s transfers."""
        for req in reqs:
            req.wait()

    def exchange(self, split, first, last, back, front):
        self.finish(self.start(split, first, last, back, front))

    def sum(self, x):
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.nccl else "cpu")
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())


class ThreadHub:
    """Meeting point of ranks run as threads of one process (ThreadComm)."""

    def __init__(self, nranks, timeout=300.0):
        self.barrier = threading.Barrier(nranks, timeout=timeout)
        self.slots = [None] * nranks


class ThreadComm:
    """Ranks as threads of one process on one GPU: every exchange and sum
    meets the other ranks at a host barrier; no kernel waits for another."""

    def __init__(self, hub, rank):
        self.hub = hub
        self.rank = rank

    def exchange(self, split, first, last, back, front):
        import torch
        hub = self.hub
        if first.is_cuda:
            torch.cuda.synchronize()          # this rank's field is complete
        hub.slots[self.rank] = (first, last)
        hub.barrier.wait()
        front.copy_(hub.slots[split.prev][1])
        back.copy_(hub.slots[split.next][0])
        if first.is_cuda:
            torch.cuda.synchronize()
        hub.barrier.wait()                    # nobody overwrites a slice still being read

    # the host-synchronised exchange cannot overlap anything: start does it all
    def start(self, split, first, last, back, front):
        self.exchange(split, first, last, back, front)
        return []

    def finish(self, reqs):
        pass

    def sum(self, x):
        hub = self.hub
        hub.slots[self.rank] = float(x)
        hub.barrier.wait()
        total = 0.0
        for v in hub.slots:                   # rank order: every rank gets the same value
            total += v
        hub.barrier.wait()
        return total


class _CudaBytes:
    """A device byte range for torch.as_tensor (no copy)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3}


def extend_links(split, comm, u_local, bc_t, device="cuda"):
    """Extended lexical links of this rank from its own links alone: u_local
    is Field_G(Vol3 * nt, 4) (lexical, this rank's slices); the global t
    boundary phase is folded on the rank owning the last slice, then the
    ghost slices come from the neighbours through `comm`.  Returns a flat
    float64 tensor on `device`."""
    import torch
    nt, v3 = split.nt, split.vol3
    u = torch.as_tensor(np.asarray(u_local, dtype=np.float64)).reshape(4, nt, v3 * 18)
    ext = torch.zeros((4, nt + 2, v3 * 18), dtype=torch.float64, device=device)
    ext[:, :nt] = u.to(device)
    if split.t0 + nt == split.lattice[3]:
        ext[3, nt - 1] *= bc_t
    for mu in range(4):
        plane = ext[mu].reshape(-1)
        comm.exchange(split, *_slices(plane, nt))
    return ext.reshape(-1)


class HaloDomainWall:
    """This rank's share of DomainWall on a lattice split along t.

    mult / mult_dag take every mode of DomainWall and the force entry points
    return this rank's interior link forces; fields live on the extended
    lattice (new_field), their ghost slices filled by the plan's exchange
    hook when a stencil reads them.  overlap=True splits each exchange
    around the hop's interior sites.  norm2, dot and cg are global over the
    ranks."""

    def __init__(self, split, comm, Ls, mq, M0, b=1.0, c=0.0, alpha=1.0, bc=(1, 1, 1, -1),
                 overlap=False):
        self.split = split
        self.comm = comm
        self.Ls = Ls
        self.bc_t = bc[3]
        self.overlap = bool(overlap)
        self.op = DomainWall(split.ext, Ls, mq, M0, b, c, alpha, bc=(bc[0], bc[1], bc[2], 1))
        self._err = None
        self._pending = {}
        # the hooks are kept alive with the plan
        if self.overlap:
            self._hooks = (HALO_FN(self._start), HALO_FN(self._finish))
            check(lib().b200_dwf_set_halo_exchange_split(self.op.handle, *self._hooks, None))
        else:
            self._hooks = (HALO_FN(self._exchange),)
            check(lib().b200_dwf_set_halo_exchange(self.op.handle, self._hooks[0], None))
        self.n_interior = 24 * Ls * split.nvol_half   # reals of one parity's interior

    def close(self):
        if self.op is not None:
            if self.overlap:
                check(lib().b200_dwf_set_halo_exchange_split(self.op.handle, HALO_FN(), HALO_FN(),
                                                             None))
            else:
                check(lib().b200_dwf_set_halo_exchange(self.op.handle, HALO_FN(), None))
            self.op = None

    # the hooks --------------------------------------------------------
    def _views(self, field, prec):
        import torch
        nbytes = lib().b200_dwf_field_bytes(self.op.handle, prec)
        buf = torch.as_tensor(_CudaBytes(field, nbytes), device="cuda")
        return _slices(buf, self.split.nt)

    def _on_stream(self, stream, fn):
        import torch
        if stream:
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                return fn()
        return fn()

    def _exchange(self, ctx, field, prec, stream):
        try:
            views = self._views(field, prec)
            self._on_stream(stream, lambda: self.comm.exchange(self.split, *views))
            return 0
        except BaseException as e:                     # reported by _call
            self._err = e
            return 1

    def _start(self, ctx, field, prec, stream):
        try:
            views = self._views(field, prec)
            reqs = self._on_stream(stream, lambda: self.comm.start(self.split, *views))
            self._pending[field] = (views, reqs)       # the views live until finish
            return 0
        except BaseException as e:
            self._err = e
            return 1

    def _finish(self, ctx, field, prec, stream):
        try:
            _, reqs = self._pending.pop(field)
            self._on_stream(stream, lambda: self.comm.finish(reqs))
            return 0
        except BaseException as e:
            self._err = e
            return 1

    def _call(self, rc):
        if rc != 0 and self._err is not None:
            err, self._err = self._err, None
            raise B200Error("halo exchange failed: %r" % (err,)) from err
        check(rc)

    # operator -----------------------------------------------------------
    def set_config(self, u_ext):
        """Extended lexical links with the t phase folded (TSplit.gauge or
        extend_links)."""
        import torch
        if isinstance(u_ext, torch.Tensor):
            u_ext = u_ext.cpu().numpy()
        self.op.set_config(u_ext)

    def new_field(self, prec=F64):
        return self.op.new_field(prec)

    def convert(self, v, w_ext):
        self.op.convert(v, w_ext)

    def reverse(self, w):
        """This rank's interior slices, (Ls, nt, Lx Ly Lz / 2, 24)."""
        return self.split.interior_spinor(self.op.reverse(w), self.Ls).copy()

    def mult(self, v, w, mode):
        self._call(lib().b200_dwf_mult(self.op.handle, w.prec, v.ptr, w.ptr, mode.encode(), 0, None))

    def mult_dag(self, v, w, mode):
        self._call(lib().b200_dwf_mult(self.op.handle, w.prec, v.ptr, w.ptr, mode.encode(), 1, None))

    def _force_out(self):
        import torch
        return torch.empty(18 * 2 * self.op.nvol * 4, dtype=torch.float64, device="cuda")

    def _interior_force(self, f):
        # the force kernels form link-free outer products and apply the
        # boundary phase of the x -> x+t hop themselves; the plan's t
        # boundary is periodic, so the rank owning the global last slice
        # applies bc_t to that slice's t-link forces
        out = self.split.interior_links(f.cpu().numpy()).copy()
        if self.split.t0 + self.split.nt == self.split.lattice[3]:
            out[3, self.split.nt - 1] *= self.bc_t
        return out

    def force_udiv1(self, mode, a, b):
        """Interior link forces, (4, nt, Lx Ly Lz, 18)."""
        f = self._force_out()
        self._call(lib().b200_dwf_force_udiv1(self.op.handle, mode.encode(), ctypes.c_void_p(f.data_ptr()),
                                              a.ptr, b.ptr, None))
        return self._interior_force(f)

    def force_udiv(self, eta):
        f = self._force_out()
        self._call(lib().b200_dwf_force_udiv(self.op.handle, ctypes.c_void_p(f.data_ptr()), eta.ptr, None))
        return self._interior_force(f)

    # global reductions and CG (FP64 fields) ----------------------------
    def _flat(self, f):
        if f.prec != F64:
            raise B200Error("global reductions and cg take FP64 fields")
        return f.ptr

    def dot(self, x, y):
        r = ctypes.c_double()
        check(lib().b200_blas_dot(0, self.n_interior, self._flat(x), self._flat(y), ctypes.byref(r), None))
        return self.comm.sum(r.value)

    def norm2(self, x):
        return self.dot(x, x)

    def _axpby(self, y, a, x, b):
        check(lib().b200_blas_axpby(0, self.n_interior, a, self._flat(x) if x is not None else None, b,
                                    self._flat(y), None))

    def cg(self, x, b, tol2, maxiter=10000):
        """CG on DdagD from x = 0, stopped when |r|^2 < tol2 |b|^2 (the
        recursive residual), as ASolver_CG (src/lib/Solver/asolver_CG-tmpl.h);
        returns (iterations, |b - DdagD x| / |b|, 0 or B200_ENOCONV)."""
        r, p, q = self.new_field(), self.new_field(), self.new_field()
        x.zero()
        self._axpby(r, 1.0, b, 0.0)
        self._axpby(p, 1.0, b, 0.0)
        bb = self.norm2(b)
        rr = bb
        n, rc = 0, -4
        if bb == 0.0:
            return 0, 0.0, 0
        for n in range(1, maxiter + 1):
            self.mult(q, p, "DdagD")
            alpha = rr / self.dot(p, q)
            self._axpby(x, alpha, p, 1.0)
            self._axpby(r, -alpha, q, 1.0)
            rr_new = self.norm2(r)
            if rr_new < tol2 * bb:
                rc = 0
                break
            self._axpby(p, 1.0, r, rr_new / rr)
            rr = rr_new
        self.mult(q, x, "DdagD")
        self._axpby(q, 1.0, b, -1.0)
        return n, float(np.sqrt(self.norm2(q) / bb)), rc
