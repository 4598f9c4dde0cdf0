"""Row-partitioned vectors and matrices over several ranks, as HiFlow3's
CoupledVector / CoupledMatrix (linear_algebra/coupled_vector.cc,
coupled_matrix.cc) lay them out, with the CG<LAD> recurrence over them.

* LaCouplings: each rank owns a contiguous block of the global rows
  (la_couplings.h), given by the offsets of all ranks.
* CoupledMatrix: the rank's rows split into the diagonal block (columns the
  rank owns, renumbered locally) and the off-diagonal block (columns owned by
  others, renumbered into the rank's ghost vector, sorted by global index),
  as CoupledMatrix::Init / diagonal() / offdiagonal() hold them.
  VectorMult (coupled_matrix.cc:327-362): exchange the ghosts, y = A_diag x,
  then y += A_offdiag x_ghost.
* CoupledVector: the owned values (interior) and the ghost values; Dot is the
  local Dot summed over the ranks (coupled_vector.cc:296-311); UpdateGhost
  (:994) sends every peer the owned values it reads and receives this rank's
  ghosts (SendBorder / ReceiveGhost, :890-973).
* CoupledCG: CG<LAD>::SolvePrecond / SolveNoPrecond (linear_solver/cg.h:
  87-246) over those, with the block-Jacobi(Jacobi) preconditioner on the
  diagonal block (preconditioner_bjacobi_standard.cc:188-196).

The local work runs on the backend's vectors and matrices (ba_b200.lmp's B200
classes on the device); the communicator carries the halo and the sums.
TorchComm uses a torch.distributed process group (one process per rank);
ThreadComm runs the ranks as threads of one process, each with its own device
context, for tests on one device.

The halo has two forms.  Host-staged (as the reference stages its MPI halo
through host buffers): GetValues / SetValues of the device vectors around a
host exchange.  Device-resident (device_halo=True): the owned values every
peer reads are gathered on the device into one send buffer (b200la_vec_gather),
the buffers move device to device -- NCCL send/recv on an NCCL group, or
device copies between thread ranks -- and the received values are scattered
into the ghost vector on the device (b200la_vec_scatter).  The CG's two dot
products after the update (r.r and r.z) go to the ranks in one all-reduce.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass, field

import numpy as np


# ---------------------------------------------------------------- communicators
class ThreadComm:
    """Ranks as threads of one process: mailboxes and a barrier.  Build one
    shared ThreadComm.World(size) and give each thread world.comm(rank)."""

    class World:
        def __init__(self, size: int):
            self.size = size
            self.barrier = threading.Barrier(size)
            self.box = {}
            self.lock = threading.Lock()

        def comm(self, rank: int, device_halo: bool = False) -> "ThreadComm":
            return ThreadComm(self, rank, device_halo)

    def __init__(self, world: "ThreadComm.World", rank: int, device_halo: bool = False):
        self.world, self.rank, self.size = world, rank, world.size
        self.device_halo = bool(device_halo)

    def _post(self, key, value):
        with self.world.lock:
            self.world.box[key] = value

    def allgather(self, obj, tag="ag"):
        self._post((tag, self.rank), obj)
        self.world.barrier.wait()
        out = [self.world.box[(tag, r)] for r in range(self.size)]
        self.world.barrier.wait()
        if self.rank == 0:
            with self.world.lock:
                for r in range(self.size):
                    self.world.box.pop((tag, r))
        self.world.barrier.wait()
        return out

    def allreduce_sum(self, value: float) -> float:
        # every rank adds the same values in rank order: identical results
        return float(sum(self.allgather(float(value), "sum")))

    def allreduce_sum_many(self, values) -> list:
        parts = self.allgather([float(v) for v in values], "sums")
        return [float(sum(p[k] for p in parts)) for k in range(len(values))]

    def exchange_device(self, halo: "DeviceHalo"):
        """Device halo between thread ranks on one device: each rank's send
        buffer is complete (its context stream synchronised) before any peer
        copies from it, and stays untouched until every peer has copied."""
        import torch
        halo.sync()
        self._post(("dh", self.rank), halo)
        self.world.barrier.wait()
        with self.world.lock:
            peers = {q: self.world.box[("dh", q)] for q in halo.recv_seg}
        for q, (o, n) in halo.recv_seg.items():
            so, sn = peers[q].send_seg[self.rank]
            assert sn == n
            halo.recv_buf[o:o + n].copy_(peers[q].send_buf[so:so + sn])
        torch.cuda.synchronize()
        self.world.barrier.wait()
        if self.rank == 0:
            with self.world.lock:
                for r in range(self.size):
                    self.world.box.pop(("dh", r), None)
        self.world.barrier.wait()

    def exchange(self, send: dict, recv_sizes: dict) -> dict:
        for q, arr in send.items():
            self._post(("x", self.rank, q), np.asarray(arr))
        self.world.barrier.wait()
        recv = {}
        with self.world.lock:
            for (t, src, dst), v in list(self.world.box.items()):
                if t == "x" and dst == self.rank:
                    recv[src] = self.world.box.pop((t, src, dst))
        self.world.barrier.wait()
        return recv


class TorchComm:
    """One process per rank over torch.distributed.  Sums run as an
    all-reduce of float64 on `group` (NCCL with device tensors, or gloo); the
    halo is exchanged through host buffers with point-to-point sends on a gloo
    group (`halo_group`, default: the world group when it is gloo)."""

    def __init__(self, group=None, halo_group=None, device=None, device_halo=False):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.halo_group = halo_group if halo_group is not None else group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.device = device
        # device_halo: buffers move device to device over `group` (NCCL), and
        # the B200 contexts must run on torch's current stream, so the gather
        # kernel precedes the sends and the scatter follows the receives
        self.device_halo = bool(device_halo)

    def allreduce_sum_many(self, values) -> list:
        import torch
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return [float(v) for v in t.tolist()]

    def exchange_device(self, halo: "DeviceHalo"):
        ops = []
        for q, (o, n) in halo.send_seg.items():
            ops.append(self.dist.P2POp(self.dist.isend, halo.send_buf[o:o + n], q, group=self.group))
        for q, (o, n) in halo.recv_seg.items():
            ops.append(self.dist.P2POp(self.dist.irecv, halo.recv_buf[o:o + n], q, group=self.group))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()

    def allgather(self, obj, tag="ag"):
        out = [None] * self.size
        self.dist.all_gather_object(out, obj, group=self.halo_group)
        return out

    def allreduce_sum(self, value: float) -> float:
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def exchange(self, send: dict, recv_sizes: dict) -> dict:
        import torch
        peers = sorted(set(send) | set(recv_sizes))
        ops = []
        recv = {}
        for q in peers:
            if q in send:
                ops.append(self.dist.P2POp(self.dist.isend, torch.from_numpy(np.ascontiguousarray(send[q],
                                                                                                   np.float64)),
                                           q, group=self.halo_group))
            if q in recv_sizes:
                recv[q] = torch.empty(int(recv_sizes[q]), dtype=torch.float64)
                ops.append(self.dist.P2POp(self.dist.irecv, recv[q], q, group=self.halo_group))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        return {q: t.numpy() for q, t in recv.items()}


# ---------------------------------------------------------------- couplings and plan
@dataclass
class LaCouplings:
    """Row ownership: rank r owns global rows offsets[r] .. offsets[r+1]-1."""
    offsets: np.ndarray

    @staticmethod
    def balanced(n: int, size: int) -> "LaCouplings":
        return LaCouplings(np.array([(n * r) // size for r in range(size + 1)], dtype=np.int64))

    def owner(self, rows: np.ndarray) -> np.ndarray:
        return np.searchsorted(self.offsets, rows, side="right") - 1


def split_rows(rowptr, col, val, begin: int, end: int):
    """The rows begin..end-1 of a global CSR split into the diagonal block
    (owned columns, renumbered from 0) and the off-diagonal block (other
    columns, numbered by their position in the sorted ghost list), keeping the
    stored order within each row.  Returns (diag, offdiag, ghosts) with diag
    and offdiag as (rowptr, col, val)."""
    rp = np.asarray(rowptr, np.int64)
    lo, hi = int(rp[begin]), int(rp[end])
    c = np.asarray(col[lo:hi], np.int64)
    v = np.asarray(val[lo:hi])
    counts = np.diff(rp[begin:end + 1])
    rows = np.repeat(np.arange(end - begin), counts)
    own = (c >= begin) & (c < end)
    ghosts = np.unique(c[~own])
    d_rp = np.zeros(end - begin + 1, np.int32)
    np.cumsum(np.bincount(rows[own], minlength=end - begin), out=d_rp[1:])
    o_rp = np.zeros(end - begin + 1, np.int32)
    np.cumsum(np.bincount(rows[~own], minlength=end - begin), out=o_rp[1:])
    diag = (d_rp, (c[own] - begin).astype(np.int32), v[own])
    off = (o_rp, np.searchsorted(ghosts, c[~own]).astype(np.int32), v[~own])
    return diag, off, ghosts


@dataclass
class HaloPlan:
    """Who sends what: recv[q] = positions in this rank's ghost vector of the
    values rank q owns; send[q] = local indices of owned values rank q reads."""
    recv: dict = field(default_factory=dict)
    send: dict = field(default_factory=dict)
    device: "DeviceHalo | None" = None  # the device form, built at the first device exchange

    @staticmethod
    def build(comm, couplings: LaCouplings, ghosts: np.ndarray) -> "HaloPlan":
        plan = HaloPlan()
        owners = couplings.owner(ghosts)
        requests = {}
        for q in np.unique(owners):
            pos = np.nonzero(owners == q)[0]
            plan.recv[int(q)] = pos.astype(np.int32)
            requests[int(q)] = ghosts[pos]
        everyone = comm.allgather(requests, "halo")
        begin = int(couplings.offsets[comm.rank])
        for q, req in enumerate(everyone):
            if comm.rank in req:
                plan.send[q] = (np.asarray(req[comm.rank]) - begin).astype(np.int32)
        return plan


class DeviceHalo:
    """A rank's halo plan on the device: device int32 indices of the owned
    values each peer reads (one segment per peer, peers in ascending order)
    and of the ghost positions each peer fills, with one device send and one
    device receive buffer of float64."""

    def __init__(self, plan: HaloPlan, platform):
        import torch
        from . import _lib
        dev = torch.device("cuda", platform.device)
        self.platform = platform
        self.send_seg, self.recv_seg = {}, {}
        send_idx, recv_idx = [], []
        o = 0
        for q in sorted(plan.send):
            self.send_seg[q] = (o, len(plan.send[q]))
            send_idx.append(np.asarray(plan.send[q], np.int32))
            o += len(plan.send[q])
        self.send_idx = torch.from_numpy(np.concatenate(send_idx) if send_idx else np.zeros(0, np.int32)).to(dev)
        self.send_buf = torch.empty(o, dtype=torch.float64, device=dev)
        o = 0
        for q in sorted(plan.recv):
            self.recv_seg[q] = (o, len(plan.recv[q]))
            recv_idx.append(np.asarray(plan.recv[q], np.int32))
            o += len(plan.recv[q])
        self.recv_idx = torch.from_numpy(np.concatenate(recv_idx) if recv_idx else np.zeros(0, np.int32)).to(dev)
        self.recv_buf = torch.empty(o, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        self._lib = _lib

    def sync(self):
        self._lib.call("b200la_ctx_synchronize", self.platform.handle)

    def pack(self, interior):
        import ctypes as C
        self._lib.call("b200la_vec_gather", interior.handle, C.c_void_p(self.send_idx.data_ptr()),
                       int(self.send_idx.numel()), C.c_void_p(self.send_buf.data_ptr()))

    def unpack(self, ghost):
        import ctypes as C
        self._lib.call("b200la_vec_scatter", ghost.handle, C.c_void_p(self.recv_idx.data_ptr()),
                       int(self.recv_idx.numel()), C.c_void_p(self.recv_buf.data_ptr()))


# ---------------------------------------------------------------- coupled objects
class CoupledVector:
    """Owned values (interior) and ghost values of one rank."""

    def __init__(self, comm, couplings: LaCouplings, plan: HaloPlan, n_ghost: int, make_vector):
        self.comm, self.couplings, self.plan = comm, couplings, plan
        begin, end = (int(x) for x in couplings.offsets[comm.rank:comm.rank + 2])
        self.interior = make_vector(end - begin)
        self.ghost = make_vector(n_ghost) if n_ghost > 0 else None
        self._make = make_vector
        self.n_ghost = n_ghost

    def CloneWithoutContent(self) -> "CoupledVector":
        return CoupledVector(self.comm, self.couplings, self.plan, self.n_ghost, self._make)

    def UpdateGhost(self):
        if getattr(self.comm, "device_halo", False):
            if self.plan.device is None:
                self.plan.device = DeviceHalo(self.plan, self.interior.platform)
            self.plan.device.pack(self.interior)
            self.comm.exchange_device(self.plan.device)
            if self.ghost is not None:
                self.plan.device.unpack(self.ghost)
            return
        send = {q: self.interior.GetValues(idx) for q, idx in self.plan.send.items()}
        recv = self.comm.exchange(send, {q: len(pos) for q, pos in self.plan.recv.items()})
        for q, pos in self.plan.recv.items():
            self.ghost.SetValues(pos, recv[q])

    def Dot(self, other: "CoupledVector") -> float:
        return self.comm.allreduce_sum(self.interior.Dot(other.interior))

    def DotMany(self, pairs) -> list:
        """Several dot products summed over the ranks in one all-reduce."""
        return self.comm.allreduce_sum_many([a.interior.Dot(b.interior) for a, b in pairs])

    def Norm2(self) -> float:
        return float(np.sqrt(self.Dot(self)))

    def Axpy(self, other: "CoupledVector", a: float):
        self.interior.Axpy(other.interior, a)

    def ScaleAdd(self, other: "CoupledVector", a: float):
        # coupled ScaleAdd(vec, alpha) -> interior ScaleAdd(alpha, vec) (coupled_vector.cc:353-358)
        self.interior.ScaleAdd(a, other.interior)

    def CopyFrom(self, other: "CoupledVector"):
        self.interior.CopyFrom(other.interior)

    def Zeros(self):
        self.interior.Zeros()


class CoupledMatrix:
    """One rank's rows of a global CSR: diagonal and off-diagonal blocks."""

    def __init__(self, comm, couplings: LaCouplings, rowptr, col, val, make_matrix, make_vector):
        self.comm, self.couplings = comm, couplings
        begin, end = (int(x) for x in couplings.offsets[comm.rank:comm.rank + 2])
        diag, off, ghosts = split_rows(rowptr, col, val, begin, end)
        self.ghosts = ghosts
        self.plan = HaloPlan.build(comm, couplings, ghosts)
        self.diag = make_matrix(*diag, end - begin)
        self.offdiag = make_matrix(*off, len(ghosts)) if len(off[1]) > 0 else None
        self._make_vector = make_vector

    def vector(self) -> CoupledVector:
        return CoupledVector(self.comm, self.couplings, self.plan, len(self.ghosts), self._make_vector)

    def VectorMult(self, x: CoupledVector, y: CoupledVector):
        if self.offdiag is not None or self.plan.send:
            x.UpdateGhost()
        self.diag.VectorMult(x.interior, y.interior)
        if self.offdiag is not None:
            self.offdiag.VectorMultAdd(x.ghost, y.interior)


@dataclass
class CoupledCGResult:
    iters: int
    res: float
    res_init: float
    state: int


def coupled_cg(A: CoupledMatrix, b: CoupledVector, x: CoupledVector, *, maxits=1000, atol=1e-12, rtol=1e-8,
               dtol=1e8, precond=True) -> CoupledCGResult:
    """CG<LAD>::SolvePrecond / SolveNoPrecond (linear_solver/cg.h:87-246) over
    coupled objects; stopping test IterateControl::Check
    (common/iterate_control.cc:80-107): 1 success (abs), 2 (rel), 3 divergence,
    4 maxits."""
    def check(step, res, first):
        if res <= atol:
            return 1
        if res < rtol * first:
            return 2
        if res > dtol * first:
            return 3
        if step >= maxits:
            return 4
        return 0

    r, p, Ap = b.CloneWithoutContent(), b.CloneWithoutContent(), b.CloneWithoutContent()
    z = b.CloneWithoutContent() if precond else None
    invd = None
    if precond:
        invd = b.CloneWithoutContent()
        A.diag.extract_invdiagelements(invd.interior)
    A.VectorMult(x, r)
    r.ScaleAdd(b, -1.0)                      # r = b - A x
    ressq = r.Dot(r)
    res = float(np.sqrt(ressq))
    first = res
    state = check(0, res, first)
    if precond:
        z.CopyFrom(r)
        z.interior.ElementWiseMult(invd.interior)
        p.CopyFrom(z)
        beta = r.Dot(z)
    else:
        p.CopyFrom(r)
        beta = ressq
    it = 0
    while state == 0:
        it += 1
        A.VectorMult(p, Ap)
        alpha = beta / Ap.Dot(p)
        x.Axpy(p, alpha)
        r.Axpy(Ap, -alpha)
        if precond:
            # r.r (the test) and r.z (the next beta) in one all-reduce
            z.CopyFrom(r)
            z.interior.ElementWiseMult(invd.interior)
            ressq, gamma = r.DotMany([(r, r), (r, z)])
        else:
            ressq = r.Dot(r)
        res = float(np.sqrt(ressq))
        state = check(it, res, first)
        if state != 0:
            break
        if precond:
            p.ScaleAdd(z, gamma / beta)      # p = (gamma / beta) p + z
            beta = gamma
        else:
            p.ScaleAdd(r, ressq / beta)
            beta = ressq
    return CoupledCGResult(it, res, first, state)


def device_backend(platform):
    """make_matrix / make_vector for ba_b200.lmp's B200 classes on `platform`."""
    from . import lmp

    def make_vector(n):
        return lmp.B200_lVector(n, platform=platform)

    def make_matrix(rp, c, v, ncol):
        return lmp.B200_CSR_lMatrix(rp, c, v, num_col=ncol, platform=platform)
    return make_matrix, make_vector
