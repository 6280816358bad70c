"""Sharded assembly and solve over several GPUs (one process per GPU).

The reference runs on one device (FEM::Init picks one StiffAlgo, src/FEM/fem.cc:62-88);
this module splits the same problem by nodes:

* `partition` gives every node an owner rank: nodes sorted along the coordinate of
  largest extent and cut into equal contiguous runs (slabs).
* `build_shard` forms a rank's local mesh: every element touching an owned node (one
  halo layer of elements), its nodes renumbered owned-first, then halo nodes, both in
  ascending global order.  The owner-computes assembly of that mesh gives exact K rows
  for every owned node without any exchange; the halo rows are incomplete and unused.
* The send and receive lists of the halo exchange follow from the owner array alone:
  rank r sends to s the nodes it owns that lie in s's halo, in ascending global order,
  which is the order of s's halo nodes owned by r.  Set-up needs no communication.
* `DistributedPCG` is Jacobi-PCG over the owned dofs (x0 = 0, stop on
  r.r <= tol^2 b.b): per iteration one halo exchange of p (point-to-point sends and
  receives between slab neighbours) before the local SpMV, and two all-reduces (p.q,
  then r.z and r.r together).  The local operator, the vectors' device and the
  communicator are plugged in, so the same algorithm runs on GPUs (`ShardedSolver`,
  library SpMV, NCCL) and in CPU tests (gloo, a host SpMV).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import meshgen as mg


def partition(coords: np.ndarray, nranks: int) -> np.ndarray:
    """Owner rank of every node: equal contiguous runs along the longest axis."""
    x = np.asarray(coords, np.float64)
    nnodes = x.shape[0]
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    axis = int(np.argmax(x.max(0) - x.min(0))) if nnodes else 0
    order = np.lexsort((np.arange(nnodes), x[:, axis]))  # stable: ties by node id
    owner = np.empty(nnodes, np.int32)
    bounds = np.linspace(0, nnodes, nranks + 1).round().astype(np.int64)
    for r in range(nranks):
        owner[order[bounds[r]:bounds[r + 1]]] = r
    return owner


@dataclass
class Shard:
    rank: int
    nranks: int
    dim: int
    elem_type: int
    owned: np.ndarray          # global node ids (0-based) owned here, ascending
    halo: np.ndarray           # global node ids of halo nodes, ascending
    elems: np.ndarray          # global element ids of the local mesh, ascending
    coords: np.ndarray         # local nodes (owned, then halo)
    conn: np.ndarray           # local connectivity, 1-based local node ids
    E: Optional[np.ndarray]    # per local element, or None
    supports: np.ndarray       # (k, dim+1), 1-based local node ids
    f: np.ndarray              # local dofs; loads on owned dofs, 0 on halo dofs
    send: Dict[int, np.ndarray] = field(default_factory=dict)  # rank -> local owned node ids
    recv: Dict[int, np.ndarray] = field(default_factory=dict)  # rank -> local halo node ids

    @property
    def n_owned(self) -> int:
        return self.owned.size * self.dim

    @property
    def n_local(self) -> int:
        return (self.owned.size + self.halo.size) * self.dim

    def dofs(self, local_nodes: np.ndarray) -> np.ndarray:
        ln = np.asarray(local_nodes, np.int64)
        return (ln[:, None] * self.dim + np.arange(self.dim)[None, :]).ravel()


def _local_elements(conn0: np.ndarray, owner: np.ndarray, rank: int) -> np.ndarray:
    return np.flatnonzero((owner[conn0] == rank).any(axis=1))


def _halo_nodes(conn0: np.ndarray, owner: np.ndarray, rank: int, elems: np.ndarray) -> np.ndarray:
    nodes = np.unique(conn0[elems])
    return nodes[owner[nodes] != rank]


def build_shard(mesh: mg.Mesh, owner: np.ndarray, rank: int) -> Shard:
    nranks = int(owner.max()) + 1 if owner.size else 1
    conn0 = mesh.conn.astype(np.int64) - 1
    dim = mesh.dim
    owned = np.flatnonzero(owner == rank)
    elems = _local_elements(conn0, owner, rank)
    halo = _halo_nodes(conn0, owner, rank, elems)
    local_nodes = np.concatenate([owned, halo])
    g2l = np.full(mesh.nnodes, -1, np.int64)
    g2l[local_nodes] = np.arange(local_nodes.size)
    conn = (g2l[conn0[elems]] + 1).astype(np.int32)
    E = None if mesh.E is None else np.asarray(mesh.E)[elems]
    sup = np.asarray(mesh.supports, np.int32).reshape(-1, dim + 1)
    if sup.size:
        keep = g2l[sup[:, 0] - 1] >= 0
        sup = sup[keep].copy()
        sup[:, 0] = (g2l[sup[:, 0] - 1] + 1).astype(np.int32)
    f_glob = mesh.f if mesh.f is not None else np.zeros(mesh.ndof)
    f = np.zeros(local_nodes.size * dim)
    f[:owned.size * dim] = f_glob.reshape(-1, dim)[owned].ravel()
    sh = Shard(rank, nranks, dim, mesh.elem_type, owned, halo, elems,
               np.ascontiguousarray(mesh.coords[local_nodes]), conn, E, sup, f)
    # exchange lists from the owner array alone
    for s in range(nranks):
        if s == rank:
            continue
        # what I receive from s: my halo nodes owned by s (ascending global id)
        mine = halo[owner[halo] == s]
        if mine.size:
            sh.recv[s] = g2l[mine]
        # what I send to s: nodes I own in s's halo (ascending global id)
        es = _local_elements(conn0, owner, s)
        hs = _halo_nodes(conn0, owner, s, es)
        theirs = hs[owner[hs] == rank]
        if theirs.size:
            sh.send[s] = g2l[theirs]
    return sh


class _DeviceArray:
    """A device buffer of doubles described by __cuda_array_interface__ (zero-copy view)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None, "stream": None}


class TorchComm:
    """Halo exchange and all-reduce through torch.distributed (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, shard: Shard, device):
        import torch
        self.torch = torch
        self.shard = shard
        self.send = {r: torch.as_tensor(shard.dofs(v), device=device) for r, v in shard.send.items()}
        self.recv = {r: torch.as_tensor(shard.dofs(v), device=device) for r, v in shard.recv.items()}

    def exchange(self, xl) -> None:
        """Fill the halo part of the local vector xl from the owners' values."""
        import torch.distributed as dist
        torch = self.torch
        ops, bufs = [], []
        for r in sorted(self.send):
            ops.append(dist.P2POp(dist.isend, xl[self.send[r]].contiguous(), r))
        for r in sorted(self.recv):
            b = torch.empty(self.recv[r].numel(), dtype=xl.dtype, device=xl.device)
            bufs.append((r, b))
            ops.append(dist.P2POp(dist.irecv, b, r))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for r, b in bufs:
            xl[self.recv[r]] = b

    def allreduce(self, t):
        import torch.distributed as dist
        dist.all_reduce(t)
        return t


@dataclass
class SolveResult:
    x: object                 # owned dofs (torch tensor)
    iterations: int
    rel_residual: float       # recursive r.r / b.b, square-rooted
    converged: bool


class DistributedPCG:
    """Jacobi-PCG over the owned dofs of every rank.

    matvec(xl, yl): yl = K_local xl on local vectors (owned + halo dofs); only the owned
    rows of yl are used.  dinv: 1 / diag over the owned dofs (1 where the diagonal is 0).
    """

    def __init__(self, shard: Shard, matvec: Callable, dinv, comm):
        self.sh = shard
        self.matvec = matvec
        self.dinv = dinv
        self.comm = comm

    def solve(self, b, tol: float, max_iter: int) -> SolveResult:
        torch = self.comm.torch
        no, nl = self.sh.n_owned, self.sh.n_local
        dev, dt = b.device, b.dtype
        x = torch.zeros(no, dtype=dt, device=dev)
        r = b.clone()
        z = self.dinv * r
        pl = torch.zeros(nl, dtype=dt, device=dev)
        ql = torch.zeros(nl, dtype=dt, device=dev)
        pl[:no] = z
        s = self.comm.allreduce(torch.stack([torch.dot(r, z), torch.dot(r, r)]))
        rz, rr0 = float(s[0]), float(s[1])
        rr = rr0
        tol2 = tol * tol * rr0
        it = 0
        while it < max_iter and rr > tol2 and rr0 > 0.0:
            self.comm.exchange(pl)
            self.matvec(pl, ql)
            p, q = pl[:no], ql[:no]
            pq = float(self.comm.allreduce(torch.dot(p, q).reshape(1))[0])
            if not pq > 0.0:
                break
            alpha = rz / pq
            x.add_(p, alpha=alpha)
            r.add_(q, alpha=-alpha)
            z = self.dinv * r
            s = self.comm.allreduce(torch.stack([torch.dot(r, z), torch.dot(r, r)]))
            rzn, rr = float(s[0]), float(s[1])
            pl[:no] = z + (rzn / rz) * p
            rz = rzn
            it += 1
        return SolveResult(x, it, (rr / rr0) ** 0.5 if rr0 > 0 else 0.0, rr <= tol2)


class ShardedSolver:
    """One rank's part of a sharded assembly + Jacobi-PCG on its GPU (torch.distributed
    already initialised, NCCL backend)."""

    def __init__(self, mesh: mg.Mesh, rank: int, nranks: int, device: int = 0,
                 scatter: Optional[int] = None):
        import torch
        from . import _lib
        from .fem import Context
        self.torch = torch
        self.owner = partition(mesh.coords, nranks)
        self.shard = sh = build_shard(mesh, self.owner, rank)
        self.ctx = ctx = Context(device)
        ctx.mesh_create(mesh.elem_type, sh.coords, sh.conn, mesh.ngauss, mesh.E0, sh.E, mesh.nu)
        ctx.set_supports(sh.supports)
        ctx.set_force(sh.f)
        self.assembly_seconds = ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_AUTO if scatter is None
                                             else scatter)
        ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
        dev = torch.device("cuda", device)
        self.device = dev
        d = ctx.ell_diagonal(_lib.GF_F64)[:sh.n_owned]
        self.dinv = torch.as_tensor(np.where(d != 0.0, 1.0 / np.where(d != 0.0, d, 1.0), 1.0),
                                    device=dev)
        self.b = torch.as_tensor(ctx.get_force()[:sh.n_owned], device=dev)
        self.comm = TorchComm(sh, dev)
        lib, h = _lib.lib, ctx.h

        def matvec(xl, yl):
            torch.cuda.synchronize(dev)   # the library runs on its own stream
            _lib.check(lib.gf_spmv(h, _lib.GF_F64, xl.data_ptr(), yl.data_ptr()), h)

        self.pcg = DistributedPCG(sh, matvec, self.dinv, self.comm)

    def solve(self, tol: float = 1e-8, max_iter: int = 100000) -> SolveResult:
        return self.pcg.solve(self.b, tol, max_iter)

    def solve_device(self, tol: float = 1e-8, max_iter: int = 100000, check_every: int = 16):
        """The same Jacobi-PCG inside the library (gf_dist_pcg): vectors, dots and scalars
        on the device, the halo exchange and the all-reduces enqueued by torch.distributed
        (NCCL) on the library's stream from the library's callbacks, no host
        synchronisation per iteration.  Returns (owned-dof solution as a numpy array,
        SolveInfo)."""
        import torch
        import torch.distributed as dist
        from . import _lib
        sh, ctx = self.shard, self.ctx
        if not hasattr(self, "_dist_cb"):
            send_r, recv_r = sorted(sh.send), sorted(sh.recv)
            send = [sh.dofs(sh.send[r]) for r in send_r]
            recv = [sh.dofs(sh.recv[r]) for r in recv_r]
            sd = np.concatenate(send).astype(np.int32) if send else np.zeros(0, np.int32)
            rd = np.concatenate(recv).astype(np.int32) if recv else np.zeros(0, np.int32)
            _lib.check(_lib.lib.gf_dist_set_halo(ctx.h, sh.n_owned, sd.size,
                                                 sd.ctypes.data_as(C.c_void_p), rd.size,
                                                 rd.ctypes.data_as(C.c_void_p)), ctx.h)
            soff = np.concatenate([[0], np.cumsum([a.size for a in send])]).astype(int)
            roff = np.concatenate([[0], np.cumsum([a.size for a in recv])]).astype(int)
            stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=self.device)

            def dev(ptr, count):
                return torch.as_tensor(_DeviceArray(ptr, count), device=self.device)

            def allreduce(ptr, count, _stream, _user):
                try:
                    with torch.cuda.stream(stream):
                        dist.all_reduce(dev(ptr, count))
                    return 0
                except Exception:   # reported to the library as a failed collective
                    return 1

            def halo(sptr, rptr, _stream, _user):
                try:
                    sb, rb = dev(sptr, int(soff[-1])), dev(rptr, int(roff[-1]))
                    ops = [dist.P2POp(dist.isend, sb[soff[k]:soff[k + 1]], r)
                           for k, r in enumerate(send_r)]
                    ops += [dist.P2POp(dist.irecv, rb[roff[k]:roff[k + 1]], r)
                            for k, r in enumerate(recv_r)]
                    with torch.cuda.stream(stream):
                        for req in dist.batch_isend_irecv(ops):
                            req.wait()
                    return 0
                except Exception:
                    return 1

            self._dist_cb = (_lib.ALLREDUCE_FN(allreduce), _lib.HALO_FN(halo))
        o = _lib.SolveOpts(solver=_lib.GF_SOLVER_PCG, matrix=_lib.GF_F64, max_iter=max_iter,
                           tol=tol, check_every=check_every)
        info = _lib.SolveInfo()
        st = _lib.lib.gf_dist_pcg(ctx.h, C.byref(o), C.cast(self._dist_cb[0], C.c_void_p),
                                  C.cast(self._dist_cb[1], C.c_void_p), None, C.byref(info))
        _lib.check(st, ctx.h)
        return ctx.solution()[:sh.n_owned], info

    def gather(self, x) -> np.ndarray:
        """Full solution on every rank (all-gather of owned dofs; for checks)."""
        import torch.distributed as dist
        sh = self.shard
        parts: List = [None] * sh.nranks
        dist.all_gather_object(parts, (sh.owned, x.cpu().numpy()))
        u = np.zeros(self.owner.size * sh.dim)
        for owned, xv in parts:
            u.reshape(-1, sh.dim)[owned] = xv.reshape(-1, sh.dim)
        return u

    def close(self) -> None:
        self.ctx.close()
