"""Sharded assembly and solve: partition, local meshes and exchange lists on the CPU; the
distributed Jacobi-PCG over gloo with 2 and 3 ranks (local operators built by the C oracle)
against the single-domain oracle solution; the GPU path (library SpMV, NCCL) on one rank."""
import datetime
import os
import socket

import numpy as np
import pytest

from gpufem_b200 import meshgen as mg
from gpufem_b200 import shard as sd

CASES = [(mg.Q8, (6, 5)), (mg.BRICK8, (3, 3, 4)), (mg.Q4, (7, 3))]


def _mesh(et, n, seed=11):
    m = mg.structured(et, n, jitter=0.2, seed=seed, ngauss=2)
    m.E = np.exp(np.log(210e3) + 0.3 * np.random.default_rng(seed).standard_normal(m.nelem))
    return mg.clamp_and_load(m)


def _fixed(m, supports=None, nnodes=None):
    sup = m.supports if supports is None else supports
    nn = m.nnodes if nnodes is None else nnodes
    fixed = np.zeros(nn * m.dim, np.uint8)
    for row in sup:
        for c in range(m.dim):
            if row[1 + c] == 1:
                fixed[(row[0] - 1) * m.dim + c] = 1
    return fixed


@pytest.mark.parametrize("et,n", CASES)
@pytest.mark.parametrize("nranks", [1, 2, 3, 4])
def test_partition_shards_and_exchange_lists(et, n, nranks):
    m = _mesh(et, n)
    owner = sd.partition(m.coords, nranks)
    assert owner.shape == (m.nnodes,) and set(np.unique(owner)) <= set(range(nranks))
    counts = np.bincount(owner, minlength=nranks)
    assert counts.max() - counts.min() <= 1
    conn0 = m.conn - 1
    shards = [sd.build_shard(m, owner, r) for r in range(nranks)]
    for sh in shards:
        # every element touching an owned node is local; no other element is
        touch = np.flatnonzero(np.isin(conn0, sh.owned).any(axis=1))
        np.testing.assert_array_equal(sh.elems, touch)
        local = np.concatenate([sh.owned, sh.halo])
        np.testing.assert_array_equal(sh.coords, m.coords[local])
        np.testing.assert_array_equal(local[sh.conn - 1], conn0[sh.elems])
        assert sh.f.shape == (local.size * m.dim,)
        np.testing.assert_array_equal(sh.f[:sh.n_owned], m.f.reshape(-1, m.dim)[sh.owned].ravel())
        assert np.all(sh.f[sh.n_owned:] == 0)
    for r, a in enumerate(shards):
        for s, b in enumerate(shards):
            if r == s:
                continue
            sent = np.concatenate([a.owned, a.halo])[a.send.get(s, np.zeros(0, int))]
            got = np.concatenate([b.owned, b.halo])[b.recv.get(r, np.zeros(0, int))]
            np.testing.assert_array_equal(sent, got)
    # every halo node of every rank is received exactly once
    for sh in shards:
        recv = np.concatenate([v for v in sh.recv.values()] + [np.zeros(0, int)])
        assert np.array_equal(np.sort(recv), np.arange(sh.owned.size, sh.owned.size + sh.halo.size))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, nranks, port, et, n, tol, ref_path):
    import torch
    import torch.distributed as dist
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks,
                            timeout=datetime.timedelta(seconds=60))
    try:
        O = Oracle()
        m = _mesh(et, n)
        owner = sd.partition(m.coords, nranks)
        sh = sd.build_shard(m, owner, rank)
        E_loc = sh.E if sh.E is not None else None
        rn, ci, v = O.assemble(m.elem_type, m.ngauss, sh.coords, sh.conn, m.E0, m.nu, E_elem=E_loc)
        fixed = _fixed(m, sh.supports, sh.coords.shape[0])
        v, f = O.eliminate(rn, ci, v, fixed, sh.f)

        def matvec(xl, yl):
            yl.copy_(torch.as_tensor(O.spmv(rn, ci, v, xl.numpy())))

        d = np.array([v[np.flatnonzero(ci[:rn[i], i] == i)[0], i] for i in range(sh.n_owned)])
        dinv = torch.as_tensor(np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 1.0))
        comm = sd.TorchComm(sh, "cpu")
        res = sd.DistributedPCG(sh, matvec, dinv, comm).solve(torch.as_tensor(f[:sh.n_owned]),
                                                              tol, 20000)
        parts = [None] * nranks
        dist.all_gather_object(parts, (sh.owned, res.x.numpy(), res.iterations, res.converged))
        if rank == 0:
            u = np.zeros(m.ndof)
            for owned, xv, it, conv in parts:
                assert conv
                u.reshape(-1, m.dim)[owned] = xv.reshape(-1, m.dim)
            assert len({p[2] for p in parts}) == 1        # every rank took the same steps
            ref = np.load(ref_path)
            assert np.linalg.norm(u - ref) <= 1e-8 * np.linalg.norm(ref)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("et,n", CASES)
@pytest.mark.parametrize("nranks", [2, 3])
def test_distributed_pcg_gloo_matches_single_domain(tmp_path, oracle, et, n, nranks):
    import torch.multiprocessing as tmp
    m = _mesh(et, n)
    rn, ci, v = oracle.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu, E_elem=m.E)
    v, f = oracle.eliminate(rn, ci, v, _fixed(m), m.f)
    ref, _ = oracle.cg(rn, ci, v, f, maxit=20000, eps=1e-13, precond=True)
    ref_path = str(tmp_path / "ref.npy")
    np.save(ref_path, ref)
    tmp.spawn(_gloo_rank, args=(nranks, _free_port(), et, n, 1e-12, ref_path), nprocs=nranks,
              join=True)


@pytest.mark.gpu
def test_sharded_solver_one_rank_matches_single_gpu_solve():
    import torch
    import torch.distributed as dist
    from gpufem_b200 import _lib
    from gpufem_b200.fem import Context
    m = mg.workload("q8_512", scale=1 / 16)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        s = sd.ShardedSolver(m, 0, 1, device=0)
        res = s.solve(tol=1e-10, max_iter=100000)
        u = s.gather(res.x)
        s.close()
    finally:
        dist.destroy_process_group()
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-10, max_iter=100000)
    u1 = ctx.solution()
    assert res.converged and abs(res.iterations - info.iterations) <= 2
    assert np.linalg.norm(u - u1) <= 1e-8 * np.linalg.norm(u1)


@pytest.mark.gpu
def test_sharded_device_pcg_one_rank_matches_single_gpu_solve():
    """gf_dist_pcg (vectors, dots and scalars on the device; the all-reduces enqueued by
    NCCL on the library's stream from its callbacks) on one rank: same solution and
    iteration count as the single-GPU PCG, and the device time per iteration within 1.5x
    of it (the single-GPU loop replays CUDA graphs and makes no collective calls).  The
    mesh is the full Q8 512x512 workload: the ctypes callbacks cost ~70 us of host time per
    iteration, which a smaller mesh's iterations would not cover."""
    import torch.distributed as dist
    from gpufem_b200 import _lib
    from gpufem_b200.fem import Context
    m = mg.workload("q8_512")                   # Q8 512x512, 1.58M dofs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        s = sd.ShardedSolver(m, 0, 1, device=0)
        x, info_d = s.solve_device(tol=1e-8, max_iter=100000)
        x2, info_d2 = s.solve_device(tol=1e-8, max_iter=100000)   # warm (layout built)
        u = s.gather(__import__("torch").as_tensor(x2))
        s.close()
    finally:
        dist.destroy_process_group()
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-8, max_iter=100000)
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-8, max_iter=100000)
    u1 = ctx.solution()
    # (dot products are summed by atomics, so two runs agree to rounding, not bitwise; over
    # ~13,000 iterations that moves the stopping iteration by a few)
    assert info_d2.status == _lib.GF_OK
    assert abs(info_d2.iterations - info.iterations) <= max(2, info.iterations // 1000)
    assert np.linalg.norm(x - x2) <= 1e-6 * np.linalg.norm(x)
    assert np.linalg.norm(u - u1) <= 1e-6 * np.linalg.norm(u1)
    per_it_d = info_d2.seconds / info_d2.iterations
    per_it = info.seconds / info.iterations
    print(f"device time per iteration: sharded {per_it_d * 1e6:.1f} us, single {per_it * 1e6:.1f} us")
    assert per_it_d <= 1.5 * per_it, (per_it_d, per_it)
