"""The sharded build's host side on CPU: two gloo ranks, each the oracle's
restatement of the reference's MPI split of the shell-pair loop
(direct.hpp:1600-1604, :1655-1656), summed by the library's own
``allreduce_sum`` (the reference's MPIReduce, direct.hpp:2085-2107), give
the whole contraction."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import oracle as O
    from chronusq_public_b200.basis import BasisSet
    from chronusq_public_b200.fockbuilder import allreduce_sum
    from helpers import water_ref
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        b = BasisSet.build(water_ref(), "cc-pvdz")
        ob = O.OracleBasis(b)
        N = b.nbasis
        rng = np.random.default_rng(3)
        A = rng.standard_normal((N, N))
        D = 0.1 * (A + A.T)
        Z = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        Zh = 0.1 * (Z + Z.conj().T)
        full = ob.contract([D, D], [1, 1], [0, 1], nthreads=2)
        part = ob.contract([D, D], [1, 1], [0, 1], nthreads=2, mpi=(rank, world))
        fullc = ob.contract([Zh, Zh], [1, 1], [0, 1], nthreads=2)
        partc = ob.contract([Zh, Zh], [1, 1], [0, 1], nthreads=2, mpi=(rank, world))
        own = max(np.abs(part[0]).max(), np.abs(part[1]).max())
        allreduce_sum(part + partc, dist.group.WORLD)
        err = max(np.abs(p - f).max() for p, f in zip(part + partc, full + fullc))
        out.put((rank, float(err), float(own)))
    finally:
        dist.destroy_process_group()


def test_two_rank_split_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(600)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, err, own in res:
        assert own > 0.0, rank  # every rank has a share of the work
        assert err < 1e-12, (rank, err)
