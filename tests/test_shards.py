"""Multi-GPU decomposition, checked on the CPU: the strided shard rule
partitions every list exactly, and partial Fock matrices from world_size 2
gloo ranks sum (one all-reduce) to the full build.  The partial builds here
are the oracle's streaming build over each rank's share of bra rows, which
stands in for the GPU shards (the all-reduce and the assembly are the same)."""
import os

import numpy as np
import pytest

from helpers import WATER, pfk


@pytest.mark.parametrize("n", [0, 1, 2, 7, 64, 1001])
@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_shards_partition_each_list(n, nranks):
    S = pfk().shard
    seen = []
    for r in range(nranks):
        idx = list(S.shard_indices(n, r, nranks))
        assert len(idx) == S.local_count(n, r, nranks)
        seen += idx
    assert sorted(seen) == list(range(n))


def _rank_main(rank, world, port, result_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch
    import torch.distributed as dist

    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    P = pfk()
    mol, shells = P.shells_for(WATER, "6-31g**", P.basis.load_library())
    ob = oracle.Basis(shells)
    nb = ob.nbasis
    rng = np.random.default_rng(1)
    A = rng.normal(size=(nb, nb)) * 0.2
    Pm = A + A.T
    Q = ob.schwarz(oracle.OS)
    rows = np.array(list(P.shard.shard_indices(ob.npairs, rank, world)), dtype=np.int32)
    J, K, n = ob.jk_direct_rows(Pm, [Pm], rows, 1e-10, oracle.OS, Q=Q)
    G = torch.from_numpy(J - 0.5 * K[0])
    P.shard.allreduce_partial(G)
    cnt = torch.tensor([n], dtype=torch.int64)
    dist.all_reduce(cnt)
    if rank == 0:
        Jf, Kf, nf = ob.jk_direct(Pm, [Pm], 1e-10, oracle.OS, Q=Q)
        err = float(np.abs(G.numpy() - (Jf - 0.5 * Kf[0])).max())
        with open(result_path, "w") as f:
            f.write(f"{err} {int(cnt.item())} {nf}")
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_partial_builds_sum_to_full(tmp_path):
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    out = str(tmp_path / "result.txt")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    err, n_sum, n_full = open(out).read().split()
    assert float(err) < 1e-12
    assert int(n_sum) == int(n_full)
