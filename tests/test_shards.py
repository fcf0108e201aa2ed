"""Multi-GPU decomposition.

On the CPU: the strided shard rule partitions every list exactly, and
partial Fock matrices from world_size 2 gloo ranks sum (one all-reduce) to
the full build.  Each rank takes, as pfk_set_shard does, every second shell
quartet of each angular-momentum class list and digests the canonical AO
quartets inside them (integrals from the oracle's tensor), so the test runs
the product's decomposition at shell-quartet granularity.

On the GPU: two contexts on one device with set_shard(0, 2) and
set_shard(1, 2) build partial G whose sum is the unsharded G."""
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


def _class_lists(shells):
    """Canonical shell quartets grouped by class (pair classes LA >= LB,
    bra class >= ket class), in a seeded order within each class (the
    partition does not depend on the order)."""
    L = np.asarray(shells["L"])
    ns = len(L)
    pairs = [(a, b) for a in range(ns) for b in range(a, ns)]

    def pc(a, b):
        la, lb = max(L[a], L[b]), min(L[a], L[b])
        return la * (la + 1) // 2 + lb

    lists = {}
    for x in range(len(pairs)):
        for y in range(x, len(pairs)):
            p, q = pairs[x], pairs[y]
            cx, cy = pc(*p), pc(*q)
            key = (max(cx, cy), min(cx, cy))
            lists.setdefault(key, []).append((p, q))
    rng = np.random.default_rng(3)
    for k in lists:
        lists[k] = [lists[k][i] for i in rng.permutation(len(lists[k]))]
    return lists


def _digest_shell_quartets(sq, bf_off, nbf, eri, Pm):
    """J and K of the listed shell quartets: each canonical AO quartet inside
    them adds every distinct member of its 8-fold orbit (mn|rs),
    J(m,n) += P(r,s) v and K(m,r) += P(n,s) v, which is what the reference's
    tensor contraction sums (os.cpp:1512-1520); G = J - K/2."""
    nb = Pm.shape[0]
    keys = set()
    for (a, b), (c, d) in sq:
        for i in range(bf_off[a], bf_off[a] + nbf[a]):
            for j in range(bf_off[b], bf_off[b] + nbf[b]):
                for k in range(bf_off[c], bf_off[c] + nbf[c]):
                    for l in range(bf_off[d], bf_off[d] + nbf[d]):
                        p1, p2 = (min(i, j), max(i, j)), (min(k, l), max(k, l))
                        keys.add(p1 + p2 if p1 <= p2 else p2 + p1)
    J, K = np.zeros((nb, nb)), np.zeros((nb, nb))
    if not keys:
        return J, K
    q = np.array(sorted(keys))
    i, j, k, l = q.T
    v = eri[i, j, k, l]
    perms = [(i, j, k, l), (j, i, k, l), (i, j, l, k), (j, i, l, k), (k, l, i, j), (l, k, i, j), (k, l, j, i),
             (l, k, j, i)]
    for a, (m, n, r, s) in enumerate(perms):
        keep = np.ones(len(v), dtype=bool)
        for c in range(a):
            keep &= ~((perms[c][0] == m) & (perms[c][1] == n) & (perms[c][2] == r) & (perms[c][3] == s))
        np.add.at(J, (m[keep], n[keep]), Pm[r[keep], s[keep]] * v[keep])
        np.add.at(K, (m[keep], r[keep]), Pm[n[keep], s[keep]] * v[keep])
    return J, K


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
    eri, _ = ob.eri_tensor(1e-10, oracle.OS)
    L = np.asarray(shells["L"])
    nbf = (L + 1) * (L + 2) // 2
    bf_off = np.concatenate([[0], np.cumsum(nbf)[:-1]])
    mine, n = [], 0
    for key, lst in sorted(_class_lists(shells).items()):
        idx = list(P.shard.shard_indices(len(lst), rank, world))
        assert len(idx) == P.shard.local_count(len(lst), rank, world)
        mine += [lst[t] for t in idx]
        n += len(idx)
    J, K = _digest_shell_quartets(mine, bf_off, nbf, eri, Pm)
    G = torch.from_numpy(J - 0.5 * K)
    P.shard.allreduce_partial(G)
    cnt = torch.tensor([n], dtype=torch.int64)
    dist.all_reduce(cnt)
    if rank == 0:
        nf = sum(len(v) for v in _class_lists(shells).values())
        err = float(np.abs(G.numpy() - oracle.fock_rhf_tensor(eri, Pm)).max())
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


@pytest.mark.gpu
def test_two_shard_contexts_sum_to_full_build():
    """pfk_set_shard on one GPU: the partial G of shards (0, 2) and (1, 2)
    add up to the unsharded G."""
    from helpers import basis_library, random_density, water_cluster
    P = pfk()
    mol, shells = P.shells_for(water_cluster(4, seed=7), "6-31g**", basis_library())
    full = P.FockEngine(shells)
    Pm = random_density(full.nbasis, seed=41, scale=0.1)
    G = full.fock_rhf(Pm)
    parts = []
    for r in range(2):
        e = P.FockEngine(shells)
        e.set_shard(r, 2)
        parts.append(e.fock_rhf(Pm))
        e.close()
    full.close()
    assert np.abs(parts[0]).max() > 0 and np.abs(parts[1]).max() > 0
    assert np.abs(parts[0] + parts[1] - G).max() < 1e-12
