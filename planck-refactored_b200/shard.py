"""Shard arithmetic of one-process-per-GPU Fock builds.

A build split across N ranks evaluates, on rank r, the quartets
t * N + r (t = 0, 1, ...) of every class list (pfk_set_shard; the class
kernels read quartets[t * qstride + qoffset]).  The ranks' partial G
(or J, K) are summed with one all-reduce.  These helpers state that rule
for the host side and the tests.
"""


def local_count(n, rank, nranks):
    """Quartets rank `rank` evaluates out of a list of n (the same formula as
    the C runtime's launch sizing)."""
    return (n - rank + nranks - 1) // nranks if n > rank else 0


def shard_indices(n, rank, nranks):
    return range(rank, n, nranks)


def allreduce_partial(partial, group=None):
    """Sum a partial matrix (a torch tensor) over the process group in place."""
    import torch.distributed as dist
    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial
