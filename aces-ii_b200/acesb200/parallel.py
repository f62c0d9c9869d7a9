"""(T) over several GPUs: triplet shards and the reduction of their energies.

The occupied triplets i >= j >= k are independent (trp/trps2.F:418-429 loops
over them with no coupling but the energy sum), so one process per GPU
evaluates the triplets whose index t in the order (i, then j <= i, then
k <= j) satisfies t % nranks == rank -- the rule `xvcc_run` applies when
`triples_rank` / `triples_nranks` are set -- and the partial E[4]T / E[5]ST
are added with one 2-double all-reduce.  Every rank needs the converged
amplitudes and integrals (each runs the same CCSD, or receives T2).
"""
from __future__ import annotations


def triplet_order(o):
    """The triplets i >= j >= k in the engine's order."""
    for i in range(o):
        for j in range(i + 1):
            for k in range(j + 1):
                yield (i, j, k)


def triplet_shard(o, rank, nranks):
    """The triplets rank `rank` of `nranks` evaluates (same rule as the engine)."""
    if nranks < 1 or not 0 <= rank < nranks:
        raise ValueError(f"rank {rank} outside 0..{nranks - 1}")
    return [t for n, t in enumerate(triplet_order(o)) if n % nranks == rank]


def allreduce_pair(e4, e5, group=None):
    """Sum (e4, e5) over the ranks of a torch.distributed process group (NCCL:
    on the current CUDA device; gloo: on the CPU)."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.tensor([e4, e5], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t[0].item()), float(t[1].item())


def allreduce_max(x, group=None):
    """Max of a float over the ranks (timings are reported as the slowest rank)."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sharded_triples(lib, rank, nranks, group=None, **xvcc_kwargs):
    """CCSD(T) with the triplets split over the ranks of `group`: every rank
    solves CCSD, evaluates its shard of (T); returns the config of this rank's
    call with e_t4 / e_st5 replaced by the totals and seconds_triples by the
    slowest rank's."""
    cfg = lib.xvcc(triples=1, triples_rank=rank, triples_nranks=nranks, **xvcc_kwargs)
    if nranks > 1:
        cfg.e_t4, cfg.e_st5 = allreduce_pair(cfg.e_t4, cfg.e_st5, group)
        cfg.seconds_triples = allreduce_max(cfg.seconds_triples, group)
    return cfg
