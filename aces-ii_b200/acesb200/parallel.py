"""(T) over several GPUs: triplet shards and the reduction of their energies.

The occupied triplets i >= j >= k are independent (trp/trps2.F:418-429 loops
over them with no coupling but the energy sum), so one process per GPU
evaluates the triplets whose index t in the order (i, then j <= i, then
k <= j) satisfies t % nranks == rank -- the rule `xvcc_run` applies when
`triples_rank` / `triples_nranks` are set -- and the partial E[4]T / E[5]ST
are added with one 2-double all-reduce.  Every rank needs the converged
amplitudes and integrals: `triples_from_root` solves CCSD on rank 0 only and
broadcasts T1 (list 90) and T2 (list 46) -- o v + o^2 v^2 doubles, 104 MB at
o = 20, v = 180 -- after which every rank restarts from them (the TGUESS path
of xvcc_run, vcc/drdtgss.F: one cycle confirms convergence) and evaluates its
shard.  `sharded_triples` is the older scheme in which every rank repeats the
solve.

Independent systems (the 64-system batch) are split by system: `assign_systems`
deals them to ranks by flop weight (longest first, to the least-loaded rank) and
`gather_values` sums the per-system results of all ranks.
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


def _device(group=None):
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")


def _amplitude_blocks(lib):
    """(list, irrep, rows, cols) of T1 (list 90, irrep 1: the (a,i) pairs of
    type 9) and T2(AB) (list 46, pair types 13 x 14 per irrep)."""
    out = [(90, 1, lib.irpdpd(1, 9), 1)]
    for h in range(1, lib.nirrep + 1):
        out.append((46, h, lib.irpdpd(h, 13), lib.irpdpd(h, 14)))
    return out


def broadcast_amplitudes(lib, group=None, src=0):
    """Copy rank `src`'s amplitude lists 90 and 46 to every rank of `group`.
    With NCCL the lists move device to device (GETLST/PUTLST device variants
    around one broadcast), with gloo through host memory.  Every rank must
    have called aces_sym_init with the same symmetry."""
    import ctypes as C
    import numpy as np
    import torch
    import torch.distributed as dist
    dev = _device(group)
    rank = dist.get_rank()
    blocks = _amplitude_blocks(lib)
    total = sum(nr * nc for _, _, nr, nc in blocks)
    buf = torch.zeros(total, dtype=torch.float64, device=dev)
    if rank == src:
        off = 0
        for lst, h, nr, nc in blocks:
            if nr * nc:
                if dev.type == "cuda":
                    lib._chk("aces_getlst_dev", lib.h.aces_getlst_dev(
                        C.c_void_p(buf.data_ptr() + 8 * off), 1, nc, h, lst))
                else:
                    buf[off:off + nr * nc] = torch.from_numpy(
                        np.ascontiguousarray(lib.getlst(1, nc, h, lst).T).ravel())
            off += nr * nc
        if dev.type == "cuda":
            torch.cuda.synchronize()   # the list copies run on the legacy stream
    dist.broadcast(buf, src=src, group=group)
    if rank != src:
        if dev.type == "cuda":
            torch.cuda.synchronize()   # the broadcast runs on torch's stream
        lib.inipck(1, 13, 14, 46)
        lib.list_touch(1, lib.irpdpd(1, 9), 1, 90)
        off = 0
        for lst, h, nr, nc in blocks:
            if nr * nc:
                if dev.type == "cuda":
                    lib._chk("aces_putlst_dev", lib.h.aces_putlst_dev(
                        C.c_void_p(buf.data_ptr() + 8 * off), 1, nc, h, lst))
                else:
                    cols = buf[off:off + nr * nc].numpy().reshape(nc, nr).T
                    lib.putlst(cols, 1, h, lst)
            off += nr * nc
    return total


def triples_from_root(lib, rank, nranks, group=None, **xvcc_kwargs):
    """CCSD(T) over the ranks of `group` with ONE CCSD solve: rank 0 solves,
    the amplitudes are broadcast, every rank restarts from them (TGUESS; the
    first cycle finds the equations converged) and evaluates its triplet
    shard; the partial energies are all-reduced.  Every rank takes the same
    collective steps on the error path too: rank 0's status is broadcast
    first and a failure raises on every rank.  Returns this rank's config with
    e_t4 / e_st5 the totals, seconds_triples the slowest rank's, and on rank 0
    ncycle the solve's cycle count."""
    import torch
    import torch.distributed as dist
    dev = _device(group)
    solve = None
    err = ""
    status = torch.zeros(1, dtype=torch.int64, device=dev)
    if rank == 0:
        try:
            solve = lib.xvcc(triples=0, **xvcc_kwargs)
        except Exception as exc:  # noqa: BLE001 -- reported on every rank below
            err = str(exc)
            status[0] = getattr(exc, "status", -1) or -1
    dist.broadcast(status, src=0, group=group)
    if int(status.item()) != 0:
        raise RuntimeError(f"CCSD on rank 0 failed (status {int(status.item())}) {err}")
    broadcast_amplitudes(lib, group)
    cfg = lib.xvcc(triples=1, tguess=1, triples_rank=rank, triples_nranks=nranks,
                   **xvcc_kwargs)
    if nranks > 1:
        cfg.e_t4, cfg.e_st5 = allreduce_pair(cfg.e_t4, cfg.e_st5, group)
        cfg.seconds_triples = allreduce_max(cfg.seconds_triples, group)
    if solve is not None:
        cfg.ncycle = solve.ncycle
        cfg.seconds_per_iter = solve.seconds_per_iter
    return cfg


def assign_systems(weights, nranks):
    """Deal independent systems to ranks: heaviest first, each to the rank with
    the least total weight so far (ties: lowest rank).  Returns one list of
    system indices per rank."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(weights)), key=lambda k: (-weights[k], k))
    load = [0.0] * nranks
    out = [[] for _ in range(nranks)]
    for k in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += weights[k]
    return [sorted(x) for x in out]


def gather_values(values, n, mine, group=None):
    """values[k] for the systems k in `mine` of this rank -> the length-n vector
    of every rank's values (zero-filled per rank, then summed)."""
    import torch
    import torch.distributed as dist
    t = torch.zeros(n, dtype=torch.float64, device=_device(group))
    for k in mine:
        t[k] = float(values[k])
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().tolist()
