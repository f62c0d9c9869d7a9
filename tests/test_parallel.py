"""Multi-rank paths on the CPU (gloo, world size 2): the (T) triplet shards
that `xvcc_run` evaluates per GPU, the 2-double all-reduce of their partial
energies, and bench.py's max-over-ranks timing reduction."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from acesb200.parallel import triplet_order, triplet_shard
from oracle.hamiltonian import synthetic
from oracle import triples as otriples


def _amplitudes(o, v, seed):
    """Pair-symmetric random amplitudes, t2[i,j,a,b] = t2[j,i,b,a]."""
    rng = np.random.default_rng(seed)
    t1 = rng.normal(0.0, 0.05, (o, v))
    t2 = rng.normal(0.0, 0.05, (o, o, v, v))
    t2 = 0.5 * (t2 + t2.transpose(1, 0, 3, 2))
    return t1, t2


@pytest.mark.parametrize("o", [1, 3, 7])
@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_triplet_shards_partition_the_triplets(o, nranks):
    shards = [triplet_shard(o, r, nranks) for r in range(nranks)]
    flat = [t for s in shards for t in s]
    assert sorted(flat) == sorted(triplet_order(o))
    assert len(set(flat)) == len(flat) == o * (o + 1) * (o + 2) // 6
    # round robin: shard sizes differ by at most one
    sizes = [len(s) for s in shards]
    assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        triplet_shard(o, nranks, nranks)


def test_unique_triplets_sum_to_the_full_triples_energy():
    ham = synthetic(4, 7, 12, seed=3)
    t1, t2 = _amplitudes(4, 7, 5)
    full = otriples.triples(ham, t1, t2)
    part = otriples.triples_unique(ham, t1, t2, list(triplet_order(4)))
    np.testing.assert_allclose(part, full, rtol=1e-12, atol=1e-15)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from acesb200.parallel import allreduce_pair, allreduce_max, triplet_shard
        import bench
        o, v = 4, 7
        ham = synthetic(o, v, 12, seed=3)
        t1, t2 = _amplitudes(o, v, 5)
        e4, e5 = otriples.triples_unique(ham, t1, t2, triplet_shard(o, rank, world))
        tot = allreduce_pair(e4, e5)
        mx = allreduce_max(float(rank + 1) * 0.25)
        mb = bench.max_over_ranks(float(10 - rank), world)
        bench.barrier(world)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array([e4, e5, tot[0], tot[1], mx, mb]))
    finally:
        dist.destroy_process_group()


def test_sharded_triples_allreduce_gloo(tmp_path):
    world = 2
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = [np.load(tmp_path / f"rank{k}.npy") for k in range(world)]
    ham = synthetic(4, 7, 12, seed=3)
    t1, t2 = _amplitudes(4, 7, 5)
    full = otriples.triples(ham, t1, t2)
    for k in range(world):
        # every rank holds the total, equal to the single-process energy
        np.testing.assert_allclose(r[k][2:4], full, rtol=1e-12, atol=1e-15)
        assert r[k][4] == 0.5 and r[k][5] == 10.0
    # the shards are proper parts of it
    np.testing.assert_allclose(r[0][:2] + r[1][:2], full, rtol=1e-12, atol=1e-15)
    assert abs(r[0][0]) > 0 and abs(r[1][0]) > 0
