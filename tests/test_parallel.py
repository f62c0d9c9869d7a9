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


# ---------------------------------------------------------------- one CCSD solve, broadcast T
class _FakeLib:
    """The subset of acesb200.Lib that triples_from_root uses, with the lists
    in host memory (C1: list 90 holds t1 as (a,i) pairs, a fastest; list 46
    holds t2 with rows (a,b) and columns (i,j), first index fastest).  xvcc
    with triples=0 "solves" by writing the given amplitudes; with triples=1 it
    evaluates the oracle's (T) on this rank's shard of whatever amplitudes its
    lists hold."""

    class Cfg:
        pass

    def __init__(self, ham, t1, t2, fail=False):
        self.ham, self.o, self.v = ham, t1.shape[0], t1.shape[1]
        self._t1, self._t2, self.fail = t1, t2, fail
        self.nirrep = 1
        self.lists = {}
        self.calls = []

    def irpdpd(self, h, typ):
        return {9: self.o * self.v, 13: self.v * self.v, 14: self.o * self.o}[typ]

    def inipck(self, irrepx, tl, tr, lst, iset=1):
        self.lists.setdefault((lst, 1), np.zeros((self.irpdpd(1, tl), self.irpdpd(1, tr))))

    def list_touch(self, ncols, nrows, irrep, lst):
        self.lists.setdefault((lst, irrep), np.zeros((nrows, ncols)))
        return 0

    def getlst(self, first, ncols, h, lst):
        return self.lists[(lst, h)][:, first - 1:first - 1 + ncols].copy()

    def putlst(self, cols, first, h, lst):
        self.lists[(lst, h)][:, first - 1:first - 1 + cols.shape[1]] = cols

    def _write(self, t1, t2):
        o, v = self.o, self.v
        self.lists[(90, 1)] = t1.T.reshape(o * v, 1).copy()              # a + i v
        self.lists[(46, 1)] = t2.transpose(3, 2, 1, 0).reshape(v * v, o * o, order="F").copy()

    def _read(self):
        o, v = self.o, self.v
        t1 = self.lists[(90, 1)][:, 0].reshape(v, o).T
        t2 = self.lists[(46, 1)].reshape(v, v, o, o, order="F").transpose(3, 2, 1, 0)
        return t1, t2

    def xvcc(self, triples=0, tguess=0, triples_rank=0, triples_nranks=1, **kw):
        self.calls.append(dict(triples=triples, tguess=tguess, rank=triples_rank,
                               nranks=triples_nranks))
        c = self.Cfg()
        c.ncycle, c.seconds_per_iter, c.seconds_triples = 11, 0.5, 0.0
        c.e_t4 = c.e_st5 = 0.0
        if not triples:
            if self.fail:
                from acesb200 import AcesError
                raise AcesError("xvcc_run", -9, "did not converge")
            self._write(self._t1, self._t2)
            return c
        assert tguess == 1
        t1, t2 = self._read()
        c.ncycle = 1
        c.e_t4, c.e_st5 = otriples.triples_unique(
            self.ham, t1, t2, triplet_shard(self.o, triples_rank, triples_nranks))
        c.seconds_triples = 0.1 * (triples_rank + 1)
        return c


def _root_worker(rank, world, port, out_dir, fail):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from acesb200.parallel import triples_from_root
        o, v = 4, 7
        ham = synthetic(o, v, 12, seed=3)
        t1, t2 = _amplitudes(o, v, 5)
        if rank != 0:   # only rank 0 has the amplitudes
            t1, t2 = np.zeros_like(t1), np.zeros_like(t2)
        lib = _FakeLib(ham, t1, t2, fail=fail)
        try:
            c = triples_from_root(lib, rank, world, cc_conv=7)
            res = [c.e_t4, c.e_st5, c.seconds_triples, c.ncycle, len(lib.calls),
                   sum(k["triples"] == 0 for k in lib.calls)]
        except RuntimeError as exc:
            res = [np.nan] * 6
            assert "failed" in str(exc)
        np.save(os.path.join(out_dir, f"root{rank}.npy"), np.array(res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("fail", [False, True])
def test_triples_from_root_one_solve_gloo(tmp_path, fail):
    """Rank 0 alone solves CCSD; its amplitudes reach rank 1 through the
    broadcast, both evaluate their shards from them and the all-reduced (T)
    equals the single-process energy.  If rank 0's solve fails, both ranks
    raise instead of waiting on each other."""
    world = 2
    port = _free_port()
    mp.start_processes(_root_worker, args=(world, port, str(tmp_path), fail), nprocs=world,
                       join=True, start_method="spawn")
    r = [np.load(tmp_path / f"root{k}.npy") for k in range(world)]
    if fail:
        assert all(np.isnan(x).all() for x in r)
        return
    ham = synthetic(4, 7, 12, seed=3)
    t1, t2 = _amplitudes(4, 7, 5)
    full = otriples.triples(ham, t1, t2)
    for k in range(world):
        np.testing.assert_allclose(r[k][:2], full, rtol=1e-12, atol=1e-15)
        assert abs(r[k][2] - 0.2) < 1e-12          # slowest rank's (T) time
    assert r[0][3] == 11 and r[1][3] == 1            # rank 0 reports the solve's cycles
    assert r[0][5] == 1 and r[1][5] == 0             # exactly one CCSD solve, on rank 0
    assert r[0][4] == 2 and r[1][4] == 1


def test_assign_systems_balances_flop_weights():
    from acesb200.parallel import assign_systems
    from acesb200.workloads import batch_systems
    systems = batch_systems()
    w = [s["nocc"] ** 2 * s["nvir"] ** 4 for s in systems]
    for n in (1, 2, 3, 8):
        parts = assign_systems(w, n)
        assert sorted(k for p in parts for k in p) == list(range(64))
        loads = [sum(w[k] for k in p) for p in parts]
        # greedy longest-first: no rank exceeds the mean by more than the heaviest system
        assert max(loads) <= sum(w) / n + max(w)
    assert assign_systems([3.0, 1.0, 2.0], 2) == [[0], [1, 2]]
    with pytest.raises(ValueError):
        assign_systems(w, 0)


def _gather_worker(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from acesb200.parallel import assign_systems, gather_values
        w = [float(k % 5 + 1) for k in range(10)]
        mine = assign_systems(w, world)[rank]
        vals = {k: -0.1 * (k + 1) for k in mine}
        np.save(os.path.join(out_dir, f"g{rank}.npy"), np.array(gather_values(vals, 10, mine)))
    finally:
        dist.destroy_process_group()


def test_gather_values_gloo(tmp_path):
    world = 2
    mp.start_processes(_gather_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for k in range(world):
        np.testing.assert_allclose(np.load(tmp_path / f"g{k}.npy"),
                                   [-0.1 * (i + 1) for i in range(10)], rtol=0, atol=1e-15)
