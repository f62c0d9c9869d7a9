#!/usr/bin/env python
"""Benchmark: RHF-CCSD seconds per iteration on one B200.

Workload (the reference's headline configuration that fits one GPU): the
seeded synthetic closed-shell C1 Hamiltonian with nocc=20, nvir=180, naux=600
(acesb200.workloads 'c2'); <ab|cd> alone is 8.4 GB of FP64 and is streamed by
every iteration, so every step's inputs exceed the 126 MB L2.

A step is one CCSD iteration (residual, Jacobi update, energy, DIIS) through
the engine's xvcc_run entry point.  Printed JSON line:
  value      device time per iteration (CUDA events on the engine stream,
             inputs resident in HBM, W warm-up cycles excluded), BF16x3 split
             contractions on tcgen05 (default) or FP64 (--precision fp64);
             from the third cycle on, the residual pass is the replay of a
             CUDA graph captured on the second (--use-graph 0 launches every
             kernel from the host);
  e2e        the same metric through the C-ABI from HOST inputs: the MO
             density-fitting factors B[L,p,q] (the workload's definition of the
             integrals) and orbital energies from pinned memory, the device
             list producer aces_intprc_df, xvcc_run for K cycles and GETLST of
             T2, all inside the timed region, divided by K ("e2e_putlst": the
             same with the six lists built on the host and PUTLST);
  roofline   the packed particle-particle ladder (2 o^2 (np^2 + nm^2) flops
             for the symmetric and antisymmetric pair blocks, 3 BF16 products
             each), timed by CUDA events around it inside every cycle,
             against the measured sustained bf16 peak;
  cpu_baseline  the FP64 numpy restatement of the reference (oracle/) on the
             host cores, one CCSD iteration of the same system from its MP2
             amplitudes (all threads, and one thread when that fits the
             time budget).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "aces-ii_b200"))
sys.path.insert(0, ROOT)

W_NAME = "c2"


def args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=8)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="bf16x3", choices=["bf16x3", "fp64"])
    p.add_argument("--workload", default=W_NAME)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64-compare", action="store_true")
    p.add_argument("--use-graph", type=int, default=None,
                   help="1: replay each cycle's residual pass from a CUDA graph captured on "
                        "the second cycle, 0: launch every kernel from the host (default 1, "
                        "and 0 for the c5 batch, whose short solves do not amortise a capture)")
    p.add_argument("--autotune", type=int, default=None,
                   help="1: tensor-core tile variants timed once per shape class and the "
                        "fastest reused (aces_set_autotune), 0: built-in tile rules (default "
                        "1 for the c5 batch, after an untimed tuning pass over its systems; "
                        "0 otherwise)")
    p.add_argument("--batch-bscale", type=float, default=1.0,
                   help="scale of the DF factors of the 64-system batch (--workload c5)")
    p.add_argument("--no-lambda", action="store_true",
                   help="skip the Lambda / density block (C4 system)")
    p.add_argument("--kernel-case", default=None,
                   help="run one small case for ncu captures and exit: a contraction "
                        "shape through aces_xgemm (ladder-small, ladder-packed, thin-t1, "
                        "lowrank-t1) or "
                        "CCSD(T) on a small system (triples-o10-v180, triples-o6-v128, "
                        "triples-o4-v136), split CCSD cycles (ccsd-o40-v100) or Lambda + "
                        "density (lambda-c4)")
    a = p.parse_args()
    if a.use_graph is None:
        a.use_graph = 0 if a.workload == "c5" else 1
    return a


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ------------------------------------------------------------------ clocks
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        # nvidia-smi initialises NVML when it starts; let that finish before the
        # timed GPU work so it cannot overlap the measured cycles
        if self.p is not None:
            time.sleep(1.5)
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.p is None:
            return
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        pw = [float(r[3]) for r in self.rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k] == "Active"})
        loaded = [s for s, p in zip(sm, pw) if p > 250.0] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows), "power_w_max": max(pw) if pw else None}


# ------------------------------------------------------------------ inputs
def host_lists(wl, device):
    """The six integral lists + orbital energies of the workload as pinned host
    buffers in the list layout (column-major irrep block, C1), built on the
    GPU from the seeded DF factors."""
    import numpy as np
    import torch
    from acesb200 import INTEGRAL_LISTS
    from acesb200.workloads import synthetic_df

    o, v = wl["nocc"], wl["nvir"]
    # the six lists are staged in pinned host memory: refuse rather than drive
    # the host out of memory
    need = 8.0 * (v ** 4 + o * v ** 3 + 2 * o * o * v * v + o ** 3 * v + o ** 4)
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except ImportError:
        avail = None
    if avail is not None and avail < 2.0 * need:
        raise SystemExit(f"workload {wl}: host lists need {need / 1e9:.1f} GB pinned, "
                         f"only {avail / 1e9:.1f} GB available")
    eps, B, irr = synthetic_df(**wl)
    return _lists_from_df(eps, B, o, v, device)


def _lists_from_df(eps, B, o, v, device):
    import torch
    from acesb200 import INTEGRAL_LISTS
    Bt = torch.from_numpy(B).to(device)
    sl = {"o": slice(0, o), "v": slice(o, o + v)}
    out = {}
    for lst, (tl, tr, key, perm) in INTEGRAL_LISTS.items():
        # physicists' <pq|rs> = (pr|qs)
        p, q, r, s = key
        L1 = Bt[:, sl[p], sl[r]].reshape(Bt.shape[0], -1)
        L2 = Bt[:, sl[q], sl[s]].reshape(Bt.shape[0], -1)
        X = (L1.T @ L2).reshape(Bt[:, sl[p], sl[r]].shape[1:] + Bt[:, sl[q], sl[s]].shape[1:])
        phys = X.permute(0, 2, 1, 3)                  # [p,q,r,s]
        dense = phys.permute(*perm)                   # [row p, row q, col r, col s]
        buf = dense.permute(3, 2, 1, 0).contiguous()  # column-major list matrix
        host = torch.empty(buf.shape, dtype=torch.float64, pin_memory=(device.type == "cuda"))
        host.copy_(buf)
        out[lst] = (tl, tr, host)
        del X, phys, dense, buf
    del Bt
    if device.type == "cuda":
        torch.cuda.synchronize(device)
        torch.cuda.empty_cache()
    return eps, out, o, v


def put_lists_dpd(lib, eps, B, irr, o, v, device):
    """sym_init + the six integral lists + SCFEVALA of an irrep-blocked DF
    system: each list's dense <pq|rs> is built on the GPU and every irrep block
    gathered there in the list's pair order (DPD tables from the library's own
    ISYMOFF), then PUTLST from host memory.  Returns the host bytes put."""
    import numpy as np
    import torch
    from acesb200 import INTEGRAL_LISTS
    from acesb200.dpd import DPD
    irr_o, irr_v = np.asarray(irr[:o]), np.asarray(irr[o:])
    pop = [int(np.sum(irr_o == h)) for h in range(8)]
    vrt = [int(np.sum(irr_v == h)) for h in range(8)]
    lib.sym_init(pop, vrt)
    dpd = DPD(lib, irr_o, irr_v)
    lib.putrec("SCFEVALA", np.asarray(eps, dtype=np.float64))
    nbytes = eps.nbytes
    Bt = torch.from_numpy(B).to(device)
    sl = {"o": slice(0, o), "v": slice(o, o + v)}
    for lst, (tl, tr, key, perm) in INTEGRAL_LISTS.items():
        p, q, r, s_ = key
        L1 = Bt[:, sl[p], sl[r]].reshape(Bt.shape[0], -1)
        L2 = Bt[:, sl[q], sl[s_]].reshape(Bt.shape[0], -1)
        X = (L1.T @ L2).reshape(Bt[:, sl[p], sl[r]].shape[1:] + Bt[:, sl[q], sl[s_]].shape[1:])
        dense = X.permute(0, 2, 1, 3).permute(*perm)   # [row p, row q, col r, col s]
        lib.inipck(1, tl, tr, lst)
        ridx, rsgn, rh = dpd.table(tl)
        cidx, csgn, ch = dpd.table(tr)
        for h in range(lib.nirrep):
            nr, nc = lib.irpdpd(h + 1, tl), lib.irpdpd(h + 1, tr)
            if nr == 0 or nc == 0:
                continue
            P, Q = np.nonzero((rh == h) & (rsgn == 1))
            k = np.argsort(ridx[P, Q])
            P, Q = P[k], Q[k]
            R, S = np.nonzero((ch == h) & (csgn == 1))
            k = np.argsort(cidx[R, S])
            R, S = R[k], S[k]
            T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(device)
            M = dense[T(P)[:, None], T(Q)[:, None], T(R)[None, :], T(S)[None, :]]
            host = M.t().contiguous().cpu().numpy()   # column-major nr x nc
            lib.putlst_raw(host, 1, nc, h + 1, lst)
            nbytes += host.nbytes
        del X, dense
    del Bt
    torch.cuda.synchronize(device)
    torch.cuda.empty_cache()
    return nbytes


def run_batch(a, rank=0, world=1, local_rank=0):
    """The 64-system batch (C5): nocc ~ U{4..24}, nvir ~ U{30..220}, 8 irreps of
    uneven size, seeds 1000+k (all 64 converge with the generator as given).
    Each system is solved to CC_CONV 7 in split precision and in FP64, one
    after another through xvcc_run on one library instance (aces_init between
    systems; device memory is recycled by the engine's caching allocator);
    prints one JSON line with the summed times (setup + cycles).  With several
    ranks the systems are split by flop weight (o^2 v^4, heaviest first to the
    least-loaded rank), the batch time is the slowest rank's and the
    per-system results are gathered."""
    import numpy as np
    import torch
    import acesb200 as ab
    from acesb200.parallel import assign_systems, gather_values
    from acesb200.workloads import batch_systems, synthetic_df
    dev = torch.device("cuda", local_rank)
    lib = ab.load()
    systems = batch_systems()
    mine = assign_systems([s_["nocc"] ** 2 * s_["nvir"] ** 4 for s_ in systems], world)[rank]
    rows = []
    tot = {"bf16x3": 0.0, "fp64": 0.0}
    flops_ladder = 0.0
    flops_exec = 0.0
    # tile autotuner: one untimed split-precision cycle of every system of
    # this rank times the tile variants of each shape class the batch meets,
    # so the timed solves launch the cached choices
    tune = 1 if a.autotune is None else a.autotune
    lib.init(local_rank)
    lib.set_autotune(2)
    lib.set_autotune(tune)
    if tune:
        for k in mine:
            eps, B, irr = synthetic_df(**systems[k], bscale=a.batch_bscale)
            lib.init(local_rank)
            put_lists_dpd(lib, eps, B, irr, systems[k]["nocc"], systems[k]["nvir"], dev)
            lib.xvcc(cc_conv=7, cc_maxcyc=1, cc_exporder=5, precision=ab.PREC_BF16X3,
                     allow_noconv=True, use_graph=0)
    tuned_before = lib.autotune_stats()
    # warm-up, untimed: the heaviest of this rank's systems once in each
    # precision, so the timed solves find every kernel loaded and the device
    # pool holding blocks of the largest sizes (as in a long batch)
    if mine:
        kw = max(mine, key=lambda k_: systems[k_]["nocc"] ** 2 * systems[k_]["nvir"] ** 4)
        eps, B, irr = synthetic_df(**systems[kw], bscale=a.batch_bscale)
        lib.init(local_rank)
        put_lists_dpd(lib, eps, B, irr, systems[kw]["nocc"], systems[kw]["nvir"], dev)
        for prec in (ab.PREC_BF16X3, ab.PREC_FP64):
            lib.xvcc(cc_conv=7, cc_maxcyc=80, cc_exporder=5, precision=prec, allow_noconv=True,
                     use_graph=a.use_graph)
    for k, sysk in enumerate(systems):
        if k not in mine:
            continue
        eps, B, irr = synthetic_df(**sysk, bscale=a.batch_bscale)
        o, v = sysk["nocc"], sysk["nvir"]
        lib.init(local_rank)
        put_lists_dpd(lib, eps, B, irr, o, v, dev)
        # particle-particle ladder flops summed over the irrep blocks (the
        # reference's per-irrep LADAB1 products), and what the engine executes:
        # the packed symmetric / antisymmetric pair blocks of every pair irrep
        flops_ladder += sum(2.0 * lib.irpdpd(h + 1, 13) ** 2 * lib.irpdpd(h + 1, 14)
                            for h in range(lib.nirrep))
        io, iv = np.asarray(irr[:o]), np.asarray(irr[o:])
        for g in range(lib.nirrep):
            nij = int(np.sum((io[:, None] ^ io[None, :]) == g))
            pg = (iv[:, None] ^ iv[None, :]) == g
            npl = int(np.sum(np.triu(pg)))          # c <= d
            nmi = int(np.sum(np.triu(pg, 1)))       # c < d
            flops_exec += 2.0 * nij * (npl * npl + nmi * nmi)
        row = {"k": k, "nocc": o, "nvir": v}
        for prec, name in ((ab.PREC_BF16X3, "bf16x3"), (ab.PREC_FP64, "fp64")):
            c = lib.xvcc(cc_conv=7, cc_maxcyc=80, cc_exporder=5, precision=prec,
                         allow_noconv=True, use_graph=a.use_graph)
            t = c.seconds_setup + c.seconds_per_iter * c.ncycle
            tot[name] += t
            row[name] = {"e": c.e_ccsd, "cycles": c.ncycle, "converged": bool(c.converged),
                         "seconds": t, "setup_seconds": c.seconds_setup,
                         "seconds_per_iter": c.seconds_per_iter}
        rows.append(row)
    tuned_after = lib.autotune_stats()
    lib.set_autotune(0)
    lib.fin()
    dE = [abs(r["bf16x3"]["e"] - r["fp64"]["e"]) for r in rows]
    conv = all(r["bf16x3"]["converged"] and r["fp64"]["converged"] for r in rows)
    if world > 1:
        from acesb200.parallel import allreduce_max
        n = len(systems)
        e_split = gather_values({r["k"]: r["bf16x3"]["e"] for r in rows}, n, mine)
        e_fp64 = gather_values({r["k"]: r["fp64"]["e"] for r in rows}, n, mine)
        dE = [abs(x - y) for x, y in zip(e_split, e_fp64)]
        flops_ladder = sum(gather_values({0: flops_ladder}, 1, [0]))
        flops_exec = sum(gather_values({0: flops_exec}, 1, [0]))
        conv = allreduce_max(0.0 if conv else 1.0) == 0.0
        tot = {k_: allreduce_max(v_) for k_, v_ in tot.items()}
        if rank != 0:
            return
    line = {"metric": "C5 batch: 64 irrep-blocked CCSD solves (CC_CONV 7), total device time",
            "value": tot["bf16x3"], "unit": "s", "higher_is_better": False, "n_gpus": world,
            "dtype": "bf16x3",
            "data": f"synthetic: acesb200.workloads.batch_systems, B x {a.batch_bscale}",
            "config": {"workload": "c5: 64 systems, nocc 4-24, nvir 30-220, 8 irreps, "
                                   "seeds 1000-1063",
                       "warm_up": "one untimed solve of the heaviest system in each precision",
                       "execution": "sequential xvcc_run calls"
                                    + (f", systems split over {world} ranks by flop weight"
                                       if world > 1 else ""),
                       "use_graph": a.use_graph,
                       "autotune": {"on": bool(tune), "classes": tuned_after[0],
                                    "classes_off_default": tuned_after[1],
                                    "tuning_ms_untimed_pass": tuned_before[2],
                                    "classes_tuned_in_timed_solves":
                                        tuned_after[0] - tuned_before[0],
                                    "tuning_ms_in_timed_solves":
                                        tuned_after[2] - tuned_before[2]}},
            "scaling": "strong",
            "fp64_seconds": tot["fp64"], "speedup_split_vs_fp64": tot["fp64"] / tot["bf16x3"],
            "max_abs_dE": max(dE), "all_converged": conv,
            "ladder_flops_block_summed": flops_ladder,
            "ladder_flops_executed_packed_blocks": flops_exec,
            "systems": rows if world == 1 else f"{len(rows)} of {len(systems)} on rank 0"}
    print(json.dumps(line), flush=True)


def getlst_pinned(lib, host, lst, irrep=1):
    """GETLST of every column of (irrep, lst) into the pinned host tensor
    `host` (the caller-owned destination buffer of acescore/getlst.F)."""
    import ctypes
    nr, nc = lib.list_dims(irrep, lst)
    assert host.numel() >= nr * nc
    lib._chk("aces_getlst", lib.h.aces_getlst(ctypes.c_void_p(host.data_ptr()), 1, nc, irrep,
                                              lst))
    return host[:nr * nc]


def put_lists(lib, eps, lists):
    lib.putrec("SCFEVALA", eps)
    nbytes = eps.nbytes
    for lst, (tl, tr, host) in lists.items():
        lib.inipck(1, tl, tr, lst)
        a = host.numpy()
        lib.putlst_raw(a, 1, lib.irpdpd(1, tr), 1, lst)
        nbytes += a.nbytes
    return nbytes


# ------------------------------------------------------------------ arms
def run_ours(a, rank, world, local_rank):
    import numpy as np
    import torch
    import acesb200 as ab
    from acesb200.workloads import WORKLOADS, synthetic_df

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = WORKLOADS[a.workload]
    prec = ab.PREC_BF16X3 if a.precision == "bf16x3" else ab.PREC_FP64
    lib = ab.load()
    eps, lists, o, v = host_lists(wl, dev)
    K, W = a.steps, a.warmup
    # the residual graph is captured in the second cycle: with the graph on,
    # at least two cycles stay untimed whatever W is
    Wc = max(W, 2) if a.use_graph else W

    # ---- value: inputs resident, device-timed cycles after W warm-up cycles
    lib.init(local_rank)
    lib.sym_init([o], [v])
    put_lists(lib, eps, lists)
    torch.cuda.synchronize()
    barrier(world)
    with Clocks(local_rank) as clk:
        cfg = lib.xvcc(cc_conv=30, cc_maxcyc=Wc + K, cc_exporder=5, precision=prec,
                       timing_warmup=Wc, allow_noconv=True, use_graph=a.use_graph)
        torch.cuda.synchronize()
    barrier(world)
    s_iter = max_over_ranks(cfg.seconds_per_iter, world)
    s_lad = max_over_ranks(cfg.seconds_ladder, world)
    e_split = cfg.e_ccsd

    # ---- FP64 GPU path, same cycles, for the split-precision comparison
    fp64 = None
    if prec == ab.PREC_BF16X3 and not a.no_fp64_compare:
        c64 = lib.xvcc(cc_conv=30, cc_maxcyc=Wc + K, cc_exporder=5, precision=ab.PREC_FP64,
                       timing_warmup=Wc, allow_noconv=True, use_graph=a.use_graph)
        # the literal generator's iteration diverges (its <ab|cd> coupling
        # exceeds the denominators), so after W + K cycles the two paths'
        # energies are not a precision measure: the accuracy block compares
        # them on the convergent variant
        fp64 = {"seconds_per_iter": c64.seconds_per_iter,
                "speedup_split_vs_fp64": c64.seconds_per_iter / cfg.seconds_per_iter,
                "seconds_ladder": c64.seconds_ladder}
        try:
            fp64["cublas_reference"] = cublas_fp64_reference(o, v, dev)
            cb = fp64["cublas_reference"]
            fp64["ladder_vs_cublas_fp64"] = cb["ladder_seconds"] / max(c64.seconds_ladder, 1e-30)
            fp64["split_ladder_speedup_vs_cublas_fp64"] = cb["ladder_seconds"] / max(s_lad, 1e-30)
        except Exception as exc:  # noqa: BLE001
            fp64["cublas_reference"] = {"error": f"{type(exc).__name__}: {exc}"}

    # ---- e2e_putlst: host lists -> PUTLST -> xvcc_run (K cycles) -> GETLST T2
    lib.init(local_rank)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    lib.sym_init([o], [v])
    h2d_l = put_lists(lib, eps, lists)
    tp = time.perf_counter()
    ce = lib.xvcc(cc_conv=30, cc_maxcyc=K, cc_exporder=5, precision=prec, allow_noconv=True,
                  use_graph=a.use_graph)
    tx = time.perf_counter()
    nr, nc = lib.list_dims(1, 46)
    t2 = lib.getlst(1, nc, 1, 46)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    putlst_parts = {"putlst_s": tp - t0, "xvcc_s": tx - tp, "xvcc_setup_s": ce.seconds_setup,
                    "xvcc_cycles_device_s": ce.seconds_per_iter * K, "getlst_s": t1 - tx}
    barrier(world)
    e2e_l = max_over_ranks((t1 - t0) / K, world)
    d2h_l = t2.nbytes + 8
    del lists
    # ---- e2e: host DF factors -> aces_intprc_df -> xvcc_run (K cycles) -> GETLST T2,
    # once untimed (the device pool then holds blocks of every size the pass
    # asks for, as in a program that runs more than one calculation) and once timed
    eps_h, Bf, _ = synthetic_df(**wl)
    Bpin = torch.empty(Bf.shape, dtype=torch.float64, pin_memory=True)
    Bpin.copy_(torch.from_numpy(Bf))
    del Bf
    t2_host = torch.empty(o * o * v * v, dtype=torch.float64, pin_memory=True)

    def e2e_pass():
        lib.init(local_rank)
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        lib.sym_init([o], [v])
        lib.putrec("SCFEVALA", eps_h)
        lib.intprc_df(Bpin)
        tp = time.perf_counter()
        ce = lib.xvcc(cc_conv=30, cc_maxcyc=K, cc_exporder=5, precision=prec,
                      allow_noconv=True, use_graph=a.use_graph)
        tx = time.perf_counter()
        t2 = getlst_pinned(lib, t2_host, 46)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        parts = {"intprc_df_s": tp - t0, "xvcc_s": tx - tp, "xvcc_setup_s": ce.seconds_setup,
                 "xvcc_cycles_device_s": ce.seconds_per_iter * K, "getlst_s": t1 - tx}
        barrier(world)
        return max_over_ranks((t1 - t0) / K, world), parts, t2.numel() * 8

    e2e_pass()
    e2e, e2e_parts, t2_bytes = e2e_pass()
    h2d = Bpin.numel() * 8 + eps_h.nbytes
    d2h = t2_bytes + 8
    del Bpin, t2_host
    lib.fin()

    pk, pk_src = peaks()
    # the ladder runs packed (symmetric + antisymmetric pair blocks): its own
    # contraction flops, and the reference's dense 2 o^2 v^4 for comparison
    n_p, n_m = v * (v + 1) // 2, v * (v - 1) // 2
    launch_flops = 2.0 * (o * o) * (n_p * n_p + n_m * n_m)
    dense_flops = 2.0 * (o * o) * (v * v) * (v * v)
    if prec == ab.PREC_BF16X3:
        executed = 3.0 * launch_flops
        peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
        roof = {"bound": "tensor",
                "kernel": "k_gemm_bf16x3 (particle-particle ladder, symmetric + antisymmetric "
                          "pair blocks, with its pack/unpack kernels)",
                "reference_dense_flops_per_launch": dense_flops,
                "effective_dense_tflops": dense_flops / s_lad / 1e12,
                "achieved": executed / s_lad / 1e12, "peak": peak, "unit": "TFLOP/s",
                "frac": executed / s_lad / 1e12 / peak,
                "peak_source": f"bf16_tflops_sustained of {pk_src} MEASURED_PEAKS.json",
                "algorithmic_flops_per_launch": launch_flops,
                "executed_bf16_flops_per_launch": executed,
                "seconds_per_launch": s_lad,
                "seconds_note": "CUDA events around the packed ladder (external event nodes "
                                "of the replayed residual graph under --use-graph 1): the "
                                "grouped launch plus its pack/unpack kernels (~0.16 ms at c2)",
                "traffic": LADDER_TRAFFIC.get(a.workload),
                "traffic_source": LADDER_TRAFFIC_SOURCE if a.workload in LADDER_TRAFFIC else None,
                "algorithmic_bytes_per_launch": 4.0 * (n_p * n_p + n_m * n_m)
                + 4.0 * (o * o) * (v * v) + 3 * 8.0 * (o * o) * (v * v)}
    else:
        roof = {"bound": "tensor", "kernel": "k_gemm_nt_f64 (particle-particle ladder)",
                "achieved": launch_flops / s_lad / 1e12, "peak": None, "unit": "TFLOP/s",
                "frac": None, "peak_source": "no FP64 peak in MEASURED_PEAKS.json",
                "algorithmic_flops_per_launch": launch_flops, "seconds_per_launch": s_lad,
                "traffic": None}

    line = {
        "metric": f"CCSD s/iter, synthetic closed-shell o={o} v={v} naux={wl['naux']} (split BF16x3 vs FP64 GPU)",
        "value": s_iter, "unit": "s/iter", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": s_iter * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16x3" if prec == ab.PREC_BF16X3 else "f64",
        "data": f"synthetic: seeded DF generator (acesb200.workloads {a.workload})",
        "config": {"workload": f"{a.workload}: RHF-CCSD, C1, nocc={o}, nvir={v}, naux={wl['naux']}, "
                               f"seed={wl['seed']}",
                   "precision": a.precision, "cycles_timed": K, "cycles_untimed": Wc,
                   "diis_order": 5,
                   "l2": "inputs larger than L2 (<ab|cd> 8.4 GB read every step)",
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "residual_graph": bool(a.use_graph)},
        "e2e": {"value": e2e, "unit": "s/iter", "h2d_bytes_per_step": h2d // K,
                "d2h_bytes_per_step": d2h // K,
                "note": "pinned host DF factors + SCFEVALA -> aces_intprc_df (lists built on "
                        "the device) + xvcc_run(K cycles) + GETLST T2, wall clock / K; "
                        "the second of two identical passes (the first warms the device pool)",
                "parts": e2e_parts},
        "e2e_putlst": {"value": e2e_l, "unit": "s/iter", "h2d_bytes_per_step": h2d_l // K,
                       "d2h_bytes_per_step": d2h_l // K,
                       "note": "the six lists built on the host, PUTLST from pinned memory + "
                               "xvcc_run(K cycles) + GETLST T2, wall clock / K",
                       "parts": putlst_parts},
        "roofline": roof,
        "gpu_launches": int(cfg.launches_per_iter) * K,
        "clocks": clk.summary(),
        "energy": {"e_corr_after_cycles": e_split, "cycles": Wc + K,
                   "note": "the literal generator's CC iteration diverges (timing does not "
                           "depend on it); split vs FP64 accuracy is the accuracy block, "
                           "on the convergent variant"},
        "flops_per_iter": cfg.flops_per_iter,
        "setup_seconds": cfg.seconds_setup,
    }
    if fp64:
        line["fp64_gpu"] = fp64
    if prec == ab.PREC_BF16X3 and not a.no_fp64_compare:
        line["accuracy"] = accuracy(lib, a.workload + "conv", local_rank, rank, world,
                                    use_graph=a.use_graph)
    # the secondary blocks (no collectives inside) report a failure in the
    # line instead of taking the headline measurement down with them
    if prec == ab.PREC_BF16X3 and not a.no_lambda and a.workload == W_NAME:
        try:
            line["lambda"] = lambda_block(lib, "c4conv", local_rank)
        except Exception as exc:  # noqa: BLE001
            line["lambda"] = {"error": f"{type(exc).__name__}: {exc}"}
    if prec == ab.PREC_BF16X3 and not a.no_lambda and a.workload == W_NAME:
        try:
            line["eom"] = eom_block(lib, "c2conv", local_rank)
        except Exception as exc:  # noqa: BLE001
            line["eom"] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(a.workload, budget_s=90.0)
        except Exception as exc:  # noqa: BLE001
            line["cpu_baseline"] = {"error": f"{type(exc).__name__}: {exc}"}
    return line


# DRAM bytes of the grouped packed-ladder launch of the c2 cycle: an ncu
# capture of its symmetric product alone (--kernel-case ladder-packed, M = K =
# 16290, N = 400: 1161.2 MB read + 45.4 MB written) scaled by the units the
# grouped launch processes, (16290^2 + 16110^2) / 16290^2
LADDER_TRAFFIC = {"c2": (1161.2e6 + 45.4e6) * (16290 ** 2 + 16110 ** 2) / 16290 ** 2}
LADDER_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the symmetric ladder "
                         "product (--kernel-case ladder-packed) scaled to the grouped launch by "
                         "(n+^2 + n-^2) / n+^2")


def cublas_fp64_reference(o, v, dev, reps=5):
    """FP64 tensor-core throughput of the vendor library on this GPU, as the
    yardstick for the FP64 path (the measured peaks hold no FP64 figure):
    cuBLAS DGEMM (through torch.matmul) on an 8192^3 product and on the two
    products of the packed particle-particle ladder at this workload's shape
    (M = K = v(v+1)/2 and v(v-1)/2, N = o^2), CUDA-event timed after a
    warm-up.  Only a comparator: no product of the engine uses cuBLAS."""
    import torch
    out = {}

    def timed(fn):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) * 1e-3 / reps

    n = 8192
    A = torch.randn(n, n, dtype=torch.float64, device=dev)
    Bm = torch.randn(n, n, dtype=torch.float64, device=dev)
    t = timed(lambda: A @ Bm)
    out["dgemm_8192_tflops"] = 2.0 * n ** 3 / t / 1e12
    del A, Bm
    np_, nm_ = v * (v + 1) // 2, v * (v - 1) // 2
    tl = 0.0
    for m in (np_, nm_):
        U = torch.randn(m, m, dtype=torch.float64, device=dev)
        X = torch.randn(m, o * o, dtype=torch.float64, device=dev)
        tl += timed(lambda: U @ X)
        del U, X
    torch.cuda.empty_cache()
    out["ladder_seconds"] = tl
    out["ladder_tflops"] = 2.0 * o * o * (np_ * np_ + nm_ * nm_) / tl / 1e12
    out["note"] = ("cuBLAS FP64 through torch.matmul; the packed ladder's two products "
                   "without the pack/unpack kernels")
    return out


def accuracy(lib, wname, device, rank=0, world=1, use_graph=1):
    """Split BF16x3 vs FP64 GPU on the convergent variant of the workload, both
    converged to max|dT| < 1e-9 (CC_CONV=9): |dE| of the correlation energy.
    With several ranks rank 0 solves CCSD, broadcasts the amplitudes, and the
    (T) triplets are split over the ranks; the partial energies are
    all-reduced."""
    from acesb200.parallel import triples_from_root
    import torch
    import acesb200 as ab
    from acesb200.workloads import WORKLOADS
    from acesb200.workloads import synthetic_df
    wl = WORKLOADS[wname]
    eps, B, irr = synthetic_df(**wl)
    o, v = wl["nocc"], wl["nvir"]
    lists = _lists_from_df(eps, B, o, v, torch.device("cuda", device))
    lib.init(device)
    lib.sym_init([o], [v])
    put_lists(lib, eps, lists[1])
    res = {}
    for prec, name in ((ab.PREC_FP64, "fp64"), (ab.PREC_BF16X3, "bf16x3")):
        # cycle 1 (integral splits, packed ladder matrices) is setup, not an iteration
        kw = dict(cc_conv=9, cc_maxcyc=80, cc_exporder=5, precision=prec, allow_noconv=True,
                  timing_warmup=1, use_graph=use_graph)
        if world > 1:
            c = triples_from_root(lib, rank, world, **kw)
        else:
            c = lib.xvcc(triples=1, **kw)
        res[name] = {"e_corr": c.e_ccsd, "cycles": c.ncycle, "converged": bool(c.converged),
                     "seconds_per_iter": c.seconds_per_iter, "e_t4": c.e_t4, "e_st5": c.e_st5,
                     "seconds_triples": c.seconds_triples}
    lib.fin()
    # (T) work: per unique triplet three class contractions of 2 v^3 (2v + 2o)
    # flops (the 12 terms of trp/d1t2new.F), each executed as 3 BF16 products
    ntrip = o * (o + 1) * (o + 2) // 6
    tflops = ntrip * 3 * 2.0 * v ** 3 * (2 * v + 2 * o)
    pk, pk_src = peaks()
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    st = max(res["bf16x3"]["seconds_triples"], 1e-30)
    troof = {"kernel": "k_gemm_bf16x3 batched triplet classes + k_triples_energy",
             "triplets": ntrip, "algorithmic_flops": tflops,
             "achieved": 3.0 * tflops / st / 1e12 / world, "unit": "TFLOP/s per GPU",
             "peak": peak, "frac": 3.0 * tflops / st / 1e12 / world / peak,
             "peak_source": f"bf16_tflops_sustained of {pk_src} MEASURED_PEAKS.json",
             "seconds": res["bf16x3"]["seconds_triples"]}
    return {"workload": f"{wname}: nocc={o}, nvir={v}, naux={wl['naux']}, seed={wl['seed']}, "
                        f"B scaled by {wl['bscale']} (convergent variant)",
            "triples_roofline": troof,
            "triples_ranks": world,
            "fp64": res["fp64"], "bf16x3": res["bf16x3"],
            "abs_dE": abs(res["bf16x3"]["e_corr"] - res["fp64"]["e_corr"]),
            "abs_dE_T": abs(res["bf16x3"]["e_t4"] + res["bf16x3"]["e_st5"]
                            - res["fp64"]["e_t4"] - res["fp64"]["e_st5"]),
            "speedup_per_iter": res["fp64"]["seconds_per_iter"] / res["bf16x3"]["seconds_per_iter"],
            "speedup_triples": res["fp64"]["seconds_triples"] / res["bf16x3"]["seconds_triples"]}


def lambda_block(lib, wname, device, seed=4, delta=1e-4):
    """Lambda equations + one-particle density on the convergent C4 system
    (o=20, v=180, seed 3, B scaled by 1/4): Lambda s/iter for both precisions,
    and dE/dx = Tr(D h') for f -> f + x h' (h' seeded, symmetric, N(0, 0.01^2)
    entries) against a central finite difference (step delta) of FP64 CCSD
    energies, and the split-precision density against the FP64 one."""
    import time
    import numpy as np
    import torch
    import acesb200 as ab
    from acesb200.workloads import WORKLOADS, synthetic_df
    wl = WORKLOADS[wname]
    eps, B, irr = synthetic_df(**wl)
    o, v = wl["nocc"], wl["nvir"]
    n = o + v
    lists = _lists_from_df(eps, B, o, v, torch.device("cuda", device))
    rng = np.random.default_rng(seed)
    hp = rng.normal(0.0, 0.01, (n, n))
    hp = 0.5 * (hp + hp.T)
    f0 = np.diag(eps)

    def load(fock):
        lib.init(device)
        lib.sym_init([o], [v])
        put_lists(lib, lists[0], lists[1])
        lib.putrec("FOCKMAT", fock)

    out = {"workload": f"{wname}: nocc={o}, nvir={v}, naux={wl['naux']}, seed={wl['seed']}, "
                       f"B scaled by {wl.get('bscale', 1.0)}; h' seed {seed}",
           "delta": delta}
    dens = {}
    # the split path's residual floor is ~5e-10 (CC_CONV 9); FP64 converges to 1e-10
    for prec, name, conv in ((ab.PREC_FP64, "fp64", 10), (ab.PREC_BF16X3, "bf16x3", 9)):
        load(f0)
        c = lib.xvcc(cc_conv=conv, cc_maxcyc=80, cc_exporder=5, precision=prec)
        t0 = time.perf_counter()
        cl = lib.xlambda(cc_conv=conv, cc_maxcyc=80, cc_exporder=5, precision=prec,
                         timing_warmup=1)
        t1 = time.perf_counter()
        lib.xdens()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        D = lib.getrec("DENSMAT", n * n).reshape(n, n)
        dens[name] = D
        out[name] = {"cc_conv": conv, "e_ccsd": c.e_ccsd, "ccsd_cycles": c.ncycle,
                     "lambda_cycles": cl.ncycle, "lambda_converged": bool(cl.converged),
                     "lambda_seconds_per_iter": cl.seconds_per_iter,
                     "lambda_seconds_total": t1 - t0, "density_seconds": t2 - t1,
                     "dE_dx_analytic": float(np.sum(D * hp))}
    e = {}
    for sgn in (+1, -1):
        load(f0 + sgn * delta * hp)
        e[sgn] = lib.xvcc(cc_conv=11, cc_maxcyc=100, cc_exporder=5, precision=ab.PREC_FP64).e_ccsd
    fd = (e[+1] - e[-1]) / (2.0 * delta)
    out["dE_dx_finite_difference_fp64"] = fd
    out["abs_diff_analytic_fp64_vs_fd"] = abs(out["fp64"]["dE_dx_analytic"] - fd)
    out["abs_diff_bf16x3_vs_fp64"] = abs(out["bf16x3"]["dE_dx_analytic"] -
                                         out["fp64"]["dE_dx_analytic"])
    out["max_abs_density_diff_bf16x3_vs_fp64"] = float(np.abs(dens["bf16x3"] - dens["fp64"]).max())
    out["lambda_speedup_bf16x3_vs_fp64"] = (out["fp64"]["lambda_seconds_per_iter"] /
                                            out["bf16x3"]["lambda_seconds_per_iter"])
    lib.fin()
    return out


def eom_block(lib, wname, device, nroots=2):
    """Singlet EOM-EE-CCSD (xvee_run) on the convergent c2 system: the lowest
    `nroots` excitation energies in split precision and in FP64, each after
    its own CCSD (CC_CONV 9), with the Davidson's Jacobian-product count and
    time per product (one reverse replay of the residual pass each)."""
    import torch
    import acesb200 as ab
    from acesb200.workloads import WORKLOADS, synthetic_df
    wl = WORKLOADS[wname]
    eps, B, _ = synthetic_df(**wl)
    o, v = wl["nocc"], wl["nvir"]
    out = {"workload": f"{wname}: nocc={o}, nvir={v}, naux={wl['naux']}, seed={wl['seed']}, "
                       f"B scaled by {wl['bscale']}", "nroots": nroots}
    for prec, name in ((ab.PREC_BF16X3, "bf16x3"), (ab.PREC_FP64, "fp64")):
        lib.init(device)
        lib.sym_init([o], [v])
        lib.putrec("SCFEVALA", eps)
        lib.intprc_df(torch.from_numpy(B).to(torch.device("cuda", device)))
        lib.xvcc(cc_conv=9, cc_maxcyc=80, cc_exporder=5, precision=prec)
        cfg, w = lib.xvee([nroots], eom_conv=6, eom_maxcyc=60, precision=prec)
        out[name] = {"omega": w[0], "iterations": cfg.niter[0], "products": cfg.nsigma,
                     "seconds": cfg.seconds, "seconds_per_product": cfg.seconds / max(cfg.nsigma, 1)}
    lib.fin()
    out["max_abs_domega"] = max(abs(x - y) for x, y in zip(out["bf16x3"]["omega"],
                                                           out["fp64"]["omega"]))
    out["speedup_per_product"] = (out["fp64"]["seconds_per_product"] /
                                  out["bf16x3"]["seconds_per_product"])
    return out


def cpu_baseline(wname, budget_s=90.0, steps=1):
    """The oracle (FP64 numpy restatement of the reference) on the host cores:
    CCSD iterations of the same system, each from its MP2 amplitudes (finite
    data every step); integral build excluded.  With all host threads, then
    one iteration on one thread (the reference's own serial design) when the
    multi-threaded time says it fits the budget."""
    import numpy as np
    from acesb200.workloads import WORKLOADS
    from oracle.hamiltonian import synthetic
    from oracle import ccsd
    wl = WORKLOADS[wname]
    ham = synthetic(**wl)
    B = ccsd.Blocks(ham)
    t1, t2 = ccsd.mp2_guess(B)
    times = []
    t_start = time.perf_counter()
    for k in range(max(1, steps)):
        t0 = time.perf_counter()
        t1n, t2n = ccsd.update(B, t1, t2)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    assert np.isfinite(t1n).all() and np.isfinite(t2n).all()
    cores = os.cpu_count()
    out = {"value": min(times), "unit": "s/iter", "cores": cores, "kind": "port",
           "sample": f"{len(times)} full CCSD iteration(s) of the {wname} system "
                     f"(o={wl['nocc']}, v={wl['nvir']}) from its MP2 amplitudes with "
                     f"oracle/ccsd.py (numpy FP64, OpenBLAS threads = {cores}); integral "
                     f"build excluded",
           "iterations": len(times)}
    try:
        from threadpoolctl import threadpool_limits
        if min(times) * cores <= 2.0 * budget_s:
            with threadpool_limits(limits=1):
                t0 = time.perf_counter()
                ccsd.update(B, t1, t2)
                out["single_thread"] = {"value": time.perf_counter() - t0, "unit": "s/iter",
                                        "cores": 1, "iterations": 1}
        else:
            out["single_thread"] = {"skipped": f"estimated {min(times) * cores:.0f} s > "
                                               f"{2.0 * budget_s:.0f} s budget"}
    except ImportError:
        out["single_thread"] = {"skipped": "threadpoolctl unavailable"}
    return out


def run_reference(a, rank, world):
    if rank != 0:
        return None
    from acesb200.workloads import WORKLOADS
    from oracle.hamiltonian import synthetic
    from oracle import ccsd
    wl = WORKLOADS[a.workload]
    ham = synthetic(**wl)
    import numpy as np
    B = ccsd.Blocks(ham)
    t1, t2 = ccsd.mp2_guess(B)
    # every step is one CCSD iteration from the same MP2 amplitudes: the
    # literal generator's iteration diverges, and timing a chain of updates
    # would time arithmetic on overflowed values after a few steps
    W = min(a.warmup, 1)
    for _ in range(W):
        ccsd.update(B, t1, t2)
    times = []
    t_start = time.perf_counter()
    for _ in range(a.steps):
        t0 = time.perf_counter()
        n1, n2 = ccsd.update(B, t1, t2)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > 150.0:
            break
    assert np.isfinite(n1).all() and np.isfinite(n2).all()
    v = statistics.mean(times)
    cores = os.cpu_count()
    return {
        "impl": "reference",
        "metric": f"CCSD s/iter, synthetic closed-shell o={wl['nocc']} v={wl['nvir']} naux={wl['naux']} (split BF16x3 vs FP64 GPU)",
        "value": v, "unit": "s/iter", "n_gpus": world, "steps": len(times), "warmup": W,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded DF generator",
        "config": {"workload": f"{a.workload}: RHF-CCSD, C1, nocc={wl['nocc']}, nvir={wl['nvir']}, "
                               f"naux={wl['naux']}, seed={wl['seed']}",
                   "note": "the reference (Fortran xvcc) cannot be compiled here (no Fortran "
                           "compiler); this arm times its numpy FP64 restatement"},
        "cpu_baseline": {"value": v, "unit": "s/iter", "cores": cores, "kind": "port",
                         "sample": f"{len(times)} CCSD iterations of the {a.workload} system, "
                                   f"each from its MP2 amplitudes (numpy FP64, OpenBLAS "
                                   f"threads = {cores})"},
        "e2e": {"value": v, "unit": "s/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------ ranks
def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    from acesb200.parallel import allreduce_max
    return allreduce_max(x)


KERNEL_CASES = {
    # particle-particle ladder shape Z(ab,ij) = W(ab,ef) tau(ef,ij) at v=120, o=20:
    # M = K = v^2 = 14400, N = o^2 = 400; A (FP64 1.66 GB, split 0.83 GB) exceeds L2
    "ladder-small": dict(m=14400, n=400, k=14400),
    # T1-dressing shape W(ajb,i) = sum_e <ajb|e> t(i,e) at o=20, v=180:
    # M = o*v*v = 648000, N = o = 20, K = v = 180
    "thin-t1": dict(m=648000, n=20, k=180),
    # T1-dressing rank-o update W(jbm,e) += sum_n t(n,e) X(jbm,n) at o=20, v=180,
    # accumulated into the existing output: M = o*o*v = 72000, N = v = 180, K = o = 20
    "lowrank-t1": dict(m=72000, n=180, k=20, beta=1.0),
    # symmetric block of the packed particle-particle ladder at o=20, v=180:
    # M = K = v(v+1)/2 = 16290, N = o^2 = 400
    "ladder-packed": dict(m=16290, n=400, k=16290),
}
# whole-program cases: a converged CCSD(T) on a small seeded system (ncu
# captures of the (T) launches; B scaled by 0.25 so the amplitudes converge)
PROGRAM_CASES = {
    "triples-o10-v180": dict(nocc=10, nvir=180, naux=540, seed=5, bscale=0.25),
    # the same kernels on a few GB of device memory (56 triplets, one batch)
    "triples-o6-v128": dict(nocc=6, nvir=128, naux=300, seed=5, bscale=0.25),
    # v = 136 > 128: the (T) classes on 128 x 256 tiles, a few GB on the device
    "triples-o4-v136": dict(nocc=4, nvir=136, naux=200, seed=5, bscale=0.25),
    # Lambda + density on the convergent C4 system (split precision)
    "lambda-c4": dict(nocc=20, nvir=180, naux=600, seed=3, bscale=0.25, lam=True),
    # split CCSD cycles of a system whose o^2 v^2 arrays (128 MB) exceed L2 while
    # the whole run holds a few GB: DRAM counters of the bandwidth-bound kernels
    "ccsd-o40-v100": dict(nocc=40, nvir=100, naux=300, seed=7, bscale=0.25, cycles=4),
}


def run_program_case(a):
    """CCSD (split precision, CC_CONV=7) and (T) on a PROGRAM_CASES system;
    prints the (T) device time and energies."""
    import torch
    import acesb200 as ab
    from acesb200.workloads import synthetic_df
    wl = dict(PROGRAM_CASES[a.kernel_case])
    lam = wl.pop("lam", False)
    cycles = wl.pop("cycles", None)
    eps, B, _ = synthetic_df(**wl)
    e, lists, o, v = _lists_from_df(eps, B, wl["nocc"], wl["nvir"], torch.device("cuda", 0))
    lib = ab.load()
    lib.init(0)
    lib.sym_init([o], [v])
    put_lists(lib, e, lists)
    if cycles:
        c = lib.xvcc(cc_conv=30, cc_maxcyc=cycles, cc_exporder=5, precision=ab.PREC_BF16X3,
                     allow_noconv=True)
        print(json.dumps({"kernel_case": a.kernel_case, "cycles": c.ncycle,
                          "seconds_per_iter": c.seconds_per_iter,
                          "launches_per_iter": c.launches_per_iter}), flush=True)
    elif lam:
        c = lib.xvcc(cc_conv=9, cc_maxcyc=60, cc_exporder=5, precision=ab.PREC_BF16X3)
        cl = lib.xlambda(cc_conv=9, cc_maxcyc=60, cc_exporder=5, precision=ab.PREC_BF16X3,
                         timing_warmup=1)
        lib.xdens()
        print(json.dumps({"kernel_case": a.kernel_case, "e_ccsd": c.e_ccsd, "cycles": c.ncycle,
                          "lambda_cycles": cl.ncycle,
                          "lambda_seconds_per_iter": cl.seconds_per_iter}), flush=True)
    else:
        c = lib.xvcc(cc_conv=7, cc_maxcyc=60, cc_exporder=5, precision=ab.PREC_BF16X3, triples=1)
        print(json.dumps({"kernel_case": a.kernel_case, "e_ccsd": c.e_ccsd, "cycles": c.ncycle,
                          "e_t4": c.e_t4, "e_st5": c.e_st5,
                          "seconds_triples": c.seconds_triples}), flush=True)
    lib.fin()


def run_kernel_case(a):
    """One XGEMM of a ladder-like shape, FP64 inputs -> split -> tcgen05, then
    the same shape in FP64 (DMMA); prints device times (CUDA events)."""
    import torch
    import acesb200 as ab
    if a.kernel_case in PROGRAM_CASES:
        return run_program_case(a)
    c = KERNEL_CASES[a.kernel_case]
    m, n, k = c["m"], c["n"], c["k"]
    beta = c.get("beta", 0.0)
    lib = ab.load()
    lib.init(0)
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn((m, k), dtype=torch.float64, device="cuda", generator=g)   # column-major op(A)=A^T
    B = torch.randn((n, k), dtype=torch.float64, device="cuda", generator=g)
    C = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    out = {}
    for prec, name in ((ab.PREC_BF16X3, "bf16x3"), (ab.PREC_FP64, "fp64")):
        for rep in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            # C(m x n) = A^T(m x k) * B(k x n): column-major A stored (k x m) = our row-major (m,k)
            lib.xgemm("T", "N", m, n, k, 1.0, A.data_ptr(), k, B.data_ptr(), k, beta,
                      C.data_ptr(), m, precision=prec)
            e1.record()
            torch.cuda.synchronize()
            out[name] = e0.elapsed_time(e1) * 1e-3
    print(json.dumps({"kernel_case": a.kernel_case, "m": m, "n": n, "k": k, "beta": beta,
                      "seconds_including_split_pack": out}), flush=True)


def main():
    a = args()
    if a.kernel_case:
        run_kernel_case(a)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        line = run_reference(a, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    try:
        if a.workload == "c5":
            run_batch(a, rank, world, local_rank)
            return
        line = run_ours(a, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
