#!/usr/bin/env python
"""Benchmark of the MW operator apply (batched Helmholtz, config 2).

Workload (one step): 32 orbitals, each a normalised sum of 2-6 Gaussians (exponents log-U[0.5,200],
centres on 8 seeded atom sites in a 6 Bohr box), projected at prec 1e-6 with interpolating order 9
(k = 10) on the [-20,20]^3 world; one Helmholtz operator per orbital (mu ~ U[0.5,3]); the step
applies all 32 operators (out_i = H_i phi_i, adaptive, prec 1e-6).  Inputs are resident in HBM
when the timed region starts; their coefficient blocks (several GB per step) are larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1: one process per GPU (torchrun); weak scaling, each rank applies its own 32-orbital batch.
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MW Poisson/Helmholtz apply time at 1e-6 rel. error: mixed+learned vs plain FP64 GPU"
FP64_PEAK_NOMINAL = 37.0  # TFLOP/s, B200 datasheet FP64 (no measured FP64 peak on this pool)
FP32_PEAK_NOMINAL = 74.4  # TFLOP/s, 148 SMs x 128 FP32 lanes x 2 x 1.965 GHz


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="mw", choices=["mw", "reference"])
    p.add_argument("--orbitals", type=int, default=32)
    p.add_argument("--order", type=int, default=9)
    p.add_argument("--prec", type=float, default=1e-6)
    p.add_argument("--cpu-sample-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--tau", type=float, default=0.99, help="proposal threshold of the learned apply")
    p.add_argument("--mixed-engine", default="bf16x3", choices=["bf16x3", "fp32"],
                   help="contraction of the mixed path: BF16x3 (x step on the tensor cores) or FP32 CUDA cores")
    p.add_argument("--tf32x3", action="store_true", help="also time the split-TF32 tensor-core engine")
    p.add_argument("--shard", action="store_true",
                   help="N > 1: split one batch over the ranks by input node count (strong scaling) "
                        "instead of one batch per rank (weak scaling)")
    p.add_argument("--reserve-gib", type=int, default=None,
                   help="device memory pool reserved up front (GiB): the working set of the step (default 64; "
                        "150 for the exchange workload, whose 136 product and potential trees per leg need "
                        "more: a pool that has to grow inside the timed region made its steps vary 0.8-2.9 s)")
    p.add_argument("--workload", default="helmholtz", choices=["helmholtz", "exchange", "density_sweep"],
                   help="helmholtz: 32-orbital Helmholtz batch (the headline); exchange: 16 orbitals -> 136 "
                        "pair products, each followed by a Poisson apply; density_sweep: Poisson potential of "
                        "a 20-atom density at orders 7/9/11 x prec 1e-5/1e-6/1e-7, FP64 and mixed")
    a = p.parse_args()
    if a.reserve_gib is None:
        a.reserve_gib = 150 if a.workload == "exchange" else 64
    return a


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "_fallback": True}


class Clocks:
    """nvidia-smi sampling (every 50 ms) during the timed region."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.marks = []

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def mark(self):
        """record the wall time of a boundary of the timed region (samples outside are dropped)"""
        self.marks.append(time.time())

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        """median SM clock, max clock and throttle reasons of the samples inside the timed region
        (all samples when the region was shorter than the sampling period)"""
        import datetime

        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 10:
                try:
                    parts[0] = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    parts[0] = None
                rows.append(parts)
        os.unlink(self.f.name)
        if len(self.marks) >= 2:
            inside = [r for r in rows if r[0] is not None and self.marks[0] <= r[0] <= self.marks[-1]]
            if inside:
                rows = inside
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_env():
    from mrchem_b200.replicas import dist_env as de

    return de()


def workload(rank, n, seed=2):
    """Config-2 orbitals and Helmholtz mu for a rank (weak scaling: every rank its own batch)."""
    from mrchem_b200 import workloads as W

    from mrchem_b200.replicas import rank_seed

    return W.orbitals(n, seed=rank_seed(seed, rank)), W.helmholtz_mus(n, seed=rank_seed(seed, rank))


def flops_per_triple(k):
    return 6 * (2 * k) ** 4


# ----------------------------------------------------------------------------------------------
# reference arm: the CPU restatement (MRCPP itself cannot be built here), all host threads
# ----------------------------------------------------------------------------------------------
def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from mrchem_b200 import workloads as W
    from oracle import oracle as O

    orbs, mus = workload(0, args.orbitals)
    m = O.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], args.order, 15)
    # the whole batch of the GPU arm, taken in groups of a quarter of it: consecutive steps rotate over
    # the groups, so that every four steps apply every orbital once
    n = args.orbitals
    group = max(1, (n + 3) // 4)
    trees, ops = [], []
    for i in range(n):
        t = O.FunctionTree(m)
        O.project(args.prec, t, orbs[i])
        trees.append(t)
        ops.append(O.HelmholtzOperator(m, mus[i], args.prec))
    outs = [O.FunctionTree(m) for _ in range(n)]

    def step(s):
        b = (s * group) % n
        idx = [(b + q) % n for q in range(group)]
        for i in idx:
            O.apply(args.prec, outs[i], ops[i], trees[i])
        return len(idx)

    for i in range(n):  # operator tables are built on first use: build them all untimed
        O.apply(args.prec, outs[i], ops[i], trees[i])
    for s in range(args.warmup):
        step(s)
    applies = 0
    t0 = time.perf_counter()
    for s in range(args.steps):
        applies += step(args.warmup + s)
    dt = time.perf_counter() - t0
    cores = O.lib().oracle_num_threads()
    val = applies / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "applies/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "helmholtz_batch_32orb_k10_prec1e-6", "orbitals": args.orbitals,
                   "order": args.order, "prec": args.prec,
                   "step": f"{group} orbital applies (a quarter of the batch, rotating over the whole batch)"},
        "cpu_baseline": {"value": val, "unit": "applies/s", "cores": cores, "kind": "port",
                         "sample": f"{applies} Helmholtz applies of the {n}-orbital batch ({args.steps} steps of "
                                   f"{group}); FP64 CPU restatement (OpenMP), not MRCPP (not buildable here)"},
        "e2e": {"value": val, "unit": "applies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------------------------
def run_gpu(args):
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from mrchem_b200 import mrcpp as G
    from mrchem_b200 import workloads as W
    from mrchem_b200.replicas import max_over_ranks

    stream = torch.cuda.Stream()
    ctx = G.Context(local, stream=stream.cuda_stream)
    ctx.reserve(args.reserve_gib << 30)  # the whole working set, so that no timed step grows the pool
    m = G.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], args.order, 15,
                                  ctx=ctx)
    shard = args.shard and world > 1
    orbs, mus = workload(0 if shard else rank, args.orbitals)
    inps, ops, outs = [], [], []
    for i in range(args.orbitals):
        t = G.FunctionTree(m)
        G.project(args.prec, t, orbs[i])
        inps.append(t)
        ops.append(G.HelmholtzOperator(m, mus[i], args.prec))
        outs.append(G.FunctionTree(m))
    shard_range = (0, args.orbitals)
    if shard:  # this rank's contiguous range of the one batch, balanced by input node count
        from mrchem_b200.replicas import shard_ranges

        shard_range = shard_ranges([t.nnodes() for t in inps], world)[rank]
        b_, e_ = shard_range
        inps, ops, outs, orbs, mus = inps[b_:e_], ops[b_:e_], outs[b_:e_], orbs[b_:e_], mus[b_:e_]
    nloc = len(inps)
    # applies of the whole job per step: the one batch (strong) or one batch per rank (weak)
    job_applies = args.orbitals if shard else args.orbitals * world
    in_bytes = sum(t.nnodes() for t in inps) * (2 * m.k) ** 3 * 8

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    step_ms = []  # per timed region: device time of each step

    def timed(run, name):
        """W untimed + K timed steps of `run()` (returns the step's contracted triples).  The clock
        sampler starts before the warm-up steps, so that its start-up (NVML initialisation) is over
        when the timed region begins.  The timed steps sit in an NVTX range `name` (a no-op unless a
        profiler listens; `ncu --nvtx --nvtx-include name/` lists the launches of that region only)."""
        with Clocks(local) as clk:
            for _ in range(args.warmup):
                run()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
            gc.collect()  # no collector pass (tree destructors synchronise the stream) inside the region
            gc.disable()
            barrier()
            torch.cuda.synchronize()
            clk.mark()
            ctx.profile(True)
            trip = 0
            ev0.record(stream)
            evs[0].record(stream)
            torch.cuda.nvtx.range_push(name)
            for q in range(args.steps):
                trip += run()
                evs[q + 1].record(stream)
            torch.cuda.nvtx.range_pop()
            ev1.record(stream)
            torch.cuda.synchronize()
            clk.mark()
            gc.enable()
        step_ms.append([evs[q].elapsed_time(evs[q + 1]) for q in range(args.steps)])
        barrier()
        ms_ = ev0.elapsed_time(ev1)
        prof = ctx.profile_read() + (ctx.profile_ctas(),)
        ctx.profile(False)
        ms_ = max_over_ranks(ms_, device=f"cuda:{local}")
        return ms_, trip, prof, clk.summary()

    # learned tree proposal: trained (untimed) on plain applies of a disjoint seeded orbital set
    t_train = time.perf_counter()
    net = G.ProposalNet(ctx=ctx, hidden_layers=3, width=128, seed=5)
    tr_orbs, tr_mus = workload(0 if shard else rank, max(nloc, 1), seed=1000 + 7)
    tr_in = []
    for f in tr_orbs:
        t = G.FunctionTree(m)
        G.project(args.prec, t, f)
        tr_in.append(t)
    tr_ops = [G.HelmholtzOperator(m, mu, args.prec) for mu in tr_mus]
    tr_out = [G.FunctionTree(m) for _ in tr_in]
    G.apply_batched(args.prec, tr_out, tr_ops, tr_in)
    for o, op, t in zip(tr_out, tr_ops, tr_in):
        net.collect(o, op, t)
    n_train, n_pos = net.dataset()
    train_loss = net.train(epochs=40, batch=4096, lr=2e-3, seed=0)
    del tr_in, tr_out, tr_ops
    t_train = time.perf_counter() - t_train

    # contraction work split per engine, tuned (untimed) on this batch: every engine gets the same
    # treatment (mrchem_b200.autotune)
    from mrchem_b200.autotune import tune_chunk_triples

    MIXED = G.APPLY_BF16X3 if args.mixed_engine == "bf16x3" else G.APPLY_FP32
    tuning = {}
    engines = [("fp64", G.APPLY_FP64), ("fp32", G.APPLY_FP32), ("bf16x3", G.APPLY_BF16X3)]
    if args.tf32x3:
        engines.append(("tf32x3", G.APPLY_TF32X3))
    for name, fl in engines:
        tune_out = [G.FunctionTree(m) for _ in range(nloc)]

        def tune_run(fl=fl, tune_out=tune_out):
            G.apply_batched(args.prec, tune_out, ops, inps, fl)

        tuning[name] = tune_chunk_triples(ctx, tune_run, fl, reps=2, warmup=1)
        del tune_out

    # plain FP64 (the reference method on the GPU), the mixed path (BF16x3 tensor-core x step, FP32 y
    # and z steps, FP64 accumulation; or the FP32 CUDA-core engine), and mixed + learned proposal, same
    # inputs, same operators
    ms64, trip64, prof64, _ = timed(lambda: G.apply_batched(args.prec, outs, ops, inps, G.APPLY_FP64), "plain_fp64")
    outs32 = [G.FunctionTree(m) for _ in range(nloc)]
    ms32, trip32, prof32m, _ = timed(lambda: G.apply_batched(args.prec, outs32, ops, inps, MIXED), "mixed")
    outsS = [G.FunctionTree(m) for _ in range(nloc)]
    other = G.APPLY_FP32 if MIXED == G.APPLY_BF16X3 else G.APPLY_BF16X3
    msS, tripS, profS, _ = timed(lambda: G.apply_batched(args.prec, outsS, ops, inps, other), "mixed_other_engine")
    errS = [G.distance(a, b) / np.sqrt(b.square_norm()) for a, b in zip(outsS, outs)]
    outsL = [G.FunctionTree(m) for _ in range(nloc)]
    lstats = {}

    def run_learned():
        st = G.apply_learned(args.prec, outsL, ops, inps, net, tau=args.tau, flags=MIXED)
        lstats.update(st)
        return st["triples"]

    ms, triples, prof32, clocks = timed(run_learned, "mixed_learned")
    launches, apply_launches, apply_ms, apply_ctas = prof32
    if args.tf32x3:  # the split-TF32 tensor-core contraction on the same batch, no learned proposal
        outsT = [G.FunctionTree(m) for _ in range(nloc)]
        msT, tripT, profT, _ = timed(lambda: G.apply_batched(args.prec, outsT, ops, inps, G.APPLY_TF32X3), "tensor_core")
        errT = [G.distance(a, b) / np.sqrt(b.square_norm()) for a, b in zip(outsT, outs)]
    # error of the mixed + learned result against the FP64 one: ||g - g64|| / ||g64|| per orbital
    # (from the coefficient differences, mw_tree_distance: no cancellation)
    rel_err = 0.0
    same_tree = True
    for a, b in zip(outsL, outs):
        rel_err = max(rel_err, G.distance(a, b) / np.sqrt(b.square_norm()))
        same_tree &= a.nnodes() == b.nnodes()
    rel_err_mixed = max(G.distance(a, b) / np.sqrt(b.square_norm()) for a, b in zip(outs32, outs))
    total_applies = job_applies * args.steps
    value = total_applies / (ms / 1e3)

    # end to end through the public API from host buffers: every step uploads the input trees from
    # pinned host memory, applies, and downloads the output trees into pinned host memory (buffers
    # allocated once, as a caller that streams batches would)
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    host = []
    for t in inps:
        ex = t.export()
        h = {"depth": pinned(ex["depth"].shape, torch.int32), "trans": pinned(ex["trans"].shape, torch.int64),
             "parent": pinned(ex["parent"].shape, torch.int32), "child0": pinned(ex["child0"].shape, torch.int32),
             "coef": pinned(ex["coef"].shape, torch.float64)}
        for key in h:
            h[key][...] = ex[key]
        host.append(h)
    bs_k = (2 * m.k) ** 3
    out_bufs = []
    for t in outsL:  # outputs of the timed learned steps: the same batch, the same tree sizes
        cap = int(t.nnodes() * 1.25) + 64
        out_bufs.append({"depth": pinned((cap,), torch.int32), "parent": pinned((cap,), torch.int32),
                         "child0": pinned((cap,), torch.int32), "trans": pinned((3 * cap,), torch.int64),
                         "coef": pinned((cap * bs_k,), torch.float64)})
    n_e2e = 32  # a stream of 32 batches: the pipeline's fill and drain (about 1.5 steps) amortised
    h2d = sum(sum(v.nbytes for v in h.values()) for h in host)
    node_bytes = 4 + 24 + 4 + 4 + 8 * bs_k
    nb = nloc

    # Pipeline of three host threads (the library releases the interpreter lock in every call):
    #   upload:   pinned host -> staging input trees of a side context (stream), double-buffered;
    #   compute:  staging inputs -> the compute context's trees (device copy, mw_tree_assign), the
    #             learned apply of the whole batch, outputs -> staging output trees (device copy);
    #   download: staging outputs -> pinned host, on the side contexts of the output buffers.
    # Step i's uploads and step i-1's downloads overlap step i's compute.
    import queue
    import threading

    def side_world():
        # high priority: the transfers' small kernels (hash index, norms) are scheduled ahead of the
        # pending CTAs of the compute stream's long contraction launches
        st = torch.cuda.Stream(priority=-1)
        c = G.Context(local, stream=st.cuda_stream)
        w = G.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], args.order, 15,
                                      ctx=c)
        return st, c, w

    # one side context per staging buffer: a buffer's stream is idle whenever its trees are handed
    # over (mw_tree_assign waits for the source's stream and its own), so the threads never wait on
    # each other's transfers in flight
    ups = [side_world() for _ in range(2)]
    dns = [side_world() for _ in range(2)]
    stage_in = [[G.FunctionTree(ups[q][2]) for _ in range(nb)] for q in range(2)]
    stage_out = [[G.FunctionTree(dns[q][2]) for _ in range(nb)] for q in range(2)]
    c_in = [G.FunctionTree(m) for _ in range(nb)]
    c_out = [G.FunctionTree(m) for _ in range(nb)]

    def upload(q):  # the whole batch in one call: its copies stream back to back
        G.load_many(stage_in[q], host)

    def compute(q):
        for i in range(nb):
            c_in[i].assign(stage_in[q][i])

    def apply_and_stage(q):
        G.apply_learned(args.prec, c_out, ops, c_in, net, tau=args.tau, flags=MIXED)
        for i in range(nb):
            stage_out[q][i].assign(c_out[i])

    def download(q):
        return sum(G.export_many_into(stage_out[q], out_bufs)) * node_bytes

    # untimed pass through every stage (staging trees grow to size)
    for q in (0, 1):
        upload(q)
        compute(q)
        apply_and_stage(q)
        download(q)
    torch.cuda.synchronize()

    free_in = [threading.Semaphore(1) for _ in range(2)]
    free_out = [threading.Semaphore(1) for _ in range(2)]
    ready_in, ready_out = queue.Queue(), queue.Queue()
    errs, d2h_steps = [], []

    def guard(fn):
        def run():
            try:
                fn()
            except Exception as exc:  # reported by the main thread; unblock the others
                errs.append(exc)
                ready_in.put(None)
                ready_out.put(None)
        return run

    def uploader():
        for step_i in range(n_e2e):
            q = step_i % 2
            free_in[q].acquire()
            upload(q)
            ready_in.put(step_i)

    def computer():
        for _ in range(n_e2e):
            step_i = ready_in.get()
            if step_i is None:
                return
            q = step_i % 2
            compute(q)
            free_in[q].release()
            free_out[q].acquire()
            apply_and_stage(q)
            ready_out.put(step_i)

    def downloader():
        for _ in range(n_e2e):
            step_i = ready_out.get()
            if step_i is None:
                return
            q = step_i % 2
            d2h_steps.append(download(q))
            free_out[q].release()

    threads = [threading.Thread(target=guard(f)) for f in (uploader, computer, downloader)]
    barrier()
    torch.cuda.synchronize()
    gc.collect()
    gc.disable()
    t0 = time.perf_counter()
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    gc.enable()
    if errs:
        raise errs[0]
    d2h = d2h_steps[-1]
    # the e2e outputs equal the headline outputs (same inputs, same network)
    e2e_same = True
    for i in range(nb):
        ex = outsL[i].export()
        nn = c_out[i].nnodes()
        e2e_same &= nn == outsL[i].nnodes() and np.array_equal(out_bufs[i]["depth"][:nn], ex["depth"]) and \
            np.array_equal(out_bufs[i]["coef"][:nn * bs_k], ex["coef"].ravel())
    e2e_s = max_over_ranks(e2e_s, device=f"cuda:{local}")
    e2e_val = job_applies * n_e2e / e2e_s

    peaks = measured_peaks()
    k = m.k
    flops = triples * flops_per_triple(k)
    achieved = flops / (apply_ms / 1e3) / 1e12 if apply_ms > 0 else None
    peak = float(peaks.get("bf16_tflops", 1590.0))
    # DRAM traffic per contraction launch: bytes per CTA measured by ncu on a 4-orbital batch
    # (profiles/k_happly_k10_traffic.json or k_gapply_fp32_k10_traffic.json) times this step's CTAs per launch
    traffic = None
    kernel_name = f"k_happly<{k}>" if MIXED == G.APPLY_BF16X3 else f"k_gapply<{k},float>"
    prof_file = os.path.join(ROOT, "profiles", "k_happly_k10_traffic.json" if MIXED == G.APPLY_BF16X3
                             else "k_gapply_fp32_k10_traffic.json")
    if os.path.exists(prof_file) and k == 10 and apply_launches > 0:
        try:
            traffic = json.load(open(prof_file))["dram_bytes_per_cta"] * apply_ctas / apply_launches
        except Exception:
            traffic = None

    cpu, err_oracle = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, oracle_outs = cpu_baseline(args, inps, mus)
        # error of the headline (mixed + learned) results against the FP64 CPU apply of the same inputs
        errs_o = []
        for i, ex in oracle_outs:
            back = G.FunctionTree(m)
            back.load(ex["depth"], ex["trans"], ex["parent"], ex["child0"], ex["coef"])
            same = back.nnodes() == outsL[i].nnodes()
            errs_o.append((G.distance(outsL[i], back) / np.sqrt(back.square_norm()), same))
        err_oracle = {"max": max(e for e, _ in errs_o), "orbitals": len(errs_o),
                      "same_node_count": all(sm for _, sm in errs_o),
                      "definition": "||g - g_oracle|| / ||g_oracle|| per orbital, g = mixed + learned result, "
                                    "g_oracle = the FP64 CPU restatement's apply of the same input tree"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "applies/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if shard else "weak",
            "vs_baseline": None, "data": "synthetic",
            "dtype": ("bf16x3 fixed-point slices (x step, tensor cores) / f32 (y, z steps), f64 accumulation"
                      if MIXED == G.APPLY_BF16X3 else "f32 products, f64 accumulation"),
            "config": {"workload": "helmholtz_batch_32orb_k10_prec1e-6", "orbitals": args.orbitals,
                       "order": args.order, "k": k, "prec": args.prec, "mu": "U[0.5,3]", "world": "[-20,20]^3",
                       "path": f"mixed ({args.mixed_engine} contraction, FP64 accumulation) + learned tree proposal; batched",
                       "parallelism": (f"one batch sharded over {world} ranks by input node count "
                                       f"(this rank: trees {shard_range[0]}..{shard_range[1] - 1})") if shard
                       else f"replicas x{world}",
                       "l2": f"inputs larger than L2 ({in_bytes / 1e9:.2f} GB of input blocks per step)"},
            "e2e": {"value": e2e_val, "unit": "applies/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "host_memory": "pinned, allocated once",
                    "path": "per step: mw_tree_upload_many of the 32 trees (upload thread, own context), "
                            "mw_tree_assign x32 (device copy into the compute context), mw_apply_learned, "
                            "mw_tree_assign x32 (device copy out), mw_tree_download_many of the 32 trees (download "
                            "thread, own context); double-buffered staging trees, so a step's transfers overlap "
                            "the previous and next steps' compute",
                    "steps": n_e2e,
                    "outputs_equal_headline": bool(e2e_same)},
            "plain_fp64": {"value": job_applies * args.steps / (ms64 / 1e3), "unit": "applies/s",
                           "ms_per_step": ms64 / args.steps, "kernel_ms_per_step": prof64[2] / args.steps,
                           "triples_per_step": trip64 // max(1, args.steps)},
            "mixed_no_learning": {"engine": args.mixed_engine,
                                  "value": job_applies * args.steps / (ms32 / 1e3), "unit": "applies/s",
                                  "ms_per_step": ms32 / args.steps, "kernel_ms_per_step": prof32m[2] / args.steps},
            "mixed_other_engine": {"engine": "fp32" if MIXED == G.APPLY_BF16X3 else "bf16x3",
                                   "value": job_applies * args.steps / (msS / 1e3), "unit": "applies/s",
                                   "ms_per_step": msS / args.steps, "kernel_ms_per_step": profS[2] / args.steps,
                                   "rel_error_vs_fp64_max": max(errS),
                                   "same_node_count_as_fp64": all(a.nnodes() == b.nnodes() for a, b in zip(outsS, outs))},
            "step_ms": {"plain_fp64": step_ms[0], "mixed_no_learning": step_ms[1], "mixed_other_engine": step_ms[2],
                        "mixed_learned": step_ms[3]},
            "speedup_vs_plain_fp64": ms64 / ms,
            "rel_error_vs_fp64": rel_err,
            "rel_error_vs_oracle": err_oracle,
            "rel_error_vs_fp64_mixed_no_learning": rel_err_mixed,
            "rel_error_definition": "max over orbitals of ||g - g_fp64|| / ||g_fp64|| (coefficient differences)",
            "same_node_count_as_fp64": bool(same_tree),
            "learned": {"passes": lstats.get("passes"), "proposed": lstats.get("proposed"),
                        "pruned": lstats.get("pruned"), "missed": lstats.get("missed"),
                        "out_nodes": lstats.get("out_nodes"), "train_rows": n_train, "train_positive": n_pos,
                        "train_loss": train_loss, "train_s": t_train, "tau": args.tau,
                        "train_data": "plain applies of 32 other seeded orbitals (seed 1007)"},
            "roofline": {"bound": "tensor", "kernel": kernel_name, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if not peaks.get("_fallback")
                         else "fallback", "fp32_simt_peak_nominal": FP32_PEAK_NOMINAL,
                         "frac_fp32_simt_nominal": (achieved / FP32_PEAK_NOMINAL) if achieved else None,
                         "flops_per_triple": flops_per_triple(k), "triples_per_step": triples // max(1, args.steps),
                         "kernel_ms_per_step": apply_ms / args.steps, "kernel_launches": apply_launches,
                         "traffic_unit": "DRAM bytes per launch (ncu bytes per CTA x CTAs per launch)",
                         "block_write_bytes_per_launch": apply_ctas * (2 * k) ** 3 * 8 / max(1, apply_launches)},
            "cpu_baseline": cpu,
            "autotune": {k: {"chunk_triples": v["best"], "ms_per_candidate": v["ms"]} for k, v in tuning.items()},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if args.tf32x3:
            line["tensor_core_tf32x3"] = {
                "value": job_applies * args.steps / (msT / 1e3), "unit": "applies/s",
                "ms_per_step": msT / args.steps, "kernel": f"k_tapply<{m.k}>", "kernel_ms_per_step": profT[2] / args.steps,
                "rel_error_vs_fp64_max": max(errT), "rel_error_vs_fp64_median": float(np.median(errT)),
                "same_node_count_as_fp64": all(a.nnodes() == b.nnodes() for a, b in zip(outsT, outs))}
            line["step_ms"]["tensor_core_tf32x3"] = step_ms[4]
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def cpu_baseline(args, inps, mus):
    """Oracle (FP64 CPU restatement, OpenMP, all host threads) on a bounded sample of the batch."""
    from mrchem_b200 import workloads as W
    from oracle import oracle as O

    m = O.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], args.order, 15)
    done, t_used = 0, 0.0
    outs_o = []
    while done < len(inps) and t_used < args.cpu_sample_seconds:
        ex = inps[done].export()
        ti = O.FunctionTree(m)
        ti.load(ex["depth"], ex["trans"], ex["parent"], ex["child0"], ex["coef"])
        op = O.HelmholtzOperator(m, mus[done], args.prec)
        to = O.FunctionTree(m)
        O.apply(args.prec, to, op, ti)  # operator tables build lazily: warm them first
        t0 = time.perf_counter()
        O.apply(args.prec, to, op, ti)
        t_used += time.perf_counter() - t0
        outs_o.append((done, to.export()))
        done += 1
    return {"value": done / t_used, "unit": "applies/s", "cores": O.lib().oracle_num_threads(), "kind": "port",
            "sample": f"first {done} orbitals of the batch, one Helmholtz apply each ({t_used:.1f} s); "
                      "FP64 CPU restatement (OpenMP), not MRCPP"}, outs_o


def run_exchange(args):
    """Exchange pair batch: 16 orbitals (the Helmholtz batch's orbital model), the 136 pair products
    phi_i phi_j (i <= j, adaptive multiply as at ExchangePotential.cpp:253,312), each followed by a
    Poisson apply (ExchangePotential.cpp:137).  One step = all 136 products and applies; FP64, mixed and
    split-TF32 tensor-core applies (the products are FP64 in all); error per pair of the mixed and
    tensor-core potentials against FP64."""
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    from mrchem_b200 import mrcpp as G
    from mrchem_b200 import workloads as W
    from mrchem_b200.replicas import rank_seed

    stream = torch.cuda.Stream()
    ctx = G.Context(local, stream=stream.cuda_stream)
    ctx.reserve(args.reserve_gib << 30)
    m = G.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], args.order, 15, ctx=ctx)
    norb = 16
    phis = []
    for f in W.orbitals(norb, seed=rank_seed(2, rank)):
        t = G.FunctionTree(m)
        G.project(args.prec, t, f)
        phis.append(t)
    pairs = [(i, j) for i in range(norb) for j in range(i, norb)]
    P = G.PoissonOperator(m, args.prec)

    # trees allocated once and reused every step, as a caller iterating the exchange would: products are
    # emptied before each multiply (a non-empty output would be its starting grid), potentials restart
    # from their roots in the apply
    prods = [G.FunctionTree(m) for _ in pairs]
    half = (len(pairs) + 1) // 2

    def step(flags, outs):
        for p in prods:
            G.clear(p)
        G.multiply_batched(args.prec, prods, None, [phis[i] for i, _ in pairs], [phis[j] for _, j in pairs])
        for a in range(0, len(pairs), half):
            G.apply_batched(args.prec, outs[a:a + half], [P] * len(outs[a:a + half]), prods[a:a + half], flags)
        return prods, outs

    res = {}
    legs = [("fp64", G.APPLY_FP64), ("mixed", G.APPLY_FP32), ("bf16x3", G.APPLY_BF16X3)]
    if args.tf32x3:
        legs.append(("tf32x3", G.APPLY_TF32X3))
    ref_outs = None
    clk = Clocks(local)
    clk.__enter__()
    for name, flags in legs:
        leg_outs = [G.FunctionTree(m) for _ in pairs]
        for _ in range(args.warmup):
            step(flags, leg_outs)
        torch.cuda.synchronize()
        ctx.profile(True)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk.mark()
        ev0.record(stream)
        for _ in range(args.steps):
            prods, outs = step(flags, leg_outs)
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.mark()
        ms = ev0.elapsed_time(ev1) / args.steps
        launches, apply_launches, apply_ms = ctx.profile_read()
        ctx.profile(False)
        res[name] = {"ms_per_step": ms, "pairs_per_s": len(pairs) / (ms / 1e3),
                     "apply_kernel_ms_per_step": apply_ms / args.steps,
                     "product_nodes": sum(p.nnodes() for p in prods), "potential_nodes": sum(o.nnodes() for o in outs)}
        if ref_outs is None:
            ref_outs = outs
        else:  # errors against the FP64 potentials now, then this leg's trees are released (device memory)
            errs = [G.distance(a, b) / np.sqrt(b.square_norm()) for a, b in zip(outs, ref_outs)]
            res[name]["rel_error_per_pair"] = {"max": max(errs), "median": float(np.median(errs)), "min": min(errs)}
            res[name]["same_node_count_as_fp64"] = all(a.nnodes() == b.nnodes() for a, b in zip(outs, ref_outs))
            del outs, leg_outs
            gc.collect()
    clk.__exit__(None, None, None)
    if rank == 0:
        line = {"metric": "exchange pair batch: 136 pair products + Poisson applies", "workload": "exchange_16orb_136pairs_k10_prec1e-6",
                "value": res["bf16x3"]["pairs_per_s"], "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "order": args.order, "prec": args.prec, "data": "synthetic",
                "fp64": res["fp64"], "mixed_fp32": res["mixed"], "bf16x3": res["bf16x3"],
                "rel_error_per_pair_fp32": res["mixed"]["rel_error_per_pair"],
                "same_node_count_as_fp64_fp32": bool(res["mixed"]["same_node_count_as_fp64"]),
                "rel_error_per_pair_bf16x3": res["bf16x3"]["rel_error_per_pair"],
                "same_node_count_as_fp64_bf16x3": bool(res["bf16x3"]["same_node_count_as_fp64"]),
                "clocks": clk.summary()}
        if args.tf32x3:
            line["tf32x3"] = res["tf32x3"]
            line["rel_error_per_pair_tf32x3"] = res["tf32x3"]["rel_error_per_pair"]
        print(json.dumps(line), flush=True)


def run_density_sweep(args):
    """Poisson potential of a 20-atom density (4 normalised Gaussians per atom, exponents
    log-U[0.3, 1e3], atoms in a 12 Bohr box) at interpolating orders 7/9/11 and precisions
    1e-5/1e-6/1e-7: FP64, mixed (FP32 products, FP64 accumulation) and BF16x3 tensor-core applies (with
    --tf32x3 also split-TF32) on the GPU, each timed over --steps steps after --warmup, with the relative
    errors of the mixed and tensor-core potentials against FP64 (coefficient differences) and the CPU
    restatement's time for one apply at order 7, prec 1e-5.  (At order 11, k = 12, the BF16x3 flag runs
    the FP32 engine.)"""
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    from mrchem_b200 import mrcpp as G
    from mrchem_b200 import workloads as W

    stream = torch.cuda.Stream()
    ctx = G.Context(local, stream=stream.cuda_stream)
    ctx.reserve(args.reserve_gib << 30)
    rho_f = W.density_20_atoms()
    rows = []
    clk = Clocks(local)
    clk.__enter__()
    clk.mark()
    for order in (7, 9, 11):
        m = G.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], order, 15, ctx=ctx)
        for prec in (1e-5, 1e-6, 1e-7):
            rho = G.FunctionTree(m)
            G.project(prec, rho, rho_f)
            P = G.PoissonOperator(m, prec)
            row = {"order": order, "k": order + 1, "prec": prec, "input_nodes": rho.nnodes()}
            outs = {}
            legs = [("fp64", G.APPLY_FP64), ("mixed", G.APPLY_FP32), ("bf16x3", G.APPLY_BF16X3)]
            if args.tf32x3:
                legs.append(("tf32x3", G.APPLY_TF32X3))
            for name, fl in legs:
                out = G.FunctionTree(m)
                for _ in range(args.warmup):
                    G.apply(prec, out, P, rho, fl)
                torch.cuda.synchronize()
                ctx.profile(True)
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                for _ in range(args.steps):
                    st = G.apply(prec, out, P, rho, fl)
                ev1.record(stream)
                torch.cuda.synchronize()
                kms = ctx.profile_read()[2] / args.steps
                ctx.profile(False)
                row[name] = {"ms": ev0.elapsed_time(ev1) / args.steps, "kernel_ms": kms, "triples": st[0],
                             "out_nodes": out.nnodes(),
                             "tflops": st[0] * flops_per_triple(order + 1) / (kms / 1e3) / 1e12 if kms > 0 else None}
                outs[name] = out
            for name in [n for n, _ in legs if n != "fp64"]:
                row["rel_error_" + name] = G.distance(outs[name], outs["fp64"]) / np.sqrt(outs["fp64"].square_norm())
                row["same_nodes_" + name] = outs[name].nnodes() == outs["fp64"].nnodes()
                row["speedup_" + name] = row["fp64"]["ms"] / row[name]["ms"]
            rows.append(row)
            print(json.dumps(row), file=sys.stderr, flush=True)
    clk.mark()
    clk.__exit__(None, None, None)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O  # the CPU baseline (the FP64 restatement)

        mo = O.MultiResolutionAnalysis(W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"], 7, 15)
        ro = O.FunctionTree(mo)
        O.project(1e-5, ro, rho_f)
        Po = O.PoissonOperator(mo, 1e-5)
        vo = O.FunctionTree(mo)
        O.apply(1e-5, vo, Po, ro)  # operator tables are built on first use
        t0 = time.perf_counter()
        O.apply(1e-5, vo, Po, ro)
        cpu = {"order": 7, "prec": 1e-5, "s_per_apply": time.perf_counter() - t0,
               "cores": O.lib().oracle_num_threads(), "kind": "port"}
    if rank == 0:
        print(json.dumps({"metric": "Poisson apply of a 20-atom density: orders x precisions, FP64, mixed FP32, BF16x3",
                          "workload": "density_20_atoms_sweep", "data": "synthetic", "steps": args.steps,
                          "warmup": args.warmup, "rows": rows, "cpu_baseline": cpu,
                          "clocks": clk.summary()}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "exchange":
        run_exchange(args)
    elif args.workload == "density_sweep":
        run_density_sweep(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
