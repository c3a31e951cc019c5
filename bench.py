#!/usr/bin/env python
"""Benchmark: SparsePauliVector propagation throughput (terms/s, rotate+merge+clip).

Workload (default): the 8x8-lattice circuit (N=64): observable mean Z (64 terms,
coefficient 1/64), 20 Trotter layers of RZZ(0.3) on the 112 edges (rows, then
columns) followed by RX(0.25) on all 64 sites, a depolarizing channel p=1e-3
after each layer, CompositeTruncation(CoeffTruncation(1e-5), WeightTruncation(12))
at window 1.  One step = the whole 3,520-rotation evolution from the observable
plus <0...0|O|0...0>.  terms/s = sum over rotations of the live terms entering
the rotation, divided by the step time.

Arms:
  --impl ours       (default) libpauliprop on the GPU.  `value`: device time of K
                    steps (CUDA events on the engine's stream, input resident in
                    HBM).  `e2e`: the same steps through the public API with host
                    buffers (pinned upload, evolve, download of the final term
                    set and the expectation value) timed by the host clock.
  --impl reference  the reference algorithm on the host cores: the C restatement
                    of the reference's CPU path (oracle/, "port").  Each step is
                    one whole-circuit run from the observable; the K steps run
                    in min(K, host threads) concurrent single-threaded worker
                    processes, and `value` is their aggregate terms/s.  The
                    workers never load libpauliprop.so.
The GPU arm also runs the whole circuit once on the oracle (1 thread, in a
spawned process while the GPU is timed): that is its `cpu_baseline`, and the
GPU's final term set and expectation value are checked against it
(`final_check`).
--workload batch256: 256 uneven instances of the 8x8 lattice in one batched pass
(pp_evolve_batch): depth U{4..24} layers, θ_J, θ_h ~ U[0.05, 0.5], observable a
random Pauli string of weight 1-4, CoeffTruncation(1e-4), no noise.  One step =
all 256 instances; the line adds the p50 / p99 instance completion times.
--workload learned: the learned-truncation protocol on the 8x8-lattice circuit
(20 layers, depolarizing 1e-3, weight cap 12): the network is trained on labels
the engine generates (sampled terms propagated alone through the remaining
layers to relative precision 1e-3), then on held-out angle draws the GPU time
to reach |<O> - <O>_ref| <=
1e-3 is measured for budget truncation by the network and for plain threshold
truncation; the reference run is plain threshold 1e-6 (1e-7 exceeds 2^31 live
terms on this circuit).  value = median learned time (lower is better).
Multi-GPU (torchrun, N > 1): every rank runs an independent replica of the
workload (the path does not shard at this size); value = all ranks' terms over
the slowest rank's time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "paulioperators.jl_b200"))

BYTES_PER_TERM = {1: 24, 2: 40}     # B = 2*(W/8) + 8
# DRAM traffic of k_merge<1,0> per algorithmic byte, from one ncu capture of the 176
# merge launches of layer 11 of this workload (dram__bytes_read.sum +
# dram__bytes_write.sum = 115.1 MB per launch against B(n + a + m) = 150.9 MB:
# the gathered sin branches re-read live terms that are still in L2)
MERGE_TRAFFIC_PER_ALG_BYTE = 115.09 / 150.88
# DRAM traffic of k_bk_rotate<1,512,4> per algorithmic byte, from one ncu capture of
# three launches of this workload at n = 1.90e6 live terms: (dram__bytes_read.sum +
# dram__bytes_write.sum) = 60.6 MB per launch against B(n_in + n_out) = 91.0 MB (part
# of a launch's writes is still in L2 when it ends and is written back later)
BUCKET_TRAFFIC_PER_ALG_BYTE = 60.58 / 91.02


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["lattice64", "chain20", "graph127", "batch256", "learned"],
                    default="lattice64")
    ap.add_argument("--learned-scale", choices=["full", "small"], default="full",
                    help="learned: 'small' is a quick run of the same protocol on fewer draws and samples")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="config 2 only (skip the 127-qubit graph circuit's secondary record)")
    ap.add_argument("--ref-workers", type=int, default=0, help="reference arm worker processes (0: all host threads)")
    return ap.parse_args()


def workload(name):
    from pauliprop import circuits
    return {"lattice64": circuits.lattice64, "chain20": circuits.chain20,
            "graph127": circuits.random_graph127}[name]()


def strategy_of(w):
    import pauliprop as pp
    parts = [pp.CoeffTruncation(w.thresh)]
    if w.wmax:
        parts.append(pp.WeightTruncation(w.wmax))
    return pp.CompositeTruncation(*parts)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
            sm = [float(r[1]) for r in rows]
            mx = max(float(r[2]) for r in rows)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def dist_init(backend):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def reduce_max(x, ws, device=None):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x, ws, device=None):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ----------------------------------------------------------------------------- CPU legs
# The CPU legs run the C restatement of the reference path (oracle/liborc.so) in
# processes that import only the library-free host modules of pauliprop
# (circuits, truncation, paulis): libpauliprop.so is never mapped into them.
def _native_libs_loaded():
    """Shared objects of this repository mapped into the calling process."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                p = line.split()[-1] if line.strip() else ""
                if p.endswith(".so") and p.startswith(ROOT):
                    out.add(os.path.relpath(p, ROOT))
    except OSError:
        pass
    return sorted(out)


def _oracle_whole_circuit(wname, layers=None, out_path=None):
    """The whole circuit of a workload on the CPU oracle, from the observable, one
    evolve! call per Trotter layer followed by the layer's channel (the
    reference's usage: spv_evolve.jl:312-387, channels.jl:223-243).
    Returns dict(terms_in, seconds, expect, n, libs); with out_path the final term
    set is saved there (npz: z, x, c)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import orc
    from pauliprop import circuits
    from pauliprop.truncation import CoeffTruncation, CompositeTruncation, WeightTruncation, compile_filter
    w = {"lattice64": circuits.lattice64, "chain20": circuits.chain20,
         "graph127": circuits.random_graph127}[wname]()
    parts = [CoeffTruncation(w.thresh)] + ([WeightTruncation(w.wmax)] if w.wmax else [])
    f = tuple(compile_filter(CompositeTruncation(*parts)))
    kind = {"depolarizing": 0, "dephasing": 1}[w.channel[0]] if w.channel else None
    gens = [(p.z, p.x) for p in w.layer]
    v = orc.OracleSPV.from_terms(w.N, w.observable)
    terms, dt = 0, 0.0
    for _ in range(w.layers if layers is None else layers):
        n0 = len(v)
        t0 = time.perf_counter()
        _, ctr = v.evolve(gens, w.angles, window=1, strict=f, nwin=len(gens))
        if kind is not None:
            v.channel(kind, [w.channel[1]])
        dt += time.perf_counter() - t0
        # terms entering each rotation: n0, then the live count after each merge
        terms += n0 + int(ctr[2][:-1].sum())
    res = {"terms_in": terms, "seconds": dt, "expect": v.expect(0), "n": len(v), "libs": _native_libs_loaded()}
    if out_path:
        z, x, c = v.arrays()
        np.savez(out_path, z=z, x=x, c=c)
    return res


def _oracle_worker(wname, n_warm, n_runs, barrier, q):
    """Reference-arm worker: n_warm warm-up runs of the circuit's first two layers,
    then (after all workers reach the barrier) n_runs whole-circuit runs."""
    for _ in range(n_warm):
        _oracle_whole_circuit(wname, layers=2)
    barrier.wait()
    q.put([_oracle_whole_circuit(wname) for _ in range(n_runs)])


def _oracle_background(wname, out_path, q):
    """One whole-circuit oracle run for the GPU arm's CPU baseline and final check."""
    q.put(_oracle_whole_circuit(wname, out_path=out_path))


def workload_label(w):
    return (f"{w.name}: N={w.N}, {w.layers} layers x {len(w.layer)} rotations, "
            f"thresh {w.thresh}, wmax {w.wmax}, channel {w.channel}")


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    ws, rank, local = dist_init("gloo")
    if rank != 0:
        return
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    nthreads = args.ref_workers or os.cpu_count() or 1
    q = ctx.Queue()
    if args.workload == "batch256":
        return run_reference_batch(args, ctx, q, nthreads)
    if args.workload == "learned":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned truncation "
                          "(its plain threshold path is the plain arm of this workload)"}), flush=True)
        return
    # the K timed whole-circuit runs are dealt round-robin to P single-threaded
    # worker processes that run concurrently (the reference path is serial:
    # spv_kernels.jl:3-5); the W warm-up steps are short runs of the first two layers
    P = max(1, min(nthreads, args.steps))
    runs = [args.steps // P + (1 if k < args.steps % P else 0) for k in range(P)]
    warm = [args.warmup // P + (1 if k < args.warmup % P else 0) for k in range(P)]
    barrier = ctx.Barrier(P)
    procs = [ctx.Process(target=_oracle_worker, args=(args.workload, warm[k], runs[k], barrier, q))
             for k in range(P)]
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    # aggregate throughput of the concurrently running workers: the sum over
    # workers of (term-rotations they processed / seconds they spent)
    value = sum(sum(r["terms_in"] for r in rs) / sum(r["seconds"] for r in rs) for rs in res)
    flat = [r for rs in res for r in rs]
    per_run = statistics.median(r["terms_in"] / r["seconds"] for r in flat)
    libs = sorted({lib for r in flat for lib in r["libs"]})
    from pauliprop import circuits
    w = {"lattice64": circuits.lattice64, "chain20": circuits.chain20,
         "graph127": circuits.random_graph127}[args.workload]()
    line = {
        "metric": "terms/s rotate+merge+clip", "value": value, "unit": "terms/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.median(r["seconds"] for r in flat), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded circuit)", "impl": "reference",
        "config": {"workload": workload_label(w), "N": w.N, "threads": P,
                   "value_is": f"aggregate of {P} concurrent single-threaded runs (sum of per-worker terms/s)",
                   "per_run_single_thread_terms_per_s": per_run,
                   "runs_per_worker": runs, "step": "one whole-circuit run from the observable"},
        "expectation": flat[0]["expect"],
        "native_libs_loaded": libs,
        "cpu_baseline": {"value": value, "unit": "terms/s", "cores": P, "kind": "port",
                         "sample": f"{w.name} end to end ({w.layers} layers x {len(w.layer)} rotations + channels "
                                   f"from the observable), {args.steps} runs over {P} concurrent worker processes, "
                                   f"C restatement of the reference path (oracle/liborc.so)"},
        "e2e": {"value": value, "unit": "terms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


BATCH_COUNT, BATCH_SEED, BATCH_THRESH = 256, 5, 1e-4
BATCH_CPU_LIMIT = 2_000_000     # CPU sample: layers entered with at most this many live terms


def batch_setup():
    from pauliprop import circuits
    insts = circuits.batch_instances(count=BATCH_COUNT, seed=BATCH_SEED, thresh=BATCH_THRESH)
    layer = [(p.z, p.x) for p in insts[0].layer]
    acol = [0] * 112 + [1] * 64
    angs = [[w.angles[0], w.angles[-1]] for w in insts]
    depths = [w.layers for w in insts]
    obs = [w.observable for w in insts]
    return insts, layer, acol, angs, depths, obs


def _oracle_batch_sample(worker, nworkers, budget_s, q=None):
    """Worker: the batch's instances worker, worker + nworkers, ... on the CPU oracle,
    one layer at a time, entering a layer only with at most BATCH_CPU_LIMIT live
    terms, until budget_s seconds of evolution.  Returns (terms_in, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    import pauliprop as pp
    insts, layer, acol, angs, depths, obs = batch_setup()
    f = tuple(pp.compile_filter(pp.CoeffTruncation(BATCH_THRESH)))
    terms = 0
    spent = 0.0
    for i in range(worker, len(insts), nworkers):
        v = orc.OracleSPV(64, 16, 1 << 22)
        v.upload([t[0] for t in obs[i]], [t[1] for t in obs[i]], [t[2] for t in obs[i]])
        ang = [angs[i][a] for a in acol]
        for _ in range(depths[i]):
            if len(v) > BATCH_CPU_LIMIT or spent > budget_s:
                break
            n0 = len(v)
            t0 = time.perf_counter()
            _, ctr = v.evolve(layer, ang, window=1, strict=f, nwin=len(layer))
            spent += time.perf_counter() - t0
            terms += n0 + int(ctr[2][:-1].sum())
        if spent > budget_s:
            break
    out = (terms, spent)
    if q is not None:
        q.put(out)
    return out


def run_ours_batch(args):
    import numpy as np
    import torch
    ws, rank, local = dist_init("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import pauliprop as pp
    from pauliprop.batch import tagged_terms

    insts, layer, acol, angs, depths, obs = batch_setup()
    D = max(depths)
    gens = layer * D
    acols = acol * D
    rend = [d * len(layer) for d in depths]
    strat = pp.CoeffTruncation(BATCH_THRESH)
    v = pp.SparsePauliVector(128, 1 << 20, 16)
    stream = torch.cuda.ExternalStream(v.stream(), device=dev)

    def one_step(profile=False):
        return pp.evolve_batch(obs, gens, acols, angs, rend, nq=64, truncation=strat, vector=v, profile=profile)

    for _ in range(args.warmup):
        one_step()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    res = []
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            res.append(one_step())
        e1.record(stream)
        torch.cuda.synchronize()
    t = reduce_max(e0.elapsed_time(e1) * 1e-3, ws, dev)
    terms_in = res[-1].stats["terms_in"]
    total_terms = reduce_sum(terms_in * args.steps, ws, dev)
    value = total_terms / t
    launches = int(res[-1].stats["launches"])
    tdone = np.concatenate([r.t_done for r in res])
    # e2e: the public call from host arrays (upload, evolve, per-instance results back)
    z, x, c = tagged_terms(obs)
    te = []
    for _ in range(args.steps):
        if ws > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        r = one_step()
        te.append(time.perf_counter() - t0)
    t_e2e = reduce_max(sum(te), ws, dev)
    h2d = z.nbytes + x.nbytes + c.nbytes + len(gens) * (32 + 4) + len(obs) * (2 * 2 * 8 + 8)
    d2h = len(obs) * (8 + 8 + 8)
    # profiled pass: merge kernel time for the roofline
    rp = one_step(profile=True)
    sp = rp.stats
    B = BYTES_PER_TERM[2]
    if sp["bucket_rot"] > 0:
        # rotations on buckets: B*(n_in + n_out) per k_bk_rotate launch over the timed
        # graph replays (t_merge also holds any span that ran on the sorted-merge kernels)
        dom_bytes = sp["bucket_bytes"]
        tune = pp.tune.get_tuning(v)
        dom_kernel = (f"k_bk_rotate<2,{tune[0]},{tune[1]},batched> (rotation + partner merge + filter over "
                      f"bucket pairs, 40-byte instance-tagged terms)")
    else:
        dom_bytes = B * (sp["merge_in"] + sp["merge_out"])
        dom_kernel = "k_merge<2,0> (merge + reduce-by-key + filter, 40-byte batched terms)"
    achieved = dom_bytes / sp["t_merge"] / 1e9 if sp["t_merge"] > 0 else None
    hbm, src = peaks()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        ti, dt = _oracle_batch_sample(0, 1, 12.0)
        cpu = {"value": ti / dt, "unit": "terms/s", "cores": 1, "kind": "port",
               "sample": f"the batch's instances in order, one layer at a time, layers entered with at most "
                         f"{BATCH_CPU_LIMIT} live terms, about 12 s of evolution ({ti:.3g} term-rotations); "
                         f"C restatement of the reference path, 1 thread"}
    if rank == 0:
        line = {
            "metric": "terms/s rotate+merge+clip (batched instances)", "value": value, "unit": "terms/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded instances)",
            "config": {"workload": f"batch256: {len(obs)} instances of the 8x8 lattice (N=64), depth U{{4..24}} "
                                   f"layers of 176 rotations, θ_J, θ_h ~ U[0.05, 0.5], observable a random "
                                   f"weight-1-4 Pauli string, CoeffTruncation({BATCH_THRESH}), no noise",
                       "instances": len(obs), "rotations": len(gens), "terms_in_per_step": terms_in,
                       "peak_terms": res[-1].stats["peak"],
                       "n_final_p50": float(np.percentile(res[-1].n_final, 50)),
                       "n_final_max": int(res[-1].n_final.max()),
                       "completion_p50_s": float(np.percentile(tdone, 50)),
                       "completion_p99_s": float(np.percentile(tdone, 99)),
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "no flush: the live set (up to ~3e8 terms x 40 B) exceeds L2"},
            "e2e": {"value": total_terms / t_e2e, "unit": "terms/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None, "traffic": None,
                         "kernel": dom_kernel, "bucket_rotations": sp["bucket_rot"],
                         "peak_source": src, "t_merge_s": sp["t_merge"], "t_rotate_s": sp["t_rotate"],
                         "t_partition_commit_s": sp["t_partition"]},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    v.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def run_reference_batch(args, ctx, q, nthreads):
    """Reference arm of batch256: the instances split over one worker process per
    host thread, each evolving its share layer by layer on the C restatement for a
    bounded time; value = the sum of the workers' term-rotations per second."""
    budget = 10.0 * args.steps
    procs = [ctx.Process(target=_oracle_batch_sample, args=(k, nthreads, budget, q)) for k in range(nthreads)]
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    value = sum(t / s for t, s in res if s > 0)
    line = {
        "metric": "terms/s rotate+merge+clip (batched instances)", "value": value, "unit": "terms/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * max(s for _, s in res), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded instances)", "impl": "reference",
        "config": {"workload": f"batch256 instances, CoeffTruncation({BATCH_THRESH}), layers entered with at "
                               f"most {BATCH_CPU_LIMIT} live terms", "threads": nthreads},
        "cpu_baseline": {"value": value, "unit": "terms/s", "cores": nthreads, "kind": "port",
                         "sample": f"each worker: its share of the instances for about {budget:.0f} s"},
        "e2e": {"value": value, "unit": "terms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


LEARN = {
    "full": dict(n_train=8, n_test=3, sample_layers=(6, 10, 14), per_layer=6000, train_steps=4000, batch=8192,
                 budgets=(5e6, 1e7, 2e7, 5e7, 1e8), plain=(1e-5, 3e-6, 2e-6, 1.5e-6, 1.2e-6, 1.1e-6)),
    "small": dict(n_train=2, n_test=1, sample_layers=(8, 12), per_layer=2000, train_steps=800, batch=4096,
                  budgets=(2e6, 1e7), plain=(1e-5, 3e-6)),
}
# label threshold: 1e-3 x |c| (rounded up to a decade) per sampled term, floor 1e-12
LEARN_T_REF, LEARN_T_BASE, LEARN_LABEL_T, LEARN_TOL = 1e-6, 1e-6, 1e-12, 1e-3
LEARN_AUDIT = dict(layers=(5, 11), sample=1024, bound=2.5e-4, label_thresh=1e-12)


def run_learned_bench(args):
    import numpy as np
    import pauliprop as pp
    from pauliprop import learned as L
    cfg = LEARN[args.learned_scale]
    lat = L.Lattice(8, 8, 20)
    train = L.angle_draws(cfg["n_train"], seed=41)
    test = L.angle_draws(cfg["n_test"], seed=42)
    t0 = time.perf_counter()
    X, T, lab = L.training_set(lat, train, cfg["sample_layers"], cfg["per_layer"], LEARN_T_BASE, LEARN_LABEL_T)
    t_data = time.perf_counter() - t0
    # the last training draw's samples validate the fit
    nval = len(T) // cfg["n_train"] if cfg["n_train"] > 1 else len(T) // 5
    mlp = pp.MLP(L.init_params(0))
    mlp.load_data(X[:-nval], T[:-nval])
    t1 = time.perf_counter()
    losses = mlp.train(cfg["train_steps"], batch=cfg["batch"], lr=1e-3, seed=0)
    t_train = time.perf_counter() - t1
    yv = mlp.forward(X[-nval:])
    r2 = 1.0 - float(np.mean((yv - T[-nval:]) ** 2) / max(1e-30, np.var(T[-nval:])))
    rows = []
    for draw in test:
        e_ref, t_ref, peak_ref = L.run_plain(lat, draw, LEARN_T_REF)
        plain = []
        for t in cfg["plain"]:
            e, dt, pk = L.run_plain(lat, draw, t)
            plain.append({"thresh": t, "err": abs(e - e_ref), "s": dt, "peak": pk})
        learned, coeff = [], []
        for B in cfg["budgets"]:
            e, dt, pk, au = L.run_learned(lat, draw, mlp, int(B), LEARN_T_BASE, audit=LEARN_AUDIT)
            learned.append({"budget": B, "err": abs(e - e_ref), "s": dt, "peak": pk, "reverted": au["reverted"],
                            "audits": au["audits"]})
            e2, dt2, pk2, _ = L.run_learned(lat, draw, None, int(B), LEARN_T_BASE)
            coeff.append({"budget": B, "err": abs(e2 - e_ref), "s": dt2, "peak": pk2})
        # every method reaches the tolerance at the latest with the reference run
        # itself (plain t_ref; a learned run with an unbounded budget is that run)
        ref_run = [(0.0, t_ref)]
        # error at matched time: for each plain run, the best learned error among
        # learned runs that took no longer
        matched = []
        for p in plain:
            le = [r["err"] for r in learned if r["s"] <= p["s"]]
            if le:
                matched.append(p["err"] / max(min(le), 1e-12))
        rows.append({"draw": draw, "ref": {"expect": e_ref, "s": t_ref, "peak": peak_ref}, "plain": plain,
                     "learned": learned, "coeff_budget": coeff,
                     "t_learned": L.time_to_error([(r["err"], r["s"]) for r in learned] + ref_run, LEARN_TOL),
                     "t_plain": L.time_to_error([(r["err"], r["s"]) for r in plain] + ref_run, LEARN_TOL),
                     "t_coeff_budget": L.time_to_error([(r["err"], r["s"]) for r in coeff] + ref_run, LEARN_TOL),
                     "plain_over_learned_error_at_matched_time": matched,
                     "coeff_over_learned_error_at_equal_budget": [c["err"] / max(l["err"], 1e-12)
                                                                  for c, l in zip(coeff, learned)]})
    med = lambda k: statistics.median([r[k] for r in rows])
    tl, tp = med("t_learned"), med("t_plain")
    allm = [x for r in rows for x in r["plain_over_learned_error_at_matched_time"]]
    allc = [x for r in rows for x in r["coeff_over_learned_error_at_equal_budget"]]
    line = {
        "metric": "time to |Δ⟨O⟩|≤1e-3 learned vs plain truncation", "value": tl, "unit": "s",
        "higher_is_better": False, "n_gpus": 1, "steps": 1, "warmup": 0, "dtype": "f64 (terms) / bf16 (network)",
        "data": "synthetic (seeded angle draws; labels generated by the engine)", "vs_baseline": None,
        "scaling": "weak",
        "config": {"workload": "learned truncation on the 8x8 lattice circuit (N=64, 20 layers of RZZ(θ_J) on 112 "
                               "edges + RX(θ_h) on 64 sites, depolarizing 1e-3, weight cap 12); θ_J ~ U[0.22,0.32], "
                               "θ_h ~ U[0.18,0.28]",
                   "reference_threshold": LEARN_T_REF, "base_threshold": LEARN_T_BASE,
                   "label_threshold": "1e-3 x |c| of the sampled term, rounded up to a decade",
                   "tolerance": LEARN_TOL, "scale": args.learned_scale,
                   "train_draws": len(train), "test_draws": len(test), "samples": int(len(T)),
                   "validation_r2": r2, "data_seconds": t_data, "train_seconds": t_train,
                   "train_tflops": 6 * 5313 * cfg["train_steps"] * cfg["batch"] / t_train / 1e12,
                   "loss_first_last": [float(losses[:10].mean()), float(losses[-10:].mean())],
                   "audit": LEARN_AUDIT},
        "plain_time_s": tp, "coeff_budget_time_s": med("t_coeff_budget"),
        "learned_over_plain": tl / tp,
        "per_draw_learned_over_plain": [r["t_learned"] / r["t_plain"] for r in rows],
        "median_plain_over_learned_error_at_matched_time": statistics.median(allm) if allm else None,
        "median_coeff_budget_over_learned_error_at_equal_budget": statistics.median(allc) if allc else None,
        "draws": rows,
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- our arm
def _start_oracle(wname):
    """Spawns the whole-circuit oracle run of a workload (before the first CUDA call)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    path = tempfile.NamedTemporaryFile(suffix=".npz", delete=False).name
    proc = ctx.Process(target=_oracle_background, args=(wname, path, q))
    proc.start()
    return proc, q, path


def run_ours(args):
    ws, rank, local = dist_init("nccl")
    # CPU baseline and final check: one whole-circuit oracle run per measured
    # workload in a spawned process, started before the first CUDA call, running
    # while the GPU is timed.  The headline config-2 run also measures config 3
    # (the 127-qubit graph circuit) as a secondary record.
    second = ("graph127" if args.workload == "lattice64" and ws == 1 and not args.no_secondary else None)
    orc = orc2 = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        orc = _start_oracle(args.workload)
        if second:
            orc2 = _start_oracle(second)
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    line = _measure(args, args.workload, ws, rank, local, dev, orc)
    if second:
        r2 = _measure(args, second, ws, rank, local, dev, orc2)
        if rank == 0:
            line["secondary"] = {second: {k: r2[k] for k in (
                "value", "unit", "ms_per_step", "e2e", "roofline", "cpu_baseline", "final_check",
                "gpu_launches", "clocks", "config", "tuning", "expectation")}}
            if r2["cpu_baseline"]:
                line["secondary"][second]["gpu_over_cpu_baseline"] = r2["value"] / r2["cpu_baseline"]["value"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def _measure(args, wname, ws, rank, local, dev, orc):
    """Warm-up, timed steps, e2e steps and the profiled step of one workload on this
    rank's GPU; on rank 0 returns the JSON line's fields (else None)."""
    import numpy as np
    import torch
    import pauliprop as pp
    orc_proc, orc_q, orc_path = orc if orc else (None, None, None)

    w = workload(wname)
    strat = strategy_of(w)
    gens, angs = w.generators()
    ch = (w.channel[0], w.channel[1], None) if w.channel else None
    per = len(w.layer)
    nw = pp.nwords(w.N)
    B = BYTES_PER_TERM[nw]
    # reference sizing of SparsePauliVector(O::PauliSum) for the observable
    live_cap = max(16, math.ceil(2.0 * len(w.observable)))
    ps = pp.PauliSum(w.N)
    for z, x, c in w.observable:
        ps[(z, x)] = c
    obs_z, obs_x = pp.pack_keys(w.N, list(ps.keys()))
    obs_c = np.array(list(ps.values()), dtype=np.float64)
    # key order: z then x, each as an integer whose last word is the most significant
    order = np.lexsort(tuple(obs_x[:, k] for k in range(nw)) + tuple(obs_z[:, k] for k in range(nw)))
    obs_z, obs_x, obs_c = obs_z[order], obs_x[order], obs_c[order]
    dz = torch.from_numpy(obs_z.copy()).to(dev)
    dx = torch.from_numpy(obs_x.copy()).to(dev)
    dc = torch.from_numpy(obs_c.copy()).to(dev)

    g = pp.SparsePauliVector(w.N, live_cap, live_cap)
    stream = torch.cuda.ExternalStream(g.stream(), device=dev)

    def upload_dev():
        pp.spv.check(pp.spv.lib.pp_upload(g._h, dz.data_ptr(), dx.data_ptr(), dc.data_ptr(), len(obs_c), 1))

    def one_step(stats=None, profile=False):
        upload_dev()
        _, e = pp.evolve_(g, gens, angs, truncation=strat, channel=ch, channel_every=per if ch else 0,
                          return_expectation=True, stats=stats, profile=profile)
        return e

    # warm-up
    for _ in range(args.warmup):
        one_step()
    st = {}
    one_step(stats=st)
    terms_in = st["terms_in"]
    launches = int(st["launches"])

    # timed region (device time on the engine's stream)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        expect = None
        for _ in range(args.steps):
            expect = one_step()
        e1.record(stream)
        torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    t = e0.elapsed_time(e1) * 1e-3
    t = reduce_max(t, ws, dev)
    total_terms = reduce_sum(terms_in * args.steps, ws, dev)
    value = total_terms / t

    # e2e through the public API with host buffers
    hz = torch.from_numpy(obs_z.copy()).pin_memory()
    hx = torch.from_numpy(obs_x.copy()).pin_memory()
    hc = torch.from_numpy(obs_c.copy()).pin_memory()
    # pinned host buffers for the result (a caller reading tens of MB per step
    # would allocate them once), sized for this step's final set
    fcap = max(1, len(g))
    pz = torch.empty((fcap, nw), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    px = torch.empty((fcap, nw), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    pc = torch.empty(fcap, dtype=torch.float64).pin_memory().numpy()
    h2d = d2h = 0
    te = []
    final = None
    for _ in range(args.steps):
        if ws > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        pp.spv.check(pp.spv.lib.pp_upload(g._h, hz.data_ptr(), hx.data_ptr(), hc.data_ptr(), len(obs_c), 1))
        _, ev = pp.evolve_(g, gens, angs, truncation=strat, channel=ch, channel_every=per if ch else 0,
                           return_expectation=True)
        n_out = len(g)
        if n_out > fcap:                      # (the same circuit every step: not expected)
            fcap = n_out
            pz = np.empty((fcap, nw), dtype=np.uint64)
            px = np.empty((fcap, nw), dtype=np.uint64)
            pc = np.empty(fcap, dtype=np.float64)
        zf, xf, cf = pz[:n_out], px[:n_out], pc[:n_out]
        m = pp.spv.c_int64()
        pp.spv.check(pp.spv.lib.pp_download(g._h, zf.ctypes.data, xf.ctypes.data, cf.ctypes.data, n_out,
                                            pp.spv.byref(m)))
        te.append(time.perf_counter() - t0)
        h2d = obs_z.nbytes + obs_x.nbytes + obs_c.nbytes + len(gens) * (2 * 8 * nw + 16)
        d2h = zf.nbytes + xf.nbytes + cf.nbytes + 8
        final = (zf, xf, cf, ev)
    t_e2e = reduce_max(sum(te), ws, dev)
    e2e_value = total_terms / t_e2e

    # profiled pass: per-kernel device time for the roofline of the dominant kernel
    sp = {}
    one_step(stats=sp, profile=True)
    pipe_bytes = B * (sp["terms_in"] + sp["merge_out"])          # B*(n + m) per rotation, summed
    tuning = pp.tune.get_tuning(g)
    if sp["bucket_rot"] > 0:
        # bucketed rotations: one k_bk_rotate launch per rotation reads its n live
        # terms and writes its m survivors, B*(n + m) per launch
        dom_bytes, dom_launches = sp["bucket_bytes"], sp["bucket_rot"]
        dom_kernel = (f"k_bk_rotate<{nw},{tuning[0]},{tuning[1]}> (rotation + partner merge + filter + "
                      f"channel over bucket pairs)")
        traffic_ratio = BUCKET_TRAFFIC_PER_ALG_BYTE
    elif sp["t_merge"] > 0:
        dom_bytes, dom_launches = B * (sp["merge_in"] + sp["merge_out"]), len(gens)   # B*(n + a + m)
        dom_kernel = "k_merge<1,0> (merge + reduce-by-key + filter + channel + compaction)"
        traffic_ratio = MERGE_TRAFFIC_PER_ALG_BYTE if w.name == "lattice64" else None
    else:
        # the whole sequence ran in k_small_run (one CTA, the set in shared memory):
        # its bytes are the step's B*(n + m), its time the step's
        dom_bytes, dom_launches = pipe_bytes, 1
        dom_kernel = f"k_small_run<{nw}> (whole sequence in one CTA)"
        traffic_ratio = None
        sp["t_merge"] = t / args.steps
    achieved = dom_bytes / sp["t_merge"] / 1e9 if sp["t_merge"] > 0 else None
    hbm, src = peaks()

    # CPU baseline (the concurrent whole-circuit oracle run) and the final check
    cpu = None
    final_check = None
    if orc_proc is not None:
        r = orc_q.get()
        orc_proc.join()
        o = np.load(orc_path)
        os.unlink(orc_path)
        zf, xf, cf, ev = final
        keys_equal = bool(np.array_equal(zf, o["z"]) and np.array_equal(xf, o["x"]))
        cdiff = float(np.abs(cf - o["c"]).max(initial=0.0)) if keys_equal else None
        ctol = 1e-12 * max(1.0, float(np.abs(o["c"]).max(initial=1.0)))
        diag = np.all(o["x"] == 0, axis=1)
        etol = 1e-12 * max(1.0, float(np.abs(o["c"][diag]).sum()))
        final_check = {"final_matches_oracle": bool(keys_equal and cdiff <= ctol and abs(ev - r["expect"]) <= etol),
                       "keys_bit_exact": keys_equal, "max_coef_diff": cdiff, "coef_tol": ctol,
                       "expectation_gpu": ev, "expectation_oracle": r["expect"], "expectation_tol": etol,
                       "terms_final": int(len(cf))}
        cpu = {"value": r["terms_in"] / r["seconds"], "unit": "terms/s", "cores": 1, "kind": "port",
               "sample": f"{w.name} end to end ({w.layers} layers x {per} rotations + channels from the "
                         f"observable, {r['terms_in']:.4g} term-rotations, {r['seconds']:.1f} s), C restatement "
                         f"of the reference path (oracle/liborc.so), 1 thread, run while the GPU was timed",
               "native_libs_loaded": r["libs"]}

    if rank == 0:
        line = {
            "metric": "terms/s rotate+merge+clip", "value": value, "unit": "terms/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded circuit)",
            "config": {"workload": workload_label(w),
                       "terms_in_per_step": terms_in, "peak_terms": st["peak"],
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "no flush: working set exceeds L2 at peak; the step re-creates its input"},
            "expectation": expect,
            "final_check": final_check,
            "e2e": {"value": e2e_value, "unit": "terms/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None,
                         "traffic": (traffic_ratio * dom_bytes / max(1.0, dom_launches)
                                     if traffic_ratio and w.name == "lattice64" else None),
                         "traffic_unit": "bytes per launch of the kernel (ncu-measured DRAM bytes per "
                                         "algorithmic byte x this step's mean algorithmic bytes per launch)",
                         "alg_bytes_per_launch": dom_bytes / max(1.0, dom_launches),
                         "kernel": dom_kernel, "launches_per_step": dom_launches,
                         "peak_source": src,
                         "pipeline_frac": pipe_bytes / (t / args.steps) / 1e9 / hbm,
                         "pipeline_frac_is": "B*(n + m) summed over the step's rotations / the timed step time",
                         "t_kernel_s": sp["t_merge"], "t_rotate_s": sp["t_rotate"],
                         "t_partition_commit_s": sp["t_partition"]},
            "tuning": {"bucket_cap": tuning[0], "items_per_thread": tuning[1], "load_div": tuning[2],
                       "chunk": tuning[3]},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
    else:
        line = None
    g.close()
    return line


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch256":
        run_ours_batch(args)
    elif args.workload == "learned":
        run_learned_bench(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
