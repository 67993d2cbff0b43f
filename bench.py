"""Benchmark of the filter -> edge table -> enumerate path on B200.

Workload (the plain method at scale): a seeded Chung-Lu data graph with
1,000,000 vertices and 10,000,000 edges (degree exponent 2.2, unlabelled,
int32 neighbour ids), 100 seeded queries of 8 and 12 vertices (half dense:
greedy-densest growth, average degree > 3; half sparse: random-walk edges),
GQL filter, RI order, exhaustive counts capped at 10^9 per query.  Synthetic
data stands in for datasets (no network).

One step = the whole pipeline for one batch of 10 queries: NLF + GQL
filtering, candidate-edge tables, enumeration.  Steps walk through the
100-query workload batch by batch (warm-up on the first batches, timed steps
on the next ones).  `value` is queries/s over all
ranks with the data graph resident in HBM; `e2e` runs the same through the C
ABI from pinned host buffers (data-graph CSR upload, queries, counts back)
inside the timed region.  L2 (126 MB) is flushed before every timed step.

Multi-GPU: one process per GPU (torchrun); every rank runs its own 100
queries on a replica of the data graph (weak scaling, no data-path
collective); rank 0 prints the line with times = max over ranks.

--impl reference runs the reference's own CPU code (oracle/_ref, built from
the reference sources) on a bounded sample per step: the GQL filter of one
query and its enumeration to a reduced cap with all host threads, scaled to
queries/s by the measured embedding rate.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_VERT = 1_000_000
N_EDGE = 10_000_000
GAMMA = 2.2
GRAPH_SEED = 2
CAP = 1_000_000_000
WORKLOAD = "cfg2: Chung-Lu 1M V / 10M E (gamma 2.2), 100 queries of 8/12 vertices (half dense), GQL + RI, cap 1e9"
WORKLOAD3 = ("cfg3: the cfg2 graph with 32 labels drawn Zipf(1.0), queries of 16/24 vertices inheriting labels "
             "(half dense), NLF + GQL, RI, cache + failing sets, cap 1e9 as a guard")
METRIC = "queries/s & embeddings/s; learned-order vs RI-order GPU speedup at exact counts"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=10, help="queries per step")
    ap.add_argument("--impl", default="smx", choices=["smx", "reference"])
    ap.add_argument("--queries", type=int, default=100)
    ap.add_argument("--cap", type=int, default=CAP)
    ap.add_argument("--explore", type=int, default=0, help="0 candidate tables, 1 cache + failing sets")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", type=int, default=2, choices=[2, 3, 4],
                    help="2: the headline workload; 3: its labelled variant; 4: learned order + batched launch vs "
                         "RI order one query at a time")
    ap.add_argument("--chunk", type=int, default=50, help="--config 4: queries per batched launch")
    ap.add_argument("--train-queries", type=int, default=120, help="--config 4: queries that train the order model")
    return ap.parse_args()


def query_specs(nq: int, rank: int, sizes=(8, 12)):
    """(k, dense, seed) per query: two sizes, dense and sparse alternating."""
    out = []
    for i in range(nq):
        k = sizes[0] if (i // 2) % 2 == 0 else sizes[1]
        out.append((k, i % 2 == 0, 10_000 + rank * 100_000 + i))
    return out


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(prefix="smx_clocks_", suffix=".csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def ncu_traffic(launch_ms: float):
    """DRAM bytes (read + write) of one enumeration launch of launch_ms: the
    rate of the launch captured by ncu (profiles/enum_kernel_cfg2.json, a
    smaller cap of the same workload, cold caches) scaled by device time."""
    path = os.path.join(ROOT, "profiles", "enum_kernel_cfg2.json")
    if os.path.exists(path) and launch_ms > 0:
        with open(path) as f:
            rate = json.load(f).get("dram_bytes_per_ms")
        return rate * launch_ms if rate else None
    return None


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist

        backend = "nccl" if args.impl == "smx" else "gloo"
        if backend == "nccl":
            import torch

            torch.cuda.set_device(local)
        import datetime

        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if pg.get_backend() == "nccl" else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ---------------------------------------------------------------------- reference arm
def run_reference(args, world, rank, pg):
    if rank != 0:
        return
    from oracle import GQL, RefOracle, available

    if not available()["ref"]:
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle library not built (oracle/_ref)"}))
        return
    line = reference_sample(args, steps=args.steps, warmup=args.warmup)
    line["impl"] = "reference"
    line["e2e"] = {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line))


def reference_sample(args, steps: int, warmup: int, sample_cap: int = 20_000_000):
    """The reference (oracle/_ref) on a bounded sample: per step one query's
    GQL filter + RI order + enumeration to sample_cap with all host threads;
    queries/s is scaled from the filter time and the embedding rate to the
    workload's cap."""
    import subgraphmatching_b200 as smx
    from oracle import GQL, RefOracle

    R = RefOracle()
    threads = os.cpu_count() or 1
    g = smx.Graph.generate(N_VERT, N_EDGE, GAMMA, 1, 1.0, GRAPH_SEED, device=-1)
    tmp = tempfile.mkdtemp(prefix="smx_ref_")
    gpath = os.path.join(tmp, "data.txt")
    g.save(gpath)
    gr = R.load_graph(gpath)
    specs = query_specs(args.queries, 0)
    per_query_s = []
    emb_rates = []
    for step in range(warmup + steps):
        k, dense, seed = specs[step % len(specs)]
        q = smx.Query.generate(g, k, dense, seed)
        qpath = os.path.join(tmp, f"q{step}.txt")
        q.save(qpath)
        qr = R.load_query(qpath)
        t0 = time.perf_counter()
        c = R.filter(gr, qr, GQL)
        t_filter = time.perf_counter() - t0
        order = R.order_ri(qr)
        t0 = time.perf_counter()
        cnt, _, _ = R.explore(gr, qr, c, order, sample_cap, threads, R.CANDIDATES)
        t_enum = time.perf_counter() - t0
        rate = cnt / t_enum if t_enum > 0 else 0.0
        # a capped count reaches the workload cap at the measured rate; an exhaustive one is done
        t_full = t_filter + (args.cap / rate if cnt >= sample_cap and rate > 0 else t_enum)
        if step >= warmup:
            per_query_s.append(t_full)
            emb_rates.append(rate)
    mean_s = sum(per_query_s) / len(per_query_s)
    return {
        "metric": METRIC,
        "value": 1.0 / mean_s,
        "unit": "queries/s",
        "n_gpus": 0,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": mean_s * 1000.0,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded Chung-Lu graph and queries)",
        "config": {"workload": WORKLOAD, "cap": args.cap, "sample_cap": sample_cap},
        "embeddings_per_s": statistics.mean(emb_rates),
        "cpu_baseline": {"value": 1.0 / mean_s, "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": f"{steps} queries of the workload (after {warmup} warm-up), each: reference "
                                   f"Filter_GQL (1 thread) + Order_RI + explore_Intersection_Recursive to "
                                   f"{sample_cap:,} embeddings on {threads} threads, scaled to the {args.cap:,} cap "
                                   f"by the measured embedding rate"},
    }


# ---------------------------------------------------------------------- smx arm
def run_smx(args, world, rank, local, pg):
    import ctypes

    import numpy as np
    import torch

    import subgraphmatching_b200 as smx
    from subgraphmatching_b200 import _lib

    torch.cuda.set_device(local)
    dev = local
    labelled = args.config == 3
    hg = smx.Graph.generate(N_VERT, N_EDGE, GAMMA, 32 if labelled else 1, 1.0, GRAPH_SEED, device=-1)
    off, nb, lab = hg.csr()
    dg = smx.Graph.from_csr(off, nb, lab, device=dev)
    specs = query_specs(args.queries, rank, sizes=(16, 24) if labelled else (8, 12))
    if labelled:  # the labelled variant runs the cache + failing-set explorer
        args.explore = 1
    queries = [smx.Query.generate(hg, k, dense, seed) for k, dense, seed in specs]
    nb_batches = max(1, (len(queries) + args.batch - 1) // args.batch)
    batches = [queries[i * args.batch:(i + 1) * args.batch] for i in range(nb_batches)]
    opts = smx.EnumOptions(explore=args.explore)
    build_tables = args.explore == 0
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{dev}")

    n_enum = [0]
    at_cap = [0]

    def step(graph, batch):
        embeddings = 0
        kernel_ms = 0.0
        kbytes = 0
        for q in batch:
            can = smx.CandidateParam(graph, q, build_tables=build_tables)
            if smx.Filter_GQL(graph, q, can):
                st = smx.explore(graph, q, can, None, opts, args.cap)
                embeddings += st.count
                kernel_ms += st.kernel_ms
                kbytes += st.bytes
                n_enum[0] += 1
                at_cap[0] += bool(st.limit_reached)
        return embeddings, kernel_ms, kbytes

    for i in range(args.warmup):
        step(dg, batches[i % nb_batches])
    first = args.warmup  # timed steps continue through the workload
    # ---- timed: device-resident inputs
    times, emb, kms, kby = [], 0, 0.0, 0
    launches0 = _lib.lib.smx_launch_count()
    n_enum[0] = 0
    at_cap[0] = 0
    clocks = Clocks(dev)
    clocks.start()
    nq_timed = 0
    for i in range(args.steps):
        batch = batches[(first + i) % nb_batches]
        nq_timed += len(batch)
        flush.zero_()
        torch.cuda.synchronize()
        barrier(pg)
        _lib.check(_lib.lib.smx_mark_begin(dg._h))
        e, km, kb = step(dg, batch)
        ms = ctypes.c_double()
        _lib.check(_lib.lib.smx_mark_end(dg._h, ctypes.byref(ms)))
        torch.cuda.synchronize()
        barrier(pg)
        times.append(ms.value)
        emb += e
        kms += km
        kby += kb
    clock_info = clocks.stop()
    launches = _lib.lib.smx_launch_count() - launches0
    enum_launches = n_enum[0]
    timed_at_cap = at_cap[0]
    step_ms = max_over_ranks(pg, sum(times) / len(times))
    # ---- e2e: pinned host CSR -> device graph, queries, counts back, per step
    p_off = torch.from_numpy(off.view(np.int64)).pin_memory()
    p_nb = torch.from_numpy(nb.view(np.int32)).pin_memory()
    p_lab = torch.from_numpy(lab.view(np.int32)).pin_memory()
    u64p = ctypes.POINTER(ctypes.c_uint64)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    e2e_times = []
    for i in range(max(1, args.steps)):
        flush.zero_()
        torch.cuda.synchronize()
        barrier(pg)
        t0 = time.perf_counter()
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.smx_graph_create(ctypes.cast(p_off.data_ptr(), u64p), ctypes.cast(p_nb.data_ptr(), u32p),
                                             ctypes.cast(p_lab.data_ptr(), u32p), N_VERT, int(off[-1]), dev,
                                             ctypes.byref(h)))
        g2 = smx.Graph(h)
        step(g2, batches[(first + i) % nb_batches])
        del g2
        torch.cuda.synchronize()
        e2e_times.append((time.perf_counter() - t0) * 1000.0)
        barrier(pg)
    e2e_ms = max_over_ranks(pg, sum(e2e_times) / len(e2e_times))
    b0 = batches[first % nb_batches]
    h2d = off.nbytes + nb.nbytes + lab.nbytes + sum(q.csr()[0].nbytes + q.csr()[1].nbytes + q.csr()[2].nbytes
                                                    for q in b0)
    d2h = 8 * len(b0) * 3  # counts + stats read back per query
    if rank != 0:
        return
    q_per_step = nq_timed / args.steps * world
    value = q_per_step / (step_ms / 1000.0)
    hbm, peak_kind = peaks()
    achieved = (kby / 1e9) / (kms / 1000.0) if kms > 0 else 0.0
    launch_ms = kms / enum_launches if enum_launches else 0.0
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded Chung-Lu graph and queries; no dataset download)",
        "config": {"workload": WORKLOAD3 if labelled else WORKLOAD, "queries_per_gpu": len(queries),
                   "queries_per_step": args.batch,
                   "cap": args.cap,
                   "explore": "candidate tables" if args.explore == 0 else "cache + failing sets",
                   "l2": "flushed (256 MB write) before every timed step", "parallelism": f"replicas x{world}",
                   "timed_queries_at_cap": timed_at_cap},
        "embeddings_per_s": emb * world / (sum(times) / 1000.0),
        "e2e": {"value": q_per_step / (e2e_ms / 1000.0), "unit": "queries/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm if hbm else None, "traffic": ncu_traffic(launch_ms),
                     "kernel": "enum_kernel", "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": kby / enum_launches if enum_launches else None,
                     "note": "achieved = algorithmic bytes (list elements touched x 4 + row/candidate reads) / "
                             "event-timed kernel time, summed over the timed launches; traffic = DRAM bytes of "
                             "an average timed launch, from the ncu capture's bytes per ms (cold caches)"},
        "gpu_launches": int(launches),
        "clocks": clock_info,
    }
    if not args.no_cpu_baseline and world == 1:
        try:
            ref = reference_sample(args, steps=1, warmup=0)
            line["cpu_baseline"] = ref["cpu_baseline"]
        except Exception as e:  # the reference build may be absent
            line["cpu_baseline"] = {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    print(json.dumps(line))


# ---------------------------------------------------------------------- config 4
C4_VERT, C4_EDGE, C4_SEED = 4_000_000, 40_000_000, 4
C4_CAP, C4_BUDGET_MS = 100_000_000, 2000.0


def c4_specs(n: int, base: int):
    """(k, dense, seed): sizes uniform in 4..32 (seeded), dense and sparse alternating."""
    import numpy as np

    rng = np.random.default_rng(base)
    return [(int(rng.integers(4, 33)), i % 2 == 0, base + i) for i in range(n)]


def run_cfg4(args, world, rank, local, pg):
    """Learned order + one batched persistent launch per chunk (autotuned
    settings) against RI order with one launch per query, on the same
    filtered candidates; counts must agree wherever neither run hit the time
    budget.  Filtering is timed separately (it is the same for both).  Both
    sides use the cache + failing-set explorer: candidate-edge tables of
    dense 32-vertex queries on this graph would take tens of GB per query."""
    import numpy as np

    import subgraphmatching_b200 as smx
    from subgraphmatching_b200 import autotune as at
    from subgraphmatching_b200 import learned_order as lo

    dev = local
    t0 = time.perf_counter()
    hg = smx.Graph.generate(C4_VERT, C4_EDGE, GAMMA, 1, 1.0, C4_SEED, device=-1)
    off, nb, lab = hg.csr()
    dg = smx.Graph.from_csr(off, nb, lab, device=dev)
    nq = args.queries
    queries = [smx.Query.generate(hg, k, d, s) for k, d, s in c4_specs(nq, 1_000_000 + rank * 100_000)]
    train_q = [smx.Query.generate(hg, k, d, s) for k, d, s in c4_specs(args.train_queries, 2_000_000)]
    setup_s = time.perf_counter() - t0
    # the order model, trained on queries of its own
    t0 = time.perf_counter()
    opts1 = smx.EnumOptions(explore=1)
    samples = lo.collect(dg, train_q, beam=8, cap=10_000_000, budget_ms=300.0, opts=opts1, build_tables=False)
    model = smx.MLP(dev, 1024, seed=7)
    lo.train(model, samples, epochs=60, batch=128, lr=2e-3)
    train_s = time.perf_counter() - t0
    # autotuned launch settings on a sample chunk
    sample = queries[: min(20, nq)]
    cans = [smx.CandidateParam(dg, q, build_tables=False) for q in sample]
    oks = [smx.Filter_GQL(dg, q, c) for q, c in zip(sample, cans)]
    best, report = at.autotune(dg, [q for q, ok in zip(sample, oks) if ok], [c for c, ok in zip(cans, oks) if ok],
                               cap=C4_CAP, budget_ms=C4_BUDGET_MS, explore=1, repeats=1, grid=at.GRID_CACHE)
    best.time_budget_ms = C4_BUDGET_MS
    best.budget_per_query = 1  # the same budget per query as the single launches
    del cans
    ri_ms = bl_ms = filt_s = 0.0
    ri_dev = bl_dev = 0.0
    mismatches = compared = timeouts = 0
    for c0 in range(0, nq, args.chunk):
        chunk = queries[c0:c0 + args.chunk]
        t = time.perf_counter()
        cans = [smx.CandidateParam(dg, q, build_tables=False) for q in chunk]
        oks = [smx.Filter_GQL(dg, q, c) for q, c in zip(chunk, cans)]
        filt_s += time.perf_counter() - t
        qs = [q for q, ok in zip(chunk, oks) if ok]
        cs = [c for c, ok in zip(cans, oks) if ok]
        # RI order, one launch per query
        t = time.perf_counter()
        ri = [smx.explore(dg, q, c, None, smx.EnumOptions(explore=1, time_budget_ms=C4_BUDGET_MS), C4_CAP)
              for q, c in zip(qs, cs)]
        ri_ms += (time.perf_counter() - t) * 1000.0
        ri_dev += sum(r.kernel_ms for r in ri)
        # learned order (inference included) + one batched launch
        t = time.perf_counter()
        orders = [smx.Order_Learned(model, q, c, 32, 7) for q, c in zip(qs, cs)]
        counts, st = smx.explore_batch(dg, qs, cs, orders, best, C4_CAP)
        bl_ms += (time.perf_counter() - t) * 1000.0
        bl_dev += st.kernel_ms
        for r, c, s_ in zip(ri, counts, st.query_status):
            if r.status == 0 and s_ == 0:
                compared += 1
                mismatches += r.count != c
        timeouts += sum(r.status != 0 for r in ri) + sum(s_ != 0 for s_ in st.query_status)
        del cans, cs
    if rank != 0:
        return
    line = {
        "metric": "queries/s: learned order + batched persistent launch vs RI order, one launch per query",
        "value": nq / (bl_ms / 1000.0), "unit": "queries/s", "n_gpus": world, "higher_is_better": True,
        "ri_single_value": nq / (ri_ms / 1000.0),
        "speedup_vs_ri_single": ri_ms / bl_ms if bl_ms else None,
        "device_ms": {"ri_single": ri_dev, "learned_batched": bl_dev},
        "counts": {"compared": compared, "mismatches": mismatches, "query_runs_at_time_budget": timeouts},
        "dtype": "u32", "data": "synthetic (seeded Chung-Lu graph and queries)",
        "config": {"workload": f"cfg4: Chung-Lu {C4_VERT:,} V / {C4_EDGE:,} E (gamma {GAMMA}), {nq} queries of "
                               f"4-32 vertices (half dense), GQL, cache + failing-set explorer, cap {C4_CAP:.0e}, budget {C4_BUDGET_MS:.0f} ms",
                   "chunk": args.chunk, "train_queries": args.train_queries, "train_samples": int(len(samples.t)),
                   "autotuned": report["best"]},
        "seconds": {"setup": setup_s, "train": train_s, "filter": filt_s},
    }
    print(json.dumps(line))


def main():
    args = parse()
    world, rank, local, pg = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, pg)
        elif args.config == 4:
            run_cfg4(args, world, rank, local, pg)
        else:
            run_smx(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
