"""Benchmark of the B200 triple-pattern exploration step.

Workload: the seeded LUBM-shaped synthetic graph (1,000 organisations by default) resident in
HBM, and the heavy queries of the heavy-query configuration: (a) a 3-pattern star from the
PersonA type index, (b) the memberOf / subOrgOf / degreeFrom triangle from the memberOf
predicate index.  One step = both heavy queries, each from its index start to its final table.

  value   heavy queries/s, device-resident: CUDA-graph replays timed with CUDA events on the
          library's stream, L2 flushed between steps (outside the timed brackets)
  e2e     the same through wk_query_execute_host: plan in, final table copied to pinned host
          memory every step, timed on the host clock
  plain   the one-launch-per-pattern path with a host sync per step (reference-shaped)

`--impl reference` times the CPU restatement of the reference engine (oracle/) on the host
cores with the reference's own intra-query split (mt_factor = cores) on the same config.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "wukong-cube_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def step_bytes(s):
    """Algorithmic bytes of one step (4-byte ids, 16-byte slots)."""
    k, R, C, Rp, D = s["kind"], s["rows_in"], s["cols_in"], s["rows_out"], s["sum_deg"]
    if k in ("index_to_unknown", "const_to_unknown"):
        return 16 + Rp * 4 + Rp * 4
    if k == "known_to_unknown":
        return R * C * 4 + R * 16 + D * 4 + Rp * (C + 1) * 4
    return R * C * 4 + R * 16 + D * 4 + Rp * C * 4


def build_graph(orgs, seed):
    import wukong_b200 as wk
    t0 = time.time()
    tr, v = wk.synth_generate(orgs, seed=seed)
    t1 = time.time()
    g = wk.GStore(tr)
    t2 = time.time()
    return tr, v, g, {"triples": int(tr.shape[0]), "gen_s": round(t1 - t0, 2),
                      "build_s": round(t2 - t1, 2), **g.info()}


def run_reference(args, world, rank):
    """CPU arm: the oracle (restated reference CPU engine) on all host cores."""
    if rank != 0:
        return
    import oracle
    import workloads
    import wukong_b200 as wk
    cores = os.cpu_count() or 1
    tr, v, g, ginfo = build_graph(args.orgs, args.seed)
    del g
    o = oracle.OracleStore(tr)
    qs = [workloads.heavy_star(v), workloads.heavy_triangle(v)]
    for _ in range(args.warmup):
        for q in qs:
            o.run(q.flat(), q.nvars, mt_factor=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for q in qs:
            st, tab, _ = o.run(q.flat(), q.nvars, mt_factor=cores)
            assert st == 0
        times.append(time.perf_counter() - t0)
    ms = 1000 * sum(times) / len(times)
    value = 2 * args.steps / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": config(args, ginfo),
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": "port",
                             "sample": "%d steps x (heavy star + heavy triangle), mt_factor=%d" %
                                       (args.steps, cores)},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


METRIC = "light-query QPS at p99 latency; heavy-query ms; vs plain per-query GPU path"


def config(args, ginfo):
    return {"workload": "heavy queries (star from PersonA type index + memberOf/subOrgOf/"
                        "degreeFrom triangle from predicate index) on the seeded LUBM-shaped "
                        "graph, %d organisations" % args.orgs,
            "orgs": args.orgs, "seed": args.seed, "graph": ginfo,
            "l2": "flushed between timed steps (256 MiB write)"}


def run_ours(args, world, rank, local_rank):
    import torch

    import oracle
    import workloads
    import wukong_b200 as wk

    torch.cuda.set_device(local_rank)
    tr, v, g, ginfo = build_graph(args.orgs, args.seed)
    ctx = wk.Context(local_rank)
    ctx.upload_gstore(g)
    ginfo["device_store_bytes"] = ctx.store_bytes()
    qs = [workloads.heavy_star(v), workloads.heavy_triangle(v)]
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(64 << 20, dtype=torch.int32, device="cuda")

    # correctness gate on the bench config: each heavy query vs the oracle
    rows = []
    o = oracle.OracleStore(tr) if rank == 0 and not args.no_check else None
    for q in qs:
        got, _ = ctx.execute(q, wk.MODE_GRAPH)
        rows.append(int(got.shape[0]))
        if o is not None:
            st, want, _ = o.run(q.flat(), q.nvars, mt_factor=os.cpu_count() or 1)
            assert st == 0 and np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want)), \
                "GPU result differs from the oracle"

    def one_step():
        for q in qs:
            ctx.enqueue(q, wk.MODE_GRAPH)

    for _ in range(args.warmup):
        one_step()
    ctx.check()
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    torch.cuda.synchronize()
    with Clocks(local_rank) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                ev[i][0].record(stream)
            one_step()
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
        torch.cuda.synchronize()
    ctx.check()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    tot_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([tot_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        tot_ms = float(t.item())
    value = len(qs) * args.steps * world / (tot_ms / 1000.0)

    # e2e through the C ABI with pinned host buffers (result table copied to the host)
    host = [torch.empty(max(r * 3 + 64, 64), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
            for r in rows]
    for q, h in zip(qs, host):
        ctx.execute_host(q, h, wk.MODE_GRAPH)
    t0 = time.perf_counter()
    d2h = 0
    for _ in range(args.steps):
        for q, h in zip(qs, host):
            r, c = ctx.execute_host(q, h, wk.MODE_GRAPH)
            d2h += r * c * 4
    e2e_s = time.perf_counter() - t0
    e2e = len(qs) * args.steps / e2e_s
    h2d = sum(len(q.patterns) * 20 for q in qs)

    # plain path: one launch per pattern, host sync per step
    for q in qs:
        ctx.execute(q, wk.MODE_PLAIN)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for q, h in zip(qs, host):
            ctx.execute_host(q, h, wk.MODE_PLAIN)
    plain = len(qs) * args.steps / (time.perf_counter() - t0)

    # roofline of the dominant kernel: per-step kernel times on the library stream
    prof = [ctx.profile(q, iters=max(3, args.steps)) for q in qs]
    steps = [s for p in prof for s in p]
    dom = max(steps, key=lambda s: s["ms"])
    peak, src = peaks()
    algo = step_bytes(dom)
    achieved = algo / (dom["ms"] / 1000.0) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "heavy queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": config(args, ginfo),
            "heavy_ms": {"star": None, "triangle": None},
            "e2e": {"value": e2e, "unit": "heavy queries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h // max(args.steps, 1)},
            "plain_path": {"value": plain, "unit": "heavy queries/s"},
            "rows": rows,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": src,
                         "kernel": dom["kind"], "algorithmic_bytes": algo, "kernel_ms": dom["ms"]},
            "profile": prof,
            "gpu_launches": sum(len(q.patterns) for q in qs) * args.steps,
            "clocks": clk.summary()}
    for name, p in zip(("star", "triangle"), prof):
        line["heavy_ms"][name] = sum(s["ms"] for s in p)
    if rank == 0:
        if not args.no_cpu:
            import oracle as orc
            cores = os.cpu_count() or 1
            if o is None:
                o = orc.OracleStore(tr)
            t0 = time.perf_counter()
            for q in qs:
                o.run(q.flat(), q.nvars, mt_factor=cores)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": len(qs) / dt, "unit": "heavy queries/s", "cores": cores,
                                    "kind": "port", "sample": "one run of each heavy query, mt_factor=%d" % cores}
        print(json.dumps(line))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--orgs", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, world, rank, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
