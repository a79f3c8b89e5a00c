"""Benchmark of the wedge-parallel triangle count on B200.

Workload: seeded R-MAT scale 22, edge factor 16, (a, b, c, d) =
(0.57, 0.19, 0.19, 0.05), symmetrised, deduplicated, self-loops removed
(generated and preprocessed on the device). One step = one exact count of
the whole graph from the device-resident oriented CSR: wedge prefix, tile
map, bitmap and count kernels, plus the count's read-back.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--s S] [--a A]
    python bench.py --impl reference ...   # the reference's own tc (sm_100a)

Metric: wedges/s (W x steps / time); triangles/s and the HBM-roofline
fraction of the count kernel are reported beside it. For N > 1 (torchrun)
every rank holds the whole CSR and counts an equal share of the wedge range;
the partial counts are summed with one 8-byte all-reduce per step; time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "wedge-parallel-triangle-counting_b200"))

import numpy as np  # noqa: E402

SPEC_ARGS = dict(scale=22, edge_factor=16, seed=1)
METRIC = "wedges/s (exact triangle count, R-MAT s22 ef16)"
UNIT = "wedges/s"


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(workload: str, kernel: int, s: int, a: int):
    """The committed ncu figures of the count kernel for this workload,
    kernel variant, s and a (profiles/traffic.json): DRAM read + write bytes
    per launch and, where captured, L2 bytes, warp instructions and the L2
    hit rate of the bitmap's loads. None when no capture matches."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f)
    for e in t.get("count_kernel", []):
        if (e.get("workload"), e.get("kernel"), e.get("s"), e.get("a")) == (workload, kernel, s, a):
            return e
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [l.strip().split(", ") for l in self.file.read().splitlines() if l.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(og_host, W_total, triangles):
    """The CPU baseline on the whole graph: the reference's host
    preprocessing restated by the oracle (symmetrise, qsort, dedup, stable
    degree order, orientation, row sort -- tc.cu:561-787, one thread, as in
    the reference) from the same seeded R-MAT pairs, then the oracle's
    OpenMP merge-intersection count on all host threads. The oracle's
    oriented CSR and count must equal ours bit for bit."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    src, dst = oracle.gen_rmat(SPEC_ARGS["scale"], SPEC_ARGS["edge_factor"] << SPEC_ARGS["scale"],
                               seed=SPEC_ARGS["seed"])
    t0 = time.perf_counter()
    g = oracle.preprocess(oracle.csr_from_pairs(src, dst))
    prep_s = time.perf_counter() - t0
    del src, dst
    same_csr = (np.array_equal(g.row_ptr, np.asarray(og_host.row_ptr, dtype=np.uint64))
                and np.array_equal(g.col_ind, og_host.col_ind))
    t0 = time.perf_counter()
    tri = oracle.count_merge(g)
    count_s = time.perf_counter() - t0
    if not same_csr or tri != triangles:
        raise RuntimeError(f"CPU baseline disagrees: csr equal {same_csr}, {tri} vs {triangles}")
    threads = oracle.max_threads()
    return {"value": W_total / count_s, "unit": UNIT, "cores": threads, "kind": "port",
            "cpu_model": oracle.cpu_model(), "prep_s": prep_s, "count_s": count_s,
            "value_incl_prep": W_total / (prep_s + count_s),
            "oriented_csr_equal": bool(same_csr), "triangles": int(tri),
            "sample": (f"whole graph ({W_total} wedges): host preprocessing of the "
                       f"{SPEC_ARGS['edge_factor'] << SPEC_ARGS['scale']} seeded pairs (oracle "
                       f"restatement of tc.cu:561-787, qsort, 1 thread) {prep_s:.2f} s, then the "
                       f"OpenMP merge-intersection count on {threads} threads {count_s:.2f} s; "
                       f"value = wedges / count time")}


def cost_balanced_range(og, W, rank, world, dev, args):
    """This rank's wedge range when the ranks share one graph: equal device
    time rather than equal wedges. The dense core's wedges (the top of the
    wedge order, [W - core_wedges, W)) cost a fraction of the others', so
    equal wedge ranges would leave the low ranks with most of the time. One
    whole-graph count (run by every rank alike) gives the two kernels'
    times per wedge; the cuts split the piecewise-linear cost evenly."""
    import torch
    import torch.distributed as dist

    _, st = og.count(args.s, args.a, device=dev, kernel=args.kernel, core_len=args.core_len,
                     pair_streams=False)
    from wetric.parallel import cost_balanced_cuts

    cuts = cost_balanced_cuts(W, st.core_wedges, st.count_ms - st.core_ms, st.core_ms, world)
    # rank 0's cuts for every rank, so the ranges tile [0, W) exactly
    t = torch.tensor(cuts, dtype=torch.int64, device=f"cuda:{dev}")
    dist.broadcast(t, src=0)
    cuts = [int(x) for x in t.tolist()]
    return cuts[rank], cuts[rank + 1]


def run_ours(args):
    import torch
    import torch.distributed as dist

    import wetric
    from wetric import workloads as Wl

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    spec = Wl.RmatSpec(**SPEC_ARGS)

    src, dst, _ = Wl.device_pairs(spec, dev)
    og = wetric.orient_edges(src, dst, device=dev)
    prep_ms = og.stats.prep_ms
    del src, dst
    torch.cuda.empty_cache()
    rp_dev = torch.empty(og.n + 1, dtype=torch.int64, device=f"cuda:{dev}")
    ci_dev = torch.empty(og.m, dtype=torch.int32, device=f"cuda:{dev}")
    host = og.download()
    rp_dev.copy_(torch.from_numpy(host.row_ptr.view(np.int64)))
    ci_dev.copy_(torch.from_numpy(host.col_ind.view(np.int32)))
    W, maxdeg = wetric.wedge_total(rp_dev, dev)
    b_alg = wetric.algorithmic_bytes(rp_dev, ci_dev, dev)
    lo, hi = W * rank // world, W * (rank + 1) // world
    if world > 1:
        lo, hi = cost_balanced_range(og, W, rank, world, dev, args)
    stream = torch.cuda.current_stream()

    # one GPU counts the whole graph (wedge_end 0), which lets the count
    # take pair streams for its short rows
    hi_arg = hi if world > 1 else 0

    def step():
        c, st = og.count(args.s, args.a, device=dev, wedge_begin=lo, wedge_end=hi_arg,
                         stream=stream, kernel=args.kernel, core_len=args.core_len,
                         pair_streams=bool(args.pair_streams))
        if world > 1:
            t = torch.tensor([c], dtype=torch.int64, device=f"cuda:{dev}")
            dist.all_reduce(t)
            c = int(t.item())
        return c, st

    for _ in range(args.warmup):
        tri, _ = step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    count_ms, exec_ms, core_ms, pair_ms, launches = [], [], [], [], 0
    e0.record(stream)
    for _ in range(args.steps):
        tri, st = step()
        count_ms.append(st.count_ms)
        exec_ms.append(st.exec_ms)
        core_ms.append(st.core_ms)
        pair_ms.append(st.pair_ms)
        launches += st.launches
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps

    # End to end through the reference-shaped call: host (pinned) oriented
    # CSR with u32 offsets -> H2D inside the call -> count -> D2H.
    rp32 = torch.from_numpy(host.row_ptr.astype(np.uint32).view(np.int32)).pin_memory()
    ci32 = torch.from_numpy(host.col_ind.view(np.int32)).pin_memory()
    rp32_np = rp32.numpy().view(np.uint32)
    ci32_np = ci32.numpy().view(np.uint32)
    for _ in range(args.warmup):
        wetric.count(rp32_np, ci32_np, args.s, args.a, device=dev, wedge_begin=lo,
                     wedge_end=hi, kernel=args.kernel, core_len=args.core_len)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_launches = 0
    e2e_parts = []
    e2e_steps = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        c, st = wetric.count(rp32_np, ci32_np, args.s, args.a, device=dev,
                             wedge_begin=lo, wedge_end=hi, kernel=args.kernel,
                             core_len=args.core_len)
        e2e_steps.append((time.perf_counter() - t1) * 1e3)
        e2e_launches += st.launches
        e2e_parts.append((st.copy_ms, st.exec_ms, st.count_ms))
        if world > 1:
            t = torch.tensor([c], dtype=torch.int64, device=f"cuda:{dev}")
            dist.all_reduce(t)
            c = int(t.item())
        assert c == tri
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    # The same call with pageable host arrays (plain numpy memory, what a
    # caller of the reference's tc_GPU passes: tc.cu:370-392 copies from
    # malloc'd buffers).
    rp_pg = host.row_ptr.astype(np.uint32)
    ci_pg = np.array(host.col_ind, dtype=np.uint32, copy=True)
    for _ in range(args.warmup):
        wetric.count(rp_pg, ci_pg, args.s, args.a, device=dev, wedge_begin=lo,
                     wedge_end=hi, kernel=args.kernel, core_len=args.core_len)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        c, st = wetric.count(rp_pg, ci_pg, args.s, args.a, device=dev,
                             wedge_begin=lo, wedge_end=hi, kernel=args.kernel,
                             core_len=args.core_len)
        if world > 1:
            t = torch.tensor([c], dtype=torch.int64, device=f"cuda:{dev}")
            dist.all_reduce(t)
            c = int(t.item())
        assert c == tri
    torch.cuda.synchronize()
    pg_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([pg_s], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        pg_s = float(t.item())

    if rank != 0:
        og.free()
        dist.destroy_process_group()
        return
    peak, peak_kind = load_peaks()
    count_ms_avg = statistics.mean(count_ms)
    share = (hi - lo) / W if W else 1.0
    workload = spec.name
    cap = (load_traffic(workload, args.kernel, args.s, args.a)
           if world == 1 and (lo, hi) == (0, W) else None)
    traffic = cap.get("dram_bytes_per_launch") if cap else None
    # The roofline is HBM: achieved = DRAM bytes the count kernel moves per
    # launch (ncu capture of this workload, kernel, s and a) / its event time.
    achieved = traffic / (count_ms_avg / 1e3) / 1e9 if traffic else None
    # The byte model of the reference's own algorithm (every wedge charged
    # its u load, two row offsets and a full binary search, as if from DRAM)
    # over the same time: how fast a search-based count would have to stream.
    ref_equiv = b_alg * share / (count_ms_avg / 1e3) / 1e9
    line = {
        "metric": METRIC,
        "value": W * args.steps / (ms / 1e3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "u32 ids, u64 counts (integer)",
        "data": "synthetic (seeded R-MAT generated on device)",
        "config": {
            "workload": workload, "n": og.n, "m": og.m, "wedges": W, "kernel": args.kernel,
            "triangles": tri, "max_out_degree": maxdeg, "s": args.s, "a": args.a,
            "parallelism": f"wedge-range x{world} (cost-balanced)" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (col_ind %.0f MB, row offsets %.0f MB)"
                  % (og.m * 4 / 1e6, (og.n + 1) * 4 / 1e6),
            "device_prep_ms": prep_ms,
            "exec_ms_per_step": statistics.mean(exec_ms),
            "count_kernel_ms": count_ms_avg,
            "core_len": st.core_len, "core_wedges": st.core_wedges,
            "core_kernel_ms": statistics.mean(core_ms),
            "pair_rows": st.pair_rows, "pair_wedges": st.pair_wedges,
            "pair_kernel_ms": statistics.mean(pair_ms),
            "triangles_per_s": tri * args.steps / (ms / 1e3),
        },
        "roofline": {
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved is not None else None,
            "traffic": traffic, "peak_source": peak_kind,
            "traffic_source": cap.get("source") if cap else None,
            "l2_gbs": (cap["lts_bytes_per_launch"] / (count_ms_avg / 1e3) / 1e9
                       if cap and cap.get("lts_bytes_per_launch") else None),
            "bitmap_l2_hit_rate": cap.get("bitmap_l2_hit_rate") if cap else None,
            "inst_per_wedge": (cap["warp_inst_per_launch"] * 32 / W
                               if cap and cap.get("warp_inst_per_launch") else None),
            "algorithmic_bytes": b_alg,
            "reference_equivalent_gbs": ref_equiv,
        },
        "e2e": {
            "value": W * args.steps / e2e_s, "unit": UNIT,
            "h2d_bytes_per_step": int(rp32.numel() * 4 + ci32.numel() * 4),
            "d2h_bytes_per_step": 36,
            "ms_per_step": e2e_s * 1e3 / args.steps,
            # per-call device timings inside the call (means over the steps)
            "copy_ms": statistics.mean(p[0] for p in e2e_parts),
            "exec_ms": statistics.mean(p[1] for p in e2e_parts),
            "count_ms": statistics.mean(p[2] for p in e2e_parts),
            # the calls' own wall times (rank 0), to show a slow step
            "call_ms_median": statistics.median(e2e_steps),
            "call_ms_max": max(e2e_steps),
            "call_ms_steps": [round(x, 2) for x in e2e_steps],
            "exec_ms_max": max(p[1] for p in e2e_parts),
            "host_memory": "pinned",
        },
        "e2e_pageable": {
            "value": W * args.steps / pg_s, "unit": UNIT,
            "h2d_bytes_per_step": int(rp_pg.nbytes + ci_pg.nbytes),
            "d2h_bytes_per_step": 36, "ms_per_step": pg_s * 1e3 / args.steps,
            "host_memory": "pageable (numpy)",
        },
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(host, W, tri)
    print(json.dumps(line), flush=True)
    og.free()
    if world > 1:
        dist.destroy_process_group()


SWEEP_S = (1, 2, 5, 10)
SWEEP_A = (0, 4096, 8192, 16384)


def run_sweep(args):
    """The R-MAT scale-22 sweep over s in {1, 2, 5, 10} x a in {0, 4096,
    8192, 16384}: one JSON line per (s, a) with the count kernel's and the
    whole count's device time (median of --steps after --warmup) -- ours,
    or with --impl reference the reference tc's GPU exec column."""
    if args.impl == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        if not oracle.have_reference_binary():
            print(json.dumps({"impl": "reference",
                              "unavailable": "oracle/_ref/tc not built (make -C oracle ref)"}))
            return
        with tempfile.TemporaryDirectory() as tmp:
            path, W, _ = _reference_input(tmp)
            name = os.path.basename(path)[:-4]
            for s_ in SWEEP_S:
                for a_ in SWEEP_A:
                    rows = oracle.run_reference(path, s_, a_, loops=args.warmup + args.steps,
                                                timeout=1800)[args.warmup:]
                    ex = statistics.median(r["exec"] for r in rows)
                    print(json.dumps({"impl": "reference", "workload": name + "-sweep",
                                      "s": s_, "a": a_, "gpu_exec_ms": 1e3 * ex,
                                      "wedges_per_s": W / ex,
                                      "triangles": rows[0]["triangles"]}), flush=True)
        return
    import torch

    import wetric
    from wetric import workloads as Wl

    spec = Wl.RmatSpec(**SPEC_ARGS)

    torch.cuda.set_device(0)
    src, dst, _ = Wl.device_pairs(spec, 0)
    og = wetric.orient_edges(src, dst, device=0)
    del src, dst
    want = None
    for s_ in SWEEP_S:
        for a_ in SWEEP_A:
            cms, ems = [], []
            for k in range(args.warmup + args.steps):
                c, st = og.count(s_, a_, device=0, kernel=args.kernel)
                want = c if want is None else want
                if c != want:
                    raise RuntimeError(f"count {c} at s={s_} a={a_} differs from {want}")
                if k >= args.warmup:
                    cms.append(st.count_ms)
                    ems.append(st.exec_ms)
            cm = statistics.median(cms)
            print(json.dumps({"workload": spec.name + "-sweep", "kernel": args.kernel,
                              "s": s_, "a": a_, "count_kernel_ms": cm,
                              "exec_ms": statistics.median(ems),
                              "wedges_per_s": st.wedges / (cm / 1e3),
                              "triangles": int(c)}), flush=True)
    og.free()


def _reference_input(tmp):
    """The headline workload written as Matrix Market for the reference's own
    tc, made by the oracle's copy of the seeded R-MAT stream (a CPU test
    checks it against the library's), so the reference arm's process never
    loads this repository's library. Returns (path, W, max out-degree)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    sc, ef = SPEC_ARGS["scale"], SPEC_ARGS["edge_factor"]
    src, dst = oracle.gen_rmat(sc, ef << sc, seed=SPEC_ARGS["seed"])
    W, maxdeg = oracle.wedge_total_from_pairs(src, dst)
    path = os.path.join(tmp, f"rmat-s{sc}-ef{ef}-seed{SPEC_ARGS['seed']}.mtx")
    oracle.write_mm(path, 1 << sc, src, dst)
    return path, W, maxdeg


def run_core_sweep(args):
    """The dense core and shell on R-MAT scale 22: one JSON line per (s, a,
    core length, shell length) with the median of --steps counts after
    --warmup -- the count kernels' time, the core's and the shell's, and the
    share of the wedges each took. Every count must be the same."""
    import torch

    import wetric
    from wetric import workloads as Wl

    torch.cuda.set_device(0)
    spec = Wl.RmatSpec(**SPEC_ARGS)
    src, dst, _ = Wl.device_pairs(spec, 0)
    og = wetric.orient_edges(src, dst, device=0)
    del src, dst
    OFF = wetric.CORE_OFF
    configs = [(5, 8192, OFF, OFF)]
    for h in (0, 8192, 16384, 24576, 32768, 40960, 49152, 57344, 65536):
        configs.append((5, 8192, h, OFF))
    for h in (16384, 32768):
        for sh in (h, 3 * h):
            configs.append((5, 8192, h, sh))
    for s_, a_ in ((10, 16384), (5, 16384), (2, 8192), (1, 0)):
        configs += [(s_, a_, OFF, OFF), (s_, a_, 0, OFF)]
    want = None
    for s_, a_, core, shell in configs:
        cm, km, sm_, em = [], [], [], []
        for k in range(args.warmup + args.steps):
            c, st = og.count(s_, a_, device=0, core_len=core, shell_len=shell, kernel=args.kernel)
            want = c if want is None else want
            if c != want:
                raise RuntimeError(f"count {c} differs from {want} at {s_, a_, core, shell}")
            if k >= args.warmup:
                cm.append(st.count_ms)
                km.append(st.core_ms)
                sm_.append(st.shell_ms)
                em.append(st.exec_ms)
        print(json.dumps({"workload": spec.name + "-core", "s": s_, "a": a_,
                          "core_req": "off" if core == OFF else ("auto" if core == 0 else core),
                          "shell_req": "off" if shell in (OFF, 0) else shell,
                          "core_len": st.core_len, "shell_len": st.shell_len,
                          "core_share": round(st.core_wedges / st.wedges, 4),
                          "shell_share": round(st.shell_wedges / st.wedges, 4),
                          "count_kernels_ms": round(statistics.median(cm), 3),
                          "core_ms": round(statistics.median(km), 3),
                          "shell_ms": round(statistics.median(sm_), 3),
                          "exec_ms": round(statistics.median(em), 3),
                          "triangles": int(c)}), flush=True)
    og.free()


def run_reference(args):
    """The reference's own tc, compiled unmodified for sm_100a into
    oracle/_ref, on the same workload written as Matrix Market. It runs
    -l (warmup + steps) loops of its tc_GPU call and the first `warmup` rows
    are dropped, so both arms take the same number of warm-up steps."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.have_reference_binary():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/tc not built (make -C oracle ref)"}))
        return
    workload = f"rmat-s{SPEC_ARGS['scale']}-ef{SPEC_ARGS['edge_factor']}-seed{SPEC_ARGS['seed']}"
    with tempfile.TemporaryDirectory() as tmp:
        path, W, maxdeg = _reference_input(tmp)
        if maxdeg >= 65536:
            print(json.dumps({"impl": "reference", "unavailable":
                              "max out-degree >= 2^16 overflows the reference's u32 wedge math"}))
            return
        t0 = time.perf_counter()
        rows = oracle.run_reference(path, args.s, args.a, loops=args.warmup + args.steps,
                                    timeout=1800)
        wall = time.perf_counter() - t0
    rows = rows[args.warmup:]
    cpu_gpu = [r["cpu_gpu"] for r in rows]
    execs = [r["exec"] for r in rows]
    tri = rows[0]["triangles"]
    value = W * len(rows) / sum(cpu_gpu)
    line = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": len(rows), "warmup": args.warmup, "ms_per_step": 1e3 * sum(cpu_gpu) / len(rows),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32 ids, u64 counts (integer)",
        "data": "synthetic (seeded R-MAT, Matrix Market file)",
        "config": {"workload": workload, "n": rows[0]["n"], "m": rows[0]["m"], "wedges": W,
                   "triangles": tri, "s": args.s, "a": args.a,
                   "kernel_only_value": W * len(execs) / sum(execs),
                   "gpu_exec_s": statistics.mean(execs),
                   "gpu_copy_s": statistics.mean(r["copy"] for r in rows),
                   "prepro_s": rows[0]["prepro"], "process_wall_s": wall},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": (f"reference tc (sm_100a build) -s {args.s} -a {args.a} "
                                    f"-l {args.warmup + args.steps}, first {args.warmup} rows "
                                    "dropped: whole tc_GPU call (host bitmap and prefix, "
                                    "copies, kernel) per step; single-threaded host")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batch(args):
    """The uneven-batch workload: 4,096 seeded graphs (half Erdos-Renyi, half
    Chung-Lu), counted (a) batched -- resident, one persistent launch per
    size bucket per sub-batch, CUDA-graph replay -- and (b) by plain
    per-graph calls on a sample of the same graphs. Reports graphs/s of
    both; every sampled count must agree."""
    import torch

    import wetric
    from wetric import workloads as Wl

    dev = 0
    torch.cuda.set_device(dev)
    specs = Wl.mixed_batch(args.batch_graphs, seed=1000)

    def bucket_of(sp):
        kind = "er" if isinstance(sp, Wl.ErdosRenyiSpec) else "chunglu"
        dec = min(5, max(3, int(np.floor(np.log10(max(sp.n, 1))))))
        return f"{kind}-n1e{dec}"

    # Sub-batches sized to the device (pairs + union copy + sort buffers),
    # each within one size/family bucket, so every bucket's batched time is
    # measured on its own.
    cap = int(args.sub_batch_pairs)
    by_bucket = {}
    for i, sp in enumerate(specs):
        by_bucket.setdefault(bucket_of(sp), []).append(i)
    groups, group_bucket = [], []
    for bk in sorted(by_bucket):
        cur, cur_p, cur_n = [], 0, 0
        for i in by_bucket[bk]:
            sp = specs[i]
            if cur and (cur_p + sp.draws > cap or cur_n + sp.n >= (1 << 31)):
                groups.append(cur)
                group_bucket.append(bk)
                cur, cur_p, cur_n = [], 0, 0
            cur.append(i)
            cur_p += sp.draws
            cur_n += sp.n
        if cur:
            groups.append(cur)
            group_bucket.append(bk)
    t0 = time.perf_counter()
    batches = []
    for grp in groups:
        src, dst, off, n = Wl.batch_pairs_device([specs[i] for i in grp], dev)
        batches.append(wetric.Batch(src, dst, off, n, device=dev, spread=args.batch_spread,
                                    a=args.a, autotune=not args.no_autotune,
                                    pair_streams=bool(args.pair_streams)))
        del src, dst
        torch.cuda.empty_cache()
    build_s = time.perf_counter() - t0
    # warm-up (captures the CUDA graphs) and reference counts
    counts = np.zeros(len(specs), np.uint64)
    W = Wpair = Kpair = 0
    for grp, b in zip(groups, batches):
        c, st = b.count()
        counts[grp] = c
        W += st.wedges
        Wpair += st.pair_wedges
        Kpair += st.pair_rows
    torch.cuda.synchronize()
    times, launches = [], 0
    per_group = [[] for _ in batches]
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for gi, b in enumerate(batches):
            t1 = time.perf_counter()
            _, st = b.count()
            per_group[gi].append(time.perf_counter() - t1)
            launches += st.launches
        times.append(time.perf_counter() - t0)
    batched_s = statistics.median(times)
    # plain per-graph calls on every k-th graph (every graph by default)
    sample = list(range(0, len(specs), args.plain_every))
    lat = []
    lat_of = {}
    plain_ok = True
    for i in sample:
        sp = specs[i]
        s_, d_, n_ = Wl.device_pairs(sp, dev)
        og = wetric.orient_edges(s_, d_, n=n_, device=dev)
        del s_, d_
        og.count(5, args.a, device=dev, pair_streams=bool(args.pair_streams))  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c, _ = og.count(5, args.a, device=dev, pair_streams=bool(args.pair_streams))
        lat.append(time.perf_counter() - t0)
        lat_of[i] = lat[-1]
        plain_ok &= int(c) == int(counts[i])
        og.free()
    plain_gps = len(sample) / sum(lat)
    batched_gps = len(specs) / batched_s
    # Per size/family bucket: graphs, wedges, the bucket's batched time
    # (its sub-batches' median count times) and its plain per-graph time
    # (summed over the sampled graphs, scaled to the bucket).
    wedges_of = np.zeros(len(specs), np.uint64)
    for grp, b in zip(groups, batches):
        wedges_of[grp] = b.info()[0]
    buckets = {}
    for gi, (grp, bk) in enumerate(zip(groups, group_bucket)):
        e = buckets.setdefault(bk, {"graphs": 0, "wedges": 0, "batched_s": 0.0,
                                    "plain_s": 0.0, "plain_sampled": 0})
        e["graphs"] += len(grp)
        e["wedges"] += int(wedges_of[grp].sum())
        e["batched_s"] += statistics.median(per_group[gi])
        for i in grp:
            if i in lat_of:
                e["plain_s"] += lat_of[i]
                e["plain_sampled"] += 1
    for e in buckets.values():
        if e["plain_sampled"]:
            e["plain_s"] *= e["graphs"] / e["plain_sampled"]
        e["batched_vs_plain"] = e["plain_s"] / e["batched_s"] if e["batched_s"] else None
        e["batched_wedges_per_s"] = e["wedges"] / e["batched_s"] if e["batched_s"] else None
    line = {
        "metric": f"graphs/s (exact per-graph triangle counts, {len(specs):,}-graph uneven batch)",
        "value": batched_gps, "unit": "graphs/s", "n_gpus": 1, "steps": args.steps,
        "warmup": 1, "ms_per_step": batched_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 ids, u64 counts (integer)",
        "data": "synthetic (seeded ER + Chung-Lu, generated on device)",
        "config": {"workload": f"mixed-batch-{len(specs)}", "graphs": len(specs),
                   "sub_batches": len(batches), "wedges": int(W),
                   "edges_drawn": int(sum(sp.draws for sp in specs)),
                   "batch_build_s": build_s,
                   "spread": args.batch_spread or ("size table" if args.no_autotune
                                                   else "autotuned per size/skew bucket"),
                   "spreads_used": {int(k): int(v) for k, v in zip(*np.unique(
                       np.concatenate([b.spreads() for b in batches]), return_counts=True))},
                   "a": args.a, "plain_sample": len(sample),
                   "plain_graphs_per_s": plain_gps,
                   "plain_p50_ms": 1e3 * float(np.percentile(lat, 50)),
                   "plain_p99_ms": 1e3 * float(np.percentile(lat, 99)),
                   "batched_vs_plain": batched_gps / plain_gps,
                   "counts_agree": bool(plain_ok),
                   "counts_compared": len(sample),
                   "wedges_per_s": W / batched_s,
                   "pair_streams": bool(args.pair_streams),
                   "pair_rows": int(Kpair), "pair_wedges": int(Wpair),
                   "buckets": buckets},
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    for b in batches:
        b.free()


def run_serve(args):
    """Serving: Poisson arrivals at args.rate graphs/s for args.duration s,
    95% drawn from the uneven-batch mixture and 5% R-MAT scale 20-23 (edge
    factor 16), served (a) by the continuous-batching server under a 150 GB
    HBM admission cap and (b) by plain per-request calls (one worker,
    preprocess + count per request, FIFO). Reports graphs/s and p50/p99
    submit-to-result latency of both; every served count must equal the
    graph's count alone."""
    import queue
    import threading

    import torch

    import wetric
    from wetric import workloads as Wl

    dev = 0
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(7)
    mix = Wl.mixed_batch(args.serve_pool, seed=5000)
    rmats = [Wl.RmatSpec(scale=int(sc), edge_factor=16, seed=9000 + i)
             for i, sc in enumerate(rng.integers(20, 24, size=max(2, args.serve_pool // 20)))]
    pool = []
    for sp in mix + rmats:
        s_, d_, n_ = Wl.device_pairs(sp, dev)
        og = wetric.orient_edges(s_, d_, n=n_, device=dev)
        alone, _ = og.count(5, args.a, device=dev)
        og.free()
        pool.append((s_, d_, n_, int(alone), isinstance(sp, Wl.RmatSpec)))
    torch.cuda.synchronize()
    n_req = int(args.rate * args.duration)
    gaps = rng.exponential(1.0 / args.rate, size=n_req)
    arrivals = np.cumsum(gaps)
    pick_r = rng.random(n_req) < args.rmat_fraction
    mix_idx = rng.integers(0, len(mix), size=n_req)
    rm_idx = len(mix) + rng.integers(0, len(rmats), size=n_req)
    choice = np.where(pick_r, rm_idx, mix_idx)

    def drive(submit, finish):
        t0 = time.perf_counter()
        handles = []
        for k in range(n_req):
            delay = arrivals[k] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            handles.append(submit(choice[k], time.perf_counter()))
        results = [finish(h) for h in handles]
        wall = time.perf_counter() - t0
        return results, wall

    # (a) continuous batching server
    srv = wetric.Server(device=dev, hbm_budget=150 << 30, spread=5, a=args.a,
                        max_batch_graphs=4096, large_pairs=args.large_pairs,
                        resident=bool(args.serve_resident))

    def srv_submit(i, _t):
        s_, d_, n_, want, _ = pool[i]
        return srv.submit(s_, d_, n_), i

    def srv_finish(h):
        t, i = h
        try:
            c, lat = srv.wait(t, timeout_ms=120000)
        except wetric.WetricError:
            # the server's queue state for the record, then fail the run
            print(json.dumps({"ticket": t, "pool_index": int(i),
                              "pairs": int(pool[i][0].numel()), "server": srv.stats()}),
                  file=sys.stderr, flush=True)
            raise
        return c == pool[i][3], lat

    res_b, wall_b = drive(srv_submit, srv_finish)
    st = srv.stats()
    srv.close()

    # (b) plain per-request calls
    q = queue.Queue()
    done = {}

    def worker():
        while True:
            item = q.get()
            if item is None:
                return
            key, i, t_arr = item
            s_, d_, n_, want, _ = pool[i]
            og = wetric.orient_edges(s_, d_, n=n_, device=dev)
            c, _ = og.count(5, args.a, device=dev)
            og.free()
            done[key] = (c == want, 1e3 * (time.perf_counter() - t_arr))

    th = threading.Thread(target=worker)
    th.start()
    keys = iter(range(n_req))

    def plain_submit(i, t_arr):
        key = next(keys)
        q.put((key, i, t_arr))
        return key

    def plain_finish(key):
        while key not in done:
            time.sleep(0.0005)
        return done[key]

    res_p, wall_p = drive(plain_submit, plain_finish)
    q.put(None)
    th.join()

    lat_b = np.array([r[1] for r in res_b])
    lat_p = np.array([r[1] for r in res_p])
    if args.serve_trace:
        # one row per request: arrival s, input pairs, server ms, plain ms
        with open(args.serve_trace, "w") as f:
            f.write("arrival_s,pairs,server_ms,plain_ms\n")
            for k in range(n_req):
                f.write(f"{arrivals[k]:.6f},{pool[choice[k]][0].numel()},"
                        f"{lat_b[k]:.3f},{lat_p[k]:.3f}\n")
    ok = all(r[0] for r in res_b) and all(r[0] for r in res_p)
    line = {
        "metric": "graphs/s served (Poisson arrivals, exact counts)",
        "value": n_req / wall_b, "unit": "graphs/s", "n_gpus": 1, "steps": n_req,
        "warmup": 0, "ms_per_step": 1e3 * wall_b / n_req, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 ids, u64 counts (integer)",
        "data": "synthetic (seeded ER / Chung-Lu / R-MAT pool, generated on device)",
        "config": {"workload": f"serve-poisson-{args.rate:g}-per-s", "requests": n_req,
                   "offered_rate": args.rate, "pool_graphs": len(pool),
                   "rmat_fraction": float(pick_r.mean()), "hbm_budget_gb": 150,
                   "p50_ms": float(np.percentile(lat_b, 50)),
                   "p99_ms": float(np.percentile(lat_b, 99)),
                   "batches": st["batches"], "mean_batch_graphs": st["mean_batch_graphs"],
                   "server_admit_busy_s": st["admit_busy_ms"] / 1e3,
                   "server_count_busy_s": st["count_busy_ms"] / 1e3,
                   "large_pairs": args.large_pairs,
                   "queue_p50_ms": st["queue_p50_ms"],
                   "small_lane_p50_ms": st["small_p50_ms"],
                   "small_lane_p99_ms": st["small_p99_ms"],
                   "large_lane_p50_ms": st["large_p50_ms"],
                   "large_lane_p99_ms": st["large_p99_ms"],
                   "large_lane_requests": st["large_completed"],
                   "resident": bool(args.serve_resident),
                   "resident_launches": st["resident_launches"],
                   "recycles": st["recycles"],
                   "wall_s": wall_b,
                   "plain_graphs_per_s": n_req / wall_p,
                   "plain_p50_ms": float(np.percentile(lat_p, 50)),
                   "plain_p99_ms": float(np.percentile(lat_p, 99)),
                   "counts_equal_alone": bool(ok)},
    }
    print(json.dumps(line), flush=True)


def _sample_ranges(row_ptr, budget):
    """Three vertex ranges of an oriented CSR whose merge counts cost about
    `budget` element steps each: one ending at the last (highest-degree)
    vertex, one around the middle of the wedge mass and one low in it.
    Work of v = sum over w in N+(v) of (d+(v) + d+(w)), estimated with the
    mean d+(w) of v's rows as d+(v) (the hubs' out-neighbours are hubs)."""
    d = np.diff(row_ptr.astype(np.int64))
    wedges = d * (d - 1) // 2
    cum = np.cumsum(wedges)
    W = int(cum[-1])
    work = 2 * d * d
    n = len(d)
    out = []
    cw = np.cumsum(work)
    rev = np.cumsum(work[::-1])
    for kind, anchor in (("top", n), ("middle", int(np.searchsorted(cum, W // 2))),
                         ("low", int(np.searchsorted(cum, W // 10)))):
        if kind == "top":
            ve = n
            vb = max(0, n - 1 - int(np.searchsorted(rev, budget)))
        else:
            vb = min(anchor, n - 1)
            base = int(cw[vb - 1]) if vb > 0 else 0
            ve = min(n, int(np.searchsorted(cw, base + budget)) + 1)
        wb = int(cum[vb - 1]) if vb > 0 else 0
        we = int(cum[ve - 1]) if ve > 0 else 0
        out.append((kind, vb, ve, wb, we))
    return out, W, int(d.max())


def run_big(args):
    """The m > 2^32 case: R-MAT scale 27, edge factor 40 (5.37e9 draws),
    generated and preprocessed entirely on the device (u64 offsets and
    wedge indices), counted exactly. The count is pinned three ways: (1)
    size-independent properties -- equal under another (s, a), with and
    without the dense core, and equal to the sum of five wedge-range
    counts; (2) the oriented CSR, downloaded to the host, passes the
    device validation (rows sorted, columns above the row and below n), has
    non-decreasing total degree along the ids (the degree order) and the
    same W and max out-degree on the host; (3) on three vertex ranges (the
    top hubs, the middle and the low end of the wedge mass) the GPU's count
    of the ranges' wedges equals the oracle's merge-intersection count of
    the same vertices on the downloaded CSR, bit for bit."""
    import torch

    import wetric
    from wetric import workloads as Wl

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    dev = 0
    torch.cuda.set_device(dev)
    spec = Wl.RmatSpec(scale=args.big_scale, edge_factor=args.big_edge_factor, seed=1)
    t0 = time.perf_counter()
    src, dst, _ = Wl.device_pairs(spec, dev)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    og = wetric.orient_edges(src, dst, device=dev)
    prep_ms = og.stats.prep_ms
    del src, dst
    torch.cuda.empty_cache()
    c0, st = og.count(args.s, args.a, device=dev, core_len=args.core_len)
    W = st.wedges
    times, core_ms = [], []
    for _ in range(args.steps):
        c, st = og.count(args.s, args.a, device=dev, core_len=args.core_len)
        assert c == c0
        times.append(st.count_ms)
        core_ms.append(st.core_ms)
    c_alt, _ = og.count(10, 16384, device=dev)
    c_nocore, st_nc = og.count(args.s, args.a, device=dev, core_len=wetric.CORE_OFF)
    c_valid, _ = og.count(args.s, args.a, device=dev, validate=True)
    parts = [og.count(args.s, args.a, device=dev, wedge_begin=W * i // 5,
                      wedge_end=W * (i + 1) // 5)[0] for i in range(5)]
    ms = statistics.median(times)
    checks = {}
    if args.big_host_checks:
        t1 = time.perf_counter()
        host = og.download()
        rp, ci = host.row_ptr, host.col_ind
        d_minus = torch.zeros(og.n, dtype=torch.int64, device=f"cuda:{dev}")
        step = 1 << 28
        for j in range(0, og.m, step):
            blk = torch.from_numpy(ci[j:j + step].view(np.int32)).to(f"cuda:{dev}")
            d_minus += torch.bincount(blk, minlength=og.n)
        d_plus = torch.from_numpy(np.diff(rp.astype(np.int64))).to(f"cuda:{dev}")
        deg = d_plus + d_minus
        degree_order = bool((deg[1:] >= deg[:-1]).all().item())
        ranges, W_host, maxd_host = _sample_ranges(rp, args.big_sample_work)
        g = oracle.CSR(rp, ci)
        samples = []
        for kind, vb, ve, wb, we in ranges:
            gpu, _ = og.count(args.s, args.a, device=dev, wedge_begin=wb, wedge_end=we)
            t2 = time.perf_counter()
            cpu = oracle.count_merge_range(g, vb, ve)
            samples.append({"range": kind, "vbegin": vb, "vend": ve, "wedge_begin": wb,
                            "wedge_end": we, "gpu": int(gpu), "oracle": int(cpu),
                            "oracle_s": time.perf_counter() - t2})
        checks = {"host_check_s": time.perf_counter() - t1,
                  "row_ptr_ends": [int(rp[0]), int(rp[-1])],
                  "W_host": W_host, "max_out_degree_host": maxd_host,
                  "degree_order_nondecreasing": degree_order,
                  "sample_checks": samples,
                  "samples_equal": all(x["gpu"] == x["oracle"] for x in samples),
                  "oracle_threads": oracle.max_threads()}
        del host, rp, ci, g
    line = {
        "metric": "wedges/s (exact triangle count, R-MAT s27 ef40, m > 2^32)",
        "value": W / (ms / 1e3), "unit": "wedges/s", "n_gpus": 1, "steps": args.steps,
        "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u32 ids, u64 offsets and counts (integer)",
        "data": "synthetic (seeded R-MAT generated on device)",
        "config": {"workload": spec.name, "n": og.n, "m": og.m, "m_over_2^32": og.m > (1 << 32),
                   "wedges": W, "triangles": c0, "max_out_degree": st.max_out_degree,
                   "s": args.s, "a": args.a, "generate_s": gen_s, "device_prep_ms": prep_ms,
                   "core_len": st.core_len, "core_wedges": st.core_wedges,
                   "core_kernel_ms": statistics.median(core_ms),
                   "count_no_core": c_nocore, "count_ms_no_core": st_nc.count_ms,
                   "count_alt_s10_a16384": c_alt, "count_validated": c_valid,
                   "range_sum": int(sum(parts)),
                   "invariants_hold": bool(c_alt == c0 and sum(parts) == c0
                                           and c_nocore == c0 and c_valid == c0),
                   **checks},
    }
    if checks:
        line["config"]["pinned"] = bool(
            line["config"]["invariants_hold"] and checks["samples_equal"]
            and checks["degree_order_nondecreasing"] and checks["W_host"] == W
            and checks["max_out_degree_host"] == st.max_out_degree
            and checks["row_ptr_ends"] == [0, og.m])
    print(json.dumps(line), flush=True)
    og.free()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--s", type=int, default=5)
    ap.add_argument("--a", type=int, default=8192)
    ap.add_argument("--kernel", type=int, default=0,
                    help="count kernel (wetric_opts.kernel): 0 default (8), 1 block-tile, "
                         "2 warp-staged, 3-5 row-walk variants, 6 row-walk with hash "
                         "sets, 7 long-row segments with hash sets, 8 = 7 with 16-bit "
                         "near sets")
    ap.add_argument("--core-len", type=int, default=0,
                    help="dense core vertices (wetric_opts.core_len): 0 = chosen by the "
                         "library, -1 = none")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="rmat-s22",
                    choices=["rmat-s22", "rmat-s22-sweep", "rmat-s22-core", "rmat-s27", "batch",
                             "serve"],
                    help="rmat-s22: the headline single-graph count; rmat-s22-sweep: "
                         "s x a sweep of the same graph (both impls); batch: the "
                         "4,096-graph uneven batch, batched vs plain calls; serve: "
                         "Poisson arrivals, continuous batching vs plain calls; "
                         "rmat-s22-core: dense core / shell lengths on the same graph; "
                         "rmat-s27: the m > 2^32 graph")
    ap.add_argument("--big-scale", type=int, default=27)
    ap.add_argument("--big-edge-factor", type=int, default=40)
    ap.add_argument("--big-host-checks", type=int, default=1,
                    help="rmat-s27: download the CSR and check it on the host "
                         "(about 22 GB of host memory at scale 27)")
    ap.add_argument("--big-sample-work", type=float, default=4e9,
                    help="rmat-s27: merge steps per sampled vertex range")
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--duration", type=float, default=15.0)
    ap.add_argument("--serve-pool", type=int, default=240)
    ap.add_argument("--serve-trace", default="",
                    help="serve: write per-request arrival, size and latencies (CSV)")
    ap.add_argument("--rmat-fraction", type=float, default=0.05,
                    help="serve: share of requests drawn from R-MAT scale 20-23")
    ap.add_argument("--large-pairs", type=int, default=8 << 20,
                    help="serve: requests with at least this many pairs use the "
                         "server's large lane (0 = one lane)")
    ap.add_argument("--serve-resident", type=int, default=0,
                    help="serve: 0 = per-lane launches (the library default), 1 = the "
                         "resident counting kernel")
    ap.add_argument("--batch-graphs", type=int, default=4096)
    ap.add_argument("--batch-spread", type=int, default=0, help="0 = tuned per graph")
    ap.add_argument("--no-autotune", action="store_true",
                    help="batch: spread from the size table instead of the autotuner")
    ap.add_argument("--sub-batch-pairs", type=float, default=1.2e9)
    ap.add_argument("--pair-streams", type=int, default=1,
                    help="1 = pair streams for short rows (the library default), 0 = off")
    ap.add_argument("--plain-every", type=int, default=1,
                    help="batch: plain per-graph calls on every k-th graph (1 = all)")
    args = ap.parse_args()
    if args.core_len < 0:
        args.core_len = 0xFFFFFFFF
    if args.workload == "rmat-s22-sweep":
        run_sweep(args)
    elif args.workload == "rmat-s22-core":
        run_core_sweep(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "rmat-s27":
        run_big(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
