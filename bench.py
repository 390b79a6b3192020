"""Benchmark: multilevel k-way partitioning of a 2D Delaunay graph of 2^20
points at k = 64, eps = 0.03 (unit weights, int32 CSR), on B200.

One step = one full partition (coarsening, device initial partition,
uncoarsening with refinement, exact cut) of the graph.

  value   edges/s = undirected edges / device time of the partition, input CSR
          resident in HBM, output part left in HBM (CUDA events on the
          library's stream; L2 flushed between steps; max over ranks).
  e2e     the same metric through the host API gkw_partition: pinned host CSR
          in, host part out, host<->device copies inside the timed region.

--impl reference times the reference algorithm on the host cores instead: the
oracle (a C++ restatement of G-kway, with the reference's bundled METIS as the
initial partitioner, as the reference does), one process per core, each
partitioning the same graph.

Multi-GPU (--gpus N under torchrun): one independent partition per rank (the
path does not shard within a graph), weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 1 << 20
K = 64
EPS = 0.03
SEED = 1
METRIC = "edges/s partitioned (Delaunay 2^20, k=64)"
CACHE_DIR = "/tmp/gkway_bench_cache"


def load_graph():
    import __graft_entry__ as ge
    gen = ge.load_generators()
    path = os.path.join(CACHE_DIR, f"delaunay_{N_POINTS}_s{SEED}.npz")
    if os.path.exists(path):
        d = np.load(path)
        return gen.Csr(d["xadj"], d["adjncy"], d["adjwgt"], d["vwgt"])
    g = gen.delaunay(N_POINTS, SEED)
    os.makedirs(CACHE_DIR, exist_ok=True)
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, xadj=g.xadj, adjncy=g.adjncy, adjwgt=g.adjwgt, vwgt=g.vwgt)
    os.replace(tmp, path)
    return g


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of this GPU, sampled by a
    background thread every few milliseconds while the timed region runs.
    NVML (the library nvidia-smi reads) is used directly so that short timed
    regions still get many samples; nvidia-smi is the fallback."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device_index: int, period_s: float = 0.005):
        self.dev = device_index
        self.period = period_s
        self.rows = []           # (sm_mhz, max_mhz, reason bits)
        self.stop_evt = threading.Event()
        self.mode = None
        self.proc = None
        self.t = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            idx = int(vis.split(",")[self.dev]) if vis and vis.split(",")[self.dev].isdigit() else self.dev
            return pynvml.nvmlDeviceGetHandleByIndex(idx)

    def start(self):
        try:
            import pynvml
            hnd = self._nvml_handle()
            mx = pynvml.nvmlDeviceGetMaxClockInfo(hnd, pynvml.NVML_CLOCK_SM)

            def run():
                while not self.stop_evt.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(hnd, pynvml.NVML_CLOCK_SM)
                        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(hnd)
                        self.rows.append((float(sm), float(mx), int(rs)))
                    except Exception:
                        pass
                    self.stop_evt.wait(self.period)

            self.mode = "nvml"
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
            return
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)

            def read():
                for line in self.proc.stdout:
                    r = [x.strip() for x in line.split(",")]
                    if len(r) < 9 or not r[1].replace(".", "").isdigit():
                        continue
                    bits = 0
                    for i, (_, bit) in enumerate(self.REASONS[:4]):
                        if r[5 + i].lower().startswith("active"):
                            bits |= bit
                    self.rows.append((float(r[1]), float(r[2]), bits))

            self.mode = "nvidia-smi"
            self.t = threading.Thread(target=read, daemon=True)
            self.t.start()
        except Exception:
            self.mode = None

    def stop(self) -> dict:
        if self.mode is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        self.stop_evt.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        self.t.join(timeout=2)
        rows = list(self.rows)
        reasons = sorted({nm for _, _, bits in rows for nm, bit in self.REASONS if bits & bit})
        return {"sm_mhz": statistics.median(r[0] for r in rows) if rows else None,
                "sm_max_mhz": max(r[1] for r in rows) if rows else None,
                "reasons": reasons, "samples": len(rows), "source": self.mode}


def metis_cpu_baseline(g, budget_s: float = 12.0) -> dict:
    """The reference's bundled METIS k-way on one host core, whole graph."""
    import oracle
    if not oracle.has_metis():
        return None
    oracle.metis_kway(g, K)   # warm
    times = []
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end or not times:
        t0 = time.perf_counter()
        _, cut = oracle.metis_kway(g, K)
        times.append(time.perf_counter() - t0)
        if len(times) >= 10:
            break
    t = statistics.median(times)
    return {"value": g.n_edges / t, "unit": "edges/s", "cores": 1, "kind": "reference",
            "sample": f"METIS_PartGraphKway (bundled METIS 5.2.1) on the full graph, k={K}, "
                      f"{len(times)} runs, median {t:.3f}s, cut {cut}",
            "cut": int(cut)}


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The largest x over all ranks: the whole job's step time is that of its
    slowest replica."""
    import torch
    if world <= 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def bench_ours(args):
    import torch
    import __graft_entry__ as ge

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    pkg = ge.load_package()
    g = load_graph()
    h = pkg.Handle(dev.index)
    stream = torch.cuda.ExternalStream(h.stream, device=dev)
    xadj, adjncy, adjwgt, vwgt = (torch.from_numpy(a).to(dev) for a in (g.xadj, g.adjncy, g.adjwgt, g.vwgt))
    part = torch.empty(g.n, dtype=torch.int32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)   # 512 MB > 126 MB L2
    opts = pkg.default_options(eps=EPS, seed=SEED)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # launch shapes for this graph (gkw_autotune: timed candidates; results never depend on them)
    tuning = None if args.no_tune else h.autotune(xadj, adjncy, adjwgt, vwgt, K, opts)
    # warm-up
    for _ in range(args.warmup):
        h.partition_device(xadj, adjncy, adjwgt, vwgt, K, part, opts)
    torch.cuda.synchronize()

    # ---- timed: device-resident ----
    sampler = ClockSampler(dev.index) if rank == 0 else None
    if sampler:
        sampler.start()
    barrier()
    step_ms = []
    launches = 0
    cut = None
    st = None
    steps_stats = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        l0 = pkg.launch_count()
        cut, st = h.partition_device(xadj, adjncy, adjwgt, vwgt, K, part, opts)
        launches += pkg.launch_count() - l0
        steps_stats.append(st)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    barrier()
    clocks = sampler.stop() if sampler else None
    ms = sum(step_ms) / len(step_ms)
    ms_max = max_over_ranks(ms, world, dev)

    if args.device_only:
        roof, phase_roof = roofline_report(steps_stats)
        h.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": world * g.n_edges / (ms_max / 1e3), "unit": "edges/s",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                              "device_only": True, "gpu_launches": int(launches), "roofline": roof,
                              "phase_roofline": phase_roof, "cut": int(cut),
                              "phase_ms": {"coarsen": st["ms_coarsen"], "init": st["ms_init"],
                                           "refine": st["ms_refine"], "total": st["ms_total"]},
                              "clocks": clocks}))
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    # ---- e2e: host API, pinned host buffers, copies inside ----
    hx, ha, hw, hv = (torch.from_numpy(a).pin_memory() for a in (g.xadj, g.adjncy, g.adjwgt, g.vwgt))
    hpart = torch.empty(g.n, dtype=torch.int32).pin_memory()
    opts_e = pkg.default_options(eps=EPS, seed=SEED)
    h.partition(hx.numpy(), ha.numpy(), hw.numpy(), hv.numpy(), K, opts_e, part_out=hpart.numpy())
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, cut_e, _ = h.partition(hx.numpy(), ha.numpy(), hw.numpy(), hv.numpy(), K, opts_e, part_out=hpart.numpy())
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    barrier()
    e2e = sum(e2e_ms) / len(e2e_ms)
    e2e_max = max_over_ranks(e2e, world, dev)
    assert int(cut_e) == int(cut), "host and device paths disagree"

    # ---- roofline of the dominant kernel, from the timed steps ----
    roof, phase_roof = roofline_report(steps_stats)
    h.close()

    # ---- the batched and served forms (one GPU, rank 0 of a lone run) ----
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        del xadj, adjncy, adjwgt, vwgt, flush
        torch.cuda.empty_cache()
        for name, fn in (("batched", batched_summary), ("served", served_summary)):
            try:
                extras[name] = fn(args)
            except Exception as e:   # reported in the line, not fatal to the headline
                extras[name] = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        part_np = part.cpu().numpy()
        pw = np.bincount(part_np, weights=g.vwgt, minlength=K)
        W = int(g.vwgt.sum())
        cpu = metis_cpu_baseline(g) if world == 1 else None
        line = {
            "metric": METRIC, "value": world * g.n_edges / (ms_max / 1e3), "unit": "edges/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded 2D Delaunay of uniform points, unit weights)",
            "config": {"workload": f"2D Delaunay 2^20 points (n={g.n}, |E|={g.n_edges}), k={K}, eps={EPS}",
                       "n": g.n, "edges": g.n_edges, "k": K, "eps": EPS, "seed": SEED,
                       "parallelism": f"replicas x{world}", "l2": "flushed between steps (512 MB write)"},
            "e2e": {"value": world * g.n_edges / (e2e_max / 1e3), "unit": "edges/s", "ms_per_step": e2e_max,
                    "h2d_bytes_per_step": int(4 * (g.n + 1) + 8 * g.m + 4 * g.n),
                    "d2h_bytes_per_step": int(4 * g.n)},
            "gpu_launches": int(launches),
            "roofline": roof,
            "phase_roofline": phase_roof,
            "cpu_baseline": cpu,
            "quality": {"cut": int(cut), "max_part_weight": int(pw.max()),
                        "balance": float(pw.max() * K / W), "maxw": st["maxw"] if st else None,
                        "levels": st["level_n"] if st else None,
                        "refine_rounds": st["refine_rounds"] if st else None},
            "phase_ms": {"coarsen": st["ms_coarsen"], "init": st["ms_init"], "refine": st["ms_refine"],
                         "total": st["ms_total"]} if st else None,
            "clocks": clocks,
            "tuning": tuning,
        }
        line.update(extras)
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def load_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    return 6650.0, "fallback 6.65 TB/s (of fallback)"


def level_kernel_launches(st):
    """(algorithmic bytes, device ms) of each level-kernel launch of one
    partition.  Per level of n vertices and m CSR entries (4-byte words, each
    compulsory array once): one full gain pass 4(n+1) + 8m + 4n + 8n, the
    projection from the coarser level 4n + 4n_c, and 8 bytes (adjncy, adjwgt)
    per adjacency entry the gain updates of the rounds read."""
    nl, ln, lm = st["n_levels"], st["level_n"], st["level_m"]
    out = []
    for i in range(nl):
        ms = st["ms_level"][i]
        if ms < 0:
            continue
        n, m = ln[i], lm[i]
        b = 4 * (n + 1) + 8 * m + 4 * n + 8 * n + 8 * st["round_entries"][i]
        if i + 1 < nl:
            b += 4 * n + 4 * ln[i + 1]
        out.append((i, b, ms))
    return out


def coarsen_bytes(st):
    """Algorithmic bytes of coarsening, summed over the kept levels: match
    4(n+1) + 8m + 4n, grouping 12n + 4n_c, contraction 4(n+1) + 8m + 8n +
    4(n_c+1) + 8m_c."""
    nl, ln, lm = st["n_levels"], st["level_n"], st["level_m"]
    tot = 0
    for i in range(nl - 1):
        n, m, nc, mc = ln[i], lm[i], ln[i + 1], lm[i + 1]
        tot += 4 * (n + 1) + 8 * m + 4 * n
        tot += 12 * n + 4 * nc
        tot += 4 * (n + 1) + 8 * m + 8 * n + 4 * (nc + 1) + 8 * mc
    return tot


def read_traffic(kernel_file):
    """DRAM bytes per launch from a committed ncu summary (a line
    'traffic_bytes_per_launch: N'), or None."""
    path = os.path.join(ROOT, "profiles", kernel_file)
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        return None
    return None


def roofline_report(steps_stats):
    """Roofline of the dominant kernel (the level kernel: projection, balance
    and refinement rounds, one launch per level), from the CUDA events the
    library records around each of its launches in the timed steps."""
    peak, src = load_peak_gbs()
    launches = [x for st in steps_stats for x in level_kernel_launches(st)]
    tot_b = sum(b for _, b, _ in launches)
    tot_ms = sum(ms for _, _, ms in launches)
    nlaunch = max(len(launches), 1)
    achieved = tot_b / (tot_ms / 1e3) / 1e9 if tot_ms > 0 else 0.0
    roof = {"kernel": "k_level (one launch per level: projection, balance rounds, refinement rounds)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": read_traffic("k_level_delaunay2e20_k64.md"),
            "algorithmic_bytes_per_launch": tot_b / nlaunch, "ms_per_launch": tot_ms / nlaunch,
            "launches": len(launches), "peak_source": src,
            "timing": "CUDA events on the library stream around each launch, every timed step"}
    # phase fractions (coarsening, refinement) over the timed steps
    cb = sum(coarsen_bytes(st) for st in steps_stats)
    cms = sum(st["ms_coarsen"] for st in steps_stats)
    rb = sum(b for st in steps_stats for i, b, _ in level_kernel_launches(st) if i + 1 < st["n_levels"])
    rms = sum(st["ms_refine"] for st in steps_stats)
    phases = {"coarsen": {"bytes_per_step": cb / len(steps_stats), "ms_per_step": cms / len(steps_stats),
                          "frac": cb / (cms / 1e3) / 1e9 / peak if cms > 0 else None},
              "uncoarsen": {"bytes_per_step": rb / len(steps_stats), "ms_per_step": rms / len(steps_stats),
                            "frac": rb / (rms / 1e3) / 1e9 / peak if rms > 0 else None}}
    return roof, phases


# ---------------------------------------------------------------------------
# reference arm: the oracle (G-kway restated on the CPU, METIS initial
# partition) on every host core, one independent partition per process
# ---------------------------------------------------------------------------
def _ref_worker(conn, graph_path):
    import oracle
    import __graft_entry__ as ge
    gen = ge.load_generators()
    d = np.load(graph_path)
    g = gen.Csr(d["xadj"], d["adjncy"], d["adjwgt"], d["vwgt"])
    oracle.lib()
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg == "stop":
            break
        t0 = time.perf_counter()
        _, info = oracle.partition(g, K)
        conn.send((time.perf_counter() - t0, info["cut"]))


def bench_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    import oracle
    if not oracle.has_metis():
        print(json.dumps({"impl": "reference", "unavailable": "the reference's bundled METIS library is missing"}))
        return
    g = load_graph()
    path = os.path.join(CACHE_DIR, f"delaunay_{N_POINTS}_s{SEED}.npz")
    cores = len(os.sched_getaffinity(0))
    ctx = mp.get_context("spawn")
    pipes, procs = [], []
    for _ in range(cores):
        a, b = ctx.Pipe()
        p = ctx.Process(target=_ref_worker, args=(b, path), daemon=True)
        p.start()
        pipes.append(a)
        procs.append(p)
    for a in pipes:
        a.recv()

    def step():
        for a in pipes:
            a.send("go")
        res = [a.recv() for a in pipes]
        return max(r[0] for r in res), res[0][1]

    for _ in range(args.warmup):
        step()
    ts = []
    cut = None
    for _ in range(args.steps):
        t, cut = step()
        ts.append(t)
    for a in pipes:
        a.send("stop")
    for p in procs:
        p.join(timeout=10)
    s = sum(ts) / len(ts)
    value = cores * g.n_edges / s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded 2D Delaunay of uniform points, unit weights)",
        "config": {"workload": f"2D Delaunay 2^20 points (n={g.n}, |E|={g.n_edges}), k={K}, eps={EPS}",
                   "n": g.n, "edges": g.n_edges, "k": K, "eps": EPS, "seed": SEED,
                   "parallelism": f"{cores} host processes"},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": cores, "kind": "port",
                         "sample": f"oracle partition (G-kway restated in C++, METIS initial partition) of the "
                                   f"full graph on each of {cores} processes; cut {cut}"},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# batched and served forms (not the headline line): --workload batched|served
# ---------------------------------------------------------------------------
BATCH_KS = (2, 4, 8, 16, 32)


def _gen_one(spec):
    """One seeded graph of a mixed workload: (kind, n, seed) -> CSR arrays."""
    import __graft_entry__ as ge
    gen = ge.load_generators()
    kind, n, seed = spec
    if kind == 0:
        g = gen.delaunay(max(n, 4), seed)
    elif kind == 1:
        a = max(2, int(round(n ** (1.0 / 3.0))))
        g = gen.grid27(a, a, max(2, int(round(n / (a * a)))))
    else:
        g = gen.circuit(max(n, 64), seed=seed, levels=min(200, max(8, n // 200)), hub_max=max(16, min(10000, n // 10)))
    return g.xadj, g.adjncy, g.adjwgt, g.vwgt


def mixed_graphs(count, n_lo, n_hi, seed, tag):
    """``count`` seeded graphs, vertex counts log-uniform in [n_lo, n_hi],
    generator uniform over 2D Delaunay, near-cubic 27-point grid and the
    scaled circuit-like graph; cached under CACHE_DIR."""
    import multiprocessing as mp
    import __graft_entry__ as ge
    gen = ge.load_generators()
    path = os.path.join(CACHE_DIR, f"{tag}_{count}_{n_lo}_{n_hi}_s{seed}.npz")
    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(0, 3)), int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))), 1000 + i)
             for i in range(count)]
    if os.path.exists(path):
        with np.load(path) as d:   # each array read once
            X, A, Wt, V, gp, ep = d["x"], d["a"], d["w"], d["v"], d["gp"], d["ep"]
        return [gen.Csr(X[gp[i] + i:gp[i + 1] + i + 1], A[ep[i]:ep[i + 1]], Wt[ep[i]:ep[i + 1]],
                        V[gp[i]:gp[i + 1]]) for i in range(count)], specs
    with mp.get_context("spawn").Pool(max(1, min(32, os.cpu_count() or 1))) as pool:
        arrs = pool.map(_gen_one, [(k, n, sd) for k, n, sd in specs], chunksize=4)
    graphs = [gen.Csr(*a) for a in arrs]
    os.makedirs(CACHE_DIR, exist_ok=True)
    gp = np.zeros(count + 1, np.int64)
    ep = np.zeros(count + 1, np.int64)
    gp[1:] = np.cumsum([g.n for g in graphs])
    ep[1:] = np.cumsum([g.m for g in graphs])
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, x=np.concatenate([g.xadj for g in graphs]), a=np.concatenate([g.adjncy for g in graphs]),
             w=np.concatenate([g.adjwgt for g in graphs]), v=np.concatenate([g.vwgt for g in graphs]), gp=gp, ep=ep)
    os.replace(tmp, path)
    return graphs, specs


def batched_summary(args, sample_clocks=True):
    """Config: many independent small graphs in one call (gkw_partition_batch)
    against the plain path partitioning them one after another on the same
    GPU.  Both sides go host arrays -> host parts; wall-clock time.  Returns
    the result object (clocks sampled over both timed parts)."""
    import torch
    import __graft_entry__ as ge
    torch.cuda.set_device(0)
    pkg = ge.load_package()
    count = args.graphs
    graphs, specs = mixed_graphs(count, 1000, 64000, 7, "batch")
    rng = np.random.default_rng(11)
    ks = [int(rng.choice(BATCH_KS)) for _ in graphs]
    x, a, w, vw, gp = pkg.concat_graphs(graphs)
    edges = int(sum(g.n_edges for g in graphs))
    # plain path: one handle, one graph after another
    h = pkg.Handle(0)
    for g, k in list(zip(graphs, ks))[:8]:
        h.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
    torch.cuda.synchronize()
    sampler = ClockSampler(0) if sample_clocks else None
    if sampler:
        sampler.start()
    t0 = time.perf_counter()
    plain = [h.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k) for g, k in zip(graphs, ks)]
    t_plain = time.perf_counter() - t0
    h.close()
    srv = pkg.Server(0, slots=args.slots)
    srv.partition_batch(x[: gp[8] + 1], a[: x[gp[8]]], w[: x[gp[8]]], vw[: gp[8]], gp[:9], ks[:8])   # warm
    times = []
    part = cuts = None
    for _ in range(max(1, min(args.steps, 5))):
        t0 = time.perf_counter()
        part, cuts, sts = srv.partition_batch(x, a, w, vw, gp, ks)
        times.append(time.perf_counter() - t0)
    clocks = sampler.stop() if sampler else None
    srv.close()
    same = all(np.array_equal(part[gp[i]:gp[i + 1]], plain[i][0]) and int(cuts[i]) == plain[i][1]
               for i in range(count))
    t_b = statistics.median(times)
    return {
        "workload": "batched", "metric": "graphs/s partitioned (batched form)", "value": count / t_b,
        "unit": "graphs/s", "edges_per_s": edges / t_b, "plain_graphs_per_s": count / t_plain,
        "plain_edges_per_s": edges / t_plain, "speedup_vs_plain": t_plain / t_b, "identical_to_plain": bool(same),
        "slots": args.slots, "steps": len(times), "timing": "wall clock, host arrays in, host parts out",
        "config": {"graphs": count, "n": "log-uniform 1k-64k", "generators": "Delaunay / 27-point grid / circuit",
                   "k": list(BATCH_KS), "eps": EPS, "vertices": int(gp[-1]), "edges": edges},
        "clocks": clocks}


def bench_batched(args):
    print(json.dumps(batched_summary(args)))


def served_summary(args, sample_clocks=True):
    """Config: open-loop Poisson requests of mixed sizes at a sweep of offered
    loads, through the server (continuous batching) and through the plain
    path (one handle serving requests first come, first served).  Returns the
    result object (clocks sampled over every load)."""
    import threading
    import torch
    import __graft_entry__ as ge
    torch.cuda.set_device(0)
    pkg = ge.load_package()
    pool, _ = mixed_graphs(args.pool, 1000, args.max_n, 5, "served")
    rng = np.random.default_rng(3)
    ks_all = [2 ** int(rng.integers(1, 9)) for _ in range(4096)]
    out = []
    sampler = ClockSampler(0) if sample_clocks else None
    if sampler:
        sampler.start()
    for rate in [float(r) for r in args.rates.split(",")]:
        nreq = int(max(20, min(args.requests, rate * args.duration)))
        arr = np.cumsum(rng.exponential(1.0 / rate, nreq))
        which = rng.integers(0, len(pool), nreq)
        ks = [ks_all[i % len(ks_all)] for i in range(nreq)]
        res = {"offered_per_s": rate, "requests": nreq}
        for mode in ("served", "plain"):
            lat = [0.0] * nreq
            done_t = [0.0] * nreq
            together = [1] * nreq
            if mode == "served":
                srv = pkg.Server(0, slots=args.slots)
                tickets = [None] * nreq
                t0 = time.perf_counter()

                def submit():
                    for i in range(nreq):
                        d = t0 + arr[i] - time.perf_counter()
                        if d > 0:
                            time.sleep(d)
                        g = pool[which[i]]
                        tickets[i] = srv.submit(g.xadj, g.adjncy, g.adjwgt, g.vwgt, ks[i])

                th = threading.Thread(target=submit)
                th.start()
                for i in range(nreq):
                    while tickets[i] is None:
                        time.sleep(0.0002)
                    r = srv.poll(tickets[i], pool[which[i]].n, wait_ms=-1)
                    lat[i] = r[2]["latency_ms"]
                    together[i] = r[2]["batch_graphs"]
                    done_t[i] = time.perf_counter()
                th.join()
                srv.close()
            else:
                h = pkg.Handle(0)
                t0 = time.perf_counter()
                for i in range(nreq):
                    d = t0 + arr[i] - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    g = pool[which[i]]
                    h.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, ks[i])
                    done_t[i] = time.perf_counter()
                    lat[i] = (done_t[i] - (t0 + arr[i])) * 1e3
                h.close()
            span = max(done_t) - t0
            res[mode] = {"graphs_per_s": nreq / span, "p50_ms": float(np.percentile(lat, 50)),
                         "p99_ms": float(np.percentile(lat, 99))}
            if mode == "served":   # graphs partitioned together with a request, on average
                res[mode]["mean_union_graphs"] = float(np.mean(together))
        out.append(res)
    clocks = sampler.stop() if sampler else None
    return {"workload": "served", "metric": "served graphs/s and p50/p99 latency vs plain",
            "unit": "graphs/s", "slots": args.slots, "loads": out,
            "config": {"pool_graphs": len(pool), "n": f"log-uniform 1k-{args.max_n}",
                       "k": "2..256 powers of two", "eps": EPS, "requests_per_load": f"<= {args.requests}",
                       "arrivals_s": args.duration, "timing": "wall clock, submit to result on the host"},
            "clocks": clocks}


def bench_served(args):
    print(json.dumps(served_summary(args)))


def bench_configs(args):
    """The other plain-method configurations at full size, each on one GPU:
    27-point grid 100x100x96 (k=64), road-like graph of 12M points and
    circuit-like graph of 4M vertices (k=256).  Device-resident timing with
    CUDA events (L2 flushed between steps), as for the headline line."""
    import torch
    import __graft_entry__ as ge
    torch.cuda.set_device(0)
    pkg = ge.load_package()
    gen = ge.load_generators()
    dev = torch.device("cuda", 0)
    cases = [("grid27 100x100x96", lambda: gen.grid27(100, 100, 96), 64),
             ("road 12M points", lambda: gen.road(12000000, 1), 256),
             ("circuit 4M vertices", lambda: gen.circuit(4000000, 1), 256)]
    if args.only:
        cases = [c for c in cases if c[0].startswith(args.only)]
    out = []
    for name, make, k in cases:
        path = os.path.join(CACHE_DIR, name.replace(" ", "_") + ".npz")
        if os.path.exists(path):
            with np.load(path) as d:
                g = gen.Csr(d["x"], d["a"], d["w"], d["v"])
        else:
            g = make()
            os.makedirs(CACHE_DIR, exist_ok=True)
            np.savez(path + ".tmp.npz", x=g.xadj, a=g.adjncy, w=g.adjwgt, v=g.vwgt)
            os.replace(path + ".tmp.npz", path)
        h = pkg.Handle(0)
        stream = torch.cuda.ExternalStream(h.stream, device=dev)
        t = [torch.from_numpy(a).to(dev) for a in (g.xadj, g.adjncy, g.adjwgt, g.vwgt)]
        part = torch.empty(g.n, dtype=torch.int32, device=dev)
        flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
        for _ in range(max(1, args.warmup)):
            h.partition_device(*t, k, part)
        ms = []
        cut = st = None
        sampler = ClockSampler(0)
        sampler.start()
        for _ in range(max(1, args.steps)):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cut, st = h.partition_device(*t, k, part)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        clocks = sampler.stop()
        p = part.cpu().numpy()
        W = int(g.vwgt.astype(np.int64).sum())
        pw = np.bincount(p, weights=g.vwgt, minlength=k)
        m = statistics.median(ms)
        out.append({"config": name, "n": g.n, "edges": g.n_edges, "k": k, "ms": m, "edges_per_s": g.n_edges / (m / 1e3),
                    "cut": int(cut), "balance": float(pw.max() * k / W), "levels": st["level_n"],
                    "phase_ms": {"coarsen": st["ms_coarsen"], "init": st["ms_init"], "refine": st["ms_refine"]},
                    "clocks": clocks})
        print(json.dumps(out[-1]), flush=True)
        h.close()
        del t, part, flush
        torch.cuda.empty_cache()
    print(json.dumps({"workload": "configs", "metric": "edges/s partitioned, default mode", "steps": args.steps,
                      "warmup": args.warmup, "results": out}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "served", "configs"])
    ap.add_argument("--graphs", type=int, default=4096, help="batched: number of graphs")
    ap.add_argument("--slots", type=int, default=2, help="batched/served: concurrent partitions")
    ap.add_argument("--pool", type=int, default=96, help="served: distinct graphs requests draw from")
    ap.add_argument("--max-n", type=int, default=2000000, help="served: largest graph")
    ap.add_argument("--rates", default="20,1000", help="served: offered loads (requests/s)")
    ap.add_argument("--requests", type=int, default=400, help="served: most requests per load")
    ap.add_argument("--duration", type=float, default=10.0, help="served: seconds of arrivals per load")
    ap.add_argument("--no-tune", action="store_true",
                    help="plain workload: skip gkw_autotune (default launch shapes; profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="plain workload: leave the batched and served objects out of the line")
    ap.add_argument("--only", default="",
                    help="configs workload: run only the configurations whose name starts with this")
    ap.add_argument("--device-only", action="store_true",
                    help="plain workload: only the device-resident steps (no e2e, CPU baseline, batched or "
                         "served legs); for profiling runs")
    args = ap.parse_args()
    if args.workload == "configs":
        bench_configs(args)
    elif args.workload == "batched":
        bench_batched(args)
    elif args.workload == "served":
        bench_served(args)
    elif args.impl == "reference":
        bench_reference(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
