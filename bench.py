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
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for i, nm in enumerate(names):
                if r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


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
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        l0 = pkg.launch_count()
        cut, st = h.partition_device(xadj, adjncy, adjwgt, vwgt, K, part, opts)
        launches += pkg.launch_count() - l0
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    barrier()
    clocks = sampler.stop() if sampler else None
    ms = sum(step_ms) / len(step_ms)
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(ms_t.item())

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
    e2e_t = torch.tensor([e2e], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_max = float(e2e_t.item())
    assert int(cut_e) == int(cut), "host and device paths disagree"

    # ---- roofline of the dominant kernel (contraction at level 0) ----
    roof = None
    if rank == 0:
        roof = roofline_contract(pkg, h, g, stream, flush)

    if rank == 0:
        part_np = part.cpu().numpy()
        pw = np.bincount(part_np, weights=g.vwgt, minlength=K)
        W = int(g.vwgt.sum())
        cpu = metis_cpu_baseline(g)
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
            "cpu_baseline": cpu,
            "quality": {"cut": int(cut), "max_part_weight": int(pw.max()),
                        "balance": float(pw.max() * K / W), "maxw": st["maxw"] if st else None,
                        "levels": st["level_n"] if st else None,
                        "refine_rounds": st["refine_rounds"] if st else None},
            "phase_ms": {"coarsen": st["ms_coarsen"], "init": st["ms_init"], "refine": st["ms_refine"],
                         "total": st["ms_total"]} if st else None,
            "clocks": clocks,
        }
        print(json.dumps(line))
    h.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def roofline_contract(pkg, h, g, stream, flush):
    """Contraction of level 0 timed alone (per-phase entry point), against the
    measured HBM copy bandwidth.  Algorithmic bytes per launch:
    4(n+1) + 8m (level CSR) + 8n (own + gathered cmap) + 4(n_c+1) + 8m_c."""
    import torch
    import oracle
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"hbm_gbs": 6650.0}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    dev = torch.device("cuda", torch.cuda.current_device())
    dg = tuple(torch.from_numpy(a).to(dev) for a in (g.xadj, g.adjncy, g.adjwgt, g.vwgt))
    cand = h.match(dg)
    root, dist, _ = h.union_find(cand)
    cmap, nc = h.group_map(root, dist, 6)
    times = []
    mc = 0
    for i in range(8):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cx, ca, cw, cv = h.contract(dg, cmap, nc)
        e1.record(stream)
        e1.synchronize()
        if i >= 2:
            times.append(e0.elapsed_time(e1))
        mc = int(ca.shape[0])
    ms = statistics.median(times)
    alg = 4 * (g.n + 1) + 8 * g.m + 8 * g.n + 4 * (nc + 1) + 8 * mc
    achieved = alg / (ms / 1e3) / 1e9
    tr = None
    tf = os.path.join(ROOT, "profiles", "contract_traffic.json")
    if os.path.exists(tf):
        try:
            tr = json.load(open(tf)).get("bytes_per_launch")
        except Exception:
            tr = None
    return {"kernel": "contraction, level 0 (gkw_contract: accum + scan + hash rows + scan + copy)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr, "algorithmic_bytes": int(alg), "ms": ms,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    if args.impl == "reference":
        bench_reference(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
