"""Benchmark of the SpMV hot path on B200.

Workload (one "step"): y = A x, FP32 plus-times SpMV over the whole R-MAT
scale-22 graph (4,194,304 vertices, edge factor 16, a/b/c/d = .57/.19/.19/.05,
self loops and duplicates removed, int32 indices, values and x uniform in
[0,1), seeded), CSR storage -- the format-sweep configuration at full size.

Metric: achieved SpMV bandwidth in GB/s over algorithmic bytes
  B = 4 (n+1) [row_ptr] + 8 nnz [col + val] + 4 n [x, read once] + 4 n [y write]
divided by the device time of one step (CUDA events on the launching
stream, max over ranks).  Also reported: % of measured HBM peak, GTEPS
(nnz / t) and the reference's own GB/s formula 16 nnz / t (spmv.cpp:94-98).

  python bench.py [--gpus N --steps K --warmup W] [--format CSR|SELL_C|CSR_SEG|LAV]
  python bench.py --impl reference   # the reference's OpenMP CPU SpMV, same config

Other workloads, one JSON line each:
  python bench.py --mode batched     # 64-source BFS, 32-column PPR / SSSP, R-MAT s22
  python bench.py --mode serve       # Poisson BFS/SSSP/PPR requests on resident R-MAT s24
  python bench.py --mode algorithms  # BFS/CC/PR/SSSP/TC on R-MAT s23 vs the reference CPU

Multi-GPU: the hot path does not need an exchange at these sizes, so
``--gpus N`` (under torchrun) runs N independent replicas, one per GPU, and
``value`` sums their work ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SpMV GB/s (% HBM peak) & GTEPS; served-query QPS + p50/p99 vs plain GPU"
FALLBACK_HBM_GBS = 6650.0
# Format the reference CPU code runs in: "auto" maps to CSR_SEG, the
# reference's fastest format in its own SpMV measurements.
REF_FORMAT = {"auto": 3, "CSR": 0, "SELL_C": 6, "CSR_SEG": 3, "LAV": 4}
REF_FORMAT_NAME = {0: "CSR", 3: "CSR_SEG", 4: "LAV", 6: "SELL_C"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--sweep", action="store_true", help="add the storage-format sweep to the JSON line")
    p.add_argument("--sweep-steps", type=int, default=200)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--graph", default="rmat", choices=["rmat", "er"])
    p.add_argument("--format", default="auto", choices=["auto", "CSR", "SELL_C", "CSR_SEG", "LAV"],
                   help="storage format; auto = the per-graph autotuner's choice")
    p.add_argument("--sigma", type=int, default=0, help="SELL-C sorting window for --format SELL_C")
    p.add_argument("--staged", type=int, default=0,
                   help="--format SELL_C: 1 = SELL-C-sigma inside staged x windows; CSR_SEG / LAV: -1 = unstaged")
    p.add_argument("--reorder", type=int, default=0, help="--format SELL_C: renumber columns by in-degree")
    p.add_argument("--csr-kernel", type=int, default=0,
                   help="--format CSR: 0 default (degree bins), 1 merge-path, 2 degree bins, 3 runs of 256 entries")
    p.add_argument("--seed", type=int, default=42)
    p.add_argument("--cpu-baseline-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--mode", default="spmv",
                   choices=["spmv", "batched", "serve", "algorithms", "single", "ingest", "spgemm"],
                   help="spmv: the SpMV line (default); batched: 64-source BFS + 32-column PPR / SSSP on "
                        "R-MAT s22; serve: Poisson request stream on a resident undirected R-MAT s24; "
                        "algorithms: BFS/CC/PR/SSSP/TC on undirected R-MAT s23 vs the reference CPU code; "
                        "single: the device-loop BFS/SSSP/CC/PageRank calls on undirected R-MAT (--alg-scale), "
                        "--steps sources; "
                        "ingest: the R-MAT graph as .mtx / .mtxbin files into device CSR vs the reference reader; "
                        "spgemm: unmasked A*A and triangle counting on undirected R-MAT vs the reference")
    p.add_argument("--queries", type=int, default=1000, help="serve: requests in the trace")
    p.add_argument("--rate", type=float, default=2000.0, help="serve: mean arrival rate (queries/s)")
    p.add_argument("--serial-queries", type=int, default=60, help="serve: requests run one at a time")
    p.add_argument("--serve-scale", type=int, default=24, help="serve: R-MAT scale of the resident graph")
    p.add_argument("--alg-scale", type=int, default=23, help="algorithms: R-MAT scale")
    p.add_argument("--ingest-reps", type=int, default=3, help="ingest: timed reads per file")
    p.add_argument("--spgemm-scale", type=int, default=15, help="spgemm: R-MAT scale (undirected)")
    p.add_argument("--no-extras", action="store_true",
                   help="default line without the batched / served summaries (SpMV only)")
    return p.parse_args()


def hbm_peak():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def make_input(args):
    from gb_kun_b200 import graphgen as gg
    if args.graph == "rmat":
        g = gg.rmat(args.scale, args.edge_factor, seed=args.seed)
    else:
        g = gg.uniform(args.scale, args.edge_factor, seed=args.seed)
    val = gg.values_f32(g, seed=args.seed + 1)
    x = gg.vector_f32(g.n, seed=args.seed + 2)
    return g, val, x


def alg_bytes(g):
    return 4 * (g.n + 1) + 8 * g.nnz + 4 * g.n + 4 * g.n


def workload_config(args, g):
    """The workload both arms run (identical for --impl ours and reference);
    the storage format each arm actually ran is reported beside it."""
    return {"workload": f"spmv_fp32_plus_times_{args.format.lower()}_{args.graph}{args.scale}",
            "graph": f"{'R-MAT' if args.graph == 'rmat' else 'Erdos-Renyi'} scale {args.scale}, edge factor "
                     f"{args.edge_factor}, seed {args.seed}",
            "n": g.n, "nnz": g.nnz, "format": args.format, "index": "int32", "semiring": "plus_times",
            "l2": "inputs larger than L2 (matrix arrays stream from HBM each step; x is L2-resident by design)"}


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()  # the timed region starts once sampling runs
            while not self.samples and time.time() - t0 < 10:
                time.sleep(0.02)
            self.skip = len(self.samples)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        samples = self.samples[getattr(self, "skip", 0):] or self.samples[-1:]
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in samples for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(samples)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(args, g, val, x):
    """The reference's own OpenMP CSR SpMV on this host, bounded sample."""
    try:
        from oracle.cpu import Reference
        if not Reference.available():
            return None
        R = Reference()
        fmt = REF_FORMAT[args.format]
        _, ms = R.spmv(g, val, x, fmt=fmt, semiring=0, warmup=1, reps=1)
        reps = max(3, min(200, int(args.cpu_baseline_seconds * 1000 / max(ms, 1e-3))))
        _, ms = R.spmv(g, val, x, fmt=fmt, semiring=0, warmup=0, reps=reps)
        return {"value": alg_bytes(g) / (ms * 1e-3) / 1e9, "unit": "GB/s", "cores": R.max_threads(),
                "cpu_model": cpu_model(), "kind": "reference",
                "sample": f"full matrix, median of {reps} GrB_mxv calls (reference CPU code, "
                          f"format {REF_FORMAT_NAME[fmt]}, OMP_NUM_THREADS={R.max_threads()})",
                "ms_per_spmv": ms}
    except Exception as e:  # reported, never fatal for the GPU number
        return {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"failed: {e}"}


def read_traffic(profile):
    """DRAM bytes of one SpMV from the committed ncu summary.

    Prefers the whole-SpMV sum (`traffic_bytes_per_spmv:`, all kernels of one
    SpMV from the launch list), else the dominant kernel's own launch.  The
    summary names the kernel sources it was captured from
    (`kernel_source_sha256: <path> <hex>`); when a source has changed since,
    the figure describes other code and None is returned."""
    f = ROOT / "profiles" / f"{profile}.md"
    if not f.exists():
        return None
    found = {}
    for line in f.read_text().splitlines():
        if line.startswith("kernel_source_sha256:"):
            parts = line.split(":", 1)[1].split()
            src = ROOT / parts[0]
            if len(parts) < 2 or not src.exists() or hashlib.sha256(src.read_bytes()).hexdigest() != parts[1]:
                return None
        for key in ("traffic_bytes_per_spmv:", "traffic_bytes_per_launch:"):
            if line.startswith(key) and key not in found:
                try:
                    found[key] = float(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    pass
    return found.get("traffic_bytes_per_spmv:", found.get("traffic_bytes_per_launch:"))


def dominant_kernel(fmt_name, scale, graph, staged=False, csr_kernel=0, nnz=0):
    """(kernel description, profile summary) for the storage format that ran
    (the default CSR kernel takes runs of 256 entries from 2^23 entries on)."""
    tag = f"{graph}{scale}"
    if fmt_name == "CSR" and (csr_kernel == 3 or (csr_kernel == 0 and nnz >= 1 << 23)):
        return ("k_spmv_chunks (256 entries per warp; + k_spmv_chunks_fixup for rows across chunks); achieved "
                "counts the whole SpMV", f"spmv_csr_chunks_{tag}")
    if fmt_name == "SELL_C" and staged:
        return ("k_sellw (SELL-C-sigma inside x windows staged in shared memory; + k_sw_prologue for y and the "
                "renumbered x); achieved counts the whole SpMV", f"spmv_sell_c_staged_{tag}")
    if fmt_name == "SELL_C":
        return ("k_sell_items (+ k_piece_fold for long-row pieces, k_sell_fold, k_spmv_binned for the few "
                "problematic slices); achieved counts the whole SpMV", f"spmv_sell_c_{tag}")
    if fmt_name == "CSR_SEG":
        return "k_segsmem (x windows staged in shared memory; + k_ss_identity for y); achieved counts the whole " \
            "SpMV", f"spmv_csr_seg_staged_{tag}"
    if fmt_name == "CSR":
        return "k_spmv_binned (+ k_spmv_split_fixup); achieved counts the whole SpMV", f"spmv_csr_kernels_{tag}"
    return f"{fmt_name} kernels; achieved counts the whole SpMV", f"spmv_{fmt_name.lower()}_{tag}"


def time_spmv(A, dx, dy, steps, warmup, semiring="plus_times"):
    """Average device time (ms) of one SpMV over `steps` launches (CUDA events)."""
    import torch
    for _ in range(warmup):
        A.mxv(dx, dy, semiring=semiring)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        A.mxv(dx, dy, semiring=semiring)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def format_sweep(args, peak):
    """The format-sweep configuration: every storage format on R-MAT and
    Erdos-Renyi graphs of the same scale, plus-times and or-and semirings.
    GB/s counts CSR-equivalent algorithmic bytes (padding is not credited)."""
    import torch
    from gb_kun_b200 import capi
    from gb_kun_b200 import graphgen as gg
    from oracle.cpu import Oracle
    O = Oracle()
    out = {}
    fmts = [("CSR_bins", {"fmt": "CSR", "csr_kernel": 2}), ("CSR_merge", {"fmt": "CSR", "csr_kernel": 1}),
            ("CSR_chunks", {"fmt": "CSR", "csr_kernel": 3}),
            ("SELL_C_s1", {"fmt": "SELL_C", "sigma": 1}), ("SELL_C_s256", {"fmt": "SELL_C", "sigma": 256}),
            ("SELL_C_s4096", {"fmt": "SELL_C", "sigma": 4096}),
            ("SELL_C_s4096_reorder", {"fmt": "SELL_C", "sigma": 4096, "reorder": 1}),
            ("SELL_C_s256_reorder", {"fmt": "SELL_C", "sigma": 256, "reorder": 1}),
            ("CSR_SEG", {"fmt": "CSR_SEG"}), ("LAV", {"fmt": "LAV"}),
            ("SELL_C_staged", {"fmt": "SELL_C", "staged": 1}),
            ("SELL_C_staged_reorder", {"fmt": "SELL_C", "staged": 1, "reorder": 1})]
    for gname in ("rmat", "er"):
        g = gg.rmat(args.scale, args.edge_factor, seed=args.seed) if gname == "rmat" else \
            gg.uniform(args.scale, args.edge_factor, seed=args.seed)
        val = gg.values_f32(g, seed=args.seed + 1)
        x = gg.vector_f32(g.n, seed=args.seed + 2)
        ref = O.spmv_f64(g, val, x)
        B = alg_bytes(g)
        A = capi.Matrix.from_graph(g, val)
        dx = torch.from_numpy(x).cuda()
        dy = torch.zeros(g.n, device="cuda")
        for name, f in fmts:
            A.set_format(f["fmt"], sigma=f.get("sigma", 0), csr_kernel=f.get("csr_kernel", 0), hot_cols=f.get("hot", 0),
                         reorder_cols=f.get("reorder", 0), seg_staged=f.get("staged", 0))
            ms = time_spmv(A, dx, dy, args.sweep_steps, 3)
            err = float(np.abs(dy.cpu().numpy().astype(np.float64) - ref).sum() / np.abs(ref).sum())
            ms_or = time_spmv(A, dx, dy, args.sweep_steps, 3, semiring="lor_land")
            inf = A.info()
            out[f"{gname}{args.scale}.{name}"] = {
                "plus_times_gbs": round(B / (ms * 1e-3) / 1e9, 1), "plus_times_ms": round(ms, 4),
                "pct_hbm_peak": round(100 * B / (ms * 1e-3) / 1e9 / peak, 1),
                "or_and_gbs": round(B / (ms_or * 1e-3) / 1e9, 1), "rel_l1_vs_fp64": err,
                "stored_entries": int(inf.padded_nnz), "nnz": g.nnz}
        A.close()
    return out


def e2e_pipelined(A, hx, g, steps, depth=3, parts=2):
    """End-to-end SpMV through the public API with host buffers: every step
    copies its x from pinned host memory to the device, runs gbk_mxv and
    copies its y back to pinned host memory.  Steps are independent
    requests, so step i+1's upload, step i's SpMV and step i-1's download run
    at once; each copy is cut into `parts` pieces on as many streams per
    direction (two pieces in flight per direction moved 11 % more than one
    copy per direction, four fewer), and `depth` device and host buffers
    rotate.  Returns the device time per step (CUDA events; the end event
    waits for every stream)."""
    import torch
    n = g.n
    ups = [torch.cuda.Stream() for _ in range(parts)]
    downs = [torch.cuda.Stream() for _ in range(parts)]
    comp = torch.cuda.Stream()
    dxs = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(depth)]
    dys = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(depth)]
    hys = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(depth)]
    copied = [[torch.cuda.Event() for _ in range(parts)] for _ in range(depth)]  # x_i pieces on the device
    done = [torch.cuda.Event() for _ in range(depth)]                            # y_i computed
    freed = [[torch.cuda.Event() for _ in range(parts)] for _ in range(depth)]   # y_i pieces downloaded
    cut = [n * p // parts for p in range(parts + 1)]

    def run(cnt):
        for i in range(cnt):
            k = i % depth
            for p in range(parts):
                if i >= depth:
                    for q in range(parts):  # buffers k are free once all of y_{i-depth} is home
                        ups[p].wait_event(freed[k][q])
                with torch.cuda.stream(ups[p]):
                    dxs[k][cut[p]:cut[p + 1]].copy_(hx[cut[p]:cut[p + 1]], non_blocking=True)
                    copied[k][p].record(ups[p])
            for p in range(parts):
                comp.wait_event(copied[k][p])
            A.mxv(dxs[k], dys[k], stream=comp)
            done[k].record(comp)
            for p in range(parts):
                downs[p].wait_event(done[k])
                with torch.cuda.stream(downs[p]):
                    hys[k][cut[p]:cut[p + 1]].copy_(dys[k][cut[p]:cut[p + 1]], non_blocking=True)
                    freed[k][p].record(downs[p])

    run(2 * depth)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ups[0])
    for st in ups[1:] + downs + [comp]:
        st.wait_event(e0)
    run(steps)
    for st in ups[1:] + downs + [comp]:
        ups[0].wait_stream(st)
    e1.record(ups[0])
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, hys[(steps - 1) % depth]


def e2e_serial(A, hx, dx, dy, hy, steps, stream):
    """The same, one step after another on one stream (no overlap)."""
    import torch
    for _ in range(2):
        dx.copy_(hx, non_blocking=True)
        A.mxv(dx, dy)
        hy.copy_(dy, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        dx.copy_(hx, non_blocking=True)
        A.mxv(dx, dy)
        hy.copy_(dy, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def c1_csr_s18(args, peak):
    """Plain FP32 plus-times SpMV on CSR over R-MAT scale 18 (262,144 vertices,
    edge factor 16), the reference's CPU CSR SpMV beside it.  The matrix
    (about 37 MB) fits in L2, so every timed SpMV follows an L2 flush (a
    write of twice the L2 size) and is timed alone with CUDA events; the
    warm (back-to-back) rate is reported too.  Both CSR kernels run (degree
    bins, runs of 256 entries per warp); the line carries the faster."""
    import torch
    from gb_kun_b200 import capi
    from gb_kun_b200 import graphgen as gg
    g = gg.rmat(18, 16, seed=args.seed)
    val = gg.values_f32(g, seed=args.seed + 1)
    x = gg.vector_f32(g.n, seed=args.seed + 2)
    dx = torch.from_numpy(x).cuda()
    dy = torch.zeros(g.n, device="cuda")
    l2 = torch.cuda.get_device_properties(0).L2_cache_size
    flush = torch.empty(2 * l2 // 4, dtype=torch.float32, device="cuda")
    B = alg_bytes(g)
    from oracle.cpu import Oracle
    ref64 = Oracle().spmv_f64(g, val, x)
    kernels = {}
    for name, kern in (("degree_bins", 2), ("entry_chunks", 3)):
        A = capi.Matrix.from_graph(g, val)
        A.set_format("CSR", csr_kernel=kern)
        for _ in range(5):
            A.mxv(dx, dy)
        ts = []
        for i in range(50):
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            A.mxv(dx, dy)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        warm = time_spmv(A, dx, dy, 200, 3)
        err = float(np.abs(dy.cpu().numpy().astype(np.float64) - ref64).sum() / np.abs(ref64).sum())
        kernels[name] = {"ms_flushed": round(statistics.median(ts), 5), "ms_warm_l2": round(warm, 5),
                         "rel_l1_vs_fp64": err}
        A.close()
    best = min(kernels, key=lambda k: kernels[k]["ms_flushed"])
    cold, warm = kernels[best]["ms_flushed"], kernels[best]["ms_warm_l2"]
    out = {"workload": "spmv_fp32_plus_times_csr_rmat18", "n": g.n, "nnz": g.nnz,
           "ms_flushed": round(cold, 5), "gbs_flushed": round(B / (cold * 1e-3) / 1e9, 1),
           "frac_flushed": round(B / (cold * 1e-3) / 1e9 / peak, 4),
           "ms_warm_l2": round(warm, 5), "gbs_warm_l2": round(B / (warm * 1e-3) / 1e9, 1),
           "rel_l1_vs_fp64": kernels[best]["rel_l1_vs_fp64"],
           "csr_kernel": {"degree_bins": "degree bins (k_spmv_binned)",
                          "entry_chunks": "256 entries per warp (k_spmv_chunks)"}[best],
           "csr_kernels": kernels}
    try:
        from oracle.cpu import Reference
        if Reference.available():
            R = Reference()
            _, ms = R.spmv(g, val, x, fmt=0, semiring=0, warmup=3, reps=50)
            out["cpu_baseline"] = {"value": round(B / (ms * 1e-3) / 1e9, 2), "unit": "GB/s", "ms": round(ms, 4),
                                   "cores": R.max_threads(), "cpu_model": cpu_model(), "kind": "reference",
                                   "sample": "median of 50 GrB_mxv calls, reference CPU code, CSR"}
            out["speedup_vs_reference_flushed"] = round(ms / cold, 1)
    except Exception as e:
        out["cpu_baseline"] = {"error": str(e)[:200]}
    return out


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from gb_kun_b200 import capi
    capi.init(local)
    g, val, x = make_input(args)
    A = capi.Matrix.from_graph(g, val)
    stream = torch.cuda.current_stream()
    dx = torch.from_numpy(x).cuda()
    dy = torch.zeros(g.n, device="cuda")
    B = alg_bytes(g)
    tuned = None
    # clocks are sampled from the tuning runs through the end of the timed
    # steps: the timed region alone is a few milliseconds at small --steps
    with ClockSampler(local) as clk:
        if args.format == "auto":
            tuned = A.autotune(reps=20).describe()
        else:
            A.set_format(args.format, sigma=args.sigma, seg_staged=args.staged, reorder_cols=args.reorder,
                         csr_kernel=args.csr_kernel)
        for _ in range(args.warmup):
            A.mxv(dx, dy)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        l0 = capi.launch_count()
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        t_all0.record(stream)
        for i in range(args.steps):
            A.mxv(dx, dy)
        t_all1.record(stream)
        torch.cuda.synchronize()
        launches = capi.launch_count() - l0
    barrier(world)
    torch.cuda.synchronize()
    total_ms = max_over_ranks(t_all0.elapsed_time(t_all1), world)
    ms_per_step = total_ms / args.steps

    # end to end through the public API: pinned host x -> device, SpMV, y -> pinned host
    hx = torch.from_numpy(x).pin_memory()
    hy1 = torch.empty(g.n, dtype=torch.float32).pin_memory()
    e2e_serial_ms = max_over_ranks(e2e_serial(A, hx, dx, dy, hy1, args.steps, stream), world)
    barrier(world)
    e2e_ms, hy = e2e_pipelined(A, hx, g, args.steps)
    e2e_ms = max_over_ranks(e2e_ms, world)

    # correctness of the timed output (checker only)
    ok = None
    if rank == 0:
        from oracle.cpu import Oracle
        ref = Oracle().spmv_f64(g, val, x)
        got = hy.numpy().astype(np.float64)
        ok = float(np.abs(got - ref).sum() / np.abs(ref).sum())

    peak, peak_kind = hbm_peak()
    ran_format = tuned["format"] if tuned else args.format
    staged = bool(tuned.get("staged_windows")) if tuned else args.staged == 1
    ran_csr_kernel = tuned.get("csr_kernel") if tuned else args.csr_kernel
    ran_csr_kernel = {"entry-chunks": 3}.get(ran_csr_kernel, ran_csr_kernel)
    kern_desc, kern_profile = dominant_kernel(ran_format, args.scale, args.graph, staged,
                                              ran_csr_kernel if isinstance(ran_csr_kernel, int) else 0, g.nnz)
    # one launch = one SpMV (the y initialisation and the main kernel, which
    # starts under programmatic dependent launch); its average duration is
    # the per-step time of the timed region
    achieved = B / (ms_per_step * 1e-3) / 1e9
    value = world * B / (ms_per_step * 1e-3) / 1e9
    cfg = workload_config(args, g)
    cfg["parallelism"] = f"replicas{world}" if world > 1 else "single"
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded R-MAT, generated in-process)",
        "config": cfg,
        "format_ran": tuned if tuned else {"format": args.format, "sigma": args.sigma, "staged": args.staged,
                                           "reorder_cols": args.reorder},
        "pct_hbm_peak": round(100 * achieved / peak, 2),
        "gteps": round(world * g.nnz / (ms_per_step * 1e-3) / 1e9, 3),
        "ref_formula_gbs": round(world * 16 * g.nnz / (ms_per_step * 1e-3) / 1e9, 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6650 GB/s",
                     "traffic": read_traffic(kern_profile),
                     "kernel": kern_desc,
                     "algorithmic_bytes_per_launch": B,
                     "launch_ms": round(ms_per_step, 5)},
        "e2e": {"value": round(world * B / (e2e_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
                "h2d_bytes_per_step": 4 * g.n, "d2h_bytes_per_step": 4 * g.n, "ms_per_step": round(e2e_ms, 5),
                "pipelining": "upload of step i+1, SpMV of step i and download of step i-1 at once; each copy in two "
                              "halves on two streams per direction",
                "serial_ms_per_step": round(e2e_serial_ms, 5),
                "serial_gbs": round(world * B / (e2e_serial_ms * 1e-3) / 1e9, 2)},
        "gpu_launches": int(launches),
        "clocks": dict(clk.summary(), window="autotune, warm-up and timed steps"),
        "check_rel_l1_vs_fp64": ok,
    }
    A.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, g, val, x)
    if args.sweep and rank == 0:
        out["format_sweep"] = format_sweep(args, peak)
    if rank == 0 and world == 1 and not args.no_extras:
        try:
            out["c1_csr_s18"] = c1_csr_s18(args, peak)
        except Exception as e:
            out["c1_csr_s18"] = {"error": str(e)[:300]}
        out.update(extras_summary(args))
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _median_ms(fn, reps):
    """Median device time of fn() over reps calls (CUDA events on the current stream)."""
    import torch
    ts = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts), ts


def _ref_threads():
    try:
        from oracle.cpu import Reference
        return Reference() if Reference.available() else None
    except Exception:
        return None


def run_batched(args):
    """64-source BFS and 32-column PPR / SSSP on R-MAT scale 22 (directed)."""
    import torch
    from gb_kun_b200 import capi, graphgen as gg, lablas_capi as lc
    capi.init(0)
    g = gg.rmat(args.scale, args.edge_factor, seed=args.seed)
    w = gg.weights_i32(g, seed=args.seed + 3)
    A = capi.Matrix.from_graph(g, val=w.astype(np.float32))
    deg = torch.from_numpy(np.diff(g.row_ptr).astype(np.int64)).cuda()
    src = gg.sources(g, 64, seed=args.seed + 4)
    reps = max(3, min(args.steps, 10))
    warm = max(3, args.warmup)
    lv = torch.zeros((64, g.n), dtype=torch.int32, device="cuda")
    rk = torch.zeros((32, g.n), dtype=torch.float32, device="cuda")
    dd = torch.zeros((32, g.n), dtype=torch.int32, device="cuda")
    tuned = {"bfs": A.batch_autotune("bfs", src).describe(), "ppr": A.batch_autotune("ppr", src[:32]).describe(),
             "sssp": A.batch_autotune("sssp", src[:32]).describe()}
    for _ in range(warm):
        A.msbfs(src, lv)
        A.ppr(src[:32], rk)
        A.sssp_multi(src[:32], dd)
    torch.cuda.synchronize()
    l0 = capi.launch_count()
    with ClockSampler(0) as clk:
        bfs_ms, bfs_ts = _median_ms(lambda: A.msbfs(src, lv), reps)
        ppr_ms, _ = _median_ms(lambda: A.ppr(src[:32], rk), reps)
        sssp_ms, _ = _median_ms(lambda: A.sssp_multi(src[:32], dd), reps)
    launches = capi.launch_count() - l0
    depths = A.msbfs(src, lv)
    ppr_it = A.ppr(src[:32], rk)
    sssp_it = A.sssp_multi(src[:32], dd)
    edges = int(((lv > 0).to(torch.int64) * deg).sum())
    gteps = edges / (bfs_ms * 1e-3) / 1e9
    # single-query paths, one at a time: lablas bfs_blast / sssp and one-lane PPR
    G = lc.Graph(g, weights=w)
    G.bfs(int(src[0]))
    one_bfs = statistics.median([G.bfs(int(s))[1] for s in src[:8]])
    G.sssp_i32(int(src[0]))
    one_sssp = statistics.median([G.sssp_i32(int(s))[1] for s in src[:4]])
    one_ppr, _ = _median_ms(lambda: A.ppr(src[:1], rk[:1]), 3)
    # end to end: levels of all 64 sources back in pinned host memory
    hl = torch.empty((64, g.n), dtype=torch.int32).pin_memory()
    e2e_ms, _ = _median_ms(lambda: (A.msbfs(src, lv), hl.copy_(lv, non_blocking=True)), 3)
    # checker: some lanes against the oracle
    from oracle.cpu import Oracle
    O = Oracle()
    lvh, rkh, ddh = lv.cpu().numpy(), rk.cpu().numpy(), dd.cpu().numpy()
    ok_bfs = all(np.array_equal(lvh[k], O.bfs(g, int(src[k]))) for k in (0, 31, 63))
    d0 = O.sssp(g, w, int(src[0]))
    ok_sssp = bool(np.array_equal(ddh[0], np.where(d0 < 0, np.iinfo(np.int32).max, d0).astype(np.int32)))
    r0, _ = O.ppr(g, int(src[0]), tol=1e-6, itermax=100)
    ppr_err = float(np.abs(rkh[0] - r0).sum() / np.abs(r0).sum())
    # roofline of the PPR SpMM (per iteration, 32 columns): 4(n+1) + 4 nnz + 2 n 32 4
    peak, peak_kind = hbm_peak()
    spmm_bytes = 4 * (g.n + 1) + 4 * g.nnz + 2 * g.n * 32 * 4
    spmm_gbs = spmm_bytes * int(ppr_it.max()) / (ppr_ms * 1e-3) / 1e9
    R = _ref_threads()
    cpu = None
    if R is not None and not args.no_cpu_baseline:
        r_edges, r_ms = 0, 0.0
        for s in src[:2]:
            lvr, ms = R.bfs(g, int(s))
            r_edges += int(np.diff(g.row_ptr)[lvr > 0].sum())
            r_ms += ms
        cpu = {"value": round(r_edges / (r_ms * 1e-3) / 1e9, 4), "unit": "GTEPS", "cores": R.max_threads(),
               "kind": "reference", "sample": "bfs_blast from 2 of the 64 sources, one at a time"}
    out = {
        "metric": "batched BFS GTEPS (64 sources per launch); PPR / SSSP queries/s",
        "value": round(gteps, 3), "unit": "GTEPS", "n_gpus": 1, "steps": reps, "warmup": warm,
        "ms_per_step": round(bfs_ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64 lanes (BFS), f32 (PPR), i32 (SSSP)", "data": "synthetic (seeded R-MAT, generated in-process)",
        "config": {"workload": f"msbfs64_ppr32_sssp32_rmat{args.scale}", "n": g.n, "nnz": g.nnz,
                   "graph": f"R-MAT scale {args.scale}, edge factor {args.edge_factor}, directed, seed {args.seed}",
                   "sources": "64 seeded non-isolated vertices", "loop": "one CUDA graph per batch (while node)",
                   "autotuned": tuned,
                   "l2": "state and matrix larger than L2"},
        "msbfs": {"ms": round(bfs_ms, 3), "edges_traversed": edges, "max_depth": int(depths.max()),
                  "bfs_per_s": round(64 / (bfs_ms * 1e-3), 1), "one_at_a_time_ms": round(one_bfs, 3),
                  "speedup_vs_one_at_a_time": round(64 * one_bfs / bfs_ms, 2), "bit_exact_checked": ok_bfs},
        "ppr": {"ms": round(ppr_ms, 3), "seeds": 32, "iterations_max": int(ppr_it.max()),
                "queries_per_s": round(32 / (ppr_ms * 1e-3), 1), "one_lane_ms": round(one_ppr, 3),
                "rel_l1_vs_fp64_lane0": ppr_err},
        "sssp": {"ms": round(sssp_ms, 3), "sources": 32, "rounds_max": int(sssp_it.max()),
                 "queries_per_s": round(32 / (sssp_ms * 1e-3), 1), "one_at_a_time_ms": round(one_sssp, 3),
                 "speedup_vs_one_at_a_time": round(32 * one_sssp / sssp_ms, 2), "bit_exact_checked": ok_sssp},
        "roofline": {"bound": "hbm", "kernel": "k_ppr_spmm (+ k_ppr_fix, k_ppr_control); bytes per iteration "
                                               "4(n+1) + 4 nnz + 2*n*32*4",
                     "achieved": round(spmm_gbs, 2), "peak": peak, "unit": "GB/s", "frac": round(spmm_gbs / peak, 4),
                     "traffic": read_traffic("batched_traversals_rmat22") if args.scale == 22 else None},
        "e2e": {"value": round(edges / (e2e_ms * 1e-3) / 1e9, 3), "unit": "GTEPS", "h2d_bytes_per_step": 4 * 64,
                "d2h_bytes_per_step": 4 * 64 * g.n, "ms_per_step": round(e2e_ms, 3)},
        "gpu_launches": int(launches), "clocks": clk.summary(), "cpu_baseline": cpu,
    }
    return out


def run_serve(args):
    """Poisson stream of BFS / SSSP / PPR requests on a resident undirected R-MAT graph."""
    import torch
    from gb_kun_b200 import capi, graphgen as gg, lablas_capi as lc
    from gb_kun_b200.serve import Server, latency_stats, poisson_trace
    capi.init(0)
    t_gen = time.time()
    g = gg.rmat(args.serve_scale, args.edge_factor, seed=args.seed, undirected=True)
    w = gg.weights_i32(g, seed=args.seed + 3)
    t_gen = time.time() - t_gen
    A = capi.Matrix.from_graph(g, val=w.astype(np.float32))
    cand = gg.sources(g, 1 << 16, seed=args.seed + 5)
    arr, kinds, srcs = poisson_trace(args.queries, args.rate, mix=(0.5, 0.25, 0.25), candidates=cand,
                                     seed=args.seed + 6)
    nq = len(arr)
    srv = Server(A, iters_per_launch=4)
    # warm-up: builds the three batches and their graphs
    wa, wk, ws = poisson_trace(12, 1e5, candidates=cand, seed=args.seed + 7)
    srv.run_trace(wa, wk, ws)
    l0 = capi.launch_count()
    with ClockSampler(0) as clk:
        res, wall = srv.run_trace(arr, kinds, srcs)
    launches = capi.launch_count() - l0
    burst, wall_b = srv.run_trace(np.zeros(nq), kinds, srcs)
    # below capacity: the same mix at 60 % of the burst capacity, so the
    # latencies are service times rather than queueing
    sub_rate = 0.6 * nq / wall_b
    sub_n = min(nq, max(100, int(sub_rate * 2.0)))
    sa, sk, ss = poisson_trace(sub_n, sub_rate, mix=(0.5, 0.25, 0.25), candidates=cand, seed=args.seed + 8)
    sub, sub_wall = srv.run_trace(sa, sk, ss)
    # capacity per query kind (a burst of one kind only)
    per_kind = {}
    for k, name in ((0, "bfs"), (1, "ppr"), (2, "sssp")):
        sel = np.flatnonzero(kinds == k)[:128]
        if len(sel):
            _, wk_s = srv.run_trace(np.zeros(len(sel)), kinds[sel], srcs[sel])
            per_kind[name] = round(len(sel) / wk_s, 2)
    used, budget, nb = srv.memory()
    srv.close()
    # one query at a time through the same engine (one lane, nothing overlaps)
    m = min(args.serial_queries, nq)
    one = Server(A, lanes_per_batch=1, max_inflight=1)
    one.run_trace(wa[:3], wk[:3], ws[:3])
    res1, wall1 = one.run_trace(arr[:m], kinds[:m], srcs[:m])
    one_b, wall1_b = one.run_trace(np.zeros(m), kinds[:m], srcs[:m])
    one.close()
    # plain single-query algorithms (lablas bfs_blast / sssp), per-query device time
    G = lc.Graph(g, weights=w)
    G.bfs(int(cand[0]))
    plain_bfs = statistics.median([G.bfs(int(s))[1] for s in cand[1:6]])
    G.bfs_ops(int(cand[0]))
    plain_bfs_ops = statistics.median([G.bfs_ops(int(s))[1] for s in cand[1:6]])
    plain_sssp = statistics.median([G.sssp_i32(int(s))[1] for s in cand[1:4]])
    G.ppr(int(cand[0]))
    plain_ppr = statistics.median([G.ppr(int(s))[2] for s in cand[1:4]])
    G.close()
    ser = {k: float(np.mean((one_b["t_done"] - one_b["t_admit"])[one_b["kind"] == k]) * 1e3)
           if (one_b["kind"] == k).any() else None for k in (0, 1, 2)}
    # one-at-a-time capacity with the faster single-query path per kind
    best = {0: min(x for x in (ser[0], plain_bfs) if x), 1: min(x for x in (ser[1], plain_ppr) if x),
            2: min(x for x in (ser[2], plain_sssp) if x)}
    mix = {0: 0.5, 1: 0.25, 2: 0.25}
    one_best_qps = 1e3 / sum(mix[k] * best[k] for k in mix if best[k])
    qps = nq / wall
    cap = nq / wall_b
    cap1 = m / wall1_b
    lat = latency_stats(res)
    out = {
        "metric": "served-query QPS + p50/p99 vs one-at-a-time GPU", "value": round(qps, 2), "unit": "queries/s",
        "n_gpus": 1, "steps": nq, "warmup": 12, "ms_per_step": round(1e3 * wall / nq, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 lanes (BFS), f32 (PPR), i32 (SSSP)",
        "data": "synthetic (seeded R-MAT, seeded Poisson trace)",
        "config": {"workload": f"serve_rmat{args.serve_scale}u_poisson{int(args.rate)}",
                   "graph": f"R-MAT scale {args.serve_scale}, edge factor {args.edge_factor}, undirected, "
                            f"int32 weights in [1,255] as FP32 values", "n": g.n, "nnz": g.nnz,
                   "trace": f"{nq} queries, Poisson mean {args.rate}/s, 50% BFS / 25% SSSP / 25% PPR, sources "
                            "uniform over non-isolated vertices", "iters_per_launch": 4,
                   "l2": "graph and batch state larger than L2"},
        "latency_ms": lat, "qps_offered": args.rate, "qps_capacity_burst": round(cap, 2),
        "below_capacity": {"qps_offered": round(sub_rate, 2), "queries": int(sub_n),
                           "qps": round(sub_n / sub_wall, 2), "latency_ms": latency_stats(sub)},
        "qps_capacity_per_kind": per_kind,
        "batches": nb, "device_bytes_used": used, "memory_budget": budget,
        "one_at_a_time": {"qps_poisson": round(m / wall1, 2), "qps_capacity": round(cap1, 2),
                          "latency_ms": latency_stats(res1), "queries": m,
                          "service_ms_engine": ser, "service_ms_plain_lablas": {"bfs": plain_bfs, "bfs_graphblas_calls": plain_bfs_ops,
                                                      "sssp": plain_sssp, "ppr": plain_ppr},
                          "qps_capacity_best_single_query_path": round(one_best_qps, 2)},
        "speedup_qps_vs_one_at_a_time": round(cap / max(cap1, one_best_qps), 2),
        "e2e": {"value": round(qps, 2), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 24, "note": "requests enter and summaries leave through the host loop"},
        "gpu_launches": int(launches), "clocks": clk.summary(), "graph_gen_s": round(t_gen, 1),
    }
    return out


def extras_summary(args):
    """Compact batched and served results for the default line (each guarded:
    a failure there is reported, the SpMV line still prints)."""
    res = {}
    try:
        b = run_batched(args)
        res["batched"] = {"workload": b["config"]["workload"], "msbfs64_ms": b["msbfs"]["ms"],
                          "msbfs64_gteps": b["value"], "msbfs_speedup_vs_one_at_a_time":
                              b["msbfs"]["speedup_vs_one_at_a_time"],
                          "ppr32_ms": b["ppr"]["ms"], "ppr_rel_l1_vs_fp64": b["ppr"]["rel_l1_vs_fp64_lane0"],
                          "sssp32_ms": b["sssp"]["ms"], "sssp_speedup_vs_one_at_a_time":
                              b["sssp"]["speedup_vs_one_at_a_time"],
                          "bit_exact_checked": b["msbfs"]["bit_exact_checked"] and b["sssp"]["bit_exact_checked"],
                          "autotuned": b["config"]["autotuned"]}
    except Exception as e:  # reported, never fatal for the SpMV number
        res["batched"] = {"error": str(e)[:300]}
    try:
        v = run_serve(args)
        o = v["one_at_a_time"]
        res["served"] = {"workload": v["config"]["workload"], "qps": v["value"], "p50_ms": v["latency_ms"]["p50_ms"],
                         "p99_ms": v["latency_ms"]["p99_ms"], "qps_capacity": v["qps_capacity_burst"],
                         "below_capacity": {"qps_offered": v["below_capacity"]["qps_offered"],
                                            "p50_ms": v["below_capacity"]["latency_ms"]["p50_ms"],
                                            "p99_ms": v["below_capacity"]["latency_ms"]["p99_ms"]},
                         "qps_capacity_per_kind": v["qps_capacity_per_kind"],
                         "one_at_a_time_qps_same_engine": o["qps_capacity"],
                         "one_at_a_time_qps_best_single_query_path": o["qps_capacity_best_single_query_path"],
                         "speedup_vs_same_engine_one_at_a_time": round(v["qps_capacity_burst"] / o["qps_capacity"], 2),
                         "speedup_vs_best_single_query_path": v["speedup_qps_vs_one_at_a_time"]}
    except Exception as e:
        res["served"] = {"error": str(e)[:300]}
    try:
        a = run_algorithms(args, light=True)
        res["algorithms"] = {"workload": a["config"]["workload"], "n": a["config"]["n"], "nnz": a["config"]["nnz"],
                             **{k: {kk: vv for kk, vv in v.items() if kk in (
                                 "gpu_ms", "ref_cpu_ms", "speedup", "matches_reference", "gteps", "iterations",
                                 "rel_l1_vs_fp64_oracle", "triangles", "scale", "launches")}
                                for k, v in a["algorithms"].items()}}
    except Exception as e:
        res["algorithms"] = {"error": str(e)[:300]}
    return res


def run_single(args):
    """Single-query loops on the device (gbk_bfs_levels, gbk_sssp_dist, gbk_cc_labels,
    gbk_pagerank) on undirected R-MAT, CUDA events around each call; a few
    sources each, the levels / distances / labels checked against the oracle."""
    import torch
    from gb_kun_b200 import capi, graphgen as gg
    from oracle.cpu import Oracle
    capi.init(0)
    g = gg.rmat(args.alg_scale, args.edge_factor, seed=args.seed, undirected=True)
    w = gg.weights_i32(g, seed=args.seed + 3)
    A = capi.Matrix.from_graph(g)
    Aw = capi.Matrix.from_graph(g, w)
    src = [int(s) for s in gg.sources(g, max(1, args.steps), seed=args.seed + 4)]
    deg = np.diff(g.row_ptr)
    lv = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    dist = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    lab = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    rk = torch.zeros(g.n, device="cuda")
    A.autotune(reps=10, semiring="plus_second")
    for _ in range(max(1, args.warmup)):  # lazy CSC, format and degree builds
        A.bfs(src[0], lv)
        Aw.sssp(src[0], dist)
        A.cc(lab)
        A.pagerank(rk, itermax=100, damping=0.85, tol=1e-6)
    torch.cuda.synchronize()

    def ev(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    l0 = capi.launch_count()
    bfs = [ev(lambda: A.bfs(s, lv)) for s in src]
    edges = int(deg[lv.cpu().numpy() > 0].sum())
    sssp = [ev(lambda: Aw.sssp(s, dist)) for s in src]
    cc_ms, _ = ev(lambda: A.cc(lab))
    pr_ms, (pr_it, _) = ev(lambda: A.pagerank(rk, itermax=100, damping=0.85, tol=1e-6))
    launches = capi.launch_count() - l0
    O = Oracle()
    d64 = O.sssp(g, w, src[-1])
    checks = {"bfs": bool(np.array_equal(lv.cpu().numpy(), O.bfs(g, src[-1]))),
              "sssp": bool(np.array_equal(dist.cpu().numpy(),
                                          np.where(d64 < 0, np.iinfo(np.int32).max, d64).astype(np.int32))),
              "cc": bool(np.array_equal(lab.cpu().numpy(), O.cc(g)))}
    r64, _, _ = O.pagerank(g, tol=0.0, itermax=pr_it)
    checks["pagerank_rel_l1_vs_fp64"] = float(np.abs(rk.cpu().numpy() - r64).sum() / np.abs(r64).sum())
    bfs_ms = statistics.median(t for t, _ in bfs)
    A.close()
    Aw.close()
    return {
        "metric": "single-query loops on the device: ms per query", "value": round(edges / (bfs_ms * 1e-3) / 1e9, 3),
        "unit": "GTEPS (BFS)", "n_gpus": 1, "steps": len(src), "warmup": max(1, args.warmup),
        "ms_per_step": round(bfs_ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "i32 levels / i32 distances / f32 ranks", "data": "synthetic (seeded R-MAT, generated in-process)",
        "config": {"workload": f"single_query_rmat{args.alg_scale}u", "n": g.n, "nnz": g.nnz,
                   "graph": f"R-MAT scale {args.alg_scale}, edge factor {args.edge_factor}, undirected; int32 "
                            "weights in [1, 255] for SSSP", "sources": f"{len(src)} seeded non-isolated vertices",
                   "timing": "CUDA events around each call (one graph launch per query)"},
        "bfs_ms": [round(t, 4) for t, _ in bfs], "bfs_depth": bfs[-1][1],
        "sssp_ms": [round(t, 4) for t, _ in sssp], "sssp_rounds": sssp[-1][1],
        "cc_ms": round(cc_ms, 4), "pagerank_ms": round(pr_ms, 4), "pagerank_iterations": pr_it,
        "gpu_launches": int(launches), "checked_against_oracle": checks,
    }


def run_algorithms(args, light=False):
    """BFS, CC, PageRank, SSSP and TC on undirected R-MAT (lablas:: path) vs the reference CPU code.

    Each algorithm runs once untimed on the same inputs (lazy CSC / bins /
    format set-up), then once timed; the reference CPU code runs on the same
    graph and its output is compared (bit-exact, PageRank both against the
    reference and against the FP64 oracle).  light=True (the default bench
    line) checks the reference's triangle count at scale 17 instead of
    alg_scale - 4 and skips the unmasked SpGEMM."""
    from gb_kun_b200 import capi, graphgen as gg, lablas_capi as lc
    from oracle.cpu import Oracle
    capi.init(0)
    g = gg.rmat(args.alg_scale, args.edge_factor, seed=args.seed, undirected=True)
    w = gg.weights_i32(g, seed=args.seed + 3)
    G = lc.Graph(g, weights=w)
    src = gg.sources(g, 4, seed=args.seed + 4)
    R = _ref_threads()
    degs = np.diff(g.row_ptr)
    res = {}

    def rec(name, gpu_ms, ref_ms, exact, extra=None):
        res[name] = {"gpu_ms": round(gpu_ms, 3), "ref_cpu_ms": None if ref_ms is None else round(ref_ms, 1),
                     "speedup": None if not ref_ms else round(ref_ms / gpu_ms, 1), "matches_reference": exact}
        if extra:
            res[name].update(extra)

    def twice(fn):
        fn()
        return fn()

    lv, ms = twice(lambda: G.bfs(int(src[1])))
    ref = R.bfs(g, int(src[1])) if R else (None, None)
    teps = int(degs[lv > 0].sum()) / (ms * 1e-3) / 1e9
    rec("bfs", ms, ref[1], None if ref[0] is None else bool(np.array_equal(lv, ref[0])),
        {"gteps": round(teps, 3), "path": "gbk_bfs_levels: level loop on the device, one graph launch"})
    lv2, ms2 = twice(lambda: G.bfs_ops(int(src[1])))
    rec("bfs_graphblas_calls", ms2, ref[1], None if ref[0] is None else bool(np.array_equal(lv2, ref[0])),
        {"gteps": round(int(degs[lv2 > 0].sum()) / (ms2 * 1e-3) / 1e9, 3),
         "path": "bfs_blast's assign / masked vxm / reduce per level, a host read per level"})
    lab, ms = twice(G.cc)
    ref = R.cc(g) if R else (None, None)
    rec("cc", ms, ref[1], None if ref[0] is None else bool(np.array_equal(lab, ref[0])),
        {"path": "gbk_cc_labels: union-find, three launches"})
    lab2, it2, ms2 = twice(G.cc_fastsv)
    rec("cc_fastsv_calls", ms2, ref[1], None if ref[0] is None else bool(np.array_equal(lab2, ref[0])),
        {"iterations": it2, "path": "cc.hpp's FastSV GraphBLAS calls, a host read per iteration"})
    d, ms = twice(lambda: G.sssp_f32(int(src[2])))
    ref = R.sssp(g, w, int(src[2])) if R else (None, None)
    rec("sssp", ms, ref[1], None if ref[0] is None else bool(np.array_equal(d, ref[0])))
    r, it, ms = twice(lambda: G.pagerank(itermax=100, damping=0.85, tol=1e-6))
    r64, _, _ = Oracle().pagerank(g, tol=0.0, itermax=it)
    gpu_err = float(np.abs(r - r64).sum() / np.abs(r64).sum())
    ref = R.pagerank(g, it) if R else (None, None)
    ref_err = None if ref[0] is None else float(np.abs(ref[0] - r64).sum() / np.abs(r64).sum())
    err = None if ref[0] is None else float(np.abs(r - ref[0]).sum() / np.abs(ref[0]).sum())
    # PageRank's criterion is the FP64 oracle (1e-5 relative L1): the
    # reference's own FP32 result is itself ~1e-3 from it at this size
    rec("pagerank", ms, ref[1], bool(gpu_err < 1e-5),
        {"iterations": it, "criterion": "rel. L1 < 1e-5 vs the FP64 oracle", "rel_l1_vs_reference": err,
         "rel_l1_vs_fp64_oracle": gpu_err, "reference_rel_l1_vs_fp64_oracle": ref_err,
         "sinks_fraction": float((np.bincount(g.col, minlength=g.n) == 0).mean())})
    t, ms = twice(G.tc)
    rec("tc", ms, None, None, {"triangles": t, "reference": "not run at this scale (bounded CPU sample)"})
    # triangle counting against the reference on a smaller graph of the same family
    ts = 17 if light else max(10, args.alg_scale - 4)
    gs = gg.rmat(ts, args.edge_factor, seed=args.seed, undirected=True)
    Gs = lc.Graph(gs)
    ts_cnt, ts_ms = twice(Gs.tc)
    ref = R.tc(gs) if R else (None, None)
    res["tc_small"] = {"scale": ts, "gpu_ms": round(ts_ms, 3), "ref_cpu_ms": None if ref[1] is None else round(ref[1], 1),
                       "speedup": None if not ref[1] else round(ref[1] / ts_ms, 1),
                       "matches_reference": None if ref[0] is None else ref[0] == ts_cnt, "triangles": ts_cnt}
    if light:
        G.close()
        Gs.close()
        return {"config": {"workload": f"algorithms_rmat{args.alg_scale}u", "n": g.n, "nnz": g.nnz},
                "algorithms": res}
    # unmasked SpGEMM A (+.x) A (SpMSpM_unmasked_ikj) on a smaller graph of the same family
    ms_scale = max(10, args.alg_scale - 8)
    gm = gg.rmat(ms_scale, args.edge_factor, seed=args.seed, undirected=True)
    vm = gg.values_f32(gm, seed=args.seed + 5)
    Am = capi.Matrix.from_graph(gm, vm)
    Am.mxm(Am).close()  # warm-up (allocations, CUB scratch)
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Cm = Am.mxm(Am)
    torch.cuda.synchronize()
    mxm_ms = (time.perf_counter() - t0) * 1e3
    deg = np.diff(gm.row_ptr).astype(np.int64)
    products = int(deg[gm.col].sum())
    cnnz = Cm.nnz
    ref = R.mxm(gm, vm, 0) if R else None
    same = None
    if ref is not None:
        rp, col, v = Cm.download_csr()
        rrp, rcol, rv, ref_ms = ref
        rows = np.repeat(np.arange(gm.n), np.diff(rrp))
        o = np.lexsort((rcol, rows))
        same = bool(np.array_equal(rp, rrp) and np.array_equal(col, rcol[o]) and np.allclose(v, rv[o], rtol=2e-6))
    res["mxm_unmasked"] = {"scale": ms_scale, "gpu_ms": round(mxm_ms, 3), "products": products, "nnz_c": cnnz,
                           "G_products_per_s": round(products / (mxm_ms * 1e-3) / 1e9, 3),
                           "ref_cpu_ms": None if ref is None else round(ref[3], 1),
                           "speedup": None if ref is None else round(ref[3] / mxm_ms, 1), "matches_reference": same}
    Cm.close()
    Am.close()
    out = {
        "metric": "full algorithms: device time per run vs the reference CPU code", "value": res["bfs"]["gteps"],
        "unit": "GTEPS (BFS)", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": res["bfs"]["gpu_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 / i32",
        "data": "synthetic (seeded R-MAT, generated in-process)",
        "config": {"workload": f"algorithms_rmat{args.alg_scale}u", "n": g.n, "nnz": g.nnz,
                   "graph": f"R-MAT scale {args.alg_scale}, edge factor {args.edge_factor}, undirected",
                   "timing": "host timer around each lablas:: algorithm call (device work synchronised), "
                             "second of two runs on the same inputs"},
        "algorithms": res,
        "cpu_baseline": None if R is None else {"value": res["bfs"]["ref_cpu_ms"], "unit": "ms (BFS)",
                                                "cores": R.max_threads(), "kind": "reference",
                                                "sample": "one run per algorithm on the same graph"},
    }
    return out


def run_ingest(args):
    """Graph file -> device CSR (lablas::Matrix<T>::init_from_mtx, read_file.hpp:565-617) for the R-MAT
    graph written as .mtx text and as .mtxbin, the CSR cache reload, and the reference's own reader on the
    same files.  Files sit in a temporary directory on the local disk and are read warm (page cache): the
    first read of each is untimed, then the median of --ingest-reps timed reads."""
    import shutil
    import tempfile
    import torch
    from gb_kun_b200 import capi, graphgen as gg
    capi.init(0)
    g = gg.rmat(args.scale, args.edge_factor, seed=args.seed)
    s, d = gg.edge_list(g)
    tmp = Path(tempfile.mkdtemp(prefix="gbk_ingest_"))
    try:
        f_mtx, f_bin, f_csr = tmp / "g.mtx", tmp / "g.mtxbin", tmp / "g.gbkcsr"
        gg.write_mtx(f_mtx, g.n, g.n, s, d)
        gg.write_mtxbin(f_bin, g.n, g.n, s, d)

        def timed(path):
            ts, A = [], None
            for i in range(args.ingest_reps + 1):
                if A is not None:
                    A.close()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                A = capi.Matrix.from_file(path)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
            return A, statistics.median(ts[1:])

        def same(A):
            rp, col, val = A.download_csr()
            return bool(np.array_equal(rp, g.row_ptr) and np.array_equal(col, g.col) and np.all(val == 1))

        A, t_mtx = timed(f_mtx)
        ok_mtx = same(A)
        A.save_csr(f_csr)
        A.close()
        B, t_bin = timed(f_bin)
        ok_bin = same(B)
        B.close()
        Cm, t_csr = timed(f_csr)
        Cm.close()
        sizes = {k: os.path.getsize(f) for k, f in (("mtx", f_mtx), ("mtxbin", f_bin), ("gbkcsr", f_csr))}
        # the link every file byte crosses once: pinned host -> device copy bandwidth
        hb = torch.empty(1 << 30, dtype=torch.uint8).pin_memory()
        db = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
        db.copy_(hb, non_blocking=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            db.copy_(hb, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        h2d_gbs = 5 * (1 << 30) / (e0.elapsed_time(e1) * 1e-3) / 1e9
        del hb, db
        R = _ref_threads()
        ref = {}
        if R is not None:
            for kind, f in (("mtx", f_mtx), ("mtxbin", f_bin)):
                n, rp, col, val, ms = R.graph_read(f)
                rows_equal = bool(np.array_equal(rp, g.row_ptr))
                ref[kind] = {"ms": round(ms, 1), "MB_per_s": round(sizes[kind] / (ms * 1e-3) / 1e6, 1),
                             "same_csr_as_ours": rows_equal and bool(np.array_equal(col, g.col)) if kind == "mtx"
                             else rows_equal}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    mbs = sizes["mtx"] / t_mtx / 1e6
    out = {
        "metric": "graph file ingest: .mtx text into device CSR (MB of file per second)", "value": round(mbs, 1),
        "unit": "MB/s", "n_gpus": 1, "steps": args.ingest_reps, "warmup": 1, "ms_per_step": round(t_mtx * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32 ids",
        "data": "synthetic (seeded R-MAT written as .mtx / .mtxbin in a temporary directory)",
        "config": {"workload": f"ingest_rmat{args.scale}", "n": g.n, "nnz": g.nnz, "file_bytes": sizes,
                   "timing": "host timer around gbk_matrix_create_from_file (device synchronised), warm page "
                             "cache, median of --ingest-reps after one untimed read"},
        "mtx": {"ms": round(t_mtx * 1e3, 2), "MB_per_s": round(mbs, 1),
                "M_entries_per_s": round(g.nnz / t_mtx / 1e6, 1), "bit_exact": ok_mtx},
        "mtxbin": {"ms": round(t_bin * 1e3, 2), "MB_per_s": round(sizes["mtxbin"] / t_bin / 1e6, 1),
                   "bit_exact": ok_bin},
        "csr_cache": {"ms": round(t_csr * 1e3, 2), "MB_per_s": round(sizes["gbkcsr"] / t_csr / 1e6, 1)},
        "roofline": {"bound": "host-to-device link (every file byte crosses it once)", "achieved": round(mbs / 1e3, 2),
                     "peak": round(h2d_gbs, 2), "unit": "GB/s", "frac": round(mbs / 1e3 / h2d_gbs, 3),
                     "peak_source": "measured here: pinned 1 GiB host-to-device copies"},
        "reference": ref,
        "cpu_baseline": None if not ref else {
            "value": ref["mtx"]["MB_per_s"], "unit": "MB/s", "cores": R.max_threads(), "kind": "reference",
            "sample": "one init_from_mtx of the same .mtx file (read_mtx_file_pipelined + CSR/CSC build)"},
    }
    if ref:
        out["speedup_vs_reference"] = {k: round(ref[k]["ms"] / (1e3 * (t_mtx if k == "mtx" else t_bin)), 1)
                                       for k in ref}
    return out


def run_spgemm(args):
    """Sparse products on undirected R-MAT (--spgemm-scale): unmasked A (+.x) A (SpMSpM_unmasked_ikj), the
    masked plus-one product C<A> = A A of Burkhardt's triangle count (SpMSpM_masked_ikj), and the triangle
    count itself, each against the reference CPU code on the same graph (second of two runs timed)."""
    import torch
    from gb_kun_b200 import capi, graphgen as gg
    capi.init(0)
    g = gg.rmat(args.spgemm_scale, args.edge_factor, seed=args.seed, undirected=True)
    val = gg.values_f32(g, seed=args.seed + 5)
    A = capi.Matrix.from_graph(g, val)
    Ai = capi.Matrix.from_graph(g, np.ones(g.nnz, np.int32))
    R = _ref_threads()

    def timed(fn):
        out = fn()
        if hasattr(out, "close"):
            out.close()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, (time.perf_counter() - t0) * 1e3

    deg = np.diff(g.row_ptr).astype(np.int64)
    products = int(deg[g.col].sum())
    C, mxm_ms = timed(lambda: A.mxm(A))
    res = {"mxm_unmasked": {"gpu_ms": round(mxm_ms, 3), "products": products, "nnz_c": C.nnz,
                            "G_products_per_s": round(products / (mxm_ms * 1e-3) / 1e9, 3)}}
    if R is not None:
        rp, col, v = C.download_csr()
        rrp, rcol, rv, ref_ms = R.mxm(g, val, 0)
        rows = np.repeat(np.arange(g.n), np.diff(rrp))
        o = np.lexsort((rcol, rows))
        res["mxm_unmasked"].update({"ref_cpu_ms": round(ref_ms, 1), "speedup": round(ref_ms / mxm_ms, 1),
                                    "matches_reference": bool(np.array_equal(rp, rrp) and np.array_equal(col, rcol[o])
                                                              and np.allclose(v, rv[o], rtol=2e-6))})
    C.close()
    tri, tc_ms = timed(lambda: Ai.triangle_count())
    res["triangle_count"] = {"gpu_ms": round(tc_ms, 3), "triangles": tri}
    from gb_kun_b200 import lablas_capi as lc
    G = lc.Graph(g)
    mtri, mtc_ms = timed(lambda: G.tc_method(2)[0])  # Cohen: select + masked plus-one product
    res["triangle_count_masked_product"] = {"gpu_ms": round(mtc_ms, 3), "triangles": mtri}
    if R is not None:
        rtri, rms = R.tc(g)
        res["triangle_count"].update({"ref_cpu_ms": round(rms, 1), "speedup": round(rms / tc_ms, 1),
                                      "matches_reference": rtri == tri})
        res["triangle_count_masked_product"]["matches_reference"] = rtri == mtri
    out = {
        "metric": "sparse products: unmasked A*A G products/s; triangle count vs the reference CPU code",
        "value": res["mxm_unmasked"]["G_products_per_s"], "unit": "G products/s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": res["mxm_unmasked"]["gpu_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 / i32", "data": "synthetic (seeded R-MAT, generated in-process)",
        "config": {"workload": f"spgemm_rmat{args.spgemm_scale}u", "n": g.n, "nnz": g.nnz,
                   "timing": "host timer around each call (device synchronised), second of two runs"},
        "products": res,
        "cpu_baseline": None if R is None else {"value": res["mxm_unmasked"].get("ref_cpu_ms"), "unit": "ms (A*A)",
                                                "cores": R.max_threads(), "kind": "reference",
                                                "sample": "one unmasked mxm and one LAGr_TriangleCount"},
    }
    return out


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.cpu import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU library not built (oracle/_ref)"}))
        return
    g, val, x = make_input(args)
    R = Reference()
    fmt = REF_FORMAT[args.format]
    steps = max(1, args.steps)
    warm = max(0, args.warmup)
    _, ms = R.spmv(g, val, x, fmt=fmt, semiring=0, warmup=warm, reps=steps)
    B = alg_bytes(g)
    value = B / (ms * 1e-3) / 1e9
    cfg = workload_config(args, g)
    cfg["parallelism"] = "single"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": steps, "warmup": warm, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded R-MAT, generated in-process)",
        "config": cfg,
        "format_ran": {"format": REF_FORMAT_NAME[fmt], "note": "the reference's fastest format in its own SpMV "
                                                               "measurements; OpenMP threads = all host threads"},
        "cpu_baseline": {"value": round(value, 2), "unit": "GB/s", "cores": R.max_threads(), "cpu_model": cpu_model(),
                         "kind": "reference", "sample": f"full matrix, median of {steps} GrB_mxv calls after "
                                                        f"{warm} warm-up calls"},
        "e2e": {"value": round(value, 2), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    args = parse()
    if args.mode != "spmv":
        out = {"batched": run_batched, "serve": run_serve, "algorithms": run_algorithms, "single": run_single,
               "ingest": run_ingest, "spgemm": run_spgemm}[args.mode](args)
        print(json.dumps(out), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
