"""Benchmark: non-rigid Gauss-Newton solves per second on B200.

Workload (one step): a batch of independent multi-view solves, each 3 views at
640x480 around a torso-like ellipsoid, 4096 nodes, 8-NN graph, 4-NN skinning,
all terms (dense depth, foreground mask, 1000 sparse feature pairs per view,
2000 cross-view pairs per adjacent view pair), 5 Gauss-Newton x 15 PCG
iterations, mixed precision (float Jacobians and PCG vectors; double residual
chain, JtJ blocks, reductions and block Cholesky).
Each instance shares the synthetic geometry and has its own random initial
warp field. Every step re-binds the inputs (which resets each warp field) and
runs the index build plus all Gauss-Newton iterations of every instance. The
16 instances are solved in two lanes of 8 (`--streams`): each lane is a
member batch whose whole solve is one captured CUDA graph on a stream of its
own, so one lane's kernels run in the gaps that the other's latency-bound
kernels leave.

Outputs one JSON line (rank 0). `value` uses inputs resident in HBM; `e2e`
uploads every input from pinned host memory and reads every solved warp field
back inside the timed region. `--impl reference` times the CPU restatement of
the reference algorithm (the reference itself cannot be built here) on all
host cores, one instance per thread.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0
WORKLOAD = "torso_3view_640x480_4096nodes_5gn_15pcg"
METRIC = "non-rigid GN solves/s (batched mixed vs plain FP32) at <=1e-4 rel err vs FP64"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batch", type=int, default=16, help="instances per GPU")
    p.add_argument("--streams", type=int, default=2,
                   help="lanes of the timed batch: member batches of batch/streams instances, each solved as its "
                        "own graph on its own stream (1: one batch, one graph)")
    p.add_argument("--nodes", type=int, default=4096)
    p.add_argument("--width", type=int, default=640)
    p.add_argument("--height", type=int, default=480)
    p.add_argument("--gn", type=int, default=5)
    p.add_argument("--pcg", type=int, default=15)
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp32"])
    p.add_argument("--mode", default="materialized", choices=["materialized", "matrix_free"])
    p.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison leg")
    p.add_argument("--pcg-persistent", action="store_true",
                   help="run each PCG solve as one persistent cooperative launch")
    p.add_argument("--spmv-shape", type=int, default=-1,
                   help="use this SpMV tile shape (index into abi.SPMV_SHAPES) instead of the autotuner's")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--workload", default="torso", choices=["torso", "sphere", "uneven", "body", "solver_maps", "deform"],
                   help="torso: the headline batch (default); sphere: the 1-view 2048-node plain-method "
                        "configuration; uneven: 16 instances with 1024-16384 nodes and 1-4 views; body: one "
                        "32768-node, 5-view 1280x720 solve; solver_maps: the renderer's solver maps of the "
                        "body workload's surfels in its 5 views; deform: the post-solve warp, node error and "
                        "correction on the body workload")
    p.add_argument("--no-accuracy", action="store_true", help="skip the FP64 check of the timed configuration")
    p.add_argument("--no-e2e", action="store_true",
                   help="skip the end-to-end leg (for profiler captures only; the bench line then has no e2e)")
    return p.parse_args()


def instance_seeds(rank, batch):
    """Seeds of the initial warp fields of one rank's instances: every rank
    solves its own, disjoint set of instances (weak scaling, no collective in
    the solve)."""
    return [1000 * rank + i for i in range(batch)]


def max_over_ranks(ms, dist, device):
    """The slowest rank's time; every rank must call it (one all-reduce)."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, batch, ms):
    """Whole-job solves/s: all ranks' instances over the slowest rank's time."""
    return world * batch / (ms / 1e3)


def make_scenes(args, rank):
    from multiviewdynrecon_b200 import synth
    base = synth.torso_multi_view(seed=2, num_nodes=args.nodes, width=args.width, height=args.height)
    scenes = [synth.perturb_warp_field(base, seed=sd) for sd in instance_seeds(rank, args.batch)]
    return base, scenes


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples every 100 ms while the timed region
    runs (one streaming nvidia-smi process)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._proc = None
        self._t = None

    def _read(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                           "--format=csv,noheader,nounits", "-lms", "100"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def __exit__(self, *a):
        if self._proc is not None:
            time.sleep(0.15)  # one more sample after the region
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            if self._t:
                self._t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


PROFILE_SPMV = "profiles/pcg_spmv_scaled_torso_3view_4096nodes_16inst.md"
PROFILE_MATRIX_FREE = "profiles/apply_pair_matrix_free_torso_3view_4096nodes_8inst.md"


def measured_traffic(args):
    """DRAM bytes (read + write) per launch of the roofline kernel from the ncu
    capture of this workload summarised under profiles/: the headline SpMV
    (pcg_spmv_scaled_kernel, PROFILE_SPMV) or, in the matrix-free mode, the
    product pair (PROFILE_MATRIX_FREE, an 8-instance capture scaled to the
    batch: each instance moves the same bytes); None for other workloads or
    when no summary exists."""
    default = (args.batch == 16 and args.nodes == 4096 and args.width == 640 and args.height == 480
               and args.precision == "mixed")
    if not default:
        return None, None
    import re
    if args.mode == "materialized":
        rel, row, scale = PROFILE_SPMV, "| DRAM read + write |", 1.0
    else:
        rel, row, scale = PROFILE_MATRIX_FREE, "| DRAM bytes (rate x duration) |", args.batch / 8.0
    path = os.path.join(ROOT, rel)
    if not os.path.exists(path):
        return None, None
    with open(path) as f:
        for line in f:
            if line.startswith(row):
                # the first number of each of the next two cells (SpMV: "R + W MB";
                # matrix-free: one cell per kernel)
                cells = line.split("|")[2:4] if rel == PROFILE_MATRIX_FREE else [line.split("|")[2]]
                nums = [float(x) for c in cells for x in re.findall(r"[0-9]+(?:\.[0-9]+)?", c)[:2]]
                if len(nums) >= 2:
                    return int((nums[0] + nums[1]) * 1e6 * scale), rel
    return None, None


def spmv_tile_desc(shape):
    """The SpMV tile shape (rows, split, form) in words."""
    rows, split, form = shape
    return {"rows_per_cta": rows, "threads_per_row": 6 * split,
            "lower_blocks": "row reads, shared-memory exchange" if form == 0 else "column reads"}


def spmv_tile_label(shape):
    rows, split, form = shape
    return f"{'row' if form == 0 else 'col'}{rows}x{6 * split}"


def algorithmic_bytes(counts, N, mixed=True, materialized=True):
    """Compulsory HBM bytes per stage and instance (each array read or written
    once). JtJ is kept as half storage (N diagonal + P upper 6x6 blocks) with
    N + 2P entries of (position, column) in the full block-row layout.
    Mixed precision, materialised: the assembly writes the blocks in double,
    the scaling turns the P upper blocks into float blocks of the
    block-Jacobi scaled operator, whose identity diagonal the SpMV does not
    read; the SpMV reads the float copy of the direction (24 B per node) and
    the double direction (48 B) and the residual (48 B, for r.q), and writes
    the double product (48 B); the PCG update needs no preconditioner and
    forms the next direction (the direction kernel runs once per solve).
    Plain FP32: float blocks with the diagonal, float vectors, the 6x6
    inverse per node."""
    Td, Ts, Tf, Tp, Tc = (counts.dense_terms, counts.smooth_terms, counts.foreground_terms, counts.feature_terms,
                          counts.cross_terms)
    P = counts.half_pairs
    elem = 8 if mixed else 4
    scaled = mixed and materialized
    term_data = 52 * (Td + Tf) + 29 * Ts + 88 * (Tp + Tc)
    precond = 168 * N if mixed else 144 * N
    if scaled:
        spmv = 144 * P + 8 * 2 * P + 4 * (N + 1) + 24 * N + 48 * N + 48 * N + 48 * N
        direction = 3 * 48 * N + 24 * N      # r and d_prev read, d and its float copy written
        pcg_update = 7 * 48 * N + 32 * N      # x rw, r rw, d, q read; next d and its padded float copy written
    else:
        spmv = 36 * elem * (N + P) + 8 * (N + 2 * P) + 4 * (N + 1) + 2 * 6 * elem * N
        direction = 3 * 6 * elem * N          # s and d_prev read, d written
        pcg_update = 7 * 6 * elem * N + precond  # x rw, r rw, d, q read, s written
    # index build (once per solve), the per-unit bytes of a radix-sort build:
    # the node -> term pairs (6 B) read and written once per 8-bit pass over
    # ceil(log2 N) key bits, their scan; the node-pair pairs (8 B) over
    # 2 ceil(log2 N) key bits; the symmetric pass over 2P entries of 12 B
    lg = max(1, math.ceil(math.log2(max(N, 2))))
    K1, K2 = counts.node2term_entries, counts.nodepair_entries
    index = (6 * K1 * 2 * math.ceil(lg / 8) + 8 * K1 + 8 * K2 * 2 * math.ceil(2 * lg / 8) + 2 * (2 * P) * 12)
    return {
        "index": index,
        "terms": 122 * Td + 86 * Tf + 29 * Ts + 72 * (Tp + Tc) + 32 * N,
        "diag": term_data + 4 * counts.node2term_entries + 144 * N + 36 * elem * N + 24 * N + precond,
        "offdiag": term_data + 4 * counts.nodepair_entries + 12 * P + 36 * elem * P,
        # the double upper blocks and their pair keys read, the float scaled blocks
        # written, each node's Cholesky factor read once
        "scale": 288 * P + 4 * P + 144 * P + 168 * N,
        "spmv": spmv,
        "direction": direction,
        "pcg_update": pcg_update,
        "update": 24 * N + 64 * N,
        # matrix-free product: J.d reads each term's record, nodes and weights
        # (pixel 56 B, smooth 52 B, point-to-point 56 B) and d, and writes J.d
        # (one value per pixel term, three otherwise); Jt reads the node-term
        # entries and their weights, each pixel record again (32 B) or the
        # other terms' data, J.d and d, and writes q
        "matrix_free": (56 * (Td + Tf) + 52 * Ts + 56 * (Tp + Tc) + elem * (Td + Tf) + 3 * elem * (Ts + Tp + Tc)
                        + 6 * elem * N)
                       + (8 * counts.node2term_entries + 4 * (N + 1) + 32 * (Td + Tf) + 52 * Ts + 56 * (Tp + Tc)
                          + elem * (Td + Tf) + 3 * elem * (Ts + Tp + Tc) + 12 * elem * N),
    }


def run_ours(args, rank, world, dist):
    import torch
    from multiviewdynrecon_b200 import abi, lib
    from multiviewdynrecon_b200.solver import BatchSolver, DeviceScene, NonRigidSolver, StreamedBatch

    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    base, scenes = make_scenes(args, rank)
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP32
    mode = abi.MODE_MATERIALIZED if args.mode == "materialized" else abi.MODE_MATRIX_FREE
    cfg = abi.make_config(base, precision=prec, mode=mode)
    B = args.batch
    batch = BatchSolver(cfg, B)
    dev_scenes = [DeviceScene(s) for s in scenes]
    stream = torch.cuda.Stream()

    def bind_all():
        for i, ds in enumerate(dev_scenes):
            batch.set_input(i, ds, stream=stream)

    # SpMV tile shape for this workload (one timed sweep of the candidates,
    # or the shape given on the command line)
    with torch.cuda.stream(stream):
        bind_all()
        if args.pcg_persistent:
            batch.set_pcg_persistent(True)
        if args.spmv_shape >= 0:
            batch.set_spmv_shape(args.spmv_shape)
            spmv_shape, spmv_shape_ms = abi.SPMV_SHAPES[args.spmv_shape], []
        else:
            spmv_shape, spmv_shape_ms = batch.autotune(stream=stream)

    # the timed solver: the batch itself, or its instances in lanes of
    # concurrent graphs on streams of their own (same tile shape, same
    # arithmetic per instance)
    if args.streams > 1:
        timed = StreamedBatch(cfg, B, lanes=args.streams)
        timed.set_spmv_shape(abi.SPMV_SHAPES.index(tuple(spmv_shape)))
        if args.pcg_persistent:
            timed.set_pcg_persistent(True)
    else:
        timed = batch

    def bind_timed():
        for i, ds in enumerate(dev_scenes):
            timed.set_input(i, ds, stream=stream)

    def step():
        bind_timed()
        timed.solve(args.gn, args.pcg, use_graph=True, stream=stream)

    # kernels per solve: one direct (non-graph) solve counted through the ABI
    with torch.cuda.stream(stream):
        bind_timed()
        k0 = lib().mvdr_kernel_launch_count()
        timed.solve(args.gn, args.pcg, use_graph=False, stream=stream)
        kernels_per_step = lib().mvdr_kernel_launch_count() - k0
        stream.synchronize()
        for _ in range(args.warmup):
            step()
        stream.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clocks, torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, "cuda")
    if dist:
        dist.barrier()
    value = job_value(world, B, ms)

    # instance 0's counts, from the timed solver (solved in the timed region)
    inst0 = timed.instance(0)
    counts = inst0.counts()

    # per-stage timing on the same stream (CUDA events), all instances
    stages = {}
    abytes = algorithmic_bytes(counts, base.num_nodes, mixed=args.precision == "mixed",
                               materialized=mode == abi.MODE_MATERIALIZED)
    reps = 20
    with torch.cuda.stream(stream):
        bind_all()
        batch.solve(args.gn, args.pcg, use_graph=True, stream=stream)
        stream.synchronize()
        # the PCG operator: the SpMV over the materialised blocks, or the
        # matrix-free pair (J.d per term, then Jt per node)
        op = ("spmv", abi.STAGE_SPMV) if mode == abi.MODE_MATERIALIZED else ("matrix_free", abi.STAGE_MATRIX_FREE)
        for name, sid in (("index", abi.STAGE_INDEX), ("terms", abi.STAGE_TERMS), ("diag", abi.STAGE_DIAG),
                          ("offdiag", abi.STAGE_OFFDIAG), ("scale", abi.STAGE_SCALE), op,
                          ("direction", abi.STAGE_DIRECTION), ("pcg_update", abi.STAGE_PCG_UPDATE),
                          ("update", abi.STAGE_UPDATE)):
            if name in ("offdiag", "scale") and mode != abi.MODE_MATERIALIZED:
                continue
            if name == "scale" and args.precision != "mixed":
                continue
            for _ in range(2):
                lib().mvdr_batch_enqueue_stage(batch.h, sid, stream.cuda_stream)
            a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(reps):
                lib().mvdr_batch_enqueue_stage(batch.h, sid, stream.cuda_stream)
            b2.record(stream)
            b2.synchronize()
            t_ms = a.elapsed_time(b2) / reps
            entry = {"ms": round(t_ms, 5)}
            if name in abytes:
                gb = B * abytes[name] / 1e9
                entry["GB_per_launch"] = round(gb, 6)
                entry["GBps"] = round(gb / (t_ms / 1e3), 1)
            stages[name] = entry
    peak, peak_kind = load_peaks()
    if mode == abi.MODE_MATERIALIZED:
        spmv = stages["spmv"]
        spmv_bytes = B * abytes["spmv"]
        if args.precision == "mixed":
            kernel = "pcg_spmv_scaled_kernel"
        else:
            kernel = "pcg_spmv_col_kernel" if spmv_shape[2] == 1 else "pcg_spmv_kernel"
        traffic, traffic_src = measured_traffic(args)
    else:
        spmv = stages["matrix_free"]
        spmv_bytes = B * abytes["matrix_free"]
        kernel = "apply_j_kernel + apply_jt_kernel"
        traffic, traffic_src = measured_traffic(args)
    roofline = {"kernel": kernel, "bound": "hbm", "achieved": spmv["GBps"], "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s", "frac": round(spmv["GBps"] / peak, 4),
                "traffic": traffic, "traffic_source": traffic_src, "algorithmic_bytes_per_launch": spmv_bytes,
                "launch_ms": spmv["ms"]}

    # e2e: host buffers -> device copies -> solve -> warp fields back to host.
    # Two batch solvers alternate. Uploads run on two copy streams (alternate
    # instances, so two DMA engines share the PCIe link) while the previous
    # step solves on the compute stream; a batch's upload waits for that
    # batch's previous solve. Every step still uploads all of its inputs and
    # reads back all of its warp fields inside the timed region.
    e2e = None
    if args.no_e2e:
        host_scenes = []
    else:
        host_scenes = [DeviceScene(s, pin=True) for s in scenes]
    if not args.no_e2e:
        e2e_batches = [batch, BatchSolver(cfg, B)]
        for i, ds in enumerate(dev_scenes):
            e2e_batches[1].set_input(i, ds, stream=stream)
        if args.pcg_persistent:
            e2e_batches[1].set_pcg_persistent(True)
        if args.spmv_shape >= 0:
            e2e_batches[1].set_spmv_shape(args.spmv_shape)
        else:
            e2e_batches[1].autotune(stream=stream)
        # two copy streams, so that two DMA engines share the uploads
        copy_streams, solve_stream = [torch.cuda.Stream(), torch.cuda.Stream()], stream
        copy_stream = copy_streams[0]
        uploaded = [[torch.cuda.Event(), torch.cuda.Event()] for _ in range(2)]
        solved = [torch.cuda.Event(), torch.cuda.Event()]
        out_host = [[torch.empty((s.num_nodes, 8), dtype=torch.float32, pin_memory=True) for s in scenes]
                    for _ in range(2)]
        h2d = sum(hs.nbytes for hs in host_scenes)
        d2h = sum(o.numel() * 4 for o in out_host[0])

        def e2e_step(k):
            j = k % 2
            bt = e2e_batches[j]
            for cs in copy_streams:
                cs.wait_event(solved[j])  # this batch's previous solve and readback are done
            for i, hs in enumerate(host_scenes):
                bt.set_input_host(i, hs, stream=copy_streams[i % 2])
            for cs, ev in zip(copy_streams, uploaded[j]):
                ev.record(cs)
                solve_stream.wait_event(ev)
            bt.solve(args.gn, args.pcg, use_graph=True, stream=solve_stream)
            for i in range(B):
                bt.node_se3_async(i, out_host[j][i], stream=solve_stream)
            solved[j].record(solve_stream)

        for k in range(max(2, args.warmup)):
            e2e_step(k)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(copy_stream)
        copy_streams[1].wait_event(a)
        solve_stream.wait_event(a)
        for k in range(args.steps):
            e2e_step(k)
        b2.record(solve_stream)
        b2.synchronize()
        e2e_ms = max_over_ranks(a.elapsed_time(b2) / args.steps, dist, "cuda")
        e2e = {"value": round(job_value(world, B, e2e_ms), 3), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3),
               "pipeline": "uploads on two copy streams (alternate instances), overlapping the previous step's "
                           "solve"}
        for bt in e2e_batches:  # device-side error record of every e2e solve
            for i in range(B):
                if bt.instance(i).counts().error_flags:
                    raise RuntimeError(f"e2e solve of instance {i} flagged errors")
        e2e_batches[1].close()

    # plain FP32 form: one instance at a time, per-kernel launches, float dots
    plain = None
    if not args.no_plain:
        pcfg = abi.make_config(base, precision=abi.PRECISION_FP32, mode=mode)
        single = NonRigidSolver(pcfg)
        n_plain = min(B, 4)
        with torch.cuda.stream(stream):
            for _ in range(2):
                single.set_solver_input(dev_scenes[0], stream=stream)
                single.solve_non_rigid_alignment(args.gn, args.pcg, stream=stream)
            stream.synchronize()
            a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for i in range(n_plain):
                single.set_solver_input(dev_scenes[i], stream=stream)
                single.solve_non_rigid_alignment(args.gn, args.pcg, stream=stream)
            b2.record(stream)
            b2.synchronize()
        p_ms = a.elapsed_time(b2) / n_plain
        plain = {"value": round(1e3 / p_ms, 3), "unit": "solves/s", "ms_per_solve": round(p_ms, 4),
                 "form": "plain FP32, one instance per solve, no graph"}
        single.close()
        # the same FP32 arithmetic batched and graph-replayed like the headline,
        # to separate the gain of the precision scheme from that of batching
        pb = StreamedBatch(pcfg, B, lanes=args.streams) if args.streams > 1 else BatchSolver(pcfg, B)
        with torch.cuda.stream(stream):
            def pstep():
                for i, ds in enumerate(dev_scenes):
                    pb.set_input(i, ds, stream=stream)
                pb.solve(args.gn, args.pcg, use_graph=True, stream=stream)
            pstep()
            if args.spmv_shape >= 0:
                pb.set_spmv_shape(args.spmv_shape)
            else:
                pb.autotune(stream=stream)
            pb_ms = time_solves(pstep, max(3, args.steps // 4), max(3, args.warmup), stream)
        plain["batched_graph"] = {"value": round(B * 1e3 / pb_ms, 3), "unit": "solves/s",
                                  "ms_per_step": round(pb_ms, 4),
                                  "form": f"plain FP32, {B} instances in {max(1, args.streams)} concurrent "
                                          f"graph lanes (as the headline)"}
        pb.close()

    # the PCG residual history of instance 0's last timed solve: delta_k /
    # delta_0 at the start of every PCG iteration, first and last GN iteration
    pcg_history = None
    with torch.cuda.stream(stream):
        bind_timed()
        timed.solve(args.gn, args.pcg, use_graph=True, stream=stream)
        stream.synchronize()
    hist = timed.instance(0).get_array(abi.ARRAY_PCG_RESIDUALS)
    if len(hist):
        def ratios(row):
            row = row[np.isfinite(row)]
            return [float("%.3g" % (v / row[0])) for v in row] if len(row) else []
        pcg_history = {"delta_over_delta0_gn_first": ratios(hist[0]), "delta_over_delta0_gn_last": ratios(hist[-1]),
                       "instance": "0 of the timed batch", "iterations": args.pcg}

    # accuracy of the timed configuration: instance 0's solve, every
    # Gauss-Newton increment against the FP64 oracle (after the timed region)
    accuracy = None
    if not args.no_accuracy:
        with torch.cuda.stream(stream):
            errs, eerrs = increment_errors_vs_fp64(scenes[0], cfg, args.gn, args.pcg, batch=timed, bind=bind_timed,
                                                   stream=stream)
        accuracy = {"dx_rel_err_vs_fp64": [float("%.3g" % e) for e in errs],
                    "dx_rel_err_max": float("%.3g" % max(errs)),
                    "energy_rel_err_vs_fp64_max": float("%.3g" % max(eerrs)),
                    "instance": "0 of the timed batch", "bar": 1e-4,
                    "method": "each GN increment vs the FP64 oracle linearised at the GPU's warp field of that "
                              "iteration, with the GPU's projected pixels and validity decisions"}

    return dict(value=value, ms=ms, kernels_per_step=kernels_per_step, clocks=clocks.summary(), stages=stages,
                spmv_tile=dict(spmv_tile_desc(spmv_shape),
                               candidates_ms={spmv_tile_label(sh): round(t, 5)
                                              for sh, t in zip(abi.SPMV_SHAPES, spmv_shape_ms)}),
                roofline=roofline, e2e=e2e, plain=plain, counts=counts, base=base, accuracy=accuracy,
                pcg_history=pcg_history)


def first_increment_errors(scenes, cfg_for, gpu_increments, pcg, threads):
    """Relative 2-norm error of the first Gauss-Newton increment of each
    instance against the FP64 oracle, with the GPU's pixel and validity
    decisions (host threads; the oracle's ctypes calls release the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    import oracle
    from multiviewdynrecon_b200 import abi

    def one(k):
        sc, (jr, sm, x) = scenes[k], gpu_increments[k]
        o = oracle.Oracle(sc, cfg_for(sc), fp64=True)
        o.build_index()
        o.freeze(jr, sm)
        o.eval_terms()
        o.assemble()
        o.pcg(pcg)
        x64 = o.get(abi.ARRAY_INCREMENT, as_double=True).reshape(-1)
        return float(np.linalg.norm(x.reshape(-1) - x64) / max(np.linalg.norm(x64), 1e-300))

    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(one, range(len(scenes))))


def increment_errors_vs_fp64(scene, cfg, gn, pcg, batch=None, bind=None, stream=None):
    """Every Gauss-Newton increment of one instance's solve against the FP64
    oracle linearised at the GPU's warp field of that iteration, with the
    GPU's projected pixels and validity decisions (relative 2-norm), and each
    iteration's energy against the oracle's. With `batch` (and `bind`, which
    rebinds every instance) the instance is instance 0 of that batch, solved
    with 1, 2, ..., gn iterations; otherwise a single solver steps through the
    iterations. Returns (errors, energy errors)."""
    import torch
    import oracle
    from multiviewdynrecon_b200 import abi
    from multiviewdynrecon_b200.solver import NonRigidSolver
    o64 = oracle.Oracle(scene, cfg, fp64=True)
    o64.build_index()
    errs, eerrs = [], []
    g = None
    if batch is None:
        g = NonRigidSolver(cfg)
        g.set_solver_input(scene)
        g.build_index()
    field = np.ascontiguousarray(scene.node_se3, np.float32)
    for k in range(gn):
        o64.set_node_se3(field)
        if g is not None:
            g.gn_iteration(pcg)
            torch.cuda.synchronize()
            inst = g
        else:
            bind()
            batch.solve(k + 1, pcg, use_graph=False, stream=stream)
            torch.cuda.synchronize()
            inst = batch.instance(0)
        o64.freeze(inst.get_array(abi.ARRAY_TERM_JACOBIAN), inst.get_array(abi.ARRAY_SMOOTH_TERMS))
        o64.eval_terms()
        o64.assemble()
        eg, eo = inst.energy(), o64.energy()
        o64.pcg(pcg)
        o64.update()
        x64 = o64.get(abi.ARRAY_INCREMENT, as_double=True).reshape(-1)
        x = inst.get_array(abi.ARRAY_INCREMENT).reshape(-1).astype(np.float64)
        errs.append(float(np.linalg.norm(x - x64) / max(np.linalg.norm(x64), 1e-300)))
        eerrs.append(abs(eg - eo) / max(abs(eo), 1e-300))
        field = inst.get_array(abi.ARRAY_NODE_SE3)
    if g is not None:
        g.close()
    return errs, eerrs


def time_solves(solve, steps, warmup, stream):
    import torch
    for _ in range(warmup):
        solve()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        solve()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / steps


def spmv_stage(lib, abi, batch, stream, reps=20):
    import torch
    for _ in range(2):
        lib().mvdr_batch_enqueue_stage(batch.h, abi.STAGE_SPMV, stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        lib().mvdr_batch_enqueue_stage(batch.h, abi.STAGE_SPMV, stream.cuda_stream)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def solver_map_bytes(S, V, W, H, drawn, any_sized):
    """Algorithmic DRAM bytes of one render of V views: every surfel's live
    vertex, colour/time and reference vertex (for its confidence; a float4
    component costs its whole 16-byte element, the sector size being 32) and,
    when a view draws sized points, its live normal and reference normal (for
    the radius) read once; per pixel the depth-index word cleared and read
    back and the five float4 maps and the index written; per drawn pixel the
    winner's five float4 attributes gathered. The depth test's atomics stay
    in L2 (a view's depth-index buffer is W*H*8 bytes)."""
    surfel = S * (16 * 3 + (16 * 2 if any_sized else 0))
    pixels = V * W * H * (8 + 8 + 5 * 16 + 4)
    return surfel + pixels + drawn * 5 * 16


def run_solver_maps(args):
    """Times mvdr_render_solver_maps on the body workload's surfels (moved by
    its warp field) in its five 1280x720 views, view 0 with sized points;
    checks the maps bit for bit against the oracle and times the oracle's
    render on one host thread."""
    import torch
    from multiviewdynrecon_b200 import abi, synth
    from multiviewdynrecon_b200.solver_maps import SolverMapRenderer, geometry_to_device
    import oracle
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    t0 = time.perf_counter()
    scene = synth.articulated_body(auto_radius=True, focal_scale=5.0)
    g = synth.solver_map_geometry(scene)
    gen_s = time.perf_counter() - t0
    S, V, W, H = scene.num_surfels, scene.num_views, scene.width, scene.height
    r = SolverMapRenderer(W, H, V, sized_view0=True)
    dg = geometry_to_device(g)
    with torch.cuda.stream(stream):
        step = lambda: r.draw_solver_maps_with_recent_observation(dg, 10.0, scene.views, stream=stream)  # noqa
        ms = time_solves(step, args.steps, max(3, args.warmup), stream)
    got = [{k: t.cpu().numpy() for k, t in r.maps(v).items()} for v in range(V)]
    prm = abi.solver_map_params(W, H)
    oracle.lib()
    t1 = time.perf_counter()
    want = oracle.render_solver_maps(g, prm, scene.views, sized=[v == 0 for v in range(V)])
    cpu_s = time.perf_counter() - t1
    same = all(np.array_equal(np.ascontiguousarray(got[v][k]).view(np.uint32),
                              np.ascontiguousarray(want[v][k]).view(np.uint32))
               for v in range(V) for k in want[v])
    drawn = int(sum((w["index_map"] != 0xFFFFFFFF).sum() for w in want))
    nbytes = solver_map_bytes(S, V, W, H, drawn, True)
    peak, peak_kind = load_peaks()
    gbs = nbytes / 1e9 / (ms / 1e3)
    line = {"workload": "solver_maps", "metric": "solver-map renders/s", "unit": "renders/s",
            "value": round(1e3 / ms, 2), "ms_per_step": round(ms, 4), "steps": args.steps,
            "config": {"surfels": S, "views": V, "image": [W, H], "sized_view0": True,
                       "l2": "surfel arrays and maps well above the 126 MB L2; no flush"},
            "drawn_pixels": drawn, "bit_exact_vs_oracle": bool(same), "generation_s": round(gen_s, 1),
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "peak_kind": peak_kind, "algorithmic_bytes": nbytes,
                         "kernels": "splat_kernel + resolve_kernel + the depth-index clears"},
            "cpu_baseline": {"value": round(1.0 / cpu_s, 3), "unit": "renders/s", "cores": 1, "kind": "port",
                             "sample": "one whole render of the workload by the oracle"}}
    print(json.dumps(line), flush=True)
    return 0


def run_deform(args):
    """Times the post-solve path on the body workload (4.0M surfels, 32,768
    nodes, 5 views of 1280x720): the forward warp of surfels and nodes, the
    node alignment error with both error maps, and the large-error
    correction, each with CUDA events over --steps calls; algorithmic bytes
    per call from the sizes (stated beside each figure)."""
    import torch
    from multiviewdynrecon_b200 import abi, synth
    from multiviewdynrecon_b200.deform import SurfelNodeDeformer
    from multiviewdynrecon_b200.solver import NonRigidSolver
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    scene = synth.articulated_body(auto_radius=True, focal_scale=5.0)
    g = synth.solver_map_geometry(scene, warped=False)
    nk, nw = synth.node_skinning(scene)
    nodes = synth.node_views(scene)
    guides = synth.correction_guides(scene)
    gen_s = time.perf_counter() - t0

    def dev(a):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(np.int16) if a.dtype == np.uint16 else a.copy()).cuda()

    S, N, V, W, H = scene.num_surfels, scene.num_nodes, scene.num_views, scene.width, scene.height
    field, knn, w = dev(scene.node_se3), dev(scene.surfel_knn), dev(scene.surfel_knn_weight)
    cv, cn = dev(g["reference_vertex_confid"]), dev(g["reference_normal_radius"])
    dnk, dnw, dnodes = dev(nk), dev(nw), dev(nodes)
    solver = NonRigidSolver(abi.make_config(scene))
    solver.set_solver_input(scene)
    stream = torch.cuda.current_stream()
    peak, peak_kind = load_peaks()
    out = {}

    def timed(name, fn, nbytes):
        ms = time_solves(fn, args.steps, max(3, args.warmup), stream)
        out[name] = {"ms": round(ms, 4), "algorithmic_bytes": int(nbytes),
                     "GBps": round(nbytes / 1e9 / (ms / 1e3), 1),
                     "frac_of_measured_hbm": round(nbytes / 1e9 / (ms / 1e3) / peak, 4)}

    res = {}

    def fwd():
        res["fwd"] = SurfelNodeDeformer.forward_warp_surfels_and_nodes(field, knn, w, cv, cn, dnk, dnw, dnodes)

    # per surfel: knn 8 + weights 16 + vertex and normal in 32 + out 32; per node 8 + 16 + 16 + 16
    timed("forward_warp", fwd, S * 88 + N * 56)
    lv, ln, live = res["fwd"]
    drawn = sum(int((v.index_map != 0xFFFFFFFF).sum()) for v in scene.views)

    def node_err():
        res["err"] = solver.compute_alignment_error_on_nodes(maps=True)

    # per pixel: index 4 + two map writes 8; per rendered pixel: reference
    # vertex and normal 32, skinning 24, the observed window (once) 32, mask 4,
    # the node-map pass's index 4, skinning 24 and node sums 32
    timed("node_error", node_err, V * W * H * 12 + drawn * (32 + 24 + 32 + 4 + 4 + 24 + 32))
    united = res["err"]["united_error"]
    dg = [tuple(dev(a) for a in gd) for gd in guides]
    se3 = field.clone()
    live_v, live_n, live_nodes = lv.clone(), ln.clone(), live.clone()

    def correct():
        solver.correct_large_error_node(dg, united, live_nodes, dnk, dnw, live_v, live_n, knn, w, node_se3=se3)

    # per surfel: knn 8 + weights 16 + vertex and normal in 32 and out 32;
    # per node: the same plus the field (32 in, 32 out) and the guide windows
    large = int((united > 0.2).sum().item())
    timed("correction", correct, S * 88 + N * (88 + 64) + large * 25 * (48 + 1 + 16))
    torch.cuda.synchronize()
    line = {"workload": "deform", "config": {"surfels": S, "nodes": N, "views": V, "image": [W, H],
                                            "rendered_pixels": drawn, "large_error_nodes": large},
            "peak": peak, "peak_kind": peak_kind, "generation_s": round(gen_s, 1), "stages": out}
    solver.close()
    print(json.dumps(line), flush=True)
    return 0


def run_extra_workload(args):
    """The uneven batch and the large single solve: one JSON line each,
    documenting configurations beside the headline."""
    import torch
    from multiviewdynrecon_b200 import abi, lib, synth
    from multiviewdynrecon_b200.solver import BatchSolver, DeviceScene, StreamedBatch
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    t0 = time.perf_counter()
    if args.workload == "uneven":
        scenes = synth.batch_instances()
        gn, pcg = 5, 15
        caps = dict(max_nodes=max(s.num_nodes for s in scenes), max_views=max(s.num_views for s in scenes),
                    width=640, height=480, use_foreground=True, use_feature=True, use_cross_view=True,
                    max_surfels=max(s.num_surfels for s in scenes),
                    max_feature_terms=max(s.feature.count for s in scenes),
                    max_cross_terms=max(s.cross_view.count for s in scenes))
        cfg_for = lambda sc: abi.make_config(sc)  # noqa: E731 - the oracle sizes each instance itself
        modes = [("materialized", abi.MODE_MATERIALIZED, abi.PRECISION_MIXED)]
    elif args.workload == "sphere":
        base = synth.sphere_single_view(seed=1, num_nodes=2048, width=640, height=480)
        scenes = [synth.perturb_warp_field(base, seed=sd) for sd in instance_seeds(0, args.batch)]
        gn, pcg = 3, 10
        caps = None
        cfg_for = lambda sc: abi.make_config(sc)  # noqa: E731
        modes = [("materialized", abi.MODE_MATERIALIZED, abi.PRECISION_MIXED),
                 ("materialized_fp32", abi.MODE_MATERIALIZED, abi.PRECISION_FP32)]
    else:
        # framed tightly (5x the focal length of the other workloads) so that
        # the body fills about 87 % of each 1280x720 view: ~4M dense terms
        scenes = [synth.articulated_body(auto_radius=True, focal_scale=5.0)]
        gn, pcg = 8, 20
        caps = None
        cfg_for = lambda sc: abi.make_config(sc)  # noqa: E731
        modes = [("materialized", abi.MODE_MATERIALIZED, abi.PRECISION_MIXED),
                 ("matrix_free", abi.MODE_MATRIX_FREE, abi.PRECISION_MIXED),
                 ("matrix_free_recompute", abi.MODE_MATRIX_FREE, abi.PRECISION_MIXED)]
    gen_s = time.perf_counter() - t0
    dev = [DeviceScene(sc) for sc in scenes]
    B = len(scenes)
    line = {"workload": args.workload, "instances": B, "nodes": [sc.num_nodes for sc in scenes],
            "views": [sc.num_views for sc in scenes], "image": [scenes[0].width, scenes[0].height],
            "gn": gn, "pcg": pcg, "generation_s": round(gen_s, 1), "modes": {}}
    incs = None
    for name, mode, prec in modes:
        rec = name.endswith("_recompute")
        cfg = (abi.make_config(None, precision=prec, mode=mode, recompute_jacobians=rec, **caps) if caps
               else abi.make_config(scenes[0], precision=prec, mode=mode, recompute_jacobians=rec))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        batch = BatchSolver(cfg, B)
        torch.cuda.synchronize()
        solver_mb = round((free0 - torch.cuda.mem_get_info()[0]) / 2**20, 1)

        def bind():
            for i, ds in enumerate(dev):
                batch.set_input(i, ds, stream=stream)

        with torch.cuda.stream(stream):
            bind()
            shape = batch.autotune(stream=stream)[0] if mode == abi.MODE_MATERIALIZED else None
            ms = time_solves(lambda: (bind(), batch.solve(gn, pcg, use_graph=True, stream=stream)), args.steps,
                             max(3, args.warmup), stream)
            entry = {"solves_per_s": round(B / (ms / 1e3), 3), "ms_per_step": round(ms, 3),
                     "solver_device_mb": solver_mb}
            if B > 1 and args.streams > 1:
                # the same instances in concurrent graph lanes (as the headline)
                lanes = StreamedBatch(cfg, B, lanes=args.streams)
                if shape is not None:
                    lanes.set_spmv_shape(abi.SPMV_SHAPES.index(tuple(shape)))

                def lane_step():
                    for i, ds in enumerate(dev):
                        lanes.set_input(i, ds, stream=stream)
                    lanes.solve(gn, pcg, use_graph=True, stream=stream)
                lms = time_solves(lane_step, args.steps, max(3, args.warmup), stream)
                entry["one_graph"] = {"solves_per_s": entry["solves_per_s"], "ms_per_step": entry["ms_per_step"]}
                entry["solves_per_s"] = round(B / (lms / 1e3), 3)
                entry["ms_per_step"] = round(lms, 3)
                entry["lanes"] = len(lanes.lanes)
                lanes.close()
            if mode == abi.MODE_MATERIALIZED:
                bind()
                batch.solve(gn, pcg, use_graph=False, stream=stream)
                sp = spmv_stage(lib, abi, batch, stream)
                counts = [batch.instance(i).counts() for i in range(B)]
                nbytes = sum(algorithmic_bytes(c, sc.num_nodes, prec == abi.PRECISION_MIXED)["spmv"]
                             for c, sc in zip(counts, scenes))  # the materialised mode
                peak, _ = load_peaks()
                entry["spmv"] = {"ms": round(sp, 5), "GBps": round(nbytes / 1e9 / (sp / 1e3), 1),
                                 "frac_of_measured_hbm": round(nbytes / 1e9 / (sp / 1e3) / peak, 4),
                                 "tile": spmv_tile_desc(shape)}
                entry["dense_terms"] = [c.dense_terms for c in counts]
                if args.workload == "sphere":
                    with torch.cuda.stream(stream):
                        errs, eerrs = increment_errors_vs_fp64(scenes[0], cfg, gn, pcg, batch=batch, bind=bind,
                                                               stream=stream)
                    entry["dx_rel_err_vs_fp64"] = [float("%.3g" % e) for e in errs]
                    entry["energy_rel_err_vs_fp64_max"] = float("%.3g" % max(eerrs))
                    batch.close()
                    line["modes"][name] = entry
                    continue
                # first increments for the FP64 comparison
                bind()
                batch.solve(1, pcg, use_graph=False, stream=stream)
                torch.cuda.synchronize()
                incs = []
                for i in range(B):
                    v = batch.instance(i)
                    v.num_nodes = scenes[i].num_nodes
                    incs.append((v.get_array(abi.ARRAY_TERM_JACOBIAN), v.get_array(abi.ARRAY_SMOOTH_TERMS),
                                 v.get_array(abi.ARRAY_INCREMENT)))
        line["modes"][name] = entry
        batch.close()
    # plain FP32 form: one instance per solve, no graph
    if args.workload in ("uneven", "sphere"):
        from multiviewdynrecon_b200.solver import NonRigidSolver
        tot = 0.0
        for sc, ds in zip(scenes, dev):
            single = NonRigidSolver(abi.make_config(sc, precision=abi.PRECISION_FP32))
            with torch.cuda.stream(stream):
                ms = time_solves(lambda: (single.set_solver_input(ds, stream=stream),
                                          single.solve_non_rigid_alignment(gn, pcg, stream=stream)), 2, 1, stream)
            tot += ms
            single.close()
        line["plain_fp32"] = {"solves_per_s": round(B / (tot / 1e3), 3), "form": "one instance per solve, no graph"}
        line["speedup_vs_plain_fp32"] = round(line["modes"]["materialized"]["solves_per_s"] /
                                              line["plain_fp32"]["solves_per_s"], 3)
    if args.workload == "sphere":
        # the plain method on the host cores: the oracle's FP32 solve, 1 thread
        v, n, dt = run_cpu_baseline(argparse.Namespace(gn=gn, pcg=pcg), scenes, 1, min(args.cpu_seconds, 10.0))
        line["cpu_baseline"] = {"value": round(v, 4), "unit": "solves/s", "cores": 1, "kind": "port",
                                "sample": f"{n} whole solves on 1 thread in {dt:.1f} s"}
    if incs is not None:
        t1 = time.perf_counter()
        errs = first_increment_errors(scenes, cfg_for, incs, pcg, os.cpu_count() or 1)
        line["first_increment_rel_err_vs_fp64"] = [float("%.3g" % e) for e in errs]
        line["fp64_check_s"] = round(time.perf_counter() - t1, 1)
    print(json.dumps(line), flush=True)
    return 0


def cpu_solve_instance(scene, gn, pcg):
    import oracle
    from multiviewdynrecon_b200 import abi
    o = oracle.Oracle(scene, abi.make_config(scene), fp64=False)
    o.solve(gn, pcg)
    return o


def run_cpu_baseline(args, scenes, threads, seconds):
    """Time whole solves of the CPU restatement on `threads` host threads, one
    instance per thread, for about `seconds`."""
    from concurrent.futures import ThreadPoolExecutor
    done = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while True:
            futs = [ex.submit(cpu_solve_instance, scenes[(done + k) % len(scenes)], args.gn, args.pcg)
                    for k in range(threads)]
            for f in futs:
                f.result()
            done += threads
            if time.perf_counter() - t0 >= seconds:
                break
    dt = time.perf_counter() - t0
    return done / dt, done, dt


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        if rank != 0:
            return 0
        import oracle
        oracle.lib()
        base, scenes = make_scenes(args, 0)
        threads = os.cpu_count() or 1
        # warm-up steps, then timed steps; a step solves one instance per thread
        for _ in range(args.warmup):
            run_cpu_baseline(args, scenes, threads, 0.0)
        vals = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            v, n, dt = run_cpu_baseline(args, scenes, threads, 0.0)
            vals.append(dt)
        total = time.perf_counter() - t0
        value = args.steps * threads / total
        line = {"metric": METRIC, "impl": "reference", "value": round(value, 4),
                "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(1e3 * total / args.steps, 2), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "instances_per_step": threads, "views": 3,
                           "image": [args.width, args.height], "nodes": args.nodes, "gn": args.gn,
                           "pcg": args.pcg, "precision": "fp32 terms, double sums (CPU restatement)"},
                "cpu_baseline": {"value": round(value, 4), "unit": "solves/s", "cores": threads, "kind": "port",
                                 "sample": f"{threads} whole solves per step, one per host thread"},
                "e2e": {"value": round(value, 4), "unit": "solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if args.workload == "solver_maps":
        return run_solver_maps(args) if rank == 0 else 0
    if args.workload == "deform":
        return run_deform(args) if rank == 0 else 0
    if args.workload != "torso":
        return run_extra_workload(args) if rank == 0 else 0

    if world > 1:
        import torch
        import torch.distributed as tdist
        import datetime
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    r = run_ours(args, rank, world, dist)
    cpu = None
    if rank == 0 and not args.no_cpu:
        base, scenes = r["base"], make_scenes(args, 0)[1]
        v, n, dt = run_cpu_baseline(args, scenes, 1, args.cpu_seconds)
        cpu = {"value": round(v, 4), "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"{n} whole solves of the workload's instances on 1 thread in {dt:.1f} s"}
    if rank == 0:
        c = r["counts"]
        line = {
            "metric": METRIC,
            "value": round(r["value"], 3), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(r["ms"], 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "instances_per_gpu": args.batch, "streams": max(1, args.streams),
                       "instances_per_stream": -(-args.batch // max(1, args.streams)), "views": 3,
                       "image": [args.width, args.height], "nodes": args.nodes, "gn": args.gn, "pcg": args.pcg,
                       "precision": args.precision, "mode": args.mode, "graph": True,
                       "pcg_form": "persistent" if args.pcg_persistent else "launches",
                       "l2": "aggregate working set of the batch well above the 126 MB L2; no flush",
                       "dense_terms": c.dense_terms, "half_pairs": c.half_pairs,
                       "parallelism": f"independent instances, {world} GPU(s), no collective in the solve"},
            "gpu_launches": int(r["kernels_per_step"] * args.steps),
            "kernels_per_step": int(r["kernels_per_step"]),
            "clocks": r["clocks"], "roofline": r["roofline"], "stages": r["stages"], "spmv_tile": r["spmv_tile"],
            "e2e": r["e2e"],
            "plain_fp32": r["plain"],
            "speedup_vs_plain_fp32": (round(r["value"] / r["plain"]["value"], 3) if r["plain"] else None),
            "speedup_vs_plain_fp32_batched": (round(r["value"] / r["plain"]["batched_graph"]["value"], 3)
                                              if r["plain"] else None),
            "accuracy": r["accuracy"],
            "pcg_history": r["pcg_history"],
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
