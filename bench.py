#!/usr/bin/env python
"""Thin-shell fit benchmark (one JSON line on stdout from rank 0).

Workload (default): the (3,5) torus-knot tube -- 4,096 rings x 128 segments = 1,048,576
faces, FP32 vertices with N(0, 1e-3) jitter (seed 1) -- normalised to the unit cube, SVO
depth 9 (256^3 voxels), fit to 1e-6 relative residual, marching cubes at 512^3.

A step is one fit from the octree and right-hand side (resident in HBM) to coefficients
whose relative residual ||b - A lambda|| / ||b|| is at most 1e-6: the learned start (share
features -> share network in BF16 on the tensor cores -> FP64 exact start) checked by the
matrix-free FP64 residual, with the plain LSCG from that start as the fallback. `value` is
its time in ms (max over ranks); `e2e` is the same call through the C ABI with the
right-hand side in pinned host memory and the coefficients read back every step.

Beside it (none of it inside the timed steps):
  * the plain FP64 LSCG from zero (assembly + CGLS, the reference's method) and the
    mixed-precision LSCG on the same octree, with the mixed fit's error against FP64;
  * marching-cubes topology: case indices of the learned fit's field against the FP64 LSCG
    from zero at 1e-12 (the reference's solution) at both shell iso levels on the MC grid;
  * the roofline of the step's dominant kernel (the share network, kMlpForwardFused) and of
    the plain path's binned SpMV;
  * the whole pipeline in the facade's call order (octree, samples, signed distance, fit,
    iso levels, field + marching cubes at three levels) with per-stage times;
  * the 256-mesh uneven batch (plain batched LSCG vs one learned batch), marching-cubes
    throughput, and the CPU oracle per stage on the host cores.

--gpus N (N > 1, not already under torchrun) starts N ranks, one process per GPU, through
torch.distributed.run; each rank fits its own replica of the workload and the batch is
sharded over the ranks by mesh (longest processing time first).

--impl reference times the CPU restatement of the reference's fit (oracle/, OpenMP on all
host cores) on the same workload; it loads nothing from libits.
"""
import argparse
import ctypes as C
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fit ms to 1e-6 rel. residual (learned+mixed vs plain FP64, 1 B200); MC Mvox/s"
WORKLOADS = {
    "c1": dict(mesh="c1", res=256, tol=1e-6, mc_res=512,
               desc="(3,5) torus-knot tube r=0.08, 4096 rings x 128 segments = 1,048,576 faces, FP32 vertices "
                    "+ N(0,1e-3) jitter (seed 1); SVO depth 9 (256^3); FP64 LSCG to 1e-6 relative residual; "
                    "MC 512^3"),
    "c2": dict(mesh="c2", res=512, tol=1e-6, mc_res=1024,
               desc="perturbed geodesic sphere subdivided 9 times, 2,621,440 faces, amplitude 0.15 (seed 2); SVO "
                    "depth 10 (512^3); fit to 1e-6 relative residual; mixed precision (FP32 SpMV, FP64 dots and "
                    "residual, 3 refinement steps) with its error against FP64; field at 1024^3"),
    "c0": dict(mesh="c0", res=32, tol=1e-6, mc_res=128,
               desc="perturbed geodesic sphere, 10,240 faces (seed 0); SVO depth 6 (32^3); FP64 LSCG to 1e-6 "
                    "relative residual; MC 128^3"),
}
MLP_MACS_PER_ROW = 64 * 128 + 128 * 128 + 128 * 128 + 128  # multiply-adds of one share-network row


def config_of(wl, n, nnz):
    """The config object both arms print (identical keys and values for one workload)."""
    return {"workload": wl["desc"], "unknowns": int(n), "nnz": int(nnz), "tol": wl["tol"], "mc_res": wl["mc_res"],
            "inputs": "octree and right-hand side resident (value); right-hand side from host memory, coefficients "
                      "back to host memory every step (e2e)",
            "l2": "the operator (A and A^T, 12 B per entry each) exceeds the 126 MB L2 at this size"}


def field_terms(pos, depth_counts, o, w, res, R):
    """Terms of the bit-exact dense field on the (R+1)^3 MC lattice over the octree's own box
    (R a multiple of res): every corner vertex at depth d adds one term to each lattice point of
    the cells it is a corner of -- points i with floor(i / s) in {X - 1, X} per axis,
    s = R / (res >> d)."""
    terms = 0
    w0 = float(w[0]) / res
    start = 0
    for d, cnt in enumerate(depth_counts):
        P = pos[start:start + cnt]
        start += cnt
        if cnt == 0:
            continue
        s = R // (res >> d)
        X = np.rint((P - np.asarray(o)[None, :]) / (w0 * (1 << d))).astype(np.int64)
        lo = np.maximum(0, s * (X - 1))
        hi = np.minimum(R, s * (X + 1) - 1)
        c = np.clip(hi - lo + 1, 0, None)
        terms += int(np.sum(c[:, 0] * c[:, 1] * c[:, 2]))
    return terms


def fp64_peak():
    """Nominal FP64 vector rate of the device (64 operations per SM per clock at the maximum
    SM clock; no measured FP64 figure is available): operations per second."""
    import torch
    props = torch.cuda.get_device_properties(0)
    try:
        mhz = float(subprocess.run(["nvidia-smi", "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits",
                                    "-i", "0"], capture_output=True, text=True, timeout=20).stdout.split()[0])
    except Exception:
        mhz = 1965.0
    return 64.0 * props.multi_processor_count * mhz * 1e6


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def profile_traffic(name, cfg):
    """DRAM bytes per launch of a kernel on workload `cfg` from its committed ncu summary (a
    line `traffic_bytes_per_launch: N` in profiles/<name>_<cfg>_*.md), or None when no capture
    of that kernel on that workload is committed."""
    pdir = os.path.join(ROOT, "profiles")
    try:
        for fn in sorted(os.listdir(pdir)):
            if fn.startswith(name + "_" + cfg + "_") and fn.endswith(".md"):
                for line in open(os.path.join(pdir, fn)):
                    if line.strip().startswith("traffic_bytes_per_launch:"):
                        return int(float(line.split(":", 1)[1].strip().split()[0]))
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def prepared(wl, host_api):
    """Mesh of the workload normalised to the unit cube, with the reference's cubic box
    (BaseModel's constructor order), by host_api's model_to_unit_cube / uniform_bbox: libits'
    for our arm, the oracle's for the reference arm (bit-identical, tested)."""
    from its_b200 import meshes
    V, F = meshes.config_mesh(wl["mesh"])
    V = host_api.model_to_unit_cube(V)
    o, _, w = host_api.uniform_bbox(V)
    return V, F, o, w


def dist_setup():
    rank, world, local = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def max_over_ranks(value, dist=None, device="cuda"):
    """Max of a per-rank time over all ranks (every rank must call it at the same point)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device="cuda"):
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def lpt_shard(costs, world):
    """Longest-processing-time-first assignment of independent meshes to ranks.

    Returns one list of item indices per rank; each list is in ascending index order."""
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]


def batch_shard(faces, world, rank):
    """This rank's meshes of the batch: LPT over ranks by face count (no data-path collective)."""
    return lpt_shard(list(faces), world)[rank]


def batch_totals(local, dist=None, device="cuda"):
    """Whole-job figures of the sharded batch from this rank's: times (keys ending in _ms) and
    keys starting with max_ are maxima over ranks (every rank waits for the slowest), the rest
    are sums. Every rank must call it with the same keys in the same order."""
    out = {}
    for k, v in local.items():
        mx = k.endswith("_ms") or k.startswith("max_")
        out[k] = max_over_ranks(v, dist, device) if mx else sum_over_ranks(v, dist, device)
    return out


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def launch_ranks(argv, gpus):
    """Re-run this script as `gpus` ranks (one process per GPU) under torch.distributed.run."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % gpus,
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)] + argv
    return subprocess.run(cmd).returncode


def mc_case_mismatches(svo, ctx, lam_a, lam_b, o, w, R, isos):
    """Per iso level: the number of voxels whose marching-cubes case index differs between the
    FP64 fields (its_eval_grid, bit-exact with the reference's sums) of two coefficient vectors,
    and the number of voxels with a surface crossing in the first field."""
    import torch
    from its_b200 import lib
    M = R + 1
    fa = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    fb = torch.empty_like(fa)
    svo.eval_grid(lam_a, o, w, R, out=fa)
    svo.eval_grid(lam_b, o, w, R, out=fb)
    ca = torch.empty(R ** 3, dtype=torch.uint8, device="cuda")
    cb = torch.empty_like(ca)
    o_np, w_np = np.ascontiguousarray(o), np.ascontiguousarray(w)
    nv = C.c_int64(0)
    out = []
    for iso in isos:
        for f, c in ((fa, ca), (fb, cb)):
            ctx.check(lib().its_marching_cubes(ctx.h, C.c_void_p(f.data_ptr()), R, o_np.ctypes.data_as(C.c_void_p),
                                               w_np.ctypes.data_as(C.c_void_p), float(iso), C.c_void_p(c.data_ptr()),
                                               None, 0, C.byref(nv)), "its_marching_cubes")
        active = int(((ca != 0) & (ca != 255)).sum().item())
        out.append({"iso": float(iso), "mismatches": int((ca != cb).sum().item()), "active_voxels": active})
    del fa, fb, ca, cb
    return out


def run_ours(args):
    import torch
    from its_b200 import OP_FP32_VALUES, PREC_MIXED, STOP_RESIDUAL, Context, Operator, Svo, lib
    from its_b200 import sharenet
    from its_b200.api import ShareNet, fit_residual_batch, learned_fit

    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    import its_b200
    wl = WORKLOADS[args.config]
    V, F, o, w = prepared(wl, its_b200)
    ctx = Context(local)
    # One non-default stream for everything: libits, torch's own ops (the L2 flush) and the
    # timing events. (Handing libits the legacy default stream, handle 0, would select the
    # context's own non-blocking stream and the events would not bracket its kernels.)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    def barrier_sync():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def max_ranks(v):
        return max_over_ranks(v, pg, "cuda")

    if args.only == "pipeline":  # the facade-order pipeline alone (for profiling its stages)
        from its_b200 import sharenet as _sn
        params, norm = _sn.load()
        net = ShareNet(ctx, batch=65536, params=params)
        pipe = run_pipeline(ctx, net, norm, V, F, o, w, wl, timed, reps=max(1, args.steps))
        if rank == 0:
            print(json.dumps({"metric": METRIC, "only": "pipeline", "pipeline": pipe}), flush=True)
        net.close()
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    # ---- setup: octree and right-hand side (signed distance at the corner vertices) ------
    # the octree build timed warm from a device-resident mesh (the host arrays' upload apart)
    Vd, Fd = torch.from_numpy(np.ascontiguousarray(V)).cuda(), torch.from_numpy(np.ascontiguousarray(F, np.int32)).cuda()
    Svo(ctx, Vd, Fd, wl["res"], o, w).close()
    svo_ms = timed(lambda: Svo(ctx, Vd, Fd, wl["res"], o, w).close(), 3)
    svo = Svo(ctx, Vd, Fd, wl["res"], o, w)  # warm: its build times in the report are steady-state
    del Vd, Fd
    pos, _ = svo.vertices()
    b = ctx.signed_distance(pos, V, F)
    n = svo.num_verts
    b_dev = torch.from_numpy(b).cuda()
    lam_dev = torch.empty_like(b_dev)
    params, norm = sharenet.load()
    net = ShareNet(ctx, batch=65536, params=params)
    rep_box = {}

    # ---- the headline fit: learned start verified by the FP64 residual -------------------
    def learned_step(b_in=b_dev, out=lam_dev):
        _, r = learned_fit(svo, net, b_in, norm, wl["tol"], out=out)
        rep_box["learned_rel"] = r["rel_residual"]
        rep_box["learned_fallback_iterations"] = r["iterations"]

    # The clock sampler starts before the warm-up so that nvidia-smi's start-up (NVML
    # initialisation, which stalls the driver) falls outside the timed steps.
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.5)
    for _ in range(args.warmup):
        learned_step()
    barrier_sync()
    launches0 = ctx.kernel_launches
    fit_ms = timed(learned_step, args.steps)
    launches = (ctx.kernel_launches - launches0) // max(args.steps, 1)
    barrier_sync()
    fit_ms = max_ranks(fit_ms)

    # ---- end to end through the C ABI: host rhs in, host coefficients out -----------------
    b_host = torch.from_numpy(b).pin_memory()
    lam_host = torch.empty(n, dtype=torch.float64).pin_memory()
    b_np, lam_np = b_host.numpy(), lam_host.numpy()
    for _ in range(max(1, args.warmup // 2)):
        learned_step(b_np, lam_np)
    barrier_sync()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        learned_step(b_np, lam_np)
    torch.cuda.synchronize()
    e2e_ms = max_ranks((time.perf_counter() - t0) * 1e3 / args.steps)

    # ---- plain FP64 LSCG from zero (the reference's method) and the mixed-precision form --
    def plain_step():
        op = Operator(svo)
        _, r = op.solve(b_dev, tol=wl["tol"], stop_rule=STOP_RESIDUAL, out=lam_plain)
        rep_box["plain"], rep_box["nnz"] = r, op.nnz
        op.close()

    lam_plain = torch.empty_like(b_dev)
    lam_mixed = torch.empty_like(b_dev)

    def mixed_step():
        op = Operator(svo, mode=OP_FP32_VALUES)
        _, r = op.solve(b_dev, tol=wl["tol"], stop_rule=STOP_RESIDUAL, precision=PREC_MIXED, ir_steps=3,
                        inner_tol=1e-3, out=lam_mixed)
        rep_box["mixed"] = r
        op.close()

    for _ in range(args.warmup):
        plain_step()
    plain_ms = max_ranks(timed(plain_step, args.steps))
    mixed_step()
    mixed_ms = max_ranks(timed(mixed_step, max(1, args.steps // 2)))
    clk = clocks.stop()
    nnz = rep_box["nnz"]
    if args.only == "fit":
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(fit_ms, 4), "unit": "ms", "only": "fit",
                              "plain_fp64_ms": round(plain_ms, 4), "gpu_launches": launches}), flush=True)
        net.close()
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    # ---- roofline of the step's dominant kernel: the share network (kMlpForwardFused) ------
    from its_b200.api import exact_start_batch
    from its_b200.api import feature_tiles
    feats, ids = svo.share_features(b, norm[:128])
    rows = int(feats.shape[0])
    # as inside the step: the input as the features kernel writes it (BF16 tiles, fetched by
    # bulk copies), each launch a programmatic dependent launch after the previous kernel; K
    # launches captured once in a CUDA graph and replayed, so the host's launch rate is not
    # what is timed
    tiles_dev = torch.from_numpy(feature_tiles(feats)).cuda()
    pred_dev = torch.empty(rows, dtype=torch.float32, device="cuda")
    for i in range(5):
        net.forward_tiles_async(tiles_dev, rows, pred_dev, after_kernel=i > 0)
    net.check()
    K = 50
    mlp_graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(mlp_graph, stream=stream, capture_error_mode="relaxed"):
        for i in range(K):
            net.forward_tiles_async(tiles_dev, rows, pred_dev, after_kernel=i > 0)
    mlp_graph.replay()
    net.check()
    mlp_ms = timed(mlp_graph.replay, 5) / K
    net.check()
    del mlp_graph
    hbm_peak, tensor_peak, peak_kind = load_peaks()
    mlp_flop = 2.0 * rows * MLP_MACS_PER_ROW
    mlp_tflops = mlp_flop / (mlp_ms * 1e-3) / 1e12
    traffic = profile_traffic("kMlpForwardFused", wl["mesh"])

    # ---- breakdown of the learned fit ----------------------------------------------------
    learned_bytes = 3 * 48 * n + 2 * 256 * rows
    feat_buf = torch.empty((rows, 64), dtype=torch.float32, device="cuda")
    ids_dev = torch.empty(rows, dtype=torch.int64, device="cuda")
    features_call = lambda: svo.share_features(b_dev, norm[:128], out=feat_buf, ids=ids_dev)  # noqa: E731
    start_call = lambda: exact_start_batch([svo], [b_dev], outs=[lam_dev])  # noqa: E731
    resid_call = lambda: fit_residual_batch([svo], [b_dev], [lam_dev])  # noqa: E731
    for _ in range(3):  # warm-up (first launches load their kernels)
        features_call(), start_call(), resid_call()
    t_features = timed(features_call, 5)
    t_start = timed(start_call, 5)
    t_resid = timed(resid_call, 5)

    # ---- field error and MC topology of the learned fit against the FP64 LSCG from zero ----
    learned_step()
    lam_learned = lam_dev.cpu().numpy()
    op = Operator(svo)
    x_ref, rep_ref = op.solve(b, tol=1e-12, max_iters=20000, stop_rule=STOP_RESIDUAL)
    op.close()
    lam_zero = svo.exact_start(b)
    samples = np.vstack([V, svo.shell_samples(V, F)[0]])
    f_ref = svo.eval_points(x_ref, samples)[0]
    G = 128
    g_ref = svo.eval_grid(x_ref, o, w, G)
    scale = float(np.abs(b).max())
    field = {"reference": "FP64 LSCG from zero to 1e-12 relative residual (%d iterations)" % rep_ref["iterations"],
             "scale": "max |b|", "grid": "%d^3 corners of the box" % (G + 1)}
    lam_plain_np = lam_plain.cpu().numpy()
    for name, lam in (("learned", lam_learned), ("zero_shares", lam_zero), ("plain_lscg_1e-6", lam_plain_np)):
        d = svo.eval_grid(lam, o, w, G) - g_ref
        e = svo.eval_points(lam, samples)[0] - f_ref
        field[name] = {"grid_max": float(np.abs(d).max() / scale), "grid_rms": float(np.sqrt(np.mean(d * d)) / scale),
                       "samples_max": float(np.abs(e).max() / scale),
                       "coef_rel": float(np.linalg.norm(lam - x_ref) / np.linalg.norm(x_ref))}
    inner, outer, _ = svo.shell_iso_values(x_ref, samples)
    il, ol, _ = svo.shell_iso_values(lam_learned, samples)
    field["iso_abs_diff"] = [abs(il - inner), abs(ol - outer)]
    R = wl["mc_res"]
    topo = {"grid": "%d^3 voxels, FP64 fields of its_eval_grid" % R,
            "reference": "FP64 LSCG from zero to 1e-12 (the converged solution the reference's LSCG approaches)",
            "bar": "0 mismatches at both shell iso levels"}
    topo["learned"] = mc_case_mismatches(svo, ctx, lam_learned, x_ref, o, w, R, (inner, outer))
    topo["plain_lscg_1e-6"] = mc_case_mismatches(svo, ctx, lam_plain_np, x_ref, o, w, R, (inner, outer))

    # ---- precision: the mixed fit against FP64 (every run) ----------------------------------
    precision = run_precision(svo, b, x_ref, lam_mixed.cpu().numpy(), samples, o, w, scale, timed,
                              wl["mc_res"], rep_box["mixed"])

    # ---- roofline of the plain path's dominant kernel, the binned CSR SpMV ------------------
    op = Operator(svo)
    x_dev = torch.randn(n, dtype=torch.float64, device="cuda")
    y_dev = torch.empty_like(x_dev)
    # A alone (120 MB at this size) nearly fits the 126 MB L2, so every timed launch starts
    # from a flushed L2 (a 256 MB write), as in the CGLS loop where A and A^T alternate.
    flush = torch.empty(32 * 2 ** 20, dtype=torch.float64, device="cuda")
    spmv, samples_t = {}, {0: [], 1: []}
    for tr in (0, 1):
        for _ in range(3):
            op.apply(x_dev, transpose=bool(tr), out=y_dev)
    for _ in range(20):
        for tr in (0, 1):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            op.apply(x_dev, transpose=bool(tr), out=y_dev)
            e1.record(stream)
            e1.synchronize()
            samples_t[tr].append(e0.elapsed_time(e1))
    for tr in (0, 1):
        spmv[tr] = statistics.median(samples_t[tr])
    del flush
    op.close()
    spmv_bytes = 12 * nnz + 24 * n  # values 8 + columns 4 per entry; rowptr 8, x 8, y 8 per row
    dom = 1 if spmv[1] >= spmv[0] else 0
    spmv_achieved = spmv_bytes / (spmv[dom] * 1e-3) / 1e9

    # ---- dense field + marching cubes ---------------------------------------------------------
    M = R + 1
    fieldbuf = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    lam_fit = torch.from_numpy(lam_learned).cuda()
    L = lib()
    o_np, w_np = np.ascontiguousarray(o), np.ascontiguousarray(w)
    cube = torch.empty(R ** 3, dtype=torch.uint8, device="cuda")
    nv = C.c_int64(0)

    def field_step():
        svo.eval_grid(lam_fit, o, w, R, out=fieldbuf)

    def mc_step():
        st = L.its_marching_cubes(ctx.h, C.c_void_p(fieldbuf.data_ptr()), R, o_np.ctypes.data_as(C.c_void_p),
                                  w_np.ctypes.data_as(C.c_void_p), float(ol), C.c_void_p(cube.data_ptr()), None, 0,
                                  C.byref(nv))
        ctx.check(st, "its_marching_cubes")

    field_step()
    mc_step()
    field_ms = timed(field_step, 2)
    mc_ms = timed(mc_step, 3)
    mc_mvox = R ** 3 / ((field_ms + mc_ms) * 1e-3) / 1e6
    mc_verts = int(nv.value)

    # the bit-exact field is bound by FP64 arithmetic (three operations per term, the terms in
    # the reference's order), not by its writes: both rooflines are reported
    f_terms = field_terms(pos, svo.depth_counts()[1], o, w, wl["res"], R) if R % wl["res"] == 0 else None
    f_bytes = 8 * M ** 3
    f_hbm = f_bytes / (field_ms * 1e-3) / 1e9
    field_roof = {"bound": "fp64", "kernel": "the bit-exact FP64 field of the MC grid (its_eval_grid: kEvalGridSep, "
                                             "lambda * ((hx * hy) * hz) summed in the reference's order)",
                  "launch_ms": round(field_ms, 4), "terms_per_launch": f_terms,
                  "traffic": profile_traffic("kEvalGridSep", wl["mesh"]),
                  "hbm": {"achieved": round(f_hbm, 1), "peak": hbm_peak, "unit": "GB/s",
                          "frac": round(f_hbm / hbm_peak, 4), "bytes_per_launch": f_bytes}}
    if f_terms:
        ops = 3.0 * f_terms
        peak64 = fp64_peak()
        field_roof.update({"achieved": round(ops / (field_ms * 1e-3) / 1e12, 3), "peak": round(peak64 / 1e12, 3),
                           "unit": "T FP64 op/s", "frac": round(ops / (field_ms * 1e-3) / peak64, 4),
                           "peak_kind": "nominal (64 FP64 operations per SM per clock at the maximum SM clock)",
                           "note": "3 FP64 operations (two multiplies, one add) per term; every term a corner "
                                   "vertex contributes to a lattice point of its cells"})

    # ---- FP32 field + marching cubes (the precision mode) ------------------------------------
    field32 = torch.empty(M ** 3, dtype=torch.float32, device="cuda")

    def field32_step():
        svo.eval_grid_f32(lam_fit, o, w, R, out=field32)

    def mc32_step():
        st = L.its_marching_cubes_f32(ctx.h, C.c_void_p(field32.data_ptr()), R, o_np.ctypes.data_as(C.c_void_p),
                                      w_np.ctypes.data_as(C.c_void_p), float(ol), C.c_void_p(cube.data_ptr()), None,
                                      0, C.byref(nv))
        ctx.check(st, "its_marching_cubes_f32")

    field32_step()
    mc32_step()
    field32_ms = timed(field32_step, 2)
    mc32_ms = timed(mc32_step, 3)
    f32_err = float((field32.double() - fieldbuf).abs().max().item()) / scale
    mc32 = {"res": R, "mvox_s": round(R ** 3 / ((field32_ms + mc32_ms) * 1e-3) / 1e6, 1),
            "field_ms": round(field32_ms, 3), "mc_ms": round(mc32_ms, 3), "tri_vertices": int(nv.value),
            "field_max_err_vs_fp64": f32_err}

    # ---- the field by prolongation on the octree's own lattice (its_eval_grid_fast) --------
    fastbuf = torch.empty_like(fieldbuf)
    cube_fast = torch.empty_like(cube)

    def fast_step():
        svo.eval_grid_fast(lam_fit, o, w, R, out=fastbuf)

    def fast32_step():
        svo.eval_grid_fast(lam_fit, o, w, R, out=field32, fp32=True)

    def mcf_step():
        st = L.its_marching_cubes(ctx.h, C.c_void_p(fastbuf.data_ptr()), R, o_np.ctypes.data_as(C.c_void_p),
                                  w_np.ctypes.data_as(C.c_void_p), float(ol), C.c_void_p(cube_fast.data_ptr()), None, 0,
                                  C.byref(nv))
        ctx.check(st, "its_marching_cubes")

    fast_step()
    fast32_step()
    mcf_step()
    fast_ms = timed(fast_step, 3)
    fast32_ms = timed(fast32_step, 3)
    mcf_ms = timed(mcf_step, 3)
    mcf_verts = int(nv.value)
    mc_step()  # the exact field's cube indices again (the FP32 run reused the buffer)
    mc_fast = {"res": R, "mvox_s": round(R ** 3 / ((fast_ms + mcf_ms) * 1e-3) / 1e6, 1),
               "field_ms": round(fast_ms, 3), "mc_ms": round(mcf_ms, 3), "tri_vertices": mcf_verts,
               "field_max_dev_vs_exact": float((fastbuf - fieldbuf).abs().max().item()) / scale,
               "cube_index_mismatches": int((cube_fast != cube).sum().item()),
               "field32_ms": round(fast32_ms, 3),
               "field32_max_err_vs_fp64": float((field32.double() - fieldbuf).abs().max().item()) / scale,
               "field": "FP64 by prolongation on the octree's lattice (its_eval_grid_fast)"}
    del field32, fastbuf, cube_fast, fieldbuf, cube

    # ---- the whole pipeline in the facade's call order ----------------------------------------
    pipeline = run_pipeline(ctx, net, norm, V, F, o, w, wl, timed)

    # ---- the uneven multi-mesh batch: plain batched LSCG vs one learned batch ---------------
    batch = None
    if not args.no_batch:
        batch = run_batch(ctx, net, norm, timed, wl["tol"], world, rank, min(args.steps, 3), pg)

    # ---- CPU baseline: the oracle on the host cores (rank 0, N = 1) ------------------------
    cpu, cpu_st = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_fit(V, F, o, w, wl, b)
        cpu_st = cpu_stages(V, F, o, w, wl)

    if rank == 0:
        plain = rep_box["plain"]
        line = {
            "metric": METRIC, "value": round(fit_ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(fit_ms, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(wl, n, nnz),
            "method": "learned start (share network, BF16 weights and activations with FP32 accumulation on the "
                      "tcgen05 tensor cores) + FP64 exact start + FP64 matrix-free residual check; plain FP64 LSCG "
                      "from that start as the fallback",
            "rel_residual": rep_box["learned_rel"],
            "fallback_iterations": rep_box["learned_fallback_iterations"],
            "parallelism": ("replicas x%d" % world) if world > 1 else "single",
            "plain_fp64": {"ms": round(plain_ms, 4), "iterations": plain["iterations"],
                           "rel_residual": plain["rel_residual"], "speedup": round(plain_ms / fit_ms, 2)},
            "mixed": {"ms": round(mixed_ms, 4), "inner_iterations": rep_box["mixed"]["inner_iterations"],
                      "rel_residual": rep_box["mixed"]["rel_residual"]},
            "learned_breakdown_ms": {"features": round(t_features, 4), "network": round(mlp_ms, 4),
                                     "exact_start": round(t_start, 4), "residual": round(t_resid, 4), "rows": rows,
                                     "octree_build_ms": round(svo.info.build_ms, 3),
                                     "octree_learned_tables_ms": round(svo.info.learned_tables_ms, 3),
                                     "note": "features, exact start and residual each called alone through their "
                                             "C-ABI entries (a synchronisation included); the network is the kernel "
                                             "alone; inside its_learned_fit all run back to back as one captured "
                                             "graph. octree_learned_tables_ms: the part of its_svo_build (octree_build_ms, "
                                             "device time) that forms the learned fit's octree-only tables (per-node "
                                             "face-sample sums, coincident vertices and their geometric features); it "
                                             "runs once per octree, outside the timed fit"},
            "field_error": field,
            "mc_topology": topo,
            "precision": precision,
            "e2e": {"value": round(e2e_ms, 4), "unit": "ms", "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 8 * n},
            "roofline": {"bound": "tensor", "kernel": "kMlpForwardFused (share-network inference, the timed step's "
                                                      "largest kernel)",
                         "achieved": round(mlp_tflops, 2), "peak": tensor_peak, "unit": "TFLOP/s",
                         "frac": round(mlp_tflops / tensor_peak, 4), "peak_kind": peak_kind + " bf16 burst",
                         "flop_per_launch": mlp_flop, "launch_ms": round(mlp_ms, 5),
                         "traffic": traffic,
                         "note": "2 x rows x %d multiply-adds per launch (64x128 + 2 x 128x128 + 128); launch time "
                                 "by CUDA events over a graph of %d back-to-back programmatic dependent launches on "
                                 "the BF16 input tiles (as inside the step; input L2-resident); traffic: ncu DRAM "
                                 "read + write bytes per launch (profiles/)" % (MLP_MACS_PER_ROW, K)},
            "roofline_spmv": {"bound": "hbm", "kernel": "kSpmvBinned (%s), the plain LSCG's dominant kernel"
                              % ("A^T" if dom else "A"),
                              "achieved": round(spmv_achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                              "frac": round(spmv_achieved / hbm_peak, 4), "peak_kind": peak_kind,
                              "bytes_per_launch": spmv_bytes, "launch_ms": round(spmv[dom], 5),
                              "traffic": profile_traffic("kSpmvBinned", wl["mesh"])},
            "roofline_learned_step": {"bound": "hbm", "kernel": "the learned fit step as a whole (its 8 kernels)",
                                      "achieved": round(learned_bytes / (fit_ms * 1e-3) / 1e9, 1), "peak": hbm_peak,
                                      "unit": "GB/s", "frac": round(learned_bytes / (fit_ms * 1e-3) / 1e9 / hbm_peak, 4),
                                      "bytes_per_launch": learned_bytes, "launch_ms": round(fit_ms, 5)},
            "cpu_baseline": cpu,
            "cpu_stages": cpu_st,
            "clocks": clk,
            "gpu_launches": launches,
            "mc": {"res": R, "mvox_s": round(mc_mvox, 1), "field_ms": round(field_ms, 3), "mc_ms": round(mc_ms, 3),
                   "iso": ol, "tri_vertices": mc_verts, "field": "FP64, bit-exact with the oracle"},
            "roofline_field": field_roof,
            "mc_f32": mc32,
            "mc_fast": mc_fast,
            "pipeline": pipeline,
            "batch": batch,
            "svo_build_ms": round(svo_ms, 3),
            "svo_build_note": "its_svo_build from a device-resident mesh, warm (host side included); the device "
                              "time alone is learned_breakdown_ms.octree_build_ms",
            "spmv_ms": {"A": round(spmv[0], 5), "AT": round(spmv[1], 5)},
        }
        print(json.dumps(line), flush=True)
    net.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def run_precision(svo, b, x_ref, x_mixed, samples, o, w, scale, timed, G, rep):
    """Error of the mixed-precision fit and of the FP32 field against FP64."""
    import torch
    out = {"reference": "FP64 LSCG from zero to 1e-12 relative residual, FP64 field",
           "mixed_rel_residual": rep["rel_residual"], "mixed_inner_iterations": rep["inner_iterations"]}
    lam_scale = float(np.abs(x_ref).max())
    d = x_mixed - x_ref
    out["coef_max"] = float(np.abs(d).max() / lam_scale)
    out["coef_rms"] = float(np.sqrt(np.mean(d * d)) / lam_scale)
    e = svo.eval_points(x_mixed, samples)[0] - svo.eval_points(x_ref, samples)[0]
    out["samples_max"] = float(np.abs(e).max() / scale)
    out["samples_rms"] = float(np.sqrt(np.mean(e * e)) / scale)
    # the FP32 field of the mixed fit on the MC grid (bricked kernel) against the FP64 field of
    # the FP64 fit, compared slab by slab on the device
    M = G + 1
    f32 = torch.empty(M ** 3, dtype=torch.float32, device="cuda")
    lam_m = torch.from_numpy(x_mixed).cuda()
    svo.eval_grid_f32(lam_m, o, w, G, out=f32)
    out["field32_ms"] = round(timed(lambda: svo.eval_grid_f32(lam_m, o, w, G, out=f32), 1), 3)
    f64 = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    svo.eval_grid(torch.from_numpy(x_ref).cuda(), o, w, G, out=f64)
    mx, ss = 0.0, 0.0
    step = M * M * 64
    for k in range(0, M ** 3, step):
        dd = f32[k:k + step].double() - f64[k:k + step]
        mx = max(mx, float(dd.abs().max().item()))
        ss += float((dd * dd).sum().item())
    out["field_grid"] = "%d^3" % M
    out["field_max"] = mx / scale
    out["field_rms"] = float(np.sqrt(ss / M ** 3)) / scale
    out["scale"] = "coefficients: max |lambda_FP64|; field: max |b|"
    del f32, f64
    return out


def run_pipeline(ctx, net, norm, V, F, o, w, wl, timed, reps=3):
    """ThinShells' call order through the C ABI, host mesh in and host triangle soups out:
    the mesh is copied to the device once, then ctor (octree) -> creatShell (samples, signed
    distance at the corner vertices, learned fit, iso levels) -> mcVisualization (field once on
    the device, marching cubes at the outer, inner and zero levels, soups to host) with every
    intermediate kept on the device. Per-stage times and the whole sequence's wall time
    (median of reps)."""
    import torch
    from its_b200 import Svo
    from its_b200.api import learned_fit
    R = wl["mc_res"]
    stages = {k: [] for k in ("upload", "octree", "samples", "signed_distance", "fit", "iso", "field_mc")}
    walls, tris = [], None
    Vh, Fh = np.ascontiguousarray(V), np.ascontiguousarray(F, np.int32)
    for _ in range(reps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t = time.perf_counter()

        def lap(name):
            nonlocal t
            torch.cuda.synchronize()
            now = time.perf_counter()
            stages[name].append((now - t) * 1e3)
            t = now

        Vd, Fd = ctx.to_device(Vh), ctx.to_device(Fh)  # its_copy_to_device
        lap("upload")
        svo = Svo(ctx, Vd, Fd, wl["res"], o, w)
        lap("octree")
        pts, _ = svo.shell_samples(Vd, Fd, device=True)
        lap("samples")
        b = torch.empty(svo.num_verts, dtype=torch.float64, device="cuda")
        ctx.signed_distance(svo.vertex_positions_device(), Vd, Fd, out=b)
        lap("signed_distance")
        lam = torch.empty_like(b)
        _, rep = learned_fit(svo, net, b, norm, wl["tol"], out=lam)
        lap("fit")
        inner, outer, _ = svo.shell_iso_values(lam, torch.cat([Vd, pts]))
        lap("iso")
        soups = svo.grid_mc(lam, o, w, R, [outer, inner, 0.0], fast=True)
        lap("field_mc")
        walls.append((time.perf_counter() - t0) * 1e3)
        tris = [int(s.shape[0] // 3) for s in soups]
        svo.close()
    med = {k: round(statistics.median(v[1:]), 3) for k, v in stages.items()}
    return {"ms": round(statistics.median(walls[1:]), 3), "stages_ms": med, "triangles": tris,
            "rel_residual": rep["rel_residual"],
            "note": "host mesh in (copied to the device once), host triangle soups out, intermediates on the "
                    "device; MC at %d^3 with the field by prolongation (its_eval_grid_mc); wall time of the whole "
                    "sequence, median of %d runs after one warm-up" % (R, reps)}


def run_batch(ctx, net, norm, timed, tol, world, rank, steps, pg):
    """The uneven multi-mesh workload (256 meshes, 2k-200k faces; this rank's LPT share):
    the plain FP64 LSCG as one batched solve per chunk of meshes (assembly included), against
    one learned batch."""
    import torch
    from its_b200 import STOP_RESIDUAL, Operator, Svo, lib, meshes, model_to_unit_cube, uniform_bbox
    from its_b200.api import fit_residual_batch, learned_start_batch, solve_batch
    mix = meshes.batch_meshes(256, 3)
    mine = batch_shard([m["faces"] for m in mix], world, rank)
    svos, bs, outs, boxes = [], [], [], []
    for k in mine:
        m = mix[k]
        V = model_to_unit_cube(m["V"])
        o, _, w = uniform_bbox(V)
        s = Svo(ctx, V, m["F"], m["res"], o, w)
        boxes.append((np.ascontiguousarray(o), np.ascontiguousarray(w)))
        svos.append(s)
        bs.append(torch.from_numpy(ctx.signed_distance(s.vertices()[0], V, m["F"])).cuda())
        outs.append(torch.empty_like(bs[-1]))
    its = []
    # chunks of at most ~1.2 G operator entries (A and A^T: ~29 GB) per batched solve
    est = [40 * s.num_verts for s in svos]
    chunks, cur, acc = [], [], 0
    for i, e in enumerate(est):
        if cur and acc + e > 1_200_000_000:
            chunks.append(cur)
            cur, acc = [], 0
        cur.append(i)
        acc += e
    if cur:
        chunks.append(cur)

    def plain():
        its.clear()
        for ch in chunks:
            ops = [Operator(svos[i]) for i in ch]
            _, reps = solve_batch(ops, [bs[i] for i in ch], tol=tol, stop_rule=STOP_RESIDUAL,
                                  outs=[outs[i] for i in ch])
            its.extend(r["iterations"] for r in reps)
            for op in ops:
                op.close()

    rel = []

    def learned():
        learned_start_batch(svos, net, bs, norm, outs=outs)
        rel[:] = list(fit_residual_batch(svos, bs, outs))

    plain()
    plain_ms = timed(plain, max(1, steps - 1))
    learned()
    learned_ms = timed(learned, steps)
    R = 256
    fld = torch.empty((R + 1) ** 3, dtype=torch.float64, device="cuda")
    cube = torch.empty(R ** 3, dtype=torch.uint8, device="cuda")
    nv = C.c_int64(0)
    tris = []

    def mc_all(fast=False):
        tris.clear()
        for s, x, (o, w) in zip(svos, outs, boxes):
            if fast:  # the octree's own box at 256^3: the field by prolongation
                s.eval_grid_fast(x, o, w, R, out=fld)
            else:
                s.eval_grid(x, o, w, R, out=fld)
            ctx.check(lib().its_marching_cubes(ctx.h, C.c_void_p(fld.data_ptr()), R, o.ctypes.data_as(C.c_void_p),
                                               w.ctypes.data_as(C.c_void_p), 0.0, C.c_void_p(cube.data_ptr()), None, 0,
                                               C.byref(nv)), "its_marching_cubes")
            tris.append(nv.value // 3)

    mc_ms = timed(mc_all, 1)
    tris_exact = sum(tris)
    mc_fast_ms = timed(lambda: mc_all(True), 1)
    tris_fast = sum(tris)
    tot = batch_totals({"plain_ms": plain_ms, "learned_ms": learned_ms, "mc_ms": mc_ms, "mc_fast_ms": mc_fast_ms,
                        "meshes": len(mine), "unknowns": sum(s.num_verts for s in svos),
                        "iterations": float(sum(its)), "triangles": tris_exact, "triangles_fast": tris_fast,
                        "max_rel_residual": float(max(rel))}, pg)
    out = {"workload": "256 meshes, faces log-uniform in [2k, 200k] (seed 3): geodesic spheres / tori / "
                       "superquadrics, SVO depth 7-9; fit to 1e-6 relative residual",
           "meshes": int(tot["meshes"]), "unknowns": int(tot["unknowns"]),
           "plain_fp64_ms": round(tot["plain_ms"], 3), "plain_iterations_mean": tot["iterations"] / tot["meshes"],
           "plain_form": "assembly + its_lscg_solve_batch (one SpMV / reduction launch per step for all meshes of a "
                         "chunk, graph-captured), %d chunk(s) per rank" % len(chunks),
           "learned_ms": round(tot["learned_ms"], 3), "learned_max_rel_residual": tot["max_rel_residual"],
           "speedup": round(tot["plain_ms"] / tot["learned_ms"], 2),
           "sharding": ("LPT by faces over %d ranks" % world) if world > 1 else "single",
           "mc_256": {"ms": round(tot["mc_ms"], 2), "mvox_s": round(256 * R ** 3 / (tot["mc_ms"] * 1e-3) / 1e6, 1),
                      "triangles": int(tot["triangles"]), "iso": 0.0, "field": "FP64, point by point (its_eval_grid)"},
           "mc_256_fast": {"ms": round(tot["mc_fast_ms"], 2),
                           "mvox_s": round(256 * R ** 3 / (tot["mc_fast_ms"] * 1e-3) / 1e6, 1),
                           "triangles": int(tot["triangles_fast"]), "iso": 0.0,
                           "field": "FP64 by prolongation on each octree's lattice (its_eval_grid_fast)"}}
    for s in svos:
        s.close()
    return out


def cpu_fit(V, F, o, w, wl, b):
    """The oracle's fit (assembly + Eigen-semantics CGLS) on all host cores."""
    import oracle
    ref = oracle.Svo(V, F, wl["res"], o, w)
    t0 = time.perf_counter()
    rp, col, val = ref.assemble()
    x, rep = oracle.cgls(rp, col, val, b, wl["tol"], 100000, 1)
    t = (time.perf_counter() - t0) * 1e3
    return {"value": round(t, 2), "unit": "ms", "cores": os.cpu_count(), "kind": "port",
            "sample": "full fit (assembly + CGLS to %g relative residual, %d iterations) of the same workload"
                      % (wl["tol"], rep["iterations"])}


def cpu_stages(V, F, o, w, wl):
    """Every stage of the pipeline on the host cores with the oracle (the C++/OpenMP
    restatement of the reference), on the same workload. The dense field and marching cubes
    run on a 4x coarser grid (64x fewer points) and are scaled to the MC grid; the
    reference-semantics solve (Eigen's defaults: tol = machine epsilon, max 2n iterations,
    the normal-equation test) runs a bounded number of iterations, reported per iteration."""
    import oracle
    out = {"cores": os.cpu_count(), "threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())),
           "kind": "port"}

    def clock(fn):
        t0 = time.perf_counter()
        r = fn()
        return r, round((time.perf_counter() - t0) * 1e3, 2)

    s, out["octree_ms"] = clock(lambda: oracle.Svo(V, F, wl["res"], o, w))
    (pts, _), out["samples_ms"] = clock(s.intersections)
    pos, _ = s.vertices()
    b, out["signed_distance_ms"] = clock(lambda: oracle.signed_distance_bvh(pos, V, F))
    (rp, col, val), out["assembly_ms"] = clock(s.assemble)
    (x, rep), out["cgls_ms"] = clock(lambda: oracle.cgls(rp, col, val, b, wl["tol"], 100000, 1))
    out["cgls_iterations"] = rep["iterations"]
    samples = np.vstack([V, pts])
    _, out["iso_ms"] = clock(lambda: s.eval_points(x, samples))
    R = wl["mc_res"]
    Rs = max(R // 4, 8)
    g, t_field = clock(lambda: s.eval_grid(x, o, w, Rs))
    _, t_mc = clock(lambda: oracle.marching_cubes(g, Rs, o, w, 0.0, with_triangles=True))
    scale = (R / Rs) ** 3
    out["field_ms"] = round(t_field * scale, 1)
    out["mc_ms"] = round(t_mc * scale, 1)
    out["field_mc_sample"] = "%d^3 grid, scaled by %d to %d^3" % (Rs, int(scale), R)
    kref = 60 if s.num_verts > 50000 else 400
    (_, rr), t_ref = clock(lambda: oracle.cgls(rp, col, val, b, 2.220446049250313e-16, kref, 0))
    out["reference_semantics"] = {"ms_per_iteration": round(t_ref / max(rr["iterations"], 1), 3),
                                  "iterations_run": rr["iterations"], "max_iterations": 2 * s.num_verts,
                                  "normal_rel_residual": rr["normal_rel_residual"],
                                  "projected_ms_at_max_iterations": round(t_ref / max(rr["iterations"], 1) * 2
                                                                          * s.num_verts, 0)}
    out["total_ms"] = round(sum(out[k] for k in ("octree_ms", "samples_ms", "signed_distance_ms", "assembly_ms",
                                                 "cgls_ms", "iso_ms", "field_ms", "mc_ms")), 1)
    return out


def run_reference(args):
    """The CPU restatement of the reference's fit (oracle/) on the host cores: octree, right-hand
    side and assembly as untimed setup where the step does not include them; each step is the
    reference's cpCoefficients (assembly + LSCG). Nothing from libits is loaded."""
    rank, world, local = dist_setup()
    if rank != 0:
        return
    import oracle
    wl = WORKLOADS[args.config]
    V, F, o, w = prepared(wl, oracle)
    ref = oracle.Svo(V, F, wl["res"], o, w)
    pos, _ = ref.vertices()
    b = oracle.signed_distance_bvh(pos, V, F)
    times, reps, nnz = [], None, 0
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        rp, col, val = ref.assemble()
        x, reps = oracle.cgls(rp, col, val, b, wl["tol"], 100000, 1)
        t = (time.perf_counter() - t0) * 1e3
        nnz = len(val)
        if k >= args.warmup:
            times.append(t)
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 2), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(wl, ref.num_verts, nnz),
            "method": "oracle (C++/OpenMP restatement of ThinShells::cpCoefficients: assembly + Eigen-semantics "
                      "CGLS to the workload's tolerance, %d iterations); right-hand side from the oracle's BVH "
                      "signed distance (untimed setup)" % reps["iterations"],
            "cpu_baseline": {"value": round(v, 2), "unit": "ms", "cores": os.cpu_count(), "kind": "port",
                             "sample": "full fit (assembly + CGLS) per step"},
            "e2e": {"value": round(v, 2), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline legs")
    ap.add_argument("--no-batch", action="store_true", help="skip the multi-mesh batch leg")
    ap.add_argument("--only", default="all", choices=["all", "fit", "pipeline"],
                    help="fit: time the fit steps only; pipeline: the facade-order pipeline only")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.gpus > 1 and "RANK" not in os.environ:
        sys.exit(launch_ranks(sys.argv[1:], args.gpus))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
