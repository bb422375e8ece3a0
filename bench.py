#!/usr/bin/env python
"""Thin-shell fit benchmark (one JSON line on stdout from rank 0).

Workload (default): the (3,5) torus-knot tube -- 4,096 rings x 128 segments = 1,048,576
faces, FP32 vertices with N(0, 1e-3) jitter (seed 1) -- normalised to the unit cube, SVO
depth 9 (256^3 voxels), plain FP64 LSCG to 1e-6 relative residual, marching cubes at 512^3.

A step is one fit: operator assembly (ThinShells::cpCoefficients) plus the LSCG solve to
the stopping tolerance, inputs (octree, right-hand side) already resident in HBM. `value`
is the fit time in ms (max over ranks); `e2e` is the same fit through the C ABI with the
right-hand side in pinned host memory and the coefficients read back every step. Also
reported: the mixed-precision fit, marching-cubes throughput, the SVO build, the SpMV
roofline and the CPU oracle on the host cores.

--impl reference times the CPU restatement of the reference's fit (oracle/, OpenMP on all
host cores) on the same workload.
"""
import argparse
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

METRIC = "fit ms to 1e-6 rel. residual (learned+mixed vs plain FP64, 1 B200); MC Mvox/s"
WORKLOADS = {
    "c1": dict(mesh="c1", res=256, tol=1e-6, mc_res=512,
               desc="(3,5) torus-knot tube r=0.08, 4096 rings x 128 segments = 1,048,576 faces, FP32 vertices "
                    "+ N(0,1e-3) jitter (seed 1); SVO depth 9 (256^3); FP64 LSCG to 1e-6 relative residual; "
                    "MC 512^3"),
    "c0": dict(mesh="c0", res=32, tol=1e-6, mc_res=128,
               desc="perturbed geodesic sphere, 10,240 faces (seed 0); SVO depth 6 (32^3); FP64 LSCG to 1e-6 "
                    "relative residual; MC 128^3"),
}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


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


def prepared(wl):
    from its_b200 import meshes, model_to_unit_cube, uniform_bbox
    V, F = meshes.config_mesh(wl["mesh"])
    V = model_to_unit_cube(V)
    o, _, w = uniform_bbox(V)
    return V, F, o, w


def dist_setup(args):
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


def run_ours(args):
    import torch
    from its_b200 import OP_FP32_VALUES, PREC_MIXED, STOP_RESIDUAL, Context, Operator, Svo, lib
    import ctypes as C

    rank, world, local = dist_setup(args)
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    wl = WORKLOADS[args.config]
    V, F, o, w = prepared(wl)
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

    # ---- setup: octree and right-hand side (signed distance at the corner vertices) ------
    svo_ms = timed(lambda: Svo(ctx, V, F, wl["res"], o, w).close(), 2)
    svo = Svo(ctx, V, F, wl["res"], o, w)
    pos, _ = svo.vertices()
    b = ctx.signed_distance(pos, V, F)
    n = svo.num_verts
    b_dev = torch.from_numpy(b).cuda()
    lam_dev = torch.empty_like(b_dev)
    rep_box = {}

    def fit_step():
        op = Operator(svo)
        _, rep = op.solve(b_dev, tol=wl["tol"], stop_rule=STOP_RESIDUAL, out=lam_dev)
        rep_box["rep"], rep_box["nnz"] = rep, op.nnz
        op.close()

    # The clock sampler starts before the warm-up so that nvidia-smi's start-up (NVML
    # initialisation, which stalls the driver) falls outside the timed steps.
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.5)
    for _ in range(args.warmup):
        fit_step()
    barrier_sync()
    launches0 = ctx.kernel_launches
    fit_ms = timed(fit_step, args.steps)
    launches = ctx.kernel_launches - launches0
    barrier_sync()
    clk = clocks.stop()
    fit_ms = max_ranks(fit_ms)
    rep, nnz = rep_box["rep"], rep_box["nnz"]
    if args.only == "fit":
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(fit_ms, 4), "unit": "ms", "only": "fit",
                              "iterations": rep["iterations"], "gpu_launches": launches}), flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    # breakdown: assembly alone, solve alone on a prepared operator
    asm_ms = timed(lambda: Operator(svo).close(), args.steps)
    op_s = Operator(svo)
    solve_ms = timed(lambda: op_s.solve(b_dev, tol=wl["tol"], stop_rule=STOP_RESIDUAL, out=lam_dev), args.steps)
    op_s.close()

    # ---- end to end through the C ABI: pinned host rhs in, coefficients out --------------
    b_host = torch.from_numpy(b).pin_memory()
    lam_host = torch.empty(n, dtype=torch.float64).pin_memory()
    b_np, lam_np = b_host.numpy(), lam_host.numpy()

    def e2e_step():
        op = Operator(svo)
        op.solve(b_np, tol=wl["tol"], stop_rule=STOP_RESIDUAL, out=lam_np)
        op.close()

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    barrier_sync()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = max_ranks((time.perf_counter() - t0) * 1e3 / args.steps)

    # ---- mixed precision fit -----------------------------------------------------------------
    rep_m = {}

    def mixed_step():
        op = Operator(svo, mode=OP_FP32_VALUES)
        _, r = op.solve(b_dev, tol=wl["tol"], stop_rule=STOP_RESIDUAL, precision=PREC_MIXED, ir_steps=3,
                        inner_tol=1e-3, out=lam_dev)
        rep_m["rep"] = r
        op.close()

    mixed_step()
    mixed_ms = max_ranks(timed(mixed_step, max(1, args.steps // 2)))

    # ---- roofline of the dominant kernel: the binned CSR SpMV ------------------------------
    op = Operator(svo)
    x_dev = torch.randn(n, dtype=torch.float64, device="cuda")
    y_dev = torch.empty_like(x_dev)
    # A alone (120 MB at this size) nearly fits the 126 MB L2, so every timed launch starts
    # from a flushed L2 (a 256 MB write), as in the CGLS loop where A and A^T alternate.
    flush = torch.empty(32 * 2 ** 20, dtype=torch.float64, device="cuda")
    spmv, samples = {}, {0: [], 1: []}
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
            samples[tr].append(e0.elapsed_time(e1))
    for tr in (0, 1):
        spmv[tr] = statistics.median(samples[tr])
    del flush
    op.close()
    spmv_bytes = 12 * nnz + 24 * n  # values 8 + columns 4 per entry; rowptr 8, x 8, y 8 per row
    dom = 1 if spmv[1] >= spmv[0] else 0
    peak, peak_kind = load_peaks()
    achieved = spmv_bytes / (spmv[dom] * 1e-3) / 1e9

    # ---- dense field + marching cubes ---------------------------------------------------------
    R = wl["mc_res"]
    M = R + 1
    field = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    lam_fit = lam_dev.clone()
    samples = np.vstack([V, svo.shell_samples(V, F)[0]])
    inner, outer, _ = svo.shell_iso_values(lam_fit.cpu().numpy(), samples)
    L = lib()
    o_np, w_np = np.ascontiguousarray(o), np.ascontiguousarray(w)
    cube = torch.empty(R ** 3, dtype=torch.uint8, device="cuda")
    nv = C.c_int64(0)

    def field_step():
        svo.eval_grid(lam_fit, o, w, R, out=field)

    def mc_step():
        st = L.its_marching_cubes(ctx.h, C.c_void_p(field.data_ptr()), R, o_np.ctypes.data_as(C.c_void_p),
                                  w_np.ctypes.data_as(C.c_void_p), float(outer), C.c_void_p(cube.data_ptr()), None, 0,
                                  C.byref(nv))
        ctx.check(st, "its_marching_cubes")

    field_step()
    mc_step()
    field_ms = timed(field_step, 2)
    mc_ms = timed(mc_step, 3)
    mc_mvox = R ** 3 / ((field_ms + mc_ms) * 1e-3) / 1e6

    # ---- CPU baseline: the oracle's fit on the host cores (rank 0, N = 1) -------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_fit(V, F, o, w, wl, b)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(fit_ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(fit_ms, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["desc"], "unknowns": n, "nnz": nnz, "iterations": rep["iterations"],
                       "rel_residual": rep["rel_residual"], "parallelism": "replicas" if world > 1 else "single",
                       "l2": "operator (A and A^T, %.0f MB) larger than the 126 MB L2" % (2 * 12 * nnz / 1e6)},
            "e2e": {"value": round(e2e_ms, 4), "unit": "ms", "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 8 * n},
            "roofline": {"bound": "hbm", "kernel": "kSpmvBinned (%s)" % ("A^T" if dom else "A"),
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                         "bytes_per_launch": spmv_bytes, "launch_ms": round(spmv[dom], 5), "traffic": None},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": launches,
            "mixed": {"fit_ms": round(mixed_ms, 4), "inner_iterations": rep_m["rep"]["inner_iterations"],
                      "rel_residual": rep_m["rep"]["rel_residual"]},
            "mc": {"res": R, "mvox_s": round(mc_mvox, 1), "field_ms": round(field_ms, 3), "mc_ms": round(mc_ms, 3),
                   "iso": outer, "tri_vertices": int(nv.value)},
            "svo_build_ms": round(svo_ms, 3),
            "fit_breakdown_ms": {"assembly": round(asm_ms, 3), "solve": round(solve_ms, 3)},
            "spmv_ms": {"A": round(spmv[0], 5), "AT": round(spmv[1], 5)},
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


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


def run_reference(args):
    rank, world, local = dist_setup(args)
    if rank != 0:
        return
    import oracle
    wl = WORKLOADS[args.config]
    V, F, o, w = prepared(wl)
    ref = oracle.Svo(V, F, wl["res"], o, w)
    pos, _ = ref.vertices()
    # Right-hand side (untimed setup): the same signed distances as the GPU arm, from libits;
    # the CPU exact winding number over 1M triangles would take hours on the host.
    from its_b200 import Context
    ctx = Context(local)
    b = ctx.signed_distance(pos, V, F)
    ctx.close()
    times, reps = [], None
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        rp, col, val = ref.assemble()
        x, reps = oracle.cgls(rp, col, val, b, wl["tol"], 100000, 1)
        t = (time.perf_counter() - t0) * 1e3
        if k >= args.warmup:
            times.append(t)
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 2), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["desc"], "unknowns": int(ref.num_verts), "iterations": reps["iterations"]},
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
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--only", default="all", choices=["all", "fit"], help="fit: time the fit steps only")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
