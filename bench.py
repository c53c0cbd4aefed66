#!/usr/bin/env python
"""Benchmark of the B200 caking hot path (kernels (a)+(b)+(c)) on a synthetic sweep.

One step = one batch of F frames of the seeded omega sweep, caked (2-D cake) and
eta-reduced (two lineouts) in one launch of the batched kernel, with the frames
already resident in HBM.  The sweep (1440 frames of 2880x2880 u16, 23.9 GB) is
larger than L2, and consecutive steps walk through it, so no step re-reads a
batch from L2.

Prints ONE JSON line (rank 0).  Besides the contract keys it reports the HBM
roofline of the batched kernel, the plain one-frame-per-launch kernel (the
reference GPU algorithm) timed on the same frames, the FP64-oracle error of a
sampled frame, the end-to-end rate through the public API with host frames,
and the reference's own CPU integrator timed on this host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "caked_frames_per_s"
# DRAM bytes (read + write) per 128-frame batch of the sweep_2880 workload: ncu
# dram__bytes_read.sum + dram__bytes_write.sum of one launch of each kernel of the batch (the
# transpose kernel k_xc plus the caking kernel of the encoding), summarised under profiles/; the
# mma figures are of the kernels of commit 6d0d9e4
TRAFFIC = {"runs": {"bytes_per_step": int(0.840295e9 + 0.761555e9 + 1.830098e9 + 1.170938e9),
                    "kernels": "k_xc + k_runs"},
           "mma": {"bytes_per_step": int(0.839898e9 + 0.762710e9 + 1.313836e9 + 0.861997e9),
                   "kernels": "k_xc + k_mma<7, 6>", "commit": "6d0d9e4",
                   # the default 8-slot pipeline runs the same tiles, runs and blob reads; only
                   # the number of stage slots in shared memory differs
                   "pipeline_captured": [7, 6]}}
SCOPE = {"runs": "whole batch: k_xc + k_runs + k_lineout (k_runs 88 %)",
         "mma": "whole batch: k_xc + k_mma + k_lineout",
         "mmad": "whole batch: k_mmad + k_lineout"}
UNIT = "frames/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sweep_2880")
    ap.add_argument("--batch", type=int, default=128, help="frames per launch (F)")
    ap.add_argument("--sweep-frames", type=int, default=1440)
    ap.add_argument("--tile-rows", type=int, default=0)
    ap.add_argument("--tile-pixels", type=int, default=0)
    ap.add_argument("--fpl", type=int, default=0)
    ap.add_argument("--encoding", default="mma", choices=["auto", "runs", "csr", "mma", "mmad"],
                    help="tile encoding of the batched plan (mma: tensor cores, the default for these u16 sweeps)")
    ap.add_argument("--run-len", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-e2e-cake", action="store_true", help="skip the end-to-end run that returns the cakes")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-fit", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the F = 1, 8, 32, 128 launch sweep")
    ap.add_argument("--no-eta-fits", action="store_true", help="skip the per-eta ring fits of the timed cake")
    ap.add_argument("--no-published", action="store_true",
                    help="skip the reference's published PILATUS3 2M configuration")
    ap.add_argument("--no-panels", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="skip the CUDA-graph replay of the batched step")
    ap.add_argument("--autotune", action="store_true", help="time candidate tile shapes / run lengths first")
    ap.add_argument("--mma-pipeline", default="", help="stages,producers of the tensor-core kernel (e.g. 6,6)")
    ap.add_argument("--no-sum", action="store_true", help="skip the SumImages sweep and its all-reduce")
    ap.add_argument("--panel-frames", type=int, default=256)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="duration of the 6-stream serving load, about 1.07 k frames/s offered "
                         "(10 s: the 10^4 frames the latency percentiles are taken over; 0 = skip)")
    ap.add_argument("--serve-trace", default="", help="write per-frame serving timestamps to <prefix>_*.npz")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def csr_map_bytes(info) -> int:
    """The map's algorithmic bytes: its CSR of the mode's coalesced terms (4 B column + 4 B
    weight each), n_bins + 1 row pointers and n_bins areas, 4 B each."""
    return int(info["nnz"]) * 8 + (int(info["n_bins"]) + 1) * 4 + int(info["n_bins"]) * 4


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def dist_max(x: float, world: int) -> float:
    """Max of x over the ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_first_frame(rank: int, sweep: int) -> int:
    """Replicas: rank r cakes its own slice of the omega sweep, frames r*sweep .. (r+1)*sweep-1
    (weak scaling; the slices never overlap, no data crosses between ranks)."""
    return rank * sweep


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
def cpu_reference_rate(pm, w, frame_u16, dark, seconds):
    """The reference's own integrator (integration_apply_map, compiled from the MIDAS
    sources into oracle/_ref; else the FP64 oracle port) on this host's cores:
    (frames/s, cores, kind, sample)."""
    import numpy as np
    import oracle
    ny, nz = w.mapper.NrPixelsY, w.mapper.NrPixelsZ
    img = frame_u16.astype(np.float64)
    dk = dark.astype(np.float64)
    recs, nmap = pm.pxList, pm.nmap_pairs()
    grad = 1 if w.mode == "gradient" else 0
    if oracle.ref_available():
        cores = oracle.ref().ref_max_threads()
        run = lambda: oracle.ref_integrate(recs, nmap, w.n_r, w.n_eta, img, ny, nz, dark=dk, bc_y=w.mapper.BC_y,
                                           bc_z=w.mapper.BC_z, gradient=grad, n_threads=cores, chunk_rows=8)
        kind = "reference"
    else:
        cores = 1
        sub = img - dk
        run = lambda: oracle.integrate(recs, nmap, pm.n_bins, ny, nz, sub, mode=w.mode, bc_y=w.mapper.BC_y,
                                       bc_z=w.mapper.BC_z)
        kind = "port"
    out = run()  # warm-up (page-in)
    n, t0 = 0, time.perf_counter()
    while True:
        run()
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 200:
            break
    return (n / el, cores, kind, f"{n} full {w.mapper.NrPixelsZ}x{w.mapper.NrPixelsY} frame(s) in {el:.1f} s",
            out)


def _rel(got, ref):
    import numpy as np
    nz = ref[ref != 0]
    tau = 1e-3 * np.median(np.abs(nz)) if nz.size else 1e-30
    return np.abs(got - ref) / np.maximum(np.abs(ref), tau)


def accuracy_check(pm, w, checked, dark, ref_out, kind, got_ic=None, encoding=""):
    """Outputs of the last timed launch (lanes 0, 1, 31, 63, 64, 95, 126, 127 of the F-frame
    batch) against the FP64 oracle, frame by frame; and, when the reference integrator ran,
    lane 0 of the same batch through a plan with IntegrationCore semantics on the same
    encoding against that integrator's own output (sums / norms of integration_apply_map)."""
    import numpy as np
    import oracle
    ny, nz = w.mapper.NrPixelsY, w.mapper.NrPixelsZ
    recs, nmap = pm.pxList, pm.nmap_pairs()
    area = oracle.area_in(recs, nmap, pm.n_bins, ny, nz)
    worst = {"cake_max_rel": 0.0, "cake_mean_rel": 0.0, "lineout_max_rel": 0.0, "lineout_sm_max_rel": 0.0}
    per_lane = []
    for i, lane in enumerate(checked["lanes"]):
        sub = (checked["frames"][i].astype(np.float32) - dark).astype(np.float64)
        ref, _ = oracle.integrate(recs, nmap, pm.n_bins, ny, nz, sub, mode=w.mode, bc_y=w.mapper.BC_y,
                                  bc_z=w.mapper.BC_z)
        aw_ref, sm_ref = oracle.profile(ref, area, w.n_r, w.n_eta)
        r = _rel(checked["cake"][i], ref)
        ra, rs = _rel(checked["lineout_aw"][i], aw_ref), _rel(checked["lineout_sm"][i], sm_ref)
        worst["cake_max_rel"] = max(worst["cake_max_rel"], float(r.max()))
        worst["cake_mean_rel"] = max(worst["cake_mean_rel"], float(r.mean()))
        worst["lineout_max_rel"] = max(worst["lineout_max_rel"], float(ra.max()))
        worst["lineout_sm_max_rel"] = max(worst["lineout_sm_max_rel"], float(rs.max()))
        per_lane.append({"lane": lane, "cake_max_rel": float(r.max())})
    acc = dict(worst, frames_checked=len(checked["lanes"]), lanes=checked["lanes"], batch=checked["batch"],
               source="outputs of the last timed launch", per_lane=per_lane)
    ic = None
    if kind == "reference" and w.mode in ("bilinear", "gradient") and got_ic is not None:
        sums, norms = ref_out
        ic_cake = np.where(norms > 1e-9, sums / np.where(norms > 1e-9, norms, 1.0), 0.0)
        ri, rp = _rel(got_ic, ic_cake), _rel(checked["cake"][0], ic_cake)
        ic = {"cake_max_rel": float(ri.max()), "cake_mean_rel": float(ri.mean()), "frames_checked": 1,
              "semantics": "ic (plan built with IntegrationCore's rounding and normaliser)",
              "encoding": encoding, "launch": "lane 0 of the timed batch, caked in one F-frame launch",
              "integrator": "integration_apply_map (IntegrationCore.c) compiled from the reference, sums / norms",
              "py_semantics_cake_max_rel": float(rp.max())}
    return acc, ic


def served_accuracy(served):
    """Max relative error of each served stream's first lineout against the FP64 oracle."""
    import numpy as np
    import oracle
    worst = 0.0
    for c, frame, lineout in served:
        pm = c.pixmap
        ck, _ = oracle.integrate(pm.pxList, pm.nmap_pairs(), pm.n_bins, c.n_pixels_y, c.n_pixels_z,
                                 (frame.astype(np.float32) - c.dark).astype(np.float64), mode=c.mode,
                                 bc_y=c.bc_y, bc_z=c.bc_z)
        area = oracle.area_in(pm.pxList, pm.nmap_pairs(), pm.n_bins, c.n_pixels_y, c.n_pixels_z)
        ref, _ = oracle.profile(ck, area, c.n_r, c.n_eta)
        worst = max(worst, float(_rel(lineout, ref).max()))
    return worst


def main_ours(args):
    import numpy as np
    import torch

    from midas_b200 import _lib as L, synth
    from midas_b200.kernels import CakePlan
    from midas_b200.mapper import build_map

    rank, world, local = dist_setup(args)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    w = synth.WORKLOADS[args.workload]()
    ny, nz = w.mapper.NrPixelsY, w.mapper.NrPixelsZ
    F = args.batch
    t_setup = time.time()
    pm, _ = build_map(w.mapper, device=local)
    t_map = time.time() - t_setup
    tuned = None
    if args.autotune:
        from midas_b200 import autotune
        sample = w.frames(0, F, device=dev)
        t1 = time.time()
        tuned = autotune.tune(pm, sample, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=ny, n_pixels_z=nz, mode=w.mode,
                              bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z, device=dev)
        tuned_s = time.time() - t1
        del sample
        args.tile_rows, args.run_len, args.tile_pixels = (tuned.best["tile_rows"], tuned.best["run_len"],
                                                          tuned.best["tile_pixels"])
        args.encoding = tuned.best["encoding"]
    t1 = time.time()
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=ny, n_pixels_z=nz, mode=w.mode,
                    bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z, device=dev,
                    tile_rows=args.tile_rows or w.tile_rows, tile_pixels=args.tile_pixels,
                    frames_per_lane=args.fpl, encoding=args.encoding, run_len=args.run_len)
    t_plan = time.time() - t1
    pipeline = None
    if tuned is not None and tuned.best.get("pipeline"):
        pipeline = tuple(tuned.best["pipeline"])
    elif args.mma_pipeline:
        pipeline = tuple(int(x) for x in args.mma_pipeline.split(","))
    if pipeline is not None:
        plan.set_mma_pipeline(*pipeline)
    info = plan.info
    dark = w.dark(device=dev)
    dark_np = dark.cpu().numpy()
    plan.set_dark(dark_np)
    sweep = max(F, (args.sweep_frames // F) * F)
    frames = torch.empty((sweep, nz, ny), dtype=torch.uint16, device=dev)
    for s in range(0, sweep, 256):
        w.frames(rank_first_frame(rank, sweep) + s, min(256, sweep - s), out=frames[s:s + 256])
    torch.cuda.synchronize()
    n_batches = sweep // F
    cake = torch.empty((F, w.n_r, w.n_eta), dtype=torch.float32, device=dev)
    aw = torch.empty((F, w.n_r), dtype=torch.float64, device=dev)
    sm = torch.empty((F, w.n_r), dtype=torch.float64, device=dev)
    bufs = {"cake": cake, "lineout_aw": aw, "lineout_sm": sm}

    def step(i):
        b = i % n_batches
        plan.integrate(frames[b * F:(b + 1) * F], out=bufs)

    # ---- the last timed step's batch: its outputs are kept for the accuracy check (lanes
    # 0, 1, 31, 63, 64, 95, 126, 127 of the timed F-frame launch)
    b_last = (args.warmup + args.steps - 1) % n_batches
    lanes = [k for k in (0, 1, 31, 63, 64, 95, 126, 127) if k < F]

    # ---- warm-up, then K timed steps
    stream = torch.cuda.current_stream()
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        step(args.warmup + i)
        ev[i][1].record(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clk = clocks.stop()
    checked = {"frames": np.stack([frames[b_last * F + k].cpu().numpy() for k in lanes]),
               "cake": np.stack([bufs["cake"][k].reshape(-1).cpu().numpy() for k in lanes]).astype(np.float64),
               "lineout_aw": np.stack([bufs["lineout_aw"][k].cpu().numpy() for k in lanes]),
               "lineout_sm": np.stack([bufs["lineout_sm"][k].cpu().numpy() for k in lanes]),
               "lanes": lanes, "batch": b_last}
    frame0 = checked["frames"][0]
    elapsed_ms = dist_max(e0.elapsed_time(e1), world)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    value = world * args.steps * F / (elapsed_ms / 1e3)
    # kernels per step: per 256-frame launch group one k_lineout, plus either one caking
    # kernel or (pixel-major staging) k_xc + k_runs per 128 frames
    groups = [min(256, F - f0) for f0 in range(0, F, 256)]
    if info["xc_pixels"] > 0:
        launches = args.steps * sum(1 + 2 * math.ceil(g / 128) for g in groups)
    else:
        launches = args.steps * 2 * len(groups)

    # ---- roofline of the batched launch: A(F) = map bytes + F * frame bytes, the map counted as
    # its CSR (nnz x (4 B column + 4 B weight) + (n_bins + 1) x 4 B row pointers + n_bins x 4 B
    # area), whatever encoding the plan keeps it in
    peak, peak_kind = measured_peak()
    frame_bytes = ny * nz * 2
    map_bytes = csr_map_bytes(info)
    alg = map_bytes + F * frame_bytes
    mean_step_s = sum(step_ms) / len(step_ms) / 1e3
    achieved = alg / mean_step_s / 1e9
    ref_bytes = map_bytes + F * (info["ref_pixels"] * 2 + w.n_r * w.n_eta * 4)
    # DRAM bytes (read + write) of the batch's kernels from the ncu captures of this workload at
    # F = 128 (TRAFFIC); other shapes: not captured
    enc = args.encoding if args.encoding != "auto" else "runs"
    traffic = None
    if w.name.startswith("sweep_2880") and F == 128 and info["xc_pixels"] > 0 and enc in TRAFFIC:
        traffic = dict(TRAFFIC[enc], source="ncu dram__bytes_read.sum + dram__bytes_write.sum")
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                "alg_bytes_per_launch": alg, "scope": SCOPE.get(enc, "whole batch"),
                "achieved_touched_bytes": round(ref_bytes / mean_step_s / 1e9, 1)}

    out = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 4), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": w.name, "frames_per_step": F, "sweep_frames": sweep,
                      "mode": w.mode, "n_bins": w.n_r * w.n_eta, "nnz": info["nnz"],
                      "map_records": info["n_records"], "tiles": info["n_tiles"],
                      "tile_rows": info["tile_rows"], "tile_pixels": info["tile_pixels"],
                      "frames_per_lane": info["frames_per_lane"],
                      "encoding": enc,
                      "mma_pipeline": list(pipeline) if pipeline else ([8, 6] if enc == "mma" else None),
                      "run_len": info["run_len"], "staged_pixels_per_frame": info["staged_pixels"],
                      "referenced_pixels": info["ref_pixels"], "map_bytes": map_bytes,
                      "plan_map_bytes_read": info["map_bytes"],
                      "l2": "inputs larger than L2: each step reads a new %.1f GB batch" % (F * frame_bytes / 1e9),
                      "parallelism": f"replicas{world}"},
           "roofline": roofline, "gpu_launches": launches,
           "setup_s": {"map_build_gpu": round(t_map, 2), "plan_build": round(t_plan, 2)}}
    if clk:
        out["clocks"] = clk
    if tuned is not None:
        out["autotune"] = {"best": tuned.best, "best_ms": tuned.best_ms, "candidates": tuned.table,
                           "seconds": round(tuned_s, 1)}

    # ---- per-eta ring fits of the timed batch's cake (IntegratorZarrOMP.c:1902-2030)
    if not args.no_eta_fits:
        out["eta_fits"] = eta_fit_bench(bufs["cake"], w, dev)

    # ---- frames per launch F = 1, 8, 32, 128: one launch per step, new frames every step
    if not args.no_sweep:
        out["f_sweep"] = f_sweep(plan, frames, bufs, F, info, w, args, world, peak)

    # ---- the same steps replayed from CUDA graphs (one graph per resident batch)
    if not args.no_graph:
        graphs = [plan.capture(frames[b * F:(b + 1) * F], bufs) for b in range(n_batches)]
        for i in range(args.warmup):
            graphs[i % n_batches].replay()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for i in range(args.steps):
            graphs[(args.warmup + i) % n_batches].replay()
        g1.record(stream)
        torch.cuda.synchronize()
        gms = dist_max(g0.elapsed_time(g1), world)
        out["graph"] = {"frames_per_s": round(world * args.steps * F / (gms / 1e3), 1),
                        "ms_per_step": round(gms / args.steps, 4), "graphs": n_batches,
                        "nodes_per_graph": "memset + k_xc + caking kernel per 128 frames, k_lineout"}
        del graphs

    # ---- SumImages over the sweep (midas_b200.sweep): every resident batch caked with its
    # cakes added to an FP64 running sum, then the sum all-reduced over the ranks (the path's
    # one collective; a no-op at N = 1)
    if not args.no_sum:
        from midas_b200.sweep import SweepSum
        ssum = SweepSum(plan)
        plan.integrate(frames[:F], out=bufs, sum_into=ssum.total)     # warm-up
        ssum.total.zero_()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for b in range(n_batches):
            ssum.add(plan, frames[b * F:(b + 1) * F], out=bufs)
        s1.record(stream)
        torch.cuda.synchronize()
        sms = dist_max(s0.elapsed_time(s1), world)
        barrier(world)
        r0 = time.perf_counter()
        total = ssum.reduce()
        torch.cuda.synchronize()
        red_ms = dist_max((time.perf_counter() - r0) * 1e3, world)
        out["sum_images"] = {"frames_summed": world * ssum.frames, "ms_per_batch_with_sum": round(sms / n_batches, 4),
                             "all_reduce_ms": round(red_ms, 3), "all_reduce_bytes": total.numel() * 8,
                             "sum_of_sum": float(total.sum().item())}
        del ssum, total

    # ---- plain one-frame-per-launch kernel (reference GPU algorithm) on the same frames
    if not args.no_plain:
        P = 16
        for k in range(2):
            plan.integrate_plain(frames[k])
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for k in range(P):
            plan.integrate_plain(frames[(k * 37) % sweep])
        b.record(stream)
        torch.cuda.synchronize()
        plain_fps = P / (a.elapsed_time(b) / 1e3)
        out["plain"] = {"frames_per_s": round(plain_fps, 1), "frames": P,
                        "speedup_batched_vs_plain": round(value / world / plain_fps, 2)}

    # ---- end to end through the public API: pinned host frames -> cake + lineouts -> host lineouts
    if not args.no_e2e:
        out["e2e"] = e2e_rate(plan, frames, F, args, w, dev, world)
        # the same with the cakes returned to host memory (the reference's Write2D consumer)
        if rank == 0 and world == 1 and not args.no_e2e_cake:
            out["e2e_with_cake"] = e2e_rate(plan, frames, F, args, w, dev, 1, with_cake=True)

    # ---- ring fits of every resident frame: all rings in one launch, PV and TCH
    fit_sample = None
    if not args.no_fit:
        out["fits"], fit_sample = fit_bench(plan, frames, w, F, dev)

    # ---- the reference's published configuration (PILATUS3 2M), beside its H100 numbers
    if rank == 0 and world == 1 and not args.no_published:
        out["published_config"] = published_bench(args, dev)

    # ---- uneven multi-panel batch: five panels, one merged Q x eta cake (rank 0, N = 1)
    panel_sample = None
    if rank == 0 and world == 1 and not args.no_panels:
        out["multipanel"], panel_sample = panel_bench(args, dev)

    # the timed batch, kept on the device for the IntegrationCore-semantics check
    frames_ic = frames[b_last * F:(b_last + 1) * F].clone() if (rank == 0 and world == 1 and not args.no_cpu
                                                               and not args.no_check) else None

    # ---- serving load: six streams with different maps, Poisson arrivals (rank 0, N = 1)
    served = []
    if rank == 0 and world == 1 and args.serve_seconds > 0:
        del frames
        plan.close()
        torch.cuda.empty_cache()
        out["serving"], served = serving_load(args, dev, plain=False)
        out["serving"]["plain_loop"], _ = serving_load(args, dev, plain=True)

    # ---- CPU leg (rank 0, N = 1): the reference integrator timed on this host's cores, and
    # the accuracy of frame 0 and of the served lineouts against it and the FP64 oracle
    if rank == 0 and world == 1 and not args.no_cpu:
        fps, cores, kind, sample, ref_out = cpu_reference_rate(pm, w, frame0, dark_np, args.cpu_seconds)
        out["cpu_baseline"] = {"value": round(fps, 3), "unit": UNIT, "cores": cores, "kind": kind,
                               "sample": sample}
        if not args.no_check:
            got_ic = None
            if kind == "reference" and w.mode in ("bilinear", "gradient"):
                # IntegrationCore semantics on the same encoding, over the whole timed batch
                plan_ic = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=ny, n_pixels_z=nz, mode=w.mode,
                                   semantics="ic", bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z, device=dev,
                                   tile_rows=args.tile_rows or w.tile_rows, encoding=args.encoding)
                plan_ic.set_dark(dark_np)
                c_ic, _, _ = plan_ic.integrate(frames_ic, lineouts=False)
                got_ic = c_ic[0].reshape(-1).cpu().numpy().astype(np.float64)
                del c_ic
                plan_ic.close()
            out["accuracy_vs_fp64_oracle"], ic = accuracy_check(pm, w, checked, dark_np, ref_out, kind, got_ic,
                                                                args.encoding)
            if ic:
                out["accuracy_vs_reference_integrator"] = ic
            if served:
                out["serving"]["lineout_max_rel_vs_fp64_oracle"] = served_accuracy(served)
            if panel_sample is not None:
                out["multipanel"]["accuracy_vs_fp64_oracle"] = panel_accuracy(panel_sample)
            if fit_sample is not None:
                for model, acc in fit_accuracy(fit_sample).items():
                    out["fits"][model].update(acc)
    if rank == 0:
        print(json.dumps(out), flush=True)
    plan.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def serving_load(args, dev, plain=False, n_distinct=8):
    """Six concurrent detector streams (synth.serving_mix) with Poisson frame arrivals served
    by CakeServer for ``--serve-seconds``; a seventh stream with a fresh map is admitted
    half way through.  Latency = scheduled arrival -> lineouts + fits on the host."""
    import threading

    import numpy as np
    import torch

    from midas_b200 import synth
    from midas_b200.server import AdmissionError, CakeServer, DeviceBackend

    T = args.serve_seconds
    mix = synth.serving_mix()

    def cfg_of(w, rate):
        c = synth.serving_stream(w, device=dev.index)
        c.max_batch = 16 if rate >= 100 else 4
        return c

    streams = [(cfg_of(w, rate), rate, synth.host_frames(w, 0, n_distinct, dev.index)) for w, rate in mix]
    late_w, late_rate = synth.late_stream()
    late_frames = synth.host_frames(late_w, 0, n_distinct, dev.index)
    backend = DeviceBackend(device=dev.index, max_batch=16, max_inflight=2, plain=plain)
    srv = CakeServer(backend=backend).start()
    sids = [srv.admit(c) for c, _, _ in streams]
    # warm-up: every stream once (plan upload, first launches), then clear the counters
    warm = [srv.submit(sid, fr[0]) for sid, (_, _, fr) in zip(sids, streams)]
    for f in warm:
        f.result(timeout=300)
    srv.latencies.clear()
    srv.completed = srv.batches = 0
    srv.reset_pass_stats()
    backend.dispatch_stats(reset=True)
    backend.alg_bytes = backend.launches = 0
    per_stream = {}
    offered = {}
    stop_at = [0.0]
    late_info = {}

    def producer(name, sid, rate, frames, seed, t_end):
        rng = np.random.default_rng(seed)
        t = time.perf_counter()
        futs = []
        i = 0
        while True:
            t += rng.exponential(1.0 / rate)
            if t >= t_end:
                break
            d = t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            futs.append(srv.submit(sid, frames[i % len(frames)], t_arrival=t))
            i += 1
        offered[name] = i
        per_stream[name] = futs

    def late():
        time.sleep(T / 2)
        t0 = time.perf_counter()
        try:
            c = cfg_of(late_w, late_rate)
            t1 = time.perf_counter()
            sid = srv.admit(c)
        except AdmissionError as e:
            late_info.update(admitted=False, reason=str(e))
            return
        t2 = time.perf_counter()
        # map_s: map on the device, dark, ring windows; plan_s: plan build, dark upload, buffers
        late_info.update(admitted=True, admit_s=round(t2 - t0, 3), map_s=round(t1 - t0, 3),
                         plan_s=round(t2 - t1, 3), name=c.name, window=(t0, t2))
        producer(c.name, sid, late_rate, late_frames, 99, stop_at[0])

    # the host loop is Python: keep the cyclic garbage collector's pauses out of the window,
    # and let the scheduler thread take the interpreter lock back within 0.5 ms of a
    # producer or writer thread holding it (the default switch interval is 5 ms)
    import gc
    import sys
    gc.collect()
    gc.freeze()
    gc.disable()
    switch = sys.getswitchinterval()
    sys.setswitchinterval(5e-4)
    t_start = time.perf_counter()
    stop_at[0] = t_start + T
    th = [threading.Thread(target=producer, args=(c.name, sid, rate, fr, k, stop_at[0]))
          for k, (sid, (c, rate, fr)) in enumerate(zip(sids, streams))]
    th.append(threading.Thread(target=late))
    for t in th:
        t.start()
    for t in th:
        t.join()
    results = {name: [f.result(timeout=600) for f in futs] for name, futs in per_stream.items()}
    t_done = time.perf_counter()
    sys.setswitchinterval(switch)
    gc.enable()
    gc.unfreeze()
    srv.stop()
    wall = t_done - t_start
    lat = srv.latency_ms()
    n_done = sum(len(v) for v in results.values())
    streams_out = {}
    for name, res in results.items():
        a = np.sort(np.array([r.latency_s for r in res])) * 1e3
        streams_out[name] = {"frames": len(res), "p50_ms": round(float(np.percentile(a, 50)), 3) if len(a) else None,
                             "p99_ms": round(float(np.percentile(a, 99)), 3) if len(a) else None,
                             "mean_batch": round(float(np.mean([r.batch_size for r in res])), 2) if res else None}
    window = late_info.pop("window", None)
    if args.serve_trace:
        names = sorted(results)
        rows = [(names.index(n), r.t_arrival - t_start, r.t_submit - t_start, r.t_dispatch - t_start,
                 r.t_complete - t_start, r.batch_size) for n in names for r in results[n]]
        np.savez(f"{args.serve_trace}_{'plain' if plain else 'batched'}.npz", rows=np.array(rows),
                 names=np.array(names), window=np.array(window if window else (0.0, 0.0)) - t_start)
    if window:
        # frames that arrived while the late stream's map and plan were being built
        lo, hi = window[0], window[1] + 0.05
        steady = np.sort(np.array([r.latency_s for v in results.values() for r in v
                                   if not lo <= r.t_arrival <= hi])) * 1e3
        late_info["p99_ms_outside_admission"] = round(float(np.percentile(steady, 99)), 3)
        late_info["frames_during_admission"] = int(sum(lo <= r.t_arrival <= hi for v in results.values()
                                                       for r in v))
    # where the slowest 1 % of frames waited: arrival -> submit() (the producer thread late),
    # submit -> launch of its batch (queued in the server), launch -> result in host memory
    allr = [r for v in results.values() for r in v]
    tail_split = None
    if allr:
        cut = np.percentile([r.latency_s for r in allr], 99)
        worst = [r for r in allr if r.latency_s >= cut]
        tail_split = {k: round(float(np.median([f(r) for r in worst])) * 1e3, 3) for k, f in (
            ("submit_late_ms", lambda r: r.t_submit - r.t_arrival),
            ("queued_ms", lambda r: r.t_dispatch - r.t_submit),
            ("in_flight_ms", lambda r: r.t_complete - r.t_dispatch))}
        tail_split["frames"] = len(worst)
    ps = srv.pass_stats()
    ps = {k: (round(v, 3) if isinstance(v, float) else int(v)) for k, v in ps.items()}
    ps["max_pass_at"] = round(ps["max_pass_at"] - t_start, 3)   # seconds into the run
    if window:
        ps["admission_s"] = [round(window[0] - t_start, 3), round(window[1] - t_start, 3)]
    ps["dispatch_max_ms"] = {k: round(v, 3) for k, v in backend.dispatch_stats().items()}
    out = {"streams": len(streams) + (1 if late_info.get("admitted") else 0), "seconds": round(T, 2),
           "offered_frames": sum(offered.values()), "completed_frames": n_done,
           "frames_per_s": round(n_done / wall, 1), "p50_ms": round(lat["p50"], 3), "p99_ms": round(lat["p99"], 3),
           "max_ms": round(lat["max"], 3), "hbm_alg_gb_s": round(backend.alg_bytes / wall / 1e9, 2),
           "launch_calls": backend.launches, "batches": srv.batches,
           "mode": "plain one-frame-per-launch" if plain else "continuous batching",
           "late_stream": late_info, "p99_tail_median_split": tail_split, "scheduler": ps,
           "per_stream": streams_out,
           "latency": "scheduled Poisson arrival -> lineouts and ring fits in host memory"}
    # each producer's first request carried frames[0] of its stream
    served = [(c, fr[0], results[c.name][0].lineout_aw) for c, _, fr in streams if results.get(c.name)]
    del streams
    torch.cuda.empty_cache()
    return out, served


def panel_bench(args, dev, reps=3):
    """Five panels (four 2048^2 u16 around the beam, one 1475x1679 int32 with masked module
    gaps), one Q binning (0.002 1/A from 1 to 8, eta 2 deg), --panel-frames frames per panel
    caked into one merged cake per frame set."""
    import numpy as np
    import torch

    from midas_b200 import synth
    from midas_b200.kernels import PanelPlan
    from midas_b200.mapper import build_map

    ws = synth.panel_set()
    t0 = time.time()
    maps = [build_map(w.mapper, device=dev.index, mask=w.mask())[0] for w in ws]
    t_map = time.time() - t0
    t0 = time.time()
    plan = PanelPlan(maps, shapes=[(w.mapper.NrPixelsY, w.mapper.NrPixelsZ) for w in ws],
                     beam_centres=[(w.mapper.BC_y, w.mapper.BC_z) for w in ws], n_r=ws[0].n_r,
                     n_eta=ws[0].n_eta, mode=ws[0].mode, device=dev)
    t_plan = time.time() - t0
    darks = [w.dark(device=dev).cpu().numpy() for w in ws]
    plan.set_dark(darks)
    F = args.panel_frames
    dts = {"uint16": torch.uint16, "int32": torch.int32}
    frames = [w.frames(0, F, device=dev, dtype=dts[w.frame_dtype]) for w in ws]
    ck = torch.empty((F, ws[0].n_r, ws[0].n_eta), dtype=torch.float32, device=dev)
    aw = torch.empty((F, ws[0].n_r), dtype=torch.float64, device=dev)
    sm = torch.empty_like(aw)
    bufs = {"cake": ck, "lineout_aw": aw, "lineout_sm": sm}
    plan.integrate(frames, out=bufs)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        plan.integrate(frames, out=bufs)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    info = plan.info
    frame_bytes = sum(w.mapper.NrPixelsY * w.mapper.NrPixelsZ * np.dtype(w.frame_dtype).itemsize for w in ws)
    out = {"panels": [w.name for w in ws], "bins": f"{ws[0].n_r} Q x {ws[0].n_eta} eta",
           "map_records": [int(pm.n_entries) for pm in maps], "frames_per_panel": F,
           "ms_per_batch": round(ms, 3), "frame_sets_per_s": round(F / (ms / 1e3), 1),
           "panel_frames_per_s": round(len(ws) * F / (ms / 1e3), 1),
           "alg_gb_s": round((csr_map_bytes(info) + F * frame_bytes) / (ms / 1e3) / 1e9, 1),
           "staging": "fp32 pixel-major (the int32 panel); one run-kernel launch per 64 frames for all panels",
           "setup_s": {"maps_gpu": round(t_map, 2), "plan_build": round(t_plan, 2)}}
    sample = (ws, maps, [f[0].cpu().numpy() for f in frames], darks, ck[0].cpu().numpy().reshape(-1),
              aw[0].cpu().numpy())
    del frames
    plan.close()
    torch.cuda.empty_cache()
    return out, sample


def panel_accuracy(sample):
    """Frame 0 of the merged cake against the FP64 oracle: each panel's raw sums and areas,
    added, then divided."""
    import numpy as np
    import oracle
    ws, maps, frames, darks, got_ck, got_aw = sample
    n_r, n_eta = ws[0].n_r, ws[0].n_eta
    nb = n_r * n_eta
    raw, area, area_in = np.zeros(nb), np.zeros(nb), np.zeros(nb)
    for w, pm, fr, dk in zip(ws, maps, frames, darks):
        m = w.mapper
        sub = (fr.astype(np.float32) - dk).astype(np.float64)
        s, a = oracle.integrate(pm.pxList, pm.nmap_pairs(), nb, m.NrPixelsY, m.NrPixelsZ, sub, mode=w.mode,
                                normalize=False, bc_y=m.BC_y, bc_z=m.BC_z)
        raw += s
        area += a
        area_in += oracle.area_in(pm.pxList, pm.nmap_pairs(), nb, m.NrPixelsY, m.NrPixelsZ)
    cake = np.where(area > 1e-9, raw / np.where(area > 1e-9, area, 1.0), 0.0)
    ref_aw, _ = oracle.profile(cake, area_in, n_r, n_eta)
    r, ra = _rel(got_ck, cake), _rel(got_aw, ref_aw)
    return {"cake_max_rel": float(r.max()), "cake_mean_rel": float(r.mean()), "lineout_max_rel": float(ra.max()),
            "frames_checked": 1, "bins_from_two_or_more_panels": int(sum((pm.counts > 0).astype(int)
                                                                          for pm in maps).__ge__(2).sum())}


FIT_HALF_WINDOW = 60   # bins: +-15 px at RBin 0.25 px, 121 samples per window


def fit_bench(plan, frames, w, F, dev, reps=5):
    """Area-weighted lineouts of every resident frame, then every ring of every frame fitted
    in one launch of the batched LM fitter (kernel d), pseudo-Voigt and TCH.  Returns the
    timing / iteration summary and a sample of windows for the FP64 check of the CPU leg."""
    import numpy as np
    import torch

    from midas_b200 import peakfit, synth

    n = frames.shape[0]
    lo = torch.empty((n, w.n_r), dtype=torch.float64, device=dev)
    sm = torch.empty((F, w.n_r), dtype=torch.float64, device=dev)
    for s0 in range(0, n, F):
        k = min(F, n - s0)
        plan.integrate(frames[s0:s0 + k], cake=False, out={"lineout_aw": lo[s0:s0 + k], "lineout_sm": sm[:k]})
    x = torch.from_numpy(synth.r_centres(w)).to(dev)
    peaks = torch.from_numpy(synth.ring_peaks(w, FIT_HALF_WINDOW)).to(dev)
    stream = torch.cuda.current_stream()
    res, params = {}, {}
    for model in ("pv", "tch"):
        kw = dict(model=model, half_window=FIT_HALF_WINDOW, x_bin=w.mapper.RBinSize, max_iter=100,
                  px_um=w.mapper.px, lsd_um=w.mapper.Lsd)
        r = peakfit.fit_batch(x, lo, peaks, **kw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            r = peakfit.fit_batch(x, lo, peaks, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        it = r.iters.cpu().numpy().reshape(-1)
        edges = [0, 5, 10, 15, 20, 30, 50, 100, 101]
        hist = np.histogram(np.clip(it, 0, 100), bins=edges)[0]
        res[model] = {"fits_per_launch": int(it.size), "ms_per_launch": round(ms, 4),
                      "fits_per_s": round(it.size / (ms / 1e3), 1), "frames": int(n), "rings": int(peaks.numel()),
                      "window_samples": 2 * FIT_HALF_WINDOW + 1,
                      "iterations_hist": {f"{edges[i]}-{edges[i + 1] - 1}": int(hist[i]) for i in range(len(hist))},
                      "iterations_mean": round(float(it[it >= 0].mean()), 2)}
        params[model] = r.params[:16].cpu().numpy()
    sample = (synth.r_centres(w), lo[:16].cpu().numpy(), peaks.cpu().numpy(), w, params)
    return res, sample


def eta_fit_bench(cake, w, dev, reps=3):
    """Every ring in every eta column of one F-frame cake, in one launch of the fit-plan
    kernel: the per-eta pseudo-Voigt fits of the OpenMP integrator (singlets; SNR > 1
    kept)."""
    import numpy as np
    import torch

    from midas_b200 import synth
    from midas_b200.peakfit import FitPlan

    x = synth.r_centres(w)
    peaks = synth.ring_peaks(w, FIT_HALF_WINDOW)
    fp = FitPlan(x, peaks, kind="eta", half_window=FIT_HALF_WINDOW, x_bin=w.mapper.RBinSize, px_um=w.mapper.px,
                 lsd_um=w.mapper.Lsd, device=dev)
    r = fp.fit_cake_eta(cake)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        r = fp.fit_cake_eta(cake)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    it = r.iters.cpu().numpy()
    kept = int((r.params[..., 6] > 1.0).sum().item())
    fp.close()
    return {"frames": int(cake.shape[0]), "eta_bins": int(cake.shape[2]), "rings": int(len(peaks)),
            "windows_per_launch": int(it.size), "ms_per_launch": round(ms, 4),
            "fits_per_s": round(it.size / (ms / 1e3), 1), "fits_kept_snr_gt_1": kept,
            "iterations_mean": round(float(it[it >= 0].mean()), 2) if (it >= 0).any() else None}


def f_sweep(plan, frames, bufs, F_max, info, w, args, world, peak, steps=10):
    """Frames per launch F in {1, 8, 32, 128}: frames/s and the HBM roofline of one launch,
    A(F) = map bytes + F * frame bytes over the launch time (CUDA events, consecutive
    batches of the resident sweep, so no launch re-reads its frames from L2)."""
    import torch
    ny, nz = w.mapper.NrPixelsY, w.mapper.NrPixelsZ
    stream = torch.cuda.current_stream()
    out = {}
    n = frames.shape[0]
    for F in (1, 8, 32, 128):
        if F > F_max:
            continue
        ob = {k: v[:F] for k, v in bufs.items()}
        nb = n // F
        for i in range(3):
            plan.integrate(frames[(i % nb) * F:(i % nb + 1) * F], out=ob)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(steps):
            b = (3 + i) % nb
            plan.integrate(frames[b * F:(b + 1) * F], out=ob)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = dist_max(e0.elapsed_time(e1), world) / steps
        alg = csr_map_bytes(info) + F * ny * nz * 2
        out[str(F)] = {"frames_per_s": round(world * F / (ms / 1e3), 1), "ms_per_launch": round(ms, 4),
                       "roofline_frac": round(alg / (ms / 1e3) / 1e9 / peak, 4),
                       "alg_bytes_per_launch": alg}
    return out


def published_bench(args, dev, F=128, reps=10):
    """The reference's published benchmark configuration (PILATUS3 2M 1475x1679 u16, 172 um,
    Lsd 500 mm, beam centre at the detector centre, no tilt, RBin 1 px over 10..1117.4 px,
    eta 5 deg: packages/midas_integrate/tests/benchmarks/run_benchmarks.py:83-86, README
    'Performance') caked F frames per launch, on the device and end to end from host frames,
    beside the reference's H100 figures (C GPU stream ~1,600 frames/s; torch CSR FP32
    ~3,250 frames/s; packages/midas_integrate/README.md:75-80)."""
    import torch

    from midas_b200 import synth
    from midas_b200.kernels import CakePlan
    from midas_b200.mapper import build_map

    w = synth.pilatus3_2m_published()
    m = w.mapper
    ny, nz = m.NrPixelsY, m.NrPixelsZ
    pm, _ = build_map(m, device=dev.index)
    res = {"workload": w.name, "n_bins": w.n_r * w.n_eta, "mode": w.mode,
           "reference_h100_frames_per_s": {"c_gpu_stream": 1600, "torch_csr_fp32": 3250}}
    frames = w.frames(0, 4 * F, device=dev)
    stream = torch.cuda.current_stream()
    for enc in ("mma", "runs"):
        plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=ny, n_pixels_z=nz, mode=w.mode, bc_y=m.BC_y,
                        bc_z=m.BC_z, device=dev, encoding=enc)
        plan.set_dark(w.dark(device=dev).cpu().numpy())
        ob = {"cake": torch.empty((F, w.n_r, w.n_eta), dtype=torch.float32, device=dev),
              "lineout_aw": torch.empty((F, w.n_r), dtype=torch.float64, device=dev),
              "lineout_sm": torch.empty((F, w.n_r), dtype=torch.float64, device=dev)}
        for i in range(3):
            plan.integrate(frames[(i % 4) * F:(i % 4 + 1) * F], out=ob)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(reps):
            plan.integrate(frames[(i % 4) * F:(i % 4 + 1) * F], out=ob)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        r = {"frames_per_s": round(F / (ms / 1e3), 1), "ms_per_launch_of_128": round(ms, 4)}
        e2 = e2e_rate(plan, frames, F, argparse.Namespace(warmup=3, steps=reps), w, dev, 1)
        r["e2e_frames_per_s"] = e2["value"]
        r["e2e_h2d_bytes_per_step"] = e2["h2d_bytes_per_step"]
        res[enc] = r
        if enc == "mma":
            P = 16
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            plan.integrate_plain(frames[0])
            torch.cuda.synchronize()
            a.record(stream)
            for k in range(P):
                plan.integrate_plain(frames[k])
            b.record(stream)
            torch.cuda.synchronize()
            res["plain_frames_per_s"] = round(P / (a.elapsed_time(b) / 1e3), 1)
        plan.close()
    return res


def fit_accuracy(sample):
    """FP64 CPU fits (oracle twin of the device LM) of the first 16 frames' windows: largest
    centre and FWHM differences of the device fits, in px."""
    import numpy as np
    import oracle
    x, lo, peaks, w, params = sample
    out = {}
    for mi, model in enumerate(("pv", "tch")):
        got = params[model]
        dc, dfw = [], []
        for f in range(got.shape[0]):
            for k, c in enumerate(peaks):
                ref, _ = oracle.fit(x, lo[f], c, half_window=FIT_HALF_WINDOW, model=mi, max_iter=500,
                                    x_bin=w.mapper.RBinSize, px_um=w.mapper.px, lsd_um=w.mapper.Lsd)
                dc.append(abs(got[f, k, 1] - ref[1]))
                dfw.append(abs(got[f, k, 4] - ref[4]))
        out[model] = {"center_max_abs_err_px_vs_fp64": float(np.max(dc)),
                      "fwhm_max_abs_err_px_vs_fp64": float(np.max(dfw)), "windows_checked": len(dc)}
    return out


def e2e_rate(plan, frames, F, args, w, dev, world, with_cake=False):
    """Host (pinned) frames -> H2D of the referenced pixels (CakePlan.upload) -> batched
    caking -> D2H lineouts, double-buffered on two streams so the copy of batch i+1 overlaps
    the caking of batch i.  with_cake: the float32 cakes come back too (the reference's
    Write2D output), on a third stream from a double-buffered device cake."""
    import torch
    nz, ny = w.shape
    pool = min(frames.shape[0], 2 * F)
    host = torch.empty((pool, nz, ny), dtype=torch.uint16, pin_memory=True)
    host.copy_(frames[:pool].cpu())
    dbuf = [torch.empty((F, nz, ny), dtype=torch.uint16, device=dev) for _ in range(2)]
    cakes = [torch.empty((F, w.n_r, w.n_eta), dtype=torch.float32, device=dev) for _ in range(2 if with_cake else 1)]
    h_cake = [torch.empty((F, w.n_r, w.n_eta), dtype=torch.float32, pin_memory=True) for _ in range(2)] \
        if with_cake else None
    aw = torch.empty((F, w.n_r), dtype=torch.float64, device=dev)
    sm = torch.empty((F, w.n_r), dtype=torch.float64, device=dev)
    h_aw = torch.empty((2, F, w.n_r), dtype=torch.float64, pin_memory=True)
    h_sm = torch.empty((2, F, w.n_r), dtype=torch.float64, pin_memory=True)
    cs, ks, ds = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    copied = [torch.cuda.Event() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    caked = [torch.cuda.Event() for _ in range(2)]
    back = [torch.cuda.Event() for _ in range(2)]
    nb = pool // F

    def run(n):
        for i in range(n):
            s = i % 2
            cake = cakes[s % len(cakes)]
            with torch.cuda.stream(cs):
                cs.wait_event(done[s])
                plan.upload(host[(i % nb) * F:(i % nb + 1) * F], dbuf[s], stream=cs)
                copied[s].record(cs)
            with torch.cuda.stream(ks):
                ks.wait_event(copied[s])
                if with_cake:
                    ks.wait_event(back[s])              # the cake buffer's previous copy is out
                plan.integrate(dbuf[s], out={"cake": cake, "lineout_aw": aw, "lineout_sm": sm}, stream=ks)
                h_aw[s].copy_(aw, non_blocking=True)
                h_sm[s].copy_(sm, non_blocking=True)
                done[s].record(ks)
                caked[s].record(ks)
            if with_cake:
                with torch.cuda.stream(ds):
                    ds.wait_event(caked[s])
                    h_cake[s].copy_(cake, non_blocking=True)
                    back[s].record(ds)
        torch.cuda.synchronize()

    run(max(2, args.warmup))
    barrier(world)
    t0 = time.perf_counter()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(cs)
    run(args.steps)
    b.record(ds if with_cake else ks)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    dev_ms = dist_max(a.elapsed_time(b), world)
    rate = world * args.steps * F / (dev_ms / 1e3)
    info = plan.info
    up = info["upload_pixels"]
    return {"value": round(rate, 1), "unit": UNIT, "h2d_bytes_per_step": F * up * 2,
            "d2h_bytes_per_step": 2 * F * w.n_r * 8 + (F * w.n_r * w.n_eta * 4 if with_cake else 0),
            "wall_s": round(wall, 3),
            "pipeline": ("3 streams (cakes back on the third)" if with_cake else "2 streams")
                        + ", double-buffered H2D of the referenced columns of each 16-row "
                        f"group of the referenced band ({info['ref_row_hi'] - info['ref_row_lo']} of {nz} "
                        f"rows, {up} of {nz * ny} pixels per frame)"}


# ---------------------------------------------------------------------------
def main_reference(args):
    """The reference's own CPU integrator (integration_apply_map from the MIDAS sources,
    oracle/_ref) on this host's cores, same workload, metric and unit."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np

    import oracle
    from midas_b200 import synth
    w = synth.WORKLOADS[args.workload]()
    m = w.mapper
    ny, nz = m.NrPixelsY, m.NrPixelsZ
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (MIDAS C sources absent)"}))
        return
    r_lo, r_hi, e_lo, e_hi = m.edges()
    t0 = time.time()
    recs, nmap, _ = oracle.ref_build_map(ny=ny, nz=nz, px=m.px, lsd=m.Lsd, bc_y=m.BC_y, bc_z=m.BC_z, tx=m.tx,
                                         ty=m.ty, tz=m.tz, rho_d=m.RhoD, p=np.array(m.p, np.float64),
                                         parallax=m.Parallax, solid_angle=m.SolidAngleCorrection,
                                         polarization=m.PolarizationCorrection,
                                         pol_fraction=m.PolarizationFraction, r_lo=r_lo, r_hi=r_hi,
                                         eta_lo=e_lo, eta_hi=e_hi)
    t_map = time.time() - t0
    rng = np.random.default_rng(w.seed)
    yy, zz = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nz, dtype=np.float64))
    R = np.hypot(yy - m.BC_y, zz - m.BC_z)
    eta = np.arctan2(-(yy - m.BC_y), zz - m.BC_z)
    tex = 1 + w.texture * np.cos(2 * eta)
    mu = np.full((nz, ny), w.background)
    for rr, aa in zip(w.ring_radii(), w.ring_amps()):
        u2 = ((R - rr) / (w.fwhm_px / 2)) ** 2
        mu += aa * tex * (w.mix_eta / (1 + u2) + (1 - w.mix_eta) * np.exp(-np.log(2) * u2))
    dark = w.dark_mean + w.dark_sigma * rng.standard_normal((nz, ny))
    frames = [np.clip(rng.poisson(mu) + np.rint(dark), 0, 65535).astype(np.float64) for _ in range(2)]
    cores = oracle.ref().ref_max_threads()
    grad = 1 if w.mode == "gradient" else 0

    def step(i):
        oracle.ref_integrate(recs, nmap, w.n_r, w.n_eta, frames[i % 2], ny, nz, dark=dark, bc_y=m.BC_y,
                             bc_z=m.BC_z, gradient=grad, n_threads=cores)

    for i in range(args.warmup):
        step(i)
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(i)
    el = time.perf_counter() - t0
    fps = args.steps / el
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": round(fps, 3), "unit": UNIT,
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": round(el / args.steps * 1e3, 3), "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": w.name, "frames_per_step": 1, "mode": w.mode,
                                 "map_records": int(recs.shape[0]), "map_build_s": round(t_map, 1)},
                      "cpu_baseline": {"value": round(fps, 3), "unit": UNIT, "cores": cores, "kind": "reference",
                                       "sample": f"{args.steps} full frames, integration_apply_map over "
                                                 f"8-row chunks with OpenMP"},
                      "e2e": {"value": round(fps, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        main_reference(args)
    else:
        main_ours(args)


if __name__ == "__main__":
    main()
