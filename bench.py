#!/usr/bin/env python
"""Benchmark: stack MP-frames/s (align + fuse + depth) on seeded synthetic stacks.

One step = the whole stacking path over one stack: registration of every
frame to the previous aligned one (Nelder-Mead on the device cost), the
brightness gains, the level-by-level fold over all frames, the residual
rule and collapse, and the depth pass (guided-filter aggregation, peaks,
median, WLS, upsampling). `value` times steps whose 16-bit frames are
already in HBM; `e2e` times the public API (Stack.push_u16 from pinned host
memory, Stack.finish reading the results back) per step.

Workloads (seeded synthetic stacks with the shapes of the reference's
published runs: a height field, band-limited texture, per-pixel defocus):
  c3  100 x 8256x5504 RGB u16, per-frame similarity warps, alignment at
      coarsen 3, 7 levels, 16-bit (UNORM16) pyramid storage   [default]
  c2  30 x 6000x4000, no alignment, 8 levels, aggregation radius 8, FP32
  c1  8 x 1024x768, no alignment, 6 levels, FP32
  c3s 16 x 2048x1536 with c3's settings: the small case the ncu captures use
  c3m 32 x 4096x2752, c3's depth settings without alignment: the capture case whose focus slices
      exceed L2 (about 3 GB on the device)

--impl reference times the CPU restatement of the reference's path (the
oracle; the Rust reference cannot be built here) on the same workload with
all host threads: per-frame work timed frame by frame over a sample of the
stack's frames, the finish (depth pass over all N slices on the full grid)
timed once, extrapolated to the whole stack; plus a 1-core per-frame figure.
It loads no part of the CUDA library (the frames come from the oracle's twin
of the generator).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "stack MP-frames/s (align+fuse+depth)"
UNIT = "MP-frames/s"
# the reference's published CUDA run of 100 x 45.7 MP frames (RTX 3060), 26 s wall
PUBLISHED_MPFS = 175.8

CONFIGS = {
    "c3": dict(w=8256, h=5504, n=100, warp=True, mag_step=0.0, noise_std=0.002, levels=0, align=True, coarsen=3,
               agg_radius=3, storage="unorm16", wls_report=True),
    "c2": dict(w=6000, h=4000, n=30, warp=False, mag_step=0.001, noise_std=0.002, levels=8, align=False, coarsen=0,
               agg_radius=8, storage="f32"),
    "c1": dict(w=1024, h=768, n=8, warp=False, mag_step=0.002, noise_std=0.003, levels=6, align=False, coarsen=0,
               agg_radius=3, storage="f32"),
    # c3's path at sizes an ncu capture finishes quickly: frames larger than L2 (c3s), and focus
    # slices larger than L2 too (c3m)
    "c3m": dict(w=4096, h=2752, n=32, warp=False, mag_step=0.002, noise_std=0.002, levels=0, align=False, coarsen=0,
                agg_radius=3, storage="unorm16"),
    "c3s": dict(w=2048, h=1536, n=16, warp=True, mag_step=0.0, noise_std=0.002, levels=0, align=True, coarsen=3,
                agg_radius=3, storage="unorm16"),
}


# Several stacks of uneven sizes and frame counts (12, 24 and 45 MP; 8 to 24 frames), aligned,
# 16-bit storage, depth on: run one after another on the whole GPU, then side by side on engines
# that each take a share of the SMs (lsb_batch_run). Not the headline: its own JSON line.
BATCH = [(4240, 2832, 16), (6000, 4000, 12), (8256, 5504, 8), (4240, 2832, 24), (6000, 4000, 20), (8256, 5504, 12),
         (4240, 2832, 10), (6000, 4000, 8)]


def params_of(cfg, mod):
    fuse = mod.FuseParams(levels=cfg["levels"])
    align = mod.AlignParams(coarsen=cfg["coarsen"]) if cfg["align"] else None
    depth = mod.DepthParams(agg_radius=cfg["agg_radius"])
    return fuse, align, depth


def workload_name(c, name):
    return (f"{name}: {c['n']} x {c['w']}x{c['h']} RGB u16 seeded synthetic focus stack"
            f"{', per-frame similarity warps, alignment coarsen ' + str(c['coarsen']) if c['align'] else ', no alignment'}, "
            f"{'auto' if not c['levels'] else c['levels']} levels, guided-filter DfF r={c['agg_radius']}, WLS MG-PCG, "
            f"{c['storage']} pyramid storage")


def spec_of(c, n=None, seed=0x1A957ACC):
    import lapstack_b200 as L
    return L.SynthSpec(c["w"], c["h"], n or c["n"], seed=seed, mag_step=c["mag_step"], noise_std=c["noise_std"],
                       warp=c["warp"])


# ------------------------------------------------------------------ clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.p, self.path = index, None, f"/tmp/lsb_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------- reference
class OracleStackTimer:
    """The oracle (the C++ restatement of the reference's CPU path, OpenMP) on a sample of the workload's
    frames, made by the oracle's twin of the seeded generator (no CUDA library is loaded).

    push(): one frame's per-frame work, timed alone -- its registration to the previous frame, warp,
    brightness gain, fold into the pyramid selection and focus slice (stack.rs:785-821). When the sample
    wraps, a new stack starts and its first frame is pushed untimed, so every timed push registers.
    finish(n): the stack's finish, timed once -- shares, residual and collapse, the depth pass over n
    focus slices (the sample's slices in order, repeated) on the full working grid, the WLS solves, the
    upsampling and the crop (stack.rs:833-853, 1047-1060)."""

    def __init__(self, c, sample, w=None, h=None, seed=0x1A957ACC):
        from oracle import oracle as O
        self.O, self.c, self.sample = O, c, sample
        self.w, self.h = w or c["w"], h or c["h"]
        self.frames, _ = O.synth_stack(self.w, self.h, c["n"], seed=seed, mag_step=c["mag_step"], noise_std=c["noise_std"],
                                       warp=c["warp"], frames=(0, sample))
        fuse, align, depth = params_of(c, O)
        self.sp = O.StackParams(fuse=fuse, align=align, depth=depth)
        self.run, self.j = None, 0

    def push(self):
        if self.run is None or self.j == self.sample:
            self.run = self.O.StackRun(self.c["n"], self.w, self.h, self.sp)
            self.run.push(self.frames[0], last=False)
            self.j = 1
        t0 = time.perf_counter()
        self.run.push(self.frames[self.j], last=False)
        self.j += 1
        return time.perf_counter() - t0

    def finish(self, n_total):
        self.run.cycle_slices(n_total)
        t0 = time.perf_counter()
        self.run.finish()
        self.run = None
        return time.perf_counter() - t0


def repo_libs():
    """The repository's shared libraries this process has mapped (what ran)."""
    try:
        maps = open("/proc/self/maps").read().split("\n")
    except Exception:
        return None
    return sorted({os.path.relpath(l.split()[-1], ROOT) for l in maps if l.strip().endswith(".so") and ROOT in l})


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count()


def cpu_baseline(c):
    """A bounded sample of the workload on the oracle (about 30 s of CPU): frames at a quarter of the
    frame area from the same generator, two timed pushes and the finish over the workload's N slices on
    the quarter-area grid, both scaled by the area ratio (the per-frame work, the depth pass and the WLS
    solve grow with the pixel count). The reference arm (--impl reference) measures the full frame size."""
    from oracle import oracle as O
    threads = O.set_threads(0)
    w, h = (c["w"] + 1) // 2, (c["h"] + 1) // 2
    area = c["w"] * c["h"] / (w * h)
    tm = OracleStackTimer(c, 3, w, h)
    pushes = [tm.push() for _ in range(2)]
    fin = tm.finish(c["n"])
    per_frame, finish = statistics.mean(pushes) * area, fin * area
    step = per_frame + finish / c["n"]
    return {"value": c["w"] * c["h"] / 1e6 / step, "unit": UNIT, "cores": threads, "nproc": host_cores(), "kind": "port",
            "extrapolated": True, "per_frame_s": per_frame, "finish_s": finish,
            "sample": (f"the oracle (C++ restatement of the reference's CPU path, OpenMP on {threads} threads): frames at a "
                       f"quarter of the area ({w}x{h}, same generator and settings), 2 registered frames pushed "
                       f"({statistics.mean(pushes):.2f} s each) and the finish with the depth pass over {c['n']} slices "
                       f"({fin:.1f} s), scaled by the area ratio {area:.2f}; MP-frames/s = N*W*H/(N*per_frame + finish)")}


def reference_arm(args, c, name):
    """The reference's CPU path (the oracle: the Rust reference cannot be built here) on this workload,
    rank 0 only: each step is one frame's per-frame work (OracleStackTimer.push) on a sample of the
    workload's first frames (at least 8 timed ones before the sample repeats); after the steps the stack's
    finish, with the depth pass over all N slices on the full grid, is timed once and spread over the N
    frames. ms_per_step = per-frame time + finish / N, so the value is the whole stack's extrapolated
    MP-frames/s. One more push on a single thread gives the 1-core per-frame figure."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    threads = O.set_threads(0)
    N, W, H = c["n"], c["w"], c["h"]
    sample = min(N, 9)
    tm = OracleStackTimer(c, sample)
    t_begin = time.perf_counter()
    for _ in range(args.warmup):
        tm.push()
    pushes = [tm.push() for _ in range(args.steps)]
    one_core = None
    if tm.sample > 1:
        O.set_threads(1)
        try:
            one_core = tm.push()
        finally:
            O.set_threads(0)
    fin = tm.finish(N)
    per_frame = statistics.mean(pushes)
    step = per_frame + fin / N
    v = W * H / 1e6 / step
    world = int(os.environ.get("WORLD_SIZE", "1"))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": v / PUBLISHED_MPFS,
            "dtype": "f32", "data": "synthetic (seeded generator: height field, band-limited texture, per-pixel defocus)",
            "impl": "reference", "config": bench_config(c, name, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "nproc": host_cores(), "kind": "port",
                             "extrapolated": True, "per_frame_s": per_frame, "finish_s": fin,
                             "one_core": ({"per_frame_s": one_core, "per_frame_mpfs": W * H / 1e6 / one_core}
                                          if one_core else None),
                             "sample": (f"the oracle (C++ restatement of the reference's CPU path; the Rust reference "
                                        f"cannot be built here) on {threads} threads: {args.steps} frames of the workload "
                                        f"pushed one per step (registration, warp, gains, fold, focus slice; the first "
                                        f"{sample} frames of the stack, repeated), then the finish with the depth pass over "
                                        f"all {N} slices on the full grid ({fin:.1f} s), spread over the {N} frames; the "
                                        f"whole run took {time.perf_counter() - t_begin:.0f} s")},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "native_so": repo_libs()}
    print(json.dumps(line), flush=True)
    return 0


def bench_config(c, name, world):
    """The workload as both arms name it."""
    return {"workload": workload_name(c, name), "global_batch": c["n"] * world, "parallelism": f"replicas x{world}",
            "l2": "inputs (frames) larger than L2 every step"}


# ------------------------------------------------------------------- ours
def traffic_per_px_frame(name):
    """DRAM bytes per pixel-frame of the fused level-0 fold kernel from its committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"fold0_kernel_{name}.md")
    try:
        for line in open(p):
            if line.startswith("TRAFFIC_BYTES_PER_PIXEL_FRAME"):
                return float(line.split("=")[1])
    except Exception:
        return None
    return None


def _device_plane(ptr, h, w):
    """A float32 device plane as a torch tensor (no copy)."""
    import torch

    class _Cuda:
        def __init__(self):
            self.__cuda_array_interface__ = {"data": (ptr, False), "shape": (h, w), "typestr": "<f4", "version": 3}
    return torch.as_tensor(_Cuda(), device="cuda")


def wls_report(L, eng, st, c):
    """WLS ms to rel-res 1e-5 on this stack's depth grid: the reference's FP32
    MG-PCG against the BF16 V-cycle, with the reference's edge weights and with
    the large-grid Gaussian ones (lambda 0.5, sigma 0.02); and this stack's
    solves started from the trained U-Net against the reference's FGS start."""
    import torch
    from lapstack_b200 import unet as U
    (g, d, cf, _), (dw, dh) = st.depth_planes()
    torch.cuda.synchronize()
    d_h, cf_h, g_h = (_device_plane(p, dh, dw).cpu().numpy() for p in (d, cf, g))
    out = {"grid": [dw, dh]}
    for name, (em, lam, sg) in {"reference_edges": (0, 3.0, 0.04), "gaussian_edges": (1, 0.5, 0.02)}.items():
        row = {}
        for mode, tag in ((0, "fp32_vcycle"), (1, "bf16_vcycle")):
            L.wls_solve(d_h, cf_h, g_h, lam, sg, 200, edge_mode=em, vcycle_mode=mode, engine=eng)  # warm
            _, rel, it, ms = L.wls_solve(d_h, cf_h, g_h, lam, sg, 200, edge_mode=em, vcycle_mode=mode, engine=eng)
            row[tag] = {"ms": ms, "iters": it, "rel": rel}
        out[name] = row
    # the scale-0 grid (one unknown per frame pixel): the depth planes brought to the frame's size
    # (nearest), the fused image's luma as the guide, the Gaussian edge weights (lambda 0.5, sigma 0.02)
    o = st.finish()
    luma = np.ascontiguousarray(np.float32(0.2126) * o.image[0] + np.float32(0.7152) * o.image[1] + np.float32(0.0722) * o.image[2])
    del o
    H0, W0 = luma.shape
    up = lambda p: np.ascontiguousarray(np.repeat(np.repeat(p, 2, 0), 2, 1)[:H0, :W0])
    d0, c0 = up(d_h), up(cf_h)
    row = {"grid": [W0, H0]}
    for mode, tag in ((0, "fp32_vcycle"), (1, "bf16_vcycle")):
        L.wls_solve(d0, c0, luma, 0.5, 0.02, 200, edge_mode=1, vcycle_mode=mode, engine=eng)  # warm
        _, rel, it, ms = L.wls_solve(d0, c0, luma, 0.5, 0.02, 200, edge_mode=1, vcycle_mode=mode, engine=eng)
        row[tag] = {"ms": ms, "iters": it, "rel": rel}
    out["scale0_gaussian_edges"] = row
    del d0, c0, luma
    # learned warm start: trained on solver pairs of this resolution, then this stack's own solves
    t0 = time.perf_counter()
    inp, d_in, tgt, _ = U.solver_pairs(6, c["w"], c["h"], frames=(8, 12), engine=eng,
                                      depth=L.DepthParams(agg_radius=c["agg_radius"]))
    net = U.UNet(seed=0)
    losses = U.train(net, inp, d_in, tgt, steps=300, batch=8, crop=256, lr=1e-3)
    train_s = time.perf_counter() - t0
    del inp, d_in, tgt
    # the network's forward pass on this stack's grid: tensor-core FLOPs against the measured bf16 peak
    Hn, Wn = U.grid_of(dw, dh)
    t_in = torch.zeros((1, Hn, Wn, U.CH), dtype=torch.bfloat16, device="cuda")
    t_d = torch.zeros((1, Hn, Wn), dtype=torch.float32, device="cuda")
    net.forward(t_in, t_d)
    reps = 5
    times = []
    for _ in range(reps):
        net.forward(t_in, t_d)
        times.append(net.forward_ms())
    fwd_ms = statistics.median(times)
    flops = U.forward_flops(Hn, Wn)
    pk, pk_kind = peaks()
    out["unet_forward"] = {"grid": [Wn, Hn], "ms": fwd_ms, "tflops": flops / (fwd_ms / 1e3) / 1e12,
                           "frac": flops / (fwd_ms / 1e3) / 1e12 / pk["bf16_tflops"], "peak_tflops": pk["bf16_tflops"],
                           "peak_kind": pk_kind, "timing": "CUDA events around the layers on the network's stream, median of 5"}
    del t_in, t_d
    res = {}
    for mode in ("plain", "learned", "plain", "learned"):
        st.set_warm_start(net if mode == "learned" else None)
        o = st.finish()
        res[mode] = {"ms": o.ms["wls_solve"], "iters": [o.depth.wls_iters_first, o.depth.wls_iters], "rel": o.depth.wls_rel64}
    st.set_warm_start(None)
    out["learned_vs_plain"] = {"plain": res["plain"], "learned": res["learned"],
                               "speedup": res["plain"]["ms"] / max(res["learned"]["ms"], 1e-9),
                               "train": {"stacks": 6, "steps": 300, "seconds": train_s,
                                         "loss_first": float(np.mean(losses[:10])), "loss_last": float(np.mean(losses[-10:]))}}
    net.close()
    return out


# ------------------------------------------------------------- replicas
def replica_seed(rank):
    """Each rank's stack: the same workload with its own seed (independent replicas)."""
    return 0x1A957ACC ^ rank


def max_over_ranks(x, dist=None, device="cpu"):
    """The slowest rank's time (multi-GPU numbers are the max over ranks)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, mp_per_rank_step, ms_max):
    """Whole-job MP-frames/s: every rank's pixel-frames over the slowest rank's step time."""
    return world * mp_per_rank_step / (ms_max / 1e3)


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--storage", default=None, choices=["f32", "unorm16", "f16"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-wls-report", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--two-kernel-fold0", action="store_true", help="fold level 0 with the separate REDUCE and select kernels")
    ap.add_argument("--fold-beside-chain", action="store_true", help="fold device-resident frames beside the registration chain")
    ap.add_argument("--batch", action="store_true", help="time the uneven batch of stacks instead (its own JSON line)")
    ap.add_argument("--engines", type=int, default=2, help="engines the batch runs on side by side")
    args = ap.parse_args()
    if args.batch:
        return batch_bench(args)
    c = dict(CONFIGS[args.config])
    if args.storage:
        c["storage"] = args.storage
    if args.impl == "reference":
        return reference_arm(args, c, args.config)

    import torch
    import lapstack_b200 as L

    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist:
            dist.barrier()

    def max_ranks(x):
        return max_over_ranks(x, dist, "cuda")

    eng = L.Engine(device=local, storage=c["storage"], fused_fold0=not args.two_kernel_fold0,
                   fold_beside_chain=args.fold_beside_chain)
    fuse, align, depth = params_of(c, L)
    W, H, N = c["w"], c["h"], c["n"]
    st = eng.stack(W, H, N, fuse, align, depth)
    # independent stacks per rank (replicas): each its own seed
    L.synth_stack_device(spec_of(c, seed=replica_seed(rank)), st.frames_device(), eng.stream)
    st.set_count(N)
    stream = torch.cuda.ExternalStream(eng.stream)

    for _ in range(args.warmup):
        st.run()
    tune = st.autotune() if not args.no_autotune else None  # untimed: picks the persistent grids
    l0 = L.load().lsb_launch_count()
    stages = []
    barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            stages.append(st.run())
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    launches = L.load().lsb_launch_count() - l0
    ms = max_ranks(e0.elapsed_time(e1) / args.steps)
    mp_step = N * W * H / 1e6
    value = job_throughput(world, mp_step, ms)
    fold0 = statistics.mean(s["fold_level0"] for s in stages)  # the fused kernel + the border tiles' launches
    fused0 = statistics.mean(s["reduce_level0"] for s in stages)  # the fused kernel alone
    stage_ms = {k: statistics.mean(s[k] for s in stages) for k in stages[0]}

    # ---- end to end through the public API: pinned host frames in, results out
    host = torch.empty((N, H, W, 3), dtype=torch.int16, pin_memory=True)
    host.copy_(_frames_tensor(st, N, H, W))
    hnp = host.numpy().view(np.uint16)
    e2e_ms = []
    for it in range(1 + max(1, args.e2e_steps)):  # the first pass warms the host result buffers, untimed
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st.set_count(0)
        for k in range(N):
            st.push_u16(hnp[k])
        out = st.finish()
        torch.cuda.synchronize()
        t = max_ranks((time.perf_counter() - t0) * 1e3)
        if it > 0:
            e2e_ms.append(t)
        has_depth = out.depth is not None
        m = out.depth.dw * out.depth.dh if has_depth else 0
        align_evals = out.align_evals
        depth_iters = (out.depth.wls_iters, out.depth.wls_rel) if has_depth else (0, 0.0)
        del out  # a caller done with a result hands its buffers back
    e2e_t = statistics.median(e2e_ms)
    h2d = N * W * H * 6
    d2h = W * H * (6 + 12 + 4) + (W * H * 8 + m * 4 if has_depth else 0)

    wls = None
    if rank == 0 and c.get("wls_report") and not args.no_wls_report:
        try:
            wls = wls_report(L, eng, st, c)
        except Exception as ex:  # reported, never the product
            wls = {"error": str(ex)}
    if rank == 0:
        pk, pk_kind = peaks()
        gs = {"f32": 4, "unorm16": 2, "f16": 2}[c["storage"]]
        ss = 2 if gs == 2 else 4  # focus slices: FP16 with 16-bit storage
        # the level-0 fold (fold0_kernel on the interior tiles, the REDUCE and select kernels on the
        # border tiles): every frame's level-0 pixels (u16 RGB) read once; G_1 (3 planes in the storage
        # type, a quarter of the pixels) and the focus slice (a quarter of the pixels) written once; the
        # level's accumulator (3 x f32) and best energy (f32) written once
        alg_bytes = N * W * H * (6 + 3 * gs / 4 + ss / 4) + W * H * 16
        achieved = alg_bytes / (fold0 / 1e3) / 1e9
        tr = traffic_per_px_frame(args.config)
        cb = None
        if not args.no_cpu_baseline:
            try:
                cb = cpu_baseline(c)
            except Exception as ex:  # the baseline is reported, never the product
                cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": value / PUBLISHED_MPFS,
            "dtype": "f32", "data": "synthetic (seeded generator: height field, band-limited texture, per-pixel defocus)",
            "config": bench_config(c, args.config, world),
            "autotune": ({"grid_select": tune["grid_select"], "grid_aggregate": tune["grid_aggregate"]} if tune else None),
            "e2e": {"value": job_throughput(world, mp_step, e2e_t), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_t},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "level-0 fold (fold0_kernel + the border tiles' two kernels)",
                         "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                         "peak_kind": pk_kind, "traffic": (tr * N * W * H if tr else None), "algorithmic_bytes": alg_bytes,
                         "kernel_ms": fold0, "fused_kernel_ms": fused0},
            "stages_ms": stage_ms,
            "align_evals": align_evals,
            "wls": {"iters": depth_iters[0], "rel": depth_iters[1],
                    "ms_to_rel_1e-5": wls},
            "cpu_baseline": cb,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    st.close()
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


def batch_bench(args):
    """The uneven batch: each stack alone on an engine with the whole GPU (the sum of their times),
    then the batch on `--engines` engines with an equal share of the SMs each, side by side
    (lsb_batch_run). Frames are generated in each stack's frame store on the device; a run is
    lsb_stack_finish (results copied to the host). Wall clock around device-synchronised runs."""
    import torch
    import lapstack_b200 as L

    torch.cuda.set_device(0)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    fuse, align, depth = L.FuseParams(), L.AlignParams(coarsen=3), L.DepthParams()

    def stacks_on(engines):
        out = []
        for i, (w, h, n) in enumerate(BATCH):
            e = engines[i % len(engines)]
            st = e.stack(w, h, n, fuse, align, depth)
            L.synth_stack_device(L.SynthSpec(w, h, n, seed=0xBA7C + i, warp=True, mag_step=0.0, noise_std=0.002),
                                 st.frames_device(), e.stream)
            st.set_count(n)
            out.append(st)
        torch.cuda.synchronize()
        return out

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3, r

    whole = L.Engine(storage="unorm16")
    stacks = stacks_on([whole])
    single = []
    for st in stacks:
        for it in range(1 + max(1, args.steps)):
            ms, out = timed(st.finish)
            del out
            if it > 0:
                single.append((st.w, st.h, st.n, ms))
    per_stack = [statistics.median(m for (w, h, n, m) in single if (w, h, n) == key) for key in BATCH]
    for st in stacks:
        st.close()
    whole.close()

    k = max(1, args.engines)
    engines = [L.Engine(storage="unorm16", grid_limit=max(1, 2 * sms // k)) for _ in range(k)]
    stacks = stacks_on(engines)
    batch = []
    for it in range(max(1, args.warmup) + max(1, args.steps)):
        ms, outs = timed(lambda: L.batch_run(stacks))
        del outs
        if it >= max(1, args.warmup):
            batch.append(ms)
    for st in stacks:
        st.close()
    for e in engines:
        e.close()
    mpf = sum(w * h * n for (w, h, n) in BATCH) / 1e6
    b = statistics.median(batch)
    print(json.dumps({
        "metric": "uneven batch of stacks MP-frames/s (align+fuse+depth)", "value": mpf / (b / 1e3), "unit": "MP-frames/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_batch": b, "higher_is_better": True,
        "dtype": "f32", "data": "synthetic (seeded generator, frames generated on the device)",
        "config": {"workload": "batch: " + ", ".join(f"{n} x {w}x{h}" for (w, h, n) in BATCH) +
                   "; aligned (coarsen 3), unorm16 storage, guided-filter DfF r=3, WLS MG-PCG", "engines": k,
                   "grid_limit": max(1, 2 * sms // k)},
        "sum_single_ms": sum(per_stack), "single_ms": per_stack, "batch_ms": batch,
        "speedup_vs_one_after_another": sum(per_stack) / b, "timing": "wall clock around device-synchronised runs",
    }))
    return 0


def _frames_tensor(st, n, h, w):
    """The stack's device frame store as a torch tensor (no copy)."""
    import torch

    class _Cuda:
        def __init__(self, ptr, shape):
            self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": "<i2", "version": 3}
    return torch.as_tensor(_Cuda(st.frames_device(), (n, h, w, 3)), device="cuda")


if __name__ == "__main__":
    sys.exit(main())
