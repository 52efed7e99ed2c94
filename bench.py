#!/usr/bin/env python
"""BIMP keypoint extraction benchmark on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (N=1 headline): one 1920x1080 uint8 synthetic image per step, 8
scales (lambda = 4*2^(k/2), float-accumulated) x 8 orientations, FP32 maps,
keypoints out.  Metric: Mpixel/s of full-resolution input pixels.

* ``value``   device-resident inputs (a 64-image pool in HBM, 133 MB > L2),
              detection through the C ABI (bimp_detect_device_async), timed
              with CUDA events over K steps, max over ranks;
* ``e2e``     the same metric through bimp_detect_host: pinned host image in,
              host keypoint records out, copies inside the timed region;
* ``roofline`` the dominant kernel (tiled-FFT Gabor filtering) timed alone
              with CUDA events, algorithmic bytes per launch / duration;
* ``batched`` 64 mixed-size images (<= 1080p) in one CUDA-graph replay vs
              the same images detected one by one;
* ``cpu_baseline`` the FP64 oracle on one 1080p image (rank 0, N=1).

``--impl reference`` times the reference pipeline's CPU restatement (the
oracle port; the reference itself cannot be built here) on this host's cores
and prints the same metric with "impl": "reference".

Multi-GPU (torchrun): one process per GPU, each detecting its own images
(replicas; the path has no exchange step), value = all pixels / max time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "cuda-bimp_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402

METRIC = "Mpixel/s at 1080p, 8 scales x 8 orients, batched vs plain; bwd/fwd time ratio"
UNIT = "Mpixel/s"
W_HD, H_HD = 1920, 1080
POOL = 64


def hd_pool(rank: int, n: int = POOL):
    """n distinct 1080p images: 4 seeded base images x flips and circular shifts."""
    from bimp_b200 import synth
    bases = [synth.synth_image(W_HD, H_HD, 150, seed=1001 + 17 * rank + k) for k in range(4)]
    rng = np.random.default_rng(77 + rank)
    out = []
    for i in range(n):
        b = bases[i % 4]
        if (i // 4) % 2:
            b = b[:, ::-1]
        if (i // 8) % 2:
            b = b[::-1, :]
        dy, dx = int(rng.integers(0, H_HD)), int(rng.integers(0, W_HD))
        out.append(np.ascontiguousarray(np.roll(b, (dy, dx), axis=(0, 1))))
    return out


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.15)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# multi-process plumbing (replicas: no collective on the data path)
# ---------------------------------------------------------------------------
def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a per-rank timing over all ranks (all_reduce MAX); identity at N=1."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(pixels_per_step: int, steps: int, world: int, max_ms: float) -> float:
    """Whole-job Mpixel/s: every rank processed `steps` images of `pixels_per_step`."""
    return world * steps * pixels_per_step / (max_ms * 1e-3) / 1e6


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def algorithmic_bytes(cs) -> dict:
    """Algorithmic bytes of one detection, per kernel (per-pixel figures of
    the path applied to every scale's dataW x dataH map)."""
    gabor = stencil = nms = 0
    for k in cs.ks:
        n = k["data_w"] * k["data_h"]
        gabor += n * (1 + 8 * 4)          # uint8 level read + 8 fp32 magnitude maps written
        stencil += n * (8 * 4 + 2 * 4)    # 8 magnitude maps read + D and S written
        nms += n * 4                      # D read once
    return {"gabor": gabor, "stencil": stencil, "nms": nms}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profiled_traffic():
    """dram bytes per launch of the Gabor kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "gabor_tiles_hd.md"
    if not f.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch\s*=\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist
    from bimp_b200 import _lib as L
    from bimp_b200 import api, synth

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(int(stream.cuda_stream))
    lam = synth.bank(8)

    pool_np = hd_pool(rank)
    pool = [torch.from_numpy(im).to(dev) for im in pool_np]
    cs = api.CudaStuff(W_HD, H_HD, lam)
    cap = 131072
    kp = torch.zeros((7, cap), dtype=torch.float32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    lib = L.lib()

    def detect(img):
        rc = lib.bimp_detect_device_async(cs.handle, C.c_void_p(img.data_ptr()), img.stride(0), W_HD, H_HD,
                                          C.c_void_p(kp.data_ptr()), kp.stride(0), cap,
                                          C.c_void_p(cnt.data_ptr()), sp)
        if rc != 0:
            L.check(rc, "bimp_detect_device_async")

    def barrier():
        if world > 1:
            dist.barrier()

    def max_ms(x: float) -> float:
        return max_over_ranks(x, world, dev)

    for i in range(args.warmup):
        detect(pool[i % POOL])
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    if rank == 0:
        clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        detect(pool[i % POOL])
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_local = e0.elapsed_time(e1)
    clk = clocks.stop() if rank == 0 else None
    ms = max_ms(ms_local)
    n_kp = int(cnt.item())
    value = replica_throughput(W_HD * H_HD, args.steps, world, ms)

    # -- dominant kernel timed alone (same stream) --------------------------
    stage_ms = {}
    reps = max(10, min(200, args.steps))
    for st, name in ((0, "pyramid"), (1, "gabor"), (2, "stencil"), (3, "nms")):
        detect(pool[0])
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            L.check(lib.bimp_ctx_run_stage(cs.handle, st, sp), "run_stage")
        b.record(stream)
        torch.cuda.synchronize()
        stage_ms[name] = a.elapsed_time(b) / reps
    alg = algorithmic_bytes(cs)
    peak, peak_kind = measured_peak()
    achieved = alg["gabor"] / (stage_ms["gabor"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_gabor_tiles", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": profiled_traffic(), "algorithmic_bytes": alg["gabor"],
                "avg_launch_ms": round(stage_ms["gabor"], 4)}
    for name in ("stencil", "nms"):
        a_gbs = alg[name] / (stage_ms[name] * 1e-3) / 1e9
        roofline[f"{name}_frac"] = round(a_gbs / peak, 4)

    # -- end to end through the host-buffer C ABI ---------------------------
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(im).pin_memory() for im in pool_np[:8]]
        outs = (L.KeyPointC * cap)()
        n = C.c_int()
        d2h = []

        def detect_host(img):
            a = img.numpy()
            rc = lib.bimp_detect_host(cs.handle, C.c_void_p(a.ctypes.data), a.strides[0], W_HD, H_HD, outs, cap,
                                      C.byref(n), sp)
            if rc not in (0, L.BIMP_ERR_CAPACITY):
                L.check(rc, "bimp_detect_host")
            d2h.append(4 + 28 * min(n.value, cap))

        for i in range(max(3, args.warmup)):
            detect_host(pinned[i % 8])
        d2h.clear()
        k_e2e = max(10, min(args.steps, 500))
        barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for i in range(k_e2e):
            detect_host(pinned[i % 8])
        b.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_ms(a.elapsed_time(b))
        e2e = {"value": round(world * k_e2e * W_HD * H_HD / (ms_e2e * 1e-3) / 1e6, 2), "unit": UNIT,
               "h2d_bytes_per_step": W_HD * H_HD, "d2h_bytes_per_step": int(np.mean(d2h)),
               "steps": k_e2e, "api": "bimp_detect_host"}

    # -- batched mixed sizes vs the same images one by one -----------------
    batched = None
    if not args.no_batched:
        imgs, lam_b = synth.workload("mixed", seed_base=1000 + 31 * rank)
        sizes = [(im.shape[1], im.shape[0]) for im in imgs]
        px = sum(w * h for w, h in sizes)
        bt = api.Batch(sizes, lam_b, kp_capacity=65536)
        bt.load(imgs)
        for _ in range(3):
            bt.run()
        torch.cuda.synchronize()
        kb = max(5, min(50, args.steps // 10))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        a.record(stream)
        for _ in range(kb):
            bt.run()
        b.record(stream)
        torch.cuda.synchronize()
        ms_b = max_ms(a.elapsed_time(b))
        # plain: one context per image, detected one after another
        ctxs = [api.CudaStuff(w, h, lam_b) for w, h in sizes]
        gimgs = [torch.from_numpy(im).to(dev) for im in imgs]
        kp2 = torch.zeros((7, 65536), dtype=torch.float32, device=dev)

        def plain_all():
            for c2, g in zip(ctxs, gimgs):
                rc = lib.bimp_detect_device_async(c2.handle, C.c_void_p(g.data_ptr()), g.stride(0), g.shape[1],
                                                  g.shape[0], C.c_void_p(kp2.data_ptr()), kp2.stride(0), 65536,
                                                  C.c_void_p(cnt.data_ptr()), sp)
                L.check(rc, "plain detect")

        plain_all()
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(kb):
            plain_all()
        b.record(stream)
        torch.cuda.synchronize()
        ms_p = max_ms(a.elapsed_time(b))
        batched = {"workload": "64 mixed images, W in [320,1920], H in [240,1080], 8 scales",
                   "value": round(world * kb * px / (ms_b * 1e-3) / 1e6, 2),
                   "plain_value": round(world * kb * px / (ms_p * 1e-3) / 1e6, 2),
                   "ratio": round(ms_p / ms_b, 3), "unit": UNIT, "graph": True}
        for c2 in ctxs:
            c2.close()
        bt.close()

    # -- CPU baseline (rank 0, N=1) -----------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import bimp_oracle as O
        t0 = time.perf_counter()
        O.run(pool_np[0], lam, keep_maps=False)
        dt = time.perf_counter() - t0
        cpu = {"value": round(W_HD * H_HD / dt / 1e6, 4), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "one 1920x1080 image, 8 scales x 8 orientations, FP64 numpy oracle, 1 thread",
               "seconds": round(dt, 2)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "plain BIMP, one 1920x1080 uint8 image per step (1/f^2 noise + 150 polygons)",
                       "scales": 8, "orientations": 8, "lambdas": [round(x, 6) for x in lam],
                       "input_pool": f"{POOL} distinct 1080p images resident in HBM (133 MB > L2), "
                                     "rotated per step; each step also streams ~200 MB of maps",
                       "keypoints_last_step": n_kp, "parallelism": f"replicas x{world}"},
            "roofline": roofline, "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "cpu_baseline": cpu, "e2e": e2e, "batched": batched,
            "gpu_launches": cs_launches(cs) * args.steps, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    cs.close()


def cs_launches(cs) -> int:
    from bimp_b200 import _lib as L
    return int(L.lib().bimp_ctx_kernel_launches(cs.handle))


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement of the reference pipeline
# ---------------------------------------------------------------------------
def _ref_scale(args):
    img, lam, i = args
    from oracle import bimp_oracle as O
    sc = O.scale_geometry(img.shape[1], img.shape[0], lam)[i]
    data = O.level_image(img, sc)
    Ct, _, _ = O.complex_cells(data, sc)
    maps = O.keypoint_maps(O.stencil_window(Ct, sc), sc)
    kp = O.extract_keypoints(maps["D"], sc, i)
    return len(kp.ix)


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    import multiprocessing as mp
    from bimp_b200 import synth
    lam = synth.bank(8)
    pool_np = hd_pool(0, 8)
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(cores, len(lam))) as pool:
        def step(img):
            return sum(pool.map(_ref_scale, [(img, lam, i) for i in range(len(lam))]))
        for i in range(args.warmup):
            step(pool_np[i % 8])
        t0 = time.perf_counter()
        for i in range(args.steps):
            step(pool_np[i % 8])
        dt = time.perf_counter() - t0
    value = args.steps * W_HD * H_HD / dt / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "plain BIMP, one 1920x1080 uint8 image per step", "scales": 8,
                       "orientations": 8},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": min(cores, len(lam)), "kind": "port",
                             "sample": "whole 1080p image per step; scales in parallel processes (FP64 oracle port; "
                                       "the reference itself needs OpenCV-CUDA and cannot be built here)"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.steps > 30:
            args.steps = 30     # keep the CPU run within a few minutes
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
