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
* ``adjoint``  forward and backward of sum(M * D) on 16 float 512x512 images
              (6 scales): bwd/fwd time ratio and the gradient against the
              FP64 CPU reference on one image;
* ``cpu_baseline`` the FP32 C restatement of the reference pipeline (own
              FFT, OpenMP) on three 1080p images (rank 0, N=1).

``--impl reference`` times the reference pipeline's FP32 C restatement
(oracle/cbimp.c; the reference itself cannot be built here) on all of this
host's cores and prints the same metric with "impl": "reference".

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
        stencil += n * (8 * 4 + 4)        # 8 magnitude maps read + D written
        nms += n * 4                      # D read once
    return {"gabor": gabor, "stencil": stencil, "nms": nms}


def fft_flops(cs) -> float:
    """FFT arithmetic of one tile-kernel launch (5 N log2 N per complex N-point
    transform): per 128 x 128 tile a forward real transform (64 packed rows
    and 65 half-spectrum columns) and per orientation the spectrum product,
    128 column and V row inverse transforms and V^2 magnitudes."""
    per_fft = 5 * 128 * 7
    total = 0.0
    for k in cs.ks:
        v = 128 - 2 * k["kernel_x"]
        tiles = -(-(k["data_w"] + 1) // v) * -(-(k["data_h"] + 2) // v)
        per_tile = (64 + 65) * per_fft + 8 * (2 * 128 * 128 + (128 + v) * per_fft + 3 * v * v)
        total += tiles * per_tile
    return total


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


def headline_config(lam, world: int) -> dict:
    """The workload both arms report (the same dict in both lines)."""
    return {"workload": "plain BIMP, one 1920x1080 uint8 image per step (1/f^2 noise + 150 polygons)",
            "scales": 8, "orientations": 8, "lambdas": [round(x, 6) for x in lam],
            "input_pool": f"{POOL} distinct 1080p images (133 MB > L2), rotated per step",
            "parallelism": f"replicas x{world}"}


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
                "traffic": profiled_traffic(), "traffic_source": "profiles/gabor_tiles_hd.md (one ncu capture "
                "of this launch; not measured in this run)", "algorithmic_bytes": alg["gabor"],
                "avg_launch_ms": round(stage_ms["gabor"], 4)}
    for name in ("stencil", "nms"):
        a_gbs = alg[name] / (stage_ms[name] * 1e-3) / 1e9
        roofline[f"{name}_frac"] = round(a_gbs / peak, 4)
    # the tile kernel is bound by FP32 FFT arithmetic, not HBM: its FFT
    # flop rate against the nominal FP32 CUDA-core peak, for context
    fl = fft_flops(cs)
    roofline["fp32_context"] = {"fft_gflop_per_launch": round(fl / 1e9, 3),
                                "tflops": round(fl / (stage_ms["gabor"] * 1e-3) / 1e12, 2),
                                "nominal_fp32_tflops": 74.4,
                                "frac_of_nominal": round(fl / (stage_ms["gabor"] * 1e-3) / 74.4e12, 3)}

    # -- end to end through the host-buffer C ABI ---------------------------
    # Pinned host frames in, host cv::KeyPoint records out, every copy inside
    # the timed region.  Headline: the pipelined entry point (frames in
    # flight, bimp_pipeline_push/pop); beside it the one-frame-per-call
    # bimp_detect_host.  Timed by the host clock from the first push to the
    # last pop (which returns only after that frame's copies are done).
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(im).pin_memory() for im in pool_np[:8]]
        arrs = [t.numpy() for t in pinned]
        outs = (L.KeyPointC * cap)()
        n = C.c_int()
        d2h = []
        depth = args.depth
        pl = api.Pipeline(W_HD, H_HD, lam, depth=depth, capacity=cap)

        def pop():
            rc = lib.bimp_pipeline_pop(pl._h, outs, cap, C.byref(n))
            if rc not in (0, L.BIMP_ERR_CAPACITY):
                L.check(rc, "bimp_pipeline_pop")
            d2h.append(8 + 28 * min(n.value, cap))

        def push(a):
            L.check(lib.bimp_pipeline_push(pl._h, C.c_void_p(a.ctypes.data), a.strides[0], W_HD, H_HD),
                    "bimp_pipeline_push")

        def stream_frames(k):
            for i in range(k):
                if lib.bimp_pipeline_in_flight(pl._h) == depth:
                    pop()
                push(arrs[i % 8])
            while lib.bimp_pipeline_in_flight(pl._h):
                pop()

        stream_frames(max(3, args.warmup))
        d2h.clear()
        k_e2e = max(10, min(args.steps, 1000))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        stream_frames(k_e2e)
        ms_e2e = max_ms((time.perf_counter() - t0) * 1e3)
        pl.close()
        e2e = {"value": round(world * k_e2e * W_HD * H_HD / (ms_e2e * 1e-3) / 1e6, 2), "unit": UNIT,
               "h2d_bytes_per_step": W_HD * H_HD, "d2h_bytes_per_step": int(np.mean(d2h)),
               "steps": k_e2e, "api": f"bimp_pipeline_push / bimp_pipeline_pop, {depth} frames in flight",
               "host_memory": "pinned frames in, caller's records array out"}

        def detect_host(a):
            rc = lib.bimp_detect_host(cs.handle, C.c_void_p(a.ctypes.data), a.strides[0], W_HD, H_HD, outs, cap,
                                      C.byref(n), sp)
            if rc not in (0, L.BIMP_ERR_CAPACITY):
                L.check(rc, "bimp_detect_host")

        for i in range(3):
            detect_host(arrs[i % 8])
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(k_e2e):
            detect_host(arrs[i % 8])
        ms_sync = max_ms((time.perf_counter() - t0) * 1e3)
        e2e["per_call_api"] = {"api": "bimp_detect_host (one frame per call, synchronous)",
                               "value": round(world * k_e2e * W_HD * H_HD / (ms_sync * 1e-3) / 1e6, 2),
                               "ms_per_frame": round(ms_sync / k_e2e, 4)}

    # -- batched mixed sizes vs the same images one by one -----------------
    batched = None
    if not args.no_batched:
        imgs, lam_b = synth.workload("mixed", seed_base=1000 + 31 * rank)
        sizes = [(im.shape[1], im.shape[0]) for im in imgs]
        px = sum(w * h for w, h in sizes)
        bt = api.Batch(sizes, lam_b, kp_capacity=65536)
        bt.load(imgs)
        tune = bt.autotune(reps=3)   # tile plan: kernel variant, valid-block policy, tile order, grid
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
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
                   "ratio": round(ms_p / ms_b, 3), "unit": UNIT, "graph": True,
                   "autotune": {"chosen": tune["chosen"], "plans_timed": len(tune["tried"]),
                                "kernels_tried": sorted({t["kernel"] for t in tune["tried"]}),
                                "valid_block_policies_tried": sorted({t["policy"] for t in tune["tried"]}),
                                "grids_tried": sorted({t["grid"] for t in tune["tried"]}),
                                # the plan a batch starts with: phased kernel, largest valid
                                # block, scale-by-scale order, split over one CTA per SM
                                "default_plan_ms": next((t["ms"] for t in tune["tried"]
                                                         if t["policy"] == 0 and t["order"] == 0
                                                         and t["grid"] == sms and t["kernel"] == 0),
                                                        None),
                                "tried": [[t["policy"], t["order"], t["kernel"], t["grid"], t["ms"]]
                                          for t in tune["tried"]],
                                "tried_fields": ["policy", "order", "kernel", "grid", "ms"]}}
        for c2 in ctxs:
            c2.close()
        bt.close()

    # -- adjoint: 16 x 512x512 float images, 6 scales, fwd vs bwd ----------
    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint_bench(args, rank, world, dev, stream, max_ms)

    # -- CPU baseline (rank 0, N=1) -----------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_port_baseline(pool_np, lam, images=3)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": headline_config(lam, world), "keypoints_last_step": n_kp,
            "roofline": roofline, "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "cpu_baseline": cpu, "e2e": e2e, "batched": batched, "adjoint": adjoint,
            "gpu_launches": cs_launches(cs) * args.steps, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    cs.close()


def run_adjoint_bench(args, rank, world, dev, stream, max_ms):
    """Forward (loss) and backward (image + 4 parameter gradients) of the
    summed keypoint maps on 16 float 512x512 images, 6 scales; bwd/fwd time
    ratio, Mpixel/s of the training step, and (rank 0, N=1) the gradient of
    image 0 against the FP64 CPU reference and a finite difference."""
    import torch
    from bimp_b200 import api, synth
    imgs, lam = synth.workload("adjoint", seed_base=1000 + 13 * rank)
    n, h, w = len(imgs), imgs[0].shape[0], imgs[0].shape[1]
    x = torch.from_numpy(np.stack(imgs)).to(dev).contiguous()
    adj = api.Adjoint(w, h, n, lam)
    rng = np.random.default_rng(99 + rank)
    masks = torch.from_numpy(rng.standard_normal(n * adj.mask_stride).astype(np.float32)).to(dev)
    for _ in range(3):
        adj.forward(x, masks)
        adj.backward()
    torch.cuda.synchronize()
    k = max(5, min(50, args.steps // 20))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd_ms = bwd_ms = 0.0
    for _ in range(k):
        ev[0].record(stream)
        adj.forward(x, masks)
        ev[1].record(stream)
        adj.backward()
        ev[2].record(stream)
        torch.cuda.synchronize()
        fwd_ms += ev[0].elapsed_time(ev[1])
        bwd_ms += ev[1].elapsed_time(ev[2])
    fwd_ms = max_ms(fwd_ms / k)
    bwd_ms = max_ms(bwd_ms / k)
    out = {"workload": "16 float 512x512 images, 6 scales x 8 orientations, L = sum(M * D), "
                       "grads wrt image, lambda scale, sigma ratio, w_tan, w_rad",
           "fwd_ms": round(fwd_ms, 3), "bwd_ms": round(bwd_ms, 3), "bwd_fwd_ratio": round(bwd_ms / fwd_ms, 3),
           "train_step_mpixel_s": round(world * n * w * h / ((fwd_ms + bwd_ms) * 1e-3) / 1e6, 1),
           "device_bytes": adj.device_bytes()}
    if rank == 0 and world == 1 and not args.no_cpu:
        # image 0 against the FP64 CPU reference gradient: branch-matched (the
        # reference takes its ReLU states and magnitude floor from the
        # device's float32 complex cells) and on its own FP64 branch
        from oracle import bimp_adjoint as A
        one = api.Adjoint(w, h, 1, lam)
        m1 = masks[:adj.mask_stride].contiguous()
        one.forward(x[:1].contiguous(), m1)
        g1, gp1 = one.backward()
        g0 = g1[0].cpu().numpy()
        gp1 = gp1.cpu().numpy().copy()
        mv = [m.cpu().numpy().astype(np.float64) for m in one.mask_views(m1)[0]]
        dec = [np.stack([one.complex_map(0, s, o).cpu().numpy() for o in range(8)]) for s in range(len(one.layout))]
        x64 = imgs[0].astype(np.float64)
        _, ref_g, ref_p = A.gradient(x64, lam, mv, decide=dec)
        _, free_g, free_p = A.gradient(x64, lam, mv)
        names = ("alpha", "rho", "w_tan", "w_rad")
        out["grad_rel_err_image0"] = float(np.linalg.norm(g0 - ref_g) / np.linalg.norm(ref_g))
        out["param_rel_err_image0"] = [float(abs(gp1[k] - ref_p[nm]) / abs(ref_p[nm])) for k, nm in enumerate(names)]
        out["grad_rel_err_image0_fp64_branch"] = float(np.linalg.norm(g0 - free_g) / np.linalg.norm(free_g))
        # central finite difference of the FP64 loss along one seeded
        # direction, step 1e-4: kink-limited on this piecewise-linear loss
        v = np.random.default_rng(11).standard_normal(x64.shape)
        hh = 1e-4
        fd = (A.loss(x64 + hh * v, lam, mv) - A.loss(x64 - hh * v, lam, mv)) / (2 * hh)
        out["fd_step_1e-4_rel_diff_image0"] = float(abs(fd - float((g0 * v).sum())) / abs(fd))
        one.close()
    adj.close()
    if rank == 0 and world == 1 and not args.no_uhd_adjoint:
        # the 32-frame UHD configuration (12 scales): timing and peak device memory
        out["uhd_32_frames"] = uhd_adjoint(synth.uhd_frames(32, 1004), dev, stream)
    return out


def run_configs(args):
    """The other workload configurations, each next to the FP32 C
    restatement on the host cores (one JSON object):

    * cfg0: one 640x480 image, 4 scales (4, 8, 16, 32), plain path;
    * cfg4: 32 correlated 3840x2160 frames, 12 scales: batched forward (one
      graph replay) and the adjoint forward + backward of all 32 frames,
      with the device memory it holds.
    """
    import torch
    from bimp_b200 import _lib as L
    from bimp_b200 import api, synth
    from oracle.cbimp import CBimp, max_threads
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(int(stream.cuda_stream))
    lib = L.lib()
    out = {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, k):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(k):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / k

    def cpu(img, lam, reps):
        with CBimp(img.shape[1], img.shape[0], lam) as cb:
            cb.detect(img)
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                cb.detect(img)
                ts.append(time.perf_counter() - t0)
        return {"mpixel_s": round(img.size / statistics.median(ts) / 1e6, 3), "cores": max_threads(),
                "median_s": round(statistics.median(ts), 4), "runs": reps}

    # cfg0: VGA, plain path, 16 distinct shifted copies resident in HBM
    imgs, lam = synth.workload("vga")
    pool = [torch.from_numpy(np.ascontiguousarray(np.roll(imgs[0], 37 * i, axis=1))).to(dev) for i in range(16)]
    cs = api.CudaStuff(640, 480, lam)
    kp = torch.zeros((7, 65536), dtype=torch.float32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    it = [0]

    def vga_step():
        g = pool[it[0] % 16]
        it[0] += 1
        L.check(lib.bimp_detect_device_async(cs.handle, C.c_void_p(g.data_ptr()), g.stride(0), 640, 480,
                                             C.c_void_p(kp.data_ptr()), kp.stride(0), 65536,
                                             C.c_void_p(cnt.data_ptr()), sp), "vga detect")
    ms = timed(vga_step, 500)
    out["cfg0"] = {"workload": "one 640x480 uint8 image, lambdas 4, 8, 16, 32, 8 orientations, plain path",
                   "ms_per_image": round(ms, 4), "mpixel_s": round(640 * 480 / (ms * 1e-3) / 1e6, 1),
                   "cpu_baseline": cpu(imgs[0], lam, 5)}
    cs.close()
    del pool

    # cfg4: 32 UHD frames, 12 scales
    frames = synth.uhd_frames(32, 1004)
    lam12 = synth.bank(12)
    free0 = torch.cuda.mem_get_info()[0]
    bt = api.Batch([(3840, 2160)] * 32, lam12, kp_capacity=1 << 20)
    bt_bytes = free0 - torch.cuda.mem_get_info()[0]
    bt.load(frames)
    ms = timed(bt.run, 5)
    n_kp = int(bt.counts().sum().item())
    bt.close()
    torch.cuda.synchronize()
    fwd = {"ms_per_batch": round(ms, 2), "mpixel_s": round(32 * 3840 * 2160 / (ms * 1e-3) / 1e6, 1),
           "device_bytes": int(bt_bytes), "keypoints": n_kp, "graph": True}
    out["cfg4"] = {"workload": "32 correlated 3840x2160 frames (subpixel shifts <= 2 px + N(0,2) noise), "
                               "12 scales x 8 orientations",
                   "forward_batched": fwd,
                   "adjoint": uhd_adjoint(frames, dev, stream),
                   "cpu_baseline_one_frame": cpu(synth.uhd_frames(1, 1004)[0], lam12, 1)}
    print(json.dumps({"configs": out}), flush=True)


def uhd_adjoint(frames, dev, stream) -> dict:
    """Adjoint forward + backward of 32 UHD frames with the 12-scale bank:
    times, bwd/fwd ratio and the device memory it holds at its peak."""
    import torch
    from bimp_b200 import api, synth
    lam12 = synth.bank(12)
    n = len(frames)
    x = torch.from_numpy(np.stack([f.astype(np.float32) / np.float32(255.0) for f in frames])).to(dev)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    adj = api.Adjoint(3840, 2160, n, lam12)
    masks = torch.randn(n * adj.mask_stride, generator=torch.Generator(device=dev).manual_seed(5), device=dev)
    adj.forward(x, masks)
    grad, _ = adj.backward()
    torch.cuda.synchronize()
    held = free0 - torch.cuda.mem_get_info()[0]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, k):
        fn()
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(k):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / k

    f_ms = timed(lambda: adj.forward(x, masks), 3)
    b_ms = timed(lambda: adj.backward(grad), 3)
    out = {"workload": f"{n} correlated 3840x2160 float frames, 12 scales x 8 orientations, L = sum(M * D)",
           "fwd_ms": round(f_ms, 2), "bwd_ms": round(b_ms, 2), "bwd_fwd_ratio": round(b_ms / f_ms, 3),
           "train_step_mpixel_s": round(n * 3840 * 2160 / ((f_ms + b_ms) * 1e-3) / 1e6, 1),
           "device_bytes_arena": adj.device_bytes(), "device_bytes_held": int(held),
           "note": "peak device memory held by the adjoint (its arena plus the gradient output), measured "
                   "as the drop in free device memory; the backward recomputes each tile's spectrum and "
                   "e + i o (nothing of the forward's responses is stored); complex cells, their gradient "
                   "and the inhibition maps exist for a chunk of frames at a time"}
    adj.close()
    del x, masks, grad
    torch.cuda.synchronize()
    return out


def cs_launches(cs) -> int:
    from bimp_b200 import _lib as L
    return int(L.lib().bimp_ctx_kernel_launches(cs.handle))


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement of the reference pipeline
# ---------------------------------------------------------------------------
def cpu_port_baseline(images_np, lam, images: int, warmup: int = 1) -> dict:
    """The FP32 C restatement of the reference pipeline (oracle/cbimp.c, own
    FFT, OpenMP over every host thread) on `images` 1080p images."""
    from oracle.cbimp import CBimp, max_threads
    with CBimp(W_HD, H_HD, lam) as cb:
        for i in range(warmup):
            cb.detect(images_np[i % len(images_np)])
        times = []
        for i in range(images):
            t0 = time.perf_counter()
            cb.detect(images_np[(warmup + i) % len(images_np)])
            times.append(time.perf_counter() - t0)
    dt = sum(times)
    return {"value": round(images * W_HD * H_HD / dt / 1e6, 4), "unit": UNIT, "cores": max_threads(),
            "kind": "port",
            "sample": f"{images} 1920x1080 images after {warmup} warm-up, 8 scales x 8 orientations; FP32 C "
                      "restatement of the reference pipeline (whole-torus FFT filtering, own mixed-radix FFT, "
                      "OpenMP over all host threads)",
            "seconds": round(dt, 3), "median_s_per_image": round(statistics.median(times), 4)}


def run_reference(args, rank: int, world: int):
    """The reference's pipeline on the host cores: the reference itself needs
    OpenCV-CUDA 3.x, Boost, CUDA-samples headers and texture references
    (removed in CUDA 12), so its FP32 C restatement stands in for it.  Same
    64-image pool, bank and config as the GPU arm; each step is one whole
    1080p image, at most 30 steps so that the run stays within minutes."""
    if rank != 0:
        return
    from bimp_b200 import synth
    from oracle.cbimp import CBimp, max_threads
    lam = synth.bank(8)
    pool_np = hd_pool(0)
    with CBimp(W_HD, H_HD, lam) as cb:
        for i in range(args.warmup):
            cb.detect(pool_np[i % POOL])
        t0 = time.perf_counter()
        n_kp = 0
        for i in range(args.steps):
            n_kp = cb.detect(pool_np[i % POOL])[1]
        dt = time.perf_counter() - t0
    value = args.steps * W_HD * H_HD / dt / 1e6
    cores = max_threads()
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": headline_config(lam, world), "keypoints_last_step": n_kp,
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} whole 1080p images of the {POOL}-image pool after "
                                       f"{args.warmup} warm-up; FP32 C restatement of the reference pipeline, "
                                       "OpenMP over all host threads (the reference needs OpenCV-CUDA 3.x and "
                                       "CUDA<=11 texture references and cannot be built here)"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--depth", type=int, default=4, help="frames in flight of the end-to-end measurement")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-uhd-adjoint", action="store_true",
                    help="skip the 32-frame UHD adjoint inside the adjoint block (N=1 only)")
    ap.add_argument("--configs", action="store_true",
                    help="the other workload configurations (VGA, 32 UHD frames forward and adjoint), 1 GPU")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="only the forward/backward measurement of the adjoint workload (1 GPU)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.configs:
        run_configs(args)
        return
    if args.adjoint_only:
        import torch
        torch.cuda.set_device(local_rank)
        out = run_adjoint_bench(args, 0, 1, torch.device("cuda", local_rank), torch.cuda.current_stream(),
                                lambda v: float(v))
        print(json.dumps({"adjoint": out}), flush=True)
        return
    if args.impl == "reference":
        # each step is a whole 1080p image on the CPU (~0.3 s): keep the run
        # within a few minutes
        args.steps = min(args.steps, 30)
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
