#!/usr/bin/env python
"""Benchmark of the BM3Dv2 basic estimate on B200.

Workload (one step): denoise a seeded synthetic YUV420PS clip, 1920x1080,
32 frames, radius 2, sigma 3, block_step 4, bm_range 16, ps_num 2,
ps_range 7, extractor_exp 0 (luma denoised, chroma passed through), the
reference benchmark's BM3D settings (benchmark/bench.py:108-121,167-180).

* value -- Mpx/s with the clip already in HBM (process_device), timed with
  CUDA events on the launch stream; the inputs (265 MB) exceed L2.
* e2e -- the same metric through the plugin-facing host call
  (vsfeel_bm3d_process_host) from pinned host memory, host->device and
  device->host copies of every frame inside the timed region.
* roofline -- the dominant kernel (block matching) timed live with CUDA
  events: algorithmic bytes per launch (8 B/px x one frame) / launch time.
* cpu_baseline -- the oracle (C++ restatement of the reference) on the host
  cores, on a bounded sample of whole stacks of the same workload.

``--impl reference`` times the reference's own shaders compiled for the CPU
(oracle/_ref) on the same workload instead; N>1 ranks other than 0 exit.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
For N > 1 launch one process per GPU with torch.distributed.run. The ranks
shard one clip of 32*N frames with vsfeel.shard.plan: each denoises its 32
output frames from its sub-clip, which carries a 2r-frame halo on each
interior side, and computes the halo's extra stacks itself (weak scaling:
32 output frames per GPU; no collective on the data path).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "vapoursynth-feel_b200"
for _p in (str(ROOT), str(PKG)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "BM3Dv2 1080p Mpx/s: plain vs batched vs fwd+bwd at ≤1e-4 max abs err"
UNIT = "Mpx/s"
WIDTH, HEIGHT, FRAMES = 1920, 1080, 32
PARAMS = dict(sigma=3.0, block_step=4, bm_range=16, radius=2, ps_num=2, ps_range=7,
              extractor_exp=0)
CONFIG = {
    "workload": "bm3dv2_plain_yuv420ps_1920x1080x32_r2",
    "format": "YUV420PS (luma denoised, 960x540 chroma passed through)",
    "width": WIDTH, "height": HEIGHT, "frames_per_step": FRAMES, **PARAMS,
    "noise_sigma_255": 3.0, "translation_px": 4,
    "l2": "inputs (265 MB of luma) larger than L2 (126 MB); no flush",
}
BYTES_PER_PX = 8  # algorithmic: read 4 + write 4 of luma per output pixel
PROFILE_FILE = ROOT / "profiles" / "bm3d_match_kernel__1080p_r2.txt"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_value(prefix: str):
    """The first number after `prefix` on a line of the committed ncu summary
    of the match kernel, or None."""
    try:
        for line in PROFILE_FILE.read_text().splitlines():
            if line.startswith(prefix):
                return float(line[len(prefix):].replace(":", " ").split()[0])
    except Exception:
        pass
    return None


def _profile_traffic():
    """dram bytes per launch of the match kernel from the committed ncu summary."""
    v = _profile_value("dram_bytes_per_launch_full_size")
    return int(v) if v is not None else None


# Useful FP32 work of the radius < 3 search, in the reference's sliding-column
# form (src/bm3d.comp:497-511): per candidate one new column SSD (8
# subtractions and 8 fused multiply-adds, 24 flops) and the three additions
# that advance the 8-column tree.
FLOPS_PER_CANDIDATE = 27


def candidates_per_stack(width: int, height: int, p: dict) -> int:
    """Candidates one stack evaluates: each block's spatial window clamped to
    the frame, plus 2r * ps_num temporal windows of (2Q+1)^2, clamped as if
    centred on the block itself (the predictors are matches near it)."""
    import numpy as np

    step = p["block_step"]

    def widths(extent, reach):
        nb = (extent - 9 + 2 * step) // step
        pos = np.minimum(np.arange(nb) * step, extent - 8)
        return np.minimum(pos + reach, extent - 8) - np.maximum(pos - reach, 0) + 1

    spatial = int(widths(width, p["bm_range"]).sum()) * int(widths(height, p["bm_range"]).sum())
    temporal = int(widths(width, p["ps_range"]).sum()) * int(widths(height, p["ps_range"]).sum())
    return spatial + 2 * p["radius"] * p["ps_num"] * temporal


def fp32_peak_tflops(torch, dev) -> tuple[float, str]:
    """FP32 CUDA-core peak: SMs x 128 lanes x 2 flops (FMA) x the max SM clock
    (MEASURED_PEAKS.json's sm_max_mhz, else 1965 MHz)."""
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz, src = 1965.0, "nominal max SM clock"
    try:
        mhz = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["sm_max_mhz"])
        src = "MEASURED_PEAKS.json sm_max_mhz"
    except Exception:
        pass
    return sms * 128 * 2 * mhz * 1e6 / 1e12, f"{sms} SMs x 128 FP32 lanes x 2 flop x {mhz:.0f} MHz ({src})"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str):
        self.device_id = device_id
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.device_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, sm_max, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                sm_max = max(sm_max, float(f[1]))
            except ValueError:
                continue
            for name, val in zip(names, f[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": sm_max,
                "reasons": sorted(reasons), "samples": len(sm)}


TILE_NAMES = ("8x4", "16x2", "4x8", "8x2", "4x4")


def matcher_config(info) -> dict:
    """Tile shape (blocks) and lanes per block of the context's matcher."""
    shape = info.match_tile_shape
    return {"tile": TILE_NAMES[shape] if 0 <= shape < len(TILE_NAMES) else "direct-read",
            "lanes_per_block": info.match_lanes, "autotuned": bool(info.autotuned)}


def _device_id(torch, dev) -> str:
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else f"GPU-{u}"
    except Exception:
        return str(dev)


def cpu_baseline_port(luma):
    """The oracle (C++ restatement of the reference) on the host cores: whole
    stacks of the workload until about 10 s have passed (at most 16)."""
    from oracle import Oracle, Params

    o = Oracle()
    p = Params(**PARAMS)
    threads = os.cpu_count() or 1
    done, t0 = 0, time.perf_counter()
    while done < 16:
        o.stack(luma, p, (luma.shape[0] // 2 + done) % luma.shape[0], nthreads=threads)
        done += 1
        if time.perf_counter() - t0 > 10.0:
            break
    dt = time.perf_counter() - t0
    return {"value": done * WIDTH * HEIGHT / dt / 1e6, "unit": UNIT, "cores": threads,
            "kind": "port",
            "sample": f"{done} stacks (one output frame each in the steady state) of the "
                      f"1920x1080 r2 workload, oracle fp32 with {threads} threads, {dt:.1f} s"}


GRAD_WORKLOADS = {
    # the differentiable workload: 16 frames 512x512, radius 1
    "fwd_bwd_512x512x16_r1": dict(frames=16, height=512, width=512, shift=3, seed=4,
                                  params=dict(sigma=5.0, block_step=4, bm_range=12, radius=1,
                                              ps_num=2, ps_range=5)),
    # the plain workload's clip and settings, forward + backward
    "fwd_bwd_1920x1080x32_r2": dict(frames=32, height=HEIGHT, width=WIDTH, shift=4, seed=2000,
                                    params=dict(PARAMS)),
    # the large workload: 24 frames 3840x2160, radius 4 (true 8x8 SSD search)
    "fwd_bwd_3840x2160x24_r4": dict(frames=24, height=2160, width=3840, shift=6, seed=4000,
                                    params=dict(sigma=8.0, block_step=4, bm_range=16, radius=4,
                                                ps_num=4, ps_range=7, extractor_exp=2)),
}


def time_fwd_bwd(torch, dev, name, steps, warmup, frames=None):
    """Forward alone (the plain path) and forward+backward through the
    autograd Function on one workload, timed with CUDA events; loss =
    sum(W * out) with W ~ N(0, 1) seeded."""
    import vsfeel
    from vsfeel.autograd import Denoiser
    from vsfeel.synthetic import make_clip_device

    wl = GRAD_WORKLOADS[name]
    n, h, w = frames or wl["frames"], wl["height"], wl["width"]
    x = make_clip_device(n, h, w, sigma=wl["params"]["sigma"], shift=wl["shift"], seed=wl["seed"],
                         device=dev)
    weights = torch.randn(x.shape, generator=torch.Generator(device=dev).manual_seed(6),
                          device=dev)
    den = Denoiser(x.shape, dev.index, **wl["params"])
    fwd_den = Denoiser(x.shape, dev.index, **wl["params"])
    plain = torch.empty_like(x)

    def fwd():
        fwd_den.plain(x, plain)

    def fwd_bwd():
        xr = x.detach().requires_grad_(True)
        out = den(xr)
        out.backward(weights)
        return xr.grad

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    fwd_ms = timed(fwd)
    fwd_den.close()
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats(dev)
    fb_ms = timed(fwd_bwd)
    torch_peak = int(torch.cuda.max_memory_allocated(dev))
    # adjoint kernel alone
    out, saved = den.forward_saved(x)
    torch.cuda.synchronize()
    adj_ms = timed(lambda: den.backward(saved, weights))
    px = n * h * w
    return {"workload": name, "fwd_mpx_s": px / fwd_ms / 1e3, "fwd_bwd_mpx_s": px / fb_ms / 1e3,
            "fwd_ms": fwd_ms, "fwd_bwd_ms": fb_ms, "backward_only_ms": adj_ms,
            "fwd_bwd_over_fwd": fb_ms / fwd_ms, "saved_state_bytes": int(den.layout.bytes),
            "peak_hbm_bytes_fwd_bwd": torch_peak + int(den.info.device_bytes),
            "peak_hbm_note": "torch's peak allocation during forward+backward (clip, output, "
                             "saved state, gradients) plus the library context's buffers",
            "steps": steps, "warmup": warmup}


def batched_clips(rng):
    """The batched workload: 64 clips of 16 frames, 16 at 640x360, 24 at
    1280x720, 16 at 1920x1080 and 8 at 3840x2160; per clip sigma U[1, 10],
    radius from {0, 1, 2}, block_step from {4, 8}; bm_range 16, ps_num 2,
    ps_range 7."""
    sizes = [(640, 360)] * 16 + [(1280, 720)] * 24 + [(1920, 1080)] * 16 + [(3840, 2160)] * 8
    out = []
    for i, (w, h) in enumerate(sizes):
        params = dict(sigma=float(rng.uniform(1.0, 10.0)), block_step=int(rng.choice([4, 8])),
                      bm_range=16, radius=int(rng.choice([0, 1, 2])), ps_num=2, ps_range=7)
        out.append((16, h, w, params))
    return out


def time_batched(torch, dev, steps, warmup):
    """The batched form on the 64-clip workload, against the same clips run
    one after another through the plain path (device-resident, CUDA events)."""
    import numpy as np

    from vsfeel.autograd import Denoiser
    from vsfeel.batch import Batch
    from vsfeel.synthetic import make_clip_device

    spec = batched_clips(np.random.default_rng(3000))
    src, dst = [], []
    for i, (n, h, w, p) in enumerate(spec):
        src.append(make_clip_device(n, h, w, p["sigma"], shift=4, seed=3000 + i, device=dev))
        dst.append(torch.empty_like(src[-1]))
    px = sum(n * h * w for n, h, w, _ in spec)
    t0 = time.perf_counter()
    batch = Batch([(s, d, p) for s, d, (_, _, _, p) in zip(src, dst, spec)], device=dev.index,
                  autotune=True)
    create_s = time.perf_counter() - t0
    for _ in range(warmup):
        batch.run()
    torch.cuda.synchronize()
    batch.finish()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        batch.run()
    b.record()
    torch.cuda.synchronize()
    batch.finish()
    batched_ms = a.elapsed_time(b) / steps
    classes = batch.classes()
    device_bytes = batch.device_bytes
    batched_out = [d.clone() for d in dst[:4]]
    batch.close()

    # the plain path, clip after clip, each at its steady state
    plain_ms = 0.0
    worst = 0.0
    for i, (s, d, (n, h, w, p)) in enumerate(zip(src, dst, spec)):
        den = Denoiser(s.shape, dev.index, **p)
        den.plain(s, d)
        torch.cuda.synchronize()
        a.record()
        for _ in range(2):
            den.plain(s, d)
        b.record()
        torch.cuda.synchronize()
        plain_ms += a.elapsed_time(b) / 2
        if i < 4:
            worst = max(worst, float((d - batched_out[i]).abs().max()))
        den.close()
    return {"workload": "batched_64_clips_mixed_360p_to_2160p_x16_frames",
            "batched_mpx_s": px / batched_ms / 1e3, "batched_ms": batched_ms,
            "plain_sequential_mpx_s": px / plain_ms / 1e3, "plain_sequential_ms": plain_ms,
            "batched_over_plain_sequential": plain_ms / batched_ms,
            "megapixels_per_step": px / 1e6, "create_and_autotune_s": create_s,
            "classes": classes, "device_bytes": device_bytes,
            "max_abs_diff_vs_plain_first4": worst, "steps": steps, "warmup": warmup}


def time_batched_sharded(torch, dev, rank, world, max_over_ranks, barrier, steps, warmup):
    """The 64-clip workload across `world` ranks: whole clips, assigned
    longest processing time first by the cost model (vsfeel.shard); every
    rank builds and runs only its clips as one batch. Device time is the max
    over ranks, and Mpx/s counts every clip's pixels once."""
    import numpy as np

    from vsfeel import shard as shard_mod
    from vsfeel.batch import Batch
    from vsfeel.synthetic import make_clip_device

    spec = batched_clips(np.random.default_rng(3000))
    costs = [shard_mod.clip_cost(*c) for c in spec]
    plan = shard_mod.assign_clips(costs, world)
    mine = plan[rank]
    src = [make_clip_device(spec[i][0], spec[i][1], spec[i][2], spec[i][3]["sigma"], shift=4,
                            seed=3000 + i, device=dev) for i in mine]
    dst = [torch.empty_like(x) for x in src]
    batch = Batch([(x, y, spec[i][3]) for x, y, i in zip(src, dst, mine)], device=dev.index,
                  autotune=True) if mine else None
    run = batch.run if batch else (lambda: None)
    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        run()
    b.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(a.elapsed_time(b) / steps)
    if batch:
        batch.finish()
        batch.close()
    px = sum(n * h * w for n, h, w, _ in spec)
    loads = [sum(costs[i] for i in part) for part in plan]
    return {"workload": "batched_64_clips_mixed_360p_to_2160p_x16_frames",
            "batched_mpx_s": px / ms / 1e3, "batched_ms": ms,
            "assignment": "whole clips, longest processing time first by the cost model",
            "clips_per_rank": [len(part) for part in plan],
            "predicted_ms_per_rank": [round(x, 2) for x in loads],
            "steps": steps, "warmup": warmup}


def time_all_planes(torch, dev, nfr, steps, warmup):
    """Per-plane denoising (the ``planes`` extension): a YUV420PS 1080p clip
    with all three planes denoised, the 960x540 chroma planes noisy like
    luma, same arguments per plane. Device-resident, one stream, CUDA events;
    Mpx/s counts the pixels of all three planes."""
    import vsfeel
    from vsfeel.synthetic import make_clip

    planes = [make_clip(nfr, HEIGHT, WIDTH, sigma=3.0, shift=4, seed=4000),
              make_clip(nfr, HEIGHT // 2, WIDTH // 2, sigma=3.0, shift=2, seed=4001),
              make_clip(nfr, HEIGHT // 2, WIDTH // 2, sigma=3.0, shift=2, seed=4002)]
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(*planes), planes=[0, 1, 2],
                         device=dev.index or 0, **PARAMS)
    src = [torch.from_numpy(x).to(dev) for x in planes]
    out = [torch.empty_like(x) for x in src]

    def step():
        for p in range(3):
            node.output_device(src[p], out[p], plane=p)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        step()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    px = sum(x.size for x in planes)
    return {"workload": f"bm3dv2_all_planes_yuv420ps_1920x1080x{nfr}_r2",
            "mpx_s": px / ms / 1e3, "ms_per_step": ms, "megapixels_per_step": px / 1e6,
            "steps": steps, "warmup": warmup}


def time_frame_requests(luma, u, v, dev_index, passes, threads):
    """The VapourSynth request path as vspipe drives it: get_frame(n) for
    n = 0..N-1 submitted in order to `threads` worker threads (that many
    requests in flight, fmParallel), the frames fetched from pageable host
    memory through the callbacks and each output copied back. Wall clock;
    each pass denoises the whole clip (the stack cache is smaller than the
    clip, so a pass recomputes every stack)."""
    from concurrent.futures import ThreadPoolExecutor

    import vsfeel

    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(luma, u, v), device=dev_index, **PARAMS)
    n = luma.shape[0]
    node.get_frame(0)
    launches0 = node.launch_count()
    with ThreadPoolExecutor(threads) as ex:
        t0 = time.perf_counter()
        for _ in range(passes):
            list(ex.map(node.get_frame, range(n)))
        sec = (time.perf_counter() - t0) / passes
    return {"workload": f"bm3dv2_get_frame_in_order_yuv420ps_1920x1080x{n}_r2",
            "threads": threads, "mpx_s": n * luma.shape[1] * luma.shape[2] / sec / 1e6,
            "ms_per_clip": sec * 1e3,
            "launches_per_frame": (node.launch_count() - launches0) / (passes * n),
            "passes": passes}


# Small workloads for ncu captures (a few GB of device memory at most, so
# that a capture of one launch ends quickly): each runs its path once per
# step, device-resident, and prints one line with the step time.
PROFILE_CASES = {
    # the radius >= 3 exact search with the 3840x2160 workload's arguments,
    # on 1080p frames (one stack per match launch)
    "exact_1920x1080x9_r4": dict(frames=9, height=HEIGHT, width=WIDTH, shift=6, seed=4100,
                                 params=dict(sigma=8.0, block_step=4, bm_range=16, radius=4,
                                             ps_num=4, ps_range=7, extractor_exp=2)),
    # the batched form on a mixed handful of clips (one persistent launch per
    # class chunk)
    "batched_small": None,
    # one 1080p radius-0 clip of 16 frames through the batched form (one
    # chunk: one persistent matching launch, one filter launch over its 16
    # stacks, one normalisation launch), 8x4 tiles
    "batched_1920x1080x16_r0": None,
}


def run_profile_case(torch, dev, name, steps, warmup):
    from vsfeel.synthetic import make_clip_device

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if name == "batched_small":
        from vsfeel.batch import Batch

        spec = [(4, 1080, 1920, dict(sigma=3.0, block_step=4, bm_range=16, radius=2, ps_num=2,
                                     ps_range=7))] * 2 + \
               [(8, 360, 640, dict(sigma=5.0, block_step=8, bm_range=16, radius=1, ps_num=2,
                                   ps_range=7))] * 4
        src = [make_clip_device(n, h, w, p["sigma"], shift=4, seed=4200 + i, device=dev)
               for i, (n, h, w, p) in enumerate(spec)]
        dst = [torch.empty_like(x) for x in src]
        batch = Batch([(x, y, p) for x, y, (_, _, _, p) in zip(src, dst, spec)],
                      device=dev.index or 0, autotune=False)
        run = batch.run
        px = sum(n * h * w for n, h, w, _ in spec)
    elif name == "batched_1920x1080x16_r0":
        from vsfeel.batch import Batch

        p = dict(sigma=5.0, block_step=4, bm_range=16, radius=0, ps_num=2, ps_range=7)
        x = make_clip_device(16, HEIGHT, WIDTH, p["sigma"], shift=4, seed=3100, device=dev)
        out = torch.empty_like(x)
        batch = Batch([(x, out, p)], device=dev.index or 0, autotune=False, tile_shape="8x4")
        run = batch.run
        px = x.numel()
    else:
        wl = PROFILE_CASES[name]
        x = make_clip_device(wl["frames"], wl["height"], wl["width"], sigma=wl["params"]["sigma"],
                             shift=wl["shift"], seed=wl["seed"], device=dev)
        from vsfeel.autograd import Denoiser

        out = torch.empty_like(x)
        den = Denoiser(x.shape, dev.index or 0, **wl["params"])
        run = lambda: den.plain(x, out)  # noqa: E731
        px = x.numel()
    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    a.record()
    for _ in range(steps):
        run()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / max(steps, 1)
    return {"profile_case": name, "ms_per_step": ms, "mpx_s": px / ms / 1e3, "steps": steps,
            "warmup": warmup}


def run_reference(args) -> int:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import Oracle, Params, ReferenceShaders
    from vsfeel.synthetic import make_clip

    luma = make_clip(5, HEIGHT, WIDTH, sigma=3.0, shift=4, seed=2000)
    p = Params(**PARAMS)
    threads = os.cpu_count() or 1
    nby = (HEIGHT - 9 + 2 * p.block_step) // p.block_step
    if ReferenceShaders.available():
        ref = ReferenceShaders()
        kind = "reference"

        def step(rows):
            # four bands spread from the top edge to the bottom edge, so that
            # edge rows (clamped, cheaper windows) are sampled in proportion
            bands = min(4, rows)
            for k in range(bands):
                n = rows // bands + (1 if k < rows % bands else 0)
                first = (nby - n) * k // max(bands - 1, 1)
                ref.stack_rows(luma, p, 2, first, n, nthreads=threads)
        what = ("reference shaders (src/bm3d.comp) compiled for the CPU, rows in four bands "
                "from the top edge to the bottom edge")
    else:
        o = Oracle()
        kind = "port"

        def step(rows):
            o.stack(luma, p, 2, nthreads=threads)
        what = "oracle restatement (reference shaders not built)"
    # size each step so that warmup + steps take about 150 s
    t0 = time.perf_counter()
    step(8)
    per_row = (time.perf_counter() - t0) / 8
    total = args.steps + args.warmup
    rows = int(max(4, min(nby, 150.0 / max(total, 1) / max(per_row, 1e-6))))
    if kind == "port":
        rows = nby
    for _ in range(args.warmup):
        step(rows)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(rows)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    px = rows * p.block_step * WIDTH
    value = px / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": CONFIG,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{rows} block rows ({px} px of reference blocks) of stack 2 "
                                   f"per step, {what}, {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--frames", type=int, default=FRAMES,
                    help="frames per step (default 32; smaller only for profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass")
    ap.add_argument("--no-grad", action="store_true",
                    help="skip the forward+backward measurements")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-form measurement")
    ap.add_argument("--no-planes", action="store_true",
                    help="skip the all-planes (chroma denoised) measurement")
    ap.add_argument("--case", choices=sorted(GRAD_WORKLOADS),
                    help="only time forward and forward+backward of this workload (a small "
                         "profiling target) and print its line")
    ap.add_argument("--case-frames", type=int, default=None,
                    help="frames of the --case clip (default: the workload's)")
    ap.add_argument("--profile-case", choices=sorted(PROFILE_CASES),
                    help="only run this small profiling workload and print its line")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_case:
        import torch

        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        print(json.dumps(run_profile_case(torch, dev, args.profile_case, args.steps, args.warmup)),
              flush=True)
        return 0
    if args.case:
        import torch

        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        line = time_fwd_bwd(torch, dev, args.case, args.steps, args.warmup, args.case_frames)
        print(json.dumps(line), flush=True)
        return 0

    import numpy as np
    import torch
    import torch.distributed as dist

    import vsfeel
    from vsfeel.synthetic import make_chroma, make_clip_range

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # one clip of nfr frames per rank, sharded by output range: this rank
    # denoises outputs out_first.. of the whole clip from its sub-clip
    # (its range plus the 2r-frame halo), generated alone
    from vsfeel import shard as shard_mod

    nfr = args.frames
    total_frames = nfr * world
    shards = shard_mod.plan(total_frames, world, PARAMS["radius"])
    sh = shards[rank]
    luma = make_clip_range(total_frames, sh.in_first, sh.in_count, HEIGHT, WIDTH, sigma=3.0,
                           shift=4, seed=2000)
    u = make_chroma(sh.in_count, HEIGHT // 2, WIDTH // 2, seed=2000 + sh.in_first)
    v = make_chroma(sh.in_count, HEIGHT // 2, WIDTH // 2, seed=3000 + sh.in_first)
    r = PARAMS["radius"]

    def stacks_of(s):
        # stacks a shard computes: its outputs' stacks, clamped to its sub-clip
        lo = max(s.local_first - r, 0)
        hi = min(s.local_first + s.out_count - 1 + r, s.in_count - 1)
        return hi - lo + 1 if s.out_count else 0

    halo_fraction = sum(stacks_of(s) for s in shards) / total_frames - 1.0

    # ---- device-resident pass ------------------------------------------------
    node = vsfeel.BM3Dv2(vsfeel.clip_from_array(luma, u, v), device=local_rank, **PARAMS)
    d_src = torch.from_numpy(luma).to(dev)
    d_out = torch.empty((sh.out_count, HEIGHT, WIDTH), dtype=torch.float32, device=dev)

    def run_device():
        node.output_device(d_src, d_out, first=sh.local_first, count=sh.out_count)

    for _ in range(args.warmup):
        run_device()
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(_device_id(torch, dev))
    clocks.start()
    time.sleep(0.3)
    node.trace(True)
    launches0 = node.launch_count()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(args.steps):
        run_device()
    stop.record()
    torch.cuda.synchronize()
    elapsed_ms = start.elapsed_time(stop)
    launches = node.launch_count() - launches0
    kt = node.trace_read()
    node.trace(False)
    clk = clocks.stop()
    barrier()
    elapsed_ms = max_over_ranks(elapsed_ms)
    ms_per_step = elapsed_ms / args.steps
    px_per_step = total_frames * WIDTH * HEIGHT  # output pixels of all ranks
    value = px_per_step / (ms_per_step / 1e3) / 1e6

    # ---- end to end through the host entry point (pinned buffers) -----------
    e2e = None
    if not args.no_e2e:
        h_src = torch.from_numpy(luma).pin_memory()
        h_out = torch.empty((sh.out_count, HEIGHT, WIDTH), dtype=torch.float32).pin_memory()
        enode = vsfeel.BM3Dv2(vsfeel.clip_from_array(h_src.numpy(), u, v), device=local_rank,
                              **PARAMS)
        out_np = h_out.numpy()
        for _ in range(max(1, args.warmup)):
            enode.output(sh.local_first, sh.out_count, out=out_np)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            enode.output(sh.local_first, sh.out_count, out=out_np)
        e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
        e2e = {"value": px_per_step / e2e_s / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(h_src.numel() * 4),
               "d2h_bytes_per_step": int(h_out.numel() * 4),
               "bytes_note": "this rank's copies (its sub-clip up, its outputs down)",
               "max_abs_diff_vs_device_path": float(np.abs(out_np - d_out.cpu().numpy()).max())}

    # ---- roofline of the dominant kernel ------------------------------------
    match_ms, match_n = kt["bm3d_match_kernel"]
    avg_s = match_ms / max(match_n, 1) / 1e3
    alg_bytes = BYTES_PER_PX * WIDTH * HEIGHT
    achieved = alg_bytes / avg_s / 1e9 if avg_s > 0 else 0.0
    peak, peak_src = _peaks()
    traffic = _profile_traffic()
    cands = candidates_per_stack(WIDTH, HEIGHT, PARAMS)
    useful_flops = cands * FLOPS_PER_CANDIDATE
    fp32_peak, fp32_src = fp32_peak_tflops(torch, dev)
    fp32_achieved = useful_flops / avg_s / 1e12 if avg_s > 0 else 0.0
    compute = {"bound": "fp32", "achieved": fp32_achieved, "peak": fp32_peak, "unit": "TFLOP/s",
               "frac": fp32_achieved / fp32_peak, "peak_source": fp32_src,
               "useful_flops_per_launch": useful_flops, "candidates_per_launch": cands,
               "flops_per_candidate": FLOPS_PER_CANDIDATE,
               "flops_note": "the reference's sliding-column SSD: one new column SSD (24 flops) "
                             "and 3 tree additions per candidate; warm-up columns, idle lanes "
                             "and selection are overhead, not counted",
               "ncu_sm_throughput_pct": _profile_value("sm__throughput (pct of peak)"),
               "ncu_fma_pipe_pct": _profile_value("sm__pipe_fma_cycles_active (pct of peak)")}
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": "bm3d_match_kernel", "peak_source": peak_src,
                "binding_roof": "compute (FP32 CUDA-core issue): see roofline.compute; the HBM "
                                "fraction is far below it by the algorithm's 8 B/px",
                "compute": compute,
                "avg_launch_ms": avg_s * 1e3, "algorithmic_bytes_per_launch": alg_bytes,
                # the matcher configuration the timed launches used
                "match_kernel": matcher_config(node.info),
                # summed event spans per kernel kind; filtering and normalisation run
                # on a second stream beside the matching, so their spans overlap it
                # and include waiting for SM space (the ncu launch list in profiles/
                # gives the serialised time shares)
                "kernel_span_ms_per_step": {k: round(ms / args.steps, 3) for k, (ms, _) in kt.items()},
                "kernel_span_share": {k: round(ms / max(sum(x[0] for x in kt.values()), 1e-9), 4)
                                    for k, (ms, _) in kt.items()}}

    # the batched form across ranks: every rank takes part (collectives)
    batched_sharded = None
    if world > 1 and not args.no_batch:
        batched_sharded = time_batched_sharded(torch, dev, rank, world, max_over_ranks, barrier,
                                               max(2, args.steps // 3), 3)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**CONFIG, "frames_per_step": total_frames,
                   "parallelism": f"frame-shard x{world}: one clip of {total_frames} frames, "
                                  f"{nfr} output frames per rank plus a {2 * r}-frame halo "
                                  f"per interior side"},
        "halo_recompute_fraction": halo_fraction,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "roofline": roofline,
        "clocks": clk,
    }
    if world == 1 and not args.no_grad:
        line["fwd_bwd"] = [time_fwd_bwd(torch, dev, name,
                                        3 if name.endswith("_r4") else max(3, args.steps // 2), 3)
                           for name in GRAD_WORKLOADS]
    if world == 1 and not args.no_batch:
        line["batched"] = time_batched(torch, dev, max(2, args.steps // 3), 3)
    if batched_sharded is not None:
        line["batched"] = batched_sharded
    if world == 1 and not args.no_e2e:
        line["frame_requests"] = [time_frame_requests(luma, u, v, local_rank, 2, t)
                                  for t in (1, 4)]
    if world == 1 and not args.no_planes:
        line["all_planes"] = time_all_planes(torch, dev, nfr, max(3, args.steps // 2), 3)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(luma)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
