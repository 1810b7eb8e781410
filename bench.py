#!/usr/bin/env python
"""Throughput of the digHolo batch path on B200: frames/s through
FFT -> window -> IFFT -> tilt removal -> HG overlap.

Workload (the batched dual-polarisation benchmark): 1024 frames of 640x512
uint16 (12-bit), two polarisations (left/right halves, carriers
+-(0.25, 0.2) Nyquist), 120 HG modes (maxMG 15), waist 250 um, 25 dB SNR,
FFT window 128x128, IFFT resolution mode 1 (window-sized reconstruction,
the mode the digHolo header recommends).  Frames are synthetic (seeded, the
hologram model of digholo_b200/synth.py, generated on the GPU).

One step = digHoloProcessBatch over one batch of 1024 frames.
  value : frames/s with the frames already resident in HBM
          (digHoloSetBatchUint16 given a device pointer, outputs left on the
          device); four different batches rotate so the 268 MB of window
          pixels they hold exceed the 126 MB L2.
  e2e   : frames/s through the plain C ABI with the frames in pinned host
          memory: the window copies host->device and the coefficient copy
          device->host are inside the timed region.
Timing: CUDA events on the library's stream (set to torch's current
stream), W untimed warm-up steps, K timed steps, max over ranks.
With torchrun each rank processes its own batches (frames are independent:
weak scaling, no collective on the data path).

--impl reference times the reference's own CPU implementation (the
reference compiled from its sources into oracle/_ref, FFT stage served by
this project's FFT library, not FFTW) on the host cores.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "batched_640x512_u16_2pol"
RES_MODE = 1
FRAMES = 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mode", type=int, default=RES_MODE, help="IFFT resolution mode (0 full, 1 window)")
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--overlap", default="tc", choices=["tc", "f32"],
                    help="overlap of full-resolution fields: split-BF16 tensor cores or FP32 CUDA cores")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autoalign", action="store_true", help="skip the AutoAlign (plain vs adjoint) measurement")
    ap.add_argument("--inverse-kernel", type=int, default=0,
                    help="digHoloB200SetInverseKernel choice (0 automatic; 3 forward and inverse fused into "
                         "one launch where they can be)")
    ap.add_argument("--no-c3", action="store_true",
                    help="skip the uneven-batch measurement (200 batches of 1-4096 frames, two frame sizes)")
    ap.add_argument("--largefield-only", action="store_true",
                    help="run only the large-field measurement and print its JSON (for profiling)")
    ap.add_argument("--largefield-frames", type=int, default=256,
                    help="frames per batch of the large-field measurement")
    ap.add_argument("--no-largefield", action="store_true",
                    help="skip the large-field measurement (2048x2048 frames, 512x512 fields, 465 modes)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_config(mode, frames, workload=WORKLOAD):
    """Hologram parameters (beam centres, tilts, window radius) and the matching digHolo configuration."""
    from digholo_b200 import synth
    kw = dict(synth.WORKLOADS[workload])
    kw["frame_count"] = 1
    hol = synth.generate(**kw)

    class Cfg:
        pass
    c = Cfg()
    c.frame_width, c.frame_height = hol.frame_width, hol.frame_height
    c.pixel_size, c.wavelength = hol.pixel_size, hol.wavelength
    c.pol_count = hol.pol_count
    c.fft_window = hol.window
    c.window_radius_deg = hol.radius_deg
    c.resolution_mode = mode
    c.max_mg = hol.max_mg
    c.fill_factor = 1
    c.pol_lock_tilt = 0
    c.pol_lock_defocus = 0
    c.pol_lock_waist = 1
    c.waist = [hol.waist, hol.waist]
    c.beam_centre = hol.beam_centres
    c.tilt_deg = hol.tilts_deg
    c.defocus = [0.0, 0.0]
    c.snr_db = synth.WORKLOADS[workload]["snr_db"]
    c.taper = bool(synth.WORKLOADS[workload].get("taper", False))
    c.frames = frames
    return c


def torch_frames(cfg, n, seed, device):
    """The synth.py hologram model evaluated on the GPU (uint16 values stored as int16)."""
    import torch
    from digholo_b200 import synth
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    W, H, P, G = cfg.frame_width, cfg.frame_height, cfg.pol_count, cfg.max_mg
    p = cfg.pixel_size
    ms, ns = synth.hg_indices(G)
    M = len(ms)
    region = W // P
    xs = (torch.arange(W, device=device, dtype=torch.float64) - W // 2) * p
    ys = (torch.arange(H, device=device, dtype=torch.float64) - H // 2) * p
    nyq = math.pi / p
    clean = torch.empty((n, H, W), device=device, dtype=torch.float32)
    for pol in range(P):
        xr = xs[pol * region:(pol + 1) * region]
        cx, cy = cfg.beam_centre[pol]
        hx = torch.tensor(synth.hg_modes_1d((xr - cx).cpu().numpy(), cfg.waist[0], G), device=device, dtype=torch.float32)
        hy = torch.tensor(synth.hg_modes_1d((ys - cy).cpu().numpy(), cfg.waist[0], G), device=device, dtype=torch.float32)
        sgn = 1.0 if pol == 0 else -1.0
        kx, ky = sgn * 0.25 * nyq, sgn * 0.2 * nyq
        ref = (torch.exp(1j * ky * ys)[:, None] * torch.exp(1j * kx * xr)[None, :]).to(torch.complex64)
        for f0 in range(0, n, 128):
            f1 = min(n, f0 + 128)
            c = torch.complex(torch.randn((f1 - f0, M), generator=g, device=device),
                              torch.randn((f1 - f0, M), generator=g, device=device)) / math.sqrt(2)
            if getattr(cfg, "taper", False):
                c = c / (torch.as_tensor(ms + ns, device=device, dtype=torch.float32) + 1.0)
            cm = torch.zeros((f1 - f0, G, G), device=device, dtype=torch.complex64)
            cm[:, torch.as_tensor(ms, device=device), torch.as_tensor(ns, device=device)] = c
            s = torch.einsum("fmn,ny,mx->fyx", cm, hy.to(torch.complex64), hx.to(torch.complex64))
            pw = (s.abs() ** 2).sum(dim=(1, 2), keepdim=True)
            s = s * torch.sqrt(0.1 * ref.numel() / pw)
            clean[f0:f1, :, pol * region:(pol + 1) * region] = (ref[None] + s).abs() ** 2
    sigma = clean.mean() * 10.0 ** (-cfg.snr_db / 20.0)
    clean += torch.randn(clean.shape, generator=g, device=device) * sigma
    scale = 4095.0 / clean.max()
    return torch.clamp(torch.round(clean * scale), 0, 4095).to(torch.int16)


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for i, name in enumerate(names):
                if r[5 + i].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def max_over_ranks(ms, device=None):
    """Slowest rank's elapsed time (ms); the identity without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_seed(rank, batch_index):
    """Seed of a rank's synthetic batch: every rank processes its own frames (weak scaling)."""
    return 1000 + 17 * rank + batch_index


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel, mode):
    """dram bytes per launch of ``kernel`` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "ncu_%s_%s_mode%d.md" % (kernel, WORKLOAD, mode))
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def reference_run(cfg, frames_host, seconds, threads):
    """Time the reference's digHoloProcessBatch on host frames; returns frames/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes as C
    import ref_lib
    L = ref_lib.load()
    # one handle per process: the reference crashes when a handle is created
    # after another was destroyed (seen in its uint16 conversion), so handles
    # are never destroyed here
    h = L.digHoloCreate()
    ref_lib.configure(L, h, cfg)
    L.digHoloConfigSetThreadCount(h, threads)
    n = frames_host.shape[0]
    L.digHoloSetBatchUint16(h, n, ref_lib.ptr(frames_host, C.c_ushort), 0)
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    calls = 0
    t0 = time.perf_counter()
    while True:
        L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
        calls += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return n * calls / el, calls, el


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import numpy as np
    from digholo_b200 import synth
    cfg = workload_config(args.mode, args.frames)
    # the whole batch of the GPU arm's step (about 0.2 s per step on 16 host cores)
    sample = args.frames
    kw = dict(synth.WORKLOADS[WORKLOAD])
    kw["frame_count"] = sample
    frames = np.ascontiguousarray(synth.generate(**kw).frames)
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes as C
    import ref_lib
    if not ref_lib.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libdigholo_ref.so missing"}))
        return 0
    L = ref_lib.load()
    h = L.digHoloCreate()
    ref_lib.configure(L, h, cfg)
    L.digHoloConfigSetThreadCount(h, threads)
    L.digHoloSetBatchUint16(h, sample, ref_lib.ptr(frames, C.c_ushort), 0)
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    for _ in range(args.warmup):
        L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    el = time.perf_counter() - t0
    fps = sample * args.steps / el
    line = {
        "impl": "reference", "metric": "frames/s (FFT->window->IFFT->tilt->HG overlap)", "value": fps,
        "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded hologram model, numpy)",
        "config": {"workload": WORKLOAD + "_mode%d" % args.mode, "frames_per_step": sample,
                   "frame": "640x512 uint16", "pol": 2, "maxMG": 15, "fft_window": "128x128",
                   "ifft_resolution_mode": args.mode},
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": threads, "kind": "reference",
                         "sample": "the full %d-frame batch per step, as the GPU arm's step; reference "
                                   "digHolo.cpp compiled here with this project's FFT library standing in for FFTW"
                                   % sample},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    import ctypes as C

    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import digholo_b200
    L = digholo_b200.load()
    if args.largefield_only:
        stream = torch.cuda.Stream(device)
        torch.cuda.set_stream(stream)
        print(json.dumps(largefield_leg(L, torch, device, stream, True, args.largefield_frames)))
        return 0
    cfg = workload_config(args.mode, args.frames)
    B = args.frames
    P, W, H = cfg.pol_count, cfg.fft_window[0], cfg.fft_window[1]
    G = cfg.max_mg
    M = G * (G + 1) // 2

    # four device-resident batches (rotated: their windows exceed L2)
    batches = [torch_frames(cfg, B, shard_seed(rank, i), device) for i in range(4)]
    torch.cuda.synchronize()
    # a dedicated (non-default) stream shared by the library and the timing events
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0

    h = L.digHoloCreate()
    from digholo_b200 import api
    api.configure(L, h, cfg)
    L.digHoloB200SetStream(h, C.c_void_p(stream.cuda_stream))
    L.digHoloB200SetOverlapKernel(h, 0 if args.overlap == "tc" else 1)
    L.digHoloB200SetInverseKernel(h, args.inverse_kernel)

    def step_device(i):
        t = batches[i % 4]
        L.digHoloSetBatchUint16(h, B, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_ushort)), 0)
        rc = L.digHoloB200ProcessBatchDevice(h)
        if rc != 0:
            raise RuntimeError("ProcessBatchDevice failed: %s" % L.digHoloB200GetLastError(h))

    # warm-up: at least one pass over the four batch buffers and one more
    # step, so that the library's CUDA graph of each buffer (captured on its
    # first use once the launches are settled) exists before the timed steps
    warmup = max(args.warmup, len(batches) + 1)
    for i in range(warmup):
        step_device(i)
    torch.cuda.synchronize()
    st = (C.c_float * 3)()
    L.digHoloB200GetStageTimes(h, st)  # reset

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(args.steps):
        step_device(i)
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    # per-stage kernel times: the same steps again with the library's stage
    # events on (events between the kernels, so kept out of the timed loop)
    L.digHoloB200SetTiming(h, 1)
    for i in range(args.steps):
        step_device(i)
    torch.cuda.synchronize()
    L.digHoloB200GetStageTimes(h, st)
    L.digHoloB200SetTiming(h, 0)
    fwd_ms, inv_ms, timed = st[0], st[1], st[2]

    elapsed_ms = max_over_ranks(elapsed_ms, device)
    value = world * B * args.steps / (elapsed_ms / 1e3)

    # end to end through the C ABI with pinned host frames
    host = torch.empty((B, H_FRAME(cfg), W_FRAME(cfg)), dtype=torch.int16, pin_memory=True)
    host.copy_(batches[0].cpu())
    e2e_steps = max(3, min(args.steps, 10))
    hp = C.cast(C.c_void_p(host.data_ptr()), C.POINTER(C.c_ushort))
    b, m, pc = C.c_int(), C.c_int(), C.c_int()
    L.digHoloB200SetTiming(h, 0)
    for _ in range(2):
        L.digHoloSetBatchUint16(h, B, hp, 0)
        L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        L.digHoloSetBatchUint16(h, B, hp, 0)
        ptr = L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(pc))
        if not ptr:
            raise RuntimeError("ProcessBatch failed: %s" % L.digHoloB200GetLastError(h))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(e2e_ms, device)
    e2e = world * B * e2e_steps / (e2e_ms / 1e3)
    h2d = B * P * W * H * 2
    d2h = B * P * M * 8

    if rank != 0:
        L.digHoloDestroy(h)
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    # kernels per step: forward + inverse, plus the separate FP32 overlap
    # kernel for full-resolution fields when that path is chosen
    per_step = 2 + (1 if (L.digHoloB200GetInverseKernel(h) == 3 and L.digHoloB200GetOverlapKernel(h) == 1) else 0)
    overlap_name = {1: "fp32 cuda cores", 2: "split-bf16 tensor cores"}.get(L.digHoloB200GetOverlapKernel(h), "?")

    # roofline of the dominant kernel (HBM bytes it must move per launch)
    peak, peak_kind = measured_peaks()
    geo = (C.c_int * 10)()
    L.digHoloB200GetGeometry(h, geo)
    w, hh, nx, ny = geo[2], geo[3], geo[4], geo[5]
    fwd_bytes = B * (P * W * H * 2 + P * w * hh * 8)
    inv_bytes = B * (P * w * hh * 8 + P * nx * ny * 4 + P * M * 8 + 7 * P * 4)
    fwd_name = {1: "k_forward", 2: "k_forward_reg", 3: "k_forward_tma", 4: "k_forward_i8"}.get(
        L.digHoloB200GetForwardKernel(h), "k_forward")
    inv_name = {1: "k_inverse", 2: "k_inverse_lo16q" if w == 16 else "k_inverse_lo", 3: "k_field_full",
                4: "k_field_big"}.get(L.digHoloB200GetInverseKernel(h), "k_inverse")
    if fwd_ms >= inv_ms:
        kname, kbytes, kms = fwd_name, fwd_bytes, fwd_ms / max(timed, 1)
    else:
        kname, kbytes, kms = inv_name, inv_bytes, inv_ms / max(timed, 1)
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = profile_traffic(kname, args.mode)

    cpu = None
    if not args.no_cpu_baseline:
        sample = np.ascontiguousarray(host.numpy().view(np.uint16))
        threads = os.cpu_count() or 1
        try:
            fps, calls, el = reference_run(cfg, sample, 12.0, threads)
            cpu = {"value": fps, "unit": "frames/s", "cores": threads, "kind": "reference",
                   "sample": "the full %d-frame batch, digHoloProcessBatch repeated for %.1f s (%d calls); "
                             "reference compiled from its sources, FFT by this project's library (not FFTW)"
                             % (B, el, calls)}
        except Exception as exc:  # the reference build may be absent on a box
            cpu = {"value": None, "unit": "frames/s", "cores": 0, "kind": "reference",
                   "sample": "unavailable: %s" % exc}

    large = None
    if not args.no_largefield:
        try:
            large = largefield_leg(L, torch, device, stream, args.no_cpu_baseline)
        except Exception as exc:
            large = {"unavailable": str(exc)}

    c3 = None
    if not args.no_c3:
        try:
            c3 = c3_leg(L, torch, device, stream)
        except Exception as exc:
            c3 = {"unavailable": str(exc)}

    align = None
    if not args.no_autoalign:
        try:
            align = autoalign_leg(L, torch, device)
        except Exception as exc:
            align = {"unavailable": str(exc)}

    line = {
        "metric": "frames/s (FFT->window->IFFT->tilt->HG overlap)",
        "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": warmup,
        "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded hologram model, generated on the GPU)",
        "config": {"workload": WORKLOAD + "_mode%d" % args.mode, "frames_per_step": B,
                   "frame": "640x512 uint16", "pol": P, "maxMG": G, "modes": M, "fft_window": "%dx%d" % (W, H),
                   "ifft_resolution_mode": args.mode, "overlap": overlap_name,
                   "launch": "one CUDA graph per batch buffer, replayed by the library (%d held)"
                             % L.digHoloB200GetGraphCount(h),
                   "parallelism": "dp%d (independent frames)" % world,
                   "l2": "4 rotating device batches; their window pixels (268 MB) exceed the 126 MB L2"},
        "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / e2e_steps, "steps": e2e_steps},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": kbytes, "avg_launch_ms": kms,
                     "stage_ms_per_step": {"k_forward": fwd_ms / max(timed, 1), "k_inverse": inv_ms / max(timed, 1)}},
        "gpu_launches": per_step * args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "autoalign": align,
        "largefield": large,
        "uneven_batches": c3,
    }
    print(json.dumps(line))
    L.digHoloDestroy(h)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def largefield_leg(L, torch, device, stream, no_cpu, frames=256):
    """frames/s on the large-field workload: 256 frames of 2048x2048 uint16,
    two polarisations, FFT window 512x512, full resolution (IFFT mode 0,
    the reference's default: 512x512 fields by the band kernels), maxMG 30
    (465 modes), waist 600 um, 20 dB SNR, 1/(group+1) coefficient taper; the
    overlap in split-BF16 on the tensor cores and in FP32 on the CUDA cores.
    Two device-resident batches (2.1 GB each, beyond L2) alternate; CUDA
    events on the library's stream; 3 warm-up and 5 timed batches each."""
    import ctypes as C
    import numpy as np
    from digholo_b200 import api
    B, steps, warmup = frames, 5, 3
    cfg = workload_config(0, B, "largefield_2048_u16_2pol")
    batches = [torch_frames(cfg, B, 5000 + i, device) for i in range(2)]
    torch.cuda.synchronize()
    out = {"metric": "frames/s (FFT->window->IFFT->tilt->HG overlap), device-resident frames",
           "workload": "largefield_2048_u16_2pol_mode0: %d frames 2048x2048 uint16, 2 pol, window 512x512, "
                       "maxMG 30 (465 modes)" % B, "steps": steps, "warmup": warmup}
    for name, ov in (("split_bf16", 0), ("fp32", 1)):
        h = L.digHoloCreate()
        api.configure(L, h, cfg)
        L.digHoloB200SetStream(h, C.c_void_p(stream.cuda_stream))
        L.digHoloB200SetTiming(h, 1)
        L.digHoloB200SetOverlapKernel(h, ov)

        def step(i):
            t = batches[i % 2]
            L.digHoloSetBatchUint16(h, B, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_ushort)), 0)
            if L.digHoloB200ProcessBatchDevice(h) != 0:
                raise RuntimeError("ProcessBatchDevice failed: %s" % L.digHoloB200GetLastError(h))
        for i in range(warmup):
            step(i)
        torch.cuda.synchronize()
        st = (C.c_float * 3)()
        L.digHoloB200GetStageTimes(h, st)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(steps):
            step(i)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        L.digHoloB200GetStageTimes(h, st)
        n = max(st[2], 1.0)
        out[name] = {"value": B * steps / (ms / 1e3), "unit": "frames/s", "ms_per_step": ms / steps,
                     "stage_ms_per_step": {"forward": st[0] / n, "inverse": st[1] / n},
                     "inverse_kernel": L.digHoloB200GetInverseKernel(h),
                     "overlap_kernel": L.digHoloB200GetOverlapKernel(h)}
        L.digHoloDestroy(h)
    if not no_cpu:
        try:
            sample = np.ascontiguousarray(batches[0][:4].cpu().numpy().view(np.uint16))
            threads = os.cpu_count() or 1
            fps, calls, el = reference_run(cfg, sample, 8.0, threads)
            out["cpu_baseline"] = {"value": fps, "unit": "frames/s", "cores": threads, "kind": "reference",
                                   "sample": "4 of the %d frames, digHoloProcessBatch repeated for %.1f s (%d calls)"
                                             % (B, el, calls)}
        except Exception as exc:
            out["cpu_baseline"] = {"value": None, "sample": "unavailable: %s" % exc}
    del batches
    torch.cuda.empty_cache()
    return out


def c3_leg(L, torch, device, stream):
    """Uneven streamed batches: 200 batches, frame counts log-uniform in
    [1, 4096], frames 320x256 or 1280x1024 float32 (two polarisations, 12-bit
    values of the synth.py hologram model, carrier (0.25, 0.2) Nyquist),
    maxMG from {6, 9, 15}, FFT windows from {64, 128, 256} (1280x1024) or
    {32, 64} (320x256: a 16-pixel window is smaller than the Fourier window
    of this carrier), low-resolution fields.  The frames come from two
    device-resident pools of 4096 frames (21.5 GB and 1.3 GB); batch k uses
    the first n_k frames of its pool.  The sequence runs with the built-in
    kernel choice (FFTW plan mode ESTIMATE) and with tuned kernel plans
    (MEASURE; an untimed pass plans every shape first); CUDA events on the
    handles' stream around the whole sequence; each mode's handles run the
    sequence once untimed first (buffers grown, shapes planned)."""
    import ctypes as C
    import numpy as np
    from digholo_b200 import api, synth
    rng = np.random.default_rng(3003)
    pools, cfgs = {}, {}
    for fw, fh in ((320, 256), (1280, 1024)):
        hol = synth.generate(frame_count=1, frame_width=fw, frame_height=fh, pol_count=2, max_mg=9, waist=fw * 0.4e-6,
                             snr_db=30, window=(fw // 5, fw // 5), dtype="float32", seed=3004)

        class G:
            pass
        g = G()
        g.frame_width, g.frame_height, g.pol_count, g.max_mg = fw, fh, 2, 9
        g.pixel_size, g.beam_centre, g.waist = hol.pixel_size, hol.beam_centres, [hol.waist] * 2
        g.snr_db, g.taper = 30, False
        pools[fw] = torch_frames(g, 4096, 3005 + fw, device).float()
        cfgs[fw] = hol
    torch.cuda.synchronize()
    batches = []
    for k in range(200):
        fw = 1280 if rng.random() < 0.5 else 320
        n = int(min(4096, max(1, round(float(np.exp(rng.uniform(0.0, np.log(4096))))))))
        mg = int(rng.choice([6, 9, 15]))
        win = int(rng.choice([64, 128, 256] if fw == 1280 else [32, 64]))
        batches.append((fw, n, mg, win))
    total = sum(b[1] for b in batches)

    def configure(h, fw, mg, win):
        hol = cfgs[fw]
        L.digHoloConfigSetFrameDimensions(h, fw, 1024 if fw == 1280 else 256)
        L.digHoloConfigSetFramePixelSize(h, float(hol.pixel_size))
        L.digHoloConfigSetWavelengthCentre(h, float(hol.wavelength))
        L.digHoloConfigSetPolCount(h, 2)
        L.digHoloConfigSetfftWindowSize(h, win, win)
        L.digHoloConfigSetFourierWindowRadius(h, float(hol.radius_deg))
        L.digHoloConfigSetIFFTResolutionMode(h, 1)
        L.digHoloConfigSetBasisGroupCount(h, mg)
        for p in range(2):
            L.digHoloConfigSetBasisWaist(h, p, float(win * 2.5e-6))
            L.digHoloConfigSetBeamCentre(h, 0, p, float(hol.beam_centres[p][0]))
            L.digHoloConfigSetBeamCentre(h, 1, p, float(hol.beam_centres[p][1]))
            L.digHoloConfigSetTilt(h, 0, p, float(hol.tilts_deg[p][0]))
            L.digHoloConfigSetTilt(h, 1, p, float(hol.tilts_deg[p][1]))

    def make(plan):
        hs = {fw: L.digHoloCreate() for fw in pools}
        for h in hs.values():
            L.digHoloB200SetStream(h, C.c_void_p(stream.cuda_stream))
            L.digHoloConfigSetFFTWPlanMode(h, plan)
        return hs

    def run(hs):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for fw, n, mg, win in batches:
            h = hs[fw]
            configure(h, fw, mg, win)
            L.digHoloSetBatch(h, n, C.cast(C.c_void_p(pools[fw].data_ptr()), C.POINTER(C.c_float)))
            if L.digHoloB200ProcessBatchDevice(h) != 0:
                raise RuntimeError("C3 batch failed: %s" % L.digHoloB200GetLastError(h))
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)
    # each plan mode on its own two handles: an untimed pass grows their
    # buffers to the sequence's largest batches (and with plans, tunes every
    # shape), then the timed pass runs the same sequence on them
    hd = make(0)
    run(hd)
    ms_default = run(hd)
    runs0 = L.digHoloB200GetKernelPlanRuns()
    hp = make(1)
    run(hp)
    plans = L.digHoloB200GetKernelPlanRuns() - runs0
    ms_planned = run(hp)
    for h in list(hd.values()) + list(hp.values()):
        L.digHoloDestroy(h)
    out = {"metric": "frames/s over the whole sequence, device-resident frames",
           "batches": len(batches), "frames": total, "shapes_planned": plans,
           "default": {"ms": ms_default, "value": total / (ms_default / 1e3), "unit": "frames/s"},
           "planned": {"ms": ms_planned, "value": total / (ms_planned / 1e3), "unit": "frames/s"},
           "planned_over_default": ms_default / ms_planned}
    del pools
    torch.cuda.empty_cache()
    return out


def autoalign_leg(L, torch, device):
    """ms per AutoAlign, plain coordinate search (digHoloAutoAlign, TWEAK) vs
    the adjoint-driven search (digHoloB200AutoAlignAdjoint), goal IL and goal
    MDL, on 512 frames of 640x512 float32, two polarisations, each frame one
    column of a Haar-random 240x240 transfer matrix over both polarisations'
    120 modes with 0-1 dB per-mode loss, full resolution (IFFT mode 0).  The
    start is off the true alignment by seeded uniform draws: beam centre
    +-60 um, tilt +-5 % of the Nyquist angle, defocus +-0.5, waist +-15 %.
    Frames are device resident; each search runs twice on its handle and
    the second is timed."""
    import ctypes as C
    import numpy as np
    from digholo_b200 import api, synth
    kw = dict(synth.WORKLOADS["align_640x512_f32_2pol"])
    B = kw["frame_count"]
    kw["coefs"] = synth.transfer_coefs(B, 2, kw["max_mg"], 1004)
    hol = synth.generate(**kw)
    frames = torch.from_numpy(np.ascontiguousarray(hol.frames)).to(device)
    rng = np.random.default_rng(4004)
    dtilt = synth.carrier_to_tilt_degrees(0.05)

    class Cfg:
        pass
    cfg = Cfg()
    cfg.frame_width, cfg.frame_height = hol.frame_width, hol.frame_height
    cfg.pixel_size, cfg.wavelength = hol.pixel_size, hol.wavelength
    cfg.pol_count, cfg.fft_window, cfg.window_radius_deg = 2, hol.window, hol.radius_deg
    cfg.resolution_mode, cfg.max_mg, cfg.fill_factor = 0, hol.max_mg, 1
    cfg.pol_lock_tilt, cfg.pol_lock_defocus, cfg.pol_lock_waist = 0, 0, 1
    cfg.beam_centre = [[bc[0] + rng.uniform(-60e-6, 60e-6), bc[1] + rng.uniform(-60e-6, 60e-6)]
                       for bc in hol.beam_centres]
    cfg.tilt_deg = [[t[0] + rng.uniform(-dtilt, dtilt), t[1] + rng.uniform(-dtilt, dtilt)] for t in hol.tilts_deg]
    cfg.defocus = [rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5)]
    cfg.waist = [hol.waist * (1.0 + rng.uniform(-0.15, 0.15))] * 2
    out = {"metric": "ms per AutoAlign, host wall clock around the call",
           "workload": "align_640x512_f32_2pol_mode0: 512 frames, carrier (0.55, 0.45) of Nyquist (the Fourier window "
                       "holds all 120 modes per polarisation), Haar 240x240 transfer over both polarisations, "
                       "perturbed start (centre +-60 um, tilt +-5% Nyquist, defocus +-0.5, waist +-15%)"}
    for goal, gname in ((0, "goal_il"), (1, "goal_mdl")):
        res = {}
        for name in ("plain", "adjoint"):
            h = L.digHoloCreate()
            ms = None
            for run in range(2):
                api.configure(L, h, cfg)
                L.digHoloSetBatch(h, B, C.cast(C.c_void_p(frames.data_ptr()), C.POINTER(C.c_float)))
                b, m, p = C.c_int(), C.c_int(), C.c_int()
                L.digHoloProcessBatch(h, C.byref(b), C.byref(m), C.byref(p))
                L.digHoloConfigSetAutoAlignMode(h, 1)
                L.digHoloConfigSetAutoAlignGoalIdx(h, goal)
                L.digHoloConfigSetAutoAlignTol(h, 0.01)
                L.digHoloConfigSetAutoAlignFourierWindowRadius(h, 0)
                L.digHoloB200Synchronize(h)
                t = time.perf_counter()
                if name == "plain":
                    L.digHoloAutoAlign(h)
                else:
                    L.digHoloB200AutoAlignAdjoint(h)
                L.digHoloB200Synchronize(h)
                ms = (time.perf_counter() - t) * 1e3
            res[name] = {"ms": ms, "il_db": L.digHoloAutoAlignGetMetric(h, 0),
                         "mdl_db": L.digHoloAutoAlignGetMetric(h, 1),
                         "evaluations": L.digHoloB200GetAutoAlignEvaluations(h)}
            L.digHoloDestroy(h)
        key = "il_db" if goal == 0 else "mdl_db"
        res["adjoint_over_plain"] = res["adjoint"]["ms"] / res["plain"]["ms"]
        res["goal_delta_db"] = res["adjoint"][key] - res["plain"][key]
        out[gname] = res
    return out


def H_FRAME(cfg):
    return cfg.frame_height


def W_FRAME(cfg):
    return cfg.frame_width


if __name__ == "__main__":
    sys.exit(main())
