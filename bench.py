"""Develop throughput benchmark (MP/s) on B200.

Workload: the 51 MP Bayer develop -- an 8736x5856 RGGB float32 mosaic of the
seeded fringed scene, AMaZE -> defringe(10, 0.1, 0.15, 10, green off) ->
axial CA guided filter (r=6, eps=1e-4, strength 0.3) -> ACES tone map
(after_scale 1.0), float32 RGB out.  A step develops one image per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs (torchrun, one process per GPU) are independent replicas:
every rank develops its own image, no data-path collective; the timed region
is bracketed by a barrier and the time is the max over ranks.

Reported (one JSON line from rank 0):
  value  -- MP/s with the mosaic resident in HBM (lre_dev_develop); the
            mosaic (205 MB) and RGB (614 MB) exceed L2, so no flush is needed;
  e2e    -- MP/s through the C ABI with pinned host buffers (lre_develop):
            H2D of the mosaic and D2H of the RGB inside every step;
  roofline -- the dominant stage (largest device time) against the measured
            HBM copy bandwidth, from its algorithmic bytes per pixel;
  cpu_baseline -- the reference's own CPU accelerator (oracle/_ref) on this
            host's cores: the same chain on the same 8736x5856 mosaic,
            a bounded number of develops.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

H, W = 5856, 8736
SEED = 2
WB = (2.0, 1.0, 1.5, 1.0)
METRIC = "develop MP/s on 1 B200 (51 MP Bayer: AMaZE->defringe->axial CA->tone map)"
# algorithmic bytes per output pixel of each stage (float32 RGB = 12 B/px)
STAGE_BYTES = {"amaze": 16.0, "defringe": 24.0, "axial": 24.0, "tone": 24.0}
# From one ncu capture of k_amaze at 4096x3072: DRAM read+write bytes and
# executed warp-instructions per output pixel.
AMAZE_DRAM_BYTES_PER_PX = (124.060416e6 + 909.380352e6) / (4096 * 3072)
AMAZE_WARP_INST_PER_PX = 925190063 / (4096 * 3072)
# issue roofline: 148 SMs x 4 schedulers x 1.965 GHz, one warp-instruction per cycle each
ISSUE_PEAK_G = 148 * 4 * 1.965


def workload_config(world=1):
    """The `config` object both arms print (same workload, same sizes)."""
    return {
        "workload": "51 MP Bayer develop: AMaZE -> defringe(r10,s10) -> axial CA(r6) -> ACES(1.0), f32 RGB out",
        "width": W,
        "height": H,
        "parallelism": f"replicas x{world}",
        "l2": "inputs 205 MB mosaic + 614 MB RGB exceed the 126 MB L2 (no flush needed)",
    }


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_mosaic():
    import numpy as np

    from libraw_enhanced_b200 import scenes

    if (H, W) != (5856, 8736):  # a reduced case (profiling): generate, no cache
        return scenes.bayer_51mp_fringed(SEED, H, W)
    cache = os.path.join(tempfile.gettempdir(), f"lre_bench_51mp_seed{SEED}.npy")
    if os.path.exists(cache):
        try:
            m = np.load(cache)
            if m.shape == (H, W):
                return m
        except Exception:
            pass
    m = scenes.bayer_51mp_fringed(SEED, H, W)
    try:
        np.save(cache, m)
    except Exception:
        pass
    return m


class ClockSampler:
    """SM clock and throttle-reason sampling during the timed region.

    Reads NVML every 20 ms (read-only queries); falls back to polling
    nvidia-smi when NVML is unavailable."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index, period=0.02):
        self.index = index
        self.period = period
        self.samples = []  # (sm_mhz, max_mhz, {reason names})
        self._stop = threading.Event()
        self._t = None

    def _run_nvml(self):
        import pynvml as nv

        nv.nvmlInit()
        try:
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while not self._stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), {n for n, b in zip(self.NAMES, bits) if rs & b}))
                self._stop.wait(self.period)
        finally:
            nv.nvmlShutdown()

    def _run_smi(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5,
                ).stdout.strip()
                s = [x.strip() for x in out.split(",")]
                if len(s) >= 6 and s[0].replace(".", "").isdigit():
                    self.samples.append((float(s[0]), float(s[1]),
                                         {n for i, n in enumerate(self.NAMES) if s[2 + i].lower() == "active"}))
            except Exception:
                pass
            self._stop.wait(0.2)

    def _run(self):
        try:
            self._run_nvml()
        except Exception:
            self._run_smi()

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        time.sleep(0.05)
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        import statistics

        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {
            "sm_mhz": statistics.median(s[0] for s in self.samples),
            "sm_max_mhz": max(s[1] for s in self.samples),
            "reasons": sorted(set().union(*(s[2] for s in self.samples))),
            "samples": len(self.samples),
        }


def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reference_chain(mosaic, threads):
    """One develop of `mosaic` by the reference's own CPU accelerator
    (oracle/_ref): AMaZE -> defringe -> axial CA -> ACES, the GPU arm's chain
    and parameters."""
    import oracle
    from libraw_enhanced_b200 import scenes

    oracle.set_threads(threads)
    sp = scenes.sparse_rgb(mosaic, "RGGB")
    x = oracle.amaze(sp, scenes.FILTERS["RGGB"], WB, 1.0)
    del sp
    x = oracle.defringe(x, 10.0, 0.1, 0.15, 10.0, False, 0.3)
    x = oracle.axial_ca(x, 6, 1e-4, 0.3)
    return oracle.tone_mapping(x, 1.0)


def cpu_baseline(mosaic, develops=2, threads=None):
    """The reference CPU accelerator on the bench's own 8736x5856 mosaic:
    one untimed develop, then `develops` timed ones (about 8 s each on 16
    cores)."""
    threads = threads or os.cpu_count() or 1
    reference_chain(mosaic, threads)  # warm-up
    t0 = time.perf_counter()
    for _ in range(develops):
        reference_chain(mosaic, threads)
    dt = time.perf_counter() - t0
    mp = mosaic.shape[0] * mosaic.shape[1] / 1e6
    return {
        "value": round(develops * mp / dt, 3),
        "unit": "MP/s",
        "cores": threads,
        "kind": "reference",
        "sample": f"{develops} develops of the full {mosaic.shape[1]}x{mosaic.shape[0]} bench mosaic "
                  f"(AMaZE->defringe->axial->ACES), reference CPUAccelerator, {threads} OpenMP threads",
    }


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/liblre_ref.so not built"}))
        return 0
    threads = os.cpu_count() or 1
    mosaic = make_mosaic()  # the GPU arm's input, generated outside the timed region
    for _ in range(args.warmup):
        reference_chain(mosaic, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        reference_chain(mosaic, threads)
    dt = time.perf_counter() - t0
    mp = H * W / 1e6 * args.steps
    v = mp / dt
    line = {
        "metric": METRIC,
        "value": round(v, 3),
        "unit": "MP/s",
        "impl": "reference",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": f"synthetic (seeded fringed scene, {W}x{H} RGGB)",
        "config": workload_config(args.gpus),
        "cpu_baseline": {"value": round(v, 3), "unit": "MP/s", "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} develops of the full {W}x{H} mosaic, host buffers, "
                                   f"{threads} OpenMP threads"},
        "e2e": {"value": round(v, 3), "unit": "MP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import numpy as np
    import torch

    import libraw_enhanced_b200 as lre

    world, rank, local = dist_setup(args.gpus)
    acc = lre.CudaAccelerator(local)
    # a dedicated stream: the library enqueues on it and the CUDA events are
    # recorded on it (the legacy default stream has handle 0, which the C ABI
    # reads as "use your own stream")
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    acc.set_stream(stream.cuda_stream)
    mosaic = make_mosaic()
    mp = H * W / 1e6
    params = lre.develop_params(cfa="RGGB", cam_mul=WB, defringe=1, axial_ca_correction=1, tone_mapping=1,
                                tone_after_scale=1.0, stage_order=1)

    d_mos = torch.from_numpy(mosaic).to(f"cuda:{local}")
    d_out = torch.empty((H, W, 3), dtype=torch.float32, device=f"cuda:{local}")
    d_tmp = torch.empty((H, W, 3), dtype=torch.float32, device=f"cuda:{local}")

    # ---------------- device-resident develop (value)
    for _ in range(args.warmup):
        acc.dev_develop(d_mos, d_out, W, H, params)
    torch.cuda.synchronize()
    barrier(world)
    n0 = acc.launch_count
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            acc.dev_develop(d_mos, d_out, W, H, params)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = acc.launch_count - n0
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms, world)
    barrier(world)
    value = world * mp / (ms / 1e3)

    # ---------------- per-stage device times (roofline of the dominant stage)
    stage_ms = {}
    if rank == 0:
        def timed(fn, reps=3):
            fn()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        stage_ms["amaze"] = timed(lambda: acc.dev_demosaic_bayer_amaze(d_mos, d_tmp, W, H, scenes_filters(), WB, 1.0))
        stage_ms["defringe"] = timed(lambda: acc.dev_defringe(d_tmp, d_out, W, H))
        stage_ms["axial"] = timed(lambda: acc.dev_ca_axial_cleanup(d_tmp, d_out, W, H, 6, 1e-4, 0.3))
        stage_ms["tone"] = timed(lambda: acc.dev_tone_mapping(d_tmp, d_out, W, H, 1.0))
    barrier(world)

    # ---------------- end to end through the C ABI with pinned host buffers
    e2e, e_ms = None, None
    e2p, ep_ms = None, None
    e2s, es_ms, es_lanes = None, None, None
    if not args.no_e2e:
        e2e, e_ms = run_e2e(acc, mosaic, params, args, world, mp)
        e2p, ep_ms = run_e2e(acc, mosaic, params, args, world, mp, pinned=False)
        e2s, es_ms, es_lanes = run_e2e_served(mosaic, params, args, world, mp, local)
    barrier(world)

    if rank == 0:
        peak, peak_kind = load_peaks()
        # dominant single kernel: k_amaze (the AMaZE stage is that kernel
        # plus a 10 us border fill)
        amaze_ms = stage_ms["amaze"]
        px = H * W
        achieved = STAGE_BYTES["amaze"] * px / (amaze_ms / 1e3) / 1e9
        warp_inst = AMAZE_WARP_INST_PER_PX * px / (amaze_ms / 1e3)
        roof = {
            "bound": "hbm",
            "kernel": "k_amaze",
            "achieved": round(achieved, 1),
            "peak": peak,
            "peak_kind": peak_kind,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": int(AMAZE_DRAM_BYTES_PER_PX * px),
            "traffic_source": "ncu dram__bytes_read+write of k_amaze at 4096x3072, scaled by pixel count",
            "algorithmic_bytes_per_px": STAGE_BYTES["amaze"],
            "issue": {
                "bound": "issue",
                "achieved": round(warp_inst / 1e9, 1),
                "peak": ISSUE_PEAK_G,
                "unit": "G warp-inst/s",
                "frac": round(warp_inst / 1e9 / ISSUE_PEAK_G, 4),
            },
            "stage_ms": {k: round(v, 3) for k, v in stage_ms.items()},
        }
        line = {
            "metric": METRIC,
            "value": round(value, 2),
            "unit": "MP/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": f"synthetic (seeded fringed scene, {W}x{H} RGGB)",
            "config": workload_config(world),
            "e2e": None if e2e is None else {
                "value": round(e2e, 2), "unit": "MP/s", "ms_per_step": round(e_ms, 3),
                "h2d_bytes_per_step": H * W * 4, "d2h_bytes_per_step": H * W * 12},
            "e2e_pageable": None if e2p is None else {
                "value": round(e2p, 2), "unit": "MP/s", "ms_per_step": round(ep_ms, 3),
                "h2d_bytes_per_step": H * W * 4, "d2h_bytes_per_step": H * W * 12,
                "how": "same call with ordinary (pageable) numpy buffers in and out, as the drop-in caller's "
                       "std::vector-backed ImageBufferFloat passes them"},
            "e2e_served": None if e2s is None else {
                "value": round(e2s, 2), "unit": "MP/s", "ms_per_request": round(es_ms, 3),
                "h2d_bytes_per_step": H * W * 4, "d2h_bytes_per_step": H * W * 12, "lanes": es_lanes,
                "how": "same develop, pinned host buffers in/out, through lre_server_submit/wait with up to "
                       "`lanes` requests in flight (copies of one request overlap another's kernels); wall clock"},
            "roofline": roof,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_xtrans:
            line["xtrans"] = run_xtrans(args, acc, stream)
        if world == 1 and not args.no_demosaics:
            line["demosaics"] = run_demosaics(args, acc, stream, d_mos, W, H)
        if world == 1 and not args.no_batch:
            line["batched"] = run_batched(args, acc)
        if world == 1 and not args.no_serve:
            line["served"] = run_served(args)
        if not args.no_cpu_baseline and world == 1:
            try:
                line["cpu_baseline"] = cpu_baseline(mosaic)
            except Exception as e:  # the oracle is test infrastructure; report, do not fail the bench
                line["cpu_baseline"] = {"value": None, "error": str(e)}
        print(json.dumps(line))
    acc.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_e2e(acc, mosaic, params, args, world, mp, pinned=True):
    """MP/s through lre_develop with host buffers (page-locked, or ordinary
    pageable numpy arrays with pinned=False): the H2D copy of the mosaic and
    the D2H copy of the RGB result are inside every timed step."""
    import numpy as np
    import torch

    if pinned:
        h_mos_np = torch.from_numpy(mosaic).pin_memory().numpy()
        h_out_np = torch.empty((H, W, 3), dtype=torch.float32).pin_memory().numpy()
    else:
        h_mos_np = np.array(mosaic, dtype=np.float32, copy=True)
        h_out_np = np.empty((H, W, 3), np.float32)
        h_out_np.fill(0.0)  # touch the pages, as a caller's filled buffer would be
    acc.set_stream(None)
    for _ in range(max(1, args.warmup // 2)):
        acc.develop(h_mos_np, params, out=h_out_np)
    barrier(world)
    t0 = time.perf_counter()
    e_steps = max(2, args.steps // 2)
    for _ in range(e_steps):
        acc.develop(h_mos_np, params, out=h_out_np)
    e_ms = (time.perf_counter() - t0) / e_steps * 1e3
    e_ms = max_over_ranks(e_ms, world)
    return world * mp / (e_ms / 1e3), e_ms


def run_e2e_served(mosaic, params, args, world, mp, device):
    """The same develop, host buffers in and out, through the request server
    (lre_server_submit / lre_server_wait): every request uploads its pinned
    mosaic and downloads its f32 RGB inside the timed region, and up to
    `lanes` requests are in flight, so one request's copies overlap another's
    kernels.  Wall-clock over K requests after a warm-up."""
    import numpy as np

    import libraw_enhanced_b200 as lre

    lanes = 3
    h_mos = _pinned(mosaic.shape, np.float32)
    h_mos[...] = mosaic
    outs = [_pinned((H, W, 3), np.float32) for _ in range(lanes)]
    srv = lre.Server(device, lanes=lanes, budget_bytes=150 * 10**9)
    try:
        def run(k):
            tickets = []
            for i in range(k):
                if len(tickets) >= lanes:
                    srv.wait(tickets.pop(0))
                tickets.append(srv.submit(h_mos, params, out=outs[i % lanes]))
            for t in tickets:
                srv.wait(t)

        run(2 * lanes)
        barrier(world)
        k = max(2 * lanes, args.steps)
        t0 = time.perf_counter()
        run(k)
        ms = (time.perf_counter() - t0) / k * 1e3
    finally:
        srv.close()
    ms = max_over_ranks(ms, world)
    return world * mp / (ms / 1e3), ms, lanes


def _pinned(shape, dtype):
    """A numpy view of page-locked host memory (torch's pinned allocator)."""
    import numpy as np
    import torch

    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    return torch.empty(n, dtype=torch.uint8).pin_memory().numpy().view(dtype).reshape(shape)


def run_batched(args, acc):
    """The 32-image batched develop: sizes {4032x3024, 6000x4000, 8256x5504,
    9504x6336}, CFAs and WB drawn by seed, AMaZE -> defringe -> axial CA,
    16-bit output.  Host f32 mosaics in, host u16 RGB out (page-locked),
    through lre_batch_run (lanes, one CUDA graph per batch, autotuned kernel
    shapes); the plain path develops the same 32 images one lre_develop call
    at a time for the comparison."""
    import numpy as np
    import torch

    import libraw_enhanced_b200 as lre
    from libraw_enhanced_b200 import scenes

    specs = scenes.batch_specs(32, 100)
    mos, outs, params = [], [], []
    for seed, h, w, cfa, wb in specs:
        d = scenes.mosaic_upscaled_torch(seed, h, w, cfa, wb)
        hm = _pinned((h, w), np.float32)
        torch.from_numpy(hm).copy_(d.cpu())
        del d
        mos.append(hm)
        outs.append(_pinned((h, w, 3), np.uint16))
        params.append(lre.develop_params(cfa=cfa, cam_mul=wb, defringe=1, axial_ca_correction=1,
                                         output_bits=16, stage_order=1))
    torch.cuda.empty_cache()
    total_mp = sum(h * w for _, h, w, _, _ in specs) / 1e6
    b = lre.Batch(acc.device, lanes=0, use_graph=True, autotune=True)
    t0 = time.perf_counter()
    b.run(mos, params, outs)  # autotune + capture
    first_s = time.perf_counter() - t0
    tune_ms = b.last_stats.tune_ms
    b.run(mos, params, outs)  # replay (warm)
    steps = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(steps):
        b.run(mos, params, outs)
    dt = (time.perf_counter() - t0) / steps
    st = b.last_stats
    tuning = b.get_tuning()
    b.close()
    # plain per-image path on the same images, same kernel shapes
    acc.set_stream(None)
    acc.set_tuning(tuning["axial_strip"], tuning["axial_rows"], tuning["blur_tile"])
    acc.develop(mos[0], params[0], out=outs[0])
    t0 = time.perf_counter()
    for m, p, o in zip(mos, params, outs):
        acc.develop(m, p, out=o)
    dt_plain = time.perf_counter() - t0
    acc.set_tuning()
    del mos, outs
    return {
        "value": round(total_mp / dt, 2),
        "unit": "MP/s",
        "ms_per_batch": round(dt * 1e3, 1),
        "images": len(specs),
        "total_mp": round(total_mp, 1),
        "plain_e2e": round(total_mp / dt_plain, 2),
        "speedup_vs_plain": round(dt_plain / dt, 3),
        "graph": int(st.graph),
        "lanes": int(st.lanes),
        "gpu_launches": int(st.launches),
        "tuning": tuning,
        "first_call_s": round(first_s, 2),
        "tune_ms": round(tune_ms, 1),
        "h2d_bytes_per_step": int(sum(h * w * 4 for _, h, w, _, _ in specs)),
        "d2h_bytes_per_step": int(sum(h * w * 6 for _, h, w, _, _ in specs)),
        "workload": "32 Bayer images (sizes/CFA/WB by seeds 100..131), AMaZE->defringe->axial CA, u16 out; "
                    "host page-locked buffers in/out, timed per whole batch",
    }


def run_xtrans(args, acc, stream):
    """The X-Trans workload: a 6240x4160 mosaic (standard 6x6 CFA) with radial
    lateral CA injected (R x1.0008, B x0.9992), 3-pass X-Trans demosaic ->
    pyramidal LK lateral CA (cell 96, 3 levels, 3 iterations, max shift 6,
    min confidence 0.02), float32 RGB out; device-resident, CUDA events on
    the library's stream."""
    import torch

    import libraw_enhanced_b200 as lre
    from libraw_enhanced_b200 import scenes

    w, h = (int(v) for v in args.xtrans_size.lower().split("x"))
    d_mos = scenes.xtrans_lateral_ca_torch(3, h, w)
    d_out = torch.empty((h, w, 3), dtype=torch.float32, device=d_mos.device)
    d_tmp = torch.empty_like(d_out)
    acc.set_stream(stream.cuda_stream)
    p = lre.develop_params(cfa=scenes.XTRANS_STD, cam_mul=(1.8, 1.0, 1.6, 1.0), xtrans_passes=3,
                           lateral_ca_correction=1, lateral_ca_cell_size=96, lateral_ca_pyramid_levels=3,
                           lateral_ca_max_iterations=3, lateral_ca_max_shift=6.0, lateral_ca_min_confidence=0.02)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    reps = max(3, min(args.steps, 10))
    ms = timed(lambda: acc.dev_develop(d_mos, d_out, w, h, p), reps)
    st = {
        "xtrans_3pass": timed(lambda: acc.dev_demosaic_xtrans(d_mos, d_tmp, w, h, scenes.XTRANS_STD, 1.0, 3), 3),
        "lateral_ca": timed(lambda: acc.dev_ca_register_lateral(d_tmp, d_out, w, h, 96, 3, 6.0, 0.02, 3), 3),
    }
    mp = h * w / 1e6
    return {
        "value": round(mp / (ms / 1e3), 2),
        "unit": "MP/s",
        "ms_per_image": round(ms, 3),
        "stage_ms": {k: round(v, 3) for k, v in st.items()},
        "workload": f"{w}x{h} X-Trans (radial lateral CA injected): 3-pass demosaic -> pyramidal LK lateral CA, "
                    "f32 RGB out, device-resident",
    }


def run_demosaics(args, acc, stream, d_mos, W, H):
    """The four Bayer demosaics the reference routes (bilinear, AMaZE, DCB,
    AAHD) alone on the 51 MP mosaic, scaled to a 14-bit raw range (AAHD
    indexes a 64 Ki gamma table with the sample); device-resident, CUDA
    events on the library's stream."""
    import torch

    from libraw_enhanced_b200 import scenes

    acc.set_stream(stream.cuda_stream)  # the e2e leg leaves the library on its own stream
    mos = (d_mos * 16383.0).contiguous()
    out = torch.empty((H, W, 3), dtype=torch.float32, device=mos.device)
    f = scenes.FILTERS["RGGB"]

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    reps = max(3, min(args.steps, 5))
    legs = {
        "linear": lambda: acc.dev_demosaic_bayer_linear(mos, out, W, H, f, 16383.0),
        "amaze": lambda: acc.dev_demosaic_bayer_amaze(mos, out, W, H, f, WB, 16383.0),
        "dcb": lambda: acc.dev_demosaic_bayer_dcb(mos, out, W, H, f, 16383.0, 1, True),
        "aahd": lambda: acc.dev_demosaic_bayer_aahd(mos, out, W, H, f, 16383.0),
    }
    res = {}
    for k, fn in legs.items():
        ms = timed(fn, reps)
        res[k] = {"ms": round(ms, 3), "mp_s": round(H * W / 1e6 / (ms / 1e3), 1)}
    res["workload"] = f"{W}x{H} RGGB mosaic, 14-bit range, f32 RGB out; DCB 1 iteration + enhance"
    return res


def run_served(args):
    """Poisson arrivals of develop requests through lre_server_*: 60% 6000x4000
    Bayer, 25% 8256x5504 Bayer, 15% 6240x4160 X-Trans; defringe p=.5, axial
    p=.5, lateral p=.2, ACES p=.3; 150 GB device budget, 4 lanes, u16 out.
    Reports p50/p99 of submit -> result-in-host-memory per arrival rate, and
    the throughput of a saturated queue."""
    import threading

    import numpy as np
    import torch

    import libraw_enhanced_b200 as lre
    from libraw_enhanced_b200 import scenes

    kinds = [("bayer", 4000, 6000, 0.60), ("bayer", 5504, 8256, 0.25), ("xtrans", 4160, 6240, 0.15)]
    pool = []  # (kind index, mosaic, base params)
    for ki, (kind, h, w, _) in enumerate(kinds):
        for j in range(2):
            seed = 500 + 10 * ki + j
            if kind == "bayer":
                cfa = ["RGGB", "BGGR", "GRBG", "GBRG"][(ki + j) % 4]
                wb = (2.0 - 0.2 * j, 1.0, 1.5 + 0.1 * j, 1.0)
                d = scenes.mosaic_upscaled_torch(seed, h, w, cfa, wb)
                p = lre.develop_params(cfa=cfa, cam_mul=wb, output_bits=16)
            else:
                wb = (1.8, 1.0, 1.6, 1.0)
                d = scenes.mosaic_upscaled_torch(seed, h, w, scenes.XTRANS_STD, wb)
                p = lre.develop_params(cfa=scenes.XTRANS_STD, cam_mul=wb, output_bits=16)
            hm = _pinned((h, w), np.float32)
            torch.from_numpy(hm).copy_(d.cpu())
            del d
            pool.append((ki, hm, p))
    torch.cuda.empty_cache()
    n_ring = 24
    max_px = max(h * w for _, h, w, _ in kinds)
    ring = [_pinned((max_px * 3,), np.uint16) for _ in range(n_ring)]
    rng = np.random.Generator(np.random.PCG64(500))

    def make_request():
        ki = int(rng.choice(3, p=[k[3] for k in kinds]))
        cand = [e for e in pool if e[0] == ki]
        _, m, base = cand[int(rng.integers(0, len(cand)))]
        p = lre.DevelopParams.from_buffer_copy(base)
        p.defringe = int(rng.random() < 0.5)
        p.axial_ca_correction = int(rng.random() < 0.5)
        p.lateral_ca_correction = int(rng.random() < 0.2)
        p.tone_mapping = 1 if rng.random() < 0.3 else 0
        return ki, m, p

    srv = lre.Server(0, lanes=4, budget_bytes=150 * 10**9)

    def run_stream(n, lam):
        reqs = [make_request() for _ in range(n)]
        gaps = rng.exponential(1.0 / lam, size=n) if lam else np.zeros(n)
        tickets = [None] * n
        stats = [None] * n
        done_evt = [threading.Event() for _ in range(n)]

        def waiter():
            for k in range(n):
                while tickets[k] is None:
                    time.sleep(0.0002)
                out, s = srv.wait(tickets[k])
                stats[k] = s
                done_evt[k].set()

        wt = threading.Thread(target=waiter)
        wt.start()
        t0 = time.perf_counter()
        t_next = t0
        for k, (_, m, p) in enumerate(reqs):
            t_next += gaps[k]
            dly = t_next - time.perf_counter()
            if dly > 0:
                time.sleep(dly)
            if k >= n_ring:
                done_evt[k - n_ring].wait()
            h, w = m.shape
            out = ring[k % n_ring][: h * w * 3].reshape(h, w, 3)
            tickets[k] = srv.submit(m, p, out=out)
        wt.join()
        t_end = time.perf_counter()
        lat = np.array([s["total_ms"] for s in stats])
        mp = sum(m.shape[0] * m.shape[1] for _, m, _ in reqs) / 1e6
        per_kind = {}
        for ki, (kind, kh, kw, _) in enumerate(kinds):
            lk = np.array([lat[k] for k in range(n) if reqs[k][0] == ki])
            if lk.size:
                per_kind[f"{kind}_{kw}x{kh}"] = {
                    "n": int(lk.size),
                    "p50_ms": round(float(np.percentile(lk, 50)), 1),
                    "p99_ms": round(float(np.percentile(lk, 99)), 1),
                }
        return {
            "lambda": lam if lam else "saturated",
            "n": n,
            "p50_ms": round(float(np.percentile(lat, 50)), 1),
            "p99_ms": round(float(np.percentile(lat, 99)), 1),
            "per_kind": per_kind,
            "mean_queue_ms": round(float(np.mean([s["queue_ms"] for s in stats])), 1),
            "mp_s": round(mp / (t_end - t0), 1),
            "mp_per_request": round(mp / n, 2),
        }

    # Warm-up, as a server does before taking traffic: every request kind with
    # every option on, twice per lane, so each lane has sized its buffers and
    # every kernel has been loaded before the timed rates.
    warm = []
    for rep in range(2 * 4):
        for ki in range(len(kinds)):
            cand = [e for e in pool if e[0] == ki]
            _, m, base = cand[rep % len(cand)]
            p = lre.DevelopParams.from_buffer_copy(base)
            p.defringe, p.axial_ca_correction, p.lateral_ca_correction, p.tone_mapping = 1, 1, 1, 1
            warm.append((m, p))
    wt_tickets = []
    for k, (m, p) in enumerate(warm):
        h, w = m.shape
        wt_tickets.append(srv.submit(m, p, out=ring[k % n_ring][: h * w * 3].reshape(h, w, 3)))
        if len(wt_tickets) >= n_ring // 2:
            srv.wait(wt_tickets.pop(0))
    for t in wt_tickets:
        srv.wait(t)
    run_stream(8, 0)
    rates = []
    for lam in (5, 10, 20, 30, 45, 60):
        rates.append(run_stream(64, lam))
    sat = run_stream(64, 0)
    _, peak = srv.memory()
    srv.close()
    del ring, pool
    return {
        "unit": "MP/s",
        "rates": rates,
        "saturated_mp_s": sat["mp_s"],
        "saturated_p50_ms": sat["p50_ms"],
        "saturated_p99_ms": sat["p99_ms"],
        "saturated_per_kind": sat["per_kind"],
        "lanes": 4,
        "budget_gb": 150,
        "peak_device_gb": round(peak / 1e9, 2),
        "workload": "Poisson arrivals, 64 requests per rate: 60% 6000x4000 Bayer, 25% 8256x5504 Bayer, "
                    "15% 6240x4160 X-Trans; defringe .5, axial .5, lateral .2, ACES .3; u16 out; "
                    "latency = submit -> result in page-locked host memory, overall and per request kind "
                    "(bayer_6000x4000 is the 24 MP class); warm-up: every kind with every "
                    "option twice per lane before the timed rates",
    }


def scenes_filters():
    from libraw_enhanced_b200 import scenes

    return scenes.FILTERS["RGGB"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the 32-image batched develop")
    ap.add_argument("--no-serve", action="store_true", help="skip the request-server sweep")
    ap.add_argument("--no-xtrans", action="store_true", help="skip the X-Trans + lateral CA workload")
    ap.add_argument("--no-demosaics", action="store_true", help="skip the per-algorithm Bayer demosaic timings")
    ap.add_argument("--xtrans-size", default="6240x4160", help="WxH of the X-Trans workload (reduced cases: profiling)")
    ap.add_argument("--size", default=None, help="WxH of a reduced case (profiling); default 8736x5856")
    args = ap.parse_args()
    if args.size:
        global H, W
        W, H = (int(v) for v in args.size.lower().split("x"))
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
