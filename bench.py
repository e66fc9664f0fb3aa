#!/usr/bin/env python
"""Benchmark of the B200 HEVC reconstruction back end.

Workload (one step): full decode of a 4032x3024 10-bit 4:2:0 HEIC still
stored as an 8x6 grid of 512x512 tiles (edge tiles cropped) from the flat
per-tile buffers the host syntax decode produces, to a packed RGB8 canvas
(BT.601 full range, `decode_heic_rgb8`): intra prediction + dequant +
inverse DCT/DST + add, deblocking, SAO, YCbCr->RGB and stitching.  Inputs are
seeded synthetic buffers with the benchmark's distributions (there is no
public corpus for this path).

Metric: decoded megapixels (output luma pixels) per second, higher is better.
  value  -- device time of the decode with inputs resident in HBM, L2
            flushed between steps, CUDA events on the launching stream.
  e2e    -- the same decode through the C-ABI host-buffer entry points
            (hpvcd_gpu_submit / wait / read) with the inputs in page-locked
            host memory and the RGB8 canvas copied back every step; beside
            it the same with ordinary (pageable) per-tile buffers.
  batched -- the mixed-size serving workload (256 images): one fused plan
            against one plan per image, device time, its reconstruction
            roofline, and the serving loop's latency percentiles.
`--impl reference` times the reference's CPU decode on the host cores: the
C++ restatement of its parallel structure (grid-row jobs, banded
deblocking / SAO / colour conversion on a work-stealing pool) with its AVX2
kernel set, on the same workload and configuration.

One process per GPU (torchrun for N > 1); every rank decodes its own image
(replicas, weak scaling); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "heic_grid_4032x3024_10bit_420_48x512_tiles_to_rgb8"
OUT_W, OUT_H = 4032, 3024
MPIX = OUT_W * OUT_H / 1e6


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--e2e-inflight", type=int, default=4, help="steps in flight in the end-to-end measurement")
    ap.add_argument("--e2e-schedule", default="default",
                    help="end-to-end: 'default' (the headline), 'network' (the selector's pick for "
                         "submits that find no other ticket in flight), or 'fixed:K' (candidate K of the "
                         "selector's list); the network and the default schedule are reported beside each other")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--coeff16", action="store_true",
                    help="keep every tile's int16 level pool (default: int8 pools where every level fits)")
    ap.add_argument("--workload", choices=["grid", "serving", "selector", "inter"], default="grid",
                    help="grid: the 4032x3024 still (default); serving: mixed-size batched serving; "
                         "selector: learned schedule selection on 3840x2160 frames; inter: 1080p GOP")
    ap.add_argument("--frames", type=int, default=60, help="selector: fresh frames to evaluate")
    ap.add_argument("--images", type=int, default=64, help="serving: number of images")
    ap.add_argument("--batched-images", type=int, default=256,
                    help="default workload: images of the mixed-size batch block (0 = leave it out)")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: Poisson arrivals per second")
    ap.add_argument("--no-serving", action="store_true",
                    help="default workload: leave the serving-loop runs out of the mixed-size batch block")
    ap.add_argument("--sched", default="network",
                    help="default workload: 'network' (the selector's pick) or a fixed schedule "
                         "'idct,chroma_warps,recon_ctas_per_sm,wave' (hpvcd_sched)")
    return ap.parse_args()


def dist_info():
    from hpvcd_b200 import replicas
    return replicas.dist_info()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM traffic of the reconstruction stage per step from the committed
    ncu summaries (profiles/recon_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "recon_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        self.t0 = self.t1 = None
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(device_index)], stdout=self.f, stderr=subprocess.DEVNULL)
            # wait for the first sample, so the sampler runs before the timed region starts
            deadline = time.time() + 5.0
            while time.time() < deadline and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        if self.t0 is not None and self.t1 is not None:  # samples taken inside the timed region
            from datetime import datetime

            def stamp(r):
                try:
                    return datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    return None
            inside = [r for r in rows if stamp(r) is not None and self.t0 - 0.05 <= stamp(r) <= self.t1 + 0.05]
            if inside:
                rows = inside
            else:  # region shorter than the sampling period: the sample closest to its middle
                mid = 0.5 * (self.t0 + self.t1)
                rows = [min(rows, key=lambda r: abs((stamp(r) or 0.0) - mid))]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(rows), "reasons": reasons}


CPU_ARM = ("C++ restatement of the hpvcd CPU decode path (Rust toolchain absent): its AVX2 kernel set "
           "(transforms, intra prediction, residual add, SAO, YCbCr->RGB) and its parallel structure "
           "(grid-row jobs, banded deblocking / SAO / RGB on a work-stealing pool)")


def headline_config(n_int8: int, n_tiles: int) -> dict:
    """The workload's description, the same in both arms' lines."""
    return {"workload": WORKLOAD, "tiles": 48, "tile": "512x512 (edge tiles cropped)",
            "out": f"{OUT_W}x{OUT_H} RGB8 BT.601 full range", "bit_depth": 10, "chroma": "4:2:0",
            "l2": "flushed between steps (256 MiB write)",
            "levels": f"int8 pools for {n_int8} of {n_tiles} tiles (every level fits), else int16",
            "inputs": "seeded synthetic flat buffers (CU/TU quadtrees, modes, QP 22-37, 85% zero levels, "
                      "Laplacian(8), deblock on, random SAO)"}


def reference_decode(pics, out, threads: int, simd: bool = True):
    from oracle import oracle as O
    return O.decode_grid_reference(pics, out, threads, simd)


def cpu_baseline(pics, out, threads: int, min_seconds: float = 3.0) -> dict:
    """The reference's CPU decode (its parallel structure and AVX2 kernel
    set, restated) on the host cores: repeated full decodes of the workload
    for ~min_seconds; beside it the scalar kernels on one thread."""
    reference_decode(pics, out, threads)  # warm
    reps, t0 = 0, time.perf_counter()
    while True:
        reference_decode(pics, out, threads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds and reps >= 2:
            break
    reference_decode(pics, out, 1, simd=False)
    r1, t1 = 0, time.perf_counter()
    while True:
        reference_decode(pics, out, 1, simd=False)
        r1 += 1
        e1 = time.perf_counter() - t1
        if e1 >= min_seconds / 2 and r1 >= 1:
            break
    return {"value": round(MPIX * reps / el, 2), "unit": "MPix/s", "cores": threads, "kind": "port",
            "sample": f"{reps} full {OUT_W}x{OUT_H} decodes (48 tiles, recon+deblock+SAO+RGB8) "
                      f"in {el:.2f} s, {threads} threads, AVX2 kernels",
            "implementation": CPU_ARM,
            "scalar_single_thread": {"value": round(MPIX * r1 / e1, 2), "unit": "MPix/s", "cores": 1,
                                     "sample": f"{r1} full decodes in {e1:.2f} s, scalar kernels, one thread"}}


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    from hpvcd_b200 import synth
    threads = os.cpu_count() or 1
    g = synth.config1_grid(seed=0)
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    c8keep = [] if args.coeff16 else synth.narrow_coeffs(pics)  # same inputs as the GPU arm
    for _ in range(max(args.warmup, 1)):
        reference_decode(pics, out, threads)
    steps = max(1, min(args.steps, 20))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        reference_decode(pics, out, threads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = MPIX * steps / total
    times_ms = sorted(t * 1e3 for t in times)
    config = headline_config(len(c8keep), len(pics))
    config["parallelism"] = f"replicas x{world}"
    line = {
        "impl": "reference", "metric": "decoded MPix/s", "value": round(value, 2), "unit": "MPix/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": round(total / steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": config,
        "latency_ms": {"p50": round(times_ms[len(times_ms) // 2], 3),
                       "p99": round(times_ms[min(len(times_ms) - 1, int(0.99 * len(times_ms)))], 3)},
        "cpu_baseline": {"value": round(value, 2), "unit": "MPix/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full decodes of the workload, {threads} threads, AVX2 kernels",
                         "implementation": CPU_ARM},
        "e2e": {"value": round(value, 2), "unit": "MPix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_e2e(pics, g, K2, warmup, local, world, dev, in_flight=2, schedule="network", pageable=False):
    """Same decode through hpvcd_gpu_submit / wait / read: inputs packed in
    page-locked host memory (one H2D DMA per step) and the RGB8 canvas DMA'd
    back to a page-locked caller buffer every step; or (pageable) the
    ordinary per-tile host buffers as the host syntax decode leaves them and
    an ordinary numpy canvas (the context stages both through its own
    page-locked buffers with the host copy pool).  `in_flight` steps are queued (each with its
    own output buffer), so one step's copies overlap another's decoding;
    throughput = steps / wall time from the first submit to the last read,
    latency = submit -> read per step."""
    import torch

    from hpvcd_b200 import abi, replicas, synth
    from hpvcd_b200.gpu import GpuDecoder, pack_pinned, pinned_empty

    packed, pkeep = pack_pinned(pics)
    h2d = pkeep[2]
    src = list(pics) if pageable else packed
    canvas_bytes = OUT_W * OUT_H * 3
    outs = []
    import numpy as np
    for _ in range(in_flight):
        # pageable: an ordinary numpy canvas (the context DMAs into its own
        # page-locked buffer and copies out in hpvcd_gpu_read)
        dst, dkeep = (np.empty(canvas_bytes, np.uint8), None) if pageable else pinned_empty(canvas_bytes)
        o, okeep = synth.grid_output(g)
        o.options = abi.OUTPUT_CANVAS_ONLY  # the product is the canvas
        o.host_dst = dst.ctypes.data
        o.host_dst_bytes = canvas_bytes
        outs.append((o, dst, dkeep, okeep))
    mlp = _selector_network() if schedule == "network" else None
    with GpuDecoder(local, max_inflight=in_flight) as decd:
        if schedule.startswith("fixed:"):
            from hpvcd_b200 import selector
            decd.set_sched(selector.SCHEDULES[int(schedule.split(":")[1])])
        if mlp is not None:  # every submit picks its schedule from the batch's features
            from hpvcd_b200 import selector
            decd.set_selector(mlp, selector.SCHEDULES)
        # warm-up in the timed loop's own pattern, so every ticket slot has
        # built its staging, device arena and plan before timing starts
        warm = []
        for k in range(max(3, warmup // 2) + 2 * in_flight):
            o, dst = outs[k % in_flight][:2]
            if len(warm) == in_flight:
                t, d = warm.pop(0)
                decd.wait(t)
                decd.read(t, d)
            warm.append((decd.submit(src, o), dst))
        for t, d in warm:
            decd.wait(t)
            decd.read(t, d)
        if world > 1:
            torch.distributed.barrier()
        lat = []
        pending = []  # (ticket, dst, submit time)
        t_start = time.perf_counter()
        for k in range(K2):
            o, dst = outs[k % in_flight][:2]
            if len(pending) == in_flight:  # the buffer of step k - in_flight is read before it is reused
                t, d, ts = pending.pop(0)
                decd.wait(t)
                decd.read(t, d)
                lat.append(time.perf_counter() - ts)
            pending.append((decd.submit(src, o), dst, time.perf_counter()))
        for t, d, ts in pending:
            decd.wait(t)
            decd.read(t, d)
            lat.append(time.perf_counter() - ts)
        e2e_total = replicas.max_over_ranks(time.perf_counter() - t_start, dev)
    lat = sorted(x * 1e3 for x in lat)
    return {"value": round(world * MPIX * K2 / e2e_total, 2), "unit": "MPix/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": canvas_bytes,
            "steps": K2, "ms_per_step": round(e2e_total / K2 * 1e3, 3),
            "p50_ms": round(lat[len(lat) // 2], 3),
            "p99_ms": round(lat[min(len(lat) - 1, int(0.99 * len(lat)))], 3),
            "in_flight": in_flight,
            "api": "hpvcd_gpu_submit/wait/read, " + ("pageable per-tile inputs, pageable RGB8 output" if pageable
                                                     else "pinned packed inputs, pinned RGB8 output"),
            "schedule": "network pick per submit" if mlp is not None else schedule}


def host_syntax(g, local, steps: int = 8, in_flight: int = 2) -> dict:
    """The grid from its coded slices: the host syntax decode (CABAC and
    coding-tree syntax of the 48 I slices, csrc/syntax.cpp) on every host
    thread alone, and bitstream -> RGB8 end to end: each step parses the
    slices on the host and submits the parsed buffers (ordinary host memory)
    to hpvcd_gpu_submit, with `in_flight` steps queued so one step's parse
    overlaps the previous step's decode; the canvas comes back to an
    ordinary numpy buffer.  Wall clock."""
    import numpy as np

    from hpvcd_b200 import abi, synth
    from hpvcd_b200.gpu import GpuDecoder
    from hpvcd_b200.syntax import decode_batch

    slices = synth.grid_slices(g)
    threads = os.cpu_count() or 1
    coded = sum(len(d) for _, d in slices)
    for r in decode_batch(slices, threads):
        r.close()
    t = []
    bins = 0
    for _ in range(steps):
        t0 = time.perf_counter()
        parsed = decode_batch(slices, threads)
        t.append(time.perf_counter() - t0)
        bins = sum(x.bins for x in parsed)
        for x in parsed:
            x.close()
    parse_s = statistics.median(t)
    out, keep = synth.grid_output(g)
    out.options = abi.OUTPUT_CANVAS_ONLY
    canvas_bytes = OUT_W * OUT_H * 3
    dsts = [np.empty(canvas_bytes, np.uint8) for _ in range(in_flight)]
    with GpuDecoder(local, max_inflight=in_flight) as dec:
        pend = []
        def step(k):
            parsed = decode_batch(slices, threads)
            o = out
            o.host_dst = dsts[k % in_flight].ctypes.data
            o.host_dst_bytes = canvas_bytes
            return dec.submit([x.picture() for x in parsed], o), parsed, dsts[k % in_flight]
        for k in range(in_flight + 1):  # warm-up: staging and plans of every slot
            if len(pend) == in_flight:
                tk, pp, d = pend.pop(0)
                dec.wait(tk)
                dec.read(tk, d)
            pend.append(step(k))
        for tk, pp, d in pend:
            dec.wait(tk)
            dec.read(tk, d)
        pend = []
        t0 = time.perf_counter()
        for k in range(steps):
            if len(pend) == in_flight:
                tk, pp, d = pend.pop(0)
                dec.wait(tk)
                dec.read(tk, d)
            pend.append(step(k))
        for tk, pp, d in pend:
            dec.wait(tk)
            dec.read(tk, d)
        e2e_s = (time.perf_counter() - t0) / steps
    return {"slices": len(slices), "coded_bytes": coded, "threads": threads,
            "parse_ms": round(parse_s * 1e3, 2), "parse_mpix_per_s": round(MPIX / parse_s, 1),
            "parse_mbins_per_s": round(bins / parse_s / 1e6, 1),
            "bitstream_to_rgb8_mpix_per_s": round(MPIX / e2e_s, 1), "bitstream_to_rgb8_ms": round(e2e_s * 1e3, 2),
            "api": "hpvcd_syntax_decode_batch -> hpvcd_gpu_submit/wait/read (ordinary host buffers), wall clock",
            "note": "the syntax decode stays on the host in the reference too; these figures bound a "
                    "bitstream-fed pipeline, the headline starts from the parsed buffers"}


def run_ours(args):
    import numpy as np
    import torch

    from hpvcd_b200 import replicas
    from hpvcd_b200 import abi, synth
    from hpvcd_b200.gpu import DevicePlan

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)
    L = abi.lib()

    g = synth.config1_grid(seed=rank)
    out, keep = synth.grid_output(g)
    out.options = abi.OUTPUT_CANVAS_ONLY  # the product is the RGB8 canvas (decode_heic_rgb8)
    pics = g.synth.pictures()
    # host transport choice: tiles whose levels all fit in int8 ship an int8
    # pool (half the bytes over PCIe); the pixels are the same
    c8keep = [] if args.coeff16 else synth.narrow_coeffs(pics)
    plan = DevicePlan(pics, out, device=local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    # stages: reconstruction (k_residual + k_recon), then deblocking + SAO +
    # RGB8 (one fused tile kernel when launched together)
    stage_names = ("recon", "filters")
    stages = [abi.STAGE_RECON, abi.STAGE_DEBLOCK | abi.STAGE_SAO | abi.STAGE_OUTPUT]
    # the learned schedule: the network picks from the batch's device features
    mlp = _selector_network() if args.sched == "network" else None
    schedule = {"selected_by": "default"}
    if args.sched != "network":
        fixed = [int(v) for v in args.sched.split(",")]
        plan.set_sched(abi.Sched(*fixed))
        schedule = {"selected_by": "fixed", "sched": fixed}
    if mlp is not None:
        import ctypes as C
        from hpvcd_b200 import selector
        chosen = C.c_uint32()
        abi.check(L.hpvcd_plan_select(plan._h, mlp.handle, selector.schedules_array(), selector.K,
                                      C.c_void_p(stream.cuda_stream), C.byref(chosen)), "hpvcd_plan_select")
        pick = int(chosen.value)
        sc = selector.SCHEDULES[pick] if pick < selector.K else None
        schedule = {"selected_by": "network", "pick": pick,
                    "sched": [sc.idct, sc.chroma_warps, sc.recon_ctas_per_sm, sc.wave] if sc is not None else None}
    # NVTX range "grid" (and "batched" below) lets a profiler pick this
    # workload's launches: ncu --nvtx --nvtx-include "grid/"
    torch.cuda.nvtx.range_push("grid")
    for _ in range(args.warmup):
        flush.zero_()
        plan.launch(abi.STAGE_ALL, stream)
    torch.cuda.synchronize(dev)
    st = plan.status(stream)
    if st != abi.OK:
        raise abi.HpvcdError(st, "device status after warm-up")

    K = args.steps
    # timed region: one whole-pipeline launch per step (segments of independent
    # pictures overlap across stages inside it)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    launches0 = L.hpvcd_kernel_launch_count()
    if world > 1:
        torch.distributed.barrier()
    clocks = Clocks(local)
    torch.cuda.synchronize(dev)
    clocks.mark_start()
    for k in range(K):
        flush.zero_()
        ev[k][0].record(stream)
        plan.launch(abi.STAGE_ALL, stream)
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    clocks.mark_end()
    clock_rec = clocks.stop()
    if world > 1:
        torch.distributed.barrier()
    launches = L.hpvcd_kernel_launch_count() - launches0
    st = plan.status(stream)
    if st != abi.OK:
        raise abi.HpvcdError(st, "device status after timed region")
    step_ms = [a.elapsed_time(b) for a, b in ev]
    default_ms = None
    if mlp is not None:  # the same steps with the default schedule, for comparison
        plan.set_sched(None)
        K4 = max(3, min(K, 30))
        dev_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K4)]
        for k in range(K4):
            flush.zero_()
            dev_ev[k][0].record(stream)
            plan.launch(abi.STAGE_ALL, stream)
            dev_ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
        default_ms = sum(a.elapsed_time(b) for a, b in dev_ev) / K4
        if schedule.get("sched") is not None:
            plan.set_sched(abi.Sched(*schedule["sched"]))

    # stage breakdown (separate, untimed for the value): the stages launched
    # one after another, each as its own plan launch
    K3 = max(3, min(K, 20))
    sev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(stages) + 1)] for _ in range(K3)]
    for k in range(K3):
        flush.zero_()
        sev[k][0].record(stream)
        for i, s_ in enumerate(stages):
            plan.launch(s_, stream)
            sev[k][i + 1].record(stream)
    torch.cuda.synchronize(dev)
    stage_ms = [sum(sev[k][i].elapsed_time(sev[k][i + 1]) for k in range(K3)) / K3 for i in range(len(stages))]
    torch.cuda.nvtx.range_pop()
    total_ms = replicas.max_over_ranks(sum(step_ms), dev)
    value = replicas.whole_job_rate(MPIX * K, total_ms / 1e3, dev)
    lat = sorted(step_ms)

    # Roofline of the dominant kernel (the reconstruction kernel): algorithmic
    # bytes per launch = dense levels of the coded TBs (int16, or int8 in a
    # narrowed pool) + TB records + CTU index + the reconstructed samples
    # written once.
    recon_bytes, written = recon_algorithmic_bytes(pics)
    peak, peak_kind = measured_peaks()
    recon_s = stage_ms[0] / 1e3
    achieved = recon_bytes / recon_s / 1e9
    traffic = profile_traffic()
    # achieved, algorithmic bytes and traffic all cover the reconstruction
    # stage: k_residual + k_recon of every group of one step
    roofline = {"kernel": "k_recon", "scope": "reconstruction stage (k_residual + k_recon, one step)",
                "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": recon_bytes,
                "traffic": traffic.get("dram_bytes_per_launch") if traffic else None}
    # per-stage algorithmic bytes: the fused filter stage reads the
    # reconstructed planes once and writes the RGB8 canvas (3 bytes per
    # output pixel; the canvas-only output keeps no final planes)
    stage_bytes = {"recon": recon_bytes, "filters": written + OUT_W * OUT_H * 3}
    # whole-pipeline bytes (reconstruction + filters), for context
    pipe_bytes = stage_bytes["recon"] + stage_bytes["filters"]
    stage_roofline = {}
    for i, name in enumerate(stage_names):
        gbs = stage_bytes[name] / (stage_ms[i] / 1e3) / 1e9 if stage_ms[i] > 0 else 0.0
        stage_roofline[name] = {"bytes": int(stage_bytes[name]), "ms": round(stage_ms[i], 4),
                                "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    stage_roofline["filters"]["kernel"] = "k_filter_tile (deblocking V + H, SAO, RGB8 per 64x64 tile)"

    # ---- end to end through the C ABI (host buffers) ----
    e2e = None
    K2 = args.e2e_steps if args.e2e_steps is not None else max(5, min(K, 200))
    if K2 > 0:
        e2e = run_e2e(pics, g, K2, args.warmup, local, world, dev, max(1, args.e2e_inflight), args.e2e_schedule)
        other = "network" if args.e2e_schedule == "default" else "default"
        alt = run_e2e(pics, g, K2, args.warmup, local, world, dev, max(1, args.e2e_inflight), other)
        e2e["other_schedule"] = {k: alt[k] for k in ("value", "ms_per_step", "p50_ms", "p99_ms", "schedule")}
        pg = run_e2e(pics, g, K2, args.warmup, local, world, dev, max(1, args.e2e_inflight), args.e2e_schedule,
                     pageable=True)
        e2e["pageable_inputs"] = {k: pg[k] for k in ("value", "ms_per_step", "p50_ms", "p99_ms", "api")}
        # the end-to-end rate against the link it crosses: the canvas read
        # back each step is the larger direction
        link = pcie_link(dev, int(e2e["h2d_bytes_per_step"]), int(e2e["d2h_bytes_per_step"]))
        e2e_d2h = e2e["d2h_bytes_per_step"] / (e2e["ms_per_step"] / 1e3) / 1e9
        e2e_h2d = e2e["h2d_bytes_per_step"] / (e2e["ms_per_step"] / 1e3) / 1e9
        link.update({"e2e_d2h_gbs": round(e2e_d2h, 1), "e2e_h2d_gbs": round(e2e_h2d, 1),
                     "frac_of_concurrent_d2h": (round(e2e_d2h / link["concurrent_d2h_gbs"], 3)
                                                if link["concurrent_d2h_gbs"] else None)})
        e2e["pcie"] = link

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(pics, out, os.cpu_count() or 1)
    syntax = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        syntax = host_syntax(g, local)
    batched = None
    if world == 1 and args.batched_images > 0:
        batched = batched_block(args, local)

    line = {
        "metric": "decoded MPix/s", "value": round(value, 2), "unit": "MPix/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": round(total_ms / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic",
        "config": {**headline_config(len(c8keep), len(pics)), "parallelism": f"replicas x{world}"},
        "latency_ms": {"p50": round(lat[len(lat) // 2], 4),
                       "p99": round(lat[min(len(lat) - 1, int(0.99 * len(lat)))], 4)},
        "stages_ms": {"recon": round(stage_ms[0], 4), "filters": round(stage_ms[1], 4),
                      "note": "stages launched one after another (separate pass); the timed step overlaps them"},
        "pipeline_gbs": round(pipe_bytes / (total_ms / K / 1e3) / 1e9, 1),
        "stage_roofline": stage_roofline,
        "schedule": schedule,
        "value_default_schedule": (round(MPIX / (default_ms / 1e3), 2) if default_ms else None),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "batched": batched,
        "host_syntax": syntax,
        "gpu_launches": int(launches),
        "launches_per_step": int(launches // K),
        "clocks": clock_rec,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def pcie_link(dev, h2d_bytes: int, d2h_bytes: int, reps: int = 20) -> dict:
    """Measured host<->device copy bandwidth of this box for one end-to-end
    step's byte counts (page-locked host buffers, one cudaMemcpyAsync per
    direction and step, CUDA events): each direction alone and both at once
    on two streams, as the end-to-end loop runs them."""
    import torch
    h_in = torch.empty(h2d_bytes, dtype=torch.uint8, pin_memory=True)
    h_out = torch.empty(d2h_bytes, dtype=torch.uint8, pin_memory=True)
    d_in = torch.empty(h2d_bytes, dtype=torch.uint8, device=dev)
    d_out = torch.empty(d2h_bytes, dtype=torch.uint8, device=dev)
    s_up, s_down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)

    def timed(up: bool, down: bool) -> tuple[float, float]:
        ev = {k: [torch.cuda.Event(enable_timing=True) for _ in range(2)] for k in ("up", "down")}
        torch.cuda.synchronize(dev)
        if up:
            ev["up"][0].record(s_up)
            for _ in range(reps):
                with torch.cuda.stream(s_up):
                    d_in.copy_(h_in, non_blocking=True)
            ev["up"][1].record(s_up)
        if down:
            ev["down"][0].record(s_down)
            for _ in range(reps):
                with torch.cuda.stream(s_down):
                    h_out.copy_(d_out, non_blocking=True)
            ev["down"][1].record(s_down)
        torch.cuda.synchronize(dev)
        gb_up = h2d_bytes * reps / (ev["up"][0].elapsed_time(ev["up"][1]) / 1e3) / 1e9 if up else 0.0
        gb_down = d2h_bytes * reps / (ev["down"][0].elapsed_time(ev["down"][1]) / 1e3) / 1e9 if down else 0.0
        return gb_up, gb_down

    timed(True, True)  # warm-up
    up, _ = timed(True, False)
    _, down = timed(False, True)
    both_up, both_down = timed(True, True)
    return {"h2d_gbs": round(up, 1), "d2h_gbs": round(down, 1), "concurrent_h2d_gbs": round(both_up, 1),
            "concurrent_d2h_gbs": round(both_down, 1),
            "how": f"page-locked copies of one step's bytes ({h2d_bytes} up, {d2h_bytes} down), "
                   f"{reps} per direction, alone and both directions at once, CUDA events"}


def recon_algorithmic_bytes(pics) -> tuple[int, int]:
    """Algorithmic bytes of one reconstruction pass over `pics`: the dense
    levels of the coded TBs (int16, or int8 in a narrowed pool), 16 bytes per
    TB record, 4 per CTU index entry (+1 per picture), and every reconstructed
    sample written once.  Returns (total, written sample bytes)."""
    from hpvcd_b200 import abi, synth
    coeff_bytes = sum(p.n_coeffs * (1 if p.flags & abi.PIC_COEFF8 else 2) for p in pics)
    n_tus = sum(p.n_tus for p in pics)
    ctus = written = 0
    for p in pics:
        g = synth.geometry(p)
        ctus += g["ctb_cols"] * g["ctb_rows"] + 1
        written += (g["w"] * g["h"] + 2 * g["cw"] * g["ch"]) * g["bytes_per_sample"]
    return coeff_bytes + n_tus * 16 + ctus * 4 + written, written


def batched_block(args, local) -> dict:
    """The mixed-size serving workload (`args.batched_images` images, sizes
    256..4096, 8/10-bit, 4:2:0/4:4:4, 512x512 grid tiles, int8 level pools
    where they fit) as a block of the default line: one fused plan against
    one plan per image (device time), the fused plan's reconstruction
    roofline under the learned schedule, and the continuous-batching server's
    saturation throughput and Poisson latency percentiles (page-locked host
    buffers, zero copy)."""
    import ctypes as C

    import torch

    from hpvcd_b200 import abi, serving, synth
    from hpvcd_b200.gpu import DevicePlan

    keep, imgs = serving.make_images(args.batched_images, seed=0)
    c8keep = synth.narrow_coeffs([p for im in imgs for p in im.pics])
    torch.cuda.nvtx.range_push("batched")
    mpix = sum(im.mpix for im in imgs)
    dev = device_batched_vs_plain(imgs, local)

    # reconstruction roofline of the fused plan: the stages launched one
    # after another (inputs of 1+ GB: nothing stays in L2 between steps)
    stream = torch.cuda.Stream(device=local)
    pics, out, out_keep = serving.fused_output(imgs)
    plan = DevicePlan(pics, out, device=local)
    mlp = _selector_network()
    pick = None
    if mlp is not None:
        from hpvcd_b200 import selector
        chosen = C.c_uint32()
        with torch.cuda.stream(stream):
            abi.check(abi.lib().hpvcd_plan_select(plan._h, mlp.handle, selector.schedules_array(), selector.K,
                                                  C.c_void_p(stream.cuda_stream), C.byref(chosen)),
                      "hpvcd_plan_select")
        pick = int(chosen.value)
    stages = [abi.STAGE_RECON, abi.STAGE_DEBLOCK | abi.STAGE_SAO | abi.STAGE_OUTPUT]
    reps = 5
    with torch.cuda.stream(stream):
        for _ in range(2):
            plan.launch(abi.STAGE_ALL, stream)
        torch.cuda.synchronize()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(reps)]
        for k in range(reps):
            for i, s_ in enumerate(stages):
                ev[k][i].record(stream)
                plan.launch(s_, stream)
            ev[k][2].record(stream)
        torch.cuda.synchronize()
    st = plan.status(stream)
    plan.close()
    if st != abi.OK:
        raise abi.HpvcdError(st, "device status of the fused batch")
    recon_ms = sum(e[0].elapsed_time(e[1]) for e in ev) / reps
    filt_ms = sum(e[1].elapsed_time(e[2]) for e in ev) / reps
    recon_bytes, written = recon_algorithmic_bytes(pics)
    peak, peak_kind = measured_peaks()
    gbs = recon_bytes / (recon_ms / 1e3) / 1e9
    filt_bytes = written + int(round(mpix * 1e6)) * 3
    filt_gbs = filt_bytes / (filt_ms / 1e3) / 1e9
    roof = {"kernel": "k_recon", "scope": "reconstruction stage (k_residual + k_recon) of the fused plan",
            "bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
            "frac": round(gbs / peak, 4), "peak_source": peak_kind, "algorithmic_bytes_per_launch": recon_bytes,
            "ms": round(recon_ms, 3), "schedule_pick": pick}
    filt = {"kernel": "k_filter_tile", "bytes": filt_bytes, "ms": round(filt_ms, 3), "gbs": round(filt_gbs, 1),
            "frac": round(filt_gbs / peak, 4)}

    if args.no_serving:
        torch.cuda.nvtx.range_pop()
        del keep, c8keep, out_keep
        return {"workload": "heic_serving_mixed", "images": len(imgs), "tiles": len(pics), "mpix": round(mpix, 2),
                "device": dev, "batched_vs_plain": dev["speedup"],
                "learned_vs_plain": dev.get("learned_speedup_vs_plain"), "recon_roofline": roof, "filters": filt}
    # the serving loop: saturation (all submitted at once) and Poisson arrivals
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    zc = dict(zero_copy=True, warmup=16)

    def brief(r):
        return {k: (round(r[k], 3) if isinstance(r[k], float) else r[k])
                for k in ("mpix_per_s", "p50_ms", "p99_ms", "mean_batch_pictures", "errors")}
    plain_sat = serving.run(imgs, batching=False, arrival_rate=None, device=local, **zc)
    batched_sat = serving.run(imgs, batching=True, arrival_rate=None, device=local, **zc)
    learned_sat = (serving.run(imgs, batching=True, arrival_rate=None, device=local, selector=mlp, **zc)
                   if mlp is not None else None)
    poi = serving.run(imgs, batching=True, arrival_rate=args.rate, device=local, zero_copy=True,
                      selector=mlp)
    # the same saturation run from ordinary host buffers: the server packs
    # every request into its page-locked arenas and copies each canvas out
    copied = serving.run(imgs, batching=True, arrival_rate=None, device=local, warmup=16, selector=mlp)
    ref_sat = learned_sat if learned_sat is not None else batched_sat
    torch.cuda.nvtx.range_pop()
    del keep, c8keep, out_keep
    return {
        "workload": "heic_serving_mixed", "images": len(imgs), "tiles": len(pics), "mpix": round(mpix, 2),
        "sizes": "256..4096 step 64", "bit_depth": "70% 8 / 30% 10", "chroma": "80% 4:2:0 / 20% 4:4:4",
        "device": dev,
        "batched_vs_plain": dev["speedup"],
        "learned_vs_plain": dev.get("learned_speedup_vs_plain"),
        "recon_roofline": roof, "filters": filt,
        "serving_saturation": {"plain": brief(plain_sat), "batched": brief(batched_sat),
                               "batched_learned": brief(learned_sat) if learned_sat else None},
        "serving_batched_vs_plain": round(batched_sat["mpix_per_s"] / plain_sat["mpix_per_s"], 3),
        "serving_learned_vs_plain": (round(learned_sat["mpix_per_s"] / plain_sat["mpix_per_s"], 3)
                                     if learned_sat else None),
        "serving_host_copies": {**brief(copied),
                                "vs_zero_copy": round(copied["mpix_per_s"] / ref_sat["mpix_per_s"], 3),
                                "host_buffers": "ordinary numpy inputs and outputs, copied by the server"},
        "poisson": {"rate_per_s": args.rate, "p50_ms": poi["p50_ms"], "p99_ms": poi["p99_ms"],
                    "mpix_per_s": poi["mpix_per_s"], "errors": poi["errors"],
                    "learned_schedule": mlp is not None},
        "host_buffers": "inputs packed in page-locked memory, page-locked RGB8 outputs (zero copy)",
    }


def device_batched_vs_plain(imgs, local, reps: int = 5):
    """Device time of the whole mixed batch as ONE fused plan (every tile of
    every image in one set of launches, one canvas per image) against the
    plain path: one plan per image, launched one after another."""
    import ctypes as C

    import torch

    from hpvcd_b200 import abi
    from hpvcd_b200.gpu import DevicePlan

    from hpvcd_b200 import serving

    stream = torch.cuda.Stream(device=local)
    pics, out, out_keep = serving.fused_output(imgs)
    fused = DevicePlan(pics, out, device=local)
    singles = []
    keep = []
    for im in imgs:
        o1, a1 = _single_output(im)
        keep.append(a1)
        singles.append(DevicePlan(im.pics, o1, device=local))

    def timed(fn):
        with torch.cuda.stream(stream):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    t_fused = timed(lambda: fused.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, stream))
    t_plain = timed(lambda: [p.launch(abi.STAGE_ALL, stream) for p in singles])
    st = fused.status(stream)
    mpix = sum(im.mpix for im in imgs)
    res = {"fused_ms": round(t_fused, 3), "plain_ms": round(t_plain, 3),
           "fused_mpix_per_s": round(mpix / (t_fused / 1e3), 1),
           "plain_mpix_per_s": round(mpix / (t_plain / 1e3), 1),
           "speedup": round(t_plain / t_fused, 3), "status": st,
           "fused_launches_per_run": fused.launches_per_run}
    # the fused batch with the learned schedule (features + network pick on
    # the device), and exhaustive autotuning as the yardstick
    mlp = _selector_network()
    if mlp is not None:
        from hpvcd_b200 import selector
        chosen = C.c_uint32()
        cs = C.c_void_p(stream.cuda_stream)
        with torch.cuda.stream(stream):
            abi.check(abi.lib().hpvcd_plan_select(fused._h, mlp.handle, selector.schedules_array(), selector.K, cs,
                                                  C.byref(chosen)), "hpvcd_plan_select")
        t_learned = timed(lambda: fused.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, stream))
        ms = (C.c_float * selector.K)()
        best = C.c_uint32()
        with torch.cuda.stream(stream):
            abi.check(abi.lib().hpvcd_plan_autotune(fused._h, selector.schedules_array(), selector.K, abi.STAGE_ALL,
                                                    3, 1, cs, ms, C.byref(best)), "hpvcd_plan_autotune")
        res.update({"learned_ms": round(t_learned, 3), "learned_pick": int(chosen.value),
                    "learned_mpix_per_s": round(mpix / (t_learned / 1e3), 1),
                    "learned_speedup_vs_plain": round(t_plain / t_learned, 3),
                    "autotuned_pick": int(best.value), "autotune_ms": [round(v, 3) for v in ms]})
    fused.close()
    for p in singles:
        p.close()
    return res


def _selector_network():
    """The committed selector network, or None when no weights are present."""
    from hpvcd_b200 import selector
    if not os.path.exists(selector.WEIGHTS_PATH):
        return None
    return selector.Mlp.load()


def run_selector(args):
    """Learned schedule selection on fresh 3840x2160 10-bit frames (a seed the
    network never saw): decode time with the network's pick against the
    fixed default schedule and exhaustive autotuning (every schedule timed on
    the frame itself)."""
    import torch

    from hpvcd_b200 import selector

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    mlp = _selector_network()
    metric = "ms per 3840x2160 frame (learned schedule)"
    if mlp is None:
        print(json.dumps({"metric": metric, "unavailable": "no selector weights"}))
        return 0
    r = selector.evaluate_live(mlp, args.frames, seed=12345 + rank)
    line = {"metric": metric, "value": round(r["ms_selected"], 4), "unit": "ms", "higher_is_better": False,
            "n_gpus": world, "data": "synthetic", "dtype": "int32",
            "config": {"workload": "selector_4k_frames", "frames": args.frames, "size": "3840x2160",
                       "bit_depth": 10, "chroma": "4:2:0", "qp": "17..42", "tb_mix": "Dirichlet(1,1,1,1)",
                       "coded_fraction": "5..60%", "intra_frames": "30%", "schedules": selector.K},
            "selector": r}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_inter(args):
    """Inter video: a 32-frame 1920x1080 8-bit 4:2:0 sequence in decode order
    (an intra frame, then frames predicting from up to 4 earlier frames held
    on the device: 40 % bi-predicted PUs, MVs N(0, 16 px) within the picture
    plus 80 px, one frame in ten with explicit weighted prediction), all of it
    one plan: motion compensation, residuals, intra CUs, deblocking and SAO
    on the GPU; decoded frames stay in HBM as references."""
    import torch

    from hpvcd_b200 import abi, synth
    from hpvcd_b200.gpu import DevicePlan

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_frames, w, h = 32, 1920, 1080
    s = synth.SynthSet()
    s.add(synth.intra_cfg(1000 + rank, w, h, bit_depth=8, chroma_idc=1))
    for i in range(1, n_frames):
        s.add(synth.inter_cfg(1000 + 97 * rank + i, w, h, bit_depth=8, weighted=(i % 10 == 5), n_refs=4))
    pics = s.pictures()
    plan = DevicePlan(pics, device=local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(max(3, args.warmup)):
        plan.launch(abi.STAGE_ALL, stream)
    torch.cuda.synchronize(dev)
    if plan.status(stream) != abi.OK:
        raise abi.HpvcdError(plan.status(stream), "device status")
    K = max(1, min(args.steps, 50))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    clocks = Clocks(local)
    for k in range(K):
        flush.zero_()
        ev[k][0].record(stream)
        plan.launch(abi.STAGE_ALL, stream)
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    clock_rec = clocks.stop()
    ms = [a.elapsed_time(b) for a, b in ev]
    from hpvcd_b200 import replicas
    total = replicas.max_over_ranks(sum(ms), dev)
    mpix = n_frames * w * h / 1e6
    line = {"metric": "decoded MPix/s (inter video)", "value": round(replicas.whole_job_rate(mpix * K, total / 1e3, dev), 2),
            "unit": "MPix/s", "n_gpus": world, "steps": K, "ms_per_step": round(total / K, 4),
            "fps": round(n_frames * K / (total / 1e3), 1), "higher_is_better": True, "scaling": "weak",
            "data": "synthetic", "dtype": "int32",
            "config": {"workload": "inter_1080p_gop32", "frames": n_frames, "size": f"{w}x{h}", "bit_depth": 8,
                       "chroma": "4:2:0", "refs": 4, "bi_pu": "40%", "weighted_frames": "10%",
                       "l2": "flushed between steps"},
            "launches_per_step": plan.launches_per_run, "clocks": clock_rec}
    plan.close()
    line["dpb"] = inter_frame_by_frame(pics, local, reps=2)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def inter_frame_by_frame(pics, local, reps=2, in_flight=2, entries=5):
    """The same sequence as a video decoder submits it: one frame per
    hpvcd_gpu_submit, reference frames kept in a 5-entry device DPB (frame k
    stored in entry k % 5, its up to 4 references read from theirs), inputs
    packed in page-locked memory, the decoded frame's planes DMA'd into a
    page-locked host buffer; `in_flight` frames queued at a time.  Wall-clock
    per frame from submit to its planes in host memory."""
    import ctypes as C
    import time

    from hpvcd_b200 import abi, synth
    from hpvcd_b200.gpu import Dpb, GpuDecoder, pack_pinned, pinned_empty

    frames, keep = [], []
    for k, p in enumerate(pics):
        q = abi.Picture()
        C.pointer(q)[0] = p
        q.flags = p.flags | abi.PIC_STORE_DPB(k % entries)
        for l in range(2):
            for r in range(abi.MAX_REFS):
                sv = p.ref_slot[l][r]
                q.ref_slot[l][r] = abi.REF_DPB(sv % entries) if 0 <= sv and k - sv < entries else -1
        (packed,), kp = pack_pinned([q])
        g = synth.geometry(q)
        nb = (g["w"] * g["h"] + 2 * g["cw"] * g["ch"]) * g["bytes_per_sample"]
        dst, kd = pinned_empty(nb)
        out = abi.Output(abi.OUT_YUV, 0, 0, 0, 0, None, C.c_void_p(dst.ctypes.data), nb)
        frames.append((packed, out, dst))
        keep.append((kp, kd))
    lat, total_s = [], 0.0
    with GpuDecoder(local, max_inflight=in_flight) as d, Dpb(local, entries) as dpb:
        d.set_dpb(dpb)
        for rep in range(reps + 1):  # the first pass warms up (allocations, plans)
            pend = []
            t0 = time.perf_counter()

            def retire(t, ts, dst):
                d.wait(t)
                d.read(t, dst)  # the planes are already in `dst` (direct DMA): releases the ticket
                if rep:
                    lat.append(time.perf_counter() - ts)

            for q, out, dst in frames:
                if len(pend) >= in_flight:
                    retire(*pend.pop(0))
                ts = time.perf_counter()
                pend.append((d.submit([q], out), ts, dst))
            for item in pend:
                retire(*item)
            if rep:
                total_s += time.perf_counter() - t0
        d.set_dpb(None)
    n = len(pics) * reps
    w, h = pics[0].width, pics[0].height
    lat_ms = sorted(x * 1e3 for x in lat)
    return {"fps": round(n / total_s, 1), "value": round(n * w * h / 1e6 / total_s, 1), "unit": "MPix/s",
            "frame_latency_ms": {"p50": round(lat_ms[len(lat_ms) // 2], 3),
                                 "p99": round(lat_ms[min(len(lat_ms) - 1, int(len(lat_ms) * 0.99))], 3)},
            "in_flight": in_flight, "dpb_entries": entries, "frames": n,
            "api": "hpvcd_gpu_submit per frame, references from hpvcd_dpb, pinned packed inputs, "
                   "YUV planes DMA'd to pinned host memory; wall clock"}


def _single_output(im):
    import ctypes as C

    from hpvcd_b200 import abi
    arr = (abi.TilePlace * len(im.places))(*[abi.TilePlace(*t) for t in im.places])
    o = abi.Output(abi.OUT_RGB8, im.matrix, int(im.full_range), im.width, im.height, C.cast(arr, C.c_void_p))
    return o, arr


def run_serving(args):
    """Mixed-size HEIC serving through the native continuous-batching server,
    against the plain path (one image per launch, one launch at a time)."""
    import torch

    from hpvcd_b200 import serving

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    keep, imgs = serving.make_images(args.images, seed=rank)
    dev = device_batched_vs_plain(imgs, local)
    # the device comparison's plans live in torch's cache: hand that memory
    # back, so every serving context sees the same free HBM for admission
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    # saturation runs start warm: every image once untimed (plans of the
    # batch layouts built, stream-ordered pool grown)
    zc = dict(zero_copy=True, warmup=len(imgs))
    plain_sat = serving.run(imgs, batching=False, arrival_rate=None, device=local, **zc)
    batched_sat = serving.run(imgs, batching=True, arrival_rate=None, device=local, **zc)
    mlp = _selector_network()
    learned_sat = (serving.run(imgs, batching=True, arrival_rate=None, device=local, selector=mlp, **zc)
                   if mlp is not None else None)
    zc = dict(zero_copy=True)
    batched_poi = serving.run(imgs, batching=True, arrival_rate=args.rate, device=local, **zc)
    plain_poi = serving.run(imgs, batching=False, arrival_rate=args.rate, device=local, **zc)
    copied_sat = serving.run(imgs, batching=True, arrival_rate=None, device=local)
    line = {
        "metric": "decoded MPix/s (batched serving)", "value": batched_sat["mpix_per_s"], "unit": "MPix/s",
        "n_gpus": world, "higher_is_better": True, "data": "synthetic", "dtype": "int32",
        "config": {"workload": "heic_serving_mixed", "images": len(imgs),
                   "sizes": "256..4096 step 64", "bit_depth": "70% 8 / 30% 10", "chroma": "80% 4:2:0 / 20% 4:4:4",
                   "tiles": sum(len(i.pics) for i in imgs), "mpix": round(sum(i.mpix for i in imgs), 2),
                   "arrivals": f"Poisson {args.rate}/s",
                   "host_buffers": "inputs packed in page-locked memory, page-locked outputs (zero copy)"},
        "batched_vs_plain_throughput": round(batched_sat["mpix_per_s"] / plain_sat["mpix_per_s"], 3),
        "batched_learned_vs_plain_throughput": (round(learned_sat["mpix_per_s"] / plain_sat["mpix_per_s"], 3)
                                                if learned_sat else None),
        "device": dev,
        "saturation": {"plain": plain_sat, "batched": batched_sat, "batched_learned": learned_sat,
                       "batched_host_copies": copied_sat},
        "poisson": {"plain": plain_poi, "batched": batched_poi},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "selector":
        return run_selector(args)
    if args.workload == "inter":
        return run_inter(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
