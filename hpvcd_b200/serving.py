"""Batched HEIC serving: requests of uneven sizes through the native
continuous-batching server (hpvcd_server_*), against the plain path (one
image per launch).

Workload (the mixed-size serving configuration): images with width and height
uniform in 256..4096 in steps of 64, 70% 8-bit / 30% 10-bit, 80% 4:2:0 / 20%
4:4:4, each split into 512x512 grid tiles; requests arrive as a Poisson
process (200/s) or all at once (saturation).  Inputs are seeded synthetic
flat buffers.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import abi, synth
from .gpu import Server, pack_pinned, pinned_empty


@dataclass
class Image:
    width: int
    height: int
    pics: list
    places: list
    matrix: int
    full_range: bool

    packed: list | None = None   # inputs packed in page-locked memory (zero-copy path)
    keep: object = None
    dst: np.ndarray | None = None

    @property
    def mpix(self) -> float:
        return self.width * self.height / 1e6

    def pin(self):
        """Pack the image's flat buffers into page-locked memory (as the host
        syntax decode would write them) and give it a page-locked output."""
        if self.packed is None:
            self.packed, k = pack_pinned(self.pics)
            self.dst, kd = pinned_empty(self.width * self.height * 3)
            self.dst = self.dst.reshape(self.height, self.width, 3)
            self.keep = (k, kd)


def make_images(n_images: int, seed: int = 0, max_side: int = 4096):
    """Seeded mixed-size images (returns the keep-alive SynthSet and the list)."""
    specs = synth.config2_images(seed, n_images, max_side)
    s = synth.SynthSet()
    imgs = []
    for k, (w, h, bd, idc) in enumerate(specs):
        g = synth.make_grid(w, h, seed=seed * 7919 + k, bit_depth=bd, chroma_idc=idc, synth=s)
        first = len(s) - g.cols * g.rows
        pics = [s.picture(first + i) for i in range(g.cols * g.rows)]
        imgs.append(Image(w, h, pics, g.places, abi.MATRIX_SMPTE170M if k % 3 else abi.MATRIX_BT709,
                          bool(k % 2)))
    return s, imgs


def fused_output(imgs):
    """All tiles of all images as one batch: (pictures, hpvcd_output with one
    RGB8 canvas per image, keep-alive arrays)."""
    import ctypes as C
    pics, places, canv = [], [], []
    for k, im in enumerate(imgs):
        pics += im.pics
        places += [(x, y, w, h, k) for (x, y, w, h) in im.places]
        canv.append(abi.Canvas(im.width, im.height, im.matrix, int(im.full_range)))
    pl_arr = (abi.TilePlace * len(places))(*[abi.TilePlace(*t) for t in places])
    cv_arr = (abi.Canvas * len(canv))(*canv)
    out = abi.Output(abi.OUT_RGB8, 0, 0, 0, 0, C.cast(pl_arr, C.c_void_p), None, 0, len(canv),
                     C.cast(cv_arr, C.c_void_p))
    return pics, out, (pl_arr, cv_arr)


def _percentile(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run(imgs, batching: bool, arrival_rate: float | None, seed: int = 1, max_inflight: int = 3,
        device: int = 0, timeout_s: float = 600.0, batch_window_us: int = 2000, warmup: int = 8,
        zero_copy: bool = False, selector=None, max_batch_bytes: int = 0) -> dict:
    """Submit every image (Poisson arrivals at `arrival_rate`/s, or all at
    once when None) and collect the completions.  Returns throughput and
    latency percentiles."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / arrival_rate, len(imgs)) if arrival_rate else np.zeros(len(imgs))
    lat, qms, batch = [], [], []
    bad = 0
    with Server(device, max_inflight=max_inflight if batching else 1, batching=batching,
                max_batch_bytes=max_batch_bytes if batching else 0,
                batch_window_us=batch_window_us if batching else 0) as srv:
        if selector is not None:  # the network picks every batch's schedule
            from .selector import SCHEDULES
            srv.set_selector(selector, SCHEDULES)
        # warm the server (page-locked arenas, device pool, plan code paths)
        def submit(im, user):
            if zero_copy:
                im.pin()
                srv.submit(im.packed, im.places, im.width, im.height, user=user, matrix=im.matrix,
                           full_range=im.full_range, dst=im.dst, zero_copy_keep=im.keep)
            else:
                srv.submit(im.pics, im.places, im.width, im.height, user=user, matrix=im.matrix,
                           full_range=im.full_range)

        if zero_copy:
            for im in imgs:
                im.pin()
        for k, im in enumerate(imgs[:warmup]):
            submit(im, 1 << 40 | k)
        got = 0
        while got < min(warmup, len(imgs)):
            got += len(srv.poll(64, timeout_ms=60000))
        t0 = time.perf_counter()
        next_t = t0
        done = 0
        for k, im in enumerate(imgs):
            next_t += gaps[k]
            while True:  # keep draining completions while waiting for the next arrival
                now = time.perf_counter()
                if now >= next_t:
                    break
                for c in srv.poll(64, timeout_ms=max(0, int((next_t - now) * 1000))):
                    done += 1
                    bad += c["status"] != abi.OK
                    lat.append(c["latency_ms"]); qms.append(c["queue_ms"]); batch.append(c["batch_pictures"])
            submit(im, k)
        deadline = time.perf_counter() + timeout_s
        while done < len(imgs) and time.perf_counter() < deadline:
            for c in srv.poll(64, timeout_ms=1000):
                done += 1
                bad += c["status"] != abi.OK
                lat.append(c["latency_ms"]); qms.append(c["queue_ms"]); batch.append(c["batch_pictures"])
        t1 = time.perf_counter()
    mpix = sum(im.mpix for im in imgs)
    return {"images": len(imgs), "completed": done, "errors": bad, "mpix": round(mpix, 2),
            "seconds": round(t1 - t0, 4), "mpix_per_s": round(mpix / (t1 - t0), 2),
            "p50_ms": _percentile(lat, 50), "p99_ms": _percentile(lat, 99),
            "queue_p50_ms": _percentile(qms, 50), "mean_batch_pictures": float(np.mean(batch)) if batch else 0.0,
            "arrival_rate": arrival_rate, "batching": batching, "zero_copy": zero_copy,
            "learned_schedule": selector is not None}
