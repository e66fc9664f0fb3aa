"""Python host side of the B200 reconstruction back end.

Two layers over the C ABI (include/hpvcd_gpu.h, libhpvcd_b200.so):

* `GpuDecoder` -- the host-buffer drop-in that sits where the reference's
  `decode_heic` grid path (lib.rs:1724 `decode_grid` -> lib.rs:1680
  `fill_grid_bands` -> lib.rs:1610 `stitch_grid_band`) and `finish_with`
  (decode.rs:1440) run: flat per-picture buffers in host memory go in, an RGB8
  canvas or YUV planes come out.  Errors raise `HpvcdError`, the analogue of
  the reference's `DecodeError`.
* `DevicePlan` -- the same reconstruction over buffers already resident in
  HBM (uploaded once through torch), launched on a CUDA stream; this is what
  the kernel-level timing uses.

There is no CPU fallback: when the CUDA library is missing these classes
raise ImportError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .synth import geometry


def _check(status: int, what: str) -> None:
    abi.check(status, what)


def _pic_array(pics):
    return (abi.Picture * len(pics))(*pics)


class GpuDecoder:
    """Host-buffer API (hpvcd_gpu_*): submit / wait / read tickets."""

    def __init__(self, device: int = 0, max_inflight: int = 4, hbm_budget: int = 0):
        self._L = abi.lib()
        cfg = abi.GpuCfg(device, max_inflight, hbm_budget)
        h = C.c_void_p()
        _check(self._L.hpvcd_gpu_create(C.byref(cfg), C.byref(h)), "hpvcd_gpu_create")
        self._h = h

    def submit(self, pics, output: abi.Output | None = None) -> int:
        arr = _pic_array(pics)
        t = C.c_uint64()
        _check(self._L.hpvcd_gpu_submit(self._h, arr, len(pics),
                                        C.byref(output) if output is not None else None, C.byref(t)),
               "hpvcd_gpu_submit")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> bool:
        s = self._L.hpvcd_gpu_wait(self._h, ticket, timeout_ms)
        if s == abi.ERR_BUSY:
            return False
        _check(s, "hpvcd_gpu_wait")
        return True

    def output_size(self, ticket: int) -> int:
        b = C.c_uint64()
        _check(self._L.hpvcd_gpu_output_size(self._h, ticket, C.byref(b)), "hpvcd_gpu_output_size")
        return b.value

    def read(self, ticket: int, dst: np.ndarray | None = None) -> np.ndarray:
        n = self.output_size(ticket)
        if dst is None:
            dst = np.empty(n, np.uint8)
        assert dst.nbytes >= n and dst.flags["C_CONTIGUOUS"]
        _check(self._L.hpvcd_gpu_read(self._h, ticket, dst.ctypes.data_as(C.c_void_p), dst.nbytes),
               "hpvcd_gpu_read")
        return dst

    def decode_rgb8(self, pics, output: abi.Output, dst: np.ndarray | None = None) -> np.ndarray:
        """Decode a grid of pictures onto an RGB8 canvas (decode_heic_rgb8)."""
        t = self.submit(pics, output)
        self.wait(t)
        out = self.read(t, dst)
        return out.reshape(output.canvas_h, output.canvas_w, 3)

    def decode_yuv(self, pics):
        """Decode pictures to their final planes (decode_heic_yuv); returns a
        list of (Y, Cb, Cr) numpy arrays in native sample type."""
        t = self.submit(pics, None)
        self.wait(t)
        raw = self.read(t)
        return split_planes(pics, raw)

    def set_selector(self, mlp, schedules) -> None:
        """Per-submit schedule from the selector network (None: default)."""
        arr = (abi.Sched * len(schedules))(*schedules)
        self._sel_keep = (mlp, arr)
        _check(self._L.hpvcd_gpu_set_selector(self._h, mlp.handle if mlp is not None else None, arr,
                                              len(schedules)), "hpvcd_gpu_set_selector")

    def set_sched(self, sched: abi.Sched | None) -> None:
        """Schedule of the submits while no selector is set (None: the default)."""
        _check(self._L.hpvcd_gpu_set_sched(self._h, C.byref(sched) if sched is not None else None),
               "hpvcd_gpu_set_sched")

    def selector_picks(self, n: int) -> list:
        """Picks per candidate schedule so far ([K]: batches outside the domain)."""
        out = (C.c_uint64 * n)()
        _check(self._L.hpvcd_gpu_selector_picks(self._h, out, n), "hpvcd_gpu_selector_picks")
        return list(out)

    def set_dpb(self, dpb: "Dpb | None") -> None:
        """Decoded-picture buffer the submits store into (flags
        abi.PIC_STORE_DPB(e)) and predict from (ref_slot abi.REF_DPB(e))."""
        self._dpb_keep = dpb
        _check(self._L.hpvcd_gpu_set_dpb(self._h, dpb.handle if dpb is not None else None), "hpvcd_gpu_set_dpb")

    def close(self):
        if getattr(self, "_h", None):
            self._L.hpvcd_gpu_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Dpb:
    """Device-resident decoded-picture buffer (hpvcd_dpb_*): `entries`
    reference pictures kept in HBM across submits of one context."""

    def __init__(self, device: int = 0, entries: int = 16):
        self._L = abi.lib()
        h = C.c_void_p()
        _check(self._L.hpvcd_dpb_create(device, entries, C.byref(h)), "hpvcd_dpb_create")
        self._h = h
        self.entries = entries

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._L.hpvcd_dpb_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pinned_empty(nbytes: int):
    """Page-locked host buffer (torch provides the allocation); returns
    (numpy view, keepalive)."""
    import torch
    t = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, pin_memory=True)
    return t.numpy()[:nbytes], t


def pack_pinned(pics):
    """Copy the host buffers of `pics` into one page-locked arena laid out as
    the device input arena, so hpvcd_gpu_submit uploads them with one DMA.
    Returns (new descriptors, keepalive)."""
    L = abi.lib()
    arr = _pic_array(pics)
    nb = L.hpvcd_gpu_packed_size(arr, len(pics))
    buf, keep = pinned_empty(nb)
    out = (abi.Picture * len(pics))()
    _check(L.hpvcd_gpu_pack_inputs(arr, len(pics), buf.ctypes.data_as(C.c_void_p), nb, out),
           "hpvcd_gpu_pack_inputs")
    return list(out), (keep, buf, nb)


def canvas_views(pics, out: abi.Output, raw: np.ndarray):
    """Split the output of a canvas batch (RGB8 or YUV canvas) into one view
    per canvas: an (h, w, 3) uint8 array for an RGB8 canvas, a (Y, Cb, Cr)
    tuple in native sample type for a native one (every canvas of an
    OUT_YUV_CANVAS output, CANVAS_NATIVE ones of an RGB8 output; Cb / Cr
    empty for 4:0:0).  A native canvas has the chroma format and sample size
    of the first picture placed on it."""
    n_c = out.n_canvases or 1
    cv = (abi.Canvas * out.n_canvases).from_address(out.canvases) if out.n_canvases else None
    place = (abi.TilePlace * len(pics)).from_address(out.place)
    res, off = [], 0
    def shape(w, h):  # rows, columns of the oriented image
        return (w, h) if orient in (abi.ORIENT_ROTATE90, abi.ORIENT_ROTATE270) else (h, w)

    for k in range(n_c):
        w, h = (cv[k].width, cv[k].height) if cv is not None else (out.canvas_w, out.canvas_h)
        matrix = cv[k].matrix if cv is not None else out.matrix
        orient = cv[k].orientation if cv is not None else out.orientation
        if out.kind == abi.OUT_RGB8 and matrix != abi.CANVAS_NATIVE:
            res.append(raw[off:off + w * h * 3].reshape(*shape(w, h), 3))
            off += w * h * 3
            continue
        first = next((p for i, p in enumerate(pics) if place[i].canvas == k), None)
        idc = first.chroma_idc if first is not None else 0
        bps = 1 if first is None or (first.bit_depth_y <= 8 and first.bit_depth_c <= 8) else 2
        sw, sh = (2 if idc in (1, 2) else 1), (2 if idc == 1 else 1)
        cw, ch = ((w + sw - 1) // sw, (h + sh - 1) // sh) if idc else (0, 0)
        dt = np.uint8 if bps == 1 else np.uint16
        planes = []
        for (pw, ph) in [(w, h), (cw, ch), (cw, ch)]:
            nb = pw * ph * bps
            planes.append(raw[off:off + nb].view(dt).reshape(*shape(pw, ph)))
            off += nb
        res.append(tuple(planes))
    return res


yuv_canvas_planes = canvas_views


def split_planes(pics, raw: np.ndarray):
    out = []
    o = 0
    for p in pics:
        g = geometry(p)
        dt = np.uint8 if g["bytes_per_sample"] == 1 else np.uint16
        planes = []
        for c in range(3 if p.chroma_idc else 1):
            w, h = (g["w"], g["h"]) if c == 0 else (g["cw"], g["ch"])
            nb = w * h * g["bytes_per_sample"]
            planes.append(raw[o:o + nb].view(dt).reshape(h, w).copy())
            o += nb
        while len(planes) < 3:
            planes.append(np.zeros((0, 0), dt))
        out.append(tuple(planes))
    return out


# ---------------------------------------------------------------------------
# Device-resident plans (torch provides the device memory and streams).
# ---------------------------------------------------------------------------

def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("DevicePlan needs a CUDA device")
    return torch


class DevicePlan:
    """Upload the flat buffers of `pics` to HBM once and build a plan."""

    def __init__(self, pics, output: abi.Output | None = None, sched: abi.Sched | None = None,
                 device: int = 0, resident: dict | None = None):
        torch = _torch()
        self._L = abi.lib()
        self.torch = torch
        self.device = torch.device("cuda", device)
        self._keep = []
        self.host_pics = list(pics)
        dev = []
        self.input_bytes = 0
        for i, p in enumerate(pics):
            if resident and i in resident:  # descriptor already pointing at device buffers
                dev.append(resident[i])
                continue
            g = geometry(p)
            ctbs = g["ctb_cols"] * g["ctb_rows"]
            d = abi.Picture()
            C.pointer(d)[0] = p
            d.tus = self._upload(p.tus, p.n_tus * 16)
            d.ctu_tu_start = self._upload(p.ctu_tu_start, (ctbs + 1) * 4)
            d.coeffs = self._upload(p.coeffs, p.n_coeffs * (1 if p.flags & abi.PIC_COEFF8 else 2))
            d.cells = self._upload(p.cells, g["gw"] * g["gh"] * 4)
            d.sao = self._upload(p.sao, ctbs * 36)
            d.pus = self._upload(p.pus, p.n_pus * 20)
            d.wp = self._upload(p.wp, C.sizeof(abi.WpTable))
            d.scaling = self._upload(p.scaling, C.sizeof(abi.Scaling))
            d.ctb_region = self._upload(p.ctb_region, ctbs * 2)
            d.slice_deblock = self._upload(p.slice_deblock, 512)
            for c in range(3):
                if p.pred[c]:
                    nb = (g["w"] * g["h"] if c == 0 else g["cw"] * g["ch"]) * g["bytes_per_sample"]
                    d.pred[c] = self._upload(p.pred[c], nb)
            dev.append(d)
        self.dev_pics = dev
        arr = _pic_array(dev)
        h = C.c_void_p()
        _check(self._L.hpvcd_plan_create(arr, len(dev), C.byref(output) if output is not None else None,
                                         C.byref(sched) if sched is not None else None, C.byref(h)),
               "hpvcd_plan_create")
        self._h = h
        self.output = output
        self.launches_per_run = self._L.hpvcd_plan_launches_per_run(h)

    def _upload(self, host_ptr, nbytes: int):
        if not host_ptr or nbytes == 0:
            return None
        torch = self.torch
        src = np.ctypeslib.as_array((C.c_uint8 * nbytes).from_address(host_ptr))
        t = torch.from_numpy(src.copy()).to(self.device)
        self._keep.append(t)
        self.input_bytes += nbytes
        return t.data_ptr()

    def launch(self, stages: int = abi.STAGE_ALL, stream=None) -> None:
        s = stream if stream is not None else self.torch.cuda.current_stream(self.device)
        _check(self._L.hpvcd_plan_launch(self._h, stages, C.c_void_p(s.cuda_stream)), "hpvcd_plan_launch")

    def status(self, stream=None) -> int:
        s = stream if stream is not None else self.torch.cuda.current_stream(self.device)
        return self._L.hpvcd_plan_device_status(self._h, C.c_void_p(s.cuda_stream))

    def set_sched(self, sched: abi.Sched | None) -> None:
        _check(self._L.hpvcd_plan_set_sched(self._h, C.byref(sched) if sched is not None else None),
               "hpvcd_plan_set_sched")

    def set_wait_test(self, spin_limit: int = 0, drop_ctu: int = -1) -> None:
        """Bound every wavefront wait to `spin_limit` polls (0: default) and
        leave work-list entry `drop_ctu` out of the launches (-1: none)."""
        _check(self._L.hpvcd_plan_set_wait_test(self._h, spin_limit, drop_ctu), "hpvcd_plan_set_wait_test")

    def canvas(self) -> np.ndarray:
        ptr, nb = C.c_void_p(), C.c_uint64()
        _check(self._L.hpvcd_plan_canvas(self._h, C.byref(ptr), C.byref(nb)), "hpvcd_plan_canvas")
        out = np.empty(nb.value, np.uint8)
        _check(self._L.hpvcd_copy(out.ctypes.data_as(C.c_void_p), ptr, nb.value, None), "hpvcd_copy")
        return out.reshape(self.output.canvas_h, self.output.canvas_w, 3)

    def canvas_ptr(self) -> tuple[int, int]:
        ptr, nb = C.c_void_p(), C.c_uint64()
        _check(self._L.hpvcd_plan_canvas(self._h, C.byref(ptr), C.byref(nb)), "hpvcd_plan_canvas")
        return ptr.value, nb.value

    def planes(self, i: int):
        p = self.host_pics[i]
        g = geometry(p)
        ptrs = [C.c_void_p() for _ in range(3)]
        _check(self._L.hpvcd_plan_planes(self._h, i, *(C.byref(x) for x in ptrs)), "hpvcd_plan_planes")
        dt = np.uint8 if g["bytes_per_sample"] == 1 else np.uint16
        res = []
        for c in range(3):
            w, h = (g["w"], g["h"]) if c == 0 else (g["cw"], g["ch"])
            a = np.zeros((h, w), dt)
            if ptrs[c].value and a.size:
                _check(self._L.hpvcd_copy(a.ctypes.data_as(C.c_void_p), ptrs[c], a.nbytes, None), "hpvcd_copy")
            res.append(a)
        return tuple(res)

    def close(self):
        if getattr(self, "_h", None):
            self._L.hpvcd_plan_destroy(self._h)
            self._h = None
        self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Serving loop (hpvcd_server_*): continuous batching of decode requests.
# ---------------------------------------------------------------------------

class Server:
    """Requests (one image each: its grid tiles + an RGB8 destination) are
    queued; a native worker fuses everything queued into one launch whenever
    a GPU slot frees.  `batching=False` gives the plain one-image-per-launch
    path with the same machinery."""

    def __init__(self, device: int = 0, max_inflight: int = 2, batching: bool = True,
                 max_batch_pictures: int = 0, max_batch_bytes: int = 0, hbm_budget: int = 0,
                 batch_window_us: int = 0):
        self._L = abi.lib()
        cfg = abi.ServerCfg(device, max_inflight, max_batch_pictures, max_batch_bytes, hbm_budget,
                            int(batching), batch_window_us)
        h = C.c_void_p()
        _check(self._L.hpvcd_server_create(C.byref(cfg), C.byref(h)), "hpvcd_server_create")
        self._h = h
        self._dst = {}
        self._keep = {}

    def submit(self, pics, places, width: int, height: int, user: int,
               matrix: int = abi.MATRIX_SMPTE170M, full_range: bool = True,
               dst: np.ndarray | None = None, zero_copy_keep=None) -> np.ndarray:
        """Queue one image.  `zero_copy_keep`: keep-alive of inputs packed by
        pack_pinned() and a page-locked `dst` (pinned_empty()); the server
        then copies nothing on the host."""
        arr = _pic_array(pics)
        pl = (abi.TilePlace * len(places))(*[abi.TilePlace(*t) for t in places])
        if dst is None:
            dst = np.empty((height, width, 3), np.uint8)
        req = abi.Request(C.cast(arr, C.c_void_p), len(pics), C.cast(pl, C.c_void_p),
                          abi.Canvas(width, height, matrix, int(full_range)),
                          dst.ctypes.data_as(C.c_void_p), dst.nbytes, user,
                          abi.REQ_ZERO_COPY if zero_copy_keep is not None else 0)
        self._dst[user] = dst
        if zero_copy_keep is not None:
            self._keep[user] = zero_copy_keep
        _check(self._L.hpvcd_server_submit(self._h, C.byref(req)), "hpvcd_server_submit")
        return dst

    def poll(self, max_n: int = 64, timeout_ms: int = -1):
        buf = (abi.Completion * max_n)()
        k = self._L.hpvcd_server_poll(self._h, buf, max_n, timeout_ms)
        out = []
        for i in range(k):
            c = buf[i]
            self._keep.pop(c.user, None)
            out.append(dict(user=c.user, status=c.status, batch_pictures=c.batch_pictures,
                            latency_ms=c.latency_ms, queue_ms=c.queue_ms,
                            image=self._dst.pop(c.user, None)))
        return out

    def pending(self) -> int:
        return self._L.hpvcd_server_pending(self._h)

    def set_selector(self, mlp, schedules) -> None:
        """Per-batch schedule from the selector network (None: default)."""
        arr = (abi.Sched * len(schedules))(*schedules)
        self._sel_keep = (mlp, arr)
        _check(self._L.hpvcd_server_set_selector(self._h, mlp.handle if mlp is not None else None, arr,
                                                 len(schedules)), "hpvcd_server_set_selector")

    def selector_picks(self, n: int) -> list:
        out = (C.c_uint64 * n)()
        _check(self._L.hpvcd_server_selector_picks(self._h, out, n), "hpvcd_server_selector_picks")
        return list(out)

    def close(self):
        if getattr(self, "_h", None):
            self._L.hpvcd_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
